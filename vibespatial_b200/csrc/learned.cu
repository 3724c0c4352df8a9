// Learned cell index (placeholder until the RMI path lands).
#include "index.cuh"
#include "join.cuh"

namespace vs {
int build_learned_index(vs_context*, vs_index*, const vs_index_options*) {
    set_error("learned cell index not available in this build");
    return VS_E_ARG;
}
void free_learned_index(vs_index*) {}
int launch_learned_join(vs_context*, const vs_index*, const vs_points*, int, int32_t*, int32_t*, int64_t) {
    set_error("learned cell index not available in this build");
    return VS_E_ARG;
}
}  // namespace vs
