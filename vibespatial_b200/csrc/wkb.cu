// WKB -> columnar geometry on the device (GeoParquet / GeoArrow WKB ingest).
//
// Replaces the reference's Arrow WKB decode (decode_wkb_arrow_array_owned,
// src/vibespatial/io/wkb.py:5224, and its GPU kernels in io/wkb_kernels.py)
// for the families the join consumes: Point, Polygon and MultiPolygon, in
// either byte order, ISO (type + 1000 * dims) or EWKB (Z / M / SRID flag
// bits) form; Z and M ordinates are dropped.  The output is the layout of a
// GeometryArray: per-row tags and point coordinates, and a MultiPolygon-form
// SoA (geom_off -> part_off -> ring_off -> x, y) over all rows (point and
// null rows own no parts).
//
//   1. wkb_size_kernel  (thread per row) parses the headers and counts, with
//      every read bounds-checked against the row's byte range; writes tags,
//      point coordinates and the row's part / ring / coordinate counts
//   2. exclusive scans of the three counts
//   3. wkb_fill_kernel  (thread per row) writes part_off and ring_off and,
//      per ring, where its coordinates start in the WKB bytes
//   4. wkb_copy_kernel  (warp per ring) copies the coordinates: lanes read
//      consecutive unaligned doubles, byte-swapping big-endian rows
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <new>

#include "primitives.cuh"
#include "vs_common.cuh"

namespace vs {
namespace {

enum : int8_t { kTagNull = -1, kTagPoint = 0, kTagPolygon = 2, kTagMultiPolygon = 5 };
enum : int32_t { kRowOk = 0, kRowUnsupported = 1, kRowMalformed = 2 };

struct WkbIn {
    const uint8_t* data;
    const int64_t* offsets;  // [n + 1] byte offsets of the rows
    const uint8_t* valid;    // nullable
    int64_t n;
};

// A cursor over one row's bytes; every read checks the end.
struct Cursor {
    const uint8_t* p;
    const uint8_t* end;
    bool ok;

    __device__ __forceinline__ uint32_t u32(bool little) {
        if (end - p < 4) {
            ok = false;
            return 0;
        }
        const uint32_t b0 = p[0], b1 = p[1], b2 = p[2], b3 = p[3];
        p += 4;
        return little ? (b0 | b1 << 8 | b2 << 16 | b3 << 24) : (b3 | b2 << 8 | b1 << 16 | b0 << 24);
    }
    __device__ __forceinline__ uint8_t u8() {
        if (end - p < 1) {
            ok = false;
            return 0;
        }
        return *p++;
    }
    __device__ __forceinline__ void skip(uint64_t bytes) {
        if ((uint64_t)(end - p) < bytes) {
            ok = false;
            p = end;
            return;
        }
        p += bytes;
    }
};

__device__ __forceinline__ double load_f64(const uint8_t* p, bool little) {
    uint64_t v = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) v |= (uint64_t)p[little ? k : 7 - k] << (8 * k);
    return __longlong_as_double((long long)v);
}

// Geometry header: byte order, base type and ordinates per coordinate.
struct Header {
    bool little;
    uint32_t base;  // 1 point, 3 polygon, 6 multipolygon, ...
    int dims;       // 2..4
};

__device__ __forceinline__ Header read_header(Cursor& c) {
    Header h{true, 0, 2};
    const uint8_t bo = c.u8();
    if (bo > 1) c.ok = false;
    h.little = bo == 1;
    uint32_t t = c.u32(h.little);
    bool z = false, m = false;
    if (t & 0x20000000u) c.skip(4);  // EWKB SRID
    if (t & 0x80000000u) z = true;
    if (t & 0x40000000u) m = true;
    t &= 0x0fffffffu;
    const uint32_t iso = t / 1000u;  // ISO: 1000 Z, 2000 M, 3000 ZM
    t %= 1000u;
    if (iso == 1 || iso == 3) z = true;
    if (iso == 2 || iso == 3) m = true;
    if (iso > 3) c.ok = false;
    h.base = t;
    h.dims = 2 + (z ? 1 : 0) + (m ? 1 : 0);
    return h;
}

// Polygon body: ring count, then per ring its point count and points.
// Adds its rings and coordinates to the counts.
__device__ __forceinline__ void polygon_body(Cursor& c, const Header& h, uint32_t& rings, uint64_t& coords) {
    const uint32_t nr = c.u32(h.little);
    for (uint32_t r = 0; r < nr && c.ok; ++r) {
        const uint32_t np = c.u32(h.little);
        c.skip((uint64_t)np * 8u * (uint64_t)h.dims);
        coords += np;
    }
    rings += nr;
}

struct RowCounts {
    int8_t tag;
    int32_t status;
    uint32_t parts, rings;
    uint64_t coords;
    double px, py;
};

__device__ RowCounts parse_row(const WkbIn& in, int64_t i) {
    RowCounts rc{kTagNull, kRowOk, 0, 0, 0, 0.0, 0.0};
    rc.px = rc.py = __longlong_as_double(0x7ff8000000000000ll);
    if (in.valid && !in.valid[i]) return rc;
    const int64_t b0 = in.offsets[i], b1 = in.offsets[i + 1];
    if (b1 <= b0) return rc;  // null / zero-length value: a null row
    Cursor c{in.data + b0, in.data + b1, true};
    const Header h = read_header(c);
    if (!c.ok) {
        rc.status = kRowMalformed;
        return rc;
    }
    if (h.base == 1) {
        if (c.end - c.p < 8 * h.dims) {
            rc.status = kRowMalformed;
            return rc;
        }
        rc.tag = kTagPoint;
        rc.px = load_f64(c.p, h.little);
        rc.py = load_f64(c.p + 8, h.little);
        return rc;
    }
    if (h.base == 3) {
        rc.tag = kTagPolygon;
        uint32_t rings = 0;
        polygon_body(c, h, rings, rc.coords);
        rc.parts = rings > 0 ? 1 : 0;  // an empty polygon owns no part
        rc.rings = rings;
    } else if (h.base == 6) {
        rc.tag = kTagMultiPolygon;
        const uint32_t np = c.u32(h.little);
        for (uint32_t k = 0; k < np && c.ok; ++k) {
            const Header ph = read_header(c);
            if (!c.ok) break;
            if (ph.base != 3) {
                c.ok = false;
                break;
            }
            uint32_t rings = 0;
            polygon_body(c, ph, rings, rc.coords);
            rc.parts += rings > 0 ? 1 : 0;  // an empty part owns no part entry
            rc.rings += rings;
        }
    } else {
        rc.status = kRowUnsupported;
        rc.tag = kTagNull;
        return rc;
    }
    if (!c.ok) {
        rc.status = kRowMalformed;
        rc.tag = kTagNull;
        rc.parts = rc.rings = 0;
        rc.coords = 0;
    }
    return rc;
}

__global__ void wkb_size_kernel(const WkbIn in, int8_t* __restrict__ tags, double* __restrict__ px,
                                double* __restrict__ py, uint32_t* __restrict__ parts, uint32_t* __restrict__ rings,
                                uint32_t* __restrict__ coords, unsigned long long* __restrict__ totals) {
    // totals: [0] points, [1] polygons, [2] multipolygons, [3] nulls, [4] unsupported, [5] malformed,
    //         [6] coordinates (64-bit sum, to check the 32-bit offsets)
    unsigned long long t[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < in.n; i += (int64_t)gridDim.x * blockDim.x) {
        const RowCounts rc = parse_row(in, i);
        tags[i] = rc.tag;
        px[i] = rc.px;
        py[i] = rc.py;
        parts[i] = rc.parts;
        rings[i] = rc.rings;
        coords[i] = rc.coords > 0xffffffffull ? 0xffffffffu : (uint32_t)rc.coords;
        t[0] += rc.tag == kTagPoint;
        t[1] += rc.tag == kTagPolygon;
        t[2] += rc.tag == kTagMultiPolygon;
        t[3] += rc.tag == kTagNull && rc.status == kRowOk;
        t[4] += rc.status == kRowUnsupported;
        t[5] += rc.status == kRowMalformed;
        t[6] += rc.coords;
    }
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        unsigned long long v = t[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&totals[k], v);
    }
}

// Pass 3: offsets of every part and ring, and where each ring's coordinates
// start in the row's bytes.
__global__ void wkb_fill_kernel(const WkbIn in, const int8_t* __restrict__ tags, const uint32_t* __restrict__ part0,
                                const uint32_t* __restrict__ ring0, const uint32_t* __restrict__ coord0,
                                int32_t* __restrict__ geom_off, int32_t* __restrict__ part_off,
                                int32_t* __restrict__ ring_off, int64_t* __restrict__ ring_src,
                                uint8_t* __restrict__ ring_fmt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < in.n; i += (int64_t)gridDim.x * blockDim.x) {
        geom_off[i] = (int32_t)part0[i];
        const int8_t tag = tags[i];
        if (tag != kTagPolygon && tag != kTagMultiPolygon) continue;
        const int64_t b0 = in.offsets[i], b1 = in.offsets[i + 1];
        Cursor c{in.data + b0, in.data + b1, true};
        const Header h = read_header(c);
        uint32_t part = part0[i], ring = ring0[i], coord = coord0[i];
        uint32_t n_parts = 1;
        if (tag == kTagMultiPolygon) n_parts = c.u32(h.little);
        for (uint32_t k = 0; k < n_parts; ++k) {
            Header ph = h;
            if (tag == kTagMultiPolygon) ph = read_header(c);
            const uint32_t nr = c.u32(ph.little);
            if (nr == 0) continue;  // an empty polygon (part) owns no part entry
            part_off[part++] = (int32_t)ring;
            for (uint32_t r = 0; r < nr; ++r) {
                const uint32_t np = c.u32(ph.little);
                ring_off[ring] = (int32_t)coord;
                ring_src[ring] = (int64_t)(c.p - in.data);
                ring_fmt[ring] = (uint8_t)((ph.little ? 1 : 0) | (ph.dims << 1));
                ++ring;
                c.skip((uint64_t)np * 8u * (uint64_t)ph.dims);
                coord += np;
            }
        }
    }
}

// Pass 4: warp per ring, lanes copy consecutive coordinates.
__global__ void wkb_copy_kernel(const uint8_t* __restrict__ data, int64_t n_rings, const int32_t* __restrict__ ring_off,
                                const int64_t* __restrict__ ring_src, const uint8_t* __restrict__ ring_fmt,
                                double* __restrict__ x, double* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gw; r < n_rings; r += nw) {
        const int32_t c0 = ring_off[r], c1 = ring_off[r + 1];
        const uint8_t* src = data + ring_src[r];
        const bool little = ring_fmt[r] & 1;
        const int stride = 8 * (ring_fmt[r] >> 1);
        for (int32_t k = lane; k < c1 - c0; k += 32) {
            x[c0 + k] = load_f64(src + (int64_t)k * stride, little);
            y[c0 + k] = load_f64(src + (int64_t)k * stride + 8, little);
        }
    }
}

}  // namespace
}  // namespace vs

struct vs_wkb_plan {
    vs_context* ctx = nullptr;
    vs::WkbIn in{};
    vs_wkb_sizes sizes{};
    // per-row scratch kept between the two calls
    int8_t* tags = nullptr;
    double* px = nullptr;
    double* py = nullptr;
    uint32_t* parts = nullptr;  // counts, then exclusive offsets
    uint32_t* rings = nullptr;
    uint32_t* coords = nullptr;
    unsigned long long* totals = nullptr;
};

namespace {

void free_wkb_plan(vs_wkb_plan* p) {
    cudaFree(p->tags);
    cudaFree(p->px);
    cudaFree(p->py);
    cudaFree(p->parts);
    cudaFree(p->rings);
    cudaFree(p->coords);
    cudaFree(p->totals);
}

}  // namespace

using namespace vs;

extern "C" {

int vs_wkb_plan_create(vs_context* ctx, const uint8_t* d_wkb, const int64_t* d_offsets, const uint8_t* d_valid,
                       int64_t n, vs_wkb_plan** out, vs_wkb_sizes* sizes) {
    if (!ctx || !out || !sizes || (n > 0 && (!d_wkb || !d_offsets))) {
        set_error("ctx/out/sizes/wkb/offsets is NULL");
        return VS_E_ARG;
    }
    *out = nullptr;
    memset(sizes, 0, sizeof(*sizes));
    if (n < 0 || n > 0x7ffffffeLL) {
        set_error("row count %lld outside [0, 2^31-2]", (long long)n);
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    vs_wkb_plan* p = new (std::nothrow) vs_wkb_plan{};
    if (!p) {
        set_error("host allocation failed");
        return VS_E_OOM;
    }
    p->ctx = ctx;
    p->in = WkbIn{d_wkb, d_offsets, d_valid, n};
    const size_t rows = (size_t)(n > 0 ? n : 1) + 1;
    if (cudaMalloc((void**)&p->tags, rows) != cudaSuccess || cudaMalloc((void**)&p->px, rows * 8) != cudaSuccess ||
        cudaMalloc((void**)&p->py, rows * 8) != cudaSuccess ||
        cudaMalloc((void**)&p->parts, rows * 4) != cudaSuccess ||
        cudaMalloc((void**)&p->rings, rows * 4) != cudaSuccess ||
        cudaMalloc((void**)&p->coords, rows * 4) != cudaSuccess ||
        cudaMalloc((void**)&p->totals, 8 * sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        set_error("WKB plan allocation failed (%lld rows)", (long long)n);
        free_wkb_plan(p);
        delete p;
        return VS_E_OOM;
    }
    cudaStream_t s = ctx->stream;
    int st = VS_OK;
    do {
        if (cudaMemsetAsync(p->totals, 0, 8 * sizeof(unsigned long long), s) != cudaSuccess) {
            st = VS_E_CUDA;
            break;
        }
        if (n > 0) {
            wkb_size_kernel<<<resident_grid(wkb_size_kernel, n, 256), 256, 0, s>>>(p->in, p->tags, p->px, p->py,
                                                                                   p->parts, p->rings, p->coords,
                                                                                   p->totals);
            if (cudaGetLastError() != cudaSuccess) {
                st = VS_E_CUDA;
                break;
            }
            ++g_launches;
        }
        unsigned long long t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (cudaMemcpyAsync(t, p->totals, sizeof(t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            st = VS_E_CUDA;
            break;
        }
        sizes->n_rows = n;
        sizes->n_points = (int64_t)t[0];
        sizes->n_polygons = (int64_t)t[1];
        sizes->n_multipolygons = (int64_t)t[2];
        sizes->n_null = (int64_t)t[3];
        sizes->n_unsupported = (int64_t)t[4];
        sizes->n_malformed = (int64_t)t[5];
        if (t[6] > 0x7fffffffull) {
            set_error("%llu coordinates: more than the 32-bit offsets address", t[6]);
            st = VS_E_ARG;
            break;
        }
        // exclusive scans in place, totals into the last (n-th) entry
        st = exclusive_scan_u32(p->parts, p->parts, n, p->parts + n, s);
        if (st == VS_OK) st = exclusive_scan_u32(p->rings, p->rings, n, p->rings + n, s);
        if (st == VS_OK) st = exclusive_scan_u32(p->coords, p->coords, n, p->coords + n, s);
        if (st != VS_OK) break;
        uint32_t tot[3] = {0, 0, 0};
        if (cudaMemcpyAsync(&tot[0], p->parts + n, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(&tot[1], p->rings + n, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(&tot[2], p->coords + n, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            st = VS_E_CUDA;
            break;
        }
        sizes->n_parts = tot[0];
        sizes->n_rings = tot[1];
        sizes->n_coords = tot[2];
    } while (false);
    if (st != VS_OK) {
        if (st == VS_E_CUDA) set_error("WKB sizing failed: %s", cudaGetErrorString(cudaGetLastError()));
        free_wkb_plan(p);
        delete p;
        return st;
    }
    p->sizes = *sizes;
    *out = p;
    return VS_OK;
}

int vs_wkb_plan_decode(vs_wkb_plan* p, const vs_wkb_out* o) {
    if (!p || !o || !o->d_tags || !o->d_px || !o->d_py || !o->d_geom_off || !o->d_part_off || !o->d_ring_off ||
        (p->sizes.n_coords > 0 && (!o->d_x || !o->d_y))) {
        set_error("plan/out or an output buffer is NULL");
        return VS_E_ARG;
    }
    vs_context* ctx = p->ctx;
    VS_TRY(use_device(ctx->device));
    cudaStream_t s = ctx->stream;
    const int64_t n = p->in.n, R = p->sizes.n_rings;
    Scratch<int64_t> ring_src;
    Scratch<uint8_t> ring_fmt;
    VS_TRY(ring_src.alloc((size_t)(R > 0 ? R : 1), s));
    VS_TRY(ring_fmt.alloc((size_t)(R > 0 ? R : 1), s));
    VS_CUDA_TRY(cudaMemcpyAsync(o->d_tags, p->tags, (size_t)n, cudaMemcpyDeviceToDevice, s));
    VS_CUDA_TRY(cudaMemcpyAsync(o->d_px, p->px, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    VS_CUDA_TRY(cudaMemcpyAsync(o->d_py, p->py, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    if (n > 0) {
        wkb_fill_kernel<<<resident_grid(wkb_fill_kernel, n, 256), 256, 0, s>>>(
            p->in, p->tags, p->parts, p->rings, p->coords, o->d_geom_off, o->d_part_off, o->d_ring_off, ring_src.p,
            ring_fmt.p);
        VS_LAUNCHED("wkb_fill", s);
    }
    // closing entries: geom_off[n] = parts, part_off[P] = rings, ring_off[R] = coords
    VS_CUDA_TRY(cudaMemcpyAsync(o->d_geom_off + n, p->parts + n, 4, cudaMemcpyDeviceToDevice, s));
    VS_CUDA_TRY(cudaMemcpyAsync(o->d_part_off + p->sizes.n_parts, p->rings + n, 4, cudaMemcpyDeviceToDevice, s));
    VS_CUDA_TRY(cudaMemcpyAsync(o->d_ring_off + R, p->coords + n, 4, cudaMemcpyDeviceToDevice, s));
    if (R > 0) {
        wkb_copy_kernel<<<resident_grid(wkb_copy_kernel, R * 32, 256), 256, 0, s>>>(
            p->in.data, R, o->d_ring_off, ring_src.p, ring_fmt.p, o->d_x, o->d_y);
        VS_LAUNCHED("wkb_copy", s);
    }
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    return VS_OK;
}

int vs_wkb_plan_free(vs_wkb_plan* p) {
    if (!p) return VS_OK;
    use_device(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    free_wkb_plan(p);
    delete p;
    return VS_OK;
}

}  // extern "C"
