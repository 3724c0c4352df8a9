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
//   1. wkb_size_kernel (256 threads, tiles of 1024 rows, 4 rows a thread).
//      A tile's bytes are staged in shared memory by a bulk copy (TMA
//      engine, cp.async.bulk on an mbarrier) when they fit -- point columns:
//      21.5 KB a tile -- double-buffered so the next tile's copy is in flight
//      while this tile is parsed; larger tiles are parsed from global memory.
//      Every read is bounds-checked against the row's byte range.  Writes
//      the caller's tags and point coordinates, the row's part count into
//      geom_off and its ring / coordinate counts into scratch, and 64-bit
//      totals.
//   2. exclusive scans of the three counts, skipped when no row owns a part
//      (a column of points needs nothing more).
//   3. wkb_fill_kernel (thread per polygon row) walks the headers and writes
//      part_off, ring_off and, per ring, where its coordinates start and
//      their byte order / ordinate count.
//   4. wkb_copy_kernel (256 rings a block): thread per output coordinate,
//      its ring found by a binary search of the tile's ring offsets in
//      shared memory, so consecutive threads read consecutive coordinates
//      and write x / y coalesced whatever the ring sizes.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <new>

#include "primitives.cuh"
#include "tma.cuh"
#include "vs_common.cuh"

namespace vs {
namespace {

enum : int8_t { kTagNull = -1, kTagPoint = 0, kTagPolygon = 2, kTagMultiPolygon = 5 };
enum : int32_t { kRowOk = 0, kRowUnsupported = 1, kRowMalformed = 2 };

constexpr int kSizeThreads = 256;
constexpr int kRowsPerTile = 1024;   // rows of one size-kernel tile (4 a thread)
constexpr int kStageBytes = 22528;   // tiles of at most this many bytes (+ alignment) are staged
constexpr int kTotals = 10;          // 9 sums + error flags
constexpr int kCopyRings = 256;      // rings of one copy-kernel tile

struct WkbIn {
    const uint8_t* data;
    const int64_t* offsets;  // [n + 1] byte offsets of the rows
    const uint8_t* valid;    // nullable
    int64_t n;
};

// 32-bit little-endian word at any byte address: the aligned words that
// cover it, joined with a funnel shift.  The second word is read only when
// the value straddles it; it lies in the same aligned word as the value's
// last byte, so it is inside the buffer's allocation.
__device__ __forceinline__ uint32_t ld_u32_le(const uint8_t* p) {
    const uintptr_t a = (uintptr_t)p;
    const uint32_t* w = (const uint32_t*)(a & ~(uintptr_t)3);
    const uint32_t sh = (uint32_t)(a & 3) * 8;
    const uint32_t w0 = w[0];
    const uint32_t w1 = sh ? w[1] : 0u;
    return __funnelshift_r(w0, w1, sh);
}

__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

__device__ __forceinline__ double ld_f64(const uint8_t* p, bool little) {
    const uint32_t a = ld_u32_le(p), b = ld_u32_le(p + 4);
    const uint32_t lo = little ? a : bswap32(b);
    const uint32_t hi = little ? b : bswap32(a);
    return __hiloint2double((int)hi, (int)lo);
}

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
        const uint32_t v = ld_u32_le(p);
        p += 4;
        return little ? v : bswap32(v);
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

// Parse one non-null row held in [p, end).
__device__ RowCounts parse_row(const uint8_t* p, const uint8_t* end) {
    RowCounts rc{kTagNull, kRowOk, 0, 0, 0, 0.0, 0.0};
    rc.px = rc.py = __longlong_as_double(0x7ff8000000000000ll);
    Cursor c{p, end, true};
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
        rc.px = ld_f64(c.p, h.little);
        rc.py = ld_f64(c.p + 8, h.little);
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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Arm `bar` for `bytes` of bulk-copy transaction (this arrival completes the
// phase once they land).
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bulk copy global -> shared completing on `bar` (already armed for it).
__device__ __forceinline__ void bulk_copy(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Shared memory of the size kernel: two stages, each the tile's bytes and
// its row offsets.
constexpr int kStageStride = kStageBytes + 32;
constexpr int kOffsStride = (kRowsPerTile + 2) * 8;
constexpr size_t kSizeSmem = 2 * (size_t)(kStageStride + kOffsStride);

// One tile of the size kernel: rows [r0, r1), bytes [b0, b1).  A staged
// tile holds byte data[b0 - lead + k] at stage[k] (lead = misalignment of
// the range start; the 16-byte-aligned interior arrives by one bulk copy)
// and, when the offsets array is 16-byte aligned, offsets[r0 + j] at
// offs[j] for j in [0, r1 - r0].
struct SizeTile {
    int64_t r0, r1, b0, b1;
    uint32_t lead;
    bool staged;
};

__device__ __forceinline__ SizeTile make_tile(const WkbIn& in, int64_t t, int64_t b0, int64_t b1) {
    SizeTile tl;
    tl.r0 = t * kRowsPerTile;
    tl.r1 = tl.r0 + kRowsPerTile < in.n ? tl.r0 + kRowsPerTile : in.n;
    tl.b0 = b0;
    tl.b1 = b1;
    tl.lead = (uint32_t)((uintptr_t)(in.data + b0) & 15);
    tl.staged = b1 > b0 && (int64_t)tl.lead + (b1 - b0) <= kStageBytes;
    return tl;
}

__device__ __forceinline__ int64_t tile_row_end(const WkbIn& in, int64_t t) {
    const int64_t r1 = (t + 1) * kRowsPerTile;
    return r1 < in.n ? r1 : in.n;
}

// Start staging tile `tl`: thread 0 arms the barrier and issues the bulk
// copies (bytes interior, row offsets); the ragged head / tail bytes and the
// offsets past the last even count are plain stores, visible after the
// caller's next barrier.
__device__ __forceinline__ void issue_tile(const WkbIn& in, const SizeTile& tl, bool offs_aligned, uint8_t* buf,
                                           int64_t* offs, uint64_t* bar) {
    if (!tl.staged) return;
    const uint8_t* base = in.data + tl.b0 - tl.lead;  // 16-byte aligned
    const int64_t total = (int64_t)tl.lead + (tl.b1 - tl.b0);
    const int64_t i0 = ((int64_t)tl.lead + 15) & ~(int64_t)15;
    const int64_t i1 = total & ~(int64_t)15;
    const int64_t rows = tl.r1 - tl.r0;
    const int64_t bulk_rows = offs_aligned ? (rows & ~(int64_t)1) : 0;  // 16-byte multiple of offsets
    if (threadIdx.x == 0) {
        const uint32_t bytes = (uint32_t)((i1 > i0 ? i1 - i0 : 0) + 8 * bulk_rows);
        if (bytes) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar, bytes);
            if (i1 > i0) bulk_copy(buf + i0, base + i0, (uint32_t)(i1 - i0), bar);
            if (bulk_rows) bulk_copy(offs, in.offsets + tl.r0, (uint32_t)(8 * bulk_rows), bar);
        } else {
            mbar_arrive(bar);
        }
    }
    const int64_t h1 = i1 > i0 ? i0 : total;  // plain-loaded head [lead, h1), tail [i1, total)
    for (int64_t k = (int64_t)tl.lead + threadIdx.x; k < h1; k += blockDim.x) buf[k] = base[k];
    if (i1 > i0)
        for (int64_t k = i1 + threadIdx.x; k < total; k += blockDim.x) buf[k] = base[k];
    if (offs_aligned)
        for (int64_t j = bulk_rows + threadIdx.x; j <= rows; j += blockDim.x) offs[j] = in.offsets[tl.r0 + j];
}

// A 21-byte row at byte `off` of a stage: if it is a 2D Point without SRID
// (byte order 1 and type 1, or byte order 0 and type 1 big-endian), its
// coordinates.  Reads the 7 aligned words covering the row (the stage has 32
// bytes of slack past any tile) and joins them with funnel shifts.
__device__ __forceinline__ bool point21(const uint8_t* stage, uint32_t off, double& x, double& y) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(stage) + (off >> 2);
    const uint32_t sh = (off & 3) * 8;
    uint32_t v[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = w[k];
    uint32_t r[6];  // row bytes [4k, 4k + 4)
#pragma unroll
    for (int k = 0; k < 6; ++k) r[k] = __funnelshift_r(v[k], v[k + 1], sh);
    const uint32_t bo = r[0] & 0xffu;
    const uint32_t type = __funnelshift_r(r[0], r[1], 8);
    uint32_t c[4];  // row bytes [5 + 4k, 9 + 4k): x lo, x hi, y lo, y hi as stored
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = __funnelshift_r(r[k + 1], r[k + 2], 8);
    if (bo == 1 && type == 1u) {
        x = __hiloint2double((int)c[1], (int)c[0]);
        y = __hiloint2double((int)c[3], (int)c[2]);
        return true;
    }
    if (bo == 0 && type == 0x01000000u) {
        x = __hiloint2double((int)bswap32(c[0]), (int)bswap32(c[1]));
        y = __hiloint2double((int)bswap32(c[2]), (int)bswap32(c[3]));
        return true;
    }
    return false;
}

// totals: [0] points, [1] polygons, [2] multipolygons, [3] nulls, [4] unsupported, [5] malformed,
//         [6] parts, [7] rings, [8] coordinates (64-bit sums, to check the 32-bit offsets),
//         [9] error flags (bit 2: a staging wait gave up)
// Ring and coordinate counts are written only for rows that own a part (the
// others have none; wkb_zero_counts_kernel clears them when a scan follows).
__global__ void __launch_bounds__(kSizeThreads) wkb_size_kernel(const WkbIn in, int8_t* __restrict__ tags,
                                                               double* __restrict__ px, double* __restrict__ py,
                                                               uint32_t* __restrict__ parts,
                                                               uint32_t* __restrict__ rings,
                                                               uint32_t* __restrict__ coords,
                                                               unsigned long long* __restrict__ totals) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar[2];
    // stage s: bytes at smem + s * kStageStride, row offsets at offs_of(s)
    auto stage_of = [&](int st) { return smem + st * kStageStride; };
    auto offs_of = [&](int st) { return reinterpret_cast<int64_t*>(smem + 2 * kStageStride + st * kOffsStride); };
    const bool offs_aligned = ((uintptr_t)in.offsets & 15) == 0;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0]);
        mbar_init(&bar[1]);
    }
    __syncthreads();
    uint32_t cls[6] = {0, 0, 0, 0, 0, 0};
    unsigned long long sums[3] = {0, 0, 0};
    const int64_t n_tiles = (in.n + kRowsPerTile - 1) / kRowsPerTile;
    const int64_t G = gridDim.x;
    uint32_t parity = 0;  // bit s: the phase stage s waits for next
    int64_t t = blockIdx.x;
    SizeTile cur{};
    // byte range of the tile after next, loaded one iteration ahead
    int64_t pre_b0 = 0, pre_b1 = 0;
    if (t < n_tiles) {
        cur = make_tile(in, t, in.offsets[t * kRowsPerTile], in.offsets[tile_row_end(in, t)]);
        issue_tile(in, cur, offs_aligned, stage_of(0), offs_of(0), &bar[0]);
        if (t + G < n_tiles) {
            pre_b0 = in.offsets[(t + G) * kRowsPerTile];
            pre_b1 = in.offsets[tile_row_end(in, t + G)];
        }
    }
    for (int k = 0; t < n_tiles; t += G, ++k) {
        const int s = k & 1;
        // stage the next tile into the other buffer (its readers finished at
        // the end of the previous iteration)
        SizeTile nxt{};
        const bool has_next = t + G < n_tiles;
        if (has_next) {
            nxt = make_tile(in, t + G, pre_b0, pre_b1);
            issue_tile(in, nxt, offs_aligned, stage_of(s ^ 1), offs_of(s ^ 1), &bar[s ^ 1]);
            if (t + 2 * G < n_tiles) {
                pre_b0 = in.offsets[(t + 2 * G) * kRowsPerTile];
                pre_b1 = in.offsets[tile_row_end(in, t + 2 * G)];
            }
        }
        bool failed = false;
        if (cur.staged) {
            failed = !mbar_wait_bounded(&bar[s], (parity >> s) & 1u);
            parity ^= 1u << s;
        }
        if (__syncthreads_or(failed)) {
            // give up: record it, let the copies in flight land (bounded) and stop
            if (threadIdx.x == 0) {
                atomicOr(&totals[9], 4ull);
                if (cur.staged) mbar_wait_bounded(&bar[s], ((parity >> s) & 1u) ^ 1u);
                if (has_next && nxt.staged) mbar_wait_bounded(&bar[s ^ 1], (parity >> (s ^ 1)) & 1u);
            }
            break;
        }
        const bool soffs = cur.staged && offs_aligned;
        const uint8_t* cstage = stage_of(s);
        const int64_t* coffs = offs_of(s);
#pragma unroll 1
        for (int j = 0; j < kRowsPerTile / kSizeThreads; ++j) {
            const int rj = threadIdx.x + j * kSizeThreads;
            const int64_t i = cur.r0 + rj;
            if (i >= cur.r1) break;
            const int64_t bi = soffs ? coffs[rj] : in.offsets[i];
            const int64_t bj = soffs ? coffs[rj + 1] : in.offsets[i + 1];
            const bool valid = !in.valid || in.valid[i];
            const bool in_stage = cur.staged && bi >= cur.b0 && bj <= cur.b1;
            if (valid && in_stage && bj - bi == 21) {
                // the common row of a point column: a 2D Point without SRID
                double x, y;
                if (point21(cstage, cur.lead + (uint32_t)(bi - cur.b0), x, y)) {
                    tags[i] = kTagPoint;
                    px[i] = x;
                    py[i] = y;
                    parts[i] = 0;
                    ++cls[0];
                    continue;
                }
            }
            RowCounts rc{kTagNull, kRowOk, 0, 0, 0, 0.0, 0.0};
            rc.px = rc.py = __longlong_as_double(0x7ff8000000000000ll);
            if (valid && bj > bi) {
                if (in_stage) {
                    const uint8_t* q = cstage + cur.lead + (bi - cur.b0);
                    rc = parse_row(q, q + (bj - bi));
                } else {
                    rc = parse_row(in.data + bi, in.data + bj);
                }
            }
            tags[i] = rc.tag;
            px[i] = rc.px;
            py[i] = rc.py;
            parts[i] = rc.parts;
            if (rc.parts) {
                rings[i] = rc.rings;
                coords[i] = rc.coords > 0xffffffffull ? 0xffffffffu : (uint32_t)rc.coords;
            }
            cls[0] += rc.tag == kTagPoint;
            cls[1] += rc.tag == kTagPolygon;
            cls[2] += rc.tag == kTagMultiPolygon;
            cls[3] += rc.tag == kTagNull && rc.status == kRowOk;
            cls[4] += rc.status == kRowUnsupported;
            cls[5] += rc.status == kRowMalformed;
            sums[0] += rc.parts;
            sums[1] += rc.rings;
            sums[2] += rc.coords;
        }
        __syncthreads();  // this buffer's readers are done before it is refilled
        cur = nxt;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        unsigned long long v = k < 6 ? (unsigned long long)cls[k] : sums[k - 6];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&totals[k], v);
    }
}

// Before the scans: rows without parts get zero ring / coordinate counts.
__global__ void wkb_zero_counts_kernel(const uint32_t* __restrict__ parts, uint32_t* __restrict__ rings,
                                       uint32_t* __restrict__ coords, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (parts[i] == 0) {
            rings[i] = 0;
            coords[i] = 0;
        }
}

// Pass 3: thread per row; polygon rows write their part and ring offsets,
// and per ring where its coordinates start (bytes) and its format (bit 0
// little-endian, bits 1.. ordinates per coordinate).  Closing entries
// part_off[P] = R, ring_off[R] = C.
__global__ void wkb_fill_kernel(const WkbIn in, const int8_t* __restrict__ tags, const int32_t* __restrict__ geom_off,
                                const uint32_t* __restrict__ ring0, const uint32_t* __restrict__ coord0,
                                int32_t* __restrict__ part_off, int32_t* __restrict__ ring_off,
                                int64_t* __restrict__ ring_src, uint8_t* __restrict__ ring_fmt, int64_t P, int64_t R,
                                int64_t C) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        part_off[P] = (int32_t)R;
        ring_off[R] = (int32_t)C;
    }
    for (int64_t i = tid; i < in.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int8_t tag = tags[i];
        if (tag != kTagPolygon && tag != kTagMultiPolygon) continue;
        const bool multi = tag == kTagMultiPolygon;
        // the size pass parsed this row without overrunning it; the cursor
        // checks stay as a guard
        Cursor c{in.data + in.offsets[i], in.data + in.offsets[i + 1], true};
        const Header h = read_header(c);
        uint32_t part = (uint32_t)geom_off[i], ring = ring0[i], coord = coord0[i];
        const uint32_t n_parts = multi ? c.u32(h.little) : 1u;
        for (uint32_t k = 0; k < n_parts && c.ok; ++k) {
            const Header ph = multi ? read_header(c) : h;
            const uint32_t nr = c.u32(ph.little);
            if (nr == 0) continue;  // an empty polygon (part) owns no part entry
            part_off[part++] = (int32_t)ring;
            const uint64_t stride = 8u * (uint64_t)ph.dims;
            for (uint32_t r = 0; r < nr && c.ok; ++r) {
                const uint32_t np = c.u32(ph.little);
                ring_off[ring] = (int32_t)coord;
                ring_src[ring] = (int64_t)(c.p - in.data);
                ring_fmt[ring] = (uint8_t)((ph.little ? 1 : 0) | (ph.dims << 1));
                ++ring;
                c.skip((uint64_t)np * stride);
                coord += np;
            }
        }
    }
}

// Pass 4: tiles of kCopyRings rings; their offsets, sources and formats go
// to shared memory, then a thread per output coordinate finds its ring (the
// last ring starting at or before it) by binary search and copies it.
__global__ void __launch_bounds__(kCopyRings) wkb_copy_kernel(const uint8_t* __restrict__ data, int64_t n_rings,
                                                             const int32_t* __restrict__ ring_off,
                                                             const int64_t* __restrict__ ring_src,
                                                             const uint8_t* __restrict__ ring_fmt,
                                                             double* __restrict__ x, double* __restrict__ y) {
    __shared__ int32_t s_off[kCopyRings + 1];
    __shared__ int64_t s_src[kCopyRings];
    __shared__ uint8_t s_fmt[kCopyRings];
    for (int64_t r0 = (int64_t)blockIdx.x * kCopyRings; r0 < n_rings; r0 += (int64_t)gridDim.x * kCopyRings) {
        const int nr = (int)(n_rings - r0 < kCopyRings ? n_rings - r0 : kCopyRings);
        const int t = threadIdx.x;
        if (t < nr) {
            s_off[t] = ring_off[r0 + t];
            s_src[t] = ring_src[r0 + t];
            s_fmt[t] = ring_fmt[r0 + t];
        }
        if (t == 0) s_off[nr] = ring_off[r0 + nr];
        __syncthreads();
        const int32_t c0 = s_off[0], c1 = s_off[nr];
        for (int32_t c = c0 + t; c < c1; c += blockDim.x) {
            int lo = 0, hi = nr - 1;  // last j with s_off[j] <= c
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_off[mid] <= c) lo = mid;
                else hi = mid - 1;
            }
            const bool little = s_fmt[lo] & 1;
            const uint8_t* src = data + s_src[lo] + (int64_t)(c - s_off[lo]) * (8 * (s_fmt[lo] >> 1));
            x[c] = ld_f64(src, little);
            y[c] = ld_f64(src + 8, little);
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace vs

struct vs_wkb_plan {
    vs_context* ctx = nullptr;
    vs::WkbIn in{};
    vs_wkb_sizes sizes{};
    const int8_t* tags = nullptr;  // the caller's row outputs
    int32_t* geom_off = nullptr;
    uint32_t* scratch = nullptr;   // ring and coordinate start offsets, 2 x (n + 1); then 2 x 9 totals
};

using namespace vs;

extern "C" {

int vs_wkb_plan_create(vs_context* ctx, const uint8_t* d_wkb, const int64_t* d_offsets, const uint8_t* d_valid,
                       int64_t n, const vs_wkb_out* rows, vs_wkb_plan** out, vs_wkb_sizes* sizes) {
    if (!ctx || !out || !sizes || !rows || (n > 0 && (!d_wkb || !d_offsets)) || !rows->d_geom_off ||
        (n > 0 && (!rows->d_tags || !rows->d_px || !rows->d_py))) {
        set_error("ctx/out/sizes/rows, wkb/offsets or a row output is NULL");
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
    p->tags = rows->d_tags;
    p->geom_off = rows->d_geom_off;
    cudaStream_t s = ctx->stream;
    const size_t rows1 = (size_t)n + 1;
    // 8-byte aligned totals after the two offset arrays
    const size_t tot_at = (2 * rows1 + 1) & ~(size_t)1;
    if (cudaMallocAsync((void**)&p->scratch, (tot_at + 2 * kTotals) * sizeof(uint32_t), s) != cudaSuccess) {
        cudaGetLastError();
        set_error("WKB plan allocation failed (%lld rows)", (long long)n);
        delete p;
        return VS_E_OOM;
    }
    uint32_t* ring0 = p->scratch;
    uint32_t* coord0 = p->scratch + rows1;
    unsigned long long* totals = reinterpret_cast<unsigned long long*>(p->scratch + tot_at);
    int st = VS_OK;
    do {
        if (cudaMemsetAsync(totals, 0, kTotals * sizeof(unsigned long long), s) != cudaSuccess) {
            st = VS_E_CUDA;
            break;
        }
        if (n > 0) {
            const int64_t tiles = (n + kRowsPerTile - 1) / kRowsPerTile;
            if (cudaFuncSetAttribute(wkb_size_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kSizeSmem) != cudaSuccess) {
                st = VS_E_CUDA;
                break;
            }
            wkb_size_kernel<<<resident_grid(wkb_size_kernel, tiles * kSizeThreads, kSizeThreads, kSizeSmem),
                              kSizeThreads, kSizeSmem, s>>>(p->in, rows->d_tags, rows->d_px, rows->d_py,
                                                            reinterpret_cast<uint32_t*>(rows->d_geom_off), ring0,
                                                            coord0, totals);
            if (cudaGetLastError() != cudaSuccess) {
                st = VS_E_CUDA;
                break;
            }
            ++g_launches;
        }
        unsigned long long t[kTotals] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (cudaMemcpyAsync(t, totals, sizeof(t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
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
        sizes->n_parts = (int64_t)t[6];
        sizes->n_rings = (int64_t)t[7];
        sizes->n_coords = (int64_t)t[8];
        if (t[9] & 4ull) {
            set_error("WKB sizing: a shared-memory staging copy did not complete in time");
            st = VS_E_TIMEOUT;
            break;
        }
        if (t[6] > 0x7fffffffull || t[7] > 0x7fffffffull || t[8] > 0x7fffffffull) {
            set_error("%llu parts, %llu rings, %llu coordinates: more than the 32-bit offsets address", t[6], t[7],
                      t[8]);
            st = VS_E_ARG;
            break;
        }
        if (t[6] == 0) {  // no row owns a part: geom_off is all zeros already
            if (cudaMemsetAsync(rows->d_geom_off + n, 0, sizeof(int32_t), s) != cudaSuccess) st = VS_E_CUDA;
            break;
        }
        wkb_zero_counts_kernel<<<resident_grid(wkb_zero_counts_kernel, n, 256), 256, 0, s>>>(
            reinterpret_cast<const uint32_t*>(rows->d_geom_off), ring0, coord0, n);
        if (cudaGetLastError() != cudaSuccess) {
            st = VS_E_CUDA;
            break;
        }
        ++g_launches;
        // exclusive scans in place; the totals land in the n-th entries
        st = exclusive_scan_u32(reinterpret_cast<uint32_t*>(rows->d_geom_off),
                                reinterpret_cast<uint32_t*>(rows->d_geom_off), n,
                                reinterpret_cast<uint32_t*>(rows->d_geom_off) + n, s);
        if (st == VS_OK) st = exclusive_scan_u32(ring0, ring0, n, ring0 + n, s);
        if (st == VS_OK) st = exclusive_scan_u32(coord0, coord0, n, coord0 + n, s);
    } while (false);
    if (st != VS_OK) {
        if (st == VS_E_CUDA) set_error("WKB sizing failed: %s", cudaGetErrorString(cudaGetLastError()));
        cudaFreeAsync(p->scratch, s);
        delete p;
        return st;
    }
    p->sizes = *sizes;
    *out = p;
    return VS_OK;
}

int vs_wkb_plan_decode(vs_wkb_plan* p, const vs_wkb_out* o) {
    if (!p || !o || !o->d_part_off || !o->d_ring_off || (p->sizes.n_coords > 0 && (!o->d_x || !o->d_y))) {
        set_error("plan/out or an output buffer is NULL");
        return VS_E_ARG;
    }
    vs_context* ctx = p->ctx;
    VS_TRY(use_device(ctx->device));
    cudaStream_t s = ctx->stream;
    const int64_t n = p->in.n, P = p->sizes.n_parts, R = p->sizes.n_rings, C = p->sizes.n_coords;
    if (P == 0) {
        VS_CUDA_TRY(cudaMemsetAsync(o->d_part_off, 0, sizeof(int32_t), s));
        VS_CUDA_TRY(cudaMemsetAsync(o->d_ring_off, 0, sizeof(int32_t), s));
    } else {
        const uint32_t* ring0 = p->scratch;
        const uint32_t* coord0 = p->scratch + n + 1;
        Scratch<int64_t> ring_src;
        Scratch<uint8_t> ring_fmt;
        VS_TRY(ring_src.alloc((size_t)R, s));
        VS_TRY(ring_fmt.alloc((size_t)R, s));
        wkb_fill_kernel<<<resident_grid(wkb_fill_kernel, n, 256), 256, 0, s>>>(
            p->in, p->tags, p->geom_off, ring0, coord0, o->d_part_off, o->d_ring_off, ring_src.p, ring_fmt.p, P, R, C);
        VS_LAUNCHED("wkb_fill", s);
        if (C > 0) {
            wkb_copy_kernel<<<resident_grid(wkb_copy_kernel, R, kCopyRings), kCopyRings, 0, s>>>(
                p->in.data, R, o->d_ring_off, ring_src.p, ring_fmt.p, o->d_x, o->d_y);
            VS_LAUNCHED("wkb_copy", s);
        }
    }
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    return VS_OK;
}

int vs_wkb_plan_free(vs_wkb_plan* p) {
    if (!p) return VS_OK;
    use_device(p->ctx->device);
    cudaFreeAsync(p->scratch, p->ctx->stream);
    cudaStreamSynchronize(p->ctx->stream);
    delete p;
    return VS_OK;
}

}  // extern "C"
