// LBVH Barnes-Hut: the replacement for Barnes_Hut::make_tree/compute_forces
// (src/solvers/barnes_hut.cpp:309-418, bh_specialization.cpp:30-46) and the
// OpenCL BH_hyper pipeline (src/solvers/full_GPU.cpp:54-339,519-527 with
// include/Aster/kernels/{morton_writer,radix,BHH_specific}.cl.h).
//
// Pipeline per force evaluation (all on one stream, no host sync):
//   box      max |coordinate| of the FP64 state (fused into the drift kernel
//            during time stepping, a separate reduction otherwise)
//   morton   30-bit code as the reference get_morton: x' = (x+B)/(2B),
//            q = min(trunc(x' * 1024), 1023), interleave z|y|x (63-bit: 21
//            bits per axis). IEEE FP64 add/div, no contraction: bit-exact.
//   sort     stable LSD radix sort of (code, body index), 8-bit digits:
//            per pass a tile histogram, a per-digit scan over tiles, a stable
//            scatter (warp match-any ranking). Ties keep body-index order.
//   karras   Karras (2012) node split exactly as barnes_hut.cpp:338-396
//            (tie-break 32 + clz(i ^ j) on sorted positions), children,
//            parents and leaf ranges; the same kernel gathers the leaves.
//   bottomup one thread per leaf climbs with an atomic arrival counter per
//            node; the second arrival merges the children: FP64 mass and
//            centre of mass in NodesArray::unite order (barnes_hut.cpp:137-152,
//            bit-exact), FP32 AABB, squared opening radius
//            r_crit = l/theta + |com - box centre| (rounded up to FP32).
//   walk     one warp per group (a subtree of <= 64 leaves whose parent holds
//            more): a shared-memory stack walk that opens a node for the whole
//            group unless its FP32 centre of mass lies farther than r_crit
//            from the group's FP32 box; accepted nodes are appended to a
//            shared interaction list and evaluated 32 at a time by every lane
//            (FP32 on group-relative double-single coordinates, or FP64).
// Node numbering is the reference's: leaves 0..n-1 (sorted order), internal
// n..2n-2, root n, -1 = no child.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "aster_internal.cuh"
#include "pn.cuh"

namespace {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;  // 2048 keys per block
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int RADIX = 256;
static_assert(SORT_THREADS == RADIX, "the scan and scatter kernels give each thread one digit");
constexpr int MAX_CLIMB = 160;     // bottom-up level cap (tree depth <= 97 for 63-bit codes)
#ifndef ASTER_WALK_WARPS
#define ASTER_WALK_WARPS 4
#endif
#ifndef ASTER_WALK_MINBLOCKS
#define ASTER_WALK_MINBLOCKS 5
#endif
#ifndef ASTER_WALK_UNROLL
#define ASTER_WALK_UNROLL 8
#endif
constexpr int WALK_WARPS = ASTER_WALK_WARPS;  // warps (groups in flight) per block
constexpr int WALK_UNROLL = ASTER_WALK_UNROLL;
constexpr int WALK_STACK = 1024;   // nodes per warp
constexpr int GROUP_MAX = 64;      // leaves per walk group (1 or 2 per lane)
// Interaction list: evaluated (and its FP32 partial sums folded into the
// compensated accumulators) every WALK_FLUSH entries; capacity = flush - 1 +
// the 64 entries one round can append. The post-Newtonian mixed walk, whose
// entries also carry a velocity, flushes every WALK_FLUSH_PN.
constexpr int WALK_FLUSH_MIXED = 128, WALK_FLUSH_FP64 = 32, WALK_FLUSH_PN = 64;
constexpr int WALK_LIST_MIXED = 192, WALK_LIST_FP64 = 96, WALK_LIST_PN = 128;

// ----------------------------------------------------------------- box
__device__ __forceinline__ double warp_max_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void __launch_bounds__(256) k_box(int64_t n, const double4* __restrict__ pm,
                                             unsigned long long* __restrict__ box_bits) {
    __shared__ double red[8];
    double b = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double4 p = pm[i];
        b = fmax(b, fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))));
    }
    b = warp_max_d(b);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_max_d(v);
        if (threadIdx.x == 0) atomicMax(box_bits, (unsigned long long)__double_as_longlong(v));
    }
}

// -------------------------------------------------------------- morton
__device__ __forceinline__ uint32_t part1by2_32(uint32_t n) {
    n = (n | (n << 16)) & 0x030000FFu;
    n = (n | (n << 8)) & 0x0300F00Fu;
    n = (n | (n << 4)) & 0x030C30C3u;
    n = (n | (n << 2)) & 0x09249249u;
    return n;
}

__device__ __forceinline__ uint64_t part1by2_64(uint64_t n) {
    n &= 0x1FFFFFull;
    n = (n | (n << 32)) & 0x001F00000000FFFFull;
    n = (n | (n << 16)) & 0x001F0000FF0000FFull;
    n = (n | (n << 8)) & 0x100F00F00F00F00Full;
    n = (n | (n << 4)) & 0x10C30C30C30C30C3ull;
    n = (n | (n << 2)) & 0x1249249249249249ull;
    return n;
}

// (x + B) / (2B) * scale truncated and clamped to maxv; NaN / negative -> 0.
__device__ __forceinline__ uint32_t quantize(double x, double B, double scale, uint32_t maxv) {
    double t = __ddiv_rn(__dadd_rn(x, B), __dmul_rn(2.0, B));
    double s = __dmul_rn(t, scale);
    if (!(s > 0.0)) return 0u;
    if (s >= 4294967296.0) return maxv;
    uint32_t q = (uint32_t)s;
    return q < maxv ? q : maxv;
}

// OpenCL gen_mortons (morton_writer.cl.h:72-122): clamp to [0,1], 1024 max,
// (ushort), so +B wraps to 0 through the 10-bit expansion mask.
__device__ __forceinline__ uint32_t quantize_compat(double x, double B) {
    double t = __ddiv_rn(__dadd_rn(x, B), __dmul_rn(2.0, B));
    t = fmin(fmax(t, 0.0), 1.0);
    uint32_t v = (uint32_t)__dmul_rn(t, 1024.0);
    v = v < 1024u ? v : 1024u;
    return (uint32_t)(uint16_t)v;
}

template <class KeyT, int MODE>  // MODE 0: 30-bit, 1: 63-bit, 2: 30-bit compat
__global__ void __launch_bounds__(256) k_morton(int64_t n, const double4* __restrict__ pm,
                                                const unsigned long long* __restrict__ box_bits,
                                                KeyT* __restrict__ codes) {
    const double B = __longlong_as_double((long long)*box_bits);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 p = pm[i];
        if (MODE == 0) {
            uint32_t ix = quantize(p.x, B, 1024.0, 1023u), iy = quantize(p.y, B, 1024.0, 1023u),
                     iz = quantize(p.z, B, 1024.0, 1023u);
            codes[i] = (KeyT)((part1by2_32(iz) << 2) | (part1by2_32(iy) << 1) | part1by2_32(ix));
        } else if (MODE == 1) {
            uint64_t ix = quantize(p.x, B, 2097152.0, 2097151u), iy = quantize(p.y, B, 2097152.0, 2097151u),
                     iz = quantize(p.z, B, 2097152.0, 2097151u);
            codes[i] = (KeyT)((part1by2_64(iz) << 2) | (part1by2_64(iy) << 1) | part1by2_64(ix));
        } else {
            uint32_t ix = quantize_compat(p.x, B), iy = quantize_compat(p.y, B), iz = quantize_compat(p.z, B);
            codes[i] = (KeyT)(part1by2_32(ix) | (part1by2_32(iy) << 1) | (part1by2_32(iz) << 2));
        }
    }
}

// ---------------------------------------------------------------- sort
template <class KeyT>
__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist(int64_t n, const KeyT* __restrict__ keys, int shift,
                                                            int nblocks, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[SORT_WARPS][RADIX];
    const int warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < SORT_WARPS * RADIX; d += SORT_THREADS) (&h[0][0])[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * SORT_TILE;
    KeyT k[SORT_ITEMS];  // all loads in flight before the first count
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const int64_t i = base + (int64_t)r * SORT_THREADS + threadIdx.x;
        k[r] = i < n ? keys[i] : (KeyT)0;
    }
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const int64_t i = base + (int64_t)r * SORT_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[warp][(uint32_t)(k[r] >> shift) & (RADIX - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) {
        uint32_t s = 0;
        for (int w = 0; w < SORT_WARPS; ++w) s += h[w][d];
        hist[(int64_t)d * nblocks + blockIdx.x] = s;
    }
}

// Block-wide exclusive scan of one uint32 per thread (blockDim.x <= 1024,
// multiple of 32); returns the exclusive prefix, *total gets the block sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem32, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem32[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? smem32[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) smem32[lane] = w;  // inclusive warp sums
    }
    __syncthreads();
    const uint32_t before = warp ? smem32[warp - 1] : 0u;
    if (total) *total = smem32[nw - 1];
    __syncthreads();
    return before + x - v;
}

// Per digit d (one block each): exclusive scan of the per-tile counts
// hist[d*nblocks + b] over b, in place; digit_tot[d] = the digit's total.
__global__ void __launch_bounds__(1024) k_scan_digits(uint32_t* __restrict__ hist, int nblocks,
                                                      uint32_t* __restrict__ digit_tot) {
    __shared__ uint32_t s32[32];
    uint32_t* row = hist + (int64_t)blockIdx.x * nblocks;
    uint32_t carry = 0;
    for (int base = 0; base < nblocks; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const uint32_t v = i < nblocks ? row[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(v, s32, &tot);
        if (i < nblocks) row[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) digit_tot[blockIdx.x] = carry;
}

// Stable scatter of one 8-bit digit. Warp w of the block owns the 256 keys
// [w*256, w*256+256) of the tile and ranks them round by round (32 consecutive
// keys per round) with __match_any_sync, so ranks follow input order.
// Global position = (keys of smaller digits) + (same digit in earlier tiles)
// + (same digit earlier in this tile).
template <class KeyT, bool IDENTITY_VALS>
__global__ void __launch_bounds__(SORT_THREADS, 4) k_sort_scatter(int64_t n, const KeyT* __restrict__ kin,
                                                               const int32_t* __restrict__ vin, KeyT* __restrict__ kout,
                                                               int32_t* __restrict__ vout, int shift, int nblocks,
                                                               const uint32_t* __restrict__ tile_off,
                                                               const uint32_t* __restrict__ digit_tot) {
    __shared__ uint32_t wh[SORT_WARPS][RADIX];
    __shared__ uint32_t dstart[RADIX];
    __shared__ uint32_t gofs[RADIX];
    __shared__ uint32_t s32[32];
    __shared__ KeyT sk[SORT_TILE];
    __shared__ int32_t sv[SORT_TILE];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t tile0 = (int64_t)blockIdx.x * SORT_TILE;
    KeyT key[SORT_ITEMS];
    int32_t val[SORT_ITEMS];
    // the tile's keys and values: all loads in flight before the ranking
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const int64_t i = tile0 + warp * (32 * SORT_ITEMS) + r * 32 + lane;
        const bool ok = i < n;
        key[r] = ok ? kin[i] : (KeyT)0;
        val[r] = ok ? (IDENTITY_VALS ? (int32_t)i : vin[i]) : 0;
    }
    const uint32_t toff = tile_off[(int64_t)threadIdx.x * nblocks + blockIdx.x];  // digit threadIdx.x
    for (int d = threadIdx.x; d < SORT_WARPS * RADIX; d += SORT_THREADS) (&wh[0][0])[d] = 0;
    // global base of each digit: exclusive scan of the digit totals
    const uint32_t gb = block_exclusive_scan(digit_tot[threadIdx.x], s32, nullptr);
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t rank[SORT_ITEMS];
    uint32_t dig[SORT_ITEMS];
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const int64_t i = tile0 + warp * (32 * SORT_ITEMS) + r * 32 + lane;
        const bool ok = i < n;
        const uint32_t d = ok ? ((uint32_t)(key[r] >> shift) & (RADIX - 1)) : 0xFFFFu;
        dig[r] = d;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = 0;
        if (ok) before = wh[warp][d];
        __syncwarp();
        rank[r] = before + __popc(peers & lt);
        if (ok && (peers & lt) == 0) wh[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps, then over digits (block-local start)
    uint32_t tot = 0;
    for (int w = 0; w < SORT_WARPS; ++w) {
        const uint32_t t = wh[w][threadIdx.x];
        wh[w][threadIdx.x] = tot;
        tot += t;
    }
    const uint32_t ds = block_exclusive_scan(tot, s32, nullptr);
    dstart[threadIdx.x] = ds;
    // output position of the tile's p-th key (digit d) = gofs[d] + p
    gofs[threadIdx.x] = gb + toff - ds;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        if (dig[r] < RADIX) {
            const uint32_t pos = dstart[dig[r]] + wh[warp][dig[r]] + rank[r];
            sk[pos] = key[r];
            sv[pos] = val[r];
        }
    }
    __syncthreads();
    const int64_t valid = min((int64_t)SORT_TILE, n - tile0);
    for (int p = threadIdx.x; p < valid; p += SORT_THREADS) {
        const KeyT k = sk[p];
        const uint32_t d = (uint32_t)(k >> shift) & (RADIX - 1);
        const int64_t g = (int64_t)(uint32_t)(gofs[d] + (uint32_t)p);
        kout[g] = k;
        vout[g] = sv[p];
    }
}

template <class KeyT>
__global__ void k_reverse(int64_t n, const KeyT* __restrict__ kin, const int32_t* __restrict__ vin,
                          KeyT* __restrict__ kout, int32_t* __restrict__ vout) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        kout[i] = kin[n - 1 - i];
        vout[i] = vin[n - 1 - i];
    }
}

// A leaf's box: its position rounded outwards to FP32 (not stored: computed
// from the leaf's node_cm wherever it is needed).
__device__ __forceinline__ float4 leaf_lo(const double4 p) {
    return make_float4(__double2float_rd(p.x), __double2float_rd(p.y), __double2float_rd(p.z), 0.f);
}
__device__ __forceinline__ float4 leaf_hi(const double4 p) {
    return make_float4(__double2float_ru(p.x), __double2float_ru(p.y), __double2float_ru(p.z), 0.f);
}

// Traversal data of a node (the walk's view of it): h = (rn(com), rn(mass)),
// l = (com - rn(com), rcrit2). Internal node: the squared opening radius
// r_crit = l/theta + |com - box centre| (l = longest AABB side; FP64, rounded
// up to FP32). Leaf: rcrit2 = 0.
__device__ __forceinline__ void node_trav(const double4 c, const float4 lo, const float4 hi, double theta, float4& h,
                                          float4& l) {
    const double ex = __dsub_rn((double)hi.x, (double)lo.x), ey = __dsub_rn((double)hi.y, (double)lo.y),
                 ez = __dsub_rn((double)hi.z, (double)lo.z);
    double lmax = 0.0;
    lmax = ex > lmax ? ex : lmax;
    lmax = ey > lmax ? ey : lmax;
    lmax = ez > lmax ? ez : lmax;
    const double cx = __dmul_rn(0.5, __dadd_rn((double)lo.x, (double)hi.x));
    const double cy = __dmul_rn(0.5, __dadd_rn((double)lo.y, (double)hi.y));
    const double cz = __dmul_rn(0.5, __dadd_rn((double)lo.z, (double)hi.z));
    const double dx = __dsub_rn(c.x, cx), dy = __dsub_rn(c.y, cy), dz = __dsub_rn(c.z, cz);
    const double delta = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    const double rc = __dadd_rn(__ddiv_rn(lmax, theta), delta);
    ds_split(c.x, h.x, l.x);
    ds_split(c.y, h.y, l.y);
    ds_split(c.z, h.z, l.z);
    h.w = __double2float_rn(c.w);
    l.w = __double2float_ru(__dmul_rn(rc, rc));
}
__device__ __forceinline__ void leaf_trav(const double4 c, float4& h, float4& l) {
    ds_split(c.x, h.x, l.x);
    ds_split(c.y, h.y, l.y);
    ds_split(c.z, h.z, l.z);
    h.w = __double2float_rn(c.w);
    l.w = 0.f;
}

// The child record of an internal node: the traversal data of both children
// in one contiguous 64 bytes, so opening a node costs one load, each field as
// a (left, right) pair so that the walk's paired FP32 opening test and
// list-entry arithmetic read aligned register pairs:
// (xL xR yL yR) (zL zR mL mR) (lxL lxR lyL lyR) (lzL lzR rcrit2L rcrit2R).
// Child ids below n are leaves (their boxes are not needed).
__device__ __forceinline__ void put_child_record(float4* __restrict__ dst, int64_t n, double theta, int32_t L,
                                                 const double4 cL, const float4 loL, const float4 hiL, int32_t R,
                                                 const double4 cR, const float4 loR, const float4 hiR) {
    float4 hL, lL, hR, lR;
    if (L < n) leaf_trav(cL, hL, lL);
    else node_trav(cL, loL, hiL, theta, hL, lL);
    if (R < n) leaf_trav(cR, hR, lR);
    else node_trav(cR, loR, hiR, theta, hR, lR);
    dst[0] = make_float4(hL.x, hR.x, hL.y, hR.y);
    dst[1] = make_float4(hL.z, hR.z, hL.w, hR.w);
    dst[2] = make_float4(lL.x, lR.x, lL.y, lR.y);
    dst[3] = make_float4(lL.z, lR.z, lL.w, lR.w);
}

// -------------------------------------------------------------- karras
template <class KeyT, bool COMPAT>
__device__ __forceinline__ int kdelta(const KeyT* __restrict__ codes, const int32_t* __restrict__ perm,
                                      int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const KeyT a = codes[i], b = codes[j];
    if (a == b) {
        const uint32_t t = COMPAT ? (uint32_t)(perm[i] ^ perm[j]) : (uint32_t)(i ^ j);
        return (sizeof(KeyT) == 8 ? 64 : 32) + __clz((int)t);
    }
    return sizeof(KeyT) == 8 ? __clzll((long long)(a ^ b)) : __clz((int)(uint32_t)(a ^ b));
}

// Walk groups: a node whose subtree holds at most GROUP_MAX leaves while its
// parent's holds more (the root when n <= GROUP_MAX). Its leaves are a
// contiguous sorted run sharing a Morton prefix, so the group is spatially
// compact (a fixed run of consecutive sorted bodies is not: it can straddle a
// Morton jump and span the whole system). Listed here as (first leaf, size):
// internal node n + i knows its own range and both children's, and thread i
// lists the groups among its children, so groups come roughly in sorted-leaf
// order, which keeps consecutive walk groups close in space. Groups of more
// than 32 bodies (a second pass over the list, or two bodies per lane) fill
// the array from the front, groups of at most 32 (one pass) from the back;
// the walk takes the front part first, so its last wave is made of the
// cheaper groups and warps finish closer together.
constexpr int GROUP_SMALL = 32;
__device__ __forceinline__ void list_group(int2* groups, unsigned int* ngroups, int64_t n, int64_t first,
                                           int64_t size) {
    if (size > GROUP_SMALL)
        groups[atomicAdd(&ngroups[0], 1u)] = make_int2((int32_t)first, (int32_t)size);
    else
        groups[n - 1 - atomicAdd(&ngroups[3], 1u)] = make_int2((int32_t)first, (int32_t)size);
}
template <class KeyT, bool COMPAT>
__global__ void __launch_bounds__(256) k_karras(int64_t n, const KeyT* __restrict__ codes, const int32_t* __restrict__ perm,
                                                const double4* __restrict__ pm, int32_t* __restrict__ parent,
                                                int32_t* __restrict__ sib, int32_t* __restrict__ rlo, int32_t* __restrict__ rhi,
                                                int2* __restrict__ child, uint32_t* __restrict__ counters,
                                                double4* __restrict__ node_cm, int2* __restrict__ groups,
                                                unsigned int* __restrict__ ngroups) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        // leaf i: gather body perm[i]
        {
            node_cm[i] = pm[perm[i]];
            rlo[i] = (int32_t)i;
            rhi[i] = (int32_t)i;
            if (n == 1) {
                parent[0] = -1;
                list_group(groups, ngroups, n, 0, 1);
            }
        }
        if (i == n - 1) {
            parent[n] = -1;  // root (n >= 2) or unused slot
            continue;
        }
        const int dl = i == 0 ? -1 : kdelta<KeyT, COMPAT>(codes, perm, n, i, i - 1);
        const int dr = kdelta<KeyT, COMPAT>(codes, perm, n, i, i + 1);
        const int64_t d = dr > dl ? 1 : -1;
        const int dmin = d == 1 ? dl : dr;
        int64_t lmax = 2;
        while (kdelta<KeyT, COMPAT>(codes, perm, n, i, i + lmax * d) > dmin) lmax *= 2;
        int64_t l = 0;
        for (int64_t t = lmax / 2; t >= 1; t /= 2)
            if (kdelta<KeyT, COMPAT>(codes, perm, n, i, i + (l + t) * d) > dmin) l += t;
        const int64_t j = i + l * d;
        const int dnode = kdelta<KeyT, COMPAT>(codes, perm, n, i, j);
        int64_t s = 0;
        const int64_t range = j > i ? j - i : i - j;
        for (int64_t t = (range + 1) / 2; t >= 1; t = (t + 1) / 2) {
            if (kdelta<KeyT, COMPAT>(codes, perm, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        const int64_t gamma = i + s * d + (d < 0 ? d : 0);
        const int64_t lo = i < j ? i : j, hi = i < j ? j : i;
        const int64_t node = n + i;
        const int32_t L = (int32_t)(lo == gamma ? gamma : n + gamma);
        const int32_t R = (int32_t)(hi == gamma + 1 ? gamma + 1 : n + gamma + 1);
        child[node] = make_int2(L, R);
        parent[L] = (int32_t)node;
        parent[R] = (int32_t)node;
        sib[L] = R;   // >= 0: the node is a left child
        sib[R] = ~L;  // <  0: a right child, sibling ~sib
        rlo[node] = (int32_t)lo;
        rhi[node] = (int32_t)hi;
        counters[i] = 0u;
        if (hi - lo + 1 > GROUP_MAX) {
            const int64_t szL = gamma - lo + 1, szR = hi - gamma;
            if (szL <= GROUP_MAX) list_group(groups, ngroups, n, lo, szL);
            if (szR <= GROUP_MAX) list_group(groups, ngroups, n, gamma + 1, szR);
        } else if (i == 0) {  // the root holds at most GROUP_MAX leaves
            list_group(groups, ngroups, n, 0, n);
        }
    }
}

// ------------------------------------------------------------ bottom-up
__device__ __forceinline__ double4 ld_cg(const double4* p) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ld_cg(const float4* p) { return __ldcg(p); }

// Bottom-up merge: every leaf climbs towards the root; at each internal node
// the first arrival stops and the second merges the two children in
// NodesArray::unite order. Two phases, so that the climbs through global
// memory are short and all in flight at once:
//  1. k_bottom_up_local: a block owns BU_LEAVES consecutive sorted leaves and
//     completes every node whose leaf range lies inside them, with arrival
//     counters and node data in shared memory (block-scope fences). A node
//     whose parent's range leaves the block is a frontier node.
//  2. k_bottom_up_front: one climb per frontier node through the remaining
//     (boundary-crossing) nodes with global counters and device-scope fences.
// sib[v] names v's sibling and side (>= 0: v is a left child), so a climb
// reads both children without loading child[parent] first.
#ifndef ASTER_BU_LEAVES
#define ASTER_BU_LEAVES 64
#endif
constexpr int BU_LEAVES = ASTER_BU_LEAVES;

__device__ __forceinline__ void bu_merge(const double4 cl, const double4 cr, const float4 l0, const float4 l1,
                                         const float4 h0, const float4 h1, double4& cm, float4& lo, float4& hi) {
    // NodesArray::unite order: M = m_R + m_L; c = (c_R m_R + c_L m_L) / M.
    // A node without mass (M <= 0: only massless bodies below it) takes the
    // midpoint (c_R + c_L) / 2, finite, so that its ancestors' centres stay
    // finite too (unite leaves such a node's previous contents in place).
    const double M = __dadd_rn(cr.w, cl.w);
    if (M > 0.0) {
        cm.x = __ddiv_rn(__dadd_rn(__dmul_rn(cr.x, cr.w), __dmul_rn(cl.x, cl.w)), M);
        cm.y = __ddiv_rn(__dadd_rn(__dmul_rn(cr.y, cr.w), __dmul_rn(cl.y, cl.w)), M);
        cm.z = __ddiv_rn(__dadd_rn(__dmul_rn(cr.z, cr.w), __dmul_rn(cl.z, cl.w)), M);
    } else {
        cm.x = __dmul_rn(0.5, __dadd_rn(cr.x, cl.x));
        cm.y = __dmul_rn(0.5, __dadd_rn(cr.y, cl.y));
        cm.z = __dmul_rn(0.5, __dadd_rn(cr.z, cl.z));
    }
    cm.w = M;
    lo = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.f);
    hi = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.f);
}

__global__ void __launch_bounds__(BU_LEAVES, 1024 / BU_LEAVES) k_bottom_up_local(
    int64_t n, const int32_t* __restrict__ parent, const int32_t* __restrict__ sib, const int32_t* __restrict__ rlo,
    const int32_t* __restrict__ rhi, double4* __restrict__ node_cm, float4* __restrict__ bmin,
    float4* __restrict__ bmax, int32_t* __restrict__ front, unsigned int* __restrict__ nfront, int* __restrict__ err,
    double theta, const int2* __restrict__ child, float4* __restrict__ crec) {
    // [0][j]: leaf B0 + j; [1][j]: internal node n + B0 + j (Karras numbering:
    // an internal node inside the block has its index inside the block too)
    __shared__ double4 s_cm[2][BU_LEAVES];
    __shared__ float4 s_lo[2][BU_LEAVES], s_hi[2][BU_LEAVES];
    __shared__ int32_t s_par[2][BU_LEAVES], s_sib[2][BU_LEAVES];
    __shared__ int32_t s_rlo[BU_LEAVES], s_rhi[BU_LEAVES];
    __shared__ unsigned int s_cnt[BU_LEAVES];
    __shared__ int32_t s_front[BU_LEAVES];  // frontier nodes are disjoint subtrees: at most one per leaf
    __shared__ unsigned int s_nf, s_fbase;
    const int j = threadIdx.x;
    const int64_t B0 = (int64_t)blockIdx.x * BU_LEAVES;
    const int64_t B1 = (B0 + BU_LEAVES < n ? B0 + BU_LEAVES : n) - 1;
    const int64_t k = B0 + j;
    s_cnt[j] = 0u;
    if (j == 0) s_nf = 0u;
    if (k < n) {
        const double4 lc = node_cm[k];
        s_cm[0][j] = lc;
        s_lo[0][j] = leaf_lo(lc);
        s_hi[0][j] = leaf_hi(lc);
        s_par[0][j] = parent[k];
        s_sib[0][j] = sib[k];
    }
    if (k < n - 1) {
        s_par[1][j] = parent[n + k];
        s_sib[1][j] = sib[n + k];
        s_rlo[j] = rlo[n + k];
        s_rhi[j] = rhi[n + k];
    }
    __syncthreads();
    int side = 0, slot = j;
    int32_t cur = (int32_t)k;
    double4 cm = make_double4(0, 0, 0, 0);
    float4 lo = make_float4(0, 0, 0, 0), hi = lo;
    if (k < n) {
        cm = s_cm[0][j];
        lo = s_lo[0][j];
        hi = s_hi[0][j];
    }
    for (int level = 0; k < n; ++level) {
        const int32_t par = s_par[side][slot];
        if (par < 0) break;  // the root
        const int64_t ip = (int64_t)par - n;
        const bool local = ip >= B0 && ip <= B1 && s_rlo[ip - B0] >= B0 && s_rhi[ip - B0] <= B1;
        if (!local) {
            s_front[atomicAdd(&s_nf, 1u)] = cur;  // its data is in global memory already
            break;
        }
        if (level >= MAX_CLIMB) {
            atomicOr(err, ASTER_DEVERR_TREE);
            break;
        }
        const int pslot = (int)(ip - B0);
        __threadfence_block();  // own node data (shared) before the arrival count
        if (atomicAdd(&s_cnt[pslot], 1u) == 0u) break;
        __threadfence_block();
        const int32_t sb = s_sib[side][slot];
        const int32_t so = sb >= 0 ? sb : ~sb;
        const int oside = so >= n ? 1 : 0;
        const int oslot = (int)(oside ? (int64_t)so - n - B0 : (int64_t)so - B0);
        const double4 oc = s_cm[oside][oslot];
        const float4 ol = s_lo[oside][oslot], oh = s_hi[oside][oslot];
        const bool right = sb < 0;  // cur is the right child
        double4 pc;
        float4 plo, phi;
        bu_merge(right ? oc : cm, right ? cm : oc, right ? ol : lo, right ? lo : ol, right ? oh : hi, right ? hi : oh,
                 pc, plo, phi);
        s_cm[1][pslot] = pc;
        s_lo[1][pslot] = plo;
        s_hi[1][pslot] = phi;
        cm = pc;
        lo = plo;
        hi = phi;
        side = 1;
        slot = pslot;
        cur = par;
    }
    __syncthreads();  // one global reservation per block for its frontier nodes
    if (j == 0) s_fbase = s_nf ? atomicAdd(nfront, s_nf) : 0u;
    // the block's completed internal nodes (both children arrived) go to global
    // memory in one coalesced pass, not from inside the climb, so that the
    // block-scope fences there wait for shared-memory stores only; with them
    // their child records, from the children's data still in shared memory
    // (a completed node's children lie in the block: leaves B0..B1, internal
    // nodes n + B0..B1)
    if (k < n - 1 && s_cnt[j] == 2u) {
        node_cm[n + k] = s_cm[1][j];
        bmin[n + k] = s_lo[1][j];
        bmax[n + k] = s_hi[1][j];
        const int2 ch = child[n + k];
        const int sL = (int)(ch.x < n ? ch.x - B0 : ch.x - n - B0), sR = (int)(ch.y < n ? ch.y - B0 : ch.y - n - B0);
        const int tL = ch.x < n ? 0 : 1, tR = ch.y < n ? 0 : 1;
        put_child_record(crec + 4 * k, n, theta, ch.x, s_cm[tL][sL], s_lo[tL][sL], s_hi[tL][sL], ch.y, s_cm[tR][sR],
                         s_lo[tR][sR], s_hi[tR][sR]);
    }
    __syncthreads();
    if ((unsigned)j < s_nf) front[s_fbase + j] = s_front[j];
}

// Arrival at a node in the global phase: one atomic with acquire-release
// semantics at GPU scope. Its release half publishes this climb's node data
// (written before it) to the climb that arrives second; its acquire half
// makes the sibling's data, published by the first arrival's release, visible
// to the loads that follow. (ASTER_BU_FENCES=1: the equivalent form with a
// full fence on either side of a relaxed atomicAdd.)
#ifndef ASTER_BU_FENCES
#define ASTER_BU_FENCES 0
#endif
__device__ __forceinline__ unsigned int bu_arrive(unsigned int* counter) {
#if ASTER_BU_FENCES
    __threadfence();
    const unsigned int old = atomicAdd(counter, 1u);
    __threadfence();
    return old;
#else
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
    return old;
#endif
}

__global__ void __launch_bounds__(256) k_bottom_up_front(int64_t n, const int32_t* __restrict__ front,
                                                         const unsigned int* __restrict__ nfront,
                                                         const int32_t* __restrict__ parent,
                                                         const int32_t* __restrict__ sib,
                                                         uint32_t* __restrict__ counters, double4* __restrict__ node_cm,
                                                         float4* __restrict__ bmin, float4* __restrict__ bmax,
                                                         int* __restrict__ err) {
    const int64_t nf = *nfront;
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x) {
        int32_t cur = front[f];
        // the climb's own node data stays in registers; only the sibling's is loaded
        double4 cm = ld_cg(node_cm + cur);
        float4 lo = cur < n ? leaf_lo(cm) : ld_cg(bmin + cur), hi = cur < n ? leaf_hi(cm) : ld_cg(bmax + cur);
        int32_t par = parent[cur], sb = sib[cur];
        for (int level = 0; par >= 0; ++level) {
            if (level >= MAX_CLIMB) {
                atomicOr(err, ASTER_DEVERR_TREE);
                break;
            }
            // the next level's links load while this level synchronises
            const int32_t par_next = parent[par], sb_next = sib[par];
            if (bu_arrive(&counters[par - n]) == 0u) break;  // first arrival: the sibling finishes it
            const int32_t so = sb >= 0 ? sb : ~sb;
            const double4 oc = ld_cg(node_cm + so);
            const float4 ol = so < n ? leaf_lo(oc) : ld_cg(bmin + so), oh = so < n ? leaf_hi(oc) : ld_cg(bmax + so);
            const bool right = sb < 0;  // cur is the right child
            double4 pc;
            float4 plo, phi;
            bu_merge(right ? oc : cm, right ? cm : oc, right ? ol : lo, right ? lo : ol, right ? oh : hi,
                     right ? hi : oh, pc, plo, phi);
            node_cm[par] = pc;
            bmin[par] = plo;
            bmax[par] = phi;
            cm = pc;
            lo = plo;
            hi = phi;
            cur = par;
            par = par_next;
            sb = sb_next;
        }
    }
}

// Node velocities for the post-Newtonian walk, in NodesArray::unite form
// (src/solvers/barnes_hut.cpp:150): leaf k holds the velocity of sorted body k,
// an internal node the mass-weighted mean of its children,
// v = (v_R m_R + v_L m_L) / M, with M the node mass from the bottom-up pass
// (M <= 0: (v_R + v_L) / 2). One climb per leaf with the arrival counters of
// the internal nodes (zero on entry); the second arrival merges. Only the
// post-Newtonian walk needs it, so it is a pass of its own.
__global__ void __launch_bounds__(256) k_node_vel(int64_t n, const int32_t* __restrict__ parent,
                                                  const int32_t* __restrict__ sib, const int32_t* __restrict__ perm,
                                                  const double4* __restrict__ vel, const double4* __restrict__ node_cm,
                                                  uint32_t* __restrict__ counters, double4* __restrict__ node_v,
                                                  int* __restrict__ err) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double4 v = vel[perm[k]];
        v.w = 0.0;
        node_v[k] = v;
        int32_t cur = (int32_t)k;
        int32_t par = n >= 2 ? parent[cur] : -1, sb = n >= 2 ? sib[cur] : 0;
        for (int level = 0; par >= 0; ++level) {
            if (level >= MAX_CLIMB) {
                atomicOr(err, ASTER_DEVERR_TREE);
                break;
            }
            if (bu_arrive(&counters[par - n]) == 0u) break;  // first arrival: the sibling finishes it
            const int32_t so = sb >= 0 ? sb : ~sb;
            const double4 ov = ld_cg(node_v + so);
            const double mc = node_cm[cur].w, mo = node_cm[so].w, M = node_cm[par].w;
            const bool right = sb < 0;  // cur is the right child
            const double4 vR = right ? v : ov, vL = right ? ov : v;
            const double mR = right ? mc : mo, mL = right ? mo : mc;
            double4 pv;
            if (M > 0.0) {
                pv.x = __ddiv_rn(__dadd_rn(__dmul_rn(vR.x, mR), __dmul_rn(vL.x, mL)), M);
                pv.y = __ddiv_rn(__dadd_rn(__dmul_rn(vR.y, mR), __dmul_rn(vL.y, mL)), M);
                pv.z = __ddiv_rn(__dadd_rn(__dmul_rn(vR.z, mR), __dmul_rn(vL.z, mL)), M);
            } else {
                pv.x = __dmul_rn(0.5, __dadd_rn(vR.x, vL.x));
                pv.y = __dmul_rn(0.5, __dadd_rn(vR.y, vL.y));
                pv.z = __dmul_rn(0.5, __dadd_rn(vR.z, vL.z));
            }
            pv.w = 0.0;
            node_v[par] = pv;
            v = pv;
            cur = par;
            par = parent[cur];
            sb = sib[cur];
        }
    }
}

// Child records of the internal nodes completed by the global phase of the
// bottom-up merge (their arrival counters read 2; the block-local phase writes
// the records of the nodes it completes and leaves their counters at 0).
// Those nodes are sparse (~10% of the internal nodes at N = 2^20), so each block
// first compacts the ones in its span of REC_SPAN counters into shared memory
// and then gives them to consecutive threads: the latency-bound loads of the
// children's data run in full warps instead of one lane per warp.
constexpr int REC_SPAN = 2048;
__global__ void __launch_bounds__(256) k_front_records(int64_t n, double theta, const uint32_t* __restrict__ counters,
                                                       const int2* __restrict__ child,
                                                       const double4* __restrict__ node_cm,
                                                       const float4* __restrict__ bmin,
                                                       const float4* __restrict__ bmax, float4* __restrict__ crec) {
    __shared__ int32_t s_list[REC_SPAN];
    __shared__ unsigned int s_n;
    const int lane = threadIdx.x & 31;
    const int64_t m = n - 1;  // internal nodes 0 .. n - 2
    for (int64_t base = (int64_t)blockIdx.x * REC_SPAN; base < m; base += (int64_t)gridDim.x * REC_SPAN) {
        if (threadIdx.x == 0) s_n = 0u;
        __syncthreads();
        bool hit[REC_SPAN / 256];
#pragma unroll
        for (int r = 0; r < REC_SPAN / 256; ++r) {
            const int64_t i = base + r * 256 + threadIdx.x;
            hit[r] = i < m && counters[i] == 2u;
        }
#pragma unroll
        for (int r = 0; r < REC_SPAN / 256; ++r) {
            const uint32_t mask = __ballot_sync(0xffffffffu, hit[r]);
            unsigned int wb = 0u;
            if (lane == 0 && mask) wb = atomicAdd(&s_n, (unsigned int)__popc(mask));
            wb = __shfl_sync(0xffffffffu, wb, 0);
            if (hit[r]) s_list[wb + __popc(mask & ((1u << lane) - 1u))] = r * 256 + (int)threadIdx.x;
        }
        __syncthreads();
        const unsigned int cnt = s_n;
        for (unsigned int k = threadIdx.x; k < cnt; k += blockDim.x) {
            const int64_t i = base + s_list[k];
            const int2 ch = child[n + i];
            const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
            put_child_record(crec + 4 * i, n, theta, ch.x, node_cm[ch.x], ch.x < n ? z : bmin[ch.x],
                             ch.x < n ? z : bmax[ch.x], ch.y, node_cm[ch.y], ch.y < n ? z : bmin[ch.y],
                             ch.y < n ? z : bmax[ch.y]);
        }
        __syncthreads();  // s_n and s_list are reused by the next span
    }
}

// ----------------------------------------------------------------- walk
template <bool MIXED>
struct WalkShared {
    int stack[WALK_WARPS][WALK_STACK];
    // mixed list, two entries per slot so that each paired FP32 operand is an
    // aligned register pair: lpa = (x0, x1, y0, y1), lpb = (z0, z1, m0, m1),
    // positions relative to the group centre
    float4 lpa[WALK_WARPS][MIXED ? WALK_LIST_MIXED / 2 : 1];
    float4 lpb[WALK_WARPS][MIXED ? WALK_LIST_MIXED / 2 : 1];
    double4 lcm[WALK_WARPS][MIXED ? 1 : WALK_LIST_FP64];  // FP64 (com, mass)
};

// Post-Newtonian walk: each list entry also carries the node's velocity
// (vx, vy, vz, |v|^2), FP32 for the mixed walk and FP64 for the FP64 walk.
template <bool MIXED>
struct WalkSharedPn : WalkShared<MIXED> {
    // mixed: paired like lpa/lpb, lva = (vx0, vx1, vy0, vy1), lvb = (vz0, vz1, w0, w1), w = |v|^2
    float4 lva[WALK_WARPS][MIXED ? WALK_LIST_PN / 2 : 1];
    float4 lvb[WALK_WARPS][MIXED ? WALK_LIST_PN / 2 : 1];
    double4 lvd[WALK_WARPS][MIXED ? 1 : WALK_LIST_FP64];
};

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
__device__ __forceinline__ float warp_min_f(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max_f(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Two interactions at once with the paired FP32 instructions of sm_100
// (add/mul/fma .f32x2): list entries (A.x|A.y, A.z|A.w, B.x|B.y) positions,
// B.z|B.w masses; nb = -(body position) broadcast to both halves.
template <bool GUARD>
__device__ __forceinline__ void interact2_f32(const float4 A, const float4 B, const float2 nbx, const float2 nby,
                                              const float2 nbz, const float2 eps2, float2& ax, float2& ay, float2& az) {
    const float2 dx = __fadd2_rn(make_float2(A.x, A.y), nbx);
    const float2 dy = __fadd2_rn(make_float2(A.z, A.w), nby);
    const float2 dz = __fadd2_rn(make_float2(B.x, B.y), nbz);
    float2 r2 = __ffma2_rn(dz, dz, eps2);
    r2 = __ffma2_rn(dy, dy, r2);
    r2 = __ffma2_rn(dx, dx, r2);
    float2 inv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    if (GUARD) {
        inv.x = r2.x > 0.f ? inv.x : 0.f;
        inv.y = r2.y > 0.f ? inv.y : 0.f;
    }
    const float2 inv2 = __fmul2_rn(inv, inv);
    const float2 sN = __fmul2_rn(__fmul2_rn(make_float2(B.z, B.w), inv), inv2);
    ax = __ffma2_rn(dx, sN, ax);
    ay = __ffma2_rn(dy, sN, ay);
    az = __ffma2_rn(dz, sN, az);
}

template <bool GUARD>
__device__ __forceinline__ void interact_f64(const double4 e, const double4 b, double eps2, double& ax, double& ay,
                                             double& az) {
    const double dx = e.x - b.x, dy = e.y - b.y, dz = e.z - b.z;
    const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
    double inv = rsqrt(r2);
    if (GUARD) inv = r2 > 0.0 ? inv : 0.0;
    const double s = e.w * inv * inv * inv;
    ax = fma(dx, s, ax);
    ay = fma(dy, s, ay);
    az = fma(dz, s, az);
}

// One entry with a post-Newtonian force law, FP64: the Newtonian term as
// interact_f64 forms it plus the terms pk selects (pn.cuh), all divided by G.
// Entry e (position, mass; velocity ev) acts on the body b (velocity vi).
template <int PNL, bool GUARD>
__device__ __forceinline__ void interact_pn_f64(const double4 e, const double4 ev, const double4 b, const double4 vi,
                                                double eps2, double G, const PnK<double>& k, double& ax, double& ay,
                                                double& az) {
    const double dx = e.x - b.x, dy = e.y - b.y, dz = e.z - b.z;
    const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
    double inv = rsqrt(r2);
    if (GUARD) inv = r2 > 0.0 ? inv : 0.0;
    const double s = e.w * inv * inv * inv;
    ax = fma(dx, s, ax); ay = fma(dy, s, ay); az = fma(dz, s, az);
    PnPair<double> w;
    w.nx = -dx * inv; w.ny = -dy * inv; w.nz = -dz * inv;
    w.dvx = vi.x - ev.x; w.dvy = vi.y - ev.y; w.dvz = vi.z - ev.z;
    w.inv = inv; w.inv2 = inv * inv; w.mi = b.w; w.mj = e.w; w.vi2 = vi.w; w.vj2 = ev.w;
    w.v12 = vi.x * ev.x + vi.y * ev.y + vi.z * ev.z;
    w.nv1 = w.nx * vi.x + w.ny * vi.y + w.nz * vi.z;
    w.nv2 = w.nx * ev.x + w.ny * ev.y + w.nz * ev.z;
    w.G = G;
    pn_terms<PNL>(k, w, ax, ay, az, ax, ay, az);
}

// Two entries at once with the paired FP32 instructions, force law Newton +
// 1PN: the Newtonian term into (ax, ay, az) as interact2_f32 forms it and the
// 1PN sum of newton_pn1_x2 into (px, py, pz) (the 1PN term divided by G is
// -c^-2 times it). A, B: entry positions and masses as in interact2_f32;
// VA = (vx0, vx1, vy0, vy1), VB = (vz0, vz1, |v0|^2, |v1|^2) the entries'
// velocities. Per body, broadcast to both halves: nb = -(position),
// vi = velocity, vi4 = 4 vi, nvi2 = -|vi|^2, mi5G = 5 G m_i; G4 = 4 G.
template <bool GUARD>
__device__ __forceinline__ void interact2_pn1_f32(const float4 A, const float4 B, const float4 VA, const float4 VB,
                                                  const float2 nbx, const float2 nby, const float2 nbz,
                                                  const float2 vix, const float2 viy, const float2 viz,
                                                  const float2 vi4x, const float2 vi4y, const float2 vi4z,
                                                  const float2 nvi2, const float2 mi5G, const float2 eps2,
                                                  const float2 G4, float2& ax, float2& ay, float2& az, float2& px,
                                                  float2& py, float2& pz) {
    const float2 dx = __fadd2_rn(make_float2(A.x, A.y), nbx);  // entry - body
    const float2 dy = __fadd2_rn(make_float2(A.z, A.w), nby);
    const float2 dz = __fadd2_rn(make_float2(B.x, B.y), nbz);
    newton_pn1_x2<GUARD>(dx, dy, dz, make_float2(B.z, B.w), make_float2(VA.x, VA.y), make_float2(VA.z, VA.w),
                         make_float2(VB.x, VB.y), make_float2(VB.z, VB.w), vix, viy, viz, vi4x, vi4y, vi4z, nvi2,
                         mi5G, eps2, G4, ax, ay, az, px, py, pz);
}

__device__ __forceinline__ float4 vel_f4(const double4 v) {
    return make_float4((float)v.x, (float)v.y, (float)v.z, (float)(v.x * v.x + v.y * v.y + v.z * v.z));
}
__device__ __forceinline__ double4 vel_d4(const double4 v) {
    return make_double4(v.x, v.y, v.z, v.x * v.x + v.y * v.y + v.z * v.z);
}

__device__ __forceinline__ float max3_f32(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Opening test of both children of a node for the whole group, FP32
// round-to-nearest without FMA (the CPU restatement reproduces it bit for
// bit), the two children in the halves of paired FP32 operations: the squared
// distance from a child's FP32 centre of mass to the group box is
// sum over axes of max(lo - c, c - hi, 0)^2; the child is accepted when it
// exceeds the child's r_crit^2. lo - c is formed as fma(c, -1, lo), which is
// the correctly rounded difference; nhi = -hi.
__device__ __forceinline__ float2 box_dist2_pair(const float2 cx, const float2 cy, const float2 cz, const float2 lox,
                                                 const float2 loy, const float2 loz, const float2 nhix,
                                                 const float2 nhiy, const float2 nhiz) {
    const float2 m1 = make_float2(-1.f, -1.f);
    const float2 ux = __ffma2_rn(cx, m1, lox), wx = __fadd2_rn(cx, nhix);
    const float2 uy = __ffma2_rn(cy, m1, loy), wy = __fadd2_rn(cy, nhiy);
    const float2 uz = __ffma2_rn(cz, m1, loz), wz = __fadd2_rn(cz, nhiz);
    const float2 tx = make_float2(max3_f32(ux.x, wx.x, 0.f), max3_f32(ux.y, wx.y, 0.f));
    const float2 ty = make_float2(max3_f32(uy.x, wy.x, 0.f), max3_f32(uy.y, wy.y, 0.f));
    const float2 tz = make_float2(max3_f32(uz.x, wz.x, 0.f), max3_f32(uz.y, wz.y, 0.f));
    return __fadd2_rn(__fadd2_rn(__fmul2_rn(tx, tx), __fmul2_rn(ty, ty)), __fmul2_rn(tz, tz));
}

// Persistent walk: each warp takes groups from a global work counter until
// none are left. Per group: lane l holds sorted leaf l of the group; the r
// leaves beyond 32 are each shared by 32/r (rounded down to a power of two)
// lanes that split the interaction list between them, so groups of 33..64
// bodies keep every lane busy. The warp pops up to 32 opened internal nodes
// per round from its shared stack; each lane loads the contiguous record of
// its node's two children (centres of mass, masses, opening radii: one
// 64-byte load, issued together with the child indices) and tests both:
// leaves and accepted cells go to the shared interaction list, opened
// internal children to the stack. The list is evaluated 32 entries at a
// time by every lane.
// Mixed precision: list entries and bodies are stored relative to the group
// centre cg (FP32 of hi - cg plus the double-single low part), so an
// interaction needs one subtraction per axis; the group is compact, so the
// relative coordinates keep FP32 precision of the separation.
// PNL > 0: the post-Newtonian walk (the terms pk selects, with the nodes'
// velocities node_v); PNL == 0 is the Newtonian kernel.
template <bool MIXED, bool GUARD, bool KICK, int PNL = 0>
__global__ void __launch_bounds__(WALK_WARPS * 32, PNL ? 4 : (MIXED ? ASTER_WALK_MINBLOCKS : 6)) k_walk(
    int64_t n, const int2* __restrict__ groups, const unsigned int* __restrict__ ngroups_p,
    unsigned int* __restrict__ work,
    const float4* __restrict__ crec, const double4* __restrict__ node_cm, const int2* __restrict__ child,
    const int32_t* __restrict__ perm, double G, double eps2, double half_dt, double4* __restrict__ acc,
    double4* __restrict__ vel, int* __restrict__ err, int* __restrict__ stack_hw, int stack_limit,
    int32_t* __restrict__ body_counts, unsigned long long* __restrict__ inter_count,
    const double4* __restrict__ node_v, PnK<double> pk, double4* __restrict__ pm_next, double dt_next,
    unsigned long long* __restrict__ box_next) {
    using Shared = typename std::conditional<PNL != 0, WalkSharedPn<MIXED>, WalkShared<MIXED>>::type;
    __shared__ Shared sm;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    // ngroups_p[0] groups of more than GROUP_SMALL bodies at groups[0..), then
    // ngroups_p[3] smaller ones at groups[n - 1], groups[n - 2], ...
    const unsigned int nbig = ngroups_p[0], ngroups = nbig + ngroups_p[3];
    int* stack = sm.stack[warp];
    int hw = 1;
    unsigned long long wtotal = 0;
    double bmax = 0.0;  // fused next drift: max |coordinate| of the drifted bodies

    for (;;) {
        unsigned int g = 0;
        if (lane == 0) g = atomicAdd(work, 1u);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= ngroups) break;
        const int2 gr = groups[g < nbig ? (int64_t)g : n - 1 - (int64_t)(g - nbig)];
        // Bodies 0..31 of the group: one per lane (primary). Bodies 32.. (r of
        // them, "secondary"): each shared by lps lanes that split the list.
        const int r = gr.y > 32 ? gr.y - 32 : 0;
        const bool two = r > 0;  // warp-uniform
        int lps = 32;
        while (lps > 1 && lps * r > 32) lps >>= 1;
        const int sb = lane / lps, sub = lane & (lps - 1);
        const bool v0 = lane < gr.y, v1 = two && sb < r;
        const int64_t k0 = (int64_t)gr.x + (v0 ? lane : 0);
        const int64_t k1 = (int64_t)gr.x + (v1 ? 32 + sb : 0);
        // the bodies' input indices, for the results (loaded now, used at the end)
        const int32_t pb0 = perm[k0], pb1 = perm[k1];

        float4 h0, l0, h1, l1;  // the bodies' traversal data, from their leaves
        leaf_trav(node_cm[k0], h0, l0);
        if (two) {
            leaf_trav(node_cm[k1], h1, l1);
        } else {
            h1 = h0;
            l1 = l0;
        }
        const float glox = warp_min_f(fminf(v0 ? h0.x : INFINITY, v1 ? h1.x : INFINITY));
        const float gloy = warp_min_f(fminf(v0 ? h0.y : INFINITY, v1 ? h1.y : INFINITY));
        const float gloz = warp_min_f(fminf(v0 ? h0.z : INFINITY, v1 ? h1.z : INFINITY));
        const float ghix = warp_max_f(fmaxf(v0 ? h0.x : -INFINITY, v1 ? h1.x : -INFINITY));
        const float ghiy = warp_max_f(fmaxf(v0 ? h0.y : -INFINITY, v1 ? h1.y : -INFINITY));
        const float ghiz = warp_max_f(fmaxf(v0 ? h0.z : -INFINITY, v1 ? h1.z : -INFINITY));
        const float cgx = 0.5f * (glox + ghix), cgy = 0.5f * (gloy + ghiy), cgz = 0.5f * (gloz + ghiz);
        const float3 b0 = make_float3((h0.x - cgx) + l0.x, (h0.y - cgy) + l0.y, (h0.z - cgz) + l0.z);
        const float3 b1 = make_float3((h1.x - cgx) + l1.x, (h1.y - cgy) + l1.y, (h1.z - cgz) + l1.z);
        const float2 nb0x = make_float2(-b0.x, -b0.x), nb0y = make_float2(-b0.y, -b0.y), nb0z = make_float2(-b0.z, -b0.z);
        const float2 nb1x = make_float2(-b1.x, -b1.x), nb1y = make_float2(-b1.y, -b1.y), nb1z = make_float2(-b1.z, -b1.z);
        const float2 eps2f2 = make_float2((float)eps2, (float)eps2);
        double4 c0 = make_double4(0, 0, 0, 0), c1 = c0;
        if (!MIXED) {
            c0 = node_cm[k0];
            c1 = two ? node_cm[k1] : c0;
        }
        // post-Newtonian walk: the bodies' own velocities and the running
        // 1PN (p) and 2PN + 2.5PN (q) sums of the mixed walk
        float4 vf0 = make_float4(0.f, 0.f, 0.f, 0.f), vf1 = vf0;
        double4 vd0 = make_double4(0, 0, 0, 0), vd1 = vd0;
        float3 p0 = make_float3(0.f, 0.f, 0.f), q0 = p0, p1 = p0, q1 = p0;
        if constexpr (PNL > 0) {
            if (MIXED) {
                vf0 = vel_f4(node_v[k0]);
                vf1 = two ? vel_f4(node_v[k1]) : vf0;
            } else {
                vd0 = vel_d4(node_v[k0]);
                vd1 = two ? vel_d4(node_v[k1]) : vd0;
            }
        }

        CompSum sx0, sy0, sz0, sx1, sy1, sz1;
        double dx0 = 0, dy0 = 0, dz0 = 0, dx1 = 0, dy1 = 0, dz1 = 0;
        int top = 0, lc = 0;
        int total = 0;
        bool overflow = false;

        // store list entry `pos` (lane-private): mixed = group-relative position and mass
        auto put = [&](int pos, float x, float y, float z, float mass) {
            float* A = reinterpret_cast<float*>(&sm.lpa[warp][0]);
            float* B = reinterpret_cast<float*>(&sm.lpb[warp][0]);
            const int o = ((pos >> 1) << 2) | (pos & 1);
            A[o] = x;
            A[o + 2] = y;
            B[o] = z;
            B[o + 2] = mass;
        };

        // post-Newtonian walk: the velocity of list entry `pos`
        auto put_v = [&](int pos, const double4 v) {
            if constexpr (PNL > 0) {
                if (MIXED) {
                    const float4 f = vel_f4(v);
                    float* VA = reinterpret_cast<float*>(&sm.lva[warp][0]);
                    float* VB = reinterpret_cast<float*>(&sm.lvb[warp][0]);
                    const int o = ((pos >> 1) << 2) | (pos & 1);
                    VA[o] = f.x;
                    VA[o + 2] = f.y;
                    VB[o] = f.z;
                    VB[o + 2] = f.w;
                } else {
                    sm.lvd[warp][pos] = vel_d4(v);
                }
            }
        };

        auto evaluate = [&](int cnt) {
            if constexpr (PNL > 0) {
                if constexpr (MIXED && PNL == 1) {  // Newton + 1PN only: two entries per paired instruction
                    // an odd cnt has its last slot half zero-padded by the caller
                    const int np = (cnt + 1) >> 1;
                    const float Gf = (float)G, mc2 = -(float)pk.c2;
                    const float2 G4 = make_float2(4.f * Gf, 4.f * Gf);
                    auto body = [&](const float2 nbx, const float2 nby, const float2 nbz, const float4 vf, float mi,
                                    int q0i, int step, CompSum& sx, CompSum& sy, CompSum& sz, float3& p) {
                        const float2 vix = make_float2(vf.x, vf.x), viy = make_float2(vf.y, vf.y),
                                     viz = make_float2(vf.z, vf.z), nvi2 = make_float2(-vf.w, -vf.w),
                                     vi4x = make_float2(4.f * vf.x, 4.f * vf.x),
                                     vi4y = make_float2(4.f * vf.y, 4.f * vf.y),
                                     vi4z = make_float2(4.f * vf.z, 4.f * vf.z),
                                     mi5G = make_float2(5.f * Gf * mi, 5.f * Gf * mi);
                        float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax, px = ax, py = ax, pz = ax;
#pragma unroll 2
                        for (int q = q0i; q < np; q += step)
                            interact2_pn1_f32<GUARD>(sm.lpa[warp][q], sm.lpb[warp][q], sm.lva[warp][q],
                                                     sm.lvb[warp][q], nbx, nby, nbz, vix, viy, viz, vi4x, vi4y,
                                                     vi4z, nvi2, mi5G, eps2f2, G4, ax, ay, az, px, py, pz);
                        sx.add(ax.x + ax.y); sy.add(ay.x + ay.y); sz.add(az.x + az.y);
                        p.x = fmaf(mc2, px.x + px.y, p.x);
                        p.y = fmaf(mc2, py.x + py.y, p.y);
                        p.z = fmaf(mc2, pz.x + pz.y, p.z);
                    };
                    body(nb0x, nb0y, nb0z, vf0, h0.w, 0, 1, sx0, sy0, sz0, p0);
                    if (two) body(nb1x, nb1y, nb1z, vf1, h1.w, sub, lps, sx1, sy1, sz1, p1);
                } else if (MIXED) {  // any of the PN terms by flags: two entries per paired instruction as well
                    const int np = (cnt + 1) >> 1;  // an odd cnt: last slot half zero-padded by the caller
                    const float Gf = (float)G, mc2 = -(float)pk.c2, mc4 = -(float)pk.c4;
                    const float2 G4 = make_float2(4.f * Gf, 4.f * Gf), G2 = make_float2(Gf, Gf);
                    const float nkf = -0.8f * (float)pk.ic;
                    const float2 nk = make_float2(nkf, nkf);
                    auto body = [&](const float2 nbx, const float2 nby, const float2 nbz, const float4 vf, float mi,
                                    int q0i, int step, CompSum& sx, CompSum& sy, CompSum& sz, float3& p, float3& qq) {
                        const float2 vix = make_float2(vf.x, vf.x), viy = make_float2(vf.y, vf.y),
                                     viz = make_float2(vf.z, vf.z), nvi2 = make_float2(-vf.w, -vf.w),
                                     vi2 = make_float2(vf.w, vf.w),
                                     vi4x = make_float2(4.f * vf.x, 4.f * vf.x),
                                     vi4y = make_float2(4.f * vf.y, 4.f * vf.y),
                                     vi4z = make_float2(4.f * vf.z, 4.f * vf.z),
                                     mi5G = make_float2(5.f * Gf * mi, 5.f * Gf * mi),
                                     Gmi = make_float2(Gf * mi, Gf * mi);
                        float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax, px = ax, py = ax, pz = ax, qx = ax,
                               qy = ax, qz = ax;
                        for (int q = q0i; q < np; q += step) {
                            const float4 A = sm.lpa[warp][q], B = sm.lpb[warp][q], VA = sm.lva[warp][q],
                                         VB = sm.lvb[warp][q];
                            const float2 dx = __fadd2_rn(make_float2(A.x, A.y), nbx);  // entry - body
                            const float2 dy = __fadd2_rn(make_float2(A.z, A.w), nby);
                            const float2 dz = __fadd2_rn(make_float2(B.x, B.y), nbz);
                            newton_pn_all_x2<GUARD>(dx, dy, dz, make_float2(B.z, B.w), make_float2(VA.x, VA.y),
                                                    make_float2(VA.z, VA.w), make_float2(VB.x, VB.y),
                                                    make_float2(VB.z, VB.w), vix, viy, viz, vi4x, vi4y, vi4z, nvi2,
                                                    vi2, mi5G, Gmi, eps2f2, G4, G2, nk, pk.f, ax, ay, az, px, py, pz,
                                                    qx, qy, qz);
                        }
                        sx.add(ax.x + ax.y); sy.add(ay.x + ay.y); sz.add(az.x + az.y);
                        p.x = fmaf(mc2, px.x + px.y, p.x);
                        p.y = fmaf(mc2, py.x + py.y, p.y);
                        p.z = fmaf(mc2, pz.x + pz.y, p.z);
                        qq.x = fmaf(mc4, qx.x + qx.y, qq.x);
                        qq.y = fmaf(mc4, qy.x + qy.y, qq.y);
                        qq.z = fmaf(mc4, qz.x + qz.y, qq.z);
                    };
                    body(nb0x, nb0y, nb0z, vf0, h0.w, 0, 1, sx0, sy0, sz0, p0, q0);
                    if (two) body(nb1x, nb1y, nb1z, vf1, h1.w, sub, lps, sx1, sy1, sz1, p1, q1);
                } else {
                    for (int e = 0; e < cnt; ++e)
                        interact_pn_f64<PNL, GUARD>(sm.lcm[warp][e], sm.lvd[warp][e], c0, vd0, eps2, G, pk, dx0, dy0,
                                                    dz0);
                    if (two)
                        for (int e = sub; e < cnt; e += lps)
                            interact_pn_f64<PNL, GUARD>(sm.lcm[warp][e], sm.lvd[warp][e], c1, vd1, eps2, G, pk, dx1,
                                                        dy1, dz1);
                }
                total += cnt;
                return;
            }
            if (MIXED) {
                // an odd cnt has its last slot half zero-padded by the caller
                const int np = (cnt + 1) >> 1;
                float2 ax0 = make_float2(0.f, 0.f), ay0 = ax0, az0 = ax0;
                if (two && lps == 1) {  // 49..64 bodies: both bodies of a lane share each list load
                    float2 ax1 = make_float2(0.f, 0.f), ay1 = ax1, az1 = ax1;
#pragma unroll 4
                    for (int q = 0; q < np; ++q) {
                        const float4 A = sm.lpa[warp][q], B = sm.lpb[warp][q];
                        interact2_f32<GUARD>(A, B, nb0x, nb0y, nb0z, eps2f2, ax0, ay0, az0);
                        interact2_f32<GUARD>(A, B, nb1x, nb1y, nb1z, eps2f2, ax1, ay1, az1);
                    }
                    sx0.add(ax0.x + ax0.y); sy0.add(ay0.x + ay0.y); sz0.add(az0.x + az0.y);
                    sx1.add(ax1.x + ax1.y); sy1.add(ay1.x + ay1.y); sz1.add(az1.x + az1.y);
                    total += cnt;
                    return;
                }
#pragma unroll WALK_UNROLL
                for (int q = 0; q < np; ++q)
                    interact2_f32<GUARD>(sm.lpa[warp][q], sm.lpb[warp][q], nb0x, nb0y, nb0z, eps2f2, ax0, ay0, az0);
                sx0.add(ax0.x + ax0.y); sy0.add(ay0.x + ay0.y); sz0.add(az0.x + az0.y);
                if (two) {
                    float2 ax1 = make_float2(0.f, 0.f), ay1 = ax1, az1 = ax1;
#pragma unroll 4
                    for (int q = sub; q < np; q += lps)
                        interact2_f32<GUARD>(sm.lpa[warp][q], sm.lpb[warp][q], nb1x, nb1y, nb1z, eps2f2, ax1, ay1, az1);
                    sx1.add(ax1.x + ax1.y); sy1.add(ay1.x + ay1.y); sz1.add(az1.x + az1.y);
                }
            } else {
#pragma unroll 4
                for (int e = 0; e < cnt; ++e) interact_f64<GUARD>(sm.lcm[warp][e], c0, eps2, dx0, dy0, dz0);
                if (two) {
#pragma unroll 4
                    for (int e = sub; e < cnt; e += lps) interact_f64<GUARD>(sm.lcm[warp][e], c1, eps2, dx1, dy1, dz1);
                }
            }
            total += cnt;
        };

        const int nI = (int)n;  // node ids are int32: leaves < nI <= internal nodes
        if (n >= 2) {
            if (lane == 0) stack[0] = nI;  // the root is internal: start by opening it
            top = 1;
        } else {
            if (lane == 0) {  // a single body: its own leaf
                if (MIXED) {
                    float4 h, l;
                    leaf_trav(node_cm[0], h, l);
                    put(0, (h.x - cgx) + l.x, (h.y - cgy) + l.y, (h.z - cgz) + l.z, h.w);
                } else {
                    sm.lcm[warp][0] = node_cm[0];
                }
                put_v(0, PNL > 0 ? node_v[0] : make_double4(0, 0, 0, 0));
            }
            lc = 1;
        }
        __syncwarp();
        const float2 lox2 = make_float2(glox, glox), loy2 = make_float2(gloy, gloy), loz2 = make_float2(gloz, gloz);
        const float2 nhix2 = make_float2(-ghix, -ghix), nhiy2 = make_float2(-ghiy, -ghiy),
                     nhiz2 = make_float2(-ghiz, -ghiz);
        const float2 ncgx2 = make_float2(-cgx, -cgx), ncgy2 = make_float2(-cgy, -cgy), ncgz2 = make_float2(-cgz, -cgz);

        while (top > 0) {
            const int cnt = top < 32 ? top : 32;
            const bool act = lane < cnt;
            // inactive lanes read the root's record (valid memory) and are masked off
            int v = nI;
            if (act) v = stack[top - 1 - lane];
            __syncwarp();
            top -= cnt;
            const float4* rec = crec + 4 * (int64_t)(v - nI);
            const float4 r0 = rec[0], r1 = rec[1], r2 = rec[2], r3 = rec[3];
            const int2 ch = child[v];
            const float2 cx = make_float2(r0.x, r0.y), cy = make_float2(r0.z, r0.w), cz = make_float2(r1.x, r1.y);
            const float2 d2 = box_dist2_pair(cx, cy, cz, lox2, loy2, loz2, nhix2, nhiy2, nhiz2);
            const bool fL = ch.x < nI || d2.x > r3.z, fR = ch.y < nI || d2.y > r3.w;  // leaf or far enough
            const bool aL = act && fL, aR = act && fR, oL = act && !fL, oR = act && !fR;
            const uint32_t mAL = __ballot_sync(0xffffffffu, aL), mAR = __ballot_sync(0xffffffffu, aR);
            const uint32_t mOL = __ballot_sync(0xffffffffu, oL), mOR = __ballot_sync(0xffffffffu, oR);
            const int npush = __popc(mOL) + __popc(mOR);
            if (top + npush > stack_limit) {
                overflow = true;
                break;
            }
            {
                const int pos = top + __popc(mOL & lt) + __popc(mOR & lt);
                if (oL) stack[pos] = ch.x;
                if (oR) stack[pos + (oL ? 1 : 0)] = ch.y;
            }
            top += npush;
            hw = top > hw ? top : hw;
            {
                const int pos = lc + __popc(mAL & lt) + __popc(mAR & lt);
                if (MIXED) {
                    // both children's group-relative positions: (c - cg) + remainder
                    const float2 ex = __fadd2_rn(__fadd2_rn(cx, ncgx2), make_float2(r2.x, r2.y));
                    const float2 ey = __fadd2_rn(__fadd2_rn(cy, ncgy2), make_float2(r2.z, r2.w));
                    const float2 ez = __fadd2_rn(__fadd2_rn(cz, ncgz2), make_float2(r3.x, r3.y));
                    if (aL) put(pos, ex.x, ey.x, ez.x, r1.z);
                    if (aR) put(pos + (aL ? 1 : 0), ex.y, ey.y, ez.y, r1.w);
                } else {
                    if (aL) sm.lcm[warp][pos] = node_cm[ch.x];
                    if (aR) sm.lcm[warp][pos + (aL ? 1 : 0)] = node_cm[ch.y];
                }
                if constexpr (PNL > 0) {
                    if (aL) put_v(pos, node_v[ch.x]);
                    if (aR) put_v(pos + (aL ? 1 : 0), node_v[ch.y]);
                }
            }
            lc += __popc(mAL) + __popc(mAR);
            __syncwarp();
            constexpr int FL = MIXED ? (PNL ? WALK_FLUSH_PN : WALK_FLUSH_MIXED) : WALK_FLUSH_FP64;
            while (lc >= FL) {
                evaluate(FL);
                __syncwarp();
                const int rest = lc - FL;  // < 64
                if (MIXED) {  // whole slots (FL is even), at most 32; read all, then write
                    const int ns = (rest + 1) >> 1;
                    float4 a = make_float4(0, 0, 0, 0), b = a;
                    if (lane < ns) { a = sm.lpa[warp][FL / 2 + lane]; b = sm.lpb[warp][FL / 2 + lane]; }
                    __syncwarp();
                    if (lane < ns) { sm.lpa[warp][lane] = a; sm.lpb[warp][lane] = b; }
                } else {
                    const bool m0 = lane < rest, m1 = lane + 32 < rest;
                    double4 x0 = make_double4(0, 0, 0, 0), x1 = x0;
                    if (m0) x0 = sm.lcm[warp][32 + lane];
                    if (m1) x1 = sm.lcm[warp][64 + lane];
                    __syncwarp();
                    if (m0) sm.lcm[warp][lane] = x0;
                    if (m1) sm.lcm[warp][32 + lane] = x1;
                }
                if constexpr (PNL > 0) {  // the entries' velocities: [FL, FL + rest) -> [0, rest), rest < 64
                    const bool m0 = lane < rest, m1 = lane + 32 < rest;
                    if (MIXED) {  // whole slots, as for the positions
                        const int ns = (rest + 1) >> 1;
                        float4 a = make_float4(0, 0, 0, 0), b = a;
                        if (lane < ns) { a = sm.lva[warp][FL / 2 + lane]; b = sm.lvb[warp][FL / 2 + lane]; }
                        __syncwarp();
                        if (lane < ns) { sm.lva[warp][lane] = a; sm.lvb[warp][lane] = b; }
                    } else {
                        double4 x0 = make_double4(0, 0, 0, 0), x1 = x0;
                        if (m0) x0 = sm.lvd[warp][FL + lane];
                        if (m1) x1 = sm.lvd[warp][FL + 32 + lane];
                        __syncwarp();
                        if (m0) sm.lvd[warp][lane] = x0;
                        if (m1) sm.lvd[warp][32 + lane] = x1;
                    }
                }
                lc = rest;
                __syncwarp();
            }
        }
        if (overflow) {
            if (lane == 0) atomicOr(err, ASTER_DEVERR_STACK);
            break;
        }
        if (MIXED && (lc & 1) && lane == 0) {  // zero mass, zero offset: contributes nothing
            float* A = reinterpret_cast<float*>(&sm.lpa[warp][0]);
            float* B = reinterpret_cast<float*>(&sm.lpb[warp][0]);
            const int q = lc >> 1;
            A[4 * q + 1] = 0.f; A[4 * q + 3] = 0.f; B[4 * q + 1] = 0.f; B[4 * q + 3] = 0.f;
            if constexpr (PNL > 0) {  // and zero velocity, so the 1PN term is 0 * finite
                float* VA = reinterpret_cast<float*>(&sm.lva[warp][0]);
                float* VB = reinterpret_cast<float*>(&sm.lvb[warp][0]);
                VA[4 * q + 1] = 0.f; VA[4 * q + 3] = 0.f; VB[4 * q + 1] = 0.f; VB[4 * q + 3] = 0.f;
            }
        }
        __syncwarp();
        if (KICK) {  // the closing kick's operands into L1 while the last list is evaluated
            prefetch_l1(vel + pb0);
            if (pm_next) prefetch_l1(pm_next + pb0);
            if (v1 && sub == 0) {
                prefetch_l1(vel + pb1);
                if (pm_next) prefetch_l1(pm_next + pb1);
            }
        }
        if (lc > 0) evaluate(lc);
        __syncwarp();
        wtotal += (unsigned long long)total * (unsigned long long)gr.y;
        // secondary bodies: add the lps partial sums (aligned lane groups)
        double s1x = MIXED ? sx1.value() : dx1, s1y = MIXED ? sy1.value() : dy1, s1z = MIXED ? sz1.value() : dz1;
        if constexpr (PNL > 0) {
            if (MIXED) {
                s1x += (double)p1.x + (double)q1.x;
                s1y += (double)p1.y + (double)q1.y;
                s1z += (double)p1.z + (double)q1.z;
            }
        }
        if (two) {
            for (int o = lps >> 1; o >= 1; o >>= 1) {
                s1x += __shfl_xor_sync(0xffffffffu, s1x, o);
                s1y += __shfl_xor_sync(0xffffffffu, s1y, o);
                s1z += __shfl_xor_sync(0xffffffffu, s1z, o);
            }
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const bool vq = q ? (v1 && sub == 0) : v0;
            if (!vq) continue;
            double ax, ay, az;
            if (q) {
                ax = G * s1x; ay = G * s1y; az = G * s1z;
            } else if (MIXED) {
                if constexpr (PNL > 0) {
                    ax = G * (sx0.value() + ((double)p0.x + (double)q0.x));
                    ay = G * (sy0.value() + ((double)p0.y + (double)q0.y));
                    az = G * (sz0.value() + ((double)p0.z + (double)q0.z));
                } else {
                    ax = G * sx0.value(); ay = G * sy0.value(); az = G * sz0.value();
                }
            } else {
                ax = G * dx0; ay = G * dy0; az = G * dz0;
            }
            const int32_t b = q ? pb1 : pb0;
            acc[b] = make_double4(ax, ay, az, 0.0);
            if (body_counts) body_counts[b] = total;
            if (KICK) {
                double4 vv = vel[b];
                vv.x += ax * half_dt; vv.y += ay * half_dt; vv.z += az * half_dt;
                if (pm_next) {
                    // the next step's opening kick and drift, the same operations
                    // in the same order as its kick-drift kernel would apply them
                    // (that kernel does not run then); other bodies' positions
                    // are read from the tree, never from pm
                    vv.x += ax * half_dt; vv.y += ay * half_dt; vv.z += az * half_dt;
                    double4 pp = pm_next[b];
                    pp.x += vv.x * dt_next; pp.y += vv.y * dt_next; pp.z += vv.z * dt_next;
                    pm_next[b] = pp;
                    bmax = fmax(bmax, fmax(fabs(pp.x), fmax(fabs(pp.y), fabs(pp.z))));
                }
                vel[b] = vv;
            }
        }
    }
    if (box_next) {
        for (int o = 16; o > 0; o >>= 1) bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
        // non-negative doubles order like their bit patterns
        if (lane == 0) atomicMax(box_next, (unsigned long long)__double_as_longlong(bmax));
    }
    if (lane == 0) {
        atomicMax(stack_hw, hw);
        atomicAdd(inter_count, wtotal);
    }
}

template <bool MIXED, bool GUARD, bool KICK, int PNL = 0>
int launch_walk(aster_ctx* c, const aster_params* p, int32_t* counts, bool fuse_next) {
    LbvhBufs& t = c->tree;
    auto kern = k_walk<MIXED, GUARD, KICK, PNL>;
    int per_sm = 0;
    ASTER_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WALK_WARPS * 32, 0));
    if (per_sm < 1) per_sm = 1;
    int64_t blocks = (int64_t)c->sm_count * per_sm;
    const int64_t need = (c->n + WALK_WARPS - 1) / WALK_WARPS;  // groups <= n
    if (blocks > need) blocks = need;
    unsigned int* gcount = red_groups(c);
    kern<<<(unsigned)blocks, WALK_WARPS * 32, 0, c->stream>>>(
        c->n, t.groups.as<int2>(), gcount, gcount + 1,
        t.crec.as<float4>(), t.node_cm.as<double4>(), t.child.as<int2>(), t.perm.as<int32_t>(), p->G, p->eps2, 0.5 * p->dt,
        c->acc.as<double4>(), c->vel.as<double4>(), c->err_dev, c->stack_hw_dev, c->walk_stack_limit, counts,
        red_inter(c), PNL > 0 ? t.node_v.as<double4>() : nullptr, make_pn(p),
        KICK && fuse_next ? c->pm.as<double4>() : nullptr, p->dt, KICK && fuse_next ? red_box(c) : nullptr);
    ASTER_CUDA(cudaGetLastError());
    return ASTER_OK;
}

template <class KeyT>
int run_sort(aster_ctx* c, int bits) {
    LbvhBufs& t = c->tree;
    const int64_t n = c->n;
    const int nblocks = (int)((n + SORT_TILE - 1) / SORT_TILE);
    const int passes = (bits + 7) / 8;  // 30 -> 4, 63 -> 8 (even: result lands in sorted_codes)
    uint32_t* hist = t.hist.as<uint32_t>();
    uint32_t* dtot = t.digit_off.as<uint32_t>();
    const KeyT* kin = t.codes.as<KeyT>();
    const int32_t* vin = nullptr;
    for (int ps = 0; ps < passes; ++ps) {
        KeyT* kout = (ps & 1) ? t.sorted_codes.as<KeyT>() : t.codes_alt.as<KeyT>();
        int32_t* vout = (ps & 1) ? t.perm.as<int32_t>() : t.perm_alt.as<int32_t>();
        const int shift = 8 * ps;
        k_sort_hist<KeyT><<<nblocks, SORT_THREADS, 0, c->stream>>>(n, kin, shift, nblocks, hist);
        k_scan_digits<<<RADIX, 1024, 0, c->stream>>>(hist, nblocks, dtot);
        if (ps == 0)
            k_sort_scatter<KeyT, true><<<nblocks, SORT_THREADS, 0, c->stream>>>(n, kin, nullptr, kout, vout, shift,
                                                                             nblocks, hist, dtot);
        else
            k_sort_scatter<KeyT, false><<<nblocks, SORT_THREADS, 0, c->stream>>>(n, kin, vin, kout, vout, shift,
                                                                              nblocks, hist, dtot);
        ASTER_CUDA(cudaGetLastError());
        c->stats.kernels += 3;
        kin = kout;
        vin = vout;
    }
    return ASTER_OK;
}

int launch_bottom_up(aster_ctx* c, int64_t n, double theta) {
    LbvhBufs& t = c->tree;
    unsigned int* nfront = red_groups(c) + 2;  // zeroed at the start of the build
    const int64_t blocks = (n + BU_LEAVES - 1) / BU_LEAVES;
    k_bottom_up_local<<<(unsigned)blocks, BU_LEAVES, 0, c->stream>>>(
        n, t.parent.as<int32_t>(), t.sib.as<int32_t>(), t.rlo.as<int32_t>(), t.rhi.as<int32_t>(),
        t.node_cm.as<double4>(), t.bmin.as<float4>(), t.bmax.as<float4>(), t.front.as<int32_t>(), nfront, c->err_dev,
        theta, t.child.as<int2>(), t.crec.as<float4>());
    ASTER_CUDA(cudaGetLastError());
    const int64_t fb = std::min<int64_t>(blocks, (int64_t)c->sm_count * 8);
    k_bottom_up_front<<<(unsigned)fb, 256, 0, c->stream>>>(n, t.front.as<int32_t>(), nfront, t.parent.as<int32_t>(),
                                                           t.sib.as<int32_t>(), t.counters.as<uint32_t>(),
                                                           t.node_cm.as<double4>(), t.bmin.as<float4>(),
                                                           t.bmax.as<float4>(), c->err_dev);
    ASTER_CUDA(cudaGetLastError());
    c->stats.kernels += 2;
    return ASTER_OK;
}

template <class KeyT>
int run_build(aster_ctx* c, const aster_params* p) {
    LbvhBufs& t = c->tree;
    const int64_t n = c->n;
    const int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)c->sm_count * 16);
    const unsigned long long* box = red_box(c);
    const int mode = p->compat_mode ? 2 : (p->morton_bits == 63 ? 1 : 0);
    if (mode == 0) k_morton<KeyT, 0><<<grid, 256, 0, c->stream>>>(n, c->pm.as<double4>(), box, t.codes.as<KeyT>());
    else if (mode == 1) k_morton<KeyT, 1><<<grid, 256, 0, c->stream>>>(n, c->pm.as<double4>(), box, t.codes.as<KeyT>());
    else k_morton<KeyT, 2><<<grid, 256, 0, c->stream>>>(n, c->pm.as<double4>(), box, t.codes.as<KeyT>());
    ASTER_CUDA(cudaGetLastError());
    c->stats.kernels += 1;
    ASTER_TRY(run_sort<KeyT>(c, p->morton_bits == 63 ? 64 : 32));
    if (p->compat_mode) {
        // OpenCL order is descending by (code, index): reverse the ascending sort
        k_reverse<KeyT><<<grid, 256, 0, c->stream>>>(n, t.sorted_codes.as<KeyT>(), t.perm.as<int32_t>(),
                                                     t.codes_alt.as<KeyT>(), t.perm_alt.as<int32_t>());
        ASTER_CUDA(cudaMemcpyAsync(t.sorted_codes.ptr, t.codes_alt.ptr, (size_t)n * sizeof(KeyT),
                                   cudaMemcpyDeviceToDevice, c->stream));
        ASTER_CUDA(cudaMemcpyAsync(t.perm.ptr, t.perm_alt.ptr, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                   c->stream));
        c->stats.kernels += 1;
    }
    unsigned int* gcount = red_groups(c);  // [0] large groups, [1] walk work counter, [2] bottom-up frontier,
                                           // [3] small groups
    ASTER_CUDA(cudaMemsetAsync(gcount, 0, 4 * sizeof(unsigned int), c->stream));
    ASTER_TRY(aster_apply_pending_mass(c));  // the leaf gather below is the first reader of the masses
    const KeyT* sc = t.sorted_codes.as<KeyT>();
    if (p->compat_mode)
        k_karras<KeyT, true><<<grid, 256, 0, c->stream>>>(
            n, sc, t.perm.as<int32_t>(), c->pm.as<double4>(), t.parent.as<int32_t>(), t.sib.as<int32_t>(),
            t.rlo.as<int32_t>(), t.rhi.as<int32_t>(), t.child.as<int2>(), t.counters.as<uint32_t>(),
            t.node_cm.as<double4>(), t.groups.as<int2>(), gcount);
    else
        k_karras<KeyT, false><<<grid, 256, 0, c->stream>>>(
            n, sc, t.perm.as<int32_t>(), c->pm.as<double4>(), t.parent.as<int32_t>(), t.sib.as<int32_t>(),
            t.rlo.as<int32_t>(), t.rhi.as<int32_t>(), t.child.as<int2>(), t.counters.as<uint32_t>(),
            t.node_cm.as<double4>(), t.groups.as<int2>(), gcount);
    ASTER_CUDA(cudaGetLastError());
    ASTER_TRY(launch_bottom_up(c, n, p->theta));
    const int64_t spans = (n - 2 + REC_SPAN) / REC_SPAN;  // ceil((n - 1) / REC_SPAN); 0 for n == 1
    const int rgrid = (int)std::max<int64_t>(1, std::min<int64_t>(spans, (int64_t)c->sm_count * 8));
    k_front_records<<<rgrid, 256, 0, c->stream>>>(n, p->theta, t.counters.as<uint32_t>(), t.child.as<int2>(),
                                                 t.node_cm.as<double4>(), t.bmin.as<float4>(), t.bmax.as<float4>(),
                                                 t.crec.as<float4>());
    ASTER_CUDA(cudaGetLastError());
    c->stats.kernels += 2;
    return ASTER_OK;
}

int ensure_tree(aster_ctx* c) {
    LbvhBufs& t = c->tree;
    const int64_t n = c->n, m = 2 * n;  // 2n-1 nodes, +1 slot so parent[n] exists for n == 1
    const int64_t nblocks = (n + SORT_TILE - 1) / SORT_TILE;
    ASTER_TRY(t.codes.ensure((size_t)n * 8));
    ASTER_TRY(t.codes_alt.ensure((size_t)n * 8));
    ASTER_TRY(t.sorted_codes.ensure((size_t)n * 8));
    ASTER_TRY(t.perm.ensure((size_t)n * 4));
    ASTER_TRY(t.perm_alt.ensure((size_t)n * 4));
    ASTER_TRY(t.hist.ensure((size_t)nblocks * RADIX * 4));
    ASTER_TRY(t.digit_off.ensure((size_t)RADIX * 4));
    ASTER_TRY(t.parent.ensure((size_t)m * 4));
    ASTER_TRY(t.sib.ensure((size_t)m * 4));
    ASTER_TRY(t.front.ensure((size_t)n * 4));
    ASTER_TRY(t.rlo.ensure((size_t)m * 4));
    ASTER_TRY(t.rhi.ensure((size_t)m * 4));
    ASTER_TRY(t.counters.ensure((size_t)n * 4));
    ASTER_TRY(t.node_cm.ensure((size_t)m * sizeof(double4)));
    ASTER_TRY(t.bmin.ensure((size_t)m * sizeof(float4)));
    ASTER_TRY(t.bmax.ensure((size_t)m * sizeof(float4)));
    ASTER_TRY(t.child.ensure((size_t)m * sizeof(int2)));
    ASTER_TRY(t.groups.ensure((size_t)n * sizeof(int2)));
    ASTER_TRY(t.crec.ensure((size_t)4 * n * sizeof(float4)));
    ASTER_TRY(c->red.ensure(4096));
    t.n = n;
    return ASTER_OK;
}

}  // namespace

int aster_lbvh_build_dev(aster_ctx* c, const aster_params* p, bool box_ready) {
    ASTER_TRY(ensure_tree(c));
    if (!box_ready) {
        unsigned long long* box = red_box(c);
        ASTER_CUDA(cudaMemsetAsync(box, 0, sizeof(unsigned long long), c->stream));
        const int grid = (int)std::min<int64_t>((c->n + 255) / 256, (int64_t)c->sm_count * 8);
        k_box<<<grid, 256, 0, c->stream>>>(c->n, c->pm.as<double4>(), box);
        ASTER_CUDA(cudaGetLastError());
        c->stats.kernels += 1;
    }
    if (p->morton_bits == 63) ASTER_TRY(run_build<uint64_t>(c, p));
    else ASTER_TRY(run_build<uint32_t>(c, p));
    c->tree.built = true;
    return ASTER_OK;
}

int aster_lbvh_walk_launch(aster_ctx* c, const aster_params* p, int precision, bool kick, int32_t* counts,
                           bool fuse_next) {
    if (kick) c->mixed_valid = false;  // the closing kick moves the velocities
    fuse_next = fuse_next && kick;
    ASTER_CUDA(cudaMemsetAsync(red_groups(c) + 1, 0, sizeof(unsigned int), c->stream));  // work counter
    // the fused drift's box (the build that just ran has read the previous one)
    if (fuse_next) ASTER_CUDA(cudaMemsetAsync(red_box(c), 0, sizeof(unsigned long long), c->stream));
    const bool guard = !(p->eps2 > 0.0);
    if (precision != ASTER_MIXED && precision != ASTER_FP64) return ASTER_ERR_INVALID_ARG;
    const bool mixed = precision == ASTER_MIXED;
    if (pn_level(p) > 0) {
        // post-Newtonian law: node velocities from the current body velocities
        // (one climb, fresh arrival counters), then the walk with the pair law
        LbvhBufs& t = c->tree;
        const int64_t n = c->n;
        ASTER_TRY(t.node_v.ensure((size_t)2 * n * sizeof(double4)));
        if (n >= 2) ASTER_CUDA(cudaMemsetAsync(t.counters.ptr, 0, (size_t)(n - 1) * sizeof(uint32_t), c->stream));
        const int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)c->sm_count * 8);
        k_node_vel<<<grid, 256, 0, c->stream>>>(n, t.parent.as<int32_t>(), t.sib.as<int32_t>(), t.perm.as<int32_t>(),
                                                c->vel.as<double4>(), t.node_cm.as<double4>(),
                                                t.counters.as<uint32_t>(), t.node_v.as<double4>(), c->err_dev);
        ASTER_CUDA(cudaGetLastError());
        c->stats.kernels += 1;
        if (mixed && pn_level(p) == 1) {  // Newton + 1PN: the paired-FP32 list evaluation
            if (guard) { ASTER_TRY(kick ? launch_walk<true, true, true, 1>(c, p, counts, fuse_next) : launch_walk<true, true, false, 1>(c, p, counts, fuse_next)); }
            else       { ASTER_TRY(kick ? launch_walk<true, false, true, 1>(c, p, counts, fuse_next) : launch_walk<true, false, false, 1>(c, p, counts, fuse_next)); }
        } else if (mixed) {
            if (guard) { ASTER_TRY(kick ? launch_walk<true, true, true, 2>(c, p, counts, fuse_next) : launch_walk<true, true, false, 2>(c, p, counts, fuse_next)); }
            else       { ASTER_TRY(kick ? launch_walk<true, false, true, 2>(c, p, counts, fuse_next) : launch_walk<true, false, false, 2>(c, p, counts, fuse_next)); }
        } else {
            if (guard) { ASTER_TRY(kick ? launch_walk<false, true, true, 2>(c, p, counts, fuse_next) : launch_walk<false, true, false, 2>(c, p, counts, fuse_next)); }
            else       { ASTER_TRY(kick ? launch_walk<false, false, true, 2>(c, p, counts, fuse_next) : launch_walk<false, false, false, 2>(c, p, counts, fuse_next)); }
        }
        c->stats.kernels += 1;
        return ASTER_OK;
    }
    if (mixed) {
        if (guard) { ASTER_TRY(kick ? launch_walk<true, true, true>(c, p, counts, fuse_next) : launch_walk<true, true, false>(c, p, counts, fuse_next)); }
        else       { ASTER_TRY(kick ? launch_walk<true, false, true>(c, p, counts, fuse_next) : launch_walk<true, false, false>(c, p, counts, fuse_next)); }
    } else {
        if (guard) { ASTER_TRY(kick ? launch_walk<false, true, true>(c, p, counts, fuse_next) : launch_walk<false, true, false>(c, p, counts, fuse_next)); }
        else       { ASTER_TRY(kick ? launch_walk<false, false, true>(c, p, counts, fuse_next) : launch_walk<false, false, false>(c, p, counts, fuse_next)); }
    }
    c->stats.kernels += 1;
    return ASTER_OK;
}

// ---- tree export -------------------------------------------------------------
namespace {
// Node i of m = 2n - 1 in the view's layout: leaves (i < n) have no children
// and the box of their position; internal nodes' children come from child[].
__global__ void k_export_nodes(int64_t n, int64_t m, double theta, const double4* __restrict__ cm,
                               const float4* __restrict__ bmin, const float4* __restrict__ bmax,
                               const int2* __restrict__ child, double* __restrict__ mass, double* __restrict__ com,
                               float* __restrict__ fmin3, float* __restrict__ fmax3, float* __restrict__ rc2,
                               int32_t* __restrict__ left, int32_t* __restrict__ right) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 c = cm[i];
        mass[i] = c.w;
        com[3 * i] = c.x; com[3 * i + 1] = c.y; com[3 * i + 2] = c.z;
        const bool leaf = i < n;
        const float4 a = leaf ? leaf_lo(c) : bmin[i], b = leaf ? leaf_hi(c) : bmax[i];
        const int2 ch = leaf ? make_int2(-1, -1) : child[i];
        left[i] = ch.x;
        right[i] = ch.y;
        fmin3[3 * i] = a.x; fmin3[3 * i + 1] = a.y; fmin3[3 * i + 2] = a.z;
        fmax3[3 * i] = b.x; fmax3[3 * i + 1] = b.y; fmax3[3 * i + 2] = b.z;
        float4 h, l;
        if (leaf) leaf_trav(c, h, l);
        else node_trav(c, a, b, theta, h, l);
        rc2[i] = l.w;
    }
}
template <class KeyT>
__global__ void k_widen(int64_t n, const KeyT* __restrict__ in, uint64_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (uint64_t)in[i];
}
}  // namespace

static int export_tree(aster_ctx* c, const aster_params* p, aster_tree_view* v) {
    LbvhBufs& t = c->tree;
    const int64_t n = c->n, m = 2 * n - 1;
    cudaStream_t st = c->stream;
    const size_t need = (size_t)m * (8 + 24 + 12 + 12 + 4 + 8) + (size_t)n * 16 + 1024;
    ASTER_TRY(c->stage.ensure(need));
    char* base = c->stage.as<char>();
    double* mass = (double*)base;
    double* com = mass + m;
    float* fmin3 = (float*)(com + 3 * m);
    float* fmax3 = fmin3 + 3 * m;
    float* rc2 = fmax3 + 3 * m;
    int32_t* lft = (int32_t*)(rc2 + m);
    int32_t* rgt = lft + m;
    uint64_t* wide = (uint64_t*)(((uintptr_t)(rgt + m) + 15) & ~(uintptr_t)15);
    uint64_t* wide2 = wide + n;
    const int grid = (int)std::min<int64_t>((m + 255) / 256, (int64_t)c->sm_count * 16);
    k_export_nodes<<<grid, 256, 0, st>>>(n, m, p->theta, t.node_cm.as<double4>(), t.bmin.as<float4>(),
                                         t.bmax.as<float4>(), t.child.as<int2>(), mass, com, fmin3, fmax3, rc2, lft,
                                         rgt);
    if (p->morton_bits == 63) {
        k_widen<uint64_t><<<grid, 256, 0, st>>>(n, t.codes.as<uint64_t>(), wide);
        k_widen<uint64_t><<<grid, 256, 0, st>>>(n, t.sorted_codes.as<uint64_t>(), wide2);
    } else {
        k_widen<uint32_t><<<grid, 256, 0, st>>>(n, t.codes.as<uint32_t>(), wide);
        k_widen<uint32_t><<<grid, 256, 0, st>>>(n, t.sorted_codes.as<uint32_t>(), wide2);
    }
    ASTER_CUDA(cudaGetLastError());
    auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
        if (dst) ASTER_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
        return ASTER_OK;
    };
    ASTER_TRY(cp(v->codes, wide, (size_t)n * 8));
    ASTER_TRY(cp(v->sorted_codes, wide2, (size_t)n * 8));
    ASTER_TRY(cp(v->perm, t.perm.ptr, (size_t)n * 4));
    ASTER_TRY(cp(v->left, lft, (size_t)m * 4));
    ASTER_TRY(cp(v->right, rgt, (size_t)m * 4));
    ASTER_TRY(cp(v->parent, t.parent.ptr, (size_t)m * 4));
    ASTER_TRY(cp(v->range_lo, t.rlo.ptr, (size_t)m * 4));
    ASTER_TRY(cp(v->range_hi, t.rhi.ptr, (size_t)m * 4));
    ASTER_TRY(cp(v->node_mass, mass, (size_t)m * 8));
    ASTER_TRY(cp(v->node_com, com, (size_t)m * 24));
    ASTER_TRY(cp(v->node_bmin, fmin3, (size_t)m * 12));
    ASTER_TRY(cp(v->node_bmax, fmax3, (size_t)m * 12));
    ASTER_TRY(cp(v->node_rcrit2, rc2, (size_t)m * 4));
    unsigned long long bits = 0;
    ASTER_CUDA(cudaMemcpyAsync(&bits, red_box(c), 8, cudaMemcpyDeviceToHost, st));
    ASTER_CUDA(cudaStreamSynchronize(st));
    double box;
    memcpy(&box, &bits, 8);
    v->box = box;
    return ASTER_OK;
}

extern "C" int aster_lbvh_build(aster_ctx* c, const aster_params* p, aster_tree_view* view) {
    if (!c) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    cudaEventRecord(c->ev[0], c->stream);
    ASTER_TRY(aster_lbvh_build_dev(c, p, false));
    cudaEventRecord(c->ev[1], c->stream);
    ASTER_TRY(aster_finish(c));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_build = c->stats.ms_total = ms;
    if (view) ASTER_TRY(export_tree(c, p, view));
    return ASTER_OK;
}

extern "C" int aster_lbvh_forces(aster_ctx* c, const aster_params* p, int precision, double* acc_out,
                                 int32_t* list_counts) {
    if (!c) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    int32_t* cnt = nullptr;
    if (list_counts) {
        ASTER_TRY(c->targets.ensure((size_t)c->n * 4));
        cnt = c->targets.as<int32_t>();
    }
    ASTER_TRY(ensure_tree(c));
    unsigned long long* inter = red_inter(c);
    ASTER_CUDA(cudaMemsetAsync(inter, 0, 8, c->stream));
    cudaEventRecord(c->ev[0], c->stream);
    ASTER_TRY(aster_lbvh_build_dev(c, p, false));
    cudaEventRecord(c->ev[1], c->stream);
    ASTER_TRY(aster_lbvh_walk_launch(c, p, precision, false, cnt));
    cudaEventRecord(c->ev[2], c->stream);
    unsigned long long ic = 0;
    ASTER_CUDA(cudaMemcpyAsync(&ic, inter, 8, cudaMemcpyDeviceToHost, c->stream));
    if (list_counts)
        ASTER_CUDA(cudaMemcpyAsync(list_counts, cnt, (size_t)c->n * 4, cudaMemcpyDeviceToHost, c->stream));
    ASTER_TRY(aster_finish(c));
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&b, c->ev[1], c->ev[2]);
    c->stats.ms_build = a;
    c->stats.ms_force = b;
    c->stats.ms_total = a + b;
    c->stats.interactions = (double)ic;
    c->acc_valid = true;
    return aster_copy_acc_out(c, acc_out);
}
