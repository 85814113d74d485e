// sort.cuh -- stable LSD radix sort of (cell key, particle index) pairs, the
// scans it needs, and the grouping of sorted particles into warp items.
//
// Cell key of a particle: the cell holding it, from the reference's
// floor((x - min) / dx) by division (ForwardSimulation.cpp:19), shifted so that
// clamped out-of-grid cells stay non-negative,
//   c_a = stencil_base_a + 1 + 4            (in [1, dim_a + 5]),
// ordered brick-major: bricks of 4 x 4 x 4 cells, b_a = c_a >> 2, numbered
// linearly over nb_a = (dim_a + 5) / 4 + 1 bricks per axis, and the 64 cells of
// a brick in Morton order of their local coordinates l_a = c_a & 3,
//   key = ((b_0 nb_1 + b_1) nb_2 + b_2) 64 + morton(l_0, l_1, l_2),
//   morton = (l_0>>1) 32 + (l_1>>1) 16 + (l_2>>1) 8 + (l_0&1) 4 + (l_1&1) 2 + (l_2&1).
// So the particles of one cell (a run of equal keys), of one 2 x 2 x 2 octant
// of a brick (equal key >> 3) and of one brick (equal key >> 6) are contiguous
// in the sorted order.  Sorting is stable, so equal keys keep their index
// order and the permutation equals a CPU std::stable_sort / numpy
// argsort(kind="stable") of the keys.
//
// Radix sort: 8-bit digits, per pass three kernels --
//   upsweep   per-tile digit histograms  -> counts[digit][tile]
//   scan      exclusive scan of counts in digit-major order -> global offsets
//   downsweep stable scatter: within a tile, warps walk their 256 keys in 8
//             rounds of 32; __match_any_sync ranks equal digits inside a
//             round, per-warp digit counters carry ranks across rounds, and a
//             scan over warps orders the warps of a tile.
// Warp items: runs of equal keys cut into pieces of at most 8 particles; a
// particle kernel gives each item one warp (8 particles x 4 stencil slabs).
#pragma once
#include <cstdint>
#include "kernels.cuh"

namespace dmpm {

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROUNDS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;  // 2048 keys per tile
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// ------------------------------------------------------------------ keys
template <class T> struct KeyArgs {
    int n;
    size_t np;
    GridGeom geo;
    const T* st;  // layer state (x planes)
    int xlo;      // st carries the low parts of compensated positions (planes PXL)
    uint32_t* keys;
    uint32_t* vals;
};

DMPM_HD uint32_t bricks_per_axis(int dim) { return (uint32_t)(dim + 5) / 4u + 1u; }
// number of distinct keys of a grid (keys lie in [0, key_span))
DMPM_HD uint64_t key_span(const int dim[3]) {
    return (uint64_t)bricks_per_axis(dim[0]) * bricks_per_axis(dim[1]) * bricks_per_axis(dim[2]) * 64u;
}
DMPM_HD uint32_t cell_key(const int base[3], const int dim[3]) {
    const uint32_t c0 = (uint32_t)(base[0] + 5), c1 = (uint32_t)(base[1] + 5), c2 = (uint32_t)(base[2] + 5);
    const uint32_t brick = ((c0 >> 2) * bricks_per_axis(dim[1]) + (c1 >> 2)) * bricks_per_axis(dim[2]) + (c2 >> 2);
    const uint32_t l0 = c0 & 3u, l1 = c1 & 3u, l2 = c2 & 3u;
    const uint32_t morton = ((l0 >> 1) << 5) | ((l1 >> 1) << 4) | ((l2 >> 1) << 3) | ((l0 & 1u) << 2) |
                            ((l1 & 1u) << 1) | (l2 & 1u);
    return brick * 64u + morton;
}
// First cell (c_0, c_1, c_2) of the unit of 2^(shift/3) cells per axis whose keys
// share key >> shift (shift 6: a brick, 3: an octant of a brick, 0: a cell).
DMPM_HD void unit_first_cell(uint32_t key_hi, int shift, const int dim[3], int c[3]) {
    const uint32_t key = key_hi << shift;
    uint32_t brick = key >> 6;
    const uint32_t nb1 = bricks_per_axis(dim[1]), nb2 = bricks_per_axis(dim[2]);
    const uint32_t b2 = brick % nb2;
    brick /= nb2;
    const uint32_t b1 = brick % nb1, b0 = brick / nb1;
    const uint32_t m = key & 63u;
    c[0] = (int)(4u * b0 + (((m >> 5) & 1u) << 1) + ((m >> 2) & 1u));
    c[1] = (int)(4u * b1 + (((m >> 4) & 1u) << 1) + ((m >> 1) & 1u));
    c[2] = (int)(4u * b2 + (((m >> 3) & 1u) << 1) + (m & 1u));
}

template <class T> __global__ void k_cell_keys(KeyArgs<T> a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    int base[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (a.xlo)  // the base the FP32 stencil kernels form (load_xd, stencil_coord)
            (void)stencil_coord<float>(load_xd(a.st, a.np, p, c, 1), a.geo.mn[c], 1.0 / a.geo.dx, a.geo.dim[c], base[c]);
        else
            base[c] = stencil_base<T>(a.st[(size_t)(PX + c) * a.np + p] - (T)a.geo.mn[c], (T)a.geo.dx, a.geo.dim[c]);
    }
    a.keys[p] = cell_key(base, a.geo.dim);
    a.vals[p] = (uint32_t)p;
}

// ------------------------------------------------------------------ scan
// Three-phase exclusive scan (tile scan, scan of tile totals, add) with a sum
// or max operator, in place on n uint32 values.
struct OpSum {
    __device__ static uint32_t id() { return 0u; }
    __device__ static uint32_t op(uint32_t a, uint32_t b) { return a + b; }
};
struct OpMax {
    __device__ static uint32_t id() { return 0u; }
    __device__ static uint32_t op(uint32_t a, uint32_t b) { return a > b ? a : b; }
};

// Block-wide exclusive scan of one value per thread; returns the block total.
template <class Op> __device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t& total) {
    __shared__ uint32_t s_w[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = Op::op(y, x);
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t t = lane < nw ? s_w[lane] : Op::id();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t = Op::op(y, t);
        }
        s_w[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t warp_prefix = w > 0 ? s_w[w - 1] : Op::id();
    total = s_w[nw - 1];
    const uint32_t excl_in_warp = __shfl_up_sync(0xffffffffu, x, 1);
    const uint32_t r = Op::op(warp_prefix, lane > 0 ? excl_in_warp : Op::id());
    __syncthreads();
    return r;
}

// Phase 1: each block scans SCAN_TILE elements (blocked: thread t owns
// SCAN_ITEMS consecutive elements) and records its total.
template <class Op> __global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(uint32_t* data, int n, uint32_t* totals) {
    const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t acc = Op::id();
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        const size_t k = base + i;
        v[i] = k < (size_t)n ? data[k] : Op::id();
        acc = Op::op(acc, v[i]);
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan<Op>(acc, total);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        const size_t k = base + i;
        const uint32_t x = v[i];
        if (k < (size_t)n) data[k] = run;
        run = Op::op(run, x);
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = total;
}

// Phase 2: one block scans the tile totals in place (any count, looping).
template <class Op> __global__ void __launch_bounds__(1024) k_scan_totals(uint32_t* totals, int m, uint32_t* grand) {
    __shared__ uint32_t s_carry;
    if (threadIdx.x == 0) s_carry = Op::id();
    __syncthreads();
    for (int start = 0; start < m; start += blockDim.x) {
        const int k = start + threadIdx.x;
        const uint32_t v = k < m ? totals[k] : Op::id();
        uint32_t chunk_total;
        const uint32_t ex = block_exclusive_scan<Op>(v, chunk_total);
        const uint32_t carry = s_carry;
        if (k < m) totals[k] = Op::op(carry, ex);
        __syncthreads();
        if (threadIdx.x == 0) s_carry = Op::op(carry, chunk_total);
        __syncthreads();
    }
    if (threadIdx.x == 0 && grand) *grand = s_carry;
}

// Phase 3: combine each tile's local exclusive scan with its tile prefix.
template <class Op> __global__ void __launch_bounds__(SCAN_THREADS) k_scan_add(uint32_t* data, int n, const uint32_t* totals) {
    const uint32_t pre = totals[blockIdx.x];
    const size_t base = (size_t)blockIdx.x * SCAN_TILE;
    for (int i = threadIdx.x; i < SCAN_TILE; i += blockDim.x) {
        const size_t k = base + i;
        if (k < (size_t)n) data[k] = Op::op(pre, data[k]);
    }
}

// ------------------------------------------------------------------ radix sort
static __global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const uint32_t* __restrict__ keys, int n, int shift,
                                                          uint32_t* counts, int ntiles) {
    __shared__ uint32_t hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * RS_TILE;
    for (int i = threadIdx.x; i < RS_TILE; i += RS_THREADS) {
        const size_t k = base + i;
        if (k < (size_t)n) atomicAdd(&hist[(keys[k] >> shift) & 255u], 1u);
    }
    __syncthreads();
    counts[(size_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

static __global__ void __launch_bounds__(RS_THREADS) k_rs_downsweep(const uint32_t* __restrict__ keys_in,
                                                            const uint32_t* __restrict__ vals_in, uint32_t* keys_out,
                                                            uint32_t* vals_out, int n, int shift,
                                                            const uint32_t* __restrict__ offsets, int ntiles) {
    __shared__ uint32_t wcnt[RS_WARPS][256];
    __shared__ uint32_t toff[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
    toff[threadIdx.x] = offsets[(size_t)threadIdx.x * ntiles + blockIdx.x];
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * RS_TILE + (size_t)w * (32 * RS_ROUNDS);
    uint32_t key[RS_ROUNDS], val[RS_ROUNDS], rank[RS_ROUNDS];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; r++) {
        const size_t k = base + (size_t)r * 32 + lane;
        const bool ok = k < (size_t)n;
        key[r] = ok ? keys_in[k] : 0xffffffffu;
        val[r] = ok ? vals_in[k] : 0u;
        // out-of-range lanes use the pseudo-digit 256 so they never match a real one
        const uint32_t d = ok ? ((key[r] >> shift) & 255u) : 256u;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = ok ? wcnt[w][d] : 0u;
        rank[r] = before + (uint32_t)__popc(peers & lt);
        __syncwarp();
        if (ok && (peers & lt) == 0) wcnt[w][d] = before + (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {  // exclusive scan over warps, one digit per thread
        uint32_t acc = 0;
#pragma unroll
        for (int ww = 0; ww < RS_WARPS; ww++) {
            const uint32_t c = wcnt[ww][threadIdx.x];
            wcnt[ww][threadIdx.x] = acc;
            acc += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; r++) {
        const size_t k = base + (size_t)r * 32 + lane;
        if (k < (size_t)n) {
            const uint32_t d = (key[r] >> shift) & 255u;
            const uint32_t pos = toff[d] + wcnt[w][d] + rank[r];
            keys_out[pos] = key[r];
            vals_out[pos] = val[r];
        }
    }
}

// ------------------------------------------------------------------ warp items
// head[i] = i if a run of equal keys starts at i, else 0 (max-scan -> run start)
static __global__ void k_run_heads(const uint32_t* __restrict__ keys, int n, uint32_t* head) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    head[i] = (i == 0 || keys[i] != keys[i - 1]) ? (uint32_t)i : 0u;
}
// after an inclusive max-scan of head (exclusive scan combined with the own
// value), flag item starts: every 8th element of a run.
static __global__ void k_item_flags(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ run_excl, int n,
                             uint32_t* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t own = (i == 0 || keys[i] != keys[i - 1]) ? (uint32_t)i : 0u;
    const uint32_t start = run_excl[i] > own ? run_excl[i] : own;
    flags[i] = ((uint32_t)i - start) % 8u == 0u ? 1u : 0u;
}
// flags has been exclusive-sum-scanned into idx; write item starts.
static __global__ void k_item_starts(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ run_excl,
                              const uint32_t* __restrict__ idx, int n, uint32_t* item_start) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {  // sentinel: one past the last item
        return;
    }
    const uint32_t own = (i == 0 || keys[i] != keys[i - 1]) ? (uint32_t)i : 0u;
    const uint32_t start = run_excl[i] > own ? run_excl[i] : own;
    if (((uint32_t)i - start) % 8u == 0u) item_start[idx[i]] = (uint32_t)i;
}
static __global__ void k_item_sentinel(uint32_t* item_start, const uint32_t* n_items, int n) {
    item_start[*n_items] = (uint32_t)n;
}

// ------------------------------------------------------------------ units
// A unit is a run of sorted particles with equal key >> shift: the particles of
// one brick (shift 6) or one brick octant (shift 3).  flags[i] = 1 where a unit
// starts; after an exclusive sum scan of flags into idx, k_unit_starts writes
// each unit's first sorted position and its key >> shift.
__device__ __forceinline__ bool unit_head(const uint32_t* keys, int i, int shift) {
    return i == 0 || (keys[i] >> shift) != (keys[i - 1] >> shift);
}
static __global__ void k_unit_flags(const uint32_t* __restrict__ keys, int n, int shift, uint32_t* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = unit_head(keys, i, shift) ? 1u : 0u;
}
static __global__ void k_unit_starts(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ idx, int n,
                                     int shift, uint32_t* unit_start, uint32_t* unit_key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !unit_head(keys, i, shift)) return;
    unit_start[idx[i]] = (uint32_t)i;
    unit_key[idx[i]] = keys[i] >> shift;
}
// Items never straddle units (an item is part of one cell's run), so unit u's
// items are [unit_item[u], unit_item[u + 1]): item i starts unit idx[p] where
// its first sorted position p starts one.  The last entry is the item count.
static __global__ void k_unit_items(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ item_start,
                                    const uint32_t* __restrict__ n_items, const uint32_t* __restrict__ idx,
                                    const uint32_t* __restrict__ n_units, int shift, uint32_t* unit_item) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int ni = (int)*n_items;
    if (i == ni) unit_item[*n_units] = (uint32_t)ni;
    if (i >= ni) return;
    const uint32_t p = item_start[i];
    if (unit_head(keys, (int)p, shift)) unit_item[idx[p]] = (uint32_t)i;
}

}  // namespace dmpm
