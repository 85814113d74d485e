// kernels_warp.cuh -- FP32 path kernels organised around cell-sorted warp items.
//
// GENERAL (a test switch) forces the per-lane reductions everywhere.
//
// A warp item is a run of at most 8 particles that share a cell in the sorted
// order (sort.cuh).  One warp serves one item: lane = 4 q + s handles particle
// slot q (0..7) and stencil slab s (0..3), i.e. the 16 nodes
// (base_x + s, base_y + j, base_z + k), j, k in 0..3, fully unrolled with
// compile-time j, k.  When all 8 particles of the warp share the cell (the
// common case), scatters combine the 8 particles' contributions with a
// butterfly reduce-scatter over the lanes of equal s, so each lane ends up
// owning one node's complete sum and issues a single vector
// red.global.add.v4.f32 per 8 nodes x 4 values; otherwise every lane issues
// its own reductions.  Gathers sum the 16-node partial results of the 4 slab
// lanes with two xor-shuffles.  The FP64 polar decomposition lives in the
// per-particle kernels k_stress (forward) and k_adj_finalize (adjoint), so
// the node loops keep a small register footprint.
//
// Math per stage is that of kernels.cuh (which cites the reference).
//
// Strain storage: the FP32 path keeps each layer's deformation gradient as its
// strain H = F - I in the F planes (PF).  Strains of a few 1e-3 keep float's
// full relative precision this way, where F itself (about 1) would round them
// to ~1e-4 relative at every step.  Kernels form F = I + H where they need it
// -- in FP64 for the polar decomposition -- and update H directly:
//   H' = (1 - s)(D + dt C' (I + D)) + s H,  D = H + dFc.
// The host converts at upload and download; the FP64 path stores F.
#pragma once
#include "fixpoint.cuh"
#include "sort.cuh"

namespace dmpm {

// F + dFc = I + H + dFc of layer n, in float and (exactly) in double
__device__ __forceinline__ m3<float> fe_from_strain(const m3<float>& H, const m3<float>& dfc) {
    m3<float> r = H + dfc;
    r.a[0][0] += 1.f;
    r.a[1][1] += 1.f;
    r.a[2][2] += 1.f;
    return r;
}
__device__ __forceinline__ m3<double> fe_from_strain_d(const m3<float>& H, const m3<float>& dfc) {
    m3<double> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = (double)H.a[i][j] + (double)dfc.a[i][j] + (i == j ? 1.0 : 0.0);
    return r;
}

struct WarpItems {
    const uint32_t* order;       // sorted particle indices
    const uint32_t* item_start;  // n_items + 1 entries
    int n_items;
};

struct ItemLane {
    int p;       // particle index (slot 0's particle for idle lanes)
    bool valid;  // lane carries a particle
    int q, s;
};

__device__ __forceinline__ ItemLane item_lane(const WarpItems& it, int item) {
    ItemLane r;
    const int lane = threadIdx.x & 31;
    r.q = lane >> 2;
    r.s = lane & 3;
    const uint32_t st = it.item_start[item];
    const uint32_t cnt = it.item_start[item + 1] - st;
    r.valid = (uint32_t)r.q < cnt;
    r.p = (int)it.order[st + (r.valid ? r.q : 0)];
    return r;
}

// true when every lane's stencil base equals lane 0's
__device__ __forceinline__ bool warp_uniform_base(const int b[3]) {
    const int b0 = __shfl_sync(0xffffffffu, b[0], 0), b1 = __shfl_sync(0xffffffffu, b[1], 0),
              b2 = __shfl_sync(0xffffffffu, b[2], 0);
    return __all_sync(0xffffffffu, b[0] == b0 && b[1] == b1 && b[2] == b2);
}

// Butterfly reduce-scatter over the 8 lanes that share lane & 3, for vectors
// whose 8 blocks of N/8 entries the lanes hold in a lane-permuted order: lane
// L's block b holds stencil node b ^ perm(L), perm(L) = 4 (L>>4 & 1) +
// 2 (L>>3 & 1) + (L>>2 & 1) (scatter_perm).  Then at every stage each lane
// keeps the lower half and sends the upper half -- the partner holds the same
// nodes there -- with no per-lane selects.  On return v[0 .. N/8) of lane L
// hold the sums of node perm(L)'s entries over the 8 lanes.
template <int N> __device__ __forceinline__ void reduce_scatter8(float (&v)[N]) {
#pragma unroll
    for (int i = 0; i < N / 2; i++) v[i] += __shfl_xor_sync(0xffffffffu, v[i + N / 2], 16);
#pragma unroll
    for (int i = 0; i < N / 4; i++) v[i] += __shfl_xor_sync(0xffffffffu, v[i + N / 4], 8);
#pragma unroll
    for (int i = 0; i < N / 8; i++) v[i] += __shfl_xor_sync(0xffffffffu, v[i + N / 8], 4);
}
// this lane's node permutation for reduce_scatter8: row bit (jp) and axis-2 bits (kp)
struct ScatterPerm {
    int jp, kp;
};
__device__ __forceinline__ ScatterPerm scatter_perm() {
    const int lane = threadIdx.x & 31;
    return ScatterPerm{(lane >> 4) & 1, ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1)};
}

template <int N> __device__ __forceinline__ void reduce_slabs(float (&v)[N]) {
#pragma unroll
    for (int i = 0; i < N; i++) {
        v[i] += __shfl_xor_sync(0xffffffffu, v[i], 1);
        v[i] += __shfl_xor_sync(0xffffffffu, v[i], 2);
    }
}

__device__ __forceinline__ bool in_grid(const GridGeom& g, int i, int j, int k) {
    return i >= 0 && i < g.dim[0] && j >= 0 && j < g.dim[1] && k >= 0 && k < g.dim[2];
}
__device__ __forceinline__ size_t node_id(const GridGeom& g, int i, int j, int k) {
    return ((size_t)i * g.dim[1] + j) * g.dim[2] + k;
}

// Node addressing of a lane's 16 stencil nodes (base_x + s, base_y + j, base_z + k):
// node (j, k) = g00 + j * dim_z + k in 32-bit arithmetic (grids are limited to
// 2^31 nodes) and bit 4j + k of mask says whether that node lies in the grid.
// g00 may point outside the grid; it is only dereferenced under the mask.
struct LaneNodes {
    int g00, sj;
    unsigned mask;
};
__device__ __forceinline__ LaneNodes lane_nodes(const GridGeom& g, const int base[3], int s) {
    LaneNodes r;
    const int gi = base[0] + s;
    r.sj = g.dim[2];
    r.g00 = (gi * g.dim[1] + base[1]) * g.dim[2] + base[2];
    unsigned mj = 0, mk = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        mj |= ((unsigned)(base[1] + t) < (unsigned)g.dim[1]) ? (1u << t) : 0u;
        mk |= ((unsigned)(base[2] + t) < (unsigned)g.dim[2]) ? (1u << t) : 0u;
    }
    unsigned m = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) m |= ((mj >> j) & 1u) ? (mk << (4 * j)) : 0u;
    r.mask = ((unsigned)gi < (unsigned)g.dim[0]) ? m : 0u;
    return r;
}

// Per-lane stencil weights: slab s of axis 0, all 4 nodes of axes 1 and 2.
struct LaneW {
    float d0, n0, s0;
    float d1[4], n1[4], s1[4];
    float d2[4], n2[4], s2[4];
};
// Branch-free cubic B-spline and slope (same piecewise polynomials as
// Interpolation.h:5-30, evaluated with selects so divergent lanes do not
// serialise).
__device__ __forceinline__ float bsp(float q) {
    const float a = fabsf(q);
    const float inner = (0.5f * a - 1.f) * a * a + 2.f / 3.f;
    const float t = 2.f - a;
    const float outer = t * t * t * (1.f / 6.f);
    return a < 1.f ? inner : (a < 2.f ? outer : 0.f);
}
__device__ __forceinline__ float bsp_slope(float q) {
    const float a = fabsf(q);
    const float inner = (1.5f * a - 2.f) * q;
    const float outer = (-0.5f * a + 2.f - 2.f / a) * q;
    return a < 1.f ? inner : (a < 2.f ? outer : 0.f);
}

// The 4 lanes of a particle (equal lane >> 2) each evaluate the weights of
// stencil node s on all three axes; axis-1 and axis-2 values of the other
// nodes come from the sibling lanes by shuffles.  Every lane of the warp must
// call this (full-mask shuffles).
__device__ __forceinline__ void lane_weights(const float t[3], const GridGeom& g, int s, LaneW& w, bool slopes) {
    const float dx = (float)g.dx;
    float d[3], n[3], sl[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float q = (float)s - t[c];  // node offset in cells (exact for t in [1, 2))
        d[c] = q * dx;
        n[c] = bsp(q);
        sl[c] = slopes ? bsp_slope(q) : 0.f;
    }
    w.d0 = d[0];
    w.n0 = n[0];
    w.s0 = sl[0];
    const int grp = (threadIdx.x & 31) & ~3;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        w.d1[t] = __shfl_sync(0xffffffffu, d[1], grp + t);
        w.n1[t] = __shfl_sync(0xffffffffu, n[1], grp + t);
        w.d2[t] = __shfl_sync(0xffffffffu, d[2], grp + t);
        w.n2[t] = __shfl_sync(0xffffffffu, n[2], grp + t);
        if (slopes) {
            w.s1[t] = __shfl_sync(0xffffffffu, sl[1], grp + t);
            w.s2[t] = __shfl_sync(0xffffffffu, sl[2], grp + t);
        } else {
            w.s1[t] = 0.f;
            w.s2[t] = 0.f;
        }
    }
}

// As lane_weights, but axis 1 is left to the caller: it gets this lane's own
// axis-1 offset, weight and slope in own1 and fetches row j's values with
// row_weights (three shuffles) when it reaches that row, so only one row's
// values are live at a time.  Fills d0, n0, s0 and the axis-2 arrays of w,
// the latter in the order of node k ^ kperm (reduce_scatter8's permutation).
__device__ __forceinline__ void lane_weights_k(const float t[3], const GridGeom& g, int s, LaneW& w, float own1[3],
                                               bool slopes, int kperm = 0) {
    const float dx = (float)g.dx;
    float d[3], n[3], sl[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float q = (float)s - t[c];
        d[c] = q * dx;
        n[c] = bsp(q);
        sl[c] = slopes ? bsp_slope(q) : 0.f;
    }
    w.d0 = d[0];
    w.n0 = n[0];
    w.s0 = sl[0];
    own1[0] = d[1];
    own1[1] = n[1];
    own1[2] = sl[1];
    const int grp = (threadIdx.x & 31) & ~3;
#pragma unroll
    for (int t = 0; t < 4; t++) {  // entry t holds axis-2 node t ^ kperm
        w.d2[t] = __shfl_sync(0xffffffffu, d[2], grp + (t ^ kperm));
        w.n2[t] = __shfl_sync(0xffffffffu, n[2], grp + (t ^ kperm));
        w.s2[t] = slopes ? __shfl_sync(0xffffffffu, sl[2], grp + (t ^ kperm)) : 0.f;
    }
}
// row j's axis-1 (offset, weight, slope) from the lane of slab j; every lane must call it
__device__ __forceinline__ void row_weights(const float own1[3], int j, float& d1, float& n1, float& s1) {
    const int src = ((threadIdx.x & 31) & ~3) + j;
    d1 = __shfl_sync(0xffffffffu, own1[0], src);
    n1 = __shfl_sync(0xffffffffu, own1[1], src);
    s1 = __shfl_sync(0xffffffffu, own1[2], src);
}

// stencil base and lattice coordinates t = (x - mn) / dx - base of particle p
// (compensated positions when xlo: load_xd, stencil_coord); xd, if given,
// receives the positions
__device__ __forceinline__ void load_x_base(const float* st, size_t np, int p, const GridGeom& g, float t[3],
                                            int base[3], int xlo, double* xd = nullptr) {
    const double idx = 1.0 / g.dx;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const double x = load_xd(st, np, p, c, xlo);
        if (xd) xd[c] = x;
        t[c] = stencil_coord<float>(x, g.mn[c], idx, g.dim[c], base[c]);
    }
}
// x' = x + dt v of axis c from the position x read by load_x_base, into the
// next layer's planes (hi and, when xlo, lo); returns the stored hi.  The
// brick G2P keeps x in registers from its first load (64.6 us per step on the
// 64^3, 267k-particle workload, against 67.4 us re-reading it before the
// store); the warp-item G2P re-reads it (advance_x), as holding it there
// costs 52 bytes of spill at its 64-register budget.
__device__ __forceinline__ float store_x(float* st_next, size_t npn, int p, int c, double x, float dt, float v,
                                         int xlo) {
    if (!xlo) {
        const float xn = (float)x + dt * v;
        st_next[(size_t)(PX + c) * npn + p] = xn;
        return xn;
    }
    const double xn = x + (double)(dt * v);
    const float hi = (float)xn;
    st_next[(size_t)(PX + c) * npn + p] = hi;
    st_next[(size_t)(PXL + c) * npn + p] = (float)(xn - (double)hi);
    return hi;
}
// the same, re-reading x from layer n's planes
__device__ __forceinline__ float advance_x(const float* st, float* st_next, size_t npl, size_t npn, int p, int c,
                                           float dt, float v, int xlo) {
    return store_x(st_next, npn, p, c, load_xd(st, npl, p, c, xlo), dt, v, xlo);
}

// ------------------------------------------------------------------ args
// Minimum resident blocks per SM (the register cap the compiler works to) for
// the per-particle FP64 kernels: k_stress at 256 threads per block (2: 128
// registers, no spills; 1 lets it take 132 and run one block per SM),
// k_adj_finalize at 128 (4: 128 registers with a 40-byte spill, 11 % faster
// than the 168-register build on the 64^3, 267k-particle workload), and its
// FP64 part alone (5: 96 registers with a 144-byte spill, 40.6 against 45.2 us
// at 4 and 44.4 us at 6 on the same workload: the extra warps hide more of the
// load latency than the spills cost).
// k_stress takes the FP64 polar factors from the scaled Newton iteration
// (polar_newton) where det(F + dFc) > 0 and from the SVD (polar3) otherwise;
// 0 uses the SVD everywhere
#ifndef DMPM_NEWTON_POLAR
#define DMPM_NEWTON_POLAR 1
#endif
#ifndef DMPM_STRESS_MIN_BLOCKS
#define DMPM_STRESS_MIN_BLOCKS 2
#endif
#ifndef DMPM_FINALIZE_MIN_BLOCKS
#define DMPM_FINALIZE_MIN_BLOCKS 4
#endif
#ifndef DMPM_FINALIZE_STRESS_MIN_BLOCKS
#define DMPM_FINALIZE_STRESS_MIN_BLOCKS 5
#endif
// and for the warp-item kernels: the adjoint gather and P2G in blocks of
// DMPM_GATHER_THREADS / DMPM_P2G_THREADS (256), the adjoint scatter below in
// blocks of DMPM_ADJ_SCATTER_THREADS (128)
#ifndef DMPM_GATHER_MIN_BLOCKS
#define DMPM_GATHER_MIN_BLOCKS 3
#endif
#ifndef DMPM_GATHER_THREADS
#define DMPM_GATHER_THREADS 256
#endif
#ifndef DMPM_SCATTER_MIN_BLOCKS
#define DMPM_SCATTER_MIN_BLOCKS 3
#endif
#ifndef DMPM_P2G_THREADS
#define DMPM_P2G_THREADS 256
#endif
// CTAs per SM of the persistent grids (no more than the register budget above lets reside)
#ifndef DMPM_GATHER_CTAS
#define DMPM_GATHER_CTAS DMPM_GATHER_MIN_BLOCKS
#endif
#ifndef DMPM_SCATTER_CTAS
#define DMPM_SCATTER_CTAS DMPM_SCATTER_MIN_BLOCKS
#endif
// the adjoint scatter on its own, in blocks of 128 threads: 7 per SM (72
// registers, 28-byte spill, 28 warps) take 53.3 us on the 64^3, 267k-particle
// workload, against 55.4 us for 4 blocks of 256 (64 registers, 68-byte
// spill), 59.4 us for 3 of 256 and 55.7 us for 5 of 128 (95 registers, no
// spill); P2G is faster at 3 blocks of 256 (the gather at 4: 87.0 against 78.9 us)
#ifndef DMPM_ADJ_SCATTER_MIN_BLOCKS
#define DMPM_ADJ_SCATTER_MIN_BLOCKS 7
#endif
#ifndef DMPM_ADJ_SCATTER_THREADS
#define DMPM_ADJ_SCATTER_THREADS 128
#endif
#ifndef DMPM_ADJ_SCATTER_CTAS
#define DMPM_ADJ_SCATTER_CTAS DMPM_ADJ_SCATTER_MIN_BLOCKS
#endif

// Grid of one instance of a batch: its geometry, the offset of its first node
// in the batch's concatenated grids and of its first cell key.
struct InstGeo {
    GridGeom g;
    int goff;
    uint32_t koff;
};

// Plane strides: np for the per-particle constants, controls and adjoint
// scratch; npl for the state, affine/polar planes and adjoint of layer n;
// npn for the state and adjoint of layer n + 1.  One scene: all three equal.
// A batch stores each layer for the instances still running, so its layers
// have their own strides.
struct WArgs {
    int n;
    size_t np, npl, npn;
    GridGeom geo;
    float dt, drag, s, fext[3];
    WarpItems items;
    const uint32_t* n_items_dev;  // item count on the device (grid-stride launches), or null: items.n_items
    const InstGeo* ig;            // batch: per-instance grids, indexed by item_inst
    const uint16_t* item_inst;
    const float* st;       // layer n state
    float* st_next;        // layer n+1 state
    int xlo;               // st and st_next carry the low parts of compensated positions (planes PXL)
    const float* cst;      // constants
    const float* dfc;      // dFc of layer n
    float* G;              // [24][npl] per layer: G (9), polar R (9), polar S (6: s00 s01 s02 s11 s12 s22)
    node4<float>* grid;    // layer n grid: (p, m) after P2G, (v, m) after k_gop_inplace
    float* P;              // debug: stress of layer n (or null)
    unsigned* status;
    // adjoint
    const float* adj_next;
    float* adj;
    float* adjn;           // [12][np]: dLdv_next (3), dLdC_next (9)
    float* gath;           // [18][np]: M (9), X (3), u (3), z (3)
    node4<float>* gadj;    // (dLdv.xyz, 0)
    node4<float>* gadj2;   // per node two records: (dLdp.xyz, dLdm), (v.xyz, m)
    float* ctrl_grad;      // per-layer dL/d dFc [9][np] or null
    double* ctrl_acc;      // tied FP64 accumulator or null
    float* dbg_dLdP;
    float* dbg_vnext;
    float* dbg_Cnext;
    // G2P with the next step's stress stage (kernels_brick.cuh): dFc of layer n + 1,
    // its G planes and its debug P (or null)
    const float* dfc_next;
    float* G_next;
    float* P_next;
    // deterministic mode (fixpoint.cuh): integer node sums and their bound slots, or null
    fix4* fix;
    unsigned* fixb;
    // brick units of the sorted order (kernels_brick.cuh): unit u holds the
    // sorted positions [unit_start[u], unit_start[u + 1]), all with key >> shift
    // equal to unit_key[u]; the unit count stays on the device
    const uint32_t* unit_start;
    const uint32_t* unit_key;
    const uint32_t* n_units_dev;
    const uint32_t* unit_item;  // first warp item of each unit (n_units + 1 entries), or null
};

// How a warp-item launch walks its items:
//   ITEMS_PER_WARP   one warp per item, the grid sized on the host from the item count
//   ITEMS_PERSISTENT a persistent grid sized to the SMs loops over the items, whose
//                    count stays on the device (no host read-back, so capturable)
//   ITEMS_BATCH      persistent, items of several instances, each item's grid looked up
enum : int { ITEMS_PER_WARP = 0, ITEMS_PERSISTENT = 1, ITEMS_BATCH = 2 };
__device__ __forceinline__ int item_count(const WArgs& a) {
    return a.n_items_dev ? (int)*a.n_items_dev : a.items.n_items;
}
__device__ __forceinline__ int first_warp() { return (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); }
template <int MODE> __device__ __forceinline__ int next_item(int item, int nit) {
    return MODE != ITEMS_PER_WARP ? item + (int)((gridDim.x * blockDim.x) >> 5) : nit;
}
template <int MODE> __device__ __forceinline__ void item_grid(const WArgs& a, int item, GridGeom& g, int& goff) {
    if constexpr (MODE == ITEMS_BATCH) {
        const InstGeo& ig = a.ig[a.item_inst[item]];
        g = ig.g;
        goff = ig.goff;
    } else {
        g = a.geo;
        goff = 0;
    }
}

// G2P and the adjoint gather over a warp whose 32 lanes share one stencil base
// (all 8 particles of the item in one cell, the common case after the cell sort)
// first copies the item's 64 stencil nodes, R consecutive node4 records each,
// from global memory into the warp's shared-memory slice: 2R independent
// 16-byte loads per lane, all in flight together, instead of 16 R dependent
// loads per lane.  Record r of stencil node (s, j, k) lands at
// dst[stage_index<R>(16 s + 4 j + k, r)]; nodes outside the grid are stored as
// zeros.  Each slab's 16 R records are followed by one padding record, so the
// four slabs that a warp's lanes read at the same time fall into different
// shared-memory banks (without it the reads conflict 4-way; with it the
// gather takes 86 instead of 116 us and G2P 56 instead of 73 us on the 64^3,
// 267k-particle workload).  Warp kernels run 256-thread blocks (8 warps), one
// slice per warp.
#ifndef DMPM_STAGE_NODES
#define DMPM_STAGE_NODES 1
#endif
template <int R> __device__ __forceinline__ int stage_index(int n, int r) { return R * n + r + (n >> 4); }
template <int R> struct StageRecords { static constexpr int value = 64 * R + 4; };
template <int R>
__device__ __forceinline__ void stage_stencil(const node4<float>* __restrict__ src, const GridGeom& g, int goff,
                                              const int base[3], node4<float>* dst) {
    const int lane = threadIdx.x & 31;
    __syncwarp();  // the previous item's readers are done with the slice
#pragma unroll
    for (int i = 0; i < 2 * R; i++) {
        const int t = lane + 32 * i;
        const int n = t / R, r = t % R;
        const int gi = base[0] + (n >> 4), gj = base[1] + ((n >> 2) & 3), gk = base[2] + (n & 3);
        const bool in = (unsigned)gi < (unsigned)g.dim[0] && (unsigned)gj < (unsigned)g.dim[1] &&
                        (unsigned)gk < (unsigned)g.dim[2];
        dst[stage_index<R>(n, r)] = in ? src[(size_t)R * (unsigned)((gi * g.dim[1] + gj) * g.dim[2] + gk + goff) + r]
                                       : node4<float>{0.f, 0.f, 0.f, 0.f};
    }
    __syncwarp();
}

// ------------------------------------------------------------------ forward
// P = PK(F + dFc) in FP64;  G = -3/dx^2 dt vol P Fe^T + m C  (P_op_1 and the
// particle-constant part of SingleParticle_to_grid, ForwardSimulation.cpp:6-9, 38)
// The stress stage of particle p: the FP64 polar decomposition of
// Fe = I + H + dFc (scaled Newton where det > 0, SVD otherwise), P, and
// G = -3/dx^2 dt vol P Fe^T + m C.  Writes G and the polar factors R, S (for
// the adjoint's k_adj_finalize) into the planes at Gp (stride ng) and P into Pp
// unless it is null; returns G.  cfetch() gives C, fetched after the polar so
// that it holds no registers through it.
template <class CFetch>
__device__ __forceinline__ m3<float> stress_particle(const WArgs& a, int p, const m3<float>& H, const m3<float>& dfc,
                                                     const CFetch& cfetch, float* Gp, size_t ng, float* Pp) {
    const size_t np = a.np;
    const m3<float> Fe = fe_from_strain(H, dfc);
    const m3<double> Fed = fe_from_strain_d(H, dfc);
    m3<double> Rd, Sd;
    if (!DMPM_NEWTON_POLAR || !polar_newton(Fed, Rd, Sd)) polar3(Fed, Rd, Sd);
    const m3<double> Pd = pk_from_polar(Fed, Rd, (double)a.cst[(size_t)KLAM * np + p], (double)a.cst[(size_t)KMU * np + p]);
    const m3<float> P = m3_cast<float>(Pd);
    if (Pp) store_m3(Pp, ng, p, P);
    store_m3(Gp + 9 * ng, ng, p, m3_cast<float>(Rd));
    Gp[18 * ng + p] = (float)Sd.a[0][0];
    Gp[19 * ng + p] = (float)Sd.a[0][1];
    Gp[20 * ng + p] = (float)Sd.a[0][2];
    Gp[21 * ng + p] = (float)Sd.a[1][1];
    Gp[22 * ng + p] = (float)Sd.a[1][2];
    Gp[23 * ng + p] = (float)Sd.a[2][2];
    const float dx = (float)a.geo.dx;
    const float k = -3.f / (dx * dx) * a.dt * a.cst[(size_t)KVOL * np + p];
    const m3<float> G = (k * P) * transpose(Fe) + a.cst[(size_t)KM * np + p] * cfetch();
    store_m3(Gp, ng, p, G);
    return G;
}

// DET: also raise the deterministic mode's P2G bounds (fixpoint.cuh) in a.fixb.
template <bool DET = false> __global__ void __launch_bounds__(256, DMPM_STRESS_MIN_BLOCKS) k_stress(WArgs a) {
    const size_t np = a.np, npl = a.npl;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    float cmom = 0.f, cmass = 0.f;
    if (p < a.n) {
        const m3<float> H = load_m3(a.st + (size_t)PF * npl, npl, p), dfc = load_m3(a.dfc, np, p);
        const m3<float> G = stress_particle(
            a, p, H, dfc, [&]() { return load_m3(a.st + (size_t)PC * npl, npl, p); }, a.G, npl, a.P);
        if constexpr (DET) {
            const float dx = (float)a.geo.dx;
            // bound on P2G's per-particle values: |m v damp + G d| with |d| < 2 dx, and m
            const float mp = a.cst[(size_t)KM * np + p], damp = 1.f - a.dt * a.drag;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float t = fabsf(mp * a.st[(size_t)(PV + c) * npl + p] * damp) +
                                2.f * dx * (fabsf(G.a[c][0]) + fabsf(G.a[c][1]) + fabsf(G.a[c][2]));
                cmom = fmaxf(cmom, t);
            }
            cmass = mp;
        }
    }
    if constexpr (DET) {  // every lane of every warp reaches these
        fix_bound(a.fixb + FIXB_MOMENTUM, cmom * 1.001f);
        fix_bound(a.fixb + FIXB_MASS, cmass * 1.001f);
    }
}

// P2G: m_g += w m_p;  p_g += w (m_p v (1 - dt drag) + G (x_g - x_p))
// One warp item of P2G.  DET: integer node sums (fixpoint.cuh) into a.fix
// instead of float atomics into a.grid; with a tile (ft.t non-null), the sums
// of an item whose stencil lies in the tile go to its shared-memory integers.
template <bool GENERAL, int MODE, bool DET, bool TILE>
__device__ __forceinline__ void p2g_item(const WArgs& a, int item, const FixScale& sp, const FixScale& sm,
                                         const FixTile& ft) {
    const size_t np = a.np, npl = a.npl;
    {
        GridGeom geo;
        int goff;
        item_grid<MODE>(a, item, geo, goff);
        const ItemLane L = item_lane(a.items, item);
        float t[3];
        int base[3];
        load_x_base(a.st, npl, L.p, geo, t, base, a.xlo);
        const bool uniform = !GENERAL && warp_uniform_base(base);
        // slot (jj, kk) of each half holds node (2 half + (jj ^ P.jp), kk ^ P.kp)
        const ScatterPerm P = scatter_perm();
        LaneW w;
        float own1[3];
        lane_weights_k(t, geo, L.s, w, own1, false, P.kp);
        const float mp = L.valid ? a.cst[(size_t)KM * np + L.p] : 0.f;
        const float damp = 1.f - a.dt * a.drag;
        float mvd[3], g0[3];
        m3<float> G = load_m3(a.G, npl, L.p);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            mvd[c] = mp * a.st[(size_t)(PV + c) * npl + L.p] * damp;
            g0[c] = G.a[c][0] * w.d0;
        }
        LaneNodes N = lane_nodes(geo, base, L.s);
        N.g00 += goff;
        // tile offset of node (0, 0, 0) of the item's stencil, or -1 when the stencil is not inside the tile
        const int tile_l = TILE && uniform ? fix_tile_offset(ft, base) : -1;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            float v[32];
#pragma unroll
            for (int jj = 0; jj < 2; jj++) {
                float d1, n1, s1;
                row_weights(own1, 2 * half + (jj ^ P.jp), d1, n1, s1);
                float g1[3];
#pragma unroll
                for (int c = 0; c < 3; c++) g1[c] = g0[c] + G.a[c][1] * d1;
                const float w01 = L.valid ? w.n0 * n1 : 0.f;
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    const float wt = w01 * w.n2[kk];
                    const int o = (jj * 4 + kk) * 4;
#pragma unroll
                    for (int c = 0; c < 3; c++) v[o + c] = wt * (mvd[c] + g1[c] + G.a[c][2] * w.d2[kk]);
                    v[o + 3] = wt * mp;
                }
            }
            if (uniform) {
                reduce_scatter8<32>(v);
                const int j = 2 * half + P.jp, k = P.kp;
                if (((N.mask >> (4 * j + k)) & 1u) && (v[0] != 0.f || v[1] != 0.f || v[2] != 0.f || v[3] != 0.f)) {
                    if (TILE && tile_l >= 0)
                        fix_red4_tile(ft, tile_l + (L.s * ft.E + j) * ft.E + k, v[0], v[1], v[2], v[3], sp.s, sm.s);
                    else if (DET) fix_red4(a.fix + (N.g00 + j * N.sj + k), v[0], v[1], v[2], v[3], sp.s, sm.s);
                    else red_add4(a.grid + (N.g00 + j * N.sj + k), v[0], v[1], v[2], v[3]);
                }
            } else if (L.valid) {
#pragma unroll
                for (int nd = 0; nd < 8; nd++) {
                    const int j = 2 * half + ((nd >> 2) ^ P.jp), k = (nd & 3) ^ P.kp;
                    if (!((N.mask >> (4 * j + k)) & 1u)) continue;
                    if (DET)
                        fix_red4(a.fix + (N.g00 + j * N.sj + k), v[nd * 4], v[nd * 4 + 1], v[nd * 4 + 2], v[nd * 4 + 3],
                                 sp.s, sm.s);
                    else
                        red_add4(a.grid + (N.g00 + j * N.sj + k), v[nd * 4], v[nd * 4 + 1], v[nd * 4 + 2], v[nd * 4 + 3]);
                }
            }
        }
    }
}

// P2G over warp items (one item per warp, persistent grid-stride)
template <bool GENERAL, int MODE, bool DET = false>
__global__ void __launch_bounds__(DMPM_P2G_THREADS, DMPM_SCATTER_MIN_BLOCKS) k_p2g_w(WArgs a) {
    const int nit = item_count(a);
    FixScale sp{1.f, 1.f}, sm{1.f, 1.f};
    if (DET) {
        sp = fix_scale(a.fixb + FIXB_MOMENTUM, a.n);
        sm = fix_scale(a.fixb + FIXB_MASS, a.n);
    }
    const FixTile none{nullptr, 0, {0, 0, 0}, 0};
    for (int item = first_warp(); item < nit; item = next_item<MODE>(item, nit))
        p2g_item<GENERAL, MODE, DET, false>(a, item, sp, sm, none);
}

// G_op in place: (p, m) -> (v, m), v = p/m + dt f where |m| > FLT_EPSILON, else 0
static __global__ void k_gop_inplace(node4<float>* grid, size_t G, float dt, float f0, float f1, float f2) {
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    node4<float> nd = grid[g];
    const float f[3] = {f0, f1, f2};
    float v[3];
    node_velocity(nd, dt, f, v);
    nd.x = v[0];
    nd.y = v[1];
    nd.z = v[2];
    grid[g] = nd;
}

// G2P + P_op_2: v' = sum w v_g;  C' = 3/dx^2 sum w v_g d^T;
// F' = (1 - s)(I + dt C')(F + dFc) + s F;  x' = x + dt v'
// G2P keeps 64 registers without spills, so four 256-thread CTAs reside per SM
#ifndef DMPM_G2P_CTAS
#define DMPM_G2P_CTAS 4
#endif
template <int MODE> __global__ void __launch_bounds__(256, 4) k_g2p_w(WArgs a) {
    const int nit = item_count(a);
    const size_t np = a.np, npl = a.npl, npn = a.npn;
    for (int item = first_warp(); item < nit; item = next_item<MODE>(item, nit)) {
        GridGeom geo;
        int goff;
        item_grid<MODE>(a, item, geo, goff);
        const ItemLane L = item_lane(a.items, item);
        float t[3];
        int base[3];
        load_x_base(a.st, npl, L.p, geo, t, base, a.xlo);
        LaneW w;
        float own1[3];
        lane_weights_k(t, geo, L.s, w, own1, false);
        // v = sum w v_g and C = sum w v_g d^T (scaled by 3/dx^2 at the end), with the
        // weight w = n0 n1[j] n2[k] and d = (d0, d1[j], d2[k]) factored per stencil row:
        // the node loop accumulates only the k-dependent sums, the row applies n0 n1[j]
        // and d1[j], and the d0 column is d0 v.
        float nd2[4];
#pragma unroll
        for (int k = 0; k < 4; k++) nd2[k] = w.n2[k] * w.d2[k];
        float V[3] = {0.f, 0.f, 0.f}, C1[3] = {0.f, 0.f, 0.f}, C2[3] = {0.f, 0.f, 0.f};
        // one stencil row j from its four node records
        auto row_sum = [&](int j, const node4<float> (&row)[4]) {
            float Vj[3] = {0.f, 0.f, 0.f}, Wj[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float vg[3] = {row[k].x, row[k].y, row[k].z};
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    Vj[r] += w.n2[k] * vg[r];
                    Wj[r] += nd2[k] * vg[r];
                }
            }
            float d1, n1, s1;
            row_weights(own1, j, d1, n1, s1);
            const float w01 = w.n0 * n1, w01d = w01 * d1;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                V[r] += w01 * Vj[r];
                C1[r] += w01d * Vj[r];
                C2[r] += w01 * Wj[r];
            }
        };
        // a uniform item stages its 64 stencil nodes in shared memory (stage_stencil);
        // otherwise each lane loads its slab's nodes, a row at a time (the row's four
        // records before any is used; nodes outside the grid read as zero)
        __shared__ node4<float> s_nodes[8][StageRecords<1>::value];
        if (DMPM_STAGE_NODES && warp_uniform_base(base)) {
            node4<float>* sw = s_nodes[threadIdx.x >> 5];
            stage_stencil<1>(a.grid, geo, goff, base, sw);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                node4<float> row[4];
#pragma unroll
                for (int k = 0; k < 4; k++) row[k] = sw[stage_index<1>(16 * L.s + 4 * j + k, 0)];
                row_sum(j, row);
            }
        } else {
            LaneNodes N = lane_nodes(geo, base, L.s);
            N.g00 += goff;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                node4<float> row[4];
#pragma unroll
                for (int k = 0; k < 4; k++)
                    row[k] = ((N.mask >> (4 * j + k)) & 1u) ? a.grid[N.g00 + j * N.sj + k]
                                                            : node4<float>{0.f, 0.f, 0.f, 0.f};
                row_sum(j, row);
            }
        }
        float acc[12];  // v (3), C (9) row-major
#pragma unroll
        for (int r = 0; r < 3; r++) {
            acc[r] = V[r];
            acc[3 + 3 * r] = w.d0 * V[r];
            acc[4 + 3 * r] = C1[r];
            acc[5 + 3 * r] = C2[r];
        }
        reduce_slabs<12>(acc);
        if (!L.valid) continue;
        const float dx = (float)geo.dx;
        const float k3 = 3.f / (dx * dx);
        const int p = L.p;
        m3<float> Cn;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) Cn.a[r][c] = k3 * acc[3 + 3 * r + c];
        // lane s = 0 stores x' and v', s = 1 C'; lanes s = 0, 2, 3 each one column
        // c of F' = (1-s)(I + dt C') Fe[:,c] + s F[:,c]
        bool finite = true;
        if (L.s == 0) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float xn = advance_x(a.st, a.st_next, npl, npn, p, c, a.dt, acc[c], a.xlo);
                a.st_next[(size_t)(PV + c) * npn + p] = acc[c];
                finite &= isfinite(xn);
            }
        }
        if (L.s == 1) {
            store_m3(a.st_next + (size_t)PC * npn, npn, p, Cn);
        } else {
            // column c of the strain: H' = (1 - s)(D + dt C' (I + D)) + s H,  D = H + dFc
            const int c = L.s == 0 ? 0 : L.s - 1;
            float Hc[3], Dc[3];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                Hc[r] = a.st[(size_t)(PF + r + 3 * c) * npl + p];
                Dc[r] = Hc[r] + a.dfc[(size_t)(r + 3 * c) * np + p];
            }
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const float t = Dc[r] + a.dt * (Cn.a[r][c] + (Cn.a[r][0] * Dc[0] + Cn.a[r][1] * Dc[1] + Cn.a[r][2] * Dc[2]));
                const float hn = (1.f - a.s) * t + a.s * Hc[r];
                a.st_next[(size_t)(PF + r + 3 * c) * npn + p] = hn;
                finite &= isfinite(hn);
            }
        }
        if (!finite) atomicOr(a.status, ST_NONFINITE_FWD);
    }
}

// ------------------------------------------------------------------ adjoint
// dLdv_next = dt dLdx' + dLdv';  dLdC_next = c dt dLdF' Fe^T + dLdC'
// dLdv_g += w dLdv_next + 3/dx^2 w dLdC_next (x_g - x_p)   (BackPropagation.cpp:14-44)
// The per-particle sources of the adjoint scatter: vn = dt dLdx' + dLdv' and
// Cn = cf dLdF' Fe^T + dLdC' (cf = (1 - s) dt exact, dt refcompat), from layer
// n + 1's adjoint and layer n's F + dFc.
template <bool EXACT>
__device__ __forceinline__ void adj_sources(const WArgs& a, int p, float vn[3], m3<float>& Cn) {
    const size_t np = a.np, npl = a.npl, npn = a.npn;
#pragma unroll
    for (int c = 0; c < 3; c++) vn[c] = a.dt * a.adj_next[(size_t)(PX + c) * npn + p] + a.adj_next[(size_t)(PV + c) * npn + p];
    const m3<float> Fe = fe_from_strain(load_m3(a.st + (size_t)PF * npl, npl, p), load_m3(a.dfc, np, p));
    const float cf = EXACT ? (1.f - a.s) * a.dt : a.dt;
    Cn = (cf * load_m3(a.adj_next + (size_t)PF * npn, npn, p)) * transpose(Fe) +
         load_m3(a.adj_next + (size_t)PC * npn, npn, p);
}

// Deterministic mode: the scatter's sources per particle into adjn (which the
// gather reads too) and their bound |vn + 3/dx^2 Cn d| with |d| < 2 dx into
// the adjoint bound slot, before the scatter adds anything.
template <bool EXACT> __global__ void __launch_bounds__(256) k_adj_sources(WArgs a) {
    const size_t np = a.np;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    float c = 0.f;
    if (p < a.n) {
        float vn[3];
        m3<float> Cn;
        adj_sources<EXACT>(a, p, vn, Cn);
#pragma unroll
        for (int r = 0; r < 3; r++) a.adjn[(size_t)r * np + p] = vn[r];
        store_m3(a.adjn + 3 * np, np, p, Cn);
        if (a.dbg_vnext) {
#pragma unroll
            for (int r = 0; r < 3; r++) a.dbg_vnext[(size_t)r * np + p] = vn[r];
        }
        if (a.dbg_Cnext) store_m3(a.dbg_Cnext, np, p, Cn);
        const float dx = (float)a.geo.dx, k3 = 3.f / (dx * dx);
#pragma unroll
        for (int r = 0; r < 3; r++)
            c = fmaxf(c, fabsf(vn[r]) + k3 * 2.f * dx * (fabsf(Cn.a[r][0]) + fabsf(Cn.a[r][1]) + fabsf(Cn.a[r][2])));
    }
    fix_bound(a.fixb + FIXB_ADJ, c * 1.001f);
}

// Warp items first, first + stride, ... below end of the adjoint scatter.
// DET: the sources come from k_adj_sources (adjn) and the node sums go to
// a.fix as integers (fixpoint.cuh) instead of float atomics into a.gadj; with a
// tile, those of an item whose stencil lies in it go to the tile's
// shared-memory integers.
template <bool EXACT, bool GENERAL, int MODE, bool DET, bool TILE>
__device__ __forceinline__ void adj_scatter_items(const WArgs& a, int first, int end, int stride, const FixScale& sa,
                                                  const FixTile& ft) {
    const size_t np = a.np, npl = a.npl;
    for (int item = first; item < end; item += stride) {
        GridGeom geo;
        int goff;
        item_grid<MODE>(a, item, geo, goff);
        const ItemLane L = item_lane(a.items, item);
        const int p = L.p;
        float t[3];
        int base[3];
        load_x_base(a.st, npl, p, geo, t, base, a.xlo);
        const bool uniform = !GENERAL && warp_uniform_base(base);
        const ScatterPerm P = scatter_perm();  // as in k_p2g_w
        LaneW w;
        float own1[3];
        lane_weights_k(t, geo, L.s, w, own1, false, P.kp);
        float vn[3];
        m3<float> Cn;
        if constexpr (DET) {
#pragma unroll
            for (int c = 0; c < 3; c++) vn[c] = a.adjn[(size_t)c * np + p];
            Cn = load_m3(a.adjn + 3 * np, np, p);
        } else {
            const size_t npn = a.npn;
#pragma unroll
            for (int c = 0; c < 3; c++)
                vn[c] = a.dt * a.adj_next[(size_t)(PX + c) * npn + p] + a.adj_next[(size_t)(PV + c) * npn + p];
            const m3<float> Fe = fe_from_strain(load_m3(a.st + (size_t)PF * npl, npl, p), load_m3(a.dfc, np, p));
            const float cf = EXACT ? (1.f - a.s) * a.dt : a.dt;
            Cn = (cf * load_m3(a.adj_next + (size_t)PF * npn, npn, p)) * transpose(Fe) +
                 load_m3(a.adj_next + (size_t)PC * npn, npn, p);
        }
        if (!DET && L.valid) {
            if (L.s == 0) {
#pragma unroll
                for (int c = 0; c < 3; c++) a.adjn[(size_t)c * np + p] = vn[c];
                if (a.dbg_vnext) {
#pragma unroll
                    for (int c = 0; c < 3; c++) a.dbg_vnext[(size_t)c * np + p] = vn[c];
                }
            } else if (L.s == 1) {
                store_m3(a.adjn + 3 * np, np, p, Cn);
                if (a.dbg_Cnext) store_m3(a.dbg_Cnext, np, p, Cn);
            }
        }
        const float dx = (float)geo.dx;
        const float k3 = 3.f / (dx * dx);
        float c0[3];
#pragma unroll
        for (int r = 0; r < 3; r++) c0[r] = k3 * Cn.a[r][0] * w.d0;
        LaneNodes N = lane_nodes(geo, base, L.s);
        N.g00 += goff;
        const int tile_l = TILE && uniform ? fix_tile_offset(ft, base) : -1;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            float v[24];  // 8 nodes x dLdv_g (3)
#pragma unroll
            for (int jj = 0; jj < 2; jj++) {
                float d1, n1, s1;
                row_weights(own1, 2 * half + (jj ^ P.jp), d1, n1, s1);
                float c1[3];
#pragma unroll
                for (int r = 0; r < 3; r++) c1[r] = c0[r] + k3 * Cn.a[r][1] * d1;
                const float w01 = L.valid ? w.n0 * n1 : 0.f;
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    const float wt = w01 * w.n2[kk];
                    const int o = (jj * 4 + kk) * 3;
#pragma unroll
                    for (int r = 0; r < 3; r++) v[o + r] = wt * (vn[r] + c1[r] + k3 * Cn.a[r][2] * w.d2[kk]);
                }
            }
            if (uniform) {
                reduce_scatter8<24>(v);
                const int j = 2 * half + P.jp, k = P.kp;
                if (((N.mask >> (4 * j + k)) & 1u) && (v[0] != 0.f || v[1] != 0.f || v[2] != 0.f)) {
                    if (TILE && tile_l >= 0)
                        fix_red4_tile(ft, tile_l + (L.s * ft.E + j) * ft.E + k, v[0], v[1], v[2], 0.f, sa.s, sa.s);
                    else if (DET) fix_red4(a.fix + (N.g00 + j * N.sj + k), v[0], v[1], v[2], 0.f, sa.s, sa.s);
                    else red_add4(a.gadj + (N.g00 + j * N.sj + k), v[0], v[1], v[2], 0.f);
                }
            } else if (L.valid) {
#pragma unroll
                for (int nd = 0; nd < 8; nd++) {
                    const int j = 2 * half + ((nd >> 2) ^ P.jp), k = (nd & 3) ^ P.kp;
                    if (!((N.mask >> (4 * j + k)) & 1u)) continue;
                    if (DET)
                        fix_red4(a.fix + (N.g00 + j * N.sj + k), v[nd * 3], v[nd * 3 + 1], v[nd * 3 + 2], 0.f, sa.s,
                                 sa.s);
                    else
                        red_add4(a.gadj + (N.g00 + j * N.sj + k), v[nd * 3], v[nd * 3 + 1], v[nd * 3 + 2], 0.f);
                }
            }
        }
    }
}

// adjoint scatter over warp items (one item per warp, persistent grid-stride)
template <bool EXACT, bool GENERAL, int MODE, bool DET = false>
__global__ void __launch_bounds__(DMPM_ADJ_SCATTER_THREADS, DMPM_ADJ_SCATTER_MIN_BLOCKS) k_adj_scatter_w(WArgs a) {
    const int nit = item_count(a);
    FixScale sa{1.f, 1.f};
    if (DET) sa = fix_scale(a.fixb + FIXB_ADJ, a.n);
    const FixTile none{nullptr, 0, {0, 0, 0}, 0};
    const int stride = MODE != ITEMS_PER_WARP ? (int)((gridDim.x * blockDim.x) >> 5) : nit;  // as next_item
    adj_scatter_items<EXACT, GENERAL, MODE, DET, false>(a, first_warp(), nit, stride, sa, none);
}

// adjoint G_op per node: (dLdp, dLdm) from dLdv and the layer's (v, m)
// The record pair (dLdp, dLdm), (v, m) of a node is stored contiguously (32 B)
// so the gather reads one sector per node.
template <bool EXACT>
__global__ void k_adj_gop_w(const node4<float>* __restrict__ grid, const node4<float>* __restrict__ gadj,
                            node4<float>* gadj2, size_t G, float dt, float f0, float f1, float f2) {
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const node4<float> nd = grid[g];
    const node4<float> dv = gadj[g];
    node4<float> o{0.f, 0.f, 0.f, 0.f};
    if (fabsf(nd.w) > (float)kFltEps) {
        float v[3] = {nd.x, nd.y, nd.z};
        if (EXACT) { v[0] -= dt * f0; v[1] -= dt * f1; v[2] -= dt * f2; }
        o.x = dv.x / nd.w;
        o.y = dv.y / nd.w;
        o.z = dv.z / nd.w;
        o.w = -1.f / nd.w * (v[0] * dv.x + v[1] * dv.y + v[2] * dv.z);
    }
    gadj2[2 * g] = o;
    gadj2[2 * g + 1] = nd;
}

// adjoint P2G gather: per particle, over its 64 nodes,
//   M += w d dLdp^T,  X += sigma (N'NN, NN'N, NNN'),  u += w dLdp,  z += w v_g
//   sigma = m dLdm + dLdp.(m v c_d + G d) + v_g.(dLdv_next + 3/dx^2 dLdC_next d)
// (the algebra of kernels.cuh:k_adj_gather); written to gath for k_adj_finalize.
// One warp item of the adjoint gather: the item's particles (lane L, stencil
// coordinates t, base) read their 64 stencil node pairs from sw, the item's
// staged copy, or from global memory when sw is null.
template <bool EXACT>
__device__ __forceinline__ void gather_item(const WArgs& a, const GridGeom& geo, int goff, const ItemLane& L,
                                            const float t[3], const int base[3], const node4<float>* sw) {
    const size_t np = a.np, npl = a.npl;
    const int p = L.p;
    LaneW w;
    float own1[3];
    lane_weights_k(t, geo, L.s, w, own1, true);
    const float mp = a.cst[(size_t)KM * np + p];
    const float cd = EXACT ? (1.f - a.dt * a.drag) : 1.f;
    const float dx = (float)geo.dx;
    const float k3 = 3.f / (dx * dx);
    float mvp[3], vn[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        mvp[c] = mp * a.st[(size_t)(PV + c) * npl + p] * cd;
        vn[c] = a.adjn[(size_t)c * np + p];
    }
    const m3<float> G = load_m3(a.G, npl, p);
    const m3<float> Cn = load_m3(a.adjn + 3 * np, np, p);
    // sigma's node-dependent pieces: h_g = mvp + G d,  e_g = vn + k3 Cn d
    float h0[3], e0[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        h0[r] = mvp[r] + G.a[r][0] * w.d0;
        e0[r] = vn[r] + k3 * Cn.a[r][0] * w.d0;
    }
    float acc[18];  // M (9, row-major: M[r][c] = sum w d_r dLdp_c), X (3), u (3), z (3)
#pragma unroll
    for (int i = 0; i < 18; i++) acc[i] = 0.f;
    // Factored sums: on this lane d0, n0 and s0 are constant and on a row d1, n1, s1, so
    //   M[0][c] = d0 u_c (formed after the loop),
    //   X0 = s0 sum_j n1 S_j,  X1 = n0 sum_j s1 S_j,  X2 = n0 sum_j n1 T_j,
    // with the row sums S_j = sum_k n2_k sigma, T_j = sum_k s2_k sigma.
    float S = 0.f, T = 0.f;
    // one node (j, k) of the lane's slab, with row j's axis-1 values d1, n1
    auto node = [&](const node4<float>& o, const node4<float>& vg, float d1, float n1, int k) {
        float h[3], e[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            h[r] = h0[r] + G.a[r][1] * d1 + G.a[r][2] * w.d2[k];
            e[r] = e0[r] + k3 * Cn.a[r][1] * d1 + k3 * Cn.a[r][2] * w.d2[k];
        }
        const float wt = (w.n0 * n1) * w.n2[k];
        const float sig = mp * o.w + o.x * h[0] + o.y * h[1] + o.z * h[2] + vg.x * e[0] + vg.y * e[1] + vg.z * e[2];
        S += w.n2[k] * sig;
        T += w.s2[k] * sig;
        const float wo[3] = {wt * o.x, wt * o.y, wt * o.z};
        acc[15] += wt * vg.x;
        acc[16] += wt * vg.y;
        acc[17] += wt * vg.z;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            acc[12 + c] += wo[c];
            acc[3 + c] += d1 * wo[c];
            acc[6 + c] += w.d2[k] * wo[c];
        }
    };
    auto end_row = [&](float n1, float s1) {
        acc[9] += n1 * S;
        acc[10] += s1 * S;
        acc[11] += n1 * T;
        S = 0.f;
        T = 0.f;
    };
    if (sw) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float d1, n1, s1;
            row_weights(own1, j, d1, n1, s1);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int n = 16 * L.s + 4 * j + k;
                node(sw[stage_index<2>(n, 0)], sw[stage_index<2>(n, 1)], d1, n1, k);
            }
            end_row(n1, s1);
        }
    } else {
        LaneNodes N = lane_nodes(geo, base, L.s);
        N.g00 += goff;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float d1, n1, s1;
            row_weights(own1, j, d1, n1, s1);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (!((N.mask >> (4 * j + k)) & 1u)) continue;
                const int g = N.g00 + j * N.sj + k;
                node(a.gadj2[2 * g], a.gadj2[2 * g + 1], d1, n1, k);
            }
            end_row(n1, s1);
        }
    }
    acc[9] *= w.s0;
    acc[10] *= w.n0;
    acc[11] *= w.n0;
#pragma unroll
    for (int c = 0; c < 3; c++) acc[c] = w.d0 * acc[12 + c];
    reduce_slabs<18>(acc);
    if (!L.valid) return;
    if (L.s == 0) {
#pragma unroll
        for (int i = 0; i < 9; i++) a.gath[(size_t)i * np + p] = acc[i];
    } else if (L.s == 1) {
#pragma unroll
        for (int i = 9; i < 18; i++) a.gath[(size_t)i * np + p] = acc[i];
    }
}

template <bool EXACT, int MODE>
__global__ void __launch_bounds__(DMPM_GATHER_THREADS, DMPM_GATHER_MIN_BLOCKS) k_adj_gather_w(WArgs a) {
    const int nit = item_count(a);
    const size_t npl = a.npl;
    __shared__ node4<float> s_rec[8][StageRecords<2>::value];
    for (int item = first_warp(); item < nit; item = next_item<MODE>(item, nit)) {
        GridGeom geo;
        int goff;
        item_grid<MODE>(a, item, geo, goff);
        const ItemLane L = item_lane(a.items, item);
        float t[3];
        int base[3];
        load_x_base(a.st, npl, L.p, geo, t, base, a.xlo);
        node4<float>* sw = nullptr;
        if (DMPM_STAGE_NODES && warp_uniform_base(base)) {
            sw = s_rec[threadIdx.x >> 5];
            stage_stencil<2>(a.gadj2, geo, goff, base, sw);
        }
        gather_item<EXACT>(a, geo, goff, L, t, base, sw);
    }
}

// ------------------------------------------------------------------ finalize
// per particle: P, polar factors and dP/dF in FP64, then the adjoint of layer n
//   dLdP = -3/dx^2 dt vol M^T Fe,  dLdF(stress) = -3/dx^2 dt vol M P,  dLdC = m M^T
//   dLdx = -X/dx - G^T u - 3/dx^2 dLdC_next^T z + dLdx',  dLdv = m (1 - dt drag) u
//   REFCOMPAT: dLdF = (1-s)T + s dLdF' + stress + T + dP:dLdP,  T = (I + dt C')^T dLdF'
//   EXACT:     dLdFe = (1-s)T + stress + dP:dLdP,  dLdF = dLdFe + s dLdF'
//
// Its inputs are 94 FP32 planes per particle (slots below) and, with tied
// controls, the 9 FP64 planes of the control-gradient accumulator.
enum : int {
    FS_GATH = 0,    // 18: M (9, row-major), X (3), u (3), z (3)
    FS_F = 18,      // 9: strain H = F - I of layer n
    FS_DFC = 27,    // 9: dFc
    FS_AUX = 36,    // 24: G (9), polar R (9), polar S (6)
    FS_CST = 60,    // 4: m, vol, lam, mu
    FS_CN = 64,     // 9: dLdC_next
    FS_AX = 73,     // 3: dLdx of layer n+1
    FS_AF = 76,     // 9: dLdF of layer n+1
    FS_CNEXT = 85,  // 9: C of layer n+1
    FS_COUNT = 94
};

// first element and stride of a slot's plane
__device__ __forceinline__ const float* fin_plane(const WArgs& a, int slot, size_t& stride) {
    if (slot < FS_F) { stride = a.np; return a.gath + (size_t)slot * a.np; }
    if (slot < FS_DFC) { stride = a.npl; return a.st + (size_t)(PF + slot - FS_F) * a.npl; }
    if (slot < FS_AUX) { stride = a.np; return a.dfc + (size_t)(slot - FS_DFC) * a.np; }
    if (slot < FS_CST) { stride = a.npl; return a.G + (size_t)(slot - FS_AUX) * a.npl; }
    if (slot < FS_CN) { stride = a.np; return a.cst + (size_t)(slot - FS_CST) * a.np; }
    if (slot < FS_AX) { stride = a.np; return a.adjn + (size_t)(3 + slot - FS_CN) * a.np; }
    if (slot < FS_AF) { stride = a.npn; return a.adj_next + (size_t)(PX + slot - FS_AX) * a.npn; }
    if (slot < FS_CNEXT) { stride = a.npn; return a.adj_next + (size_t)(PF + slot - FS_AF) * a.npn; }
    stride = a.npn;
    return a.st_next + (size_t)(PC + slot - FS_CNEXT) * a.npn;
}

// the finalize inputs of particle p, read from global memory
struct FinGlobal {
    const WArgs* a;
    int p;
    __device__ __forceinline__ float operator()(int slot) const {
        size_t st;
        return fin_plane(*a, slot, st)[p];
    }
    __device__ __forceinline__ double acc(int i) const { return a->ctrl_acc[(size_t)i * a->np + p]; }
};
// PART selects what one launch computes: 0 everything; FIN_STRESS the FP64 part
// (P, dP/dF:dLdP, dLdF, the control gradient); FIN_TRANSPORT the FP32 outputs
// dLdx, dLdv, dLdC, which need neither the polar factors nor dLdF.
enum : int { FIN_ALL = 0, FIN_STRESS = 1, FIN_TRANSPORT = 2 };
template <bool EXACT, class In, int PART = FIN_ALL>
__device__ __forceinline__ void finalize_particle(const WArgs& a, int p, const In& in) {
    constexpr bool kStress = PART != FIN_TRANSPORT, kTransport = PART != FIN_STRESS;
    const size_t np = a.np, npl = a.npl;
    auto mat = [&](int slot) {  // 9 column-major planes -> m3
        m3<float> m;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) m.a[r][c] = in(slot + r + 3 * c);
        return m;
    };
    m3<float> M;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) M.a[r][c] = in(FS_GATH + 3 * r + c);
    const float dx = (float)a.geo.dx;
    const float k3 = 3.f / (dx * dx);
    // dLdx = -X/dx - G^T u - 3/dx^2 dLdC_next^T z + dLdx',  dLdv = m (1 - dt drag) u,  dLdC = m M^T
    auto transport = [&]() {
        const float mp = in(FS_CST + KM);
        const m3<float> G = mat(FS_AUX);
        const m3<float> Cn = mat(FS_CN);
        float u[3], z[3], gtu[3], ctz[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            u[c] = in(FS_GATH + 12 + c);
            z[c] = in(FS_GATH + 15 + c);
        }
        mtv(G, u, gtu);
        mtv(Cn, z, ctz);
        float ax0 = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float X = in(FS_GATH + 9 + c);
            const float ax = -X / dx - gtu[c] - k3 * ctz[c] + in(FS_AX + c);
            if (c == 0) ax0 = ax;
            a.adj[(size_t)(PX + c) * npl + p] = ax;
            a.adj[(size_t)(PV + c) * npl + p] = mp * (1.f - a.dt * a.drag) * u[c];
        }
        store_m3(a.adj + (size_t)PC * npl, npl, p, mp * transpose(M));
        return ax0;
    };
    if constexpr (!kStress) {
        if (!isfinite(transport())) atomicOr(a.status, ST_NONFINITE_ADJ);
        return;
    }
    const m3<float> H = mat(FS_F), dfc = mat(FS_DFC);
    const m3<float> Fe = fe_from_strain(H, dfc);
    const m3<double> Fed = fe_from_strain_d(H, dfc);
    // polar factors computed in FP64 by k_stress for this layer
    const m3<double> Rd = m3_cast<double>(mat(FS_AUX + 9));
    m3<double> Sd;
    Sd.a[0][0] = in(FS_AUX + 18);
    Sd.a[0][1] = Sd.a[1][0] = in(FS_AUX + 19);
    Sd.a[0][2] = Sd.a[2][0] = in(FS_AUX + 20);
    Sd.a[1][1] = in(FS_AUX + 21);
    Sd.a[1][2] = Sd.a[2][1] = in(FS_AUX + 22);
    Sd.a[2][2] = in(FS_AUX + 23);
    const double lam = (double)in(FS_CST + KLAM), mu = (double)in(FS_CST + KMU);
    const m3<float> P = m3_cast<float>(pk_from_polar(Fed, Rd, lam, mu));
    const float vol = in(FS_CST + KVOL);
    const float kk = -k3 * a.dt * vol;
    const m3<float> dLdP = kk * mtm(M, Fe);
    const m3<float> dFstress = kk * (M * P);
    float ax0 = 0.f;
    if constexpr (kTransport) ax0 = transport();
    const m3<float> Cnext = mat(FS_CNEXT);
    const m3<float> dFn = mat(FS_AF);
    const m3<float> Tr = mtm(m3_eye<float>() + a.dt * Cnext, dFn);
    const m3<float> d2 = m3_cast<float>(d2_mult_from_polar<EXACT>(Fed, Rd, Sd, lam, mu, m3_cast<double>(dLdP)));
    m3<float> dLdF, dLdFe;
    if (EXACT) {
        dLdFe = (1.f - a.s) * Tr + dFstress + d2;
        dLdF = dLdFe + a.s * dFn;
    } else {
        dLdF = ((1.f - a.s) * Tr + a.s * dFn) + dFstress + Tr + d2;
        dLdFe = dLdF;
    }
    store_m3(a.adj + (size_t)PF * npl, npl, p, dLdF);
    if (a.ctrl_grad) store_m3(a.ctrl_grad, np, p, dLdFe);
    if (a.ctrl_acc) {
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int r = 0; r < 3; r++)
                a.ctrl_acc[(size_t)(r + 3 * c) * np + p] = in.acc(r + 3 * c) + (double)dLdFe.a[r][c];
    }
    if (a.dbg_dLdP) store_m3(a.dbg_dLdP, np, p, dLdP);
    if (!isfinite(dLdF.a[0][0] + dLdF.a[1][1] + dLdF.a[2][2] + ax0)) atomicOr(a.status, ST_NONFINITE_ADJ);
}

// one thread per particle, inputs read from global memory (the REFCOMPAT
// variant, with its finite-difference dJFit, keeps the compiler's own
// register budget)
template <bool EXACT, int PART = FIN_ALL>
__global__ void __launch_bounds__(128, !EXACT ? 1 : PART == FIN_STRESS ? DMPM_FINALIZE_STRESS_MIN_BLOCKS
                                                                         : DMPM_FINALIZE_MIN_BLOCKS)
    k_adj_finalize(WArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < a.n) finalize_particle<EXACT, FinGlobal, PART>(a, p, FinGlobal{&a, p});
}
// the transport part alone: few registers, many resident warps
static __global__ void __launch_bounds__(256) k_adj_finalize_transport(WArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < a.n) finalize_particle<true, FinGlobal, FIN_TRANSPORT>(a, p, FinGlobal{&a, p});
}

// host side: one thread per particle (a variant that first staged each
// block's 94 input planes in shared memory with cp.async.bulk copies measured
// 7 % slower on the 64^3, 267k-particle workload -- 57 KB of shared memory
// per 128 particles cut residency to 12 warps per SM, and the kernel is bound
// by its dependent FP64 chains, not by load latency -- so it was dropped)
inline void launch_finalize(const WArgs& a, bool exact, cudaStream_t st) {
    if (a.n <= 0) return;
    const unsigned b = (unsigned)((a.n + 127) / 128);
    if (exact) k_adj_finalize<true><<<b, 128, 0, st>>>(a);
    else k_adj_finalize<false><<<b, 128, 0, st>>>(a);
}
// The single-scene engine runs the finalize as the two launches below, the
// transport part on a second stream beside the FP64 part: the FP64 part keeps
// 128 registers per thread and 16 warps per SM, and the transport part's warps
// (60 registers) fill the rest of the SMs meanwhile (60.0 against 60.9 ms per
// gradient evaluation on the 64^3, 267k-particle workload).  0 runs the
// single kernel.
#ifndef DMPM_SPLIT_FINALIZE
#define DMPM_SPLIT_FINALIZE 1
#endif
// one part of the finalize (FIN_STRESS or FIN_TRANSPORT) on st
inline void launch_finalize_part(const WArgs& a, bool exact, int part, cudaStream_t st) {
    if (a.n <= 0) return;
    if (part == FIN_TRANSPORT) {
        k_adj_finalize_transport<<<(unsigned)((a.n + 255) / 256), 256, 0, st>>>(a);
        return;
    }
    const unsigned b = (unsigned)((a.n + 127) / 128);
    if (exact) k_adj_finalize<true, FIN_STRESS><<<b, 128, 0, st>>>(a);
    else k_adj_finalize<false, FIN_STRESS><<<b, 128, 0, st>>>(a);
}
// the same work as two launches: the FP64 part on st, the transport part on side
inline void launch_finalize_split(const WArgs& a, bool exact, cudaStream_t st, cudaStream_t side) {
    launch_finalize_part(a, exact, FIN_TRANSPORT, side);
    launch_finalize_part(a, exact, FIN_STRESS, st);
}

}  // namespace dmpm
