// kernels_brick.cuh -- FP32 path stencil kernels over cell bricks.
//
// The cell sort orders particles brick-major (sort.cuh), so the particles of a
// unit -- a brick of 4 x 4 x 4 cells (B = 4) or one 2 x 2 x 2 octant of a
// brick (B = 2) -- are one contiguous run of the sorted order.  Every stencil
// of a particle whose cell lies in the unit falls inside the unit's node tile
// of (B + 3)^3 nodes (stencil bases c - 1 .. c + B - 2 plus 3).  G2P, which
// only reads the grid, runs over units: a CTA takes a unit, stages its node
// tile in shared memory once, and each thread handles one particle of the unit,
// all 64 stencil nodes of it, reading the tile (the particles of a warp share a
// cell most of the time, so the reads are broadcasts).  On the 64^3,
// 267k-particle workload this takes 36.7 us per step against 48.1 us for the
// warp-item G2P; at 8 particles per cell, 21.5 against 22.2 us.  The other
// stencil kernels stay warp-item kernels (kernels_warp.cuh), which measured
// faster: the adjoint gather over brick tiles took 95-115 us against 79 us
// (its 18 sums per particle need 128-170 registers per thread, so few warps
// reside) -- and so did the warp-item gather reading a per-CTA octant tile
// instead of staging each item's stencil (101 against 79.5 us: the CTA-wide
// barriers around each octant's staging idle its warps) -- and P2G and the
// adjoint scatter adding into shared tiles with
// shared-memory atomics took 3-4x longer than the warp's butterfly reduction
// followed by one vector red.global.add per node.
// A particle that has left the unit since the sort (the sort runs every few
// steps) is handled by the same code with its nodes read from global memory.
// The G2P thread also forms the next step's stress stage (the FP64 polar
// decomposition, P and G of layer n + 1) from the strain and C it has just
// written, so the forward step after it skips the stress kernel: 62.3 against
// 36.7 + 30.0 us per step on the 64^3, 267k-particle workload.
//
// Math per stage is that of kernels.cuh (which cites the reference) and of the
// warp-item kernels in kernels_warp.cuh, summed in a different order.
#pragma once
#include "kernels_warp.cuh"

namespace dmpm {

#ifndef DMPM_BRICK_THREADS
#define DMPM_BRICK_THREADS 128
#endif
// minimum resident CTAs per SM (the register cap the compiler works to)
#ifndef DMPM_BRICK_G2P_MINB
#define DMPM_BRICK_G2P_MINB 4
#endif

template <int B> struct BrickShape {
    static constexpr int shift = B == 4 ? 6 : 3;  // key >> shift names the unit
    static constexpr int E = B + 3;               // tile nodes per axis
    static constexpr int NT = E * E * E;
};

// Tile origin (stencil base of the unit's first cell, c - 5 in key coordinates)
__device__ __forceinline__ void unit_origin(uint32_t ukey, int shift, const GridGeom& g, int o[3]) {
    int c[3];
    unit_first_cell(ukey, shift, g.dim, c);
#pragma unroll
    for (int a = 0; a < 3; a++) o[a] = c[a] - 5;
}

// Per-axis stencil offsets d = x_g - x, weights N(d / dx) and slopes of the
// four nodes k = 0..3 of the stencil, from the lattice coordinate t of the
// particle (load_x_base): d = (k - t) dx.
__device__ __forceinline__ void axis_stencil(float t, float dx, float n[4], float d[4], float* s) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float q = (float)k - t;
        d[k] = q * dx;
        n[k] = bsp(q);
        if (s) s[k] = bsp_slope(q);
    }
}

// Offset, weight and slope of stencil node k on one axis -- the slab and row
// loops are not unrolled, so these come from t instead of per-node arrays.
struct Axis0 {
    float t, dx;
    __device__ __forceinline__ void operator()(int k, float& n, float& d, float* s) const {
        const float q = (float)k - t;
        d = q * dx;
        n = bsp(q);
        if (s) *s = bsp_slope(q);
    }
};

// Node record fetch: from the unit's shared tile, or from global memory (zeros
// outside the grid).  (i, j, k) are stencil offsets from the particle's base.
template <int B, int R> struct TileFetch {
    const node4<float>* tile;  // R records per node, node-major
    int l0, l1, l2;            // particle base relative to the tile origin
    __device__ __forceinline__ node4<float> operator()(int i, int j, int k, int r) const {
        constexpr int E = BrickShape<B>::E;
        return tile[R * (((l0 + i) * E + (l1 + j)) * E + (l2 + k)) + r];
    }
};
template <int R> struct GlobalFetch {
    const node4<float>* grid;
    GridGeom g;
    int goff;
    int b0, b1, b2;  // particle base
    __device__ __forceinline__ node4<float> operator()(int i, int j, int k, int r) const {
        const int gi = b0 + i, gj = b1 + j, gk = b2 + k;
        if ((unsigned)gi < (unsigned)g.dim[0] && (unsigned)gj < (unsigned)g.dim[1] && (unsigned)gk < (unsigned)g.dim[2])
            return grid[(size_t)R * ((size_t)goff + ((size_t)gi * g.dim[1] + gj) * g.dim[2] + gk) + r];
        return node4<float>{0.f, 0.f, 0.f, 0.f};
    }
};

// Stage the unit's tile: R consecutive records per node from src (zeros
// outside the grid).  Every thread of the block calls it.
template <int B, int R>
__device__ __forceinline__ void stage_tile(const node4<float>* __restrict__ src, const GridGeom& g, int goff,
                                           const int o[3], node4<float>* tile) {
    constexpr int E = BrickShape<B>::E, NT = BrickShape<B>::NT;
    for (int q = threadIdx.x; q < NT * R; q += blockDim.x) {
        const int nd = q / R, r = q - nd * R;
        const int i = nd / (E * E), j = (nd / E) % E, k = nd % E;
        const int gi = o[0] + i, gj = o[1] + j, gk = o[2] + k;
        const bool in = (unsigned)gi < (unsigned)g.dim[0] && (unsigned)gj < (unsigned)g.dim[1] &&
                        (unsigned)gk < (unsigned)g.dim[2];
        tile[q] = in ? src[(size_t)R * ((size_t)goff + ((size_t)gi * g.dim[1] + gj) * g.dim[2] + gk) + r]
                     : node4<float>{0.f, 0.f, 0.f, 0.f};
    }
}

// is the particle's stencil inside the unit's tile?
template <int B> __device__ __forceinline__ bool in_unit(const int base[3], const int o[3], int l[3]) {
    bool in = true;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        l[a] = base[a] - o[a];
        in &= (unsigned)l[a] < (unsigned)B;
    }
    return in;
}

// ------------------------------------------------------------------ G2P + P_op_2
// v' = sum w v_g;  C' = 3/dx^2 sum w v_g d^T;  F' = (1 - s)(I + dt C')(F + dFc) + s F;  x' = x + dt v'
template <class Fetch>
__device__ __forceinline__ void g2p_sums(const Fetch& f, const Axis0& ax0, const float n1[4], const float d1[4],
                                         const float n2[4], const float d2[4], float V[3], float Cm[3][3]) {
    float nd2[4];
#pragma unroll
    for (int k = 0; k < 4; k++) nd2[k] = n2[k] * d2[k];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        V[r] = 0.f;
        Cm[r][0] = Cm[r][1] = Cm[r][2] = 0.f;
    }
#pragma unroll 1
    for (int i = 0; i < 4; i++) {
        float n0, d0;
        ax0(i, n0, d0, nullptr);
        float Vi[3] = {0.f, 0.f, 0.f}, C1i[3] = {0.f, 0.f, 0.f}, C2i[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float Vj[3] = {0.f, 0.f, 0.f}, Wj[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const node4<float> g = f(i, j, k, 0);
                const float vg[3] = {g.x, g.y, g.z};
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    Vj[r] += n2[k] * vg[r];
                    Wj[r] += nd2[k] * vg[r];
                }
            }
            const float n1d1 = n1[j] * d1[j];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                Vi[r] += n1[j] * Vj[r];
                C1i[r] += n1d1 * Vj[r];
                C2i[r] += n1[j] * Wj[r];
            }
        }
        const float n0d0 = n0 * d0;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            V[r] += n0 * Vi[r];
            Cm[r][0] += n0d0 * Vi[r];
            Cm[r][1] += n0 * C1i[r];
            Cm[r][2] += n0 * C2i[r];
        }
    }
}

// STRESS: also the next step's stress stage for each particle, from the strain
// and C just formed (stress_particle, the arithmetic of k_stress), into
// a.G_next -- one pass over the particles fewer per step.
template <int B, bool STRESS = false>
__global__ void __launch_bounds__(DMPM_BRICK_THREADS, DMPM_BRICK_G2P_MINB) k_g2p_b(WArgs a) {
    using S = BrickShape<B>;
    __shared__ node4<float> tile[S::NT];
    const int nun = (int)*a.n_units_dev;
    const size_t np = a.np, npl = a.npl, npn = a.npn;
    const GridGeom geo = a.geo;
    const float dx = (float)geo.dx, k3 = 3.f / (dx * dx);
    for (int u = blockIdx.x; u < nun; u += gridDim.x) {
        int o[3];
        unit_origin(a.unit_key[u], S::shift, geo, o);
        const uint32_t q0 = a.unit_start[u], q1 = a.unit_start[u + 1];
        __syncthreads();  // the previous unit's readers are done with the tile
        stage_tile<B, 1>(a.grid, geo, 0, o, tile);
        __syncthreads();
        for (uint32_t q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
            const int p = (int)a.items.order[q];
            float t[3];
            int base[3];
            double xd[3];
            load_x_base(a.st, npl, p, geo, t, base, a.xlo, xd);
            float n[3][4], d[3][4];
#pragma unroll
            for (int c = 1; c < 3; c++) axis_stencil(t[c], dx, n[c], d[c], nullptr);
            const Axis0 ax0{t[0], dx};
            float V[3], Cm[3][3];
            int l[3];
            if (in_unit<B>(base, o, l))
                g2p_sums(TileFetch<B, 1>{tile, l[0], l[1], l[2]}, ax0, n[1], d[1], n[2], d[2], V, Cm);
            else
                g2p_sums(GlobalFetch<1>{a.grid, geo, 0, base[0], base[1], base[2]}, ax0, n[1], d[1], n[2], d[2], V,
                         Cm);
            m3<float> Cn;
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) Cn.a[r][c] = k3 * Cm[r][c];
            bool finite = true;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float xn = store_x(a.st_next, npn, p, c, xd[c], a.dt, V[c], a.xlo);
                a.st_next[(size_t)(PV + c) * npn + p] = V[c];
                finite &= isfinite(xn);
            }
            store_m3(a.st_next + (size_t)PC * npn, npn, p, Cn);
            // strain update H' = (1 - s)(D + dt C' (I + D)) + s H,  D = H + dFc
            const m3<float> H = load_m3(a.st + (size_t)PF * npl, npl, p);
            const m3<float> D = H + load_m3(a.dfc, np, p);
            m3<float> Hn;
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    const float t = D.a[r][c] + a.dt * (Cn.a[r][c] + (Cn.a[r][0] * D.a[0][c] + Cn.a[r][1] * D.a[1][c] +
                                                                       Cn.a[r][2] * D.a[2][c]));
                    const float hn = (1.f - a.s) * t + a.s * H.a[r][c];
                    a.st_next[(size_t)(PF + r + 3 * c) * npn + p] = hn;
                    Hn.a[r][c] = hn;
                    finite &= isfinite(hn);
                }
            if (!finite) atomicOr(a.status, ST_NONFINITE_FWD);
            if constexpr (STRESS)
                stress_particle(a, p, Hn, load_m3(a.dfc_next, np, p), [&]() { return Cn; }, a.G_next, npn, a.P_next);
        }
    }
}

// ------------------------------------------------------------------ deterministic P2G / adjoint scatter
// The deterministic mode's integer node sums (fixpoint.cuh) over units: a CTA
// takes a unit, its warps take the unit's warp items, and each item whose
// stencil lies in the unit's node tile adds its (reduce-scattered) node sums to
// the tile's shared-memory integers; the tile is then added to the global
// integer sums, one 64-bit atomic per nonzero value.  Integer adds in any order
// give the same sums, so the result is that of k_p2g_w / k_adj_scatter_w with
// DET, with about (B + 3)^3 global atomics per unit instead of 64 per item and
// node value.  Items that are not uniform or have left the unit add to global
// memory directly.
template <int B> __device__ __forceinline__ void fix_tile_flush(const FixTile& ft, const GridGeom& g, fix4* dst) {
    constexpr int E = BrickShape<B>::E, NT = BrickShape<B>::NT;
    for (int q = threadIdx.x; q < NT; q += blockDim.x) {
        const fix4 t{ft.t[q], ft.t[NT + q], ft.t[2 * NT + q], ft.t[3 * NT + q]};
        if ((t.x | t.y | t.z | t.w) == 0) continue;
        const int i = q / (E * E), j = (q / E) % E, k = q % E;
        const int gi = ft.o[0] + i, gj = ft.o[1] + j, gk = ft.o[2] + k;
        if (!((unsigned)gi < (unsigned)g.dim[0] && (unsigned)gj < (unsigned)g.dim[1] && (unsigned)gk < (unsigned)g.dim[2]))
            continue;  // nothing is added there: items skip nodes outside the grid
        fix4* p = dst + ((size_t)gi * g.dim[1] + gj) * g.dim[2] + gk;
        fix_red(&p->x, t.x);
        fix_red(&p->y, t.y);
        fix_red(&p->z, t.z);
        fix_red(&p->w, t.w);
    }
}

template <int B>
__device__ __forceinline__ void fix_tile_begin(FixTile& ft, long long* tile, uint32_t ukey, const GridGeom& g) {
    constexpr int NT = BrickShape<B>::NT;
    unit_origin(ukey, BrickShape<B>::shift, g, ft.o);
    ft.t = tile;
    ft.nt = NT;
    ft.E = BrickShape<B>::E;
    __syncthreads();  // the previous unit's flush has read the tile
    for (int q = threadIdx.x; q < 4 * NT; q += blockDim.x) tile[q] = 0;
    __syncthreads();
}

// resident CTAs per SM the compiler budgets registers for (6: 80 registers;
// measured per step on the 64^3, 267k-particle workload: P2G 105.6 us at 6,
// 110.0 at 8 (64 registers, spills), 116 at the compiler's own choice of 95
// registers; the scatter 104.2 / 106.3 / 118)
#ifndef DMPM_FIX_P2G_MINB
#define DMPM_FIX_P2G_MINB 6
#endif
#ifndef DMPM_FIX_SCATTER_MINB
#define DMPM_FIX_SCATTER_MINB 6
#endif
template <int B, bool GENERAL>
__global__ void __launch_bounds__(DMPM_BRICK_THREADS, DMPM_FIX_P2G_MINB) k_p2g_fix_b(WArgs a) {
    __shared__ long long tile[4 * BrickShape<B>::NT];
    const int nun = (int)*a.n_units_dev;
    const FixScale sp = fix_scale(a.fixb + FIXB_MOMENTUM, a.n), sm = fix_scale(a.fixb + FIXB_MASS, a.n);
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int u = blockIdx.x; u < nun; u += gridDim.x) {
        FixTile ft;
        fix_tile_begin<B>(ft, tile, a.unit_key[u], a.geo);
        for (uint32_t it = a.unit_item[u] + warp; it < a.unit_item[u + 1]; it += nw)
            p2g_item<GENERAL, ITEMS_PERSISTENT, true, true>(a, (int)it, sp, sm, ft);
        __syncthreads();
        fix_tile_flush<B>(ft, a.geo, a.fix);
    }
}

template <int B, bool EXACT, bool GENERAL>
__global__ void __launch_bounds__(DMPM_BRICK_THREADS, DMPM_FIX_SCATTER_MINB) k_adj_scatter_fix_b(WArgs a) {
    __shared__ long long tile[4 * BrickShape<B>::NT];
    const int nun = (int)*a.n_units_dev;
    const FixScale sa = fix_scale(a.fixb + FIXB_ADJ, a.n);
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int u = blockIdx.x; u < nun; u += gridDim.x) {
        FixTile ft;
        fix_tile_begin<B>(ft, tile, a.unit_key[u], a.geo);
        adj_scatter_items<EXACT, GENERAL, ITEMS_PERSISTENT, true, true>(a, (int)a.unit_item[u] + warp,
                                                                        (int)a.unit_item[u + 1], nw, sa, ft);
        __syncthreads();
        fix_tile_flush<B>(ft, a.geo, a.fix);
    }
}

}  // namespace dmpm
