// kernels.cuh -- the MLS-MPM forward step, end-layer mass loss and adjoint
// step as sm_100a kernels.
//
// Data layout in HBM (all per-particle arrays are SoA "planes" of stride np):
//   layer state   T[24][np]: x(0..2) v(3..5) F(6..14) C(15..23)
//   adjoint state T[24][np]: dLdx dLdv dLdF dLdC, same plane layout
//   constants     T[4][np]:  m vol lam mu
//   controls      T[9][np]:  dFc (one array per layer, or one tied array)
//   3x3 matrices use column-major plane numbering: element (r, c) is plane r + 3c
//   grid          node4<T>[G]: (p.x, p.y, p.z, m), node g = (i*dim_y + j)*dim_z + k
// The stencil of a particle is the 4x4x4 node block at floor((x-min)/dx) - 1
// (reference: ForwardSimulation.cpp:17-36); nodes outside the grid are skipped.
//
// Two execution strategies share the arithmetic:
//   TILED (FP32 path): each CTA takes a contiguous chunk of particles, reduces
//     the bounding box of their stencils and, when it fits the shared-memory
//     capacity, scatters into / gathers from a shared-memory node tile; tiles
//     are flushed with one vector red.global.add per touched node.  Chunks whose
//     box does not fit use the global path.
//   plain (FP64 path): one thread per particle, global atomics and gathers,
//     one kernel per reference stage.
#pragma once
#include <cstdint>
#include "elasticity.cuh"

namespace dmpm {

enum : int { PX = 0, PV = 3, PF = 6, PC = 15, NSTATE = 24 };
// State planes of the FP32 engines: the 24 above plus the low parts of the
// positions (compensated positions, below)
enum : int { PXL = NSTATE, NSTATE_X = NSTATE + 3 };
enum : int { KM = 0, KVOL = 1, KLAM = 2, KMU = 3, NCONST = 4 };
enum : unsigned { ST_NONFINITE_FWD = 1u, ST_NONFINITE_ADJ = 2u, ST_NONFINITE_LOSS = 4u };

template <class T> struct alignas(4 * sizeof(T)) node4 { T x, y, z, w; };

struct GridGeom {
    int dim[3];
    double dx;
    double mn[3];
};

// Compensated positions.  The FP32 engines (single scene and batch) keep each
// position coordinate as two floats, x = hi + lo: hi in plane PX + c, lo (the float
// nearest x - hi) in plane PXL + c, so a position carries about 48 bits instead
// of float32's 24.  A stencil is formed from the lattice coordinate r =
// (x - mn) / dx, taken in FP64 once per particle: base = floor(r) - 1 and
// t = r - base, rounded to float.  For a particle inside the grid t lies in
// [1, 2), so the node offsets q = s - t (s = 0..3) are exact in float and a
// particle's weights are set to ~1e-7 of a cell, where the float position
// (x - mn) / dx of a particle half a unit from the origin of a 64^3 grid is
// rounded to ~4e-6 of a cell.  With xlo = 0 (the mass rasters of target
// samples, which are plain float positions) lo is taken as 0.
template <class T> __device__ __forceinline__ double load_xd(const T* st, size_t np, int p, int c, int xlo) {
    const double h = (double)st[(size_t)(PX + c) * np + p];
    return xlo ? h + (double)st[(size_t)(PXL + c) * np + p] : h;
}
// stencil base (stencil_base's clamp) and lattice coordinate t of one axis
template <class T> __device__ __forceinline__ T stencil_coord(double x, double mn, double idx, int dim, int& base) {
    const double r = (x - mn) * idx;
    base = stencil_base_lattice<double>(r, dim);
    return (T)(r - (double)base);
}
// one axis of a particle's stencil for the one-thread-per-particle kernels:
// with xlo, base and weights from the compensated position; without, from the
// stored position as the reference forms them (the FP64 path)
template <class T>
__device__ __forceinline__ void particle_axis(const T* st, size_t np, int p, int c, int xlo, const GridGeom& g,
                                              int& base, axis_w<T>& w, bool slopes) {
    if (xlo) {
        const T t = stencil_coord<T>(load_xd(st, np, p, c, 1), g.mn[c], 1.0 / g.dx, g.dim[c], base);
        axis_weights_lattice<T>(t, (T)g.dx, w, slopes);
    } else {
        const T x = st[(size_t)(PX + c) * np + p];
        base = stencil_base<T>(x - (T)g.mn[c], (T)g.dx, g.dim[c]);
        axis_weights<T>(x, (T)g.mn[c], (T)g.dx, base, w, slopes);
    }
}

template <class T> DMPM_HD m3<T> load_m3(const T* base, size_t np, int i) {
    m3<T> r;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int rr = 0; rr < 3; rr++) r.a[rr][c] = base[(size_t)(rr + 3 * c) * np + i];
    return r;
}
template <class T> DMPM_HD void store_m3(T* base, size_t np, int i, const m3<T>& m) {
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int rr = 0; rr < 3; rr++) base[(size_t)(rr + 3 * c) * np + i] = m.a[rr][c];
}

template <class T> __device__ __forceinline__ T pick4(const T (&a)[4], int k) {
    T r = a[0];
    r = (k == 1) ? a[1] : r;
    r = (k == 2) ? a[2] : r;
    r = (k == 3) ? a[3] : r;
    return r;
}

// ------------------------------------------------------------------ tiles
struct TileBox {
    int o[3], e[3], n;
    bool ok;
};

// Bounding box of the stencils of this CTA's particles.  Every thread of the
// block must call it.
__device__ __forceinline__ TileBox block_tile_box(bool valid, const int base[3], int cap) {
    __shared__ int s_red[6][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int v[6];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        v[a] = valid ? base[a] : 0x3fffffff;
        v[3 + a] = valid ? base[a] : -0x3fffffff;
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        v[a] = __reduce_min_sync(0xffffffffu, v[a]);
        v[3 + a] = __reduce_max_sync(0xffffffffu, v[3 + a]);
    }
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 6; a++) s_red[a][warp] = v[a];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            int mn = lane < nw ? s_red[a][lane] : 0x3fffffff;
            int mx = lane < nw ? s_red[3 + a][lane] : -0x3fffffff;
            mn = __reduce_min_sync(0xffffffffu, mn);
            mx = __reduce_max_sync(0xffffffffu, mx);
            if (lane == 0) { s_red[a][0] = mn; s_red[3 + a][0] = mx; }
        }
    }
    __syncthreads();
    TileBox t;
    long long n = 1;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        t.o[a] = s_red[a][0];
        int ext = s_red[3 + a][0] - s_red[a][0] + 4;
        if (ext < 4) ext = 4;  // no valid particle: empty box
        t.e[a] = ext;
        n *= ext;
    }
    t.ok = (s_red[0][0] <= s_red[3][0]) && n <= (long long)cap;
    t.n = t.ok ? (int)n : 0;
    __syncthreads();  // s_red is reused by the next call
    return t;
}

__device__ __forceinline__ int tile_index(const TileBox& t, int i, int j, int k) {
    return ((i - t.o[0]) * t.e[1] + (j - t.o[1])) * t.e[2] + (k - t.o[2]);
}

__device__ __forceinline__ void red_add4(node4<float>* p, float a, float b, float c, float d) {
    atomicAdd(reinterpret_cast<float4*>(p), make_float4(a, b, c, d));
}
__device__ __forceinline__ void red_add4(node4<double>* p, double a, double b, double c, double d) {
    atomicAdd(&p->x, a);
    atomicAdd(&p->y, b);
    atomicAdd(&p->z, c);
    atomicAdd(&p->w, d);
}

// ------------------------------------------------------------------ args
template <class T> struct FwdArgs {
    int n;
    size_t np;
    GridGeom geo;
    T dt, drag, s, fext[3];
    const T* st;        // layer n state
    T* st_next;         // layer n+1 state
    const T* cst;       // constants
    const T* dfc;       // dFc of layer n
    node4<T>* grid;     // layer n grid (p, m)
    T* gridv;           // plain path: node velocities [3][G] (G_op output)
    T* P;               // [9][np] stress of layer n (plain path, or debug copy)
    int tile_cap;
    unsigned* status;
    int strain;         // the F planes hold H = F - I (the FP32 path's layer storage)
};

// ------------------------------------------------------------------ P_op_1
// P = PK(F + dFc) with the polar decomposition in double (ForwardSimulation.cpp:6-9).
template <class T> __global__ void k_p_op1(FwdArgs<T> a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    m3<double> Fe = m3_cast<double>(load_m3(a.st + (size_t)PF * a.np, a.np, p)) + m3_cast<double>(load_m3(a.dfc, a.np, p));
    if (a.strain) Fe = Fe + m3_eye<double>();  // the F planes hold H = F - I
    const m3<double> P = pk_stress<double>(Fe, (double)a.cst[(size_t)KLAM * a.np + p], (double)a.cst[(size_t)KMU * a.np + p]);
    store_m3(a.P, a.np, p, m3_cast<T>(P));
}

// ------------------------------------------------------------------ P2G
// m_g += w m_p;  p_g += w (m_p v (1 - dt drag) + (-3/dx^2 dt vol P Fe^T + m_p C) (x_g - x_p))
// (SingleParticle_to_grid, ForwardSimulation.cpp:11-51).  FUSED_P computes P
// here (FP64 polar) instead of reading the P_op_1 output.
template <class T, bool TILED, bool FUSED_P> __global__ void __launch_bounds__(256) k_p2g(FwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < a.n;
    const T dx = (T)a.geo.dx;
    T x[3] = {0, 0, 0};
    int base[3] = {0, 0, 0};
    m3<T> G = m3_zero<T>();
    T mvd[3] = {0, 0, 0}, mp = 0;
    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            x[c] = a.st[(size_t)(PX + c) * a.np + p];
            base[c] = stencil_base<T>(x[c] - (T)a.geo.mn[c], dx, a.geo.dim[c]);
        }
        const m3<T> F = load_m3(a.st + (size_t)PF * a.np, a.np, p);
        const m3<T> Fe = F + load_m3(a.dfc, a.np, p);
        mp = a.cst[(size_t)KM * a.np + p];
        const T vol = a.cst[(size_t)KVOL * a.np + p];
        m3<T> P;
        if (FUSED_P) {
            const m3<double> Pd = pk_stress<double>(m3_cast<double>(Fe), (double)a.cst[(size_t)KLAM * a.np + p],
                                                    (double)a.cst[(size_t)KMU * a.np + p]);
            P = m3_cast<T>(Pd);
            if (a.P) store_m3(a.P, a.np, p, P);
        } else {
            P = load_m3(a.P, a.np, p);
        }
        const T k = -T(3) / (dx * dx) * a.dt * vol;
        G = (k * P) * transpose(Fe) + mp * load_m3(a.st + (size_t)PC * a.np, a.np, p);
        const T damp = T(1) - a.dt * a.drag;
#pragma unroll
        for (int c = 0; c < 3; c++) mvd[c] = mp * a.st[(size_t)(PV + c) * a.np + p] * damp;
    }
    axis_w<T> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) axis_weights(x[c], (T)a.geo.mn[c], dx, base[c], w[c], false);

    TileBox tb;
    tb.ok = false;
    node4<T>* tile = reinterpret_cast<node4<T>*>(smem_raw);
    if (TILED) {
        tb = block_tile_box(valid, base, a.tile_cap);
        if (tb.ok) {
            for (int t = threadIdx.x; t < tb.n; t += blockDim.x) tile[t] = node4<T>{0, 0, 0, 0};
            __syncthreads();
        }
    }
    if (valid) {
        const int rot = TILED ? (threadIdx.x & 63) : 0;
#pragma unroll 4
        for (int it = 0; it < 64; it++) {
            const int idx = (it + rot) & 63;
            const int di = idx >> 4, dj = (idx >> 2) & 3, dk = idx & 3;
            const int gi = base[0] + di, gj = base[1] + dj, gk = base[2] + dk;
            if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
            const T d[3] = {pick4(w[0].d, di), pick4(w[1].d, dj), pick4(w[2].d, dk)};
            const T wt = pick4(w[0].n, di) * pick4(w[1].n, dj) * pick4(w[2].n, dk);
            T gd[3];
            mv(G, d, gd);
            const T q0 = wt * (mvd[0] + gd[0]), q1 = wt * (mvd[1] + gd[1]), q2 = wt * (mvd[2] + gd[2]);
            const T qm = wt * mp;
            if (TILED && tb.ok) {
                node4<T>* nd = tile + tile_index(tb, gi, gj, gk);
                atomicAdd(&nd->w, qm);
                atomicAdd(&nd->x, q0);
                atomicAdd(&nd->y, q1);
                atomicAdd(&nd->z, q2);
            } else {
                const size_t g = ((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk;
                red_add4(a.grid + g, q0, q1, q2, qm);
            }
        }
    }
    if (TILED && tb.ok) {
        __syncthreads();
        for (int t = threadIdx.x; t < tb.n; t += blockDim.x) {
            const node4<T> v = tile[t];
            if (v.w == T(0) && v.x == T(0) && v.y == T(0) && v.z == T(0)) continue;
            const int k = t % tb.e[2], j = (t / tb.e[2]) % tb.e[1], i = t / (tb.e[2] * tb.e[1]);
            const int gi = tb.o[0] + i, gj = tb.o[1] + j, gk = tb.o[2] + k;
            if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
            red_add4(a.grid + ((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk, v.x, v.y, v.z, v.w);
        }
    }
}

// ------------------------------------------------------------------ G_op
// v = p / m + dt f_ext where |m| > FLT_EPSILON, else 0 (ForwardSimulation.cpp:53-58).
template <class T> DMPM_HD void node_velocity(const node4<T>& nd, T dt, const T* f, T* v) {
    if (fabs(nd.w) > (T)kFltEps) {
        v[0] = nd.x / nd.w + dt * f[0];
        v[1] = nd.y / nd.w + dt * f[1];
        v[2] = nd.z / nd.w + dt * f[2];
    } else {
        v[0] = v[1] = v[2] = T(0);
    }
}

template <class T> __global__ void k_gop(FwdArgs<T> a, size_t G) {
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    T v[3];
    node_velocity(a.grid[g], a.dt, a.fext, v);
    a.gridv[g] = v[0];
    a.gridv[G + g] = v[1];
    a.gridv[2 * G + g] = v[2];
}

// ------------------------------------------------------------------ G2P + P_op_2
// v' = sum w v_g;  C' = 3/dx^2 sum w v_g (x_g - x_p)^T  (ForwardSimulation.cpp:60-106)
// F' = (1 - s)(I + dt C')(F + dFc) + s F;  x' = x + dt v'  (:108-124)
// TILED fuses G_op into the tile load.
template <class T, bool TILED> __global__ void __launch_bounds__(256) k_g2p(FwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < a.n;
    const T dx = (T)a.geo.dx;
    const size_t G = (size_t)a.geo.dim[0] * a.geo.dim[1] * a.geo.dim[2];
    T x[3] = {0, 0, 0};
    int base[3] = {0, 0, 0};
    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            x[c] = a.st[(size_t)(PX + c) * a.np + p];
            base[c] = stencil_base<T>(x[c] - (T)a.geo.mn[c], dx, a.geo.dim[c]);
        }
    }
    TileBox tb;
    tb.ok = false;
    node4<T>* tile = reinterpret_cast<node4<T>*>(smem_raw);
    if (TILED) {
        tb = block_tile_box(valid, base, a.tile_cap);
        if (tb.ok) {
            for (int t = threadIdx.x; t < tb.n; t += blockDim.x) {
                const int k = t % tb.e[2], j = (t / tb.e[2]) % tb.e[1], i = t / (tb.e[2] * tb.e[1]);
                const int gi = tb.o[0] + i, gj = tb.o[1] + j, gk = tb.o[2] + k;
                T v[3] = {0, 0, 0};
                if (!(gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]))
                    node_velocity(a.grid[((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk], a.dt, a.fext, v);
                tile[t] = node4<T>{v[0], v[1], v[2], T(0)};
            }
            __syncthreads();
        }
    }
    if (!valid) return;
    axis_w<T> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) axis_weights(x[c], (T)a.geo.mn[c], dx, base[c], w[c], false);
    T vn[3] = {0, 0, 0};
    m3<T> Cn = m3_zero<T>();
    const T k3 = T(3) / (dx * dx);
#pragma unroll 2
    for (int idx = 0; idx < 64; idx++) {
        const int di = idx >> 4, dj = (idx >> 2) & 3, dk = idx & 3;
        const int gi = base[0] + di, gj = base[1] + dj, gk = base[2] + dk;
        if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
        const T d[3] = {w[0].d[di], w[1].d[dj], w[2].d[dk]};
        const T wt = w[0].n[di] * w[1].n[dj] * w[2].n[dk];
        T vg[3];
        if (TILED && tb.ok) {
            const node4<T> nd = tile[tile_index(tb, gi, gj, gk)];
            vg[0] = nd.x; vg[1] = nd.y; vg[2] = nd.z;
        } else if (TILED) {
            node_velocity(a.grid[((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk], a.dt, a.fext, vg);
        } else {
            const size_t g = ((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk;
            vg[0] = a.gridv[g]; vg[1] = a.gridv[G + g]; vg[2] = a.gridv[2 * G + g];
        }
#pragma unroll
        for (int r = 0; r < 3; r++) {
            vn[r] += wt * vg[r];
            const T kv = k3 * wt * vg[r];
#pragma unroll
            for (int c = 0; c < 3; c++) Cn.a[r][c] += kv * d[c];
        }
    }
    const m3<T> F = load_m3(a.st + (size_t)PF * a.np, a.np, p);
    const m3<T> Fe = F + load_m3(a.dfc, a.np, p);
    m3<T> Fn = (m3_eye<T>() + a.dt * Cn) * Fe;
    Fn = (T(1) - a.s) * Fn + a.s * F;
    bool finite = true;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const T xn = x[c] + a.dt * vn[c];
        a.st_next[(size_t)(PX + c) * a.np + p] = xn;
        a.st_next[(size_t)(PV + c) * a.np + p] = vn[c];
        finite &= isfinite(xn);
    }
    store_m3(a.st_next + (size_t)PF * a.np, a.np, p, Fn);
    store_m3(a.st_next + (size_t)PC * a.np, a.np, p, Cn);
    finite &= isfinite(Fn.a[0][0] + Fn.a[1][1] + Fn.a[2][2]);
    if (!finite) atomicOr(a.status, ST_NONFINITE_FWD);
}

// ------------------------------------------------------------------ loss
template <class T> struct LossArgs {
    int n;
    size_t np;           // plane stride of st and adj
    size_t npc;          // plane stride of cst
    GridGeom geo;
    const T* st;         // last layer state
    const T* cst;
    node4<T>* grid;      // mass raster written here (.w); .x/.y/.z unused
    const T* target;     // [G]
    T* dldm;             // [G]
    T* adj;              // last layer adjoint [24][np]
    double* loss;        // accumulator
    double* part;        // per-block partial sums of the loss (summed in order by k_sum_partials), or null:
                         // each block adds to *loss
    int kind;            // 0 = reference log-mass + penalty, 1 = L2
    int tile_cap;
    int xlo;             // st carries the low parts of compensated positions (planes PXL)
    unsigned* status;
};

// mass-only P2G (EndLayerMassLoss runs P2G with dt = drag = 0 and reads m only)
template <class T, bool TILED> __global__ void __launch_bounds__(256) k_p2g_mass(LossArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < a.n;
    int base[3] = {0, 0, 0};
    T mp = 0;
    axis_w<T> w[3];
    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; c++) particle_axis(a.st, a.np, p, c, a.xlo, a.geo, base[c], w[c], false);
        mp = a.cst[(size_t)KM * a.npc + p];
    }
    TileBox tb;
    tb.ok = false;
    T* tile = reinterpret_cast<T*>(smem_raw);
    if (TILED) {
        tb = block_tile_box(valid, base, a.tile_cap);
        if (tb.ok) {
            for (int t = threadIdx.x; t < tb.n; t += blockDim.x) tile[t] = T(0);
            __syncthreads();
        }
    }
    if (valid) {
        const int rot = TILED ? (threadIdx.x & 63) : 0;
#pragma unroll 4
        for (int it = 0; it < 64; it++) {
            const int idx = (it + rot) & 63;
            const int di = idx >> 4, dj = (idx >> 2) & 3, dk = idx & 3;
            const int gi = base[0] + di, gj = base[1] + dj, gk = base[2] + dk;
            if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
            const T q = pick4(w[0].n, di) * pick4(w[1].n, dj) * pick4(w[2].n, dk) * mp;
            if (TILED && tb.ok) atomicAdd(tile + tile_index(tb, gi, gj, gk), q);
            else atomicAdd(&a.grid[((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk].w, q);
        }
    }
    if (TILED && tb.ok) {
        __syncthreads();
        for (int t = threadIdx.x; t < tb.n; t += blockDim.x) {
            const T v = tile[t];
            if (v == T(0)) continue;
            const int k = t % tb.e[2], j = (t / tb.e[2]) % tb.e[1], i = t / (tb.e[2] * tb.e[1]);
            const int gi = tb.o[0] + i, gj = tb.o[1] + j, gk = tb.o[2] + k;
            if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
            atomicAdd(&a.grid[((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk].w, v);
        }
    }
}

// Per-node loss and dL/dm in FP64 (CompGraph.cpp:143-187):
//   L = sum 1/2 (log(m + 1 + eps) - log(t + 1 + eps))^2 + sum_{m < 1e-3} 10 (1e-3 - m)^2
// or, for kind 1, L = sum 1/2 (m - t)^2.  Block partial sums go to a.part
// (k_sum_partials adds them in block order, so the loss is the same in every
// run) or are added to one FP64 accumulator.
template <class T> __global__ void __launch_bounds__(256) k_node_loss(LossArgs<T> a, size_t G) {
    __shared__ double s_part[32];
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (g < G) {
        const double cm = (double)a.grid[g].w, tm = (double)a.target[g];
        double dl;
        if (a.kind == 0) {
            const double eps = 1e-4;  // CompGraph.cpp:115 (FP64 semantics: the loss is evaluated in FP64)
            const double clog = log(cm + 1.0 + eps) - log(tm + 1.0 + eps);
            l = 0.5 * clog * clog;
            dl = clog / (cm + 1.0 + eps);
            const double min_mass = 1e-3;  // CompGraph.cpp:122
            if (cm < min_mass) {
                const double diff = min_mass - cm;
                l += 10.0 * diff * diff;
                dl += -20.0 * diff;
            }
        } else {
            const double dm = cm - tm;
            l = 0.5 * dm * dm;
            dl = dm;
        }
        a.dldm[g] = (T)dl;
        if (!isfinite(l)) atomicOr(a.status, ST_NONFINITE_LOSS);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? s_part[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) {
            if (a.part) a.part[blockIdx.x] = v;
            else atomicAdd(a.loss, v);
        }
    }
}

// *out = sum of part[0 .. nb) in a fixed order (one block of 256 threads):
// strided sums per thread, then a tree over the threads
static __global__ void __launch_bounds__(256) k_sum_partials(const double* __restrict__ part, int nb, double* out) {
    __shared__ double s[256];
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += 256) v += part[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// dLdx = sum_g m_p dLdm_g grad w_gp; dLdv = dLdF = dLdC = 0 (CompGraph.cpp:192-241)
template <class T> __global__ void __launch_bounds__(256) k_loss_dldx(LossArgs<T> a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const T dx = (T)a.geo.dx;
    int base[3];
    axis_w<T> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) particle_axis(a.st, a.np, p, c, a.xlo, a.geo, base[c], w[c], true);
    const T mp = a.cst[(size_t)KM * a.npc + p];
    T acc[3] = {0, 0, 0};
    const T ndx = -T(1) / dx;
#pragma unroll 2
    for (int idx = 0; idx < 64; idx++) {
        const int di = idx >> 4, dj = (idx >> 2) & 3, dk = idx & 3;
        const int gi = base[0] + di, gj = base[1] + dj, gk = base[2] + dk;
        if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
        const T dl = mp * a.dldm[((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk];
        acc[0] += dl * (ndx * (w[0].s[di] * w[1].n[dj] * w[2].n[dk]));
        acc[1] += dl * (ndx * (w[0].n[di] * w[1].s[dj] * w[2].n[dk]));
        acc[2] += dl * (ndx * (w[0].n[di] * w[1].n[dj] * w[2].s[dk]));
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        a.adj[(size_t)(PX + c) * a.np + p] = acc[c];
        a.adj[(size_t)(PV + c) * a.np + p] = T(0);
    }
#pragma unroll
    for (int q = 0; q < 18; q++) a.adj[(size_t)(PF + q) * a.np + p] = T(0);
}

// ------------------------------------------------------------------ adjoint
template <class T> struct AdjArgs {
    int n;
    size_t np;
    GridGeom geo;
    T dt, drag, s, fext[3];
    const T* st;          // layer n state
    const T* st_next;     // layer n+1 state (C' is read)
    const T* cst;
    const T* dfc;         // dFc of layer n
    const node4<T>* grid; // layer n grid (p, m)
    const T* adj_next;    // adjoint of layer n+1
    T* adj;               // adjoint of layer n (output)
    node4<T>* gadj;       // grid scratch: (dLdv.xyz, unused)
    node4<T>* gadj2;      // plain path: (dLdp.xyz, dLdm)
    T* ctrl_grad;         // per-layer dL/d dFc of layer n [9][np] (or null)
    double* ctrl_acc;     // tied controls: FP64 accumulator [9][np] (or null)
    // debug copies of intermediates (may be null)
    T* dbg_dLdP;          // [9][np]
    T* dbg_vnext;         // [3][np]
    T* dbg_Cnext;         // [9][np]
    int tile_cap;
    unsigned* status;
};

// dLdv_next = dt dLdx' + dLdv';  dLdC_next = c dt dLdF' Fe^T + dLdC'
// (BackPropagation.cpp:14-25; EXACT uses c = 1 - s, the reference c = 1).
template <class T, bool EXACT>
__device__ __forceinline__ void adj_next_terms(const AdjArgs<T>& a, int p, const m3<T>& Fe, T vn[3], m3<T>& Cn) {
#pragma unroll
    for (int c = 0; c < 3; c++)
        vn[c] = a.dt * a.adj_next[(size_t)(PX + c) * a.np + p] + a.adj_next[(size_t)(PV + c) * a.np + p];
    const m3<T> dFn = load_m3(a.adj_next + (size_t)PF * a.np, a.np, p);
    const T c = EXACT ? (T(1) - a.s) * a.dt : a.dt;
    Cn = (c * dFn) * transpose(Fe) + load_m3(a.adj_next + (size_t)PC * a.np, a.np, p);
}

// Adjoint G2P: dLdv_g += w dLdv_next + 3/dx^2 w dLdC_next (x_g - x_p)
// (BackPropagation.cpp:27-44).
template <class T, bool TILED, bool EXACT> __global__ void __launch_bounds__(256) k_adj_scatter(AdjArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < a.n;
    const T dx = (T)a.geo.dx;
    T x[3] = {0, 0, 0};
    int base[3] = {0, 0, 0};
    T vn[3] = {0, 0, 0};
    m3<T> Cn = m3_zero<T>();
    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            x[c] = a.st[(size_t)(PX + c) * a.np + p];
            base[c] = stencil_base<T>(x[c] - (T)a.geo.mn[c], dx, a.geo.dim[c]);
        }
        const m3<T> Fe = load_m3(a.st + (size_t)PF * a.np, a.np, p) + load_m3(a.dfc, a.np, p);
        adj_next_terms<T, EXACT>(a, p, Fe, vn, Cn);
        if (a.dbg_vnext) {
#pragma unroll
            for (int c = 0; c < 3; c++) a.dbg_vnext[(size_t)c * a.np + p] = vn[c];
            store_m3(a.dbg_Cnext, a.np, p, Cn);
        }
    }
    axis_w<T> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) axis_weights(x[c], (T)a.geo.mn[c], dx, base[c], w[c], false);
    TileBox tb;
    tb.ok = false;
    node4<T>* tile = reinterpret_cast<node4<T>*>(smem_raw);
    if (TILED) {
        tb = block_tile_box(valid, base, a.tile_cap);
        if (tb.ok) {
            for (int t = threadIdx.x; t < tb.n; t += blockDim.x) tile[t] = node4<T>{0, 0, 0, 0};
            __syncthreads();
        }
    }
    const T k3 = T(3) / (dx * dx);
    if (valid) {
        const int rot = TILED ? (threadIdx.x & 63) : 0;
#pragma unroll 4
        for (int it = 0; it < 64; it++) {
            const int idx = (it + rot) & 63;
            const int di = idx >> 4, dj = (idx >> 2) & 3, dk = idx & 3;
            const int gi = base[0] + di, gj = base[1] + dj, gk = base[2] + dk;
            if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
            const T d[3] = {pick4(w[0].d, di), pick4(w[1].d, dj), pick4(w[2].d, dk)};
            const T wt = pick4(w[0].n, di) * pick4(w[1].n, dj) * pick4(w[2].n, dk);
            T cd[3];
            mv(Cn, d, cd);
            const T q0 = vn[0] * wt + k3 * wt * cd[0];
            const T q1 = vn[1] * wt + k3 * wt * cd[1];
            const T q2 = vn[2] * wt + k3 * wt * cd[2];
            if (TILED && tb.ok) {
                node4<T>* nd = tile + tile_index(tb, gi, gj, gk);
                atomicAdd(&nd->x, q0);
                atomicAdd(&nd->y, q1);
                atomicAdd(&nd->z, q2);
            } else {
                red_add4(a.gadj + ((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk, q0, q1, q2, T(0));
            }
        }
    }
    if (TILED && tb.ok) {
        __syncthreads();
        for (int t = threadIdx.x; t < tb.n; t += blockDim.x) {
            const node4<T> v = tile[t];
            if (v.x == T(0) && v.y == T(0) && v.z == T(0)) continue;
            const int k = t % tb.e[2], j = (t / tb.e[2]) % tb.e[1], i = t / (tb.e[2] * tb.e[1]);
            const int gi = tb.o[0] + i, gj = tb.o[1] + j, gk = tb.o[2] + k;
            if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
            red_add4(a.gadj + ((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk, v.x, v.y, v.z, T(0));
        }
    }
}

// Adjoint G_op: dLdp = dLdv / m; dLdm = -(1/m) v_m . dLdv where |m| > FLT_EPS
// (BackPropagation.cpp:46-59).  v_m is the node velocity v (reference) or
// p/m = v - dt f_ext (EXACT).
template <class T, bool EXACT>
DMPM_HD void node_adjoint(const node4<T>& nd, const node4<T>& gdv, T dt, const T* f, T out[4]) {
    if (fabs(nd.w) > (T)kFltEps) {
        T v[3];
        node_velocity(nd, dt, f, v);
        if (EXACT) { v[0] -= dt * f[0]; v[1] -= dt * f[1]; v[2] -= dt * f[2]; }
        out[0] = gdv.x / nd.w;
        out[1] = gdv.y / nd.w;
        out[2] = gdv.z / nd.w;
        out[3] = -T(1) / nd.w * (v[0] * gdv.x + v[1] * gdv.y + v[2] * gdv.z);
    } else {
        out[0] = out[1] = out[2] = out[3] = T(0);
    }
}

template <class T, bool EXACT> __global__ void k_adj_gop(AdjArgs<T> a, size_t G) {
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    T o[4];
    node_adjoint<T, EXACT>(a.grid[g], a.gadj[g], a.dt, a.fext, o);
    a.gadj2[g] = node4<T>{o[0], o[1], o[2], o[3]};
}

// Adjoint P2G + P_op_1 (BackPropagation.cpp:61-124), as a per-particle gather.
// With M = sum_g w d dLdp^T (d = x_g - x_p), the reference's three 3x3 sums are
//   dLdP = -3/dx^2 dt vol M^T Fe,  dLdF(stress) = -3/dx^2 dt vol M P,  dLdC = m M^T,
// and every grad-w term of dLdx is a scalar per node times grad w:
//   sigma_g = m dLdm + dLdp.(m v c_d + G d) + v_g.(dLdv_next + 3/dx^2 dLdC_next d)
//   dLdx = sum sigma_g grad w - G^T sum w dLdp - 3/dx^2 dLdC_next^T sum w v_g + dLdx'
//   dLdv = m (1 - dt drag) sum w dLdp
// (c_d = 1 for the reference, 1 - dt drag for EXACT).  Then
//   REFCOMPAT: dLdF += (I + dt C')^T dLdF' + dP/dF:dLdP     (the transport term twice)
//   EXACT:     dLdFe = (1-s)(I + dt C')^T dLdF' + stress + dP/dF:dLdP;  dLdF = dLdFe + s dLdF'
// The polar factors, P and dP/dF:dLdP are evaluated in FP64.
template <class T, bool TILED, bool EXACT> __global__ void __launch_bounds__(256) k_adj_gather(AdjArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < a.n;
    const T dx = (T)a.geo.dx;
    T x[3] = {0, 0, 0};
    int base[3] = {0, 0, 0};
    if (valid) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            x[c] = a.st[(size_t)(PX + c) * a.np + p];
            base[c] = stencil_base<T>(x[c] - (T)a.geo.mn[c], dx, a.geo.dim[c]);
        }
    }
    TileBox tb;
    tb.ok = false;
    node4<T>* tile = reinterpret_cast<node4<T>*>(smem_raw);  // [2*n]: (dLdp, dLdm), (v_g, 0)
    if (TILED) {
        tb = block_tile_box(valid, base, a.tile_cap);
        if (tb.ok) {
            for (int t = threadIdx.x; t < tb.n; t += blockDim.x) {
                const int k = t % tb.e[2], j = (t / tb.e[2]) % tb.e[1], i = t / (tb.e[2] * tb.e[1]);
                const int gi = tb.o[0] + i, gj = tb.o[1] + j, gk = tb.o[2] + k;
                T o[4] = {0, 0, 0, 0}, v[3] = {0, 0, 0};
                if (!(gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2])) {
                    const size_t g = ((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk;
                    const node4<T> nd = a.grid[g];
                    node_adjoint<T, EXACT>(nd, a.gadj[g], a.dt, a.fext, o);
                    node_velocity(nd, a.dt, a.fext, v);
                }
                tile[2 * t] = node4<T>{o[0], o[1], o[2], o[3]};
                tile[2 * t + 1] = node4<T>{v[0], v[1], v[2], T(0)};
            }
            __syncthreads();
        }
    }
    if (!valid) return;
    const size_t np = a.np;
    const T mp = a.cst[(size_t)KM * np + p], vol = a.cst[(size_t)KVOL * np + p];
    const m3<T> F = load_m3(a.st + (size_t)PF * np, np, p);
    const m3<T> Fe = F + load_m3(a.dfc, np, p);
    // polar factors and stress in FP64
    const m3<double> Fed = m3_cast<double>(Fe);
    m3<double> Rd, Sd;
    polar3(Fed, Rd, Sd);
    const double lam = (double)a.cst[(size_t)KLAM * np + p], mu = (double)a.cst[(size_t)KMU * np + p];
    const m3<T> P = m3_cast<T>(pk_from_polar(Fed, Rd, lam, mu));
    const T k3 = T(3) / (dx * dx);
    const m3<T> G = (-k3 * a.dt * vol) * P * transpose(Fe) + mp * load_m3(a.st + (size_t)PC * np, np, p);
    T vn[3];
    m3<T> Cn;
    adj_next_terms<T, EXACT>(a, p, Fe, vn, Cn);
    const T cd = EXACT ? (T(1) - a.dt * a.drag) : T(1);
    T mvp[3];
#pragma unroll
    for (int c = 0; c < 3; c++) mvp[c] = mp * a.st[(size_t)(PV + c) * np + p] * cd;

    axis_w<T> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) axis_weights(x[c], (T)a.geo.mn[c], dx, base[c], w[c], true);
    m3<T> M = m3_zero<T>();
    T X[3] = {0, 0, 0}, u[3] = {0, 0, 0}, z[3] = {0, 0, 0};
    const T ndx = -T(1) / dx;
    const size_t G_ = (size_t)a.geo.dim[0] * a.geo.dim[1] * a.geo.dim[2];
    (void)G_;
#pragma unroll 2
    for (int idx = 0; idx < 64; idx++) {
        const int di = idx >> 4, dj = (idx >> 2) & 3, dk = idx & 3;
        const int gi = base[0] + di, gj = base[1] + dj, gk = base[2] + dk;
        if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
        T o[4], vg[3];
        if (TILED && tb.ok) {
            const int t = tile_index(tb, gi, gj, gk);
            const node4<T> q = tile[2 * t], r = tile[2 * t + 1];
            o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w;
            vg[0] = r.x; vg[1] = r.y; vg[2] = r.z;
        } else {
            const size_t g = ((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk;
            const node4<T> nd = a.grid[g];
            if (TILED) {
                node_adjoint<T, EXACT>(nd, a.gadj[g], a.dt, a.fext, o);
            } else {
                const node4<T> q = a.gadj2[g];
                o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w;
            }
            node_velocity(nd, a.dt, a.fext, vg);
        }
        const T d[3] = {w[0].d[di], w[1].d[dj], w[2].d[dk]};
        const T nx = w[0].n[di], ny = w[1].n[dj], nz = w[2].n[dk];
        const T wt = nx * ny * nz;
        const T gw[3] = {ndx * (w[0].s[di] * ny * nz), ndx * (nx * w[1].s[dj] * nz), ndx * (nx * ny * w[2].s[dk])};
        T Gd[3], Cd[3];
        mv(G, d, Gd);
        mv(Cn, d, Cd);
        const T sigma = mp * o[3] + o[0] * (mvp[0] + Gd[0]) + o[1] * (mvp[1] + Gd[1]) + o[2] * (mvp[2] + Gd[2]) +
                        vg[0] * (vn[0] + k3 * Cd[0]) + vg[1] * (vn[1] + k3 * Cd[1]) + vg[2] * (vn[2] + k3 * Cd[2]);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            X[r] += sigma * gw[r];
            u[r] += wt * o[r];
            z[r] += wt * vg[r];
            const T wd = wt * d[r];
#pragma unroll
            for (int c = 0; c < 3; c++) M.a[r][c] += wd * o[c];
        }
    }
    const T kk = -k3 * a.dt * vol;
    const m3<T> dLdP = kk * mtm(M, Fe);         // kk M^T Fe
    const m3<T> dFstress = kk * (M * P);
    const m3<T> dLdC = mp * transpose(M);
    T gtu[3], ctz[3];
    mtv(G, u, gtu);
    mtv(Cn, z, ctz);
    T dLdx[3], dLdv[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        dLdx[c] = X[c] - gtu[c] - k3 * ctz[c] + a.adj_next[(size_t)(PX + c) * np + p];
        dLdv[c] = mp * (T(1) - a.dt * a.drag) * u[c];
    }
    const m3<T> Cnext = load_m3(a.st_next + (size_t)PC * np, np, p);
    const m3<T> dFn = load_m3(a.adj_next + (size_t)PF * np, np, p);
    const m3<T> transport = mtm(m3_eye<T>() + a.dt * Cnext, dFn);  // (I + dt C')^T dLdF'
    const m3<T> d2 = m3_cast<T>(d2_mult_from_polar<EXACT>(Fed, Rd, Sd, lam, mu, m3_cast<double>(dLdP)));
    m3<T> dLdF, dLdFe;
    if (EXACT) {
        dLdFe = (T(1) - a.s) * transport + dFstress + d2;
        dLdF = dLdFe + a.s * dFn;
    } else {
        dLdF = ((T(1) - a.s) * transport + a.s * dFn) + dFstress + transport + d2;
        dLdFe = dLdF;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        a.adj[(size_t)(PX + c) * np + p] = dLdx[c];
        a.adj[(size_t)(PV + c) * np + p] = dLdv[c];
    }
    store_m3(a.adj + (size_t)PF * np, np, p, dLdF);
    store_m3(a.adj + (size_t)PC * np, np, p, dLdC);
    if (a.ctrl_grad) store_m3(a.ctrl_grad, np, p, dLdFe);
    if (a.ctrl_acc) {
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int r = 0; r < 3; r++) a.ctrl_acc[(size_t)(r + 3 * c) * np + p] += (double)dLdFe.a[r][c];
    }
    if (a.dbg_dLdP) store_m3(a.dbg_dLdP, np, p, dLdP);
    if (!isfinite(dLdF.a[0][0] + dLdF.a[1][1] + dLdF.a[2][2] + dLdx[0] + dLdx[1] + dLdx[2]))
        atomicOr(a.status, ST_NONFINITE_ADJ);
}

// ------------------------------------------------------------------ volumes / target raster
// vol_p = m_p / sum_g w m_g  (CalculatePointCloudVolumes, ForwardSimulation.cpp:262-290)
template <class T> __global__ void k_volumes(LossArgs<T> a, T* vol_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    int base[3];
    axis_w<T> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) particle_axis(a.st, a.np, p, c, a.xlo, a.geo, base[c], w[c], false);
    T mg = 0;
    for (int idx = 0; idx < 64; idx++) {
        const int di = idx >> 4, dj = (idx >> 2) & 3, dk = idx & 3;
        const int gi = base[0] + di, gj = base[1] + dj, gk = base[2] + dk;
        if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
        mg += w[0].n[di] * w[1].n[dj] * w[2].n[dk] * a.grid[((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk].w;
    }
    const T mp = a.cst[(size_t)KM * a.npc + p];
    vol_out[p] = (fabs(mg) > (T)kFltEps) ? mp / mg : T(0);
}

}  // namespace dmpm
