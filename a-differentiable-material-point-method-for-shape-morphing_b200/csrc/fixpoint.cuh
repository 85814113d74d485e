// fixpoint.cuh -- node sums that do not depend on the order of the atomic adds
// (the deterministic mode of the FP32 path, dmpm_params::deterministic).
//
// P2G, the adjoint scatter and the mass rasters add each particle's (or each
// warp item's) contribution to a node with an atomic add.  In float the sum
// depends on the order in which the adds arrive, which changes from run to run,
// and a long rollout amplifies those last-bit differences.  In this mode each
// contribution x is rounded once to the integer round(x 2^k) and the integers
// are added with 64-bit atomics.  Integer addition is exact and associative, so
// every order gives the same sum; the node value is that sum times 2^-k.
//
// The exponent k is chosen per pass from a bound on every node sum.  A node
// receives at most one contribution w X per particle, with weight w <= 1 (and
// w > 0 only inside the stencil, where |x_g - x_p| < 2 dx) and |X| <= c_p, so
// |sum| <= n max_p c_p.  With max_p c_p < 2^e and n <= 2^b, k = 61 - e - b
// keeps |sum| 2^k below 2^61, and the n roundings (at most 1/2 each) keep the
// integer below 2^62.  max_p c_p is a maximum over particles -- atomicMax on the
// bit patterns of non-negative floats, the same in every order.  The
// resolution 2^-k is then at most n max c_p 2^-59: a node sum carries an
// absolute error of at most (its contributions) x 2^-(k+1), far below the one
// float rounding per atomic add that it replaces on every node whose sum is
// more than 2^-35 of that bound.
#pragma once
#include <cstdint>
#include "fixscale.h"
#include "kernels.cuh"

namespace dmpm {

struct alignas(32) fix4 {
    long long x, y, z, w;
};

#ifdef __CUDACC__
__device__ __forceinline__ long long fix_round(float x, float scale) { return __float2ll_rn(x * scale); }
__device__ __forceinline__ float fix_value(long long q, float inv_scale) { return __ll2float_rn(q) * inv_scale; }

__device__ __forceinline__ void fix_red(long long* p, long long q) {
    if (q != 0) atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)q);
}
__device__ __forceinline__ void fix_red4(fix4* p, float a, float b, float c, float d, float sa, float sd) {
    fix_red(&p->x, fix_round(a, sa));
    fix_red(&p->y, fix_round(b, sa));
    fix_red(&p->z, fix_round(c, sa));
    fix_red(&p->w, fix_round(d, sd));
}

// A CTA's shared tile of integer node sums: E^3 nodes from grid node o, one
// array of E^3 integers per value (x, y, z, w at t, t + nt, t + 2 nt, t + 3 nt):
// the lanes of a warp add to neighbouring nodes, which this layout spreads
// over the shared-memory banks (a 32-byte record per node would put a warp's
// adds into a quarter of them).
struct FixTile {
    long long* t;
    int nt;
    int o[3];
    int E;
};
// the same integers as fix_red4, added to the tile in shared memory first
__device__ __forceinline__ void fix_red_shared(long long* p, long long q) {
    if (q != 0) atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)q);
}
__device__ __forceinline__ void fix_red4_tile(const FixTile& ft, int node, float a, float b, float c, float d, float sa,
                                              float sd) {
    fix_red_shared(ft.t + node, fix_round(a, sa));
    fix_red_shared(ft.t + ft.nt + node, fix_round(b, sa));
    fix_red_shared(ft.t + 2 * ft.nt + node, fix_round(c, sa));
    fix_red_shared(ft.t + 3 * ft.nt + node, fix_round(d, sd));
}
// offset in the tile of a stencil's first node (base), or -1 when its 4^3
// nodes are not all inside the tile
__device__ __forceinline__ int fix_tile_offset(const FixTile& ft, const int base[3]) {
    const int l0 = base[0] - ft.o[0], l1 = base[1] - ft.o[1], l2 = base[2] - ft.o[2];
    const unsigned lim = (unsigned)(ft.E - 3);
    if ((unsigned)l0 < lim && (unsigned)l1 < lim && (unsigned)l2 < lim) return (l0 * ft.E + l1) * ft.E + l2;
    return -1;
}

// Raise slot to the maximum of |c| over the warp; every lane of the warp calls it.
__device__ __forceinline__ void fix_bound(unsigned* slot, float c) {
    const unsigned b = __reduce_max_sync(0xffffffffu, __float_as_uint(fabsf(c)));
    if ((threadIdx.x & 31) == 0 && b != 0u) atomicMax(slot, b);
}

// the scale 2^k of a pass and its inverse, from a bound slot
struct FixScale {
    float s, inv;
};
__device__ __forceinline__ FixScale fix_scale(const unsigned* slot, long long n) {
    const int k = fix_exponent(*slot, n);
    return FixScale{fix_pow2(k), fix_pow2(-k)};
}

// Node records from the integer sums: which = 0: (p.xyz, m) with the momentum
// and mass scales; 1: (dLdv.xyz, 0) with the adjoint scale; 2: (0, 0, 0, m)
// with the raster scale.
static __global__ void k_fix_to_node4(const fix4* __restrict__ acc, const unsigned* __restrict__ slots, long long n,
                                      size_t G, int which, node4<float>* out) {
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const fix4 q = acc[g];
    node4<float> r{0.f, 0.f, 0.f, 0.f};
    if (which == 0) {
        const FixScale sp = fix_scale(slots + FIXB_MOMENTUM, n), sm = fix_scale(slots + FIXB_MASS, n);
        r = node4<float>{fix_value(q.x, sp.inv), fix_value(q.y, sp.inv), fix_value(q.z, sp.inv), fix_value(q.w, sm.inv)};
    } else if (which == 1) {
        const FixScale sa = fix_scale(slots + FIXB_ADJ, n);
        r = node4<float>{fix_value(q.x, sa.inv), fix_value(q.y, sa.inv), fix_value(q.z, sa.inv), 0.f};
    } else {
        const FixScale sr = fix_scale(slots + FIXB_RASTER, n);
        r.w = fix_value(q.w, sr.inv);
    }
    out[g] = r;
}

// the largest particle mass of a cloud, into slot (the raster's bound)
static __global__ void k_fix_mass_bound(const float* __restrict__ m, int n, unsigned* slot) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    fix_bound(slot, p < n ? m[p] * 1.001f : 0.f);
}

// mass-only P2G (k_p2g_mass's arithmetic per contribution) as integer sums
// into acc[].w, scaled by the raster bound slot
static __global__ void __launch_bounds__(256) k_p2g_mass_fix(LossArgs<float> a, fix4* acc, const unsigned* slots) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const FixScale sr = fix_scale(slots + FIXB_RASTER, a.n);
    int base[3];
    axis_w<float> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) particle_axis(a.st, a.np, p, c, a.xlo, a.geo, base[c], w[c], false);
    const float mp = a.cst[(size_t)KM * a.npc + p];
#pragma unroll 4
    for (int idx = 0; idx < 64; idx++) {
        const int di = idx >> 4, dj = (idx >> 2) & 3, dk = idx & 3;
        const int gi = base[0] + di, gj = base[1] + dj, gk = base[2] + dk;
        if (gi < 0 || gi >= a.geo.dim[0] || gj < 0 || gj >= a.geo.dim[1] || gk < 0 || gk >= a.geo.dim[2]) continue;
        const float q = pick4(w[0].n, di) * pick4(w[1].n, dj) * pick4(w[2].n, dk) * mp;
        fix_red(&acc[((size_t)gi * a.geo.dim[1] + gj) * a.geo.dim[2] + gk].w, fix_round(q, sr.s));
    }
}
#endif

}  // namespace dmpm
