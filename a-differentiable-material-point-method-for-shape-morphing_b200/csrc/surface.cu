// surface.cu -- headless surfacing of point clouds on the GPU (include/dmpm.h,
// "surfaces"): the scalar fields the reference builds for its exported meshes
// and an isosurface extractor for them.
//
//   dmpm_surface_p2g_mass     SingleThreadMPM::P2G_Mass (ForwardSimulation.cpp:292-327)
//   dmpm_surface_g2g_mass     SingleThreadMPM::G2G_Mass (ForwardSimulation.cpp:329-367)
//   dmpm_surface_sphere_field the field of SphereUnionMarchingCubesSurfaceFromPointCloud
//                             (SphereUnionSurfacing.cpp:7-106)
//   dmpm_surface_extract      a triangle mesh of the level set {f = iso} of a grid field
//
// The fields repeat the reference's float arithmetic operation by operation
// (products, sums and quotients written as __f*_rn so nothing is contracted into
// an FMA), so G2G_Mass and the sphere field are bit-identical to the reference;
// P2G_Mass accumulates with float atomics, so its sums differ from the reference's
// point-ordered sums by rounding only.
//
// The extractor is marching tetrahedra over the Kuhn subdivision of each grid
// cube into six tetrahedra around its main diagonal, with one vertex per crossed
// grid edge (the 7 edge directions {0,1}^3 \ 0 from each node) at the linearly
// interpolated crossing and triangles oriented so that their normals point to
// decreasing field values (out of {f > iso}).  Vertices come in edge order and
// triangles in cube order, so the output is deterministic.  The reference hands
// the same fields to libigl's marching cubes (SphereUnionSurfacing.cpp:125,
// DiffMPMAnimator3D.cpp:511); both meshes approximate the same level set with
// different triangulations.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "dmpm.h"
#include "sort.cuh"

namespace dmpm {
namespace {

struct Grid3 {
    int n[3];
    float dx;
    float mn[3];
};

__device__ __forceinline__ float node_coord(const Grid3& g, int a, int i) {
    return __fadd_rn(g.mn[a], __fmul_rn((float)i, g.dx));  // min + (i, j, k) * dx (Grid.cpp:21)
}

// CubicBSpline (Interpolation.h:5-17), operation by operation
__device__ __forceinline__ float cubic_bspline_ref(float x) {
    x = fabsf(x);
    if (x < 1.f) return __fadd_rn(__fsub_rn(__fmul_rn(__fmul_rn(__fmul_rn(0.5f, x), x), x), __fmul_rn(x, x)), 2.f / 3.f);
    if (x < 2.f) {
        const float t = __fsub_rn(2.f, x);
        return __fdiv_rn(__fmul_rn(__fmul_rn(t, t), t), 6.f);
    }
    return 0.f;
}

// one term of the stencil loop of Grid::QueryPoint_CubicBSpline (Grid.cpp:40-79):
// the weight of node (bi + i, bj + j, bk + k) for point x, or -1 when outside the grid
__device__ __forceinline__ float stencil_weight(const Grid3& g, const float x[3], const int b[3], int i, int j, int k,
                                                long long& node) {
    const int id[3] = {b[0] + i, b[1] + j, b[2] + k};
    if (id[0] < 0 || id[0] >= g.n[0] || id[1] < 0 || id[1] >= g.n[1] || id[2] < 0 || id[2] >= g.n[2]) return -1.f;
    float w[3];
#pragma unroll
    for (int a = 0; a < 3; a++) w[a] = cubic_bspline_ref(__fdiv_rn(__fsub_rn(node_coord(g, a, id[a]), x[a]), g.dx));
    node = ((long long)id[0] * g.n[1] + id[1]) * g.n[2] + id[2];
    return __fmul_rn(__fmul_rn(w[0], w[1]), w[2]);
}

__device__ __forceinline__ void stencil_base_ref(const Grid3& g, const float x[3], int b[3]) {
#pragma unroll
    for (int a = 0; a < 3; a++) b[a] = (int)floorf(__fdiv_rn(__fsub_rn(x[a], g.mn[a]), g.dx)) - 1;
}

__global__ void k_p2g_mass_points(const float* __restrict__ pts, long long n, float mp_m, Grid3 g, float* mass) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float x[3] = {pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]};
    int b[3];
    stencil_base_ref(g, x, b);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++) {
                long long node;
                const float w = stencil_weight(g, x, b, i, j, k, node);
                if (w >= 0.f) atomicAdd(mass + node, __fmul_rn(w, mp_m));
            }
}

// one thread per node of grid 2, summing grid 1's stencil in the reference's order
__global__ void k_g2g_mass(const float* __restrict__ m1, Grid3 g1, Grid3 g2, float* m2) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)g2.n[0] * g2.n[1] * g2.n[2];
    if (q >= total) return;
    const int i2 = (int)(q / ((long long)g2.n[1] * g2.n[2])), j2 = (int)((q / g2.n[2]) % g2.n[1]),
              k2 = (int)(q % g2.n[2]);
    const float x[3] = {node_coord(g2, 0, i2), node_coord(g2, 1, j2), node_coord(g2, 2, k2)};
    int b[3];
    stencil_base_ref(g1, x, b);
    float acc = 0.f;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++) {
                long long node;
                const float w = stencil_weight(g1, x, b, i, j, k, node);
                if (w >= 0.f) acc = __fadd_rn(acc, __fmul_rn(w, m1[node]));
            }
    m2[q] = acc;
}

// one thread per point: radius - |x - p| on the nodes of its sphere, kept as a
// maximum (values >= 0 order like their bit patterns; a rounding-negative value
// loses to the initial 0 either way, as std::max does)
__global__ void k_sphere_max(const float* __restrict__ pts, long long n, float r, Grid3 g, int* field_bits) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float x[3] = {pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]};
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        lo[a] = max(0, (int)ceilf(__fdiv_rn(__fsub_rn(__fsub_rn(x[a], r), g.mn[a]), g.dx)));
        hi[a] = min(g.n[a] - 1, (int)ceilf(__fdiv_rn(__fsub_rn(__fadd_rn(x[a], r), g.mn[a]), g.dx)));
    }
    const float r2 = __fmul_rn(r, r);
    for (int i = lo[0]; i <= hi[0]; i++) {
        const float d0 = __fsub_rn(node_coord(g, 0, i), x[0]);
        for (int j = lo[1]; j <= hi[1]; j++) {
            const float d1 = __fsub_rn(node_coord(g, 1, j), x[1]);
            for (int k = lo[2]; k <= hi[2]; k++) {
                const float d2 = __fsub_rn(node_coord(g, 2, k), x[2]);
                // Eigen's squaredNorm of a 3-vector: d0^2 + (d1^2 + d2^2)
                const float sq = __fadd_rn(__fmul_rn(d0, d0), __fadd_rn(__fmul_rn(d1, d1), __fmul_rn(d2, d2)));
                if (sq <= r2) {
                    const float v = __fsub_rn(r, __fsqrt_rn(sq));
                    atomicMax(field_bits + ((long long)i * g.n[1] + j) * g.n[2] + k, __float_as_int(v));
                }
            }
        }
    }
}

// one blur pass (SphereUnionSurfacing.cpp:77-101): interior nodes get the
// 27-node sum (in (ii, jj, kk) order, float) divided by 9.0 in double
__global__ void k_box_blur(const float* __restrict__ src, Grid3 g, float* dst) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    if (q >= total) return;
    const int i = (int)(q / ((long long)g.n[1] * g.n[2])), j = (int)((q / g.n[2]) % g.n[1]), k = (int)(q % g.n[2]);
    if (i < 1 || j < 1 || k < 1 || i >= g.n[0] - 1 || j >= g.n[1] - 1 || k >= g.n[2] - 1) return;
    float s = 0.f;
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int c = -1; c <= 1; c++) s = __fadd_rn(s, src[((long long)(i + a) * g.n[1] + (j + b)) * g.n[2] + k + c]);
    dst[q] = __double2float_rn(__ddiv_rn((double)s, 9.0));
}

// ---------------------------------------------------------------- isosurface
// edge directions from a node: the nonzero vectors of {0,1}^3, as bits (x=4, y=2, z=1)
__constant__ int kEdgeDir[7] = {4, 2, 1, 6, 5, 3, 7};
__device__ __forceinline__ int dir_slot(int bits) {
    switch (bits) {
        case 4: return 0;
        case 2: return 1;
        case 1: return 2;
        case 6: return 3;
        case 5: return 4;
        case 3: return 5;
        default: return 6;
    }
}

__device__ __forceinline__ long long node_lin(const Grid3& g, int i, int j, int k) {
    return ((long long)i * g.n[1] + j) * g.n[2] + k;
}

// flag of edge (node, dir): the field crosses iso along it
__global__ void k_edge_flags(const float* __restrict__ f, Grid3 g, float iso, uint32_t* flag) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2] * 7;
    if (e >= total) return;
    const long long q = e / 7;
    const int bits = kEdgeDir[e % 7];
    const int i = (int)(q / ((long long)g.n[1] * g.n[2])), j = (int)((q / g.n[2]) % g.n[1]), k = (int)(q % g.n[2]);
    const int i2 = i + (bits >> 2), j2 = j + ((bits >> 1) & 1), k2 = k + (bits & 1);
    uint32_t c = 0;
    if (i2 < g.n[0] && j2 < g.n[1] && k2 < g.n[2]) c = ((f[q] > iso) != (f[node_lin(g, i2, j2, k2)] > iso)) ? 1u : 0u;
    flag[e] = c;
}

__global__ void k_edge_vertices(const float* __restrict__ f, Grid3 g, float iso, const uint32_t* __restrict__ flag,
                                const uint32_t* __restrict__ vid, float* V) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2] * 7;
    if (e >= total || !flag[e]) return;
    const long long q = e / 7;
    const int bits = kEdgeDir[e % 7];
    const int i = (int)(q / ((long long)g.n[1] * g.n[2])), j = (int)((q / g.n[2]) % g.n[1]), k = (int)(q % g.n[2]);
    const int id2[3] = {i + (bits >> 2), j + ((bits >> 1) & 1), k + (bits & 1)};
    const int id1[3] = {i, j, k};
    const float fa = f[q], fb = f[node_lin(g, id2[0], id2[1], id2[2])];
    const float t = (iso - fa) / (fb - fa);
    const long long v = vid[e];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float pa = node_coord(g, a, id1[a]), pb = node_coord(g, a, id2[a]);
        V[3 * v + a] = pa + t * (pb - pa);
    }
}

// The six Kuhn tetrahedra of a cube: corner offsets (bits x=4, y=2, z=1) of
// v0 = 0, v1 = e_a, v2 = e_a + e_b, v3 = 7 for the axis orders (a, b).
__constant__ int kTet[6][4] = {{0, 4, 6, 7}, {0, 4, 5, 7}, {0, 2, 6, 7}, {0, 2, 3, 7}, {0, 1, 5, 7}, {0, 1, 3, 7}};

__device__ __forceinline__ int3 corner_off(int c) { return make_int3(c >> 2, (c >> 1) & 1, c & 1); }
__device__ __forceinline__ int det3i(int3 a, int3 b, int3 c) {
    return a.x * (b.y * c.z - b.z * c.y) - a.y * (b.x * c.z - b.z * c.x) + a.z * (b.x * c.y - b.y * c.x);
}
__device__ __forceinline__ int3 sub3(int3 a, int3 b) { return make_int3(a.x - b.x, a.y - b.y, a.z - b.z); }

// edge slot of the tet edge between cube corners ca, cb (ca's offset <= cb's componentwise)
__device__ __forceinline__ long long edge_of(const Grid3& g, int i, int j, int k, int ca, int cb) {
    const int3 a = corner_off(ca);
    return node_lin(g, i + a.x, j + a.y, k + a.z) * 7 + dir_slot(cb ^ ca);
}

// Triangles of one tetrahedron (corner codes c[4], inside flags s[4]) as edge-slot
// triples, oriented so normals point from inside (f > iso) to outside.  Returns
// the number of triangles (0-2); writes them when out is non-null.
__device__ int tet_triangles(const Grid3& g, int i, int j, int k, const int c[4], const bool s[4], long long (*out)[3]) {
    int in[4], ou[4], ni = 0, no = 0;
    for (int t = 0; t < 4; t++) {
        if (s[t]) in[ni++] = c[t];
        else ou[no++] = c[t];
    }
    // a tet edge joins corners whose offsets are ordered componentwise, and the
    // corner codes of one Kuhn tet increase in that order
    auto E = [&](int x, int y) { return x < y ? edge_of(g, i, j, k, x, y) : edge_of(g, i, j, k, y, x); };
    if (ni == 1 || no == 1) {
        const bool lone_in = ni == 1;
        const int a = lone_in ? in[0] : ou[0];
        const int* o = lone_in ? ou : in;
        if (!out) return 1;
        // normal of (ab, ac, ad) points away from a iff det(b - a, c - a, d - a) > 0
        const int3 A = corner_off(a);
        const int d = det3i(sub3(corner_off(o[0]), A), sub3(corner_off(o[1]), A), sub3(corner_off(o[2]), A));
        const bool away = d > 0;  // the normal must point away from a lone inside corner, toward a lone outside one
        const bool keep = lone_in ? away : !away;
        out[0][0] = E(a, o[0]);
        out[0][1] = keep ? E(a, o[1]) : E(a, o[2]);
        out[0][2] = keep ? E(a, o[2]) : E(a, o[1]);
        return 1;
    }
    if (ni == 2) {
        if (!out) return 2;
        const int a = in[0], b = in[1], c0 = ou[0], d0 = ou[1];
        // quad ac, ad, bd, bc; its normal (bd - ac) x (bc - ad) must point along (c + d - a - b)
        const int3 A = corner_off(a), B = corner_off(b), C = corner_off(c0), D = corner_off(d0);
        const int3 d1 = make_int3(B.x + D.x - A.x - C.x, B.y + D.y - A.y - C.y, B.z + D.z - A.z - C.z);
        const int3 d2 = make_int3(B.x + C.x - A.x - D.x, B.y + C.y - A.y - D.y, B.z + C.z - A.z - D.z);
        const int3 gdir = make_int3(C.x + D.x - A.x - B.x, C.y + D.y - A.y - B.y, C.z + D.z - A.z - B.z);
        const bool keep = det3i(d1, d2, gdir) > 0;
        const long long q0 = E(a, c0), q1 = E(a, d0), q2 = E(b, d0), q3 = E(b, c0);
        if (keep) {
            out[0][0] = q0; out[0][1] = q1; out[0][2] = q2;
            out[1][0] = q0; out[1][1] = q2; out[1][2] = q3;
        } else {
            out[0][0] = q0; out[0][1] = q2; out[0][2] = q1;
            out[1][0] = q0; out[1][1] = q3; out[1][2] = q2;
        }
        return 2;
    }
    return 0;
}

__device__ __forceinline__ void cube_inside(const float* f, const Grid3& g, int i, int j, int k, float iso, bool s8[8]) {
    for (int c = 0; c < 8; c++) s8[c] = f[node_lin(g, i + (c >> 2), j + ((c >> 1) & 1), k + (c & 1))] > iso;
}

__global__ void k_cube_counts(const float* __restrict__ f, Grid3 g, float iso, uint32_t* count) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long cubes = (long long)(g.n[0] - 1) * (g.n[1] - 1) * (g.n[2] - 1);
    if (q >= cubes) return;
    const int i = (int)(q / ((long long)(g.n[1] - 1) * (g.n[2] - 1))), j = (int)((q / (g.n[2] - 1)) % (g.n[1] - 1)),
              k = (int)(q % (g.n[2] - 1));
    bool s8[8];
    cube_inside(f, g, i, j, k, iso, s8);
    uint32_t n = 0;
    for (int t = 0; t < 6; t++) {
        const int c[4] = {kTet[t][0], kTet[t][1], kTet[t][2], kTet[t][3]};
        const bool s[4] = {s8[c[0]], s8[c[1]], s8[c[2]], s8[c[3]]};
        n += (uint32_t)tet_triangles(g, i, j, k, c, s, nullptr);
    }
    count[q] = n;
}

__global__ void k_cube_triangles(const float* __restrict__ f, Grid3 g, float iso, const uint32_t* __restrict__ first,
                                 const uint32_t* __restrict__ vid, int* F) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long cubes = (long long)(g.n[0] - 1) * (g.n[1] - 1) * (g.n[2] - 1);
    if (q >= cubes) return;
    const int i = (int)(q / ((long long)(g.n[1] - 1) * (g.n[2] - 1))), j = (int)((q / (g.n[2] - 1)) % (g.n[1] - 1)),
              k = (int)(q % (g.n[2] - 1));
    bool s8[8];
    cube_inside(f, g, i, j, k, iso, s8);
    long long o = first[q];
    for (int t = 0; t < 6; t++) {
        const int c[4] = {kTet[t][0], kTet[t][1], kTet[t][2], kTet[t][3]};
        const bool s[4] = {s8[c[0]], s8[c[1]], s8[c[2]], s8[c[3]]};
        long long tri[2][3];
        const int m = tet_triangles(g, i, j, k, c, s, tri);
        for (int u = 0; u < m; u++, o++)
            for (int a = 0; a < 3; a++) F[3 * o + a] = (int)vid[tri[u][a]];
    }
}

// ---------------------------------------------------------------- host helpers
struct Dev {
    std::vector<void*> ptrs;
    ~Dev() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T> T* alloc(size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, count * sizeof(T) + 16) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return (T*)p;
    }
};

// exclusive sum of n u32 in place; grand total into *grand_host
bool exclusive_scan(uint32_t* d, long long n, Dev& dev, uint32_t* grand_host) {
    if (n > 0x7fffffffLL) return false;
    const int tiles = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
    uint32_t* tot = dev.alloc<uint32_t>((size_t)tiles + 1);
    uint32_t* grand = dev.alloc<uint32_t>(1);
    if (!tot || !grand) return false;
    k_scan_tiles<OpSum><<<tiles, SCAN_THREADS>>>(d, (int)n, tot);
    k_scan_totals<OpSum><<<1, 1024>>>(tot, tiles, grand);
    k_scan_add<OpSum><<<tiles, SCAN_THREADS>>>(d, (int)n, tot);
    return cudaMemcpy(grand_host, grand, 4, cudaMemcpyDeviceToHost) == cudaSuccess;
}

bool make_grid(const int* dims, float dx, const float* mn, Grid3& g) {
    if (!dims || !mn || !(dx > 0.f)) return false;
    long long total = 1;
    for (int a = 0; a < 3; a++) {
        if (dims[a] < 1 || dims[a] > (1 << 20)) return false;
        g.n[a] = dims[a];
        g.mn[a] = mn[a];
        total *= dims[a];
    }
    g.dx = dx;
    return total <= (1LL << 31);
}

long long cells(const Grid3& g) { return (long long)g.n[0] * g.n[1] * g.n[2]; }
unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

int finish(cudaError_t e) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        return DMPM_ERR_CUDA;
    }
    return DMPM_OK;
}

}  // namespace
}  // namespace dmpm

using namespace dmpm;

extern "C" int dmpm_surface_grid_dims(const float* min_point, const float* max_point, float dx, int* dims) {
    if (!min_point || !max_point || !dims || !(dx > 0.f)) return DMPM_ERR_ARG;
    const float ext = max_point[0] - min_point[0];
    const double d = std::ceil((double)(ext / dx));  // SphereUnionSurfacing.cpp:13-16: the x extent on every axis
    if (!(d >= 1.0) || d > (double)(1 << 20)) return DMPM_ERR_ARG;
    dims[0] = dims[1] = dims[2] = (int)d;
    return DMPM_OK;
}

extern "C" int dmpm_surface_p2g_mass(const float* points, int64_t n, float mp_m, const int* dims, float dx,
                                     const float* min_point, float* mass) {
    Grid3 g;
    if (n < 0 || (n > 0 && !points) || !mass || !make_grid(dims, dx, min_point, g)) return DMPM_ERR_ARG;
    Dev dev;
    float* dp = dev.alloc<float>((size_t)3 * (size_t)(n > 0 ? n : 1));
    float* dm = dev.alloc<float>((size_t)cells(g));
    if (!dp || !dm) return DMPM_ERR_OOM;
    if (n > 0 && cudaMemcpy(dp, points, (size_t)n * 12, cudaMemcpyHostToDevice) != cudaSuccess) return finish(cudaErrorUnknown);
    if (cudaMemset(dm, 0, (size_t)cells(g) * 4) != cudaSuccess) return finish(cudaErrorUnknown);
    if (n > 0) k_p2g_mass_points<<<blocks_for(n), 256>>>(dp, n, mp_m, g, dm);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return finish(e);
    return finish(cudaMemcpy(mass, dm, (size_t)cells(g) * 4, cudaMemcpyDeviceToHost));
}

extern "C" int dmpm_surface_g2g_mass(const float* mass1, const int* dims1, float dx1, const float* min1,
                                     const int* dims2, float dx2, const float* min2, float* mass2) {
    Grid3 g1, g2;
    if (!mass1 || !mass2 || !make_grid(dims1, dx1, min1, g1) || !make_grid(dims2, dx2, min2, g2)) return DMPM_ERR_ARG;
    Dev dev;
    float* d1 = dev.alloc<float>((size_t)cells(g1));
    float* d2 = dev.alloc<float>((size_t)cells(g2));
    if (!d1 || !d2) return DMPM_ERR_OOM;
    if (cudaMemcpy(d1, mass1, (size_t)cells(g1) * 4, cudaMemcpyHostToDevice) != cudaSuccess) return finish(cudaErrorUnknown);
    k_g2g_mass<<<blocks_for(cells(g2)), 256>>>(d1, g1, g2, d2);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return finish(e);
    return finish(cudaMemcpy(mass2, d2, (size_t)cells(g2) * 4, cudaMemcpyDeviceToHost));
}

extern "C" int dmpm_surface_sphere_field(const float* points, int64_t n, float radius, int blur_iterations,
                                         const int* dims, float dx, const float* min_point, float* field) {
    Grid3 g;
    if (n < 0 || (n > 0 && !points) || !field || !(radius > 0.f) || blur_iterations < 0 ||
        !make_grid(dims, dx, min_point, g))
        return DMPM_ERR_ARG;
    Dev dev;
    float* dp = dev.alloc<float>((size_t)3 * (size_t)(n > 0 ? n : 1));
    float* a = dev.alloc<float>((size_t)cells(g));
    float* b = dev.alloc<float>((size_t)cells(g));
    if (!dp || !a || !b) return DMPM_ERR_OOM;
    if (n > 0 && cudaMemcpy(dp, points, (size_t)n * 12, cudaMemcpyHostToDevice) != cudaSuccess) return finish(cudaErrorUnknown);
    if (cudaMemset(a, 0, (size_t)cells(g) * 4) != cudaSuccess) return finish(cudaErrorUnknown);
    if (n > 0) k_sphere_max<<<blocks_for(n), 256>>>(dp, n, radius, g, (int*)a);
    // blur passes ping-pong; border nodes keep the unblurred values in both buffers
    if (cudaMemcpy(b, a, (size_t)cells(g) * 4, cudaMemcpyDeviceToDevice) != cudaSuccess) return finish(cudaErrorUnknown);
    for (int it = 0; it < blur_iterations; it++) {
        k_box_blur<<<blocks_for(cells(g)), 256>>>(a, g, b);
        float* t = a;
        a = b;
        b = t;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return finish(e);
    return finish(cudaMemcpy(field, a, (size_t)cells(g) * 4, cudaMemcpyDeviceToHost));
}

extern "C" int dmpm_surface_extract(const float* field, const int* dims, float dx, const float* min_point, float iso,
                                    float* V, int64_t v_capacity, int* F, int64_t f_capacity, int64_t* nv,
                                    int64_t* nf) {
    Grid3 g;
    if (!field || !nv || !nf || v_capacity < 0 || f_capacity < 0 || (v_capacity > 0 && !V) ||
        (f_capacity > 0 && !F) || !make_grid(dims, dx, min_point, g))
        return DMPM_ERR_ARG;
    if (g.n[0] < 2 || g.n[1] < 2 || g.n[2] < 2) {
        *nv = *nf = 0;
        return DMPM_OK;
    }
    const long long N = cells(g), E = N * 7, C = (long long)(g.n[0] - 1) * (g.n[1] - 1) * (g.n[2] - 1);
    if (E > 0x7fffffffLL) return DMPM_ERR_TOO_LARGE;
    Dev dev;
    float* df = dev.alloc<float>((size_t)N);
    uint32_t* flag = dev.alloc<uint32_t>((size_t)E);
    uint32_t* vid = dev.alloc<uint32_t>((size_t)E);
    uint32_t* first = dev.alloc<uint32_t>((size_t)C);
    if (!df || !flag || !vid || !first) return DMPM_ERR_OOM;
    if (cudaMemcpy(df, field, (size_t)N * 4, cudaMemcpyHostToDevice) != cudaSuccess) return finish(cudaErrorUnknown);
    k_edge_flags<<<blocks_for(E), 256>>>(df, g, iso, flag);
    if (cudaMemcpy(vid, flag, (size_t)E * 4, cudaMemcpyDeviceToDevice) != cudaSuccess) return finish(cudaErrorUnknown);
    uint32_t nverts = 0, ntris = 0;
    if (!exclusive_scan(vid, E, dev, &nverts)) return finish(cudaErrorUnknown);
    k_cube_counts<<<blocks_for(C), 256>>>(df, g, iso, first);
    if (!exclusive_scan(first, C, dev, &ntris)) return finish(cudaErrorUnknown);
    *nv = nverts;
    *nf = ntris;
    if ((int64_t)nverts > v_capacity || (int64_t)ntris > f_capacity) return DMPM_ERR_TOO_LARGE;
    float* dV = dev.alloc<float>((size_t)3 * nverts + 3);
    int* dF = dev.alloc<int>((size_t)3 * ntris + 3);
    if (!dV || !dF) return DMPM_ERR_OOM;
    k_edge_vertices<<<blocks_for(E), 256>>>(df, g, iso, flag, vid, dV);
    k_cube_triangles<<<blocks_for(C), 256>>>(df, g, iso, first, vid, dF);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return finish(e);
    if (nverts && cudaMemcpy(V, dV, (size_t)nverts * 12, cudaMemcpyDeviceToHost) != cudaSuccess) return finish(cudaErrorUnknown);
    if (ntris && cudaMemcpy(F, dF, (size_t)ntris * 12, cudaMemcpyDeviceToHost) != cudaSuccess) return finish(cudaErrorUnknown);
    return DMPM_OK;
}
