// mesh.cu -- point cloud of a watertight triangle mesh on the GPU
// (dmpm_mesh_lattice_points, include/dmpm.h): the reference's
// GeometryLoading::GeneratePointCloudFromWatertightTriangleMesh
// (GeometryLoading.cpp:10-83), which keeps the points of the lattice
// min_point + sampling_dx (i, j, k) whose libigl signed distance with the
// winding-number sign is <= 0, i.e. whose winding number w >= 1/2
// (s = 1 - 2 w, S = s |d|; points exactly on the surface are left out here,
// see the header).
//
// One thread per lattice point sums the solid angles of all triangles in
// FP64 -- each by the formula of Van Oosterom and Strackee (1983),
// tan(Omega / 2) = a.(b x c) / (|a||b||c| + (a.b)|c| + (b.c)|a| + (c.a)|b|)
// with a, b, c the triangle's vertices relative to the point -- reading the
// triangles in tiles staged in shared memory by the whole block.  The lattice
// coordinates are formed in float with the reference's two roundings.
//
// dmpm_mesh_jittered_points uses the same inside test for jittered stratified
// sampling (the synthetic scenes' "per_axis^3 points per cell, one uniformly
// jittered point per sub-cell"), with a counter-based jitter so that the points
// depend only on the seed and the sub-cell, not on the launch.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "dmpm.h"

namespace {

constexpr int kTriTile = 256;

// the lattice point min_point + sampling_dx * (i, j, k): a product and a sum, each rounded to float
struct LatticePoints {
    float mn[3], dx;
    __device__ void operator()(int i, int j, int k, double p[3]) const {
        const int id[3] = {i, j, k};
        for (int a = 0; a < 3; a++) p[a] = (double)__fadd_rn(mn[a], __fmul_rn(dx, (float)id[a]));
    }
};

// SplitMix64 (Steele, Lea and Flood 2014): the 64-bit finaliser of a Weyl sequence
__host__ __device__ inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// one uniformly jittered point per sub-cell (i, j, k) of spacing sdx:
// min + (index + u) * sdx, u = top 24 bits of splitmix64(seed + 3 q + axis) / 2^24,
// q the sub-cell's linear index -- reproducible on any host
struct JitteredPoints {
    float mn[3], sdx;
    int d1, d2;
    uint64_t seed;
    __device__ void operator()(int i, int j, int k, double p[3]) const {
        const int id[3] = {i, j, k};
        const uint64_t q = ((uint64_t)i * d1 + j) * d2 + k;
        for (int a = 0; a < 3; a++) {
            const float u = (float)(splitmix64(seed + 3 * q + a) >> 40) * (1.f / 16777216.f);
            p[a] = (double)__fadd_rn(mn[a], __fmul_rn(__fadd_rn((float)id[a], u), sdx));
        }
    }
};

template <class Points>
__global__ void __launch_bounds__(256) k_mesh_winding(const float* __restrict__ tri, int nf, Points pts, int d0, int d1,
                                                      int d2, uint8_t* __restrict__ inside) {
    __shared__ float s_tri[kTriTile * 9];
    const long long total = (long long)d0 * d1 * d2;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = idx < total;
    const long long q = valid ? idx : 0;
    const int i = (int)(q / ((long long)d1 * d2)), j = (int)((q / d2) % d1), k = (int)(q % d2);
    double P[3];
    pts(i, j, k, P);
    const double px = P[0], py = P[1], pz = P[2];
    double ang = 0.0;
    for (int t0 = 0; t0 < nf; t0 += kTriTile) {
        const int cnt = min(kTriTile, nf - t0);
        __syncthreads();
        for (int e = threadIdx.x; e < cnt * 9; e += blockDim.x) s_tri[e] = tri[(size_t)t0 * 9 + e];
        __syncthreads();
        if (!valid) continue;
        for (int t = 0; t < cnt; t++) {
            const float* v = s_tri + 9 * t;
            const double ax = v[0] - px, ay = v[1] - py, az = v[2] - pz;
            const double bx = v[3] - px, by = v[4] - py, bz = v[5] - pz;
            const double cx = v[6] - px, cy = v[7] - py, cz = v[8] - pz;
            const double la = sqrt(ax * ax + ay * ay + az * az), lb = sqrt(bx * bx + by * by + bz * bz),
                         lc = sqrt(cx * cx + cy * cy + cz * cz);
            const double det = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
            const double den = la * lb * lc + (ax * bx + ay * by + az * bz) * lc + (bx * cx + by * cy + bz * cz) * la +
                               (cx * ax + cy * ay + cz * az) * lb;
            ang += atan2(det, den);  // Omega / 2
        }
    }
    if (valid) inside[idx] = (ang / (2.0 * M_PI) >= 0.5) ? 1 : 0;  // w = sum Omega / (4 pi)
}

// triangles gathered as 9 floats each, indices checked
int gather_triangles(const float* V, int nv, const int* F, int nf, std::vector<float>& tri) {
    tri.resize((size_t)nf * 9);
    for (int f = 0; f < nf; f++)
        for (int c = 0; c < 3; c++) {
            const int v = F[3 * f + c];
            if (v < 0 || v >= nv) return DMPM_ERR_ARG;
            std::memcpy(&tri[(size_t)f * 9 + 3 * c], V + 3 * (size_t)v, 3 * sizeof(float));
        }
    return DMPM_OK;
}

// the inside mask of d0 x d1 x d2 generated points on the GPU
template <class Points>
int inside_mask(const std::vector<float>& tri, int nf, const Points& pts, const int dims[3], std::vector<uint8_t>& mask) {
    const long long total = (long long)dims[0] * dims[1] * dims[2];
    float* dtri = nullptr;
    uint8_t* dmask = nullptr;
    if (cudaMalloc(&dtri, tri.size() * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dmask, (size_t)total) != cudaSuccess) {
        cudaFree(dtri);
        cudaGetLastError();
        return DMPM_ERR_OOM;
    }
    mask.resize((size_t)total);
    int rc = DMPM_OK;
    if (cudaMemcpy(dtri, tri.data(), tri.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = DMPM_ERR_CUDA;
    } else {
        const unsigned blocks = (unsigned)((total + 255) / 256);
        k_mesh_winding<Points><<<blocks, 256>>>(dtri, nf, pts, dims[0], dims[1], dims[2], dmask);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(mask.data(), dmask, (size_t)total, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = DMPM_ERR_CUDA;
    }
    cudaFree(dtri);
    cudaFree(dmask);
    if (rc != DMPM_OK) cudaGetLastError();
    return rc;
}

}  // namespace

extern "C" int dmpm_mesh_lattice_dims(const float* min_point, const float* max_point, float sampling_dx, int* dims) {
    if (!min_point || !max_point || !dims || !(sampling_dx > 0.f)) return DMPM_ERR_ARG;
    for (int a = 0; a < 3; a++) {
        const float ext = max_point[a] - min_point[a];
        const double d = std::ceil((double)(ext / sampling_dx)) + 1.0;  // GeometryLoading.cpp:21-23
        if (!(d >= 1.0) || d > 1e6) return DMPM_ERR_ARG;
        dims[a] = (int)d;
    }
    return DMPM_OK;
}

extern "C" int dmpm_mesh_lattice_points(const float* V, int nv, const int* F, int nf, const float* min_point,
                                        const float* max_point, float sampling_dx, float* out, int64_t capacity,
                                        int64_t* count) {
    if (!V || nv < 3 || !F || nf < 1 || !count || capacity < 0 || (capacity > 0 && !out)) return DMPM_ERR_ARG;
    int dims[3];
    int st = dmpm_mesh_lattice_dims(min_point, max_point, sampling_dx, dims);
    if (st != DMPM_OK) return st;
    const long long total = (long long)dims[0] * dims[1] * dims[2];
    if (total > (1ll << 31)) return DMPM_ERR_TOO_LARGE;
    std::vector<float> tri;
    if ((st = gather_triangles(V, nv, F, nf, tri)) != DMPM_OK) return st;
    LatticePoints pts{{min_point[0], min_point[1], min_point[2]}, sampling_dx};
    std::vector<uint8_t> mask;
    if ((st = inside_mask(tri, nf, pts, dims, mask)) != DMPM_OK) return st;
    // kept points in the reference's lattice order, coordinates rounded as it rounds them
    int64_t n = 0;
    for (long long q = 0; q < total; q++) {
        if (!mask[(size_t)q]) continue;
        if (n < capacity) {
            const int i = (int)(q / ((long long)dims[1] * dims[2])), j = (int)((q / dims[2]) % dims[1]),
                      k = (int)(q % dims[2]);
            volatile float t0 = sampling_dx * (float)i, t1 = sampling_dx * (float)j, t2 = sampling_dx * (float)k;
            out[3 * n] = min_point[0] + t0;
            out[3 * n + 1] = min_point[1] + t1;
            out[3 * n + 2] = min_point[2] + t2;
        }
        n++;
    }
    *count = n;
    return n > capacity ? DMPM_ERR_TOO_LARGE : DMPM_OK;
}

extern "C" int dmpm_mesh_jittered_points(const float* V, int nv, const int* F, int nf, const float* min_point,
                                         const float* max_point, float cell_dx, int per_axis, uint64_t seed,
                                         float* out, int64_t capacity, int64_t* count) {
    if (!V || nv < 3 || !F || nf < 1 || !count || capacity < 0 || (capacity > 0 && !out) || !min_point ||
        !max_point || !(cell_dx > 0.f) || per_axis < 1 || per_axis > 64)
        return DMPM_ERR_ARG;
    int dims[3];
    for (int a = 0; a < 3; a++) {
        const double c = std::ceil((double)((max_point[a] - min_point[a]) / cell_dx));
        if (!(c >= 1.0) || c * per_axis > 1e6) return DMPM_ERR_ARG;
        dims[a] = (int)c * per_axis;
    }
    const long long total = (long long)dims[0] * dims[1] * dims[2];
    if (total > (1ll << 31)) return DMPM_ERR_TOO_LARGE;
    std::vector<float> tri;
    int st = gather_triangles(V, nv, F, nf, tri);
    if (st != DMPM_OK) return st;
    const float sdx = cell_dx / (float)per_axis;
    JitteredPoints pts{{min_point[0], min_point[1], min_point[2]}, sdx, dims[1], dims[2], seed};
    std::vector<uint8_t> mask;
    if ((st = inside_mask(tri, nf, pts, dims, mask)) != DMPM_OK) return st;
    int64_t n = 0;
    for (long long q = 0; q < total; q++) {
        if (!mask[(size_t)q]) continue;
        if (n < capacity) {
            const long long id[3] = {q / ((long long)dims[1] * dims[2]), (q / dims[2]) % dims[1], q % dims[2]};
            for (int a = 0; a < 3; a++) {
                const float u = (float)(splitmix64(seed + 3 * (uint64_t)q + a) >> 40) * (1.f / 16777216.f);
                volatile float s = (float)id[a] + u;
                volatile float t = s * sdx;
                out[3 * n + a] = min_point[a] + t;
            }
        }
        n++;
    }
    *count = n;
    return n > capacity ? DMPM_ERR_TOO_LARGE : DMPM_OK;
}
