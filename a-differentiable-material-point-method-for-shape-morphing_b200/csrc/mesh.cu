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
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "dmpm.h"

namespace {

constexpr int kTriTile = 256;

__global__ void __launch_bounds__(256) k_mesh_winding(const float* __restrict__ tri, int nf, float mnx, float mny,
                                                      float mnz, float dx, int d0, int d1, int d2,
                                                      uint8_t* __restrict__ inside) {
    __shared__ float s_tri[kTriTile * 9];
    const long long total = (long long)d0 * d1 * d2;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = idx < total;
    const long long q = valid ? idx : 0;
    const int i = (int)(q / ((long long)d1 * d2)), j = (int)((q / d2) % d1), k = (int)(q % d2);
    // min_point + sampling_dx * Vec3(i, j, k): a product and a sum, each rounded to float
    const double px = (double)__fadd_rn(mnx, __fmul_rn(dx, (float)i));
    const double py = (double)__fadd_rn(mny, __fmul_rn(dx, (float)j));
    const double pz = (double)__fadd_rn(mnz, __fmul_rn(dx, (float)k));
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
    const int st = dmpm_mesh_lattice_dims(min_point, max_point, sampling_dx, dims);
    if (st != DMPM_OK) return st;
    const long long total = (long long)dims[0] * dims[1] * dims[2];
    if (total > (1ll << 31)) return DMPM_ERR_TOO_LARGE;
    std::vector<float> tri((size_t)nf * 9);
    for (int f = 0; f < nf; f++)
        for (int c = 0; c < 3; c++) {
            const int v = F[3 * f + c];
            if (v < 0 || v >= nv) return DMPM_ERR_ARG;
            std::memcpy(&tri[(size_t)f * 9 + 3 * c], V + 3 * (size_t)v, 3 * sizeof(float));
        }
    float* dtri = nullptr;
    uint8_t* dmask = nullptr;
    if (cudaMalloc(&dtri, tri.size() * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dmask, (size_t)total) != cudaSuccess) {
        cudaFree(dtri);
        cudaGetLastError();
        return DMPM_ERR_OOM;
    }
    std::vector<uint8_t> mask((size_t)total);
    int rc = DMPM_OK;
    if (cudaMemcpy(dtri, tri.data(), tri.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = DMPM_ERR_CUDA;
    } else {
        const unsigned blocks = (unsigned)((total + 255) / 256);
        k_mesh_winding<<<blocks, 256>>>(dtri, nf, min_point[0], min_point[1], min_point[2], sampling_dx, dims[0],
                                        dims[1], dims[2], dmask);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(mask.data(), dmask, (size_t)total, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = DMPM_ERR_CUDA;
    }
    cudaFree(dtri);
    cudaFree(dmask);
    if (rc != DMPM_OK) {
        cudaGetLastError();
        return rc;
    }
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
