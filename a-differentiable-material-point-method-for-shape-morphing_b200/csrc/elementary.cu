// elementary.cu -- batched per-matrix functions of Elasticity.h on the GPU
// (FP64): the fixed-corotated stress, its derivative applied to a direction,
// the polar decomposition and the energy.  The reference calls these per
// particle from its loops (Elasticity.cpp:74-178); here a batch of matrices
// is evaluated in one launch with the same device code the hot-path kernels
// use (svd3.cuh, elasticity.cuh).
#include <cuda_runtime.h>

#include "dmpm.h"
#include "elasticity.cuh"

namespace {

using namespace dmpm;

__device__ m3<double> ld_cm(const double* a) {
    m3<double> m;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) m.a[i][j] = a[i + 3 * j];
    return m;
}
__device__ void st_cm(const m3<double>& m, double* a) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) a[i + 3 * j] = m.a[i][j];
}

__global__ void k_elementary(int kind, int n, const double* __restrict__ F, const double* __restrict__ lam,
                             const double* __restrict__ mu, const double* __restrict__ dF, double* out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const m3<double> f = ld_cm(F + 9 * (size_t)p);
    switch (kind) {
        case DMPM_ELEM_PK:
            st_cm(pk_stress<double>(f, lam[p], mu[p]), out + 9 * (size_t)p);
            break;
        case DMPM_ELEM_D2_REFCOMPAT:
            st_cm(d2_mult<false>(f, lam[p], mu[p], ld_cm(dF + 9 * (size_t)p)), out + 9 * (size_t)p);
            break;
        case DMPM_ELEM_D2_EXACT:
            st_cm(d2_mult<true>(f, lam[p], mu[p], ld_cm(dF + 9 * (size_t)p)), out + 9 * (size_t)p);
            break;
        case DMPM_ELEM_POLAR: {
            m3<double> R, S;
            polar3(f, R, S);
            st_cm(R, out + 18 * (size_t)p);
            st_cm(S, out + 18 * (size_t)p + 9);
            break;
        }
        case DMPM_ELEM_ENERGY: {  // FixedCorotatedElasticity (Elasticity.cpp:74-86)
            m3<double> U, V;
            double s[3];
            svd3(f, U, s, V);
            double J = det3(f);
            J = J > 1e-6 ? J : 1e-6;
            out[p] = mu[p] * ((s[0] - 1) * (s[0] - 1) + (s[1] - 1) * (s[1] - 1) + (s[2] - 1) * (s[2] - 1)) +
                     0.5 * lam[p] * (J - 1) * (J - 1);
            break;
        }
    }
}

}  // namespace

extern "C" int dmpm_elementary(int kind, int n, const double* F, const double* lam, const double* mu,
                               const double* dF, double* out) {
    if (n < 0 || kind < DMPM_ELEM_PK || kind > DMPM_ELEM_ENERGY) return DMPM_ERR_ARG;
    if (n == 0) return DMPM_OK;
    if (!F || !lam || !mu || !out) return DMPM_ERR_ARG;
    const bool needs_dF = kind == DMPM_ELEM_D2_REFCOMPAT || kind == DMPM_ELEM_D2_EXACT;
    if (needs_dF && !dF) return DMPM_ERR_ARG;
    const size_t w_out = kind == DMPM_ELEM_POLAR ? 18 : (kind == DMPM_ELEM_ENERGY ? 1 : 9);
    const size_t bytes_in = (size_t)n * (9 + 1 + 1 + (needs_dF ? 9 : 0)) * sizeof(double);
    const size_t bytes_out = (size_t)n * w_out * sizeof(double);
    char* buf = nullptr;
    if (cudaMalloc(&buf, bytes_in + bytes_out) != cudaSuccess) {
        cudaGetLastError();
        return DMPM_ERR_OOM;
    }
    double* dFm = (double*)buf;
    double* dl = dFm + 9 * (size_t)n;
    double* dm = dl + n;
    double* ddF = dm + n;
    double* dout = (double*)(buf + bytes_in);
    int st = DMPM_OK;
    if (cudaMemcpy(dFm, F, 9 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dl, lam, (size_t)n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dm, mu, (size_t)n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        (needs_dF && cudaMemcpy(ddF, dF, 9 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)) {
        st = DMPM_ERR_CUDA;
    } else {
        k_elementary<<<(n + 127) / 128, 128>>>(kind, n, dFm, dl, dm, needs_dF ? ddF : nullptr, dout);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(out, dout, bytes_out, cudaMemcpyDeviceToHost) != cudaSuccess)
            st = DMPM_ERR_CUDA;
    }
    cudaFree(buf);
    if (st != DMPM_OK) cudaGetLastError();
    return st;
}
