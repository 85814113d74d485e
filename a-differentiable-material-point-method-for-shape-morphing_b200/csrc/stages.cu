// stages.cu -- single forward stages on the GPU for callers that drive the
// reference's stage-level API (SingleThreadMPM::G_op, G2P, P_op_2;
// ForwardSimulation.h:29-35) on their own grids and clouds instead of whole
// time steps.  The engine's time step (dmpm_forward) runs the same stages fused;
// these entry points take host arrays (floats, 3x3 matrices column-major, grid
// arrays in node order (i * dim_y + j) * dim_z + k), allocate their device
// scratch, run on the default stream and synchronise.
//
//   dmpm_stage_g_op   SingleNode_op over the grid (ForwardSimulation.cpp:53-58, 184-224):
//                     v = p / m + dt f where |m| > FLT_EPSILON, v unchanged elsewhere; f is
//                     f_ext, or gravity_mag times the unit vector from the node towards
//                     gravity_point (zero where every component of that vector is within
//                     1e-5, as Eigen's isZero() decides)
//   dmpm_stage_g2p    Grid_to_SingleParticle (ForwardSimulation.cpp:60-106): v' = sum w v_g,
//                     C' = 3/dx^2 sum w v_g (x_g - x_p)^T over the in-grid stencil nodes
//   dmpm_stage_p_op_2 SingleParticle_op_2 (ForwardSimulation.cpp:108-124):
//                     F' = (1 - s)(I + dt C')(F + dFc) + s F, x' = x + dt v'
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "dmpm.h"

namespace {

constexpr float kEps = 1.1920928955078125e-07f;  // FLT_EPSILON, the reference's node-mass threshold

struct Buf {
    std::vector<void*> ptrs;
    ~Buf() {
        for (void* p : ptrs) cudaFree(p);
    }
    float* get(size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, (count > 0 ? count : 1) * sizeof(float)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return (float*)p;
    }
};

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return DMPM_OK;
    cudaGetLastError();
    return DMPM_ERR_CUDA;
}

unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

__device__ __forceinline__ float bspline(float x) {  // CubicBSpline (Interpolation.h:5-17)
    x = fabsf(x);
    if (x < 1.f) return 0.5f * x * x * x - x * x + 2.f / 3.f;
    if (x < 2.f) return (2.f - x) * (2.f - x) * (2.f - x) / 6.f;
    return 0.f;
}

struct GridDesc {
    int n[3];
    float dx, mn[3];
};

__global__ void k_stage_g_op(GridDesc g, const float* __restrict__ m, const float* __restrict__ p, float dt, float f0,
                             float f1, float f2, int point_gravity, float gx, float gy, float gz, float gmag,
                             float* v) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    if (q >= total) return;
    const float mq = m[q];
    if (!(fabsf(mq) > kEps)) return;  // the reference leaves v as it is
    float f[3] = {f0, f1, f2};
    if (point_gravity) {
        const int i = (int)(q / ((long long)g.n[1] * g.n[2])), j = (int)((q / g.n[2]) % g.n[1]), k = (int)(q % g.n[2]);
        const int id[3] = {i, j, k};
        const float gp[3] = {gx, gy, gz};
        float d[3], nn = 0.f;
        bool zero = true;  // Eigen's isZero(): every component within 1e-5 (float's dummy precision)
        for (int a = 0; a < 3; a++) {
            d[a] = gp[a] - (g.mn[a] + (float)id[a] * g.dx);
            nn += d[a] * d[a];
            zero = zero && fabsf(d[a]) <= 1e-5f;
        }
        if (zero) {
            f[0] = f[1] = f[2] = 0.f;
        } else {
            const float len = sqrtf(nn);
            for (int a = 0; a < 3; a++) f[a] = d[a] / len * gmag;
        }
    }
    for (int a = 0; a < 3; a++) v[3 * q + a] = p[3 * q + a] / mq + dt * f[a];
}

__global__ void k_stage_g2p(int n, const float* __restrict__ x, GridDesc g, const float* __restrict__ gv, float* v_out,
                            float* C_out) {
    const int pi = blockIdx.x * blockDim.x + threadIdx.x;
    if (pi >= n) return;
    const float xp[3] = {x[3 * pi], x[3 * pi + 1], x[3 * pi + 2]};
    int b[3];
    for (int a = 0; a < 3; a++) b[a] = (int)floorf((xp[a] - g.mn[a]) / g.dx) - 1;
    const float k3 = 3.f / (g.dx * g.dx);
    float v[3] = {0.f, 0.f, 0.f}, C[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++) {
                const int id[3] = {b[0] + i, b[1] + j, b[2] + k};
                if (id[0] < 0 || id[0] >= g.n[0] || id[1] < 0 || id[1] >= g.n[1] || id[2] < 0 || id[2] >= g.n[2])
                    continue;
                float d[3];
                for (int a = 0; a < 3; a++) d[a] = (g.mn[a] + (float)id[a] * g.dx) - xp[a];
                const float w = bspline(d[0] / g.dx) * bspline(d[1] / g.dx) * bspline(d[2] / g.dx);
                const long long q = ((long long)id[0] * g.n[1] + id[1]) * g.n[2] + id[2];
                const float vg[3] = {gv[3 * q], gv[3 * q + 1], gv[3 * q + 2]};
                for (int r = 0; r < 3; r++) {
                    v[r] += w * vg[r];
                    for (int c = 0; c < 3; c++) C[r][c] += k3 * w * vg[r] * d[c];
                }
            }
    for (int r = 0; r < 3; r++) {
        v_out[3 * pi + r] = v[r];
        for (int c = 0; c < 3; c++) C_out[9 * pi + r + 3 * c] = C[r][c];  // column-major
    }
}

__global__ void k_stage_p_op_2(int n, const float* __restrict__ x, const float* __restrict__ F,
                               const float* __restrict__ dFc, const float* __restrict__ v, const float* __restrict__ C,
                               float dt, float s, float* x_out, float* F_out) {
    const int pi = blockIdx.x * blockDim.x + threadIdx.x;
    if (pi >= n) return;
    const float* Fp = F + 9 * (size_t)pi;
    const float* Dp = dFc + 9 * (size_t)pi;
    const float* Cp = C + 9 * (size_t)pi;
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            float t = 0.f;  // ((I + dt C)(F + dFc))(r, c), column-major storage (r + 3 c)
            for (int k = 0; k < 3; k++) {
                const float a = (r == k ? 1.f : 0.f) + dt * Cp[r + 3 * k];
                t += a * (Fp[k + 3 * c] + Dp[k + 3 * c]);
            }
            F_out[9 * (size_t)pi + r + 3 * c] = t * (1.f - s) + Fp[r + 3 * c] * s;
        }
    for (int a = 0; a < 3; a++) x_out[3 * pi + a] = x[3 * pi + a] + dt * v[3 * pi + a];
}

bool grid_desc(int dx_, int dy_, int dz_, float dx, const float* mn, GridDesc& g) {
    if (dx_ < 1 || dy_ < 1 || dz_ < 1 || !(dx > 0.f) || !mn) return false;
    if ((long long)dx_ * dy_ * dz_ > (1LL << 31)) return false;
    g.n[0] = dx_;
    g.n[1] = dy_;
    g.n[2] = dz_;
    g.dx = dx;
    for (int a = 0; a < 3; a++) g.mn[a] = mn[a];
    return true;
}

}  // namespace

extern "C" int dmpm_stage_g_op(int dim_x, int dim_y, int dim_z, float dx, const float* min_point, const float* m,
                               const float* p, float dt, const float* f_ext, const float* gravity_point,
                               float gravity_mag, float* v) {
    GridDesc g;
    if (!grid_desc(dim_x, dim_y, dim_z, dx, min_point, g) || !m || !p || !v || (!f_ext && !gravity_point))
        return DMPM_ERR_ARG;
    const size_t G = (size_t)dim_x * dim_y * dim_z;
    Buf b;
    float *dm = b.get(G), *dp = b.get(3 * G), *dv = b.get(3 * G);
    if (!dm || !dp || !dv) return DMPM_ERR_OOM;
    cudaError_t e = cudaMemcpy(dm, m, G * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dp, p, 3 * G * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dv, v, 3 * G * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e);
    const float f0 = f_ext ? f_ext[0] : 0.f, f1 = f_ext ? f_ext[1] : 0.f, f2 = f_ext ? f_ext[2] : 0.f;
    k_stage_g_op<<<blocks_for((long long)G), 256>>>(g, dm, dp, dt, f0, f1, f2, gravity_point ? 1 : 0,
                                                      gravity_point ? gravity_point[0] : 0.f,
                                                      gravity_point ? gravity_point[1] : 0.f,
                                                      gravity_point ? gravity_point[2] : 0.f, gravity_mag, dv);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(v, dv, 3 * G * 4, cudaMemcpyDeviceToHost);
    return cuda_status(e);
}

extern "C" int dmpm_stage_g2p(int n, const float* x, int dim_x, int dim_y, int dim_z, float dx, const float* min_point,
                              const float* grid_v, float* v_out, float* C_out) {
    GridDesc g;
    if (n < 0 || (n > 0 && (!x || !v_out || !C_out)) || !grid_v || !grid_desc(dim_x, dim_y, dim_z, dx, min_point, g))
        return DMPM_ERR_ARG;
    if (n == 0) return DMPM_OK;
    const size_t G = (size_t)dim_x * dim_y * dim_z;
    Buf b;
    float *dx_ = b.get(3 * (size_t)n), *dg = b.get(3 * G), *dv = b.get(3 * (size_t)n), *dC = b.get(9 * (size_t)n);
    if (!dx_ || !dg || !dv || !dC) return DMPM_ERR_OOM;
    cudaError_t e = cudaMemcpy(dx_, x, 12 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dg, grid_v, 12 * G, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e);
    k_stage_g2p<<<blocks_for(n), 256>>>(n, dx_, g, dg, dv, dC);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(v_out, dv, 12 * (size_t)n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(C_out, dC, 36 * (size_t)n, cudaMemcpyDeviceToHost);
    return cuda_status(e);
}

extern "C" int dmpm_stage_p_op_2(int n, const float* x, const float* F, const float* dFc, const float* v,
                                 const float* C, float dt, float smoothing, float* x_out, float* F_out) {
    if (n < 0 || (n > 0 && (!x || !F || !dFc || !v || !C || !x_out || !F_out))) return DMPM_ERR_ARG;
    if (n == 0) return DMPM_OK;
    Buf b;
    const size_t N = (size_t)n;
    float *dx_ = b.get(3 * N), *dF = b.get(9 * N), *dD = b.get(9 * N), *dv = b.get(3 * N), *dC = b.get(9 * N),
          *ox = b.get(3 * N), *oF = b.get(9 * N);
    if (!dx_ || !dF || !dD || !dv || !dC || !ox || !oF) return DMPM_ERR_OOM;
    cudaError_t e = cudaMemcpy(dx_, x, 12 * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dF, F, 36 * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dD, dFc, 36 * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dv, v, 12 * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dC, C, 36 * N, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e);
    k_stage_p_op_2<<<blocks_for(n), 256>>>(n, dx_, dF, dD, dv, dC, dt, smoothing, ox, oF);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(x_out, ox, 12 * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(F_out, oF, 36 * N, cudaMemcpyDeviceToHost);
    return cuda_status(e);
}
