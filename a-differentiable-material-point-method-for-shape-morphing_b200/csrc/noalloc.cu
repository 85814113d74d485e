// noalloc.cu -- particle volumes (the computation of dmpm_compute_volumes)
// for callers that must not allocate device memory.
//
// Why: some callers cannot call cudaMalloc.  A simulation embedded in a
// frame loop cannot afford the device-wide synchronisation that cudaMalloc
// and cudaFree imply, and a process whose device memory is already reserved
// by another framework's caching allocator may have nothing left to hand out.
// This entry point takes the caller's device buffers for inputs and outputs
// and keeps its only scratch -- the grid of accumulated node masses -- in the
// file-scope device array below, which every GPU that loads the library
// holds until the process exits.
//
// Limits and rules:
//   * at most kNoAllocMaxNodes grid nodes (dim_x * dim_y * dim_z); larger
//     grids are rejected with DMPM_ERR_TOO_LARGE before any GPU work;
//   * all calls on a device share the one scratch array; the part a call uses
//     is cleared at the start of the call, so nothing carries over, but two
//     calls whose GPU work overlaps (different streams, or different host
//     threads) race on the array and give wrong results;
//   * the first call in each CUDA context looks the array's device address
//     up (cudaGetSymbolAddress, with that context's device current) and keeps
//     it for that context; make that first call before any stream capture.
//     The address is keyed by the context's unique id (cuCtxGetId), so a
//     caller that runs under its own (non-primary) context, or that reset the
//     device (cudaDeviceReset, after which the library's module is loaded
//     again, possibly at another address), gets the array of the context it
//     is calling from.
#include <cuda.h>  // CUcontext / CUresult for the two driver entry points below
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "dmpm.h"
#include "mat3.cuh"

namespace {

constexpr size_t kNoAllocMaxNodes = size_t(1) << 20;  // 1,048,576 nodes = 4 MiB of float

// The scratch grid.  Host code must never pass this name to a kernel: on the
// host it is a stand-in symbol, not a device address; kernels get the address
// from cudaGetSymbolAddress.
static __device__ __align__(256) float g_noalloc_mass[kNoAllocMaxNodes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
// per device: the context the address was looked up in (its unique id) and the address
struct ScratchAddr {
    unsigned long long ctx_id = 0;  // 0: not looked up yet
    float* ptr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];

struct Geom {
    int dim[3];
    float dx;
    float mn[3];
};

// mass-only P2G: m_g += w m_p (ForwardSimulation.cpp:11-51 with dt = drag = 0)
__global__ void k_na_p2g_mass(int n, const float* __restrict__ x, const float* __restrict__ m, Geom g,
                              float* grid) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)n) return;
    float xp[3];
    int base[3];
    dmpm::axis_w<float> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        xp[c] = x[3 * (size_t)p + c];
        base[c] = dmpm::stencil_base<float>(xp[c] - g.mn[c], g.dx, g.dim[c]);
        dmpm::axis_weights(xp[c], g.mn[c], g.dx, base[c], w[c], false);
    }
    const float mp = m[p];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int gi = base[0] + i, gj = base[1] + j, gk = base[2] + k;
                if (gi < 0 || gi >= g.dim[0] || gj < 0 || gj >= g.dim[1] || gk < 0 || gk >= g.dim[2]) continue;
                atomicAdd(grid + ((size_t)gi * g.dim[1] + gj) * g.dim[2] + gk, w[0].n[i] * w[1].n[j] * w[2].n[k] * mp);
            }
}

// vol_p = m_p / sum_g w m_g  (CalculatePointCloudVolumes, ForwardSimulation.cpp:262-290)
__global__ void k_na_volumes(int n, const float* __restrict__ x, const float* __restrict__ m, Geom g,
                             const float* __restrict__ grid, float* vol) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)n) return;
    float xp[3];
    int base[3];
    dmpm::axis_w<float> w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        xp[c] = x[3 * (size_t)p + c];
        base[c] = dmpm::stencil_base<float>(xp[c] - g.mn[c], g.dx, g.dim[c]);
        dmpm::axis_weights(xp[c], g.mn[c], g.dx, base[c], w[c], false);
    }
    float mg = 0.f;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int gi = base[0] + i, gj = base[1] + j, gk = base[2] + k;
                if (gi < 0 || gi >= g.dim[0] || gj < 0 || gj >= g.dim[1] || gk < 0 || gk >= g.dim[2]) continue;
                mg += w[0].n[i] * w[1].n[j] * w[2].n[k] * grid[((size_t)gi * g.dim[1] + gj) * g.dim[2] + gk];
            }
    vol[p] = (fabsf(mg) > (float)dmpm::kFltEps) ? m[p] / mg : 0.f;
}

// Unique id of the CUDA context current on the calling thread, 0 when there
// is none (or the driver cannot say).  The two driver functions come through
// the runtime's entry-point query, so the library needs no link to libcuda.
unsigned long long current_context_id() {
    using GetCurrentFn = CUresult (*)(CUcontext*);
    using GetIdFn = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {  // under g_setup_mutex
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0{}, q1{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) == cudaSuccess &&
            q0 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrentFn>(f0);
            get_id = reinterpret_cast<GetIdFn>(f1);
        }
        cudaGetLastError();
        resolved = true;
    }
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch array in the calling thread's context: looked
// up with cudaGetSymbolAddress the first time a context calls, then reused
// while that context stays current.  Where the context id cannot be read the
// address is looked up on every call.
int scratch_for_current_context(float** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return DMPM_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long id = current_context_id();
    ScratchAddr& slot = g_scratch[dev];
    if (id != 0 && slot.ctx_id == id) {
        *out = slot.ptr;
        return DMPM_OK;
    }
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_mass);
    if (e != cudaSuccess || !ptr) {
        std::fprintf(stderr, "dmpm_compute_volumes_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                     cudaGetErrorString(e));
        cudaGetLastError();
        return DMPM_ERR_CUDA;
    }
    // the lookup makes the device's primary context current when none was:
    // read the id again so the next call from this context reuses the address
    slot.ctx_id = id != 0 ? id : current_context_id();
    slot.ptr = static_cast<float*>(ptr);
    *out = slot.ptr;
    return DMPM_OK;
}

}  // namespace

extern "C" int dmpm_compute_volumes_noalloc(int n, const float* x, const float* m, int dim_x, int dim_y, int dim_z,
                                            float dx, const float* min_point, float* vol, void* stream) {
    if (n < 0 || dim_x <= 0 || dim_y <= 0 || dim_z <= 0 || !(dx > 0.f) || !min_point) return DMPM_ERR_ARG;
    if (n > 0 && (!x || !m || !vol)) return DMPM_ERR_ARG;
    const size_t G = (size_t)dim_x * (size_t)dim_y * (size_t)dim_z;
    if (G > kNoAllocMaxNodes) {
        std::fprintf(stderr,
                     "dmpm_compute_volumes_noalloc: grid of %zu nodes exceeds the no-allocation scratch capacity of "
                     "%zu nodes\n",
                     G, kNoAllocMaxNodes);
        return DMPM_ERR_TOO_LARGE;
    }
    float* grid = nullptr;
    const int st = scratch_for_current_context(&grid);
    if (st != DMPM_OK) return st;
    if (n == 0) return DMPM_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Geom g{{dim_x, dim_y, dim_z}, dx, {min_point[0], min_point[1], min_point[2]}};
    // the previous call's masses are still in the array: clear the part this call uses
    if (cudaMemsetAsync(grid, 0, G * sizeof(float), s) != cudaSuccess) {
        cudaGetLastError();
        return DMPM_ERR_CUDA;
    }
    const unsigned blocks = (unsigned)(((size_t)n + 255) / 256);
    k_na_p2g_mass<<<blocks, 256, 0, s>>>(n, x, m, g, grid);
    k_na_volumes<<<blocks, 256, 0, s>>>(n, x, m, g, grid, vol);
    return cudaGetLastError() == cudaSuccess ? DMPM_OK : DMPM_ERR_CUDA;
}
