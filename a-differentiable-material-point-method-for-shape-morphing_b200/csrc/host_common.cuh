// host_common.cuh -- host-side helpers shared by the one-scene engine
// (engine.cu) and the batch engine (batch.cu): error types, the CUDA call
// check, the device allocation owner and the SoA <-> row-major copy kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace dmpm_host {

struct CudaError {
    cudaError_t code;
    std::string what;
};

#define DMPM_CK(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) throw CudaError{e_, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

struct ArgError {
    std::string what;
};
struct StateError {
    std::string what;
};

inline size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }

// Device bytes held by the arenas of one context, and an optional cap on them
// (0 = none): an allocation that would go above the cap fails the way a failed
// cudaMalloc does, with cudaErrorMemoryAllocation, before any device call.
struct DeviceBudget {
    size_t cap = 0;
    size_t used = 0;
};

// Device allocation owner.
class Arena {
   public:
    Arena() = default;
    explicit Arena(DeviceBudget* budget) : budget_(budget) {}
    void set_budget(DeviceBudget* budget) { budget_ = budget; }  // before the first allocation
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;
    ~Arena() { release(); }
    void* alloc(size_t bytes) {
        if (bytes == 0) return nullptr;
        const size_t want = round_up(bytes, 256);
        if (budget_ && budget_->cap && budget_->used + want > budget_->cap)
            throw CudaError{cudaErrorMemoryAllocation, "allocation of " + std::to_string(bytes) +
                                                           " bytes exceeds the context's device byte limit of " +
                                                           std::to_string(budget_->cap)};
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw CudaError{e, "cudaMalloc(" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e)};
        }
        ptrs_.push_back(p);
        bytes_ += want;
        if (budget_) budget_->used += want;
        return p;
    }
    void release() {
        for (void* p : ptrs_) cudaFree(p);
        ptrs_.clear();
        if (budget_) budget_->used -= bytes_;
        bytes_ = 0;
    }
    size_t bytes() const { return bytes_; }

   private:
    DeviceBudget* budget_ = nullptr;
    std::vector<void*> ptrs_;
    size_t bytes_ = 0;
};


// ---------------------------------------------------------------- layout kernels
// Host arrays hold width values per particle in the caller's order; device
// planes hold particle i at plane offset i.  perm (or null: the identity) maps
// a device index to the caller's index, for a cloud stored in cell order.
__device__ __forceinline__ size_t caller_index(const uint32_t* perm, int i) { return perm ? perm[i] : (size_t)i; }
template <class T>
__global__ void k_unpack(const double* __restrict__ src, int width, int n, T* dst, size_t np,
                         const uint32_t* __restrict__ perm = nullptr) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * width) return;
    const int i = (int)(t / width), q = (int)(t % width);
    dst[(size_t)q * np + i] = (T)src[caller_index(perm, i) * width + q];
}
template <class T>
__global__ void k_pack(const T* __restrict__ src, size_t np, int width, int n, double* dst,
                       const uint32_t* __restrict__ perm = nullptr) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * width) return;
    const int i = (int)(t / width), q = (int)(t % width);
    dst[caller_index(perm, i) * width + q] = (double)src[(size_t)q * np + i];
}
// dst plane q, entry i = src plane q, entry perm[i] (planes planes of stride np)
template <class T>
__global__ void k_gather_planes(const T* __restrict__ src, int planes, size_t np, int n,
                                const uint32_t* __restrict__ perm, T* dst) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * planes) return;
    const int q = (int)(t / n), i = (int)(t % n);
    dst[(size_t)q * np + i] = src[(size_t)q * np + perm[i]];
}
// n x 3 doubles to compensated position planes (three hi planes from hi, three
// lo planes from lo, plane stride np): hi = the float nearest x, lo = the float
// nearest x - hi; and back, x = hi + lo
static __global__ void k_unpack_x2(const double* __restrict__ src, int n, float* hi, float* lo, size_t np,
                                   const uint32_t* __restrict__ perm = nullptr) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * 3) return;
    const int i = (int)(t / 3), c = (int)(t % 3);
    const size_t o = (size_t)c * np + i;
    const double x = src[caller_index(perm, i) * 3 + c];
    const float h = (float)x;
    hi[o] = h;
    lo[o] = (float)(x - (double)h);
}
static __global__ void k_pack_x2(const float* __restrict__ hi, const float* __restrict__ lo, size_t np, int n,
                                 double* dst, const uint32_t* __restrict__ perm = nullptr) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * 3) return;
    const int i = (int)(t / 3), c = (int)(t % 3);
    const size_t o = (size_t)c * np + i;
    dst[caller_index(perm, i) * 3 + c] = (double)hi[o] + (double)lo[o];
}
// add s to the diagonal (entries 0, 4, 8) of n 3x3 matrices stored as 9
// consecutive doubles each: F <-> the FP32 path's strain planes H = F - I
static __global__ void k_diag_add(double* a, int n, double s) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * 3) return;
    a[9 * (i / 3) + 4 * (i % 3)] += s;
}
template <class T>
__global__ void k_pack_acc(const double* __restrict__ src, size_t np, int n, double* dst,
                           const uint32_t* __restrict__ perm = nullptr) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * 9) return;
    const int i = (int)(t / 9), q = (int)(t % 9);
    dst[caller_index(perm, i) * 9 + q] = src[(size_t)q * np + i];
}
}  // namespace dmpm_host
