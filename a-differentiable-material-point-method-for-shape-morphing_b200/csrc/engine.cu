// engine.cu -- host engine and C ABI (include/dmpm.h) of the B200 MLS-MPM
// forward + adjoint path.
//
// One context = one scene (point cloud, grid, target), one CUDA stream and
// its device memory.  Layers follow the reference's CompGraph
// (CompGraph.cpp:7-17, 246-267): layer 0 is the uploaded cloud, layer i+1 is
// ForwardTimeStep(layer i), EndLayerMassLoss reads the last layer, and the
// backward pass walks the layers in reverse.
//
// Layer storage.  With checkpoint interval k = 1 every layer's particle state
// (24 planes) and grid (node4 per node) stays in HBM.  With k > 1 only layers
// 0, k, 2k, ... and the last are kept; the backward pass recomputes each
// segment's states and grids from its checkpoint into segment scratch before
// running the segment's adjoint steps (recompute-in-between).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "dmpm.h"
#include "kernels.cuh"
#include "kernels_warp.cuh"
#include "kernels_brick.cuh"
#include "host_common.cuh"

using namespace dmpm;
using namespace dmpm_host;

namespace {

constexpr int kDefaultBlock = 256;
constexpr int kDefaultTileCap = 1024;

// Kernel identifiers for the per-kernel device-time accounting
// (dmpm_set_profiling / dmpm_kernel_stats).
enum KernelId {
    K_P_OP1 = 0, K_P2G, K_GOP, K_G2P, K_MASS, K_NODE_LOSS, K_LOSS_DLDX, K_ADJ_SCATTER, K_ADJ_GOP, K_ADJ_GATHER,
    K_ADJ_FINALIZE, K_ADJ_TRANSPORT, K_COUNT
};
const char* const kKernelNames[K_COUNT] = {"p_op1", "p2g", "g_op", "g2p_p_op2", "p2g_mass", "node_loss",
                                          "loss_dldx", "adj_g2p_scatter", "adj_g_op", "adj_p2g_gather",
                                          "adj_finalize", "adj_finalize_transport"};
constexpr int kDefaultSortEvery = 8;
// per-layer auxiliary planes of the FP32 path: G (9), polar R (9), polar S (6)
constexpr int kAuxPlanes = 24;

// Reference MaterialPoint (118 floats): x 0, v 3, F 6, C 15, P 24, m 33, vol 34,
// lam 35, mu 36, dFc 37 (MaterialPoint.h:18-46).
template <class T>
__global__ void k_unpack_ref(const float* __restrict__ pts, int n, size_t np, T* st, T* cst, T* dfc, T diag) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float* m = pts + (size_t)p * 118;
    for (int q = 0; q < 24; q++) st[(size_t)q * np + p] = (T)m[q];  // x v F C share the plane order
    for (int q = 0; q < 3; q++) st[(size_t)(PF + 4 * q) * np + p] += diag;  // strain planes: F - I
    cst[(size_t)KM * np + p] = (T)m[33];
    cst[(size_t)KVOL * np + p] = (T)m[34];
    cst[(size_t)KLAM * np + p] = (T)m[35];
    cst[(size_t)KMU * np + p] = (T)m[36];
    for (int q = 0; q < 9; q++) dfc[(size_t)q * np + p] = (T)m[37 + q];
}
// Grid fields of one layer.  The stored node holds (p, m), or, where the
// FP32 path's grid update has overwritten p in place (stored_v), (v, m): then
// v is read as stored and p is recovered as (v - dt f) m on nodes with
// |m| > FLT_EPSILON (0 on the others, whose momentum the update discards).
template <class T>
__global__ void k_grid_field(const node4<T>* __restrict__ g, size_t G, int field, int stored_v, double dt, double f0,
                             double f1, double f2, double* out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G) return;
    const node4<T> nd = g[i];
    if (field == DMPM_G_M) {
        out[i] = (double)nd.w;
    } else if (stored_v) {
        const double f[3] = {f0, f1, f2}, v[3] = {(double)nd.x, (double)nd.y, (double)nd.z};
        const bool occupied = fabs((double)nd.w) > kFltEps;
        for (int c = 0; c < 3; c++)
            out[3 * i + c] = field == DMPM_G_V ? v[c] : (occupied ? (v[c] - dt * f[c]) * (double)nd.w : 0.0);
    } else if (field == DMPM_G_P) {
        out[3 * i] = nd.x; out[3 * i + 1] = nd.y; out[3 * i + 2] = nd.z;
    } else {
        const T f[3] = {(T)f0, (T)f1, (T)f2};
        T v[3];
        node_velocity(nd, (T)dt, f, v);
        out[3 * i] = v[0]; out[3 * i + 1] = v[1]; out[3 * i + 2] = v[2];
    }
}
template <class T> __global__ void k_node4_field(const node4<T>* __restrict__ g, size_t G, int comp, double* out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G) return;
    const node4<T> nd = g[i];
    if (comp == 3) { out[3 * i] = nd.x; out[3 * i + 1] = nd.y; out[3 * i + 2] = nd.z; }
    else out[i] = nd.w;
}
template <class T> __global__ void k_scalar_field(const T* __restrict__ g, size_t G, double* out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < G) out[i] = (double)g[i];
}
template <class T> __global__ void k_set_node_mass(const double* __restrict__ src, size_t G, T* dst) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < G) dst[i] = (T)src[i];
}
template <class T> __global__ void k_copy_node_mass(const node4<T>* __restrict__ g, size_t G, T* dst) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < G) dst[i] = g[i].w;
}
// sum of squares of 9 planes (Compute_dLdF_Norm), FP64: block partial sums into
// part (summed in order by k_sum_partials)
template <class T> __global__ void k_sqnorm9(const T* __restrict__ a, size_t np, int n, double* part) {
    __shared__ double s[32];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (p < n)
        for (int q = 0; q < 9; q++) { const double t = (double)a[(size_t)q * np + p]; v += t * t; }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

// Adam step on one set of controls (PointCloud::Descend_Adam, PointCloud.cpp:83-99):
//   g = grad / norm;  m = b1 m + (1-b1) g;  v = b2 v + (1-b2) g^2;
//   dFc -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps)
// norm = ||grad|| from *norm2 (sum of squares) when normalising, else 1.
template <class T, class G>
__global__ void k_adam(T* dfc, const G* __restrict__ grad, T* mom, T* vec, size_t np, int n, const double* norm2,
                       int normalize, float lr, float b1, float b2, float eps, float c1, float c2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)9 * np) return;
    if ((int)(i % np) >= n) return;
    const float inv = normalize ? (float)(1.0 / sqrt(*norm2)) : 1.f;
    const float g = (float)grad[i] * inv;
    const float m = b1 * (float)mom[i] + (1.f - b1) * g;
    const float v = b2 * (float)vec[i] + (1.f - b2) * g * g;
    mom[i] = (T)m;
    vec[i] = (T)v;
    dfc[i] = (T)((float)dfc[i] - lr * ((m / c1) / (sqrtf(v / c2) + eps)));
}
// The other descent rules of PointCloud (PointCloud.cpp:101-204), one element of
// one control matrix per thread, g = grad / norm as in k_adam:
//   AMSGRAD  m, v as Adam; vmax = max(vmax, v / (1 - b2^t)); dFc -= lr (m / (1 - b1^t)) / (sqrt(vmax) + eps)
//   LION     m = b1 m + (1 - b1) sign(g); dFc -= lr m           (sign(0) = 0, SignFloat)
//   GD       dFc -= lr g
//   DLDF     d = g clipped to [-1, 1] with |d| >= 1e-3 (sign kept, 0 -> +1e-3);
//            m = 0.9 m + lr d; dFc -= m                           (Descend_dLdF)
template <class T, class G>
__global__ void k_descend(int kind, T* dfc, const G* __restrict__ grad, T* mom, T* vec, T* vmax, size_t np, int n,
                          const double* norm2, int normalize, float lr, float b1, float b2, float eps, float c1,
                          float c2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)9 * np) return;
    if ((int)(i % np) >= n) return;
    const float inv = normalize ? (float)(1.0 / sqrt(*norm2)) : 1.f;
    const float g = (float)grad[i] * inv;
    float d = (float)dfc[i];
    if (kind == DMPM_DESCEND_AMSGRAD) {
        const float m = b1 * (float)mom[i] + (1.f - b1) * g;
        const float v = b2 * (float)vec[i] + (1.f - b2) * g * g;
        const float vm = fmaxf((float)vmax[i], v / c2);
        mom[i] = (T)m;
        vec[i] = (T)v;
        vmax[i] = (T)vm;
        d -= lr * ((m / c1) / (sqrtf(vm) + eps));
    } else if (kind == DMPM_DESCEND_LION) {
        const float sg = g > 0.f ? 1.f : (g < 0.f ? -1.f : 0.f);
        const float m = b1 * (float)mom[i] + (1.f - b1) * sg;
        mom[i] = (T)m;
        d -= lr * m;
    } else if (kind == DMPM_DESCEND_GD) {
        d -= lr * g;
    } else {  // DMPM_DESCEND_DLDF
        float c = g;
        if (c > 1.f) c = 1.f;
        if (c < -1.f) c = -1.f;
        if (fabsf(c) < 1e-3f) c = c < 0.f ? -1e-3f : 1e-3f;
        const float m = 0.9f * (float)mom[i] + lr * c;
        mom[i] = (T)m;
        d -= m;
    }
    dfc[i] = (T)d;
}
// sum of squares of a gradient's 9 planes: block partial sums into part
template <class G> __global__ void k_sumsq(const G* __restrict__ a, size_t np, int n, double* part) {
    __shared__ double s[32];
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < (size_t)9 * np && (int)(i % np) < n) { const double t = (double)a[i]; v = t * t; }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

}  // namespace

// ====================================================================== engine
struct EngineBase {
    virtual ~EngineBase() {}
};

struct dmpm_ctx {
    int device = 0;
    int precision = DMPM_FP32_MIXED;
    cudaStream_t stream = nullptr;
    std::string err;
    dmpm_params prm{};
    int64_t prm_gen = 0;  // bumped by dmpm_set_params (captured graphs hold the parameters)
    int64_t launches = 0;
    DeviceBudget budget;  // device bytes held by the engine's arenas, optional cap (dmpm_set_device_limit)
    std::unique_ptr<EngineBase> eng;
};

namespace {

template <class T> class Engine : public EngineBase {
   public:
    // FP32 path: cell-sorted warp items (kernels_warp.cuh); FP64 path: plain kernels (kernels.cuh)
    static constexpr bool kTiled = std::is_same<T, float>::value;
    static constexpr bool kWarp = kTiled;
    // the FP32 path stores each layer's strain H = F - I in the F planes (kernels_warp.cuh)
    static constexpr bool kStrain = kWarp;
    // state planes per layer: the FP32 path adds the low parts of its
    // compensated positions (PXL); adjoint layers keep NSTATE planes
    static constexpr int kNst = kWarp ? (int)NSTATE_X : (int)NSTATE;
    // one cell sort: the stable order and warp items used for steps
    // [e * sort_every, (e + 1) * sort_every)
    struct Epoch {
        uint32_t* order = nullptr;
        uint32_t* items = nullptr;
        uint32_t* n_items = nullptr;  // device scalar: the warp kernels read it, the host never does
        // brick units (kernels_brick.cuh) of the same order, when the sort made them:
        // unit_shift 3 (2^3-cell octants) or 6 (4^3-cell bricks), -1 when the
        // warp-item kernels serve this epoch
        uint32_t* units = nullptr;
        uint32_t* unit_keys = nullptr;
        uint32_t* unit_items = nullptr;  // first warp item of each unit
        uint32_t* n_units = nullptr;
        int unit_shift = -1;
        bool valid = false;
    };

    explicit Engine(dmpm_ctx* c) : ctx_(c) {
        for (Arena* a : {&scene_arena_, &scene_arena_grid_, &layer_arena_, &staging_arena_, &misc_arena_, &fix_arena_})
            a->set_budget(&ctx_->budget);
    }

    // ---------------------------------------------------------- configuration
    void set_grid(int dx_, int dy_, int dz_, double h, const double* mn) {
        if (dx_ <= 0 || dy_ <= 0 || dz_ <= 0 || !(h > 0)) throw ArgError{"grid dims and dx must be positive"};
        if ((double)dx_ * dy_ * dz_ > 2e9) throw ArgError{"grid has more than 2e9 nodes"};
        {
            const int d[3] = {dx_, dy_, dz_};
            if (key_span(d) > (1ull << 32)) throw ArgError{"grid too large for 32-bit cell keys"};
        }
        const bool same = grid_set_ && geo_.dim[0] == dx_ && geo_.dim[1] == dy_ && geo_.dim[2] == dz_;
        drop_graphs();  // the grid geometry is a kernel argument of every captured launch
        geo_.dim[0] = dx_; geo_.dim[1] = dy_; geo_.dim[2] = dz_;
        geo_.dx = h;
        for (int a = 0; a < 3; a++) geo_.mn[a] = mn ? mn[a] : 0.0;
        G_ = (size_t)dx_ * dy_ * dz_;
        grid_set_ = true;
        if (same) return;
        layers_.clear();
        layout_ = Layout{};
        target_ = nullptr;
        scene_arena_grid_.release();
        target_ = (T*)scene_arena_grid_.alloc(G_ * sizeof(T));
        DMPM_CK(cudaMemsetAsync(target_, 0, G_ * sizeof(T), ctx_->stream));
        dldm_ = (T*)scene_arena_grid_.alloc(G_ * sizeof(T));
        scratch_grid_ = (node4<T>*)scene_arena_grid_.alloc(G_ * sizeof(node4<T>));
    }

    void alloc_particles(int n) {
        if (n <= 0) throw ArgError{"particle count must be positive"};
        permuted_ = false;  // a new cloud arrives in the caller's order
        if (n == n_ && cst_) {
            // same cloud size: overwrite in place and keep the layer storage
            DMPM_CK(cudaMemsetAsync(cst_, 0, NCONST * np_ * sizeof(T), ctx_->stream));
            DMPM_CK(cudaMemsetAsync(st0_, 0, kNst * np_ * sizeof(T), ctx_->stream));
            DMPM_CK(cudaMemsetAsync(dfc0_, 0, 9 * np_ * sizeof(T), ctx_->stream));
            return;
        }
        drop_graphs();
        n_ = n;
        np_ = round_up((size_t)n, 64);
        layers_.clear();
        layout_ = Layout{};
        scene_arena_.release();
        perm_ = nullptr;
        cst_ = (T*)scene_arena_.alloc(NCONST * np_ * sizeof(T));
        st0_ = (T*)scene_arena_.alloc(kNst * np_ * sizeof(T));
        dfc0_ = (T*)scene_arena_.alloc(9 * np_ * sizeof(T));
        DMPM_CK(cudaMemsetAsync(cst_, 0, NCONST * np_ * sizeof(T), ctx_->stream));
        DMPM_CK(cudaMemsetAsync(st0_, 0, kNst * np_ * sizeof(T), ctx_->stream));
        DMPM_CK(cudaMemsetAsync(dfc0_, 0, 9 * np_ * sizeof(T), ctx_->stream));
    }

    const uint32_t* perm() const { return permuted_ ? perm_ : nullptr; }

    // Store the cloud in the order of its cell keys (the stable cell sort of
    // layer 0): particles that share stencil nodes then sit together in every
    // plane, as they do when the caller's order is spatial.  Transfers map
    // indices through perm_ from here on, so callers see their own order.
    void reorder_scene() {
        if constexpr (kWarp) {
            // scratch: the first epoch's order and items (recomputed by the next forward
            // pass) and layer 0's state planes (overwritten from st0_ right after)
            Epoch& e = epochs_[0];
            cell_sort(st0_, e);  // e.order[i] = index of the i-th particle in cell order
            if (!perm_) perm_ = (uint32_t*)scene_arena_.alloc((size_t)n_ * 4);
            DMPM_CK(cudaMemcpyAsync(perm_, e.order, (size_t)n_ * 4, cudaMemcpyDeviceToDevice, ctx_->stream));
            T* buf = layers_[0].st;
            auto permute = [&](T* a, int planes) {
                const size_t tot = (size_t)n_ * planes;
                k_gather_planes<T><<<(unsigned)((tot + 255) / 256), 256, 0, ctx_->stream>>>(a, planes, np_, n_, perm_,
                                                                                            buf);
                launched();
                DMPM_CK(cudaMemcpyAsync(a, buf, (size_t)planes * np_ * sizeof(T), cudaMemcpyDeviceToDevice,
                                        ctx_->stream));
            };
            permute(st0_, kNst);
            permute(cst_, NCONST);
            permute(dfc0_, 9);
            permuted_ = true;
            for (Epoch& ep : epochs_) ep.valid = false;
        }
    }

    double* staging(size_t count) {
        if (count > staging_count_) {
            staging_arena_.release();
            staging_ = (double*)staging_arena_.alloc(count * sizeof(double));
            staging_count_ = count;
        }
        return staging_;
    }

    // host doubles (width per particle) -> planes; diag is added to the diagonal of
    // 3x3 matrices first (F -> strain H = F - I on the FP32 path)
    void upload_planes(const double* host, int width, T* dst, double diag = 0.0) {
        double* s = staging((size_t)n_ * width);
        DMPM_CK(cudaMemcpyAsync(s, host, (size_t)n_ * width * sizeof(double), cudaMemcpyHostToDevice, ctx_->stream));
        if (diag != 0.0) {
            k_diag_add<<<(unsigned)(((size_t)n_ * 3 + 255) / 256), 256, 0, ctx_->stream>>>(s, n_, diag);
            launched();
        }
        const size_t tot = (size_t)n_ * width;
        k_unpack<T><<<(unsigned)((tot + 255) / 256), 256, 0, ctx_->stream>>>(s, width, n_, dst, np_, perm());
        launched();
    }

    // positions: compensated planes (hi, lo) on the FP32 path, plain planes otherwise
    void upload_x(const double* host, T* st) {
        if constexpr (kWarp) {
            double* s = staging((size_t)n_ * 3);
            DMPM_CK(cudaMemcpyAsync(s, host, (size_t)n_ * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx_->stream));
            k_unpack_x2<<<(unsigned)(((size_t)n_ * 3 + 255) / 256), 256, 0, ctx_->stream>>>(
                s, n_, (float*)st + (size_t)PX * np_, (float*)st + (size_t)PXL * np_, np_, perm());
            launched();
        } else {
            upload_planes(host, 3, st + (size_t)PX * np_);
        }
    }
    void download_x(const T* st, double* host) {
        if constexpr (kWarp) {
            double* s = staging((size_t)n_ * 3);
            k_pack_x2<<<(unsigned)(((size_t)n_ * 3 + 255) / 256), 256, 0, ctx_->stream>>>(
                (const float*)st + (size_t)PX * np_, (const float*)st + (size_t)PXL * np_, np_, n_, s, perm());
            launched();
            DMPM_CK(cudaMemcpyAsync(host, s, (size_t)n_ * 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
            DMPM_CK(cudaStreamSynchronize(ctx_->stream));
        } else {
            download_planes(st + (size_t)PX * np_, 3, host);
        }
    }

    void download_planes(const T* src, int width, double* host, double diag = 0.0) {
        double* s = staging((size_t)n_ * width);
        const size_t tot = (size_t)n_ * width;
        k_pack<T><<<(unsigned)((tot + 255) / 256), 256, 0, ctx_->stream>>>(src, np_, width, n_, s, perm());
        launched();
        if (diag != 0.0) {
            k_diag_add<<<(unsigned)(((size_t)n_ * 3 + 255) / 256), 256, 0, ctx_->stream>>>(s, n_, diag);
            launched();
        }
        DMPM_CK(cudaMemcpyAsync(host, s, tot * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
        DMPM_CK(cudaStreamSynchronize(ctx_->stream));
    }

    void set_particles(int n, const double* x, const double* v, const double* F, const double* C, const double* dFc,
                       const double* m, const double* vol, const double* lam, const double* mu) {
        if (!x || !m || !lam || !mu) throw ArgError{"x, m, lam and mu are required"};
        alloc_particles(n);
        upload_x(x, st0_);
        if (v) upload_planes(v, 3, st0_ + (size_t)PV * np_);
        if (F) {
            upload_planes(F, 9, st0_ + (size_t)PF * np_, kStrain ? -1.0 : 0.0);
        } else {
            std::vector<double> eye((size_t)n * 9, 0.0);
            for (int p = 0; p < n; p++) eye[9 * p] = eye[9 * p + 4] = eye[9 * p + 8] = 1.0;
            upload_planes(eye.data(), 9, st0_ + (size_t)PF * np_, kStrain ? -1.0 : 0.0);
        }
        if (C) upload_planes(C, 9, st0_ + (size_t)PC * np_);
        if (dFc) upload_planes(dFc, 9, dfc0_);
        upload_planes(m, 1, cst_ + (size_t)KM * np_);
        if (vol) upload_planes(vol, 1, cst_ + (size_t)KVOL * np_);
        upload_planes(lam, 1, cst_ + (size_t)KLAM * np_);
        upload_planes(mu, 1, cst_ + (size_t)KMU * np_);
    }

    void set_points_ref(const void* pts, int n) {
        if (!pts) throw ArgError{"points is NULL"};
        alloc_particles(n);
        const size_t bytes = (size_t)n * 118 * sizeof(float);
        double* s = staging((bytes + 7) / 8);
        DMPM_CK(cudaMemcpyAsync(s, pts, bytes, cudaMemcpyHostToDevice, ctx_->stream));
        k_unpack_ref<T><<<(n + 255) / 256, 256, 0, ctx_->stream>>>((const float*)s, n, np_, st0_, cst_, dfc0_,
                                                                   kStrain ? T(-1) : T(0));
        launched();
    }

    void check_scene() {
        if (!grid_set_) throw StateError{"dmpm_set_grid has not been called"};
        if (n_ <= 0) throw StateError{"no particles uploaded"};
    }

    FwdArgs<T> fwd_args() const {
        FwdArgs<T> a{};
        a.n = n_;
        a.np = np_;
        a.geo = geo_;
        a.dt = (T)ctx_->prm.dt;
        a.drag = (T)ctx_->prm.drag;
        a.s = (T)ctx_->prm.smoothing;
        for (int c = 0; c < 3; c++) a.fext[c] = (T)ctx_->prm.f_ext[c];
        a.cst = cst_;
        a.tile_cap = tile_cap();
        a.status = status_;
        return a;
    }

    LossArgs<T> loss_args() const {
        LossArgs<T> a{};
        a.n = n_;
        a.np = a.npc = np_;
        a.geo = geo_;
        a.cst = cst_;
        a.target = target_;
        a.dldm = dldm_;
        a.kind = ctx_->prm.loss_kind;
        a.tile_cap = tile_cap();
        a.xlo = kWarp ? 1 : 0;
        a.status = status_;
        return a;
    }

    int block() const { return ctx_->prm.block_size > 0 ? ctx_->prm.block_size : kDefaultBlock; }
    int tile_cap() const { return ctx_->prm.tile_cap > 0 ? ctx_->prm.tile_cap : kDefaultTileCap; }
    unsigned pgrid() const { return (unsigned)((n_ + block() - 1) / block()); }
    // deterministic mode of the FP32 path: order-independent node sums (fixpoint.cuh)
    bool det() const { return kWarp && ctx_->prm.deterministic != 0; }
    void ensure_fix() {
        if (!det() || (fix_ && fix_G_ == G_)) return;
        fix_arena_.release();
        fix_ = nullptr;
        fixb_ = nullptr;
        fix_ = (fix4*)fix_arena_.alloc(G_ * sizeof(fix4));
        fixb_ = (unsigned*)fix_arena_.alloc(FIXB_SLOTS * sizeof(unsigned));
        fix_G_ = G_;
    }
    void clear_fix(int slot) {  // zero the integer sums and one bound slot (-1: all) before a pass
        DMPM_CK(cudaMemsetAsync(fix_, 0, G_ * sizeof(fix4), ctx_->stream));
        if (slot < 0) DMPM_CK(cudaMemsetAsync(fixb_, 0, FIXB_SLOTS * sizeof(unsigned), ctx_->stream));
        else DMPM_CK(cudaMemsetAsync(fixb_ + slot, 0, sizeof(unsigned), ctx_->stream));
    }
    // sum part_[0 .. nb) into *out in block order
    void sum_partials(unsigned nb, double* out) {
        if (nb > part_n_) throw StateError{"internal: partial-sum buffer too small"};
        k_sum_partials<<<1, 256, 0, ctx_->stream>>>(part_, (int)nb, out);
        launched();
    }
    unsigned pgrid256() const { return (unsigned)((n_ + 255) / 256); }
    // persistent grid of a warp-item kernel: ctas CTAs of 256 threads per SM (the
    // residency its register budget allows), fewer when the particles could not
    // fill them (at most one item per particle)
    // persistent grid of a warp-item kernel: ctas blocks of `threads` per SM, or
    // one warp per particle when that is fewer
    unsigned warp_blocks(int ctas = 3, int threads = 256) {
        if (sms_ == 0) {
            int dev = 0;
            DMPM_CK(cudaGetDevice(&dev));
            DMPM_CK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
        }
        const size_t most = ((size_t)n_ * 32 + threads - 1) / threads;
        return (unsigned)std::max<size_t>(1, std::min<size_t>(most, (size_t)sms_ * ctas));
    }
    unsigned ggrid() const { return (unsigned)((G_ + 255) / 256); }
    // Brick units of an epoch into the kernel arguments; returns the unit shift
    // (3, 6) or -1 when the epoch has none (warp-item kernels)
    int set_units(WArgs& a, const Epoch& ep) const {
        a.unit_start = ep.units;
        a.unit_key = ep.unit_keys;
        a.n_units_dev = ep.n_units;
        a.unit_item = ep.unit_items;
        return ep.units ? ep.unit_shift : -1;
    }
    // persistent grid of a brick kernel: as many CTAs as can be resident at once
    // (its register and shared-memory budget), looked up once per kernel
    template <class K> unsigned brick_blocks(K kernel) {
        if (sms_ == 0) warp_blocks();
        const void* key = reinterpret_cast<const void*>(kernel);
        auto it = brick_occ_.find(key);
        if (it == brick_occ_.end()) {
            int per_sm = 0;
            DMPM_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, DMPM_BRICK_THREADS, 0));
            it = brick_occ_.emplace(key, std::max(1, per_sm)).first;
        }
        return (unsigned)(sms_ * it->second);
    }

    // the deterministic adjoint scatter: through each unit's shared node tile when the epoch has units
    template <bool EX, bool GEN> void launch_adj_scatter_fix_t(const WArgs& a, int ush, unsigned ws) {
        const unsigned bt = DMPM_BRICK_THREADS;
        if (ush == 3) k_adj_scatter_fix_b<2, EX, GEN><<<brick_blocks(k_adj_scatter_fix_b<2, EX, GEN>), bt, 0, ctx_->stream>>>(a);
        else if (ush == 6) k_adj_scatter_fix_b<4, EX, GEN><<<brick_blocks(k_adj_scatter_fix_b<4, EX, GEN>), bt, 0, ctx_->stream>>>(a);
        else k_adj_scatter_w<EX, GEN, ITEMS_PERSISTENT, true><<<ws, DMPM_ADJ_SCATTER_THREADS, 0, ctx_->stream>>>(a);
    }
    void launch_adj_scatter_fix(const WArgs& a, bool ex, bool gen, int ush, unsigned ws) {
        if (ex && gen) launch_adj_scatter_fix_t<true, true>(a, ush, ws);
        else if (ex) launch_adj_scatter_fix_t<true, false>(a, ush, ws);
        else if (gen) launch_adj_scatter_fix_t<false, true>(a, ush, ws);
        else launch_adj_scatter_fix_t<false, false>(a, ush, ws);
    }

    void launched() {
        ctx_->launches++;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) throw CudaError{e, std::string("kernel launch: ") + cudaGetErrorString(e)};
    }

    // ---------------------------------------------------------- profiling
    void set_profiling(bool on) {
        harvest();
        prof_ = on;
        for (int k = 0; k < K_COUNT; k++) { prof_ms_[k] = 0.0; prof_cnt_[k] = 0; }
    }
    void pbeg(int kid) {
        if (!prof_) return;
        cudaEvent_t e0 = take_event(), e1 = take_event();
        DMPM_CK(cudaEventRecord(e0, ctx_->stream));
        pend_.push_back(Pending{kid, e0, e1});
    }
    void pend() {
        if (!prof_) return;
        DMPM_CK(cudaEventRecord(pend_.back().e1, ctx_->stream));
    }
    cudaEvent_t take_event() {
        if (!event_pool_.empty()) {
            cudaEvent_t e = event_pool_.back();
            event_pool_.pop_back();
            return e;
        }
        cudaEvent_t e;
        DMPM_CK(cudaEventCreate(&e));
        return e;
    }
    // called after the stream has been synchronised
    void harvest() {
        for (const Pending& q : pend_) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, q.e0, q.e1) == cudaSuccess) {
                prof_ms_[q.kid] += ms;
                prof_cnt_[q.kid] += 1;
            }
            event_pool_.push_back(q.e0);
            event_pool_.push_back(q.e1);
        }
        pend_.clear();
    }
    void kernel_stats(int kid, double* ms, int64_t* cnt) {
        if (kid < 0 || kid >= K_COUNT) throw ArgError{"kernel id out of range"};
        DMPM_CK(cudaStreamSynchronize(ctx_->stream));
        harvest();
        if (ms) *ms = prof_ms_[kid];
        if (cnt) *cnt = prof_cnt_[kid];
    }

    void ensure_status() {
        if (!status_) {
            status_ = (unsigned*)misc_arena_.alloc(sizeof(unsigned) + sizeof(double) * 2);
            loss_acc_ = (double*)((char*)status_ + 8);
            DMPM_CK(cudaMallocHost(&host_misc_, 64));
        }
    }

    unsigned read_status() {
        DMPM_CK(cudaMemcpyAsync(host_misc_, status_, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx_->stream));
        DMPM_CK(cudaStreamSynchronize(ctx_->stream));
        harvest();
        return *(unsigned*)host_misc_;
    }

    void compute_volumes() {
        check_scene();
        ensure_status();
        LossArgs<T> a = loss_args();
        a.st = st0_;
        a.grid = scratch_grid_;
        DMPM_CK(cudaMemsetAsync(scratch_grid_, 0, G_ * sizeof(node4<T>), ctx_->stream));
        launch_mass(a);
        k_volumes<T><<<pgrid(), block(), 0, ctx_->stream>>>(a, cst_ + (size_t)KVOL * np_);
        launched();
    }

    void launch_mass(const LossArgs<T>& a) {
        if constexpr (kWarp) {
            if (det()) {  // integer sums: the raster does not depend on the order of the adds
                ensure_fix();
                clear_fix(FIXB_RASTER);
                k_fix_mass_bound<<<(a.n + 255) / 256, 256, 0, ctx_->stream>>>(a.cst + (size_t)KM * a.npc, a.n,
                                                                              fixb_ + FIXB_RASTER);
                launched();
                k_p2g_mass_fix<<<(a.n + 255) / 256, 256, 0, ctx_->stream>>>(a, fix_, fixb_);
                launched();
                k_fix_to_node4<<<ggrid(), 256, 0, ctx_->stream>>>(fix_, fixb_, a.n, G_, 2, a.grid);
                launched();
                return;
            }
        }
        if (kTiled)
            k_p2g_mass<T, true><<<pgrid(), block(), tile_cap() * sizeof(T), ctx_->stream>>>(a);
        else
            k_p2g_mass<T, false><<<pgrid(), block(), 0, ctx_->stream>>>(a);
        launched();
    }

    void set_target_mass(const double* m) {
        if (!grid_set_) throw StateError{"dmpm_set_grid has not been called"};
        double* s = staging(G_);
        DMPM_CK(cudaMemcpyAsync(s, m, G_ * sizeof(double), cudaMemcpyHostToDevice, ctx_->stream));
        k_set_node_mass<T><<<ggrid(), 256, 0, ctx_->stream>>>(s, G_, target_);
        launched();
    }

    void get_target_mass(double* out) {
        if (!grid_set_) throw StateError{"dmpm_set_grid has not been called"};
        if (!out) throw ArgError{"out is NULL"};
        double* s = staging(G_);
        k_scalar_field<T><<<ggrid(), 256, 0, ctx_->stream>>>(target_, G_, s);
        launched();
        DMPM_CK(cudaMemcpyAsync(out, s, G_ * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
        DMPM_CK(cudaStreamSynchronize(ctx_->stream));
    }

    // LoadCompGraph: target grid = ResetValues + P2G(target samples, dt = drag = 0),
    // of which EndLayerMassLoss reads only m (MPMPolyscope.cpp:155-160).
    void rasterize_target(int n, const double* x, double mp) {
        if (!grid_set_) throw StateError{"dmpm_set_grid has not been called"};
        if (n < 0 || (n > 0 && !x)) throw ArgError{"bad target samples"};
        ensure_status();
        DMPM_CK(cudaMemsetAsync(scratch_grid_, 0, G_ * sizeof(node4<T>), ctx_->stream));
        if (n > 0) {
            const size_t npt = round_up((size_t)n, 64);
            Arena tmp(&ctx_->budget);
            T* st = (T*)tmp.alloc(3 * npt * sizeof(T));
            T* cst = (T*)tmp.alloc(npt * sizeof(T));
            double* s = staging((size_t)n * 3);
            DMPM_CK(cudaMemcpyAsync(s, x, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx_->stream));
            k_unpack<T><<<(unsigned)(((size_t)n * 3 + 255) / 256), 256, 0, ctx_->stream>>>(s, 3, n, st, npt);
            launched();
            std::vector<double> mh((size_t)n, mp);
            double* s2 = staging((size_t)n * 3);
            DMPM_CK(cudaMemcpyAsync(s2, mh.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx_->stream));
            k_unpack<T><<<(unsigned)((n + 255) / 256), 256, 0, ctx_->stream>>>(s2, 1, n, cst, npt);
            launched();
            LossArgs<T> a = loss_args();
            a.n = n;
            a.np = a.npc = npt;
            a.st = st;
            a.xlo = 0;  // target samples: plain float positions
            a.cst = cst;
            a.grid = scratch_grid_;
            launch_mass(a);
            k_copy_node_mass<T><<<ggrid(), 256, 0, ctx_->stream>>>(scratch_grid_, G_, target_);
            launched();
            DMPM_CK(cudaStreamSynchronize(ctx_->stream));
        } else {
            DMPM_CK(cudaMemsetAsync(target_, 0, G_ * sizeof(T), ctx_->stream));
        }
    }

    // ---------------------------------------------------------- layers
    bool stored(int l) const { return k_ == 1 || l % k_ == 0 || l == L_ - 1; }
    int control_stride() const { return ctx_->prm.control_stride > 1 ? ctx_->prm.control_stride : 1; }
    // per-layer controls: does layer l own its dFc and gradient (a control frame)?
    bool owns_controls(int l) const {
        return ctx_->prm.control_mode == DMPM_CTRL_PER_LAYER &&
               (control_stride() == 1 || (l % control_stride() == 0 && l < L_ - 1));
    }
    int num_control_layers() const {
        int c = 0;
        for (int l = 0; l < L_; l++) c += owns_controls(l) ? 1 : 0;
        return c;
    }

    void setup(int num_layers) {
        check_scene();
        if (num_layers < 1) throw ArgError{"num_layers must be >= 1"};
        ensure_status();
        const dmpm_params& P = ctx_->prm;
        Layout want;
        want.L = num_layers; want.k_req = P.checkpoint_every; want.control = P.control_mode;
        want.keep_adj = P.keep_adjoints; want.keep_int = P.keep_intermediates; want.np = np_; want.G = G_;
        want.sort_every = P.sort_every;
        want.stride = control_stride();
        want.brick = P.brick_cells != 0;
        if (want == layout_ && (int)layers_.size() == num_layers) {
            reset_layers();
            return;
        }
        drop_graphs();
        try {
            allocate_layers(num_layers);
        } catch (...) {
            // out of device memory (or over the context's device byte limit):
            // drop the partial storage so the context reads as not set up, and
            // a later dmpm_setup with a smaller request (or a higher limit) works
            layer_arena_.release();
            layers_.clear();
            epochs_.clear();
            L_ = 0;
            layout_ = Layout{};
            forward_done_ = loss_done_ = false;
            throw;
        }
        layout_ = want;
        reset_layers();
    }

    void allocate_layers(int num_layers) {
        const dmpm_params& P = ctx_->prm;
        L_ = num_layers;
        layer_arena_.release();
        layers_.assign(L_, LayerSlots{});
        const size_t st_bytes = kNst * np_ * sizeof(T);
        const size_t adj_bytes = NSTATE * np_ * sizeof(T);
        const size_t gr_bytes = G_ * sizeof(node4<T>);
        const bool per_layer = P.control_mode == DMPM_CTRL_PER_LAYER;
        // choose the checkpoint interval
        int k = P.checkpoint_every;
        if (k <= 0) {
            size_t free_b = 0, total_b = 0;
            DMPM_CK(cudaMemGetInfo(&free_b, &total_b));
            const double need = (double)L_ * (st_bytes + gr_bytes) +
                                (per_layer ? 2.0 * num_control_layers() * 9 * np_ * sizeof(T) : 0.0) +
                                (P.keep_adjoints ? (double)L_ * adj_bytes : 0.0);
            k = need < 0.8 * (double)free_b ? 1 : std::max(2, (int)std::ceil(std::sqrt((double)L_)));
        }
        k_ = std::min(k, std::max(1, L_ - 1));
        if (k_ < 1) k_ = 1;
        // particle states
        int nstored = 0;
        for (int l = 0; l < L_; l++) nstored += stored(l) ? 1 : 0;
        T* sbase = (T*)layer_arena_.alloc((size_t)nstored * st_bytes);
        for (int l = 0, s = 0; l < L_; l++)
            if (stored(l)) layers_[l].st = sbase + (size_t)(s++) * kNst * np_;
        if (k_ > 1) {
            ring_[0] = (T*)layer_arena_.alloc(st_bytes);
            ring_[1] = (T*)layer_arena_.alloc(st_bytes);
            seg_st_.assign(k_ - 1, nullptr);
            for (int i = 0; i < k_ - 1; i++) seg_st_[i] = (T*)layer_arena_.alloc(st_bytes);
            seg_grid_.assign(k_, nullptr);
            for (int i = 0; i < k_; i++) seg_grid_[i] = (node4<T>*)layer_arena_.alloc(gr_bytes);
        } else {
            node4<T>* gbase = (node4<T>*)layer_arena_.alloc((size_t)L_ * gr_bytes);
            for (int l = 0; l < L_; l++) layers_[l].grid = gbase + (size_t)l * G_;
        }
        // controls
        if (per_layer) {
            // control frames own a dFc copy and a gradient; the other layers read
            // the uploaded dFc, which nothing writes
            const size_t nc = (size_t)num_control_layers();
            T* dbase = (T*)layer_arena_.alloc(nc * 9 * np_ * sizeof(T));
            T* gbase = (T*)layer_arena_.alloc(nc * 9 * np_ * sizeof(T));
            for (int l = 0, c = 0; l < L_; l++) {
                if (owns_controls(l)) {
                    layers_[l].dfc = dbase + (size_t)c * 9 * np_;
                    layers_[l].ctrl_grad = gbase + (size_t)c * 9 * np_;
                    c++;
                } else {
                    layers_[l].dfc = dfc0_;
                    layers_[l].ctrl_grad = nullptr;
                }
            }
            ctrl_acc_ = nullptr;
        } else {
            for (int l = 0; l < L_; l++) layers_[l].dfc = dfc0_;
            ctrl_acc_ = (double*)layer_arena_.alloc(9 * np_ * sizeof(double));
        }
        // adjoints
        if (P.keep_adjoints) {
            T* abase = (T*)layer_arena_.alloc((size_t)L_ * adj_bytes);
            DMPM_CK(cudaMemsetAsync(abase, 0, (size_t)L_ * adj_bytes, ctx_->stream));
            for (int l = 0; l < L_; l++) layers_[l].adj = abase + (size_t)l * NSTATE * np_;
        } else {
            adj_pp_[0] = (T*)layer_arena_.alloc(adj_bytes);
            adj_pp_[1] = (T*)layer_arena_.alloc(adj_bytes);
        }
        gadj_ = (node4<T>*)layer_arena_.alloc(gr_bytes);
        gadj2_ = (node4<T>*)layer_arena_.alloc(2 * gr_bytes);
        // block partial sums: the loss (G / 256 blocks), dLdF norms (n / 32 at the smallest block size),
        // gradient norms (9 np / 256)
        part_n_ = std::max({(G_ + 255) / 256, (np_ + 31) / 32, (9 * np_ + 255) / 256}) + 1;
        part_ = (double*)layer_arena_.alloc(part_n_ * sizeof(double));
        if (!kWarp) {
            gridv_ = (T*)layer_arena_.alloc(3 * G_ * sizeof(T));
            pscratch_ = (T*)layer_arena_.alloc(9 * np_ * sizeof(T));
        } else {
            // affine momentum matrix G of every stored/segment layer, adjoint scratch, sort state
            const size_t g_bytes = kAuxPlanes * np_ * sizeof(T);
            if (k_ == 1) {
                T* base = (T*)layer_arena_.alloc((size_t)L_ * g_bytes);
                for (int l = 0; l < L_; l++) layers_[l].G = base + (size_t)l * kAuxPlanes * np_;
            } else {
                gscratch_ = (T*)layer_arena_.alloc(g_bytes);
                seg_G_.assign(k_, nullptr);
                for (int i = 0; i < k_; i++) seg_G_[i] = (T*)layer_arena_.alloc(g_bytes);
            }
            adjn_ = (T*)layer_arena_.alloc(12 * np_ * sizeof(T));
            gath_ = (T*)layer_arena_.alloc(18 * np_ * sizeof(T));
            alloc_sort();
        }
        if (P.keep_intermediates) {
            T* b1 = (T*)layer_arena_.alloc((size_t)L_ * 9 * np_ * sizeof(T));   // P
            T* b2 = (T*)layer_arena_.alloc((size_t)L_ * 9 * np_ * sizeof(T));   // dLdP
            T* b3 = (T*)layer_arena_.alloc((size_t)L_ * 3 * np_ * sizeof(T));   // dLdv_next
            T* b4 = (T*)layer_arena_.alloc((size_t)L_ * 9 * np_ * sizeof(T));   // dLdC_next
            node4<T>* g1 = (node4<T>*)layer_arena_.alloc((size_t)L_ * gr_bytes);  // grid dLdv
            node4<T>* g2 = (node4<T>*)layer_arena_.alloc((size_t)L_ * gr_bytes);  // grid dLdp, dLdm
            DMPM_CK(cudaMemsetAsync(b1, 0, (size_t)L_ * 9 * np_ * sizeof(T), ctx_->stream));
            DMPM_CK(cudaMemsetAsync(b2, 0, (size_t)L_ * 9 * np_ * sizeof(T), ctx_->stream));
            DMPM_CK(cudaMemsetAsync(b3, 0, (size_t)L_ * 3 * np_ * sizeof(T), ctx_->stream));
            DMPM_CK(cudaMemsetAsync(b4, 0, (size_t)L_ * 9 * np_ * sizeof(T), ctx_->stream));
            DMPM_CK(cudaMemsetAsync(g1, 0, (size_t)L_ * gr_bytes, ctx_->stream));
            DMPM_CK(cudaMemsetAsync(g2, 0, (size_t)L_ * gr_bytes, ctx_->stream));
            for (int l = 0; l < L_; l++) {
                layers_[l].dbgP = b1 + (size_t)l * 9 * np_;
                layers_[l].dbgdLdP = b2 + (size_t)l * 9 * np_;
                layers_[l].dbgvn = b3 + (size_t)l * 3 * np_;
                layers_[l].dbgCn = b4 + (size_t)l * 9 * np_;
                layers_[l].dbggdv = g1 + (size_t)l * G_;
                layers_[l].dbggdp = g2 + (size_t)l * G_;
            }
        }
    }

    // SetUpCompGraph semantics on allocated storage: layer 0 = the uploaded
    // cloud, every layer's dFc = the uploaded dFc, gradients cleared.  Layer
    // states other than 0 are not copied: each is written by the forward pass
    // before anything reads it.
    void reset_layers() {
        if (ctx_->prm.reorder_particles && !permuted_) reorder_scene();
        const size_t st_bytes = kNst * np_ * sizeof(T);
        DMPM_CK(cudaMemcpyAsync(layers_[0].st, st0_, st_bytes, cudaMemcpyDeviceToDevice, ctx_->stream));
        if (ctx_->prm.control_mode == DMPM_CTRL_PER_LAYER) {
            for (int l = 0; l < L_; l++) {
                if (!owns_controls(l)) continue;
                DMPM_CK(cudaMemcpyAsync(layers_[l].dfc, dfc0_, 9 * np_ * sizeof(T), cudaMemcpyDeviceToDevice, ctx_->stream));
                DMPM_CK(cudaMemsetAsync(layers_[l].ctrl_grad, 0, 9 * np_ * sizeof(T), ctx_->stream));
            }
        } else {
            DMPM_CK(cudaMemsetAsync(ctrl_acc_, 0, 9 * np_ * sizeof(double), ctx_->stream));
        }
        for (Epoch& e : epochs_) e.valid = false;
        forward_done_ = false;
        loss_done_ = false;
        backward_lo_ = L_;
        seg_lo_ = seg_hi_ = -1;
    }

    // ---------------------------------------------------------- cell sort (FP32 path)
    int sort_every() const { return ctx_->prm.sort_every > 0 ? ctx_->prm.sort_every : kDefaultSortEvery; }

    void alloc_sort() {
        const int nep = std::max(1, (L_ - 1 + sort_every() - 1) / sort_every());
        epochs_.assign(nep, Epoch{});
        for (Epoch& e : epochs_) {
            e.order = (uint32_t*)layer_arena_.alloc((size_t)n_ * sizeof(uint32_t));
            e.items = (uint32_t*)layer_arena_.alloc(((size_t)n_ + 1) * sizeof(uint32_t));
            e.n_items = (uint32_t*)layer_arena_.alloc(16);
            if (ctx_->prm.brick_cells) {
                e.units = (uint32_t*)layer_arena_.alloc(((size_t)n_ + 1) * sizeof(uint32_t));
                e.unit_keys = (uint32_t*)layer_arena_.alloc((size_t)n_ * sizeof(uint32_t));
                e.unit_items = (uint32_t*)layer_arena_.alloc(((size_t)n_ + 1) * sizeof(uint32_t));
                e.n_units = (uint32_t*)layer_arena_.alloc(16);
            }
        }
        const size_t n = (size_t)n_;
        sk_[0] = (uint32_t*)layer_arena_.alloc(n * 4);
        sk_[1] = (uint32_t*)layer_arena_.alloc(n * 4);
        sv_[0] = (uint32_t*)layer_arena_.alloc(n * 4);
        sv_[1] = (uint32_t*)layer_arena_.alloc(n * 4);
        sh_ = (uint32_t*)layer_arena_.alloc(n * 4);
        sf_ = (uint32_t*)layer_arena_.alloc(n * 4);
        const size_t rs_tiles = (n + RS_TILE - 1) / RS_TILE;
        counts_ = (uint32_t*)layer_arena_.alloc(256 * rs_tiles * 4);
        const size_t mx = std::max(n, 256 * rs_tiles);
        tile_tot_ = (uint32_t*)layer_arena_.alloc(((mx + SCAN_TILE - 1) / SCAN_TILE + 1) * 4);
    }

    template <class Op> void device_scan(uint32_t* data, size_t n, uint32_t* grand) {
        const int tiles = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
        k_scan_tiles<Op><<<tiles, SCAN_THREADS, 0, ctx_->stream>>>(data, (int)n, tile_tot_);
        launched();
        k_scan_totals<Op><<<1, 1024, 0, ctx_->stream>>>(tile_tot_, tiles, grand);
        launched();
        k_scan_add<Op><<<tiles, SCAN_THREADS, 0, ctx_->stream>>>(data, (int)n, tile_tot_);
        launched();
    }

    // Stable sort of the particles of a layer state by cell key; fills the
    // epoch's order and warp items.  Keys stay in sk_[sorted_] for inspection.
    void cell_sort(const T* st, Epoch& e) {
        const int n = n_;
        KeyArgs<T> ka{};
        ka.n = n;
        ka.np = np_;
        ka.geo = geo_;
        ka.st = st;
        ka.xlo = kWarp ? 1 : 0;
        ka.keys = sk_[0];
        ka.vals = sv_[0];
        k_cell_keys<T><<<(n + 255) / 256, 256, 0, ctx_->stream>>>(ka);
        launched();
        const uint64_t max_key = key_span(geo_.dim);
        int bits = 1;
        while (bits < 32 && (1ull << bits) < max_key) bits++;
        const int rs_tiles = (n + RS_TILE - 1) / RS_TILE;
        int cur = 0;
        for (int shift = 0; shift < bits; shift += 8) {
            k_rs_upsweep<<<rs_tiles, RS_THREADS, 0, ctx_->stream>>>(sk_[cur], n, shift, counts_, rs_tiles);
            launched();
            device_scan<OpSum>(counts_, (size_t)256 * rs_tiles, nullptr);
            k_rs_downsweep<<<rs_tiles, RS_THREADS, 0, ctx_->stream>>>(sk_[cur], sv_[cur], sk_[cur ^ 1], sv_[cur ^ 1], n,
                                                                     shift, counts_, rs_tiles);
            launched();
            cur ^= 1;
        }
        sorted_ = cur;
        DMPM_CK(cudaMemcpyAsync(e.order, sv_[cur], (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx_->stream));
        k_run_heads<<<(n + 255) / 256, 256, 0, ctx_->stream>>>(sk_[cur], n, sh_);
        launched();
        device_scan<OpMax>(sh_, (size_t)n, nullptr);
        k_item_flags<<<(n + 255) / 256, 256, 0, ctx_->stream>>>(sk_[cur], sh_, n, sf_);
        launched();
        device_scan<OpSum>(sf_, (size_t)n, e.n_items);
        k_item_starts<<<(n + 255) / 256, 256, 0, ctx_->stream>>>(sk_[cur], sh_, sf_, n, e.items);
        launched();
        k_item_sentinel<<<1, 1, 0, ctx_->stream>>>(e.items, e.n_items, n);
        launched();
        e.unit_shift = -1;
        if (ctx_->prm.brick_cells && e.units) {
            const int shift = ctx_->prm.brick_cells == 4 ? 6 : 3;
            k_unit_flags<<<(n + 255) / 256, 256, 0, ctx_->stream>>>(sk_[cur], n, shift, sf_);
            launched();
            device_scan<OpSum>(sf_, (size_t)n, e.n_units);
            k_unit_starts<<<(n + 255) / 256, 256, 0, ctx_->stream>>>(sk_[cur], sf_, n, shift, e.units, e.unit_keys);
            launched();
            k_item_sentinel<<<1, 1, 0, ctx_->stream>>>(e.units, e.n_units, n);
            launched();
            k_unit_items<<<(n + 256) / 256, 256, 0, ctx_->stream>>>(sk_[cur], e.items, e.n_items, sf_, e.n_units, shift,
                                                                   e.unit_items);
            launched();
            e.unit_shift = shift;
        }
        e.valid = true;
    }

    Epoch& epoch_for(int l, const T* st, bool allow_sort) {
        Epoch& e = epochs_[std::min((int)epochs_.size() - 1, l / sort_every())];
        if (allow_sort && (l % sort_every() == 0 || !e.valid)) cell_sort(st, e);
        if (!e.valid) cell_sort(st, e);
        return e;
    }

    void debug_cell_sort(int l, uint32_t* keys, uint32_t* order, uint32_t* items, int* n_items) {
        if (!kWarp) throw StateError{"the cell sort belongs to the FP32 path"};
        if (l < 0 || l >= L_) throw ArgError{"layer out of range"};
        Epoch e{};
        Arena tmp(&ctx_->budget);
        e.order = (uint32_t*)tmp.alloc((size_t)n_ * 4);
        e.items = (uint32_t*)tmp.alloc(((size_t)n_ + 1) * 4);
        e.n_items = (uint32_t*)tmp.alloc(16);
        cell_sort(materialize_state(l), e);
        uint32_t ni = 0;
        DMPM_CK(cudaMemcpyAsync(&ni, e.n_items, 4, cudaMemcpyDeviceToHost, ctx_->stream));
        DMPM_CK(cudaStreamSynchronize(ctx_->stream));
        if (keys) DMPM_CK(cudaMemcpyAsync(keys, sk_[sorted_], (size_t)n_ * 4, cudaMemcpyDeviceToHost, ctx_->stream));
        if (order) DMPM_CK(cudaMemcpyAsync(order, e.order, (size_t)n_ * 4, cudaMemcpyDeviceToHost, ctx_->stream));
        if (items) DMPM_CK(cudaMemcpyAsync(items, e.items, ((size_t)ni + 1) * 4, cudaMemcpyDeviceToHost, ctx_->stream));
        std::vector<uint32_t> perm;
        if (order && permuted_) {  // positions in the caller's indices
            perm.resize((size_t)n_);
            DMPM_CK(cudaMemcpyAsync(perm.data(), perm_, (size_t)n_ * 4, cudaMemcpyDeviceToHost, ctx_->stream));
        }
        DMPM_CK(cudaStreamSynchronize(ctx_->stream));
        for (size_t i = 0; i < perm.size(); i++) order[i] = perm[order[i]];
        if (n_items) *n_items = (int)ni;
    }

    WArgs warp_args() const {
        WArgs a{};
        const dmpm_params& P = ctx_->prm;
        a.n = n_;
        a.np = a.npl = a.npn = np_;
        a.geo = geo_;
        a.dt = (float)P.dt;
        a.drag = (float)P.drag;
        a.s = (float)P.smoothing;
        for (int c = 0; c < 3; c++) a.fext[c] = (float)P.f_ext[c];
        a.cst = (const float*)cst_;
        a.xlo = 1;
        a.status = status_;
        return a;
    }

    // pointer to the state of layer l if it is materialised (stored or in the current segment)
    T* state_of(int l) {
        if (layers_[l].st) return layers_[l].st;
        if (k_ > 1 && l > seg_lo_ && l < seg_hi_) return seg_st_[l - seg_lo_ - 1];
        return nullptr;
    }
    node4<T>* grid_of(int l) {
        if (layers_[l].grid) return layers_[l].grid;
        if (k_ > 1 && l >= seg_lo_ && l < seg_hi_) return seg_grid_[l - seg_lo_];
        return nullptr;
    }
    T* G_of(int l) {
        if (layers_[l].G) return layers_[l].G;
        if (k_ > 1 && l >= seg_lo_ && l < seg_hi_) return seg_G_[l - seg_lo_];
        return nullptr;
    }

    // One ForwardTimeStep: layer l -> out (state of l+1), grid g, G of layer l
    // in Gd.  FP32 path: g_ready = Gd already holds layer l's G (the previous
    // step's G2P formed it), so the stress stage is skipped; Gd_next non-null =
    // the brick G2P also forms layer l+1's G there.  Returns whether it did.
    bool step(int l, const T* st, T* out, node4<T>* g, T* Gd, bool allow_sort, bool g_ready = false,
              T* Gd_next = nullptr) {
        if constexpr (kWarp) {
            ensure_fix();  // allocated already (a no-op) on every captured path
            Epoch& ep = epoch_for(l, st, allow_sort);
            WArgs a = warp_args();
            a.items = WarpItems{ep.order, ep.items, 0};
            a.n_items_dev = ep.n_items;
            a.st = (const float*)st;
            a.st_next = (float*)out;
            a.dfc = (const float*)layers_[l].dfc;
            a.G = (float*)Gd;
            a.grid = (node4<float>*)g;
            a.P = ctx_->prm.keep_intermediates ? (float*)layers_[l].dbgP : nullptr;
            const bool dm = det();
            if (dm) {  // integer node sums, converted into the layer grid after P2G
                a.fix = fix_;
                a.fixb = fixb_;
                clear_fix(-1);
            } else {
                DMPM_CK(cudaMemsetAsync(g, 0, G_ * sizeof(node4<T>), ctx_->stream));
            }
            const unsigned ws = warp_blocks(DMPM_SCATTER_CTAS, DMPM_P2G_THREADS);
            const int ush = set_units(a, ep);
            if (dm || !g_ready) {
                pbeg(K_P_OP1);
                if (dm) k_stress<true><<<pgrid256(), 256, 0, ctx_->stream>>>(a);
                else k_stress<false><<<pgrid256(), 256, 0, ctx_->stream>>>(a);
                launched();
                pend();
            }
            pbeg(K_P2G);
            const bool gen = ctx_->prm.warp_general != 0;
            const unsigned bt = DMPM_BRICK_THREADS;
            if (dm && ush == 3) {  // integer sums through each unit's shared node tile
                if (gen) k_p2g_fix_b<2, true><<<brick_blocks(k_p2g_fix_b<2, true>), bt, 0, ctx_->stream>>>(a);
                else k_p2g_fix_b<2, false><<<brick_blocks(k_p2g_fix_b<2, false>), bt, 0, ctx_->stream>>>(a);
            } else if (dm && ush == 6) {
                if (gen) k_p2g_fix_b<4, true><<<brick_blocks(k_p2g_fix_b<4, true>), bt, 0, ctx_->stream>>>(a);
                else k_p2g_fix_b<4, false><<<brick_blocks(k_p2g_fix_b<4, false>), bt, 0, ctx_->stream>>>(a);
            } else if (dm && gen) k_p2g_w<true, ITEMS_PERSISTENT, true><<<ws, DMPM_P2G_THREADS, 0, ctx_->stream>>>(a);
            else if (dm) k_p2g_w<false, ITEMS_PERSISTENT, true><<<ws, DMPM_P2G_THREADS, 0, ctx_->stream>>>(a);
            else if (gen) k_p2g_w<true, ITEMS_PERSISTENT><<<ws, DMPM_P2G_THREADS, 0, ctx_->stream>>>(a);
            else k_p2g_w<false, ITEMS_PERSISTENT><<<ws, DMPM_P2G_THREADS, 0, ctx_->stream>>>(a);
            launched();
            if (dm) {
                k_fix_to_node4<<<ggrid(), 256, 0, ctx_->stream>>>(fix_, fixb_, n_, G_, 0, (node4<float>*)g);
                launched();
            }
            pend();
            pbeg(K_GOP);
            k_gop_inplace<<<ggrid(), 256, 0, ctx_->stream>>>((node4<float>*)g, G_, a.dt, a.fext[0], a.fext[1], a.fext[2]);
            launched();
            pend();
            // the deterministic mode keeps the standalone stress stage: it also raises the
            // next P2G's bounds, which that step clears first
            const bool fuse = Gd_next && !dm && (ush == 3 || ush == 6);
            if (fuse) {
                a.dfc_next = (const float*)layers_[l + 1].dfc;
                a.G_next = (float*)Gd_next;
                a.P_next = ctx_->prm.keep_intermediates ? (float*)layers_[l + 1].dbgP : nullptr;
            }
            pbeg(K_G2P);
            if (ush == 3 && fuse) k_g2p_b<2, true><<<brick_blocks(k_g2p_b<2, true>), bt, 0, ctx_->stream>>>(a);
            else if (ush == 6 && fuse) k_g2p_b<4, true><<<brick_blocks(k_g2p_b<4, true>), bt, 0, ctx_->stream>>>(a);
            else if (ush == 3) k_g2p_b<2><<<brick_blocks(k_g2p_b<2>), bt, 0, ctx_->stream>>>(a);
            else if (ush == 6) k_g2p_b<4><<<brick_blocks(k_g2p_b<4>), bt, 0, ctx_->stream>>>(a);
            else k_g2p_w<ITEMS_PERSISTENT><<<warp_blocks(DMPM_G2P_CTAS), 256, 0, ctx_->stream>>>(a);
            launched();
            pend();
            return fuse;
        }
        FwdArgs<T> a = fwd_args();
        a.st = st;
        a.st_next = out;
        a.dfc = layers_[l].dfc;
        a.grid = g;
        a.gridv = gridv_;
        a.P = ctx_->prm.keep_intermediates ? layers_[l].dbgP : (kTiled ? nullptr : pscratch_);
        DMPM_CK(cudaMemsetAsync(g, 0, G_ * sizeof(node4<T>), ctx_->stream));
        const size_t tile_b = (size_t)tile_cap() * sizeof(node4<T>);
        (void)tile_b;
        (void)Gd;
        (void)allow_sort;
        {
            pbeg(K_P_OP1);
            k_p_op1<T><<<pgrid(), block(), 0, ctx_->stream>>>(a);
            launched();
            pend();
            pbeg(K_P2G);
            k_p2g<T, false, false><<<pgrid(), block(), 0, ctx_->stream>>>(a);
            launched();
            pend();
            pbeg(K_GOP);
            k_gop<T><<<ggrid(), 256, 0, ctx_->stream>>>(a, G_);
            launched();
            pend();
            pbeg(K_G2P);
            k_g2p<T, false><<<pgrid(), block(), 0, ctx_->stream>>>(a);
            launched();
            pend();
        }
        (void)g_ready;
        (void)Gd_next;
        return false;
    }

    void reset_status() {
        DMPM_CK(cudaMemsetAsync(status_, 0, sizeof(unsigned), ctx_->stream));
    }

    // ---------------------------------------------------------- CUDA graphs
    // The FP32 store-all forward and backward passes enqueue a fixed sequence
    // of ~1,100 launches with no host read-back; each is captured once per
    // (start / top, control) and replayed.  Graphs are dropped whenever a
    // captured pointer or parameter can change: new particle or layer storage,
    // a new grid, dmpm_set_params.
    bool graphs_ok() const { return kWarp && k_ == 1 && !prof_ && !ctx_->prm.eager; }
    void drop_graphs() {
        for (auto& kv : graphs_)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        graphs_.clear();
    }
    template <class Fn> void run_graph(std::pair<int64_t, int64_t> key, Fn enqueue) {
        if (graph_gen_ != ctx_->prm_gen) {
            drop_graphs();
            graph_gen_ = ctx_->prm_gen;
        }
        auto it = graphs_.find(key);
        if (it != graphs_.end()) {
            DMPM_CK(cudaGraphLaunch(it->second.exec, ctx_->stream));
            ctx_->launches += it->second.launches;
            return;
        }
        const int64_t l0 = ctx_->launches;
        DMPM_CK(cudaStreamBeginCapture(ctx_->stream, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue();
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(ctx_->stream, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        cudaGraph_t g = nullptr;
        DMPM_CK(cudaStreamEndCapture(ctx_->stream, &g));
        Graph gr;
        gr.launches = ctx_->launches - l0;  // counted once here for the replay below
        const cudaError_t e = cudaGraphInstantiate(&gr.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) throw CudaError{e, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
        graphs_.emplace(key, gr);
        DMPM_CK(cudaGraphLaunch(gr.exec, ctx_->stream));
    }

    void forward(int start) {
        if (L_ <= 0) throw StateError{"dmpm_setup has not been called"};
        if (start < 0 || start >= L_) throw ArgError{"start_layer out of range"};
        reset_status();
        ensure_fix();  // before any capture: a captured launch holds the buffer's address
        if (k_ == 1) {
            auto body = [&]() {
                bool ready = false;  // layer l's G formed by the previous step
                for (int l = start; l + 1 < L_; l++)
                    ready = step(l, layers_[l].st, layers_[l + 1].st, layers_[l].grid, layers_[l].G, true, ready,
                                 l + 2 < L_ ? layers_[l + 1].G : nullptr);
            };
            if (graphs_ok()) {
                run_graph({0, start}, body);
                if constexpr (kWarp)  // the replayed sorts refreshed every epoch the pass touches
                    for (int l = start; l + 1 < L_; l++)
                        epochs_[std::min((int)epochs_.size() - 1, l / sort_every())].valid = true;
            } else {
                body();
            }
        } else {
            const T* cur = materialize_state(start);
            int r = 0;
            bool ready = false;
            for (int l = start; l + 1 < L_; l++) {
                T* out = layers_[l + 1].st ? layers_[l + 1].st : ring_[r];
                if (!layers_[l + 1].st) r ^= 1;
                // the current state may live in ring_[r] already (ping-pong); layer l's G in
                // gscratch_ is read by P2G before G2P writes layer l+1's there
                ready = step(l, cur, out, seg_grid_[0], gscratch_, true, ready, l + 2 < L_ ? gscratch_ : nullptr);
                cur = out;
            }
            seg_lo_ = seg_hi_ = -1;  // segment scratch no longer matches
        }
        forward_done_ = true;
        loss_done_ = false;
        last_status_ = read_status();
    }

    // Make layer l's state available; for a non-stored layer recompute its
    // segment (and the grids of the segment) from the checkpoint below it.
    const T* materialize_state(int l) {
        if (T* s = state_of(l)) return s;
        materialize_segment(l - l % k_);
        return state_of(l);
    }

    void materialize_segment(int c) {
        const int e = std::min(c + k_, L_ - 1);
        const T* cur = layers_[c].st;
        bool ready = false;
        for (int l = c; l < e; l++) {
            T* out = (l + 1 == e) ? nullptr : seg_st_[l - c];
            T* Gd = seg_G_.empty() ? nullptr : seg_G_[l - c];
            if (out) {
                ready = step(l, cur, out, seg_grid_[l - c], Gd, false, ready,
                             seg_G_.empty() ? nullptr : seg_G_[l + 1 - c]);
                cur = out;
            } else {
                // last step of the segment: only its grid is needed; the output
                // (layer e) is a stored layer already, write it to scratch ring
                step(l, cur, ring_[0], seg_grid_[l - c], Gd, false, ready);
            }
        }
        seg_lo_ = c;
        seg_hi_ = e;
    }

    double loss() {
        if (!forward_done_ && L_ > 1) throw StateError{"dmpm_forward has not been run"};
        if (L_ <= 0) throw StateError{"dmpm_setup has not been called"};
        reset_status();
        LossArgs<T> a = loss_args();
        a.st = layers_[L_ - 1].st;
        node4<T>* g = (k_ == 1) ? layers_[L_ - 1].grid : scratch_grid_;
        a.grid = g;
        a.adj = adj_of(L_ - 1, true);
        a.loss = loss_acc_;
        a.part = part_;
        DMPM_CK(cudaMemsetAsync(g, 0, G_ * sizeof(node4<T>), ctx_->stream));
        pbeg(K_MASS);
        launch_mass(a);
        pend();
        pbeg(K_NODE_LOSS);
        k_node_loss<T><<<ggrid(), 256, 0, ctx_->stream>>>(a, G_);
        launched();
        sum_partials(ggrid(), loss_acc_);
        pend();
        pbeg(K_LOSS_DLDX);
        k_loss_dldx<T><<<pgrid(), block(), 0, ctx_->stream>>>(a);
        launched();
        pend();
        DMPM_CK(cudaMemcpyAsync((char*)host_misc_ + 8, loss_acc_, sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
        last_status_ = read_status();
        loss_done_ = true;
        backward_lo_ = L_ - 1;
        return *(double*)((char*)host_misc_ + 8);
    }

    // adjoint buffer of layer l (ping-pong when adjoints are not kept)
    T* adj_of(int l, bool for_write) {
        (void)for_write;
        if (layers_[l].adj) return layers_[l].adj;
        return adj_pp_[l & 1];
    }

    void adjoint_step(int i) {
        const dmpm_params& P = ctx_->prm;
        if constexpr (kWarp) {
            Epoch& ep = epoch_for(i, state_of(i), false);
            WArgs a = warp_args();
            a.items = WarpItems{ep.order, ep.items, 0};
            a.n_items_dev = ep.n_items;
            a.st = (const float*)state_of(i);
            a.st_next = (float*)state_of(i + 1);
            a.dfc = (const float*)layers_[i].dfc;
            a.G = (float*)G_of(i);
            a.grid = (node4<float>*)grid_of(i);
            a.adj_next = (const float*)adj_of(i + 1, false);
            a.adj = (float*)adj_of(i, true);
            a.adjn = (float*)adjn_;
            a.gath = (float*)gath_;
            a.gadj = (node4<float>*)gadj_;
            a.gadj2 = (node4<float>*)gadj2_;
            a.ctrl_grad = (float*)layers_[i].ctrl_grad;
            a.ctrl_acc = ctrl_acc_;
            a.dbg_dLdP = P.keep_intermediates ? (float*)layers_[i].dbgdLdP : nullptr;
            a.dbg_vnext = P.keep_intermediates ? (float*)layers_[i].dbgvn : nullptr;
            a.dbg_Cnext = P.keep_intermediates ? (float*)layers_[i].dbgCn : nullptr;
            if (!a.st || !a.st_next || !a.grid || !a.G) throw StateError{"internal: layer not materialised"};
            const bool ex = P.adjoint_mode == DMPM_ADJ_EXACT;
            const bool dm = det();
            if (dm) {  // integer node sums of dLdv, converted into gadj_ after the scatter
                a.fix = fix_;
                a.fixb = fixb_;
                clear_fix(FIXB_ADJ);
            } else {
                DMPM_CK(cudaMemsetAsync(gadj_, 0, G_ * sizeof(node4<T>), ctx_->stream));
            }
            const unsigned ws = warp_blocks(DMPM_ADJ_SCATTER_CTAS, DMPM_ADJ_SCATTER_THREADS),
                           wg = warp_blocks(DMPM_GATHER_CTAS, DMPM_GATHER_THREADS);
            const int ush = set_units(a, ep);
            pbeg(K_ADJ_SCATTER);
            if (dm) {
                if (ex) k_adj_sources<true><<<pgrid256(), 256, 0, ctx_->stream>>>(a);
                else k_adj_sources<false><<<pgrid256(), 256, 0, ctx_->stream>>>(a);
                launched();
                launch_adj_scatter_fix(a, ex, P.warp_general != 0, ush, ws);
                launched();
                k_fix_to_node4<<<ggrid(), 256, 0, ctx_->stream>>>(fix_, fixb_, n_, G_, 1, (node4<float>*)gadj_);
            } else if (P.warp_general) {
                if (ex) k_adj_scatter_w<true, true, ITEMS_PERSISTENT><<<ws, DMPM_ADJ_SCATTER_THREADS, 0, ctx_->stream>>>(a);
                else k_adj_scatter_w<false, true, ITEMS_PERSISTENT><<<ws, DMPM_ADJ_SCATTER_THREADS, 0, ctx_->stream>>>(a);
            } else {
                if (ex) k_adj_scatter_w<true, false, ITEMS_PERSISTENT><<<ws, DMPM_ADJ_SCATTER_THREADS, 0, ctx_->stream>>>(a);
                else k_adj_scatter_w<false, false, ITEMS_PERSISTENT><<<ws, DMPM_ADJ_SCATTER_THREADS, 0, ctx_->stream>>>(a);
            }
            launched();
            pend();
            pbeg(K_ADJ_GOP);
            if (ex) k_adj_gop_w<true><<<ggrid(), 256, 0, ctx_->stream>>>(a.grid, a.gadj, a.gadj2, G_, a.dt, a.fext[0], a.fext[1], a.fext[2]);
            else k_adj_gop_w<false><<<ggrid(), 256, 0, ctx_->stream>>>(a.grid, a.gadj, a.gadj2, G_, a.dt, a.fext[0], a.fext[1], a.fext[2]);
            launched();
            pend();
            if (P.keep_intermediates) {
                DMPM_CK(cudaMemcpyAsync(layers_[i].dbggdv, gadj_, G_ * sizeof(node4<T>), cudaMemcpyDeviceToDevice, ctx_->stream));
                DMPM_CK(cudaMemcpy2DAsync(layers_[i].dbggdp, sizeof(node4<T>), gadj2_, 2 * sizeof(node4<T>),
                                          sizeof(node4<T>), G_, cudaMemcpyDeviceToDevice, ctx_->stream));
            }
            pbeg(K_ADJ_GATHER);
            if (ex) {
                k_adj_gather_w<true, ITEMS_PERSISTENT><<<wg, DMPM_GATHER_THREADS, 0, ctx_->stream>>>(a);
            } else {
                k_adj_gather_w<false, ITEMS_PERSISTENT><<<wg, DMPM_GATHER_THREADS, 0, ctx_->stream>>>(a);
            }
            launched();
            pend();
            if (DMPM_SPLIT_FINALIZE && !prof_) {
                // fork: the transport part on the side stream after the gather,
                // join: the main stream continues after both parts
                side_stream();
                DMPM_CK(cudaEventRecord(ev_fork_, ctx_->stream));
                DMPM_CK(cudaStreamWaitEvent(side_, ev_fork_, 0));
                launch_finalize_split(a, ex, ctx_->stream, side_);
                launched();
                launched();
                DMPM_CK(cudaEventRecord(ev_join_, side_));
                DMPM_CK(cudaStreamWaitEvent(ctx_->stream, ev_join_, 0));
            } else if (DMPM_SPLIT_FINALIZE) {
                // profiled: the two parts one after the other, each timed
                pbeg(K_ADJ_TRANSPORT);
                launch_finalize_part(a, ex, FIN_TRANSPORT, ctx_->stream);
                launched();
                pend();
                pbeg(K_ADJ_FINALIZE);
                launch_finalize_part(a, ex, FIN_STRESS, ctx_->stream);
                launched();
                pend();
            } else {
                pbeg(K_ADJ_FINALIZE);
                launch_finalize(a, ex, ctx_->stream);
                launched();
                pend();
            }
            return;
        }
        AdjArgs<T> a{};
        a.n = n_;
        a.np = np_;
        a.geo = geo_;
        a.dt = (T)P.dt;
        a.drag = (T)P.drag;
        a.s = (T)P.smoothing;
        for (int c = 0; c < 3; c++) a.fext[c] = (T)P.f_ext[c];
        a.st = state_of(i);
        a.st_next = state_of(i + 1);
        a.cst = cst_;
        a.dfc = layers_[i].dfc;
        a.grid = grid_of(i);
        a.adj_next = adj_of(i + 1, false);
        a.adj = adj_of(i, true);
        a.gadj = gadj_;
        a.gadj2 = gadj2_;
        a.ctrl_grad = layers_[i].ctrl_grad;
        a.ctrl_acc = ctrl_acc_;
        a.dbg_dLdP = P.keep_intermediates ? layers_[i].dbgdLdP : nullptr;
        a.dbg_vnext = P.keep_intermediates ? layers_[i].dbgvn : nullptr;
        a.dbg_Cnext = P.keep_intermediates ? layers_[i].dbgCn : nullptr;
        a.tile_cap = tile_cap();
        a.status = status_;
        if (!a.st || !a.st_next || !a.grid) throw StateError{"internal: layer not materialised"};
        DMPM_CK(cudaMemsetAsync(gadj_, 0, G_ * sizeof(node4<T>), ctx_->stream));
        const bool ex = P.adjoint_mode == DMPM_ADJ_EXACT;
        {
            pbeg(K_ADJ_SCATTER);
            if (ex) k_adj_scatter<T, false, true><<<pgrid(), block(), 0, ctx_->stream>>>(a);
            else k_adj_scatter<T, false, false><<<pgrid(), block(), 0, ctx_->stream>>>(a);
            launched();
            pend();
            pbeg(K_ADJ_GOP);
            if (ex) k_adj_gop<T, true><<<ggrid(), 256, 0, ctx_->stream>>>(a, G_);
            else k_adj_gop<T, false><<<ggrid(), 256, 0, ctx_->stream>>>(a, G_);
            launched();
            pend();
            if (P.keep_intermediates) debug_grid_adjoint(i, a, ex);
            pbeg(K_ADJ_GATHER);
            if (ex) k_adj_gather<T, false, true><<<pgrid(), block(), 0, ctx_->stream>>>(a);
            else k_adj_gather<T, false, false><<<pgrid(), block(), 0, ctx_->stream>>>(a);
            launched();
            pend();
        }
    }

    void debug_grid_adjoint(int i, AdjArgs<T>& a, bool ex) {
        DMPM_CK(cudaMemcpyAsync(layers_[i].dbggdv, gadj_, G_ * sizeof(node4<T>), cudaMemcpyDeviceToDevice, ctx_->stream));
        AdjArgs<T> b = a;
        b.gadj2 = layers_[i].dbggdp;
        if (ex) k_adj_gop<T, true><<<ggrid(), 256, 0, ctx_->stream>>>(b, G_);
        else k_adj_gop<T, false><<<ggrid(), 256, 0, ctx_->stream>>>(b, G_);
        launched();
    }

    void backward(int control) {
        if (!loss_done_) throw StateError{"dmpm_loss must run before dmpm_backward"};
        backward_range(L_ - 1, control);
    }

    // Adjoint steps top-1 down to control, starting from the adjoint state of
    // layer `top` (written by dmpm_loss, or by the caller for top < L-1).
    void backward_range(int top, int control) {
        if (!forward_done_ && L_ > 1) throw StateError{"dmpm_forward has not been run"};
        ensure_fix();
        if (top < 0 || top > L_ - 1) throw ArgError{"top layer out of range"};
        if (control < 0 || control > top) throw ArgError{"control_layer out of range"};
        if (top < L_ - 1 && !layers_[top].adj) throw StateError{"set keep_adjoints to start the adjoint below the last layer"};
        reset_status();
        // the finalize's second stream exists before any capture of the adjoint steps
        if (kWarp && DMPM_SPLIT_FINALIZE) side_stream();
        if (ctrl_acc_) DMPM_CK(cudaMemsetAsync(ctrl_acc_, 0, 9 * np_ * sizeof(double), ctx_->stream));
        if (k_ == 1) {
            auto body = [&]() {
                for (int i = top - 1; i >= control; i--) adjoint_step(i);
            };
            bool sorted = true;  // a captured backward pass must not contain sorts
            if constexpr (kWarp)
                for (int i = top - 1; i >= control; i--)
                    sorted &= epochs_[std::min((int)epochs_.size() - 1, i / sort_every())].valid;
            if (graphs_ok() && sorted) run_graph({1 + (int64_t)top, control}, body);
            else body();
        } else {
            int i = top - 1;
            while (i >= control) {
                const int c = i - i % k_;
                materialize_segment(c);
                for (; i >= std::max(c, control); i--) adjoint_step(i);
            }
        }
        backward_lo_ = control;
        last_status_ = read_status();
    }

    // ---------------------------------------------------------- downloads
    void get_particles(int l, int field, double* out) {
        if (l < 0 || l >= L_) throw ArgError{"layer out of range"};
        if (!out) throw ArgError{"out is NULL"};
        auto need_adj = [&]() -> const T* {
            if (layers_[l].adj) return layers_[l].adj;
            if (l >= backward_lo_ && (l == backward_lo_ || l == L_ - 1)) return adj_of(l, false);
            throw StateError{"adjoint of this layer is not kept (set keep_adjoints)"};
        };
        auto need_dbg = [&](const T* p) -> const T* {
            if (!p) throw StateError{"intermediates are not kept (set keep_intermediates)"};
            return p;
        };
        switch (field) {
            case DMPM_F_X: download_x(materialize_state(l), out); break;
            case DMPM_F_V: download_planes(materialize_state(l) + (size_t)PV * np_, 3, out); break;
            case DMPM_F_F: download_planes(materialize_state(l) + (size_t)PF * np_, 9, out, kStrain ? 1.0 : 0.0); break;
            case DMPM_F_C: download_planes(materialize_state(l) + (size_t)PC * np_, 9, out); break;
            case DMPM_F_P: {
                if (layers_[l].dbgP && l < L_ - 1) { download_planes(layers_[l].dbgP, 9, out); break; }
                // recompute P_op_1 of this layer on demand
                Arena tmp(&ctx_->budget);
                T* P = (T*)tmp.alloc(9 * np_ * sizeof(T));
                FwdArgs<T> a = fwd_args();
                a.st = materialize_state(l);
                a.dfc = layers_[l].dfc;
                a.P = P;
                a.strain = kStrain ? 1 : 0;
                k_p_op1<T><<<pgrid(), block(), 0, ctx_->stream>>>(a);
                launched();
                download_planes(P, 9, out);
                break;
            }
            case DMPM_F_M: download_planes(cst_ + (size_t)KM * np_, 1, out); break;
            case DMPM_F_VOL: download_planes(cst_ + (size_t)KVOL * np_, 1, out); break;
            case DMPM_F_LAM: download_planes(cst_ + (size_t)KLAM * np_, 1, out); break;
            case DMPM_F_MU: download_planes(cst_ + (size_t)KMU * np_, 1, out); break;
            case DMPM_F_DFC: download_planes(layers_[l].dfc, 9, out); break;
            case DMPM_F_DLDX: download_planes(need_adj() + (size_t)PX * np_, 3, out); break;
            case DMPM_F_DLDV: download_planes(need_adj() + (size_t)PV * np_, 3, out); break;
            case DMPM_F_DLDF: download_planes(need_adj() + (size_t)PF * np_, 9, out); break;
            case DMPM_F_DLDC: download_planes(need_adj() + (size_t)PC * np_, 9, out); break;
            case DMPM_F_DLDP: download_planes(need_dbg(layers_[l].dbgdLdP), 9, out); break;
            case DMPM_F_DLDV_NEXT: download_planes(need_dbg(layers_[l].dbgvn), 3, out); break;
            case DMPM_F_DLDC_NEXT: download_planes(need_dbg(layers_[l].dbgCn), 9, out); break;
            case DMPM_F_DLDFE:
                if (ctrl_acc_) throw StateError{"tied controls: use dmpm_get_control_grad"};
                if (!layers_[l].ctrl_grad) throw ArgError{"layer is not a control frame (control_stride)"};
                download_planes(layers_[l].ctrl_grad, 9, out);
                break;
            default: throw ArgError{"unknown particle field"};
        }
    }

    void set_layer_particles(int l, int field, const double* in) {
        if (l < 0 || l >= L_) throw ArgError{"layer out of range"};
        if (!in) throw ArgError{"in is NULL"};
        switch (field) {
            case DMPM_F_DFC:
                if (!ctrl_acc_ && !owns_controls(l)) throw ArgError{"layer is not a control frame (control_stride)"};
                upload_planes(in, 9, layers_[l].dfc);
                break;
            case DMPM_F_X: case DMPM_F_V: case DMPM_F_F: case DMPM_F_C: {
                if (!layers_[l].st) throw StateError{"layer state is not stored (checkpointing)"};
                if (field == DMPM_F_X) {
                    upload_x(in, layers_[l].st);
                    break;
                }
                const int off = field == DMPM_F_V ? PV : field == DMPM_F_F ? PF : PC;
                upload_planes(in, (field == DMPM_F_X || field == DMPM_F_V) ? 3 : 9, layers_[l].st + (size_t)off * np_,
                              (field == DMPM_F_F && kStrain) ? -1.0 : 0.0);
                break;
            }
            case DMPM_F_DLDX: case DMPM_F_DLDV: case DMPM_F_DLDF: case DMPM_F_DLDC: {
                if (!layers_[l].adj) throw StateError{"adjoint fields can be set with keep_adjoints only"};
                const int off = field == DMPM_F_DLDX ? PX : field == DMPM_F_DLDV ? PV : field == DMPM_F_DLDF ? PF : PC;
                upload_planes(in, (field == DMPM_F_DLDX || field == DMPM_F_DLDV) ? 3 : 9, layers_[l].adj + (size_t)off * np_);
                break;
            }
            default: throw ArgError{"field cannot be set per layer"};
        }
    }

    // one optimiser step on the controls of a layer (tied: the shared controls)
    void adam_step(int l, double lr, double b1, double b2, double eps, int t, bool normalize) {
        descend(l, DMPM_DESCEND_ADAM, lr, b1, b2, eps, t, normalize);
    }
    void descend(int l, int kind, double lr, double b1, double b2, double eps, int t, bool normalize) {
        if (L_ <= 0) throw StateError{"dmpm_setup has not been called"};
        if (kind < DMPM_DESCEND_ADAM || kind > DMPM_DESCEND_DLDF) throw ArgError{"unknown descent rule"};
        if ((kind == DMPM_DESCEND_ADAM || kind == DMPM_DESCEND_AMSGRAD) && t < 1)
            throw ArgError{"Adam timestep must be >= 1"};
        T* dfc;
        const void* grad;
        bool grad_fp64;
        if (ctrl_acc_) {
            dfc = dfc0_;
            grad = ctrl_acc_;
            grad_fp64 = true;
            l = -1;
        } else {
            if (l < 0 || l >= L_) throw ArgError{"layer out of range"};
            if (!owns_controls(l)) throw ArgError{"layer is not a control frame (control_stride)"};
            dfc = layers_[l].dfc;
            grad = layers_[l].ctrl_grad;
            grad_fp64 = false;
        }
        auto it = adam_.find(l);
        if (it == adam_.end()) {  // momentum, vector, vector_max of MaterialPoint, shared by the rules
            T* st = (T*)misc_arena_.alloc(3 * 9 * np_ * sizeof(T));
            DMPM_CK(cudaMemsetAsync(st, 0, 3 * 9 * np_ * sizeof(T), ctx_->stream));
            it = adam_.emplace(l, st).first;
        }
        T* mom = it->second;
        T* vec = it->second + 9 * np_;
        T* vmax = it->second + 18 * np_;
        double* norm2 = loss_acc_ + 1;
        const unsigned blocks = (unsigned)((9 * np_ + 255) / 256);
        if (grad_fp64) k_sumsq<double><<<blocks, 256, 0, ctx_->stream>>>((const double*)grad, np_, n_, part_);
        else k_sumsq<T><<<blocks, 256, 0, ctx_->stream>>>((const T*)grad, np_, n_, part_);
        launched();
        sum_partials(blocks, norm2);
        const float c1 = 1.f - std::pow((float)b1, (float)t), c2 = 1.f - std::pow((float)b2, (float)t);
        if (kind == DMPM_DESCEND_ADAM) {
            if (grad_fp64)
                k_adam<T, double><<<blocks, 256, 0, ctx_->stream>>>(dfc, (const double*)grad, mom, vec, np_, n_,
                                                                      norm2, normalize ? 1 : 0, (float)lr, (float)b1,
                                                                      (float)b2, (float)eps, c1, c2);
            else
                k_adam<T, T><<<blocks, 256, 0, ctx_->stream>>>(dfc, (const T*)grad, mom, vec, np_, n_, norm2,
                                                                normalize ? 1 : 0, (float)lr, (float)b1, (float)b2,
                                                                (float)eps, c1, c2);
        } else if (grad_fp64) {
            k_descend<T, double><<<blocks, 256, 0, ctx_->stream>>>(kind, dfc, (const double*)grad, mom, vec, vmax,
                                                                     np_, n_, norm2, normalize ? 1 : 0, (float)lr,
                                                                     (float)b1, (float)b2, (float)eps, c1, c2);
        } else {
            k_descend<T, T><<<blocks, 256, 0, ctx_->stream>>>(kind, dfc, (const T*)grad, mom, vec, vmax, np_, n_,
                                                               norm2, normalize ? 1 : 0, (float)lr, (float)b1,
                                                               (float)b2, (float)eps, c1, c2);
        }
        launched();
        // per-layer controls of later layers are copies made by setup; the
        // reference descends only the control layer, so nothing else changes
    }

    void get_control_grad(int l, double* out) {
        if (!out) throw ArgError{"out is NULL"};
        if (ctrl_acc_) {
            double* s = staging((size_t)n_ * 9);
            k_pack_acc<T><<<(unsigned)(((size_t)n_ * 9 + 255) / 256), 256, 0, ctx_->stream>>>(ctrl_acc_, np_, n_, s,
                                                                                            perm());
            launched();
            DMPM_CK(cudaMemcpyAsync(out, s, (size_t)n_ * 9 * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
            DMPM_CK(cudaStreamSynchronize(ctx_->stream));
            return;
        }
        if (l < 0 || l >= L_) throw ArgError{"layer out of range"};
        if (!layers_[l].ctrl_grad) throw ArgError{"layer is not a control frame (control_stride)"};
        download_planes(layers_[l].ctrl_grad, 9, out);
    }

    double dldf_norm(int l) {
        const T* a = nullptr;
        if (l < 0 || l >= L_) throw ArgError{"layer out of range"};
        if (layers_[l].adj) a = layers_[l].adj;
        else if (l == backward_lo_ || l == L_ - 1) a = adj_of(l, false);
        else throw StateError{"adjoint of this layer is not kept"};
        k_sqnorm9<T><<<pgrid(), block(), 0, ctx_->stream>>>(a + (size_t)PF * np_, np_, n_, part_);
        launched();
        sum_partials(pgrid(), loss_acc_ + 1);
        DMPM_CK(cudaMemcpyAsync((char*)host_misc_ + 16, loss_acc_ + 1, sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
        DMPM_CK(cudaStreamSynchronize(ctx_->stream));
        return std::sqrt(*(double*)((char*)host_misc_ + 16));
    }

    void get_grid(int l, int field, double* out) {
        if (l < 0 || l >= L_) throw ArgError{"layer out of range"};
        if (!out) throw ArgError{"out is NULL"};
        const dmpm_params& P = ctx_->prm;
        if (field == DMPM_G_M || field == DMPM_G_V || field == DMPM_G_P) {
            node4<T>* g = nullptr;
            if (l == L_ - 1) g = (k_ == 1) ? layers_[l].grid : scratch_grid_;
            else {
                g = grid_of(l);
                if (!g) {
                    materialize_segment(l - l % k_);
                    g = grid_of(l);
                }
            }
            double* s = staging(3 * G_);
            const int stored_v = (kWarp && l < L_ - 1) ? 1 : 0;  // the FP32 grid update wrote v over p
            k_grid_field<T><<<ggrid(), 256, 0, ctx_->stream>>>(g, G_, field, stored_v, P.dt, P.f_ext[0], P.f_ext[1],
                                                              P.f_ext[2], s);
            launched();
            const size_t cnt = (field == DMPM_G_M) ? G_ : 3 * G_;
            DMPM_CK(cudaMemcpyAsync(out, s, cnt * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
            DMPM_CK(cudaStreamSynchronize(ctx_->stream));
            return;
        }
        if (field == DMPM_G_DLDM && l == L_ - 1) {
            double* s = staging(G_);
            k_scalar_field<T><<<ggrid(), 256, 0, ctx_->stream>>>(dldm_, G_, s);
            launched();
            DMPM_CK(cudaMemcpyAsync(out, s, G_ * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
            DMPM_CK(cudaStreamSynchronize(ctx_->stream));
            return;
        }
        const node4<T>* g = nullptr;
        int comp = 3;
        if (field == DMPM_G_DLDV) g = layers_[l].dbggdv;
        else if (field == DMPM_G_DLDP) g = layers_[l].dbggdp;
        else if (field == DMPM_G_DLDM) { g = layers_[l].dbggdp; comp = 4; }
        else throw ArgError{"unknown grid field"};
        if (!g) throw StateError{"grid adjoints are not kept (set keep_intermediates)"};
        double* s = staging(3 * G_);
        k_node4_field<T><<<ggrid(), 256, 0, ctx_->stream>>>(g, G_, comp, s);
        launched();
        DMPM_CK(cudaMemcpyAsync(out, s, (comp == 3 ? 3 : 1) * G_ * sizeof(double), cudaMemcpyDeviceToHost, ctx_->stream));
        DMPM_CK(cudaStreamSynchronize(ctx_->stream));
    }

    void get_points_ref(int l, void* pts) {
        if (!pts) throw ArgError{"points is NULL"};
        float* mp = (float*)pts;
        std::vector<double> buf((size_t)n_ * 9);
        auto put = [&](int field, int off, int width) {
            get_particles(l, field, buf.data());
            for (int p = 0; p < n_; p++)
                for (int q = 0; q < width; q++) mp[(size_t)p * 118 + off + q] = (float)buf[(size_t)p * width + q];
        };
        put(DMPM_F_X, 0, 3);
        put(DMPM_F_V, 3, 3);
        put(DMPM_F_F, 6, 9);
        put(DMPM_F_C, 15, 9);
        put(DMPM_F_M, 33, 1);
        put(DMPM_F_VOL, 34, 1);
        put(DMPM_F_LAM, 35, 1);
        put(DMPM_F_MU, 36, 1);
        put(DMPM_F_DFC, 37, 9);
        if (layers_[l].adj || l == backward_lo_ || (l == L_ - 1 && loss_done_)) {
            put(DMPM_F_DLDX, 46, 3);
            put(DMPM_F_DLDV, 49, 3);
            put(DMPM_F_DLDF, 52, 9);
            put(DMPM_F_DLDC, 61, 9);
        }
    }

    void info(int64_t* out, int count) const {
        const int64_t v[] = {n_, geo_.dim[0], geo_.dim[1], geo_.dim[2], L_, ctx_->precision, k_,
                             (int64_t)(scene_arena_.bytes() + scene_arena_grid_.bytes() + layer_arena_.bytes() +
                                       staging_arena_.bytes() + misc_arena_.bytes()),
                             ctx_->launches, (int64_t)last_status_};
        for (int i = 0; i < count && i < (int)(sizeof(v) / sizeof(v[0])); i++) out[i] = v[i];
    }

    unsigned last_status() const { return last_status_; }

    ~Engine() override {
        cudaStreamSynchronize(ctx_->stream);
        drop_graphs();
        harvest();
        for (cudaEvent_t e : event_pool_) cudaEventDestroy(e);
        if (host_misc_) cudaFreeHost(host_misc_);
        if (side_) {
            cudaStreamSynchronize(side_);
            cudaStreamDestroy(side_);
            cudaEventDestroy(ev_fork_);
            cudaEventDestroy(ev_join_);
        }
    }

    // second stream (and its fork/join events) for work that runs beside the main stream
    void side_stream() {
        if (side_) return;
        DMPM_CK(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
        DMPM_CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
        DMPM_CK(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
    }

   private:
    cudaStream_t side_ = nullptr;
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
    struct LayerSlots {
        T* G = nullptr;
        T* st = nullptr;
        node4<T>* grid = nullptr;
        T* dfc = nullptr;
        T* ctrl_grad = nullptr;
        T* adj = nullptr;
        T* dbgP = nullptr;
        T* dbgdLdP = nullptr;
        T* dbgvn = nullptr;
        T* dbgCn = nullptr;
        node4<T>* dbggdv = nullptr;
        node4<T>* dbggdp = nullptr;
    };

    dmpm_ctx* ctx_;
    GridGeom geo_{};
    size_t G_ = 0;
    bool grid_set_ = false;
    int n_ = 0;
    size_t np_ = 0;
    Arena scene_arena_, scene_arena_grid_, layer_arena_, staging_arena_, misc_arena_, fix_arena_;
    T* cst_ = nullptr;
    T* st0_ = nullptr;
    T* dfc0_ = nullptr;
    // cloud stored in cell order (dmpm_params::reorder_particles): perm_[i] =
    // the caller's index of device particle i, applied to every transfer
    uint32_t* perm_ = nullptr;
    bool permuted_ = false;
    T* target_ = nullptr;
    T* dldm_ = nullptr;
    node4<T>* scratch_grid_ = nullptr;
    double* staging_ = nullptr;
    size_t staging_count_ = 0;
    unsigned* status_ = nullptr;
    double* loss_acc_ = nullptr;
    double* part_ = nullptr;  // per-block partial sums of the FP64 reductions (loss, norms)
    size_t part_n_ = 0;
    // deterministic mode: integer node sums (G fix4) and their bound slots
    fix4* fix_ = nullptr;
    unsigned* fixb_ = nullptr;
    size_t fix_G_ = 0;
    void* host_misc_ = nullptr;
    int L_ = 0, k_ = 1;
    std::vector<LayerSlots> layers_;
    T* ring_[2] = {nullptr, nullptr};
    std::vector<T*> seg_st_;
    std::vector<node4<T>*> seg_grid_;
    int seg_lo_ = -1, seg_hi_ = -1;
    T* adj_pp_[2] = {nullptr, nullptr};
    node4<T>* gadj_ = nullptr;
    node4<T>* gadj2_ = nullptr;
    T* gridv_ = nullptr;
    T* pscratch_ = nullptr;
    // FP32 path
    T* gscratch_ = nullptr;
    std::vector<T*> seg_G_;
    T* adjn_ = nullptr;
    T* gath_ = nullptr;
    std::vector<Epoch> epochs_;
    uint32_t* sk_[2] = {nullptr, nullptr};
    uint32_t* sv_[2] = {nullptr, nullptr};
    uint32_t* sh_ = nullptr;
    uint32_t* sf_ = nullptr;
    uint32_t* counts_ = nullptr;
    uint32_t* tile_tot_ = nullptr;
    int sorted_ = 0;
    std::map<int, T*> adam_;  // Adam moment buffers per control set (layer, or -1 for tied controls)
    double* ctrl_acc_ = nullptr;
    bool forward_done_ = false, loss_done_ = false;
    int backward_lo_ = 0;
    unsigned last_status_ = 0;
    // profiling
    struct Pending {
        int kid;
        cudaEvent_t e0, e1;
    };
    bool prof_ = false;
    int sms_ = 0;
    // CUDA graphs of the FP32 store-all forward pass (per start layer) and
    // backward pass (per top and control layer), with the kernel launches each holds
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;
    };
    std::map<std::pair<int64_t, int64_t>, Graph> graphs_;
    int64_t graph_gen_ = -1;
    std::vector<Pending> pend_;
    std::vector<cudaEvent_t> event_pool_;
    double prof_ms_[K_COUNT] = {};
    int64_t prof_cnt_[K_COUNT] = {};
    // the layout the layer storage was allocated for (setup reuses it when unchanged)
    std::map<const void*, int> brick_occ_;  // resident CTAs per SM of each brick kernel
    struct Layout {
        int L = -1, k_req = -1, control = -1, keep_adj = -1, keep_int = -1, sort_every = -1, stride = -1;
        bool brick = false;  // epochs carry brick units
        size_t np = 0, G = 0;
        bool operator==(const Layout& o) const {
            return L == o.L && k_req == o.k_req && control == o.control && keep_adj == o.keep_adj &&
                   keep_int == o.keep_int && sort_every == o.sort_every && stride == o.stride && np == o.np &&
                   G == o.G && brick == o.brick;
        }
    } layout_;
};

template <class Fn> int guarded(dmpm_ctx* ctx, Fn fn) {
    if (!ctx) return DMPM_ERR_ARG;
    try {
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            ctx->err = "cudaSetDevice failed";
            return DMPM_ERR_CUDA;
        }
        return fn();
    } catch (const CudaError& e) {
        ctx->err = e.what;
        return e.code == cudaErrorMemoryAllocation ? DMPM_ERR_OOM : DMPM_ERR_CUDA;
    } catch (const ArgError& e) {
        ctx->err = e.what;
        return DMPM_ERR_ARG;
    } catch (const StateError& e) {
        ctx->err = e.what;
        return DMPM_ERR_STATE;
    } catch (const std::bad_alloc&) {
        ctx->err = "host allocation failed";
        return DMPM_ERR_OOM;
    }
}

template <class Fn> int with_engine(dmpm_ctx* ctx, Fn fn) {
    return guarded(ctx, [&]() -> int {
        if (ctx->precision == DMPM_FP64) return fn(*static_cast<Engine<double>*>(ctx->eng.get()));
        return fn(*static_cast<Engine<float>*>(ctx->eng.get()));
    });
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

void dmpm_default_params(dmpm_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->dt = 1.0 / 120.0;  // CompGraph.h:56-58 defaults
    p->drag = 0.5;
    p->smoothing = 0.1;
    p->adjoint_mode = DMPM_ADJ_REFCOMPAT;
    p->control_mode = DMPM_CTRL_PER_LAYER;
    p->loss_kind = DMPM_LOSS_REF_LOGMASS;
    p->brick_cells = 2;  // G2P over 2^3-cell bricks (36.7 against 48.1 us per step on 64^3, 267k particles)
}

int dmpm_create(int device, int precision, dmpm_ctx** out) {
    if (!out) return DMPM_ERR_ARG;
    *out = nullptr;
    if (precision != DMPM_FP64 && precision != DMPM_FP32_MIXED) return DMPM_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return DMPM_ERR_CUDA;
    }
    dmpm_ctx* c = new dmpm_ctx();
    c->device = device;
    c->precision = precision;
    dmpm_default_params(&c->prm);
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return DMPM_ERR_CUDA;
    }
    if (precision == DMPM_FP64) c->eng.reset(new Engine<double>(c));
    else c->eng.reset(new Engine<float>(c));
    *out = c;
    return DMPM_OK;
}

int dmpm_destroy(dmpm_ctx* ctx) {
    if (!ctx) return DMPM_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->eng.reset();
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return DMPM_OK;
}

const char* dmpm_last_error(const dmpm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int dmpm_get_info(const dmpm_ctx* ctx, int64_t* info, int count) {
    if (!ctx || !info) return DMPM_ERR_ARG;
    if (ctx->precision == DMPM_FP64) static_cast<Engine<double>*>(ctx->eng.get())->info(info, count);
    else static_cast<Engine<float>*>(ctx->eng.get())->info(info, count);
    return DMPM_OK;
}

int dmpm_set_device_limit(dmpm_ctx* ctx, int64_t max_bytes) {
    if (!ctx) return DMPM_ERR_ARG;
    if (max_bytes < 0) {
        ctx->err = "device byte limit must be >= 0";
        return DMPM_ERR_ARG;
    }
    ctx->budget.cap = (size_t)max_bytes;
    return DMPM_OK;
}

int dmpm_set_grid(dmpm_ctx* ctx, int dim_x, int dim_y, int dim_z, double dx, const double* min_point) {
    return with_engine(ctx, [&](auto& e) { e.set_grid(dim_x, dim_y, dim_z, dx, min_point); return DMPM_OK; });
}

int dmpm_set_params(dmpm_ctx* ctx, const dmpm_params* p) {
    if (!ctx || !p) return DMPM_ERR_ARG;
    if (!(p->dt >= 0) || p->adjoint_mode < 0 || p->adjoint_mode > 1 || p->control_mode < 0 || p->control_mode > 1 ||
        p->loss_kind < 0 || p->loss_kind > 1 || p->checkpoint_every < 0 || p->block_size < 0 || p->block_size > 256 ||
        (p->block_size % 32) != 0 || p->tile_cap < 0 || p->tile_cap > 1536 || p->sort_every < 0 ||
        p->warp_general < 0 || p->warp_general > 1 || p->control_stride < 0 || p->eager < 0 || p->eager > 1 ||
        (p->brick_cells != 0 && p->brick_cells != 2 && p->brick_cells != 4) || p->deterministic < 0 ||
        p->deterministic > 1 || p->reorder_particles < 0 || p->reorder_particles > 1) {
        ctx->err = "invalid dmpm_params";
        return DMPM_ERR_ARG;
    }
    ctx->prm = *p;
    ctx->prm_gen++;
    return DMPM_OK;
}

int dmpm_set_particles(dmpm_ctx* ctx, int n, const double* x, const double* v, const double* F, const double* C,
                       const double* dFc, const double* m, const double* vol, const double* lam, const double* mu) {
    return with_engine(ctx, [&](auto& e) { e.set_particles(n, x, v, F, C, dFc, m, vol, lam, mu); return DMPM_OK; });
}

int dmpm_set_points_ref(dmpm_ctx* ctx, const void* points, int n) {
    return with_engine(ctx, [&](auto& e) { e.set_points_ref(points, n); return DMPM_OK; });
}

int dmpm_compute_volumes(dmpm_ctx* ctx) {
    return with_engine(ctx, [&](auto& e) { e.compute_volumes(); return DMPM_OK; });
}

int dmpm_set_target_mass(dmpm_ctx* ctx, const double* target_m) {
    if (!target_m) return DMPM_ERR_ARG;
    return with_engine(ctx, [&](auto& e) { e.set_target_mass(target_m); return DMPM_OK; });
}

int dmpm_get_target_mass(dmpm_ctx* ctx, double* out) {
    return with_engine(ctx, [&](auto& e) { e.get_target_mass(out); return DMPM_OK; });
}

int dmpm_rasterize_target(dmpm_ctx* ctx, int n, const double* x, double point_mass) {
    return with_engine(ctx, [&](auto& e) { e.rasterize_target(n, x, point_mass); return DMPM_OK; });
}

int dmpm_setup(dmpm_ctx* ctx, int num_layers) {
    return with_engine(ctx, [&](auto& e) { e.setup(num_layers); return DMPM_OK; });
}

int dmpm_forward(dmpm_ctx* ctx, int start_layer) {
    return with_engine(ctx, [&](auto& e) {
        e.forward(start_layer);
        return (e.last_status() & ST_NONFINITE_FWD) ? DMPM_ERR_NONFINITE : DMPM_OK;
    });
}

int dmpm_loss(dmpm_ctx* ctx, double* loss) {
    return with_engine(ctx, [&](auto& e) {
        const double L = e.loss();
        if (loss) *loss = L;
        return (e.last_status() & ST_NONFINITE_LOSS) ? DMPM_ERR_NONFINITE : DMPM_OK;
    });
}

int dmpm_backward(dmpm_ctx* ctx, int control_layer) {
    return with_engine(ctx, [&](auto& e) {
        e.backward(control_layer);
        return (e.last_status() & ST_NONFINITE_ADJ) ? DMPM_ERR_NONFINITE : DMPM_OK;
    });
}

int dmpm_backward_range(dmpm_ctx* ctx, int top_layer, int control_layer) {
    return with_engine(ctx, [&](auto& e) {
        e.backward_range(top_layer, control_layer);
        return (e.last_status() & ST_NONFINITE_ADJ) ? DMPM_ERR_NONFINITE : DMPM_OK;
    });
}

int dmpm_get_particles(dmpm_ctx* ctx, int layer, int field, double* out) {
    return with_engine(ctx, [&](auto& e) { e.get_particles(layer, field, out); return DMPM_OK; });
}

int dmpm_set_layer_particles(dmpm_ctx* ctx, int layer, int field, const double* in) {
    return with_engine(ctx, [&](auto& e) { e.set_layer_particles(layer, field, in); return DMPM_OK; });
}

int dmpm_get_grid(dmpm_ctx* ctx, int layer, int field, double* out) {
    return with_engine(ctx, [&](auto& e) { e.get_grid(layer, field, out); return DMPM_OK; });
}

int dmpm_adam_step(dmpm_ctx* ctx, int layer, double lr, double beta1, double beta2, double eps, int t,
                   int normalize) {
    return with_engine(ctx, [&](auto& e) { e.adam_step(layer, lr, beta1, beta2, eps, t, normalize != 0); return DMPM_OK; });
}

int dmpm_descend(dmpm_ctx* ctx, int layer, int rule, double lr, double beta1, double beta2, double eps, int t,
                 int normalize) {
    return with_engine(ctx, [&](auto& e) {
        e.descend(layer, rule, lr, beta1, beta2, eps, t, normalize != 0);
        return DMPM_OK;
    });
}

int dmpm_get_control_grad(dmpm_ctx* ctx, int layer, double* out) {
    return with_engine(ctx, [&](auto& e) { e.get_control_grad(layer, out); return DMPM_OK; });
}

int dmpm_dldf_norm(dmpm_ctx* ctx, int layer, double* norm) {
    if (!norm) return DMPM_ERR_ARG;
    return with_engine(ctx, [&](auto& e) { *norm = e.dldf_norm(layer); return DMPM_OK; });
}

int dmpm_get_points_ref(dmpm_ctx* ctx, int layer, void* points) {
    return with_engine(ctx, [&](auto& e) { e.get_points_ref(layer, points); return DMPM_OK; });
}

int dmpm_synchronize(dmpm_ctx* ctx) {
    return guarded(ctx, [&]() { DMPM_CK(cudaStreamSynchronize(ctx->stream)); return DMPM_OK; });
}

void* dmpm_stream(dmpm_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int dmpm_cell_sort(dmpm_ctx* ctx, int layer, uint32_t* keys, uint32_t* order, uint32_t* item_start, int* n_items) {
    return guarded(ctx, [&]() -> int {
        if (ctx->precision != DMPM_FP32_MIXED) {
            ctx->err = "the cell sort belongs to the FP32 path";
            return DMPM_ERR_STATE;
        }
        static_cast<Engine<float>*>(ctx->eng.get())->debug_cell_sort(layer, keys, order, item_start, n_items);
        return DMPM_OK;
    });
}

int dmpm_set_profiling(dmpm_ctx* ctx, int on) {
    return with_engine(ctx, [&](auto& e) { e.set_profiling(on != 0); return DMPM_OK; });
}

int dmpm_kernel_stats(dmpm_ctx* ctx, int kernel_id, double* total_ms, int64_t* launches) {
    return with_engine(ctx, [&](auto& e) { e.kernel_stats(kernel_id, total_ms, launches); return DMPM_OK; });
}

const char* dmpm_kernel_name(int kernel_id) {
    return (kernel_id >= 0 && kernel_id < K_COUNT) ? kKernelNames[kernel_id] : nullptr;
}

int64_t dmpm_launch_count(const dmpm_ctx* ctx) { return ctx ? ctx->launches : -1; }

}  // extern "C"
