// batch.cu -- many independent scenes advanced together (dmpm_batch_*,
// include/dmpm.h).
//
// Layout.  Instances are ordered by time steps, longest first (ties keep the
// creation order).  Their particles are concatenated in that order, so are
// their grids (node offset goff) and their cell-key ranges (key offset koff).
// Layer t holds the instances whose rollouts reach it (steps >= t): a prefix
// of that order, stored with its own plane stride S_t.  Time step t advances
// the instances with steps > t, again a prefix: P_t particles, G_t nodes.
//
// Launches.  Every stage of a time step is one launch over the prefix: the
// per-particle kernels (k_stress, k_adj_finalize) over P_t particles, the node
// kernels over G_t nodes, and the warp-item kernels (P2G, G2P, adjoint
// scatter and gather) as persistent grids of ctas_per_sm CTAs per SM looping
// over the warp items of the active instances.  Items never mix instances
// (cell keys carry the instance's key offset); each warp looks up its item's
// grid.  The item count lives on the device -- the cell sort writes the end
// of every instance's items -- so no result is read back inside a gradient
// evaluation and the whole evaluation can be captured once as a CUDA graph.
//
// Losses.  EndLayerMassLoss (CompGraph.cpp:110-244) of instance i is
// evaluated on its last layer when the backward sweep reaches that layer; its
// dL/dx seeds the instance's adjoint there, in the part of the layer's
// adjoint buffer that the later instances' adjoint steps leave untouched.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "dmpm.h"
#include "host_common.cuh"
#include "kernels.cuh"
#include "kernels_warp.cuh"

using namespace dmpm;
using namespace dmpm_host;

namespace {

constexpr int kAux = 24;  // G (9), polar R (9), polar S (6) per particle and step
constexpr int kDefaultSortEvery = 8;
constexpr int kDefaultCtasPerSm = 3;

// cell key of each particle of the active prefix: its instance's key offset +
// the one-scene key of sort.cuh (the stencil base the warp-item kernels form)
__global__ void k_cell_keys_batch(int n, size_t np, const float* __restrict__ st, const uint16_t* __restrict__ pinst,
                                  const InstGeo* __restrict__ ig, uint32_t* keys, uint32_t* vals) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const InstGeo g = ig[pinst[p]];
    int base[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
        (void)stencil_coord<float>(load_xd(st, np, p, c, 1), g.g.mn[c], 1.0 / g.g.dx, g.g.dim[c], base[c]);
    keys[p] = g.koff + cell_key(base, g.g.dim);
    vals[p] = (uint32_t)p;
}

// instance of every warp item, and one past the last item of each instance
// (items of an instance are contiguous: its keys form one range)
__global__ void k_item_inst(const uint32_t* __restrict__ order, const uint32_t* __restrict__ items,
                            const uint32_t* __restrict__ n_items, const uint16_t* __restrict__ pinst, int cap,
                            uint16_t* item_inst, uint32_t* item_end) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int ni = (int)*n_items;
    if (j >= ni || j >= cap) return;
    const uint16_t i = pinst[order[items[j]]];
    item_inst[j] = i;
    if (j + 1 == ni || pinst[order[items[j + 1]]] != i) item_end[i] = (uint32_t)(j + 1);
}

__global__ void k_set_target(const double* __restrict__ src, size_t G, float* dst) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < G) dst[i] = (float)src[i];
}

__global__ void k_fill_u16(uint16_t* dst, int n, uint16_t v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = v;
}

struct Inst {
    int user;  // creation index
    int n, steps;
    GridGeom geo;
    size_t G;
    size_t poff, goff;
    uint32_t koff;
};

struct BEpoch {
    uint32_t* order = nullptr;
    uint32_t* items = nullptr;
    uint16_t* item_inst = nullptr;
    uint32_t* item_end = nullptr;  // [instances]
    uint32_t* n_items = nullptr;   // device scalar
};

}  // namespace

struct dmpm_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    // second stream for the finalize's transport part, forked from and joined
    // back into stream by the two events
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::string err;
    struct Impl;
    std::unique_ptr<Impl> impl;
};

struct dmpm_batch::Impl {
    dmpm_batch* b;
    dmpm_params prm{};
    dmpm_batch_launch cfg{};
    std::vector<Inst> inst;      // internal order (steps descending)
    std::vector<int> user2int;
    int count = 0;
    size_t N = 0, np0 = 0, Gtot = 0;
    uint64_t keys_total = 0;
    int smax = 0;                // longest rollout (steps)
    int sms = 148;
    // per layer t = 0..smax: instances, particles, plane stride
    std::vector<int> A;
    std::vector<size_t> P, S;
    std::vector<size_t> node_prefix;  // nodes of the first a instances
    // device
    Arena scene, layers, epochs_arena, staging_arena;
    float* st0 = nullptr;        // layer 0 state [24][np0]
    float* cst = nullptr;        // [4][np0]
    float* dfc = nullptr;        // [9][np0]
    uint16_t* pinst = nullptr;   // instance of each particle
    InstGeo* ig = nullptr;
    float* target = nullptr;     // [Gtot]
    float* dldm = nullptr;       // [Gtot]
    node4<float>* scratch = nullptr;  // loss mass raster [Gtot]
    double* loss_acc = nullptr;  // [count]
    unsigned* status = nullptr;
    double* staging = nullptr;
    size_t staging_count = 0;
    void* host_misc = nullptr;   // pinned: losses + status
    std::vector<float*> st, aux;
    std::vector<node4<float>*> grid;
    float* adj[2] = {nullptr, nullptr};
    float *adjn = nullptr, *gath = nullptr;
    node4<float>*gadj = nullptr, *gadj2 = nullptr;
    double* ctrl_acc = nullptr;
    std::vector<BEpoch> ep;
    int ep_every = 0;
    uint32_t *sk[2] = {nullptr, nullptr}, *sv[2] = {nullptr, nullptr}, *sh = nullptr, *sf = nullptr;
    uint32_t *counts = nullptr, *tile_tot = nullptr;
    bool ready = false;
    cudaGraphExec_t gexec = nullptr;
    int64_t launches = 0;        // launches enqueued by one gradient evaluation
    bool done = false;           // a gradient has been evaluated

    explicit Impl(dmpm_batch* owner) : b(owner) {}
    ~Impl() { drop_graph(); if (host_misc) cudaFreeHost(host_misc); }

    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
    }
    void launched() {
        launches++;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) throw CudaError{e, std::string("kernel launch: ") + cudaGetErrorString(e)};
    }
    int sort_every() const { return cfg.sort_every > 0 ? cfg.sort_every : kDefaultSortEvery; }
    int ctas_per_sm() const { return cfg.ctas_per_sm > 0 ? cfg.ctas_per_sm : kDefaultCtasPerSm; }
    int particle_block() const { return cfg.particle_block > 0 ? cfg.particle_block : 256; }

    // ------------------------------------------------------------ creation
    void create(const dmpm_instance* in, int cnt) {
        if (cnt < 1 || cnt > 65535 || !in) throw ArgError{"instance count must be in 1..65535"};
        count = cnt;
        std::vector<int> idx(cnt);
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) { return in[a].steps > in[c].steps; });
        user2int.assign(cnt, 0);
        size_t poff = 0, goff = 0;
        uint64_t koff = 0;
        for (int k = 0; k < cnt; k++) {
            const dmpm_instance& d = in[idx[k]];
            if (d.n < 1 || d.steps < 1 || d.dim_x < 1 || d.dim_y < 1 || d.dim_z < 1 || !(d.dx > 0))
                throw ArgError{"instance " + std::to_string(idx[k]) + ": n, steps and dims must be >= 1, dx > 0"};
            if (d.dx != in[0].dx) throw ArgError{"instances of a batch share dx"};
            Inst s{};
            s.user = idx[k];
            s.n = d.n;
            s.steps = d.steps;
            s.geo.dim[0] = d.dim_x;
            s.geo.dim[1] = d.dim_y;
            s.geo.dim[2] = d.dim_z;
            s.geo.dx = d.dx;
            for (int c = 0; c < 3; c++) s.geo.mn[c] = d.min_point[c];
            s.G = (size_t)d.dim_x * d.dim_y * d.dim_z;
            s.poff = poff;
            s.goff = goff;
            s.koff = (uint32_t)koff;
            poff += (size_t)d.n;
            goff += s.G;
            const int dims[3] = {d.dim_x, d.dim_y, d.dim_z};
            koff += key_span(dims);
            user2int[idx[k]] = k;
            inst.push_back(s);
        }
        if (poff >= (1ull << 31) || goff >= (1ull << 31) || koff >= (1ull << 32))
            throw ArgError{"batch too large: particles and nodes must stay below 2^31, cell keys below 2^32"};
        N = poff;
        Gtot = goff;
        keys_total = koff;
        np0 = round_up(N, 64);
        smax = inst.front().steps;
        A.assign(smax + 2, 0);
        P.assign(smax + 2, 0);
        S.assign(smax + 2, 0);
        for (int t = 0; t <= smax + 1; t++) {
            for (const Inst& s : inst)
                if (s.steps >= t) { A[t]++; P[t] += (size_t)s.n; }
            S[t] = round_up(std::max<size_t>(P[t], 1), 64);
        }
        node_prefix.assign(cnt + 1, 0);
        for (int k = 0; k < cnt; k++) node_prefix[k + 1] = node_prefix[k] + inst[k].G;
        int dev = 0;
        DMPM_CK(cudaGetDevice(&dev));
        DMPM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        dmpm_default_params(&prm);
        prm.adjoint_mode = DMPM_ADJ_EXACT;
        // scene storage
        st0 = (float*)scene.alloc((size_t)NSTATE_X * np0 * sizeof(float));
        cst = (float*)scene.alloc((size_t)NCONST * np0 * sizeof(float));
        dfc = (float*)scene.alloc((size_t)9 * np0 * sizeof(float));
        pinst = (uint16_t*)scene.alloc(np0 * sizeof(uint16_t));
        ig = (InstGeo*)scene.alloc(cnt * sizeof(InstGeo));
        target = (float*)scene.alloc(Gtot * sizeof(float));
        dldm = (float*)scene.alloc(Gtot * sizeof(float));
        scratch = (node4<float>*)scene.alloc(Gtot * sizeof(node4<float>));
        loss_acc = (double*)scene.alloc(cnt * sizeof(double));
        status = (unsigned*)scene.alloc(16);
        DMPM_CK(cudaMemsetAsync(st0, 0, (size_t)NSTATE_X * np0 * sizeof(float), b->stream));
        DMPM_CK(cudaMemsetAsync(cst, 0, (size_t)NCONST * np0 * sizeof(float), b->stream));
        DMPM_CK(cudaMemsetAsync(dfc, 0, (size_t)9 * np0 * sizeof(float), b->stream));
        DMPM_CK(cudaMemsetAsync(target, 0, Gtot * sizeof(float), b->stream));
        std::vector<InstGeo> h(cnt);
        for (int k = 0; k < cnt; k++) {
            h[k].g = inst[k].geo;
            h[k].goff = (int)inst[k].goff;
            h[k].koff = inst[k].koff;
            k_fill_u16<<<(inst[k].n + 255) / 256, 256, 0, b->stream>>>(pinst + inst[k].poff, inst[k].n, (uint16_t)k);
            launched();
        }
        DMPM_CK(cudaMemcpyAsync(ig, h.data(), cnt * sizeof(InstGeo), cudaMemcpyHostToDevice, b->stream));
        DMPM_CK(cudaMallocHost(&host_misc, (size_t)(cnt + 2) * sizeof(double)));
        DMPM_CK(cudaStreamSynchronize(b->stream));
    }

    double* stage(size_t count_d) {
        if (count_d > staging_count) {
            staging_arena.release();
            staging = (double*)staging_arena.alloc(count_d * sizeof(double));
            staging_count = count_d;
        }
        return staging;
    }
    const Inst& user_inst(int u) const {
        if (u < 0 || u >= count) throw ArgError{"instance out of range"};
        return inst[user2int[u]];
    }
    // diag: added to the diagonal of 3x3 matrices on the way (F <-> strain H = F - I,
    // the layer storage of the FP32 kernels)
    void upload(const double* host, int n, int width, float* dst, size_t np, double diag = 0.0) {
        double* s = stage((size_t)n * width);
        DMPM_CK(cudaMemcpyAsync(s, host, (size_t)n * width * sizeof(double), cudaMemcpyHostToDevice, b->stream));
        if (diag != 0.0) {
            k_diag_add<<<(unsigned)(((size_t)n * 3 + 255) / 256), 256, 0, b->stream>>>(s, n, diag);
            launched();
        }
        const size_t tot = (size_t)n * width;
        k_unpack<float><<<(unsigned)((tot + 255) / 256), 256, 0, b->stream>>>(s, width, n, dst, np);
        launched();
    }
    void download(const float* src, size_t np, int n, int width, double* host, double diag = 0.0) {
        double* s = stage((size_t)n * width);
        const size_t tot = (size_t)n * width;
        k_pack<float><<<(unsigned)((tot + 255) / 256), 256, 0, b->stream>>>(src, np, width, n, s);
        launched();
        if (diag != 0.0) {
            k_diag_add<<<(unsigned)(((size_t)n * 3 + 255) / 256), 256, 0, b->stream>>>(s, n, diag);
            launched();
        }
        DMPM_CK(cudaMemcpyAsync(host, s, tot * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        DMPM_CK(cudaStreamSynchronize(b->stream));
    }

    void set_particles(int u, const double* x, const double* v, const double* F, const double* C, const double* dFc,
                       const double* m, const double* vol, const double* lam, const double* mu) {
        if (!x || !m || !lam || !mu) throw ArgError{"x, m, lam and mu are required"};
        const Inst& s = user_inst(u);
        const int n = s.n;
        float* l0 = st0 + s.poff;
        {  // compensated positions: hi and lo planes
            double* sx = stage((size_t)n * 3);
            DMPM_CK(cudaMemcpyAsync(sx, x, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice, b->stream));
            k_unpack_x2<<<(unsigned)(((size_t)n * 3 + 255) / 256), 256, 0, b->stream>>>(
                sx, n, l0 + (size_t)PX * np0, l0 + (size_t)PXL * np0, np0);
            launched();
        }
        if (v) upload(v, n, 3, l0 + (size_t)PV * np0, np0);
        else for (int c = 0; c < 3; c++) DMPM_CK(cudaMemsetAsync(l0 + (size_t)(PV + c) * np0, 0, n * sizeof(float), b->stream));
        std::vector<double> eye;
        if (!F) {
            eye.assign((size_t)n * 9, 0.0);
            for (int p = 0; p < n; p++) eye[9 * p] = eye[9 * p + 4] = eye[9 * p + 8] = 1.0;
            F = eye.data();
        }
        upload(F, n, 9, l0 + (size_t)PF * np0, np0, -1.0);
        if (C) upload(C, n, 9, l0 + (size_t)PC * np0, np0);
        else for (int c = 0; c < 9; c++) DMPM_CK(cudaMemsetAsync(l0 + (size_t)(PC + c) * np0, 0, n * sizeof(float), b->stream));
        if (dFc) upload(dFc, n, 9, dfc + s.poff, np0);
        else for (int c = 0; c < 9; c++) DMPM_CK(cudaMemsetAsync(dfc + (size_t)c * np0 + s.poff, 0, n * sizeof(float), b->stream));
        upload(m, n, 1, cst + (size_t)KM * np0 + s.poff, np0);
        if (vol) upload(vol, n, 1, cst + (size_t)KVOL * np0 + s.poff, np0);
        else DMPM_CK(cudaMemsetAsync(cst + (size_t)KVOL * np0 + s.poff, 0, n * sizeof(float), b->stream));
        upload(lam, n, 1, cst + (size_t)KLAM * np0 + s.poff, np0);
        upload(mu, n, 1, cst + (size_t)KMU * np0 + s.poff, np0);
        DMPM_CK(cudaStreamSynchronize(b->stream));
        done = false;
    }

    void set_target(int u, const double* m) {
        if (!m) throw ArgError{"target is NULL"};
        const Inst& s = user_inst(u);
        double* st_ = stage(s.G);
        DMPM_CK(cudaMemcpyAsync(st_, m, s.G * sizeof(double), cudaMemcpyHostToDevice, b->stream));
        k_set_target<<<(unsigned)((s.G + 255) / 256), 256, 0, b->stream>>>(st_, s.G, target + s.goff);
        launched();
        DMPM_CK(cudaStreamSynchronize(b->stream));
        done = false;
    }

    void set_params(const dmpm_params& p) {
        if (p.control_mode != DMPM_CTRL_TIED && p.control_mode != DMPM_CTRL_PER_LAYER)
            throw ArgError{"invalid control mode"};
        prm = p;
        if (p.sort_every > 0) cfg.sort_every = p.sort_every;
        drop_graph();
        done = false;
        if (ready && ep_every != sort_every()) alloc_epochs();
    }

    void set_launch(const dmpm_batch_launch& c) {
        if (c.sort_every < 0 || c.ctas_per_sm < 0 || c.ctas_per_sm > 8 ||
            (c.particle_block != 0 && c.particle_block != 128 && c.particle_block != 256) || c.use_graph < 0 ||
            c.use_graph > 1)
            throw ArgError{"invalid launch configuration"};
        cfg = c;
        drop_graph();
        if (ready && ep_every != sort_every()) alloc_epochs();
    }

    // ------------------------------------------------------------ storage
    void alloc_epochs() {
        drop_graph();
        epochs_arena.release();
        ep.clear();
        const int se = sort_every();
        const int nep = (smax + se - 1) / se;
        for (int e = 0; e < nep; e++) {
            const size_t n = P[e * se + 1];  // particles stepping at the epoch's first step
            BEpoch x;
            x.order = (uint32_t*)epochs_arena.alloc(n * 4);
            x.items = (uint32_t*)epochs_arena.alloc((n + 1) * 4);
            x.item_inst = (uint16_t*)epochs_arena.alloc(n * 2);
            x.item_end = (uint32_t*)epochs_arena.alloc((size_t)count * 4);
            x.n_items = (uint32_t*)epochs_arena.alloc(16);
            DMPM_CK(cudaMemsetAsync(x.item_end, 0, (size_t)count * 4, b->stream));
            DMPM_CK(cudaMemsetAsync(x.n_items, 0, 16, b->stream));
            ep.push_back(x);
        }
        ep_every = se;
    }

    size_t layer_bytes() const {
        size_t tot = 0;
        for (int t = 1; t <= smax; t++) tot += (size_t)NSTATE_X * S[t] * 4;               // states
        for (int t = 0; t < smax; t++) tot += (size_t)kAux * S[t] * 4 + node_prefix[A[t + 1]] * 16;  // aux, grids
        tot += 2 * (size_t)NSTATE * np0 * 4 + (12 + 18) * np0 * 4 + 9 * np0 * 8 + 3 * Gtot * 16;
        return tot;
    }

    void setup() {
        drop_graph();
        layers.release();
        ready = false;
        size_t free_b = 0, total_b = 0;
        DMPM_CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t need = layer_bytes();
        if (need > free_b) {
            throw CudaError{cudaErrorMemoryAllocation, "batch needs " + std::to_string(need >> 20) + " MiB of layer storage, " +
                                                           std::to_string(free_b >> 20) + " MiB free"};
        }
        st.assign(smax + 1, nullptr);
        aux.assign(smax, nullptr);
        grid.assign(smax, nullptr);
        st[0] = st0;
        for (int t = 1; t <= smax; t++) st[t] = (float*)layers.alloc((size_t)NSTATE_X * S[t] * 4);
        for (int t = 0; t < smax; t++) {
            aux[t] = (float*)layers.alloc((size_t)kAux * S[t] * 4);
            grid[t] = (node4<float>*)layers.alloc(node_prefix[A[t + 1]] * sizeof(node4<float>));
        }
        adj[0] = (float*)layers.alloc((size_t)NSTATE * np0 * 4);
        adj[1] = (float*)layers.alloc((size_t)NSTATE * np0 * 4);
        adjn = (float*)layers.alloc((size_t)12 * np0 * 4);
        gath = (float*)layers.alloc((size_t)18 * np0 * 4);
        ctrl_acc = (double*)layers.alloc((size_t)9 * np0 * 8);
        gadj = (node4<float>*)layers.alloc(Gtot * sizeof(node4<float>));
        gadj2 = (node4<float>*)layers.alloc(2 * Gtot * sizeof(node4<float>));
        for (int i = 0; i < 2; i++) {
            sk[i] = (uint32_t*)layers.alloc(np0 * 4);
            sv[i] = (uint32_t*)layers.alloc(np0 * 4);
        }
        sh = (uint32_t*)layers.alloc(np0 * 4);
        sf = (uint32_t*)layers.alloc(np0 * 4);
        const size_t rs_tiles = (N + RS_TILE - 1) / RS_TILE;
        counts = (uint32_t*)layers.alloc(256 * rs_tiles * 4);
        const size_t mx = std::max(N, 256 * rs_tiles);
        tile_tot = (uint32_t*)layers.alloc(((mx + SCAN_TILE - 1) / SCAN_TILE + 1) * 4);
        DMPM_CK(cudaMemsetAsync(adj[0], 0, (size_t)NSTATE * np0 * 4, b->stream));
        DMPM_CK(cudaMemsetAsync(adj[1], 0, (size_t)NSTATE * np0 * 4, b->stream));
        alloc_epochs();
        DMPM_CK(cudaStreamSynchronize(b->stream));
        ready = true;
        done = false;
    }

    // ------------------------------------------------------------ recording
    template <class Op> void scan(uint32_t* data, size_t n, uint32_t* grand) {
        const int tiles = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
        k_scan_tiles<Op><<<tiles, SCAN_THREADS, 0, b->stream>>>(data, (int)n, tile_tot);
        launched();
        k_scan_totals<Op><<<1, 1024, 0, b->stream>>>(tile_tot, tiles, grand);
        launched();
        k_scan_add<Op><<<tiles, SCAN_THREADS, 0, b->stream>>>(data, (int)n, tile_tot);
        launched();
    }

    // stable sort of the particles stepping at t (layer t) by instance-prefixed cell key
    void cell_sort(int t, BEpoch& e) {
        const int n = (int)P[t + 1];
        k_cell_keys_batch<<<(n + 255) / 256, 256, 0, b->stream>>>(n, S[t], st[t], pinst, ig, sk[0], sv[0]);
        launched();
        int bits = 1;
        while (bits < 32 && (1ull << bits) < keys_total) bits++;
        const int rs_tiles = (n + RS_TILE - 1) / RS_TILE;
        int cur = 0;
        for (int shift = 0; shift < bits; shift += 8) {
            k_rs_upsweep<<<rs_tiles, RS_THREADS, 0, b->stream>>>(sk[cur], n, shift, counts, rs_tiles);
            launched();
            scan<OpSum>(counts, (size_t)256 * rs_tiles, nullptr);
            k_rs_downsweep<<<rs_tiles, RS_THREADS, 0, b->stream>>>(sk[cur], sv[cur], sk[cur ^ 1], sv[cur ^ 1], n, shift,
                                                                  counts, rs_tiles);
            launched();
            cur ^= 1;
        }
        DMPM_CK(cudaMemcpyAsync(e.order, sv[cur], (size_t)n * 4, cudaMemcpyDeviceToDevice, b->stream));
        k_run_heads<<<(n + 255) / 256, 256, 0, b->stream>>>(sk[cur], n, sh);
        launched();
        scan<OpMax>(sh, (size_t)n, nullptr);
        k_item_flags<<<(n + 255) / 256, 256, 0, b->stream>>>(sk[cur], sh, n, sf);
        launched();
        scan<OpSum>(sf, (size_t)n, e.n_items);
        k_item_starts<<<(n + 255) / 256, 256, 0, b->stream>>>(sk[cur], sh, sf, n, e.items);
        launched();
        k_item_sentinel<<<1, 1, 0, b->stream>>>(e.items, e.n_items, n);
        launched();
        k_item_inst<<<(n + 255) / 256, 256, 0, b->stream>>>(e.order, e.items, e.n_items, pinst, n, e.item_inst,
                                                            e.item_end);
        launched();
    }

    WArgs args(int t) const {
        WArgs a{};
        a.n = (int)P[t + 1];
        a.np = np0;
        a.npl = S[t];
        a.npn = S[t + 1];
        a.geo = inst.front().geo;  // dx of the per-particle kernels (shared by every instance)
        a.dt = (float)prm.dt;
        a.drag = (float)prm.drag;
        a.s = (float)prm.smoothing;
        for (int c = 0; c < 3; c++) a.fext[c] = (float)prm.f_ext[c];
        const BEpoch& e = ep[t / ep_every];
        a.items = WarpItems{e.order, e.items, 0};
        a.n_items_dev = e.item_end + (A[t + 1] - 1);
        a.ig = ig;
        a.item_inst = e.item_inst;
        a.st = st[t];
        a.st_next = st[t + 1];
        a.xlo = 1;
        a.cst = cst;
        a.dfc = dfc;
        a.G = aux[t];
        a.grid = grid[t];
        a.status = status;
        return a;
    }
    unsigned warp_blocks(int t) const {
        const size_t most = (P[t + 1] * 32 + 255) / 256;  // one item per particle at most
        return (unsigned)std::max<size_t>(1, std::min<size_t>(most, (size_t)sms * ctas_per_sm()));
    }
    // the adjoint scatter's persistent grid: its own blocks per SM (kernels_warp.cuh), not the tuned setting
    unsigned scatter_blocks(int t) const {
        const size_t most = (P[t + 1] * 32 + DMPM_ADJ_SCATTER_THREADS - 1) / DMPM_ADJ_SCATTER_THREADS;
        return (unsigned)std::max<size_t>(1, std::min<size_t>(most, (size_t)sms * DMPM_ADJ_SCATTER_CTAS));
    }

    void step(int t) {
        WArgs a = args(t);
        const size_t Gt = node_prefix[A[t + 1]];
        const int pb = particle_block();
        const unsigned wb = warp_blocks(t);
        DMPM_CK(cudaMemsetAsync(grid[t], 0, Gt * sizeof(node4<float>), b->stream));
        k_stress<false><<<(unsigned)((a.n + pb - 1) / pb), pb, 0, b->stream>>>(a);
        launched();
        k_p2g_w<false, ITEMS_BATCH><<<wb, DMPM_P2G_THREADS, 0, b->stream>>>(a);
        launched();
        k_gop_inplace<<<(unsigned)((Gt + 255) / 256), 256, 0, b->stream>>>(grid[t], Gt, a.dt, a.fext[0], a.fext[1],
                                                                             a.fext[2]);
        launched();
        k_g2p_w<ITEMS_BATCH><<<wb, 256, 0, b->stream>>>(a);
        launched();
    }

    // EndLayerMassLoss of internal instance k on its last layer, seeding its adjoint there
    void loss(int k) {
        const Inst& s = inst[k];
        const int l = s.steps;
        LossArgs<float> la{};
        la.n = s.n;
        la.np = S[l];
        la.npc = np0;
        la.geo = s.geo;
        la.st = st[l] + s.poff;
        la.cst = cst + s.poff;
        la.grid = scratch + s.goff;
        la.target = target + s.goff;
        la.dldm = dldm + s.goff;
        la.adj = adj[l & 1] + s.poff;
        la.loss = loss_acc + k;
        la.kind = prm.loss_kind;
        la.tile_cap = 0;
        la.xlo = 1;
        la.status = status;
        DMPM_CK(cudaMemsetAsync(la.grid, 0, s.G * sizeof(node4<float>), b->stream));
        k_p2g_mass<float, false><<<(s.n + 255) / 256, 256, 0, b->stream>>>(la);
        launched();
        k_node_loss<float><<<(unsigned)((s.G + 255) / 256), 256, 0, b->stream>>>(la, s.G);
        launched();
        k_loss_dldx<float><<<(s.n + 255) / 256, 256, 0, b->stream>>>(la);
        launched();
    }

    void adjoint_step(int t) {
        WArgs a = args(t);
        a.adj_next = adj[(t + 1) & 1];
        a.adj = adj[t & 1];
        a.adjn = adjn;
        a.gath = gath;
        a.gadj = gadj;
        a.gadj2 = gadj2;
        a.ctrl_acc = ctrl_acc;
        const size_t Gt = node_prefix[A[t + 1]];
        const unsigned wb = warp_blocks(t);
        const bool ex = prm.adjoint_mode == DMPM_ADJ_EXACT;
        DMPM_CK(cudaMemsetAsync(gadj, 0, Gt * sizeof(node4<float>), b->stream));
        const unsigned ws = scatter_blocks(t);
        if (ex) k_adj_scatter_w<true, false, ITEMS_BATCH><<<ws, DMPM_ADJ_SCATTER_THREADS, 0, b->stream>>>(a);
        else k_adj_scatter_w<false, false, ITEMS_BATCH><<<ws, DMPM_ADJ_SCATTER_THREADS, 0, b->stream>>>(a);
        launched();
        const unsigned gb = (unsigned)((Gt + 255) / 256);
        if (ex) k_adj_gop_w<true><<<gb, 256, 0, b->stream>>>(grid[t], gadj, gadj2, Gt, a.dt, a.fext[0], a.fext[1], a.fext[2]);
        else k_adj_gop_w<false><<<gb, 256, 0, b->stream>>>(grid[t], gadj, gadj2, Gt, a.dt, a.fext[0], a.fext[1], a.fext[2]);
        launched();
        if (ex) k_adj_gather_w<true, ITEMS_BATCH><<<wb, DMPM_GATHER_THREADS, 0, b->stream>>>(a);
        else k_adj_gather_w<false, ITEMS_BATCH><<<wb, DMPM_GATHER_THREADS, 0, b->stream>>>(a);
        launched();
        DMPM_CK(cudaEventRecord(b->ev_fork, b->stream));
        DMPM_CK(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
        launch_finalize_split(a, ex, b->stream, b->side);
        launched();
        launched();
        DMPM_CK(cudaEventRecord(b->ev_join, b->side));
        DMPM_CK(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
    }

    // the whole gradient evaluation, enqueued on the stream (capturable: no
    // host synchronisation, no allocation)
    void record() {
        launches = 0;
        DMPM_CK(cudaMemsetAsync(status, 0, sizeof(unsigned), b->stream));
        DMPM_CK(cudaMemsetAsync(loss_acc, 0, count * sizeof(double), b->stream));
        DMPM_CK(cudaMemsetAsync(ctrl_acc, 0, (size_t)9 * np0 * sizeof(double), b->stream));
        for (int t = 0; t < smax; t++) {
            if (t % ep_every == 0) cell_sort(t, ep[t / ep_every]);
            step(t);
        }
        for (int t = smax - 1; t >= 0; t--) {
            for (int k = A[t + 2]; k < A[t + 1]; k++) loss(k);  // instances whose last layer is t + 1
            adjoint_step(t);
        }
    }

    void check_ready() const {
        if (!ready) throw StateError{"dmpm_batch_setup has not been called"};
    }

    int run_once() {
        if (cfg.use_graph) {
            if (!gexec) {
                DMPM_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
                try {
                    record();
                } catch (...) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(b->stream, &g);
                    if (g) cudaGraphDestroy(g);
                    cudaGetLastError();
                    throw;
                }
                cudaGraph_t g = nullptr;
                DMPM_CK(cudaStreamEndCapture(b->stream, &g));
                cudaError_t e = cudaGraphInstantiate(&gexec, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) {
                    gexec = nullptr;
                    throw CudaError{e, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
                }
            }
            DMPM_CK(cudaGraphLaunch(gexec, b->stream));
        } else {
            record();
        }
        return DMPM_OK;
    }

    int gradient(double* losses) {
        check_ready();
        run_once();
        char* hm = (char*)host_misc;
        DMPM_CK(cudaMemcpyAsync(hm, loss_acc, count * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        DMPM_CK(cudaMemcpyAsync(hm + count * sizeof(double), status, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream));
        DMPM_CK(cudaStreamSynchronize(b->stream));
        done = true;
        if (losses)
            for (int u = 0; u < count; u++) losses[u] = ((double*)hm)[user2int[u]];
        const unsigned stw = *(unsigned*)(hm + count * sizeof(double));
        if (stw) {
            b->err = "non-finite values in the batch (status " + std::to_string(stw) + ")";
            return DMPM_ERR_NONFINITE;
        }
        return DMPM_OK;
    }

    double time_config(int reps) {
        cudaEvent_t e0, e1;
        DMPM_CK(cudaEventCreate(&e0));
        DMPM_CK(cudaEventCreate(&e1));
        float ms = 0.f;
        try {
            run_once();  // capture (graph) or warm-up
            DMPM_CK(cudaEventRecord(e0, b->stream));
            for (int r = 0; r < reps; r++) run_once();
            DMPM_CK(cudaEventRecord(e1, b->stream));
            DMPM_CK(cudaEventSynchronize(e1));
            DMPM_CK(cudaEventElapsedTime(&ms, e0, e1));
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return ms / std::max(1, reps);
    }

    double autotune(int reps) {
        check_ready();
        if (reps < 1) throw ArgError{"reps must be >= 1"};
        const dmpm_batch_launch base = cfg;
        dmpm_batch_launch best = cfg;
        double best_ms = 1e300;
        for (int se : {4, 8, 16})
            for (int cps : {2, 3, 4, 6})
                for (int pb : {128, 256}) {
                    dmpm_batch_launch c = base;
                    c.sort_every = se;
                    c.ctas_per_sm = cps;
                    c.particle_block = pb;
                    set_launch(c);
                    const double ms = time_config(reps);
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = c;
                    }
                }
        set_launch(best);
        done = false;
        return best_ms;
    }

    void control_grad(int u, double* out) {
        check_ready();
        if (!out) throw ArgError{"out is NULL"};
        if (!done) throw StateError{"no gradient evaluated yet"};
        const Inst& s = user_inst(u);
        double* stg = stage((size_t)s.n * 9);
        k_pack_acc<float><<<(unsigned)(((size_t)s.n * 9 + 255) / 256), 256, 0, b->stream>>>(ctrl_acc + s.poff, np0,
                                                                                            s.n, stg);
        launched();
        DMPM_CK(cudaMemcpyAsync(out, stg, (size_t)s.n * 9 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        DMPM_CK(cudaStreamSynchronize(b->stream));
    }

    void get_particles(int u, int layer, int field, double* out) {
        if (!out) throw ArgError{"out is NULL"};
        const Inst& s = user_inst(u);
        if (layer < 0 || layer > s.steps) throw ArgError{"layer out of range"};
        if (layer > 0 && (!ready || !done)) throw StateError{"no gradient evaluated yet"};
        const float* base = (layer == 0 ? st0 : st[layer]) + s.poff;
        const size_t np = S[layer];
        switch (field) {
            case DMPM_F_X: {
                double* sx = stage((size_t)s.n * 3);
                k_pack_x2<<<(unsigned)(((size_t)s.n * 3 + 255) / 256), 256, 0, b->stream>>>(
                    base + (size_t)PX * np, base + (size_t)PXL * np, np, s.n, sx);
                launched();
                DMPM_CK(cudaMemcpyAsync(out, sx, (size_t)s.n * 3 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
                DMPM_CK(cudaStreamSynchronize(b->stream));
                break;
            }
            case DMPM_F_V: download(base + (size_t)PV * np, np, s.n, 3, out); break;
            case DMPM_F_F: download(base + (size_t)PF * np, np, s.n, 9, out, 1.0); break;
            case DMPM_F_C: download(base + (size_t)PC * np, np, s.n, 9, out); break;
            default: throw ArgError{"field must be DMPM_F_X, _V, _F or _C"};
        }
    }

    void info(int64_t* out, int cnt) const {
        const int64_t v[6] = {count, (int64_t)N, (int64_t)Gtot,
                              (int64_t)(scene.bytes() + layers.bytes() + epochs_arena.bytes()), launches,
                              gexec ? 1 : 0};
        for (int i = 0; i < cnt && i < 6; i++) out[i] = v[i];
    }
};

namespace {
template <class Fn> int bguard(dmpm_batch* b, Fn fn) {
    if (!b) return DMPM_ERR_ARG;
    try {
        if (cudaSetDevice(b->device) != cudaSuccess) {
            b->err = "cudaSetDevice failed";
            return DMPM_ERR_CUDA;
        }
        return fn(*b->impl);
    } catch (const CudaError& e) {
        b->err = e.what;
        return e.code == cudaErrorMemoryAllocation ? DMPM_ERR_OOM : DMPM_ERR_CUDA;
    } catch (const ArgError& e) {
        b->err = e.what;
        return DMPM_ERR_ARG;
    } catch (const StateError& e) {
        b->err = e.what;
        return DMPM_ERR_STATE;
    } catch (const std::bad_alloc&) {
        b->err = "host allocation failed";
        return DMPM_ERR_OOM;
    }
}
}  // namespace

extern "C" {

int dmpm_batch_create(int device, int count, const dmpm_instance* instances, dmpm_batch** out) {
    if (!out) return DMPM_ERR_ARG;
    *out = nullptr;
    if (!instances || count < 1) return DMPM_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return DMPM_ERR_CUDA;
    }
    dmpm_batch* b = new dmpm_batch();
    b->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return DMPM_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        dmpm_batch_destroy(b);
        return DMPM_ERR_CUDA;
    }
    b->impl.reset(new dmpm_batch::Impl(b));
    const int st = bguard(b, [&](dmpm_batch::Impl& im) { im.create(instances, count); return DMPM_OK; });
    if (st != DMPM_OK) {
        dmpm_batch_destroy(b);
        return st;
    }
    *out = b;
    return DMPM_OK;
}

int dmpm_batch_destroy(dmpm_batch* b) {
    if (!b) return DMPM_ERR_ARG;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    if (b->side) cudaStreamSynchronize(b->side);
    b->impl.reset();
    cudaStreamDestroy(b->stream);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    delete b;
    return DMPM_OK;
}

const char* dmpm_batch_last_error(const dmpm_batch* b) { return b ? b->err.c_str() : "null batch"; }

int dmpm_batch_set_params(dmpm_batch* b, const dmpm_params* p) {
    if (!p) return DMPM_ERR_ARG;
    if (!(p->dt >= 0) || p->adjoint_mode < 0 || p->adjoint_mode > 1 || p->loss_kind < 0 || p->loss_kind > 1 ||
        p->sort_every < 0)
        return DMPM_ERR_ARG;
    return bguard(b, [&](dmpm_batch::Impl& im) { im.set_params(*p); return DMPM_OK; });
}

int dmpm_batch_set_particles(dmpm_batch* b, int inst, const double* x, const double* v, const double* F,
                             const double* C, const double* dFc, const double* m, const double* vol,
                             const double* lam, const double* mu) {
    return bguard(b, [&](dmpm_batch::Impl& im) { im.set_particles(inst, x, v, F, C, dFc, m, vol, lam, mu); return DMPM_OK; });
}

int dmpm_batch_set_target_mass(dmpm_batch* b, int inst, const double* target_m) {
    return bguard(b, [&](dmpm_batch::Impl& im) { im.set_target(inst, target_m); return DMPM_OK; });
}

int dmpm_batch_set_launch(dmpm_batch* b, const dmpm_batch_launch* cfg) {
    if (!cfg) return DMPM_ERR_ARG;
    return bguard(b, [&](dmpm_batch::Impl& im) { im.set_launch(*cfg); return DMPM_OK; });
}

int dmpm_batch_get_launch(const dmpm_batch* b, dmpm_batch_launch* cfg) {
    if (!b || !cfg) return DMPM_ERR_ARG;
    const dmpm_batch::Impl& im = *b->impl;
    *cfg = im.cfg;
    cfg->sort_every = im.sort_every();
    cfg->ctas_per_sm = im.ctas_per_sm();
    cfg->particle_block = im.particle_block();
    return DMPM_OK;
}

int dmpm_batch_setup(dmpm_batch* b) {
    return bguard(b, [&](dmpm_batch::Impl& im) { im.setup(); return DMPM_OK; });
}

int dmpm_batch_gradient(dmpm_batch* b, double* losses) {
    return bguard(b, [&](dmpm_batch::Impl& im) { return im.gradient(losses); });
}

int dmpm_batch_autotune(dmpm_batch* b, int reps, double* best_ms) {
    return bguard(b, [&](dmpm_batch::Impl& im) {
        const double ms = im.autotune(reps);
        if (best_ms) *best_ms = ms;
        return DMPM_OK;
    });
}

int dmpm_batch_get_control_grad(dmpm_batch* b, int inst, double* out) {
    return bguard(b, [&](dmpm_batch::Impl& im) { im.control_grad(inst, out); return DMPM_OK; });
}

int dmpm_batch_get_particles(dmpm_batch* b, int inst, int layer, int field, double* out) {
    return bguard(b, [&](dmpm_batch::Impl& im) { im.get_particles(inst, layer, field, out); return DMPM_OK; });
}

int dmpm_batch_info(const dmpm_batch* b, int64_t* info, int count) {
    if (!b || !info || count < 0) return DMPM_ERR_ARG;
    b->impl->info(info, count);
    return DMPM_OK;
}

int dmpm_batch_stream(const dmpm_batch* b, void** stream) {
    if (!b || !stream) return DMPM_ERR_ARG;
    *stream = (void*)b->stream;
    return DMPM_OK;
}

}  // extern "C"
