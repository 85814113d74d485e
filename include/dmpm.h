/*
 * dmpm.h -- C ABI of the B200 MLS-MPM forward + adjoint engine (libdmpm.so).
 *
 * This ABI replaces, for one caller thread, the hot-path entry points of the
 * reference library DiffMPMLib3D (paths relative to that project):
 *
 *   dmpm_set_particles / dmpm_set_points_ref
 *                          <- CompGraph::CompGraph(initial_point_cloud, grid, target)
 *                             deep copy of the initial PointCloud          (CompGraph.h:20, CompGraph.cpp:269-278)
 *   dmpm_set_grid          <- Grid::Grid(dim_x, dim_y, dim_z, dx, min_point) (Grid.h:11, Grid.cpp:3-28)
 *   dmpm_set_target_mass / dmpm_rasterize_target
 *                          <- CompGraph::target_grid, built by LoadCompGraph as a
 *                             mass-only P2G of target samples             (CompGraph.h:52, MPMPolyscope.cpp:155-160)
 *   dmpm_compute_volumes   <- SingleThreadMPM::CalculatePointCloudVolumes   (ForwardSimulation.h:39, .cpp:262-290)
 *   dmpm_set_params        <- the dt / drag / f_ext / smoothing_factor members that
 *                             OptimizeDefGradControlSequence sets          (CompGraph.h:54-58, CompGraph.cpp:296-300)
 *   dmpm_setup             <- CompGraph::SetUpCompGraph(num_layers)         (CompGraph.h:40, CompGraph.cpp:7-17)
 *   dmpm_forward           <- CompGraph::ComputeForwardPass(start_layer), i.e. one
 *                             SingleThreadMPM::ForwardTimeStep per layer   (CompGraph.h:44, CompGraph.cpp:246-256,
 *                                                                           ForwardSimulation.h:17-18, .cpp:126-157)
 *   dmpm_loss              <- CompGraph::EndLayerMassLoss()                 (CompGraph.h:42, CompGraph.cpp:110-244)
 *   dmpm_backward          <- CompGraph::ComputeBackwardPass(control_layer), i.e. one
 *                             Back_Timestep per layer                       (CompGraph.h:45, CompGraph.cpp:258-267,
 *                                                                           BackPropagation.h:7, .cpp:6-125)
 *   dmpm_get_particles / dmpm_get_points_ref / dmpm_set_layer_particles
 *                          <- reads and writes of CompGraph::layers[i].point_cloud->points
 *                                                                           (CompGraph.h:50, MaterialPoint.h:8-75)
 *   dmpm_get_grid          <- reads of CompGraph::layers[i].grid->nodes     (GridNode.h:5-24)
 *   dmpm_get_control_grad  <- MaterialPoint::dLdF of layer i, the gradient the
 *                             reference optimisers descend                  (PointCloud.cpp:83-99)
 *   dmpm_dldf_norm         <- PointCloud::Compute_dLdF_Norm                 (PointCloud.cpp:24-35)
 *
 * Conventions
 *   - All functions return a status (DMPM_OK = 0); dmpm_last_error() gives the
 *     message of the last failure on a context.
 *   - Host arrays are double, one particle after another: vectors as 3 values,
 *     3x3 matrices as 9 values in column-major order (Eigen::Matrix3f storage,
 *     element (i, j) at [9p + i + 3j]).  Grid arrays use the reference's node
 *     order (i * dim_y + j) * dim_z + k, vectors as 3 values per node.
 *   - Host buffers may be pageable or pinned; pinned buffers make copies
 *     asynchronous with respect to the host thread.
 *   - A context owns one CUDA stream and its device memory.  It is not
 *     thread-safe (the reference's CompGraph is not either).
 *   - Units: the reference is only physically consistent with dx = 1 (its
 *     particle volume is m / sum w m_g); callers use lattice units.
 */
#ifndef DMPM_H
#define DMPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dmpm_ctx dmpm_ctx;

/* status codes */
#define DMPM_OK 0
#define DMPM_ERR_ARG 1       /* invalid argument or size */
#define DMPM_ERR_OOM 2       /* device or pinned allocation failed */
#define DMPM_ERR_CUDA 3      /* a CUDA runtime call failed */
#define DMPM_ERR_NONFINITE 4 /* a stage produced NaN/inf (results still written, as the reference does) */
#define DMPM_ERR_STATE 5     /* call order: e.g. backward before loss, or a layer that is not stored */
#define DMPM_ERR_TOO_LARGE 6 /* a size exceeds a fixed capacity: dmpm_compute_volumes_noalloc's scratch, an output buffer */

/* precision paths */
#define DMPM_FP64 0       /* plain FP64 path: one kernel per reference stage, global atomics */
#define DMPM_FP32_MIXED 1 /* FP32 state and grid, cell-sorted warp items; FP64 polar/SVD, stress
                             derivative, loss and control-gradient sums */

/* adjoint modes */
#define DMPM_ADJ_REFCOMPAT 0 /* reproduces Back_Timestep term by term */
#define DMPM_ADJ_EXACT 1     /* true derivative of the forward map */

/* control (dFc) modes */
#define DMPM_CTRL_PER_LAYER 0 /* one dFc per layer, as CompGraph::layers[i] */
#define DMPM_CTRL_TIED 1      /* one dFc shared by every layer; gradient = sum over layers */

/* loss kinds */
#define DMPM_LOSS_REF_LOGMASS 0 /* EndLayerMassLoss: log-mass L2 + min-mass penalty */
#define DMPM_LOSS_L2 1          /* 1/2 sum (m - t)^2 */

/* particle fields (dmpm_get_particles / dmpm_set_layer_particles) */
#define DMPM_F_X 0
#define DMPM_F_V 1
#define DMPM_F_F 2
#define DMPM_F_C 3
#define DMPM_F_P 4
#define DMPM_F_M 5
#define DMPM_F_VOL 6
#define DMPM_F_LAM 7
#define DMPM_F_MU 8
#define DMPM_F_DFC 9
#define DMPM_F_DLDX 10
#define DMPM_F_DLDV 11
#define DMPM_F_DLDF 12
#define DMPM_F_DLDC 13
#define DMPM_F_DLDP 14
#define DMPM_F_DLDV_NEXT 15
#define DMPM_F_DLDC_NEXT 16
#define DMPM_F_DLDFE 19 /* dL/d dFc of the layer (EXACT: differs from dLdF when smoothing != 0) */

/* grid fields (dmpm_get_grid).  On the FP32-mixed path the grid update
 * overwrites each node's momentum with its velocity in place: DMPM_G_V is then
 * read as stored and DMPM_G_P is recovered as (v - dt f_ext) m on nodes with
 * |m| > FLT_EPSILON (0 on the others); the FP64 path keeps both exactly. */
#define DMPM_G_M 0
#define DMPM_G_V 1
#define DMPM_G_P 2
#define DMPM_G_DLDV 3
#define DMPM_G_DLDP 4
#define DMPM_G_DLDM 5

typedef struct {
    double dt;               /* CompGraph::dt */
    double drag;             /* CompGraph::drag */
    double f_ext[3];         /* CompGraph::f_ext */
    double smoothing;        /* CompGraph::smoothing_factor */
    int adjoint_mode;        /* DMPM_ADJ_* */
    int control_mode;        /* DMPM_CTRL_* */
    int loss_kind;           /* DMPM_LOSS_* */
    int checkpoint_every;    /* 0: keep every layer if it fits in HBM, else checkpoint;
                                1: keep every layer; k > 1: keep layers 0, k, 2k, ... and the
                                last, recompute the others during backward */
    int keep_adjoints;       /* keep every layer's adjoint state readable after backward */
    int keep_intermediates;  /* keep P, dLdP, dLdv_next, dLdC_next and grid adjoints per layer */
    int block_size;          /* threads per CTA for particle kernels; 0 = default (256) */
    int tile_cap;            /* max nodes of a shared-memory tile; 0 = default */
    int sort_every;          /* FP32 path: re-sort particles by cell every this many steps; 0 = default (8) */
    int warp_general;        /* FP32 path: 1 disables the same-cell warp reduction (verification) */
    int control_stride;      /* DMPM_CTRL_PER_LAYER: layers 0, s, 2s, ... below the last own their
                                controls and gradients (OptInput::control_stride, the control frames
                                of CompGraph::OptimizeDefGradControlSequence, CompGraph.cpp:352);
                                the other layers read the uploaded dFc, as the reference's copies made
                                by SetUpCompGraph stay unchanged there.  0 or 1 = every layer. */
    int eager;               /* FP32 path with every layer kept: 0 = capture dmpm_forward / dmpm_backward
                                once per start (top, control) layer and replay them as CUDA graphs;
                                1 = launch kernel by kernel (per-kernel profiling also does) */
    int brick_cells;         /* FP32 path, G2P: 2 (default) or 4 = a CTA stages the node tile of a brick
                                of brick_cells^3 cells in shared memory and each thread handles one
                                particle of it; 0 = warp items (8 particles of a cell per warp).
                                Takes effect at the next cell sort. */
    int deterministic;       /* FP32 path: 1 = node sums (P2G, the adjoint scatter, the mass rasters) as
                                64-bit integer multiples of a power of two fixed per pass, added with
                                integer atomics, so gradients and losses are bit-identical from run to
                                run; 0 (default) = float atomics, whose summation order varies.  The
                                FP64 reductions (loss, norms) are summed in a fixed order either way. */
    int reorder_particles;   /* FP32 path: 1 = dmpm_setup stores the cloud in the order of its cell keys
                                (the stable cell sort of layer 0), so particles that share stencil
                                nodes sit together in memory whatever order the caller gave them in;
                                every particle array passed through this ABI stays in the caller's
                                order (the engine maps indices), dmpm_cell_sort included.  The order
                                is fixed until the next dmpm_set_particles / dmpm_set_points_ref.
                                0 (default) = the caller's order. */
} dmpm_params;

void dmpm_default_params(dmpm_params* p);

int dmpm_create(int device, int precision, dmpm_ctx** out);
int dmpm_destroy(dmpm_ctx* ctx);
const char* dmpm_last_error(const dmpm_ctx* ctx);
int dmpm_get_info(const dmpm_ctx* ctx, int64_t* info, int count); /* n, dims, layers, precision,
                                                                      checkpoint_every, device bytes, ... */

/* Cap on the device bytes this context may hold (0 = no cap, the default).
 * An allocation that would exceed it fails as a failed cudaMalloc does:
 * the call returns DMPM_ERR_OOM.  No reference counterpart (the reference
 * allocates on the host and never reports running out of memory); it lets a
 * caller bound one context's share of the GPU, and a failed dmpm_setup leaves
 * the context without layer storage -- calls that need it return
 * DMPM_ERR_STATE -- until a dmpm_setup that fits succeeds.  Storage already
 * held is not released by lowering the cap. */
int dmpm_set_device_limit(dmpm_ctx* ctx, int64_t max_bytes);

int dmpm_set_grid(dmpm_ctx* ctx, int dim_x, int dim_y, int dim_z, double dx, const double* min_point);
int dmpm_set_params(dmpm_ctx* ctx, const dmpm_params* params);

/* Initial point cloud (layer 0).  dFc, vol may be NULL (zeros).  The FP32
 * context keeps each position coordinate as a pair of floats (hi + lo, about
 * 48 bits), so x comes back from dmpm_get_particles as given to ~2^-48 of its
 * size; the other fields are stored as floats. */
int dmpm_set_particles(dmpm_ctx* ctx, int n, const double* x, const double* v, const double* F,
                       const double* C, const double* dFc, const double* m, const double* vol,
                       const double* lam, const double* mu);
/* Initial point cloud from an array of the reference's MaterialPoint structs
 * (118 floats = 472 bytes each, field order of MaterialPoint.h:18-46). */
int dmpm_set_points_ref(dmpm_ctx* ctx, const void* points, int n);

int dmpm_compute_volumes(dmpm_ctx* ctx);
int dmpm_set_target_mass(dmpm_ctx* ctx, const double* target_m);
int dmpm_rasterize_target(dmpm_ctx* ctx, int n, const double* x, double point_mass);
int dmpm_get_target_mass(dmpm_ctx* ctx, double* out);

int dmpm_setup(dmpm_ctx* ctx, int num_layers);
int dmpm_forward(dmpm_ctx* ctx, int start_layer);
int dmpm_loss(dmpm_ctx* ctx, double* loss);
int dmpm_backward(dmpm_ctx* ctx, int control_layer);
/* Adjoint steps from layer top_layer down to control_layer, starting from the
 * adjoint state already in top_layer (set with dmpm_set_layer_particles when
 * keep_adjoints is on): Back_Timestep applied top_layer - control_layer times
 * (BackPropagation.h:7, BackPropagation.cpp:6-125). */
int dmpm_backward_range(dmpm_ctx* ctx, int top_layer, int control_layer);

int dmpm_get_particles(dmpm_ctx* ctx, int layer, int field, double* out);
int dmpm_set_layer_particles(dmpm_ctx* ctx, int layer, int field, const double* in);
int dmpm_get_grid(dmpm_ctx* ctx, int layer, int field, double* out);
/* dL/d dFc: per-layer controls -> that layer's gradient; tied controls -> the
 * sum over layers (layer ignored). */
int dmpm_get_control_grad(dmpm_ctx* ctx, int layer, double* out);
int dmpm_dldf_norm(dmpm_ctx* ctx, int layer, double* norm);
/* One Adam step on the controls, on the device: PointCloud::Descend_Adam
 * (PointCloud.cpp:83-99) applied to the control gradient of `layer` (tied
 * controls: the summed gradient; layer ignored).  normalize = 1 divides the
 * gradient by its norm first, as the reference does with Compute_dLdF_Norm.
 * Moment buffers live in the context; t is the 1-based step count. */
int dmpm_adam_step(dmpm_ctx* ctx, int layer, double lr, double beta1, double beta2, double eps, int t,
                   int normalize);
/* One descent step on the controls, on the device, with one of PointCloud's
 * rules (same gradient, normalisation and moment buffers as dmpm_adam_step;
 * the buffers play the roles of MaterialPoint::momentum, vector and vector_max
 * and are shared by the rules, as in the reference):
 *   DMPM_DESCEND_ADAM     Descend_Adam            (PointCloud.cpp:83-99)
 *   DMPM_DESCEND_AMSGRAD  Descend_AMSGrad         (PointCloud.cpp:101-132)
 *   DMPM_DESCEND_LION     Descend_Lion, beta1 as its beta (PointCloud.cpp:134-162)
 *   DMPM_DESCEND_GD       Descend_GradientDescent (PointCloud.cpp:164-178)
 *   DMPM_DESCEND_DLDF     Descend_dLdF: clipped direction, momentum 0.9 (PointCloud.cpp:181-204)
 * beta2, eps and t are used by ADAM and AMSGRAD only. */
#define DMPM_DESCEND_ADAM 0
#define DMPM_DESCEND_AMSGRAD 1
#define DMPM_DESCEND_LION 2
#define DMPM_DESCEND_GD 3
#define DMPM_DESCEND_DLDF 4
int dmpm_descend(dmpm_ctx* ctx, int layer, int rule, double lr, double beta1, double beta2, double eps, int t,
                 int normalize);
/* Fill the state and gradient fields of an array of reference MaterialPoints for one layer. */
int dmpm_get_points_ref(dmpm_ctx* ctx, int layer, void* points);

/* Batched per-matrix functions of Elasticity.h, evaluated in FP64 on the
 * current CUDA device with the hot path's device code.  Host arrays; F, dF and
 * matrix outputs column-major, n matrices; lam, mu per matrix.
 *   DMPM_ELEM_PK            out[9n]  PK_FixedCorotatedElasticity          (Elasticity.cpp:88-98)
 *   DMPM_ELEM_D2_REFCOMPAT  out[9n]  d2_FCE_psi_dF2_mult_by_dF(F, dF)      (Elasticity.cpp:100-178)
 *   DMPM_ELEM_D2_EXACT      out[9n]  the exact dP/dF : dF
 *   DMPM_ELEM_POLAR         out[18n] R then S of JIXIE::polarDecomposition (ImplicitQRSVD.h:863-877)
 *   DMPM_ELEM_ENERGY        out[n]   FixedCorotatedElasticity             (Elasticity.cpp:74-86) */
#define DMPM_ELEM_PK 0
#define DMPM_ELEM_D2_REFCOMPAT 1
#define DMPM_ELEM_D2_EXACT 2
#define DMPM_ELEM_POLAR 3
#define DMPM_ELEM_ENERGY 4
int dmpm_elementary(int kind, int n, const double* F, const double* lam, const double* mu, const double* dF,
                    double* out);

int dmpm_synchronize(dmpm_ctx* ctx);
/* The context's CUDA stream (cudaStream_t) for callers that order their own work after it. */
void* dmpm_stream(dmpm_ctx* ctx);
/* Number of kernels this context has launched since creation. */
int64_t dmpm_launch_count(const dmpm_ctx* ctx);

/* The FP32 path's cell sort, run on a layer's state and returned for
 * verification: keys[n] (sorted cell keys), order[n] (the stable permutation),
 * item_start[n_items + 1] (warp items: runs of <= 8 same-cell particles). */
int dmpm_cell_sort(dmpm_ctx* ctx, int layer, uint32_t* keys, uint32_t* order, uint32_t* item_start, int* n_items);

/* Particle volumes without any device allocation.  No counterpart in the
 * reference.  It computes vol_p = m_p / sum_g w_gp m_g, where m_g = sum_q
 * w_gq m_q are the node masses of a mass-only particle-to-grid transfer and
 * w the cubic B-spline weights (the values dmpm_compute_volumes stores), for
 * callers that cannot call cudaMalloc -- a frame loop that must not take the
 * device-wide synchronisation of cudaMalloc/cudaFree, or a process whose
 * device memory is already held by another framework's caching allocator.
 *   x   device, n * 3 floats (x, y, z per particle, lattice units)
 *   m   device, n floats;  vol: device, n floats (output)
 *   min_point: host, 3 floats;  stream: a cudaStream_t (NULL = default stream)
 * Its only scratch is a grid-mass array compiled into the library (every GPU
 * that loads the library holds it until exit): grids above 1,048,576 nodes
 * (dim_x * dim_y * dim_z) return DMPM_ERR_TOO_LARGE.  The array is shared by
 * all calls on a device and cleared at the start of each call; calls whose GPU
 * work overlaps race on it.  The first call in each CUDA context (the primary
 * context of a device, a caller's own context, or the primary context again
 * after cudaDeviceReset) looks the array's address up in that context; make
 * it before any stream capture.  Asynchronous with respect to the host:
 * results are ready when the stream is. */
int dmpm_compute_volumes_noalloc(int n, const float* x, const float* m, int dim_x, int dim_y, int dim_z, float dx,
                                 const float* min_point, float* vol, void* stream);

/* Per-kernel device time.  With profiling on, every hot-path launch is
 * bracketed by CUDA events on the context's stream (the adjoint finalize's two
 * parts, which otherwise run side by side on two streams, then run one after
 * the other); dmpm_kernel_stats returns the summed milliseconds and the launch
 * count of one kernel since profiling was (re)enabled.  Kernel ids run from 0
 * to DMPM_NUM_KERNEL_IDS - 1; dmpm_kernel_name gives their names (p2g,
 * g2p_p_op2, adj_p2g_gather, adj_finalize, adj_finalize_transport, ...) and
 * NULL for any other id. */
#define DMPM_NUM_KERNEL_IDS 12
int dmpm_set_profiling(dmpm_ctx* ctx, int on);
int dmpm_kernel_stats(dmpm_ctx* ctx, int kernel_id, double* total_ms, int64_t* launches);
const char* dmpm_kernel_name(int kernel_id);

/* ------------------------------------------------------------------------
 * Batched instances.  No reference counterpart: the reference drives one
 * CompGraph per process (CompGraph.h:17-66).  A batch holds many independent
 * scenes (each its own point cloud, grid, target and number of time steps)
 * and advances all of them with one launch per stage per time step; a
 * gradient evaluation (ComputeForwardPass(0), EndLayerMassLoss and
 * ComputeBackwardPass(0) of every instance, CompGraph.cpp:246-267, 110-244)
 * can be captured once and replayed as a CUDA graph.  FP32-mixed arithmetic
 * (the FP32_MIXED path), every layer kept, tied controls (one dFc per
 * particle, gradient summed over the instance's layers).  Instances share
 * dt, drag, f_ext, smoothing, adjoint mode and loss kind (dmpm_params).
 * One batch = one CUDA stream; not thread-safe.
 * ------------------------------------------------------------------------ */
typedef struct dmpm_batch dmpm_batch;
typedef struct {
    int n;                   /* particles */
    int dim_x, dim_y, dim_z; /* grid nodes per axis */
    double dx;
    double min_point[3];
    int steps;               /* time steps of the rollout (layers = steps + 1), >= 1 */
} dmpm_instance;
typedef struct {
    int sort_every;     /* re-sort particles by cell every this many steps; 0 = 8 */
    int ctas_per_sm;    /* persistent grid of the warp-item kernels, CTAs per SM (1..8); 0 = 3 */
    int particle_block; /* threads per block of the per-particle kernels: 128 or 256; 0 = 256 */
    int use_graph;      /* 1 = capture the gradient evaluation once, replay it as a CUDA graph */
} dmpm_batch_launch;
int dmpm_batch_create(int device, int count, const dmpm_instance* instances, dmpm_batch** out);
int dmpm_batch_destroy(dmpm_batch* b);
const char* dmpm_batch_last_error(const dmpm_batch* b);
int dmpm_batch_set_params(dmpm_batch* b, const dmpm_params* params);
/* Instance `inst` (0-based, creation order): host arrays as dmpm_set_particles. */
int dmpm_batch_set_particles(dmpm_batch* b, int inst, const double* x, const double* v, const double* F,
                             const double* C, const double* dFc, const double* m, const double* vol,
                             const double* lam, const double* mu);
int dmpm_batch_set_target_mass(dmpm_batch* b, int inst, const double* target_m);
int dmpm_batch_set_launch(dmpm_batch* b, const dmpm_batch_launch* cfg);
int dmpm_batch_get_launch(const dmpm_batch* b, dmpm_batch_launch* cfg);
/* Allocate every layer of every instance (store-all); fails with DMPM_ERR_OOM
 * when the batch does not fit. */
int dmpm_batch_setup(dmpm_batch* b);
/* One gradient evaluation of every instance; losses: host, count doubles
 * (EndLayerMassLoss of each instance's last layer). */
int dmpm_batch_gradient(dmpm_batch* b, double* losses);
/* Time each launch configuration of a small grid (sort interval, CTAs per SM,
 * particle block) over `reps` gradient evaluations, keep the fastest and
 * report its milliseconds per evaluation. */
int dmpm_batch_autotune(dmpm_batch* b, int reps, double* best_ms);
/* dL/d dFc of instance `inst` (tied: summed over its layers), host n * 9 doubles. */
int dmpm_batch_get_control_grad(dmpm_batch* b, int inst, double* out);
/* DMPM_F_X, _V, _F or _C of instance `inst` at `layer` (0..steps), host doubles. */
int dmpm_batch_get_particles(dmpm_batch* b, int inst, int layer, int field, double* out);
/* info: [0] instances, [1] particles, [2] grid nodes, [3] device bytes,
 * [4] kernel launches of one gradient evaluation, [5] 1 if a graph is captured */
int dmpm_batch_info(const dmpm_batch* b, int64_t* info, int count);
int dmpm_batch_stream(const dmpm_batch* b, void** stream);

/* ------------------------------------------------------------------------
 * Scene setup: point cloud of a watertight, outward-oriented triangle mesh,
 * computed on the current CUDA device.  GeometryLoading::
 * GeneratePointCloudFromWatertightTriangleMesh (GeometryLoading.cpp:10-83),
 * as LoadMPMPointCloudFromObj calls it (MPMPolyscope.cpp:10-60, min_point and
 * max_point the vertices' bounding box): the lattice min_point +
 * sampling_dx (i, j, k), i < ceil((max - min) / sampling_dx) + 1 per axis,
 * i outermost, keeping the points whose winding number is >= 1/2 (the
 * reference's libigl signed distance with winding-number sign is <= 0
 * there).  The reference also keeps a lattice point that lies exactly on a
 * face, which this function leaves out when its winding number is below 1/2.
 *   V: nv * 3 floats;  F: nf * 3 vertex indices (0-based)
 *   out: capacity * 3 floats (NULL with capacity 0 to count only)
 *   *count: the number of points kept; DMPM_ERR_TOO_LARGE when > capacity
 * ------------------------------------------------------------------------ */
int dmpm_mesh_lattice_dims(const float* min_point, const float* max_point, float sampling_dx, int* dims);
int dmpm_mesh_lattice_points(const float* V, int nv, const int* F, int nf, const float* min_point,
                             const float* max_point, float sampling_dx, float* out, int64_t capacity,
                             int64_t* count);
/* Jittered stratified sampling of the same kind of mesh: the box [min_point,
 * max_point] is cut into ceil(extent_a / cell_dx) cells per axis a and each
 * cell into per_axis^3 sub-cells of spacing sdx = cell_dx / per_axis; sub-cell
 * (i, j, k) (linear index q = (i * n1 + j) * n2 + k over the sub-cell grid)
 * gets the point min_point + (index + u) * sdx, u_a = (splitmix64(seed + 3 q + a)
 * >> 40) / 2^24 (SplitMix64's finaliser, Steele et al. 2014; float arithmetic:
 * index + u, times sdx, plus min), and points with winding number >= 1/2 are
 * kept in q order.  Not a reference function: the synthetic scenes'
 * sampling ("jittered stratified, 8 per cell" for per_axis 2) on the GPU. */
int dmpm_mesh_jittered_points(const float* V, int nv, const int* F, int nf, const float* min_point,
                              const float* max_point, float cell_dx, int per_axis, uint64_t seed, float* out,
                              int64_t capacity, int64_t* count);

/* ------------------------------------------------------------------------
 * Single forward stages on caller-held grids and clouds: the reference's
 * stage-level API (SingleThreadMPM::G_op x2, G2P, P_op_2 x2;
 * ForwardSimulation.h:29-35), for callers that compose their own steps.  Host
 * float arrays, 3x3 matrices column-major (9 floats each), grid arrays in node
 * order (i * dim_y + j) * dim_z + k with node (i, j, k) at min_point + (i, j, k) dx.
 * Each call allocates its device scratch and synchronises (dmpm_forward runs
 * the same stages fused, without these copies).
 *   dmpm_stage_g_op    SingleNode_op over the grid (ForwardSimulation.cpp:53-58, 184-224):
 *                      v = p / m + dt f where |m| > FLT_EPSILON, v left unchanged elsewhere;
 *                      f = f_ext, or (gravity_point non-null) gravity_mag times the unit
 *                      vector from the node to gravity_point (0 where every component of that
 *                      vector is within 1e-5, Eigen's isZero()); v in/out
 *   dmpm_stage_g2p     Grid_to_SingleParticle (ForwardSimulation.cpp:60-106):
 *                      v' = sum w v_g,  C' = 3/dx^2 sum w v_g (x_g - x_p)^T
 *   dmpm_stage_p_op_2  SingleParticle_op_2 (ForwardSimulation.cpp:108-124):
 *                      F' = (1 - s)(I + dt C')(F + dFc) + s F,  x' = x + dt v'
 * ------------------------------------------------------------------------ */
int dmpm_stage_g_op(int dim_x, int dim_y, int dim_z, float dx, const float* min_point, const float* m, const float* p,
                    float dt, const float* f_ext, const float* gravity_point, float gravity_mag, float* v);
int dmpm_stage_g2p(int n, const float* x, int dim_x, int dim_y, int dim_z, float dx, const float* min_point,
                   const float* grid_v, float* v_out, float* C_out);
int dmpm_stage_p_op_2(int n, const float* x, const float* F, const float* dFc, const float* v, const float* C,
                      float dt, float smoothing, float* x_out, float* F_out);

/* ------------------------------------------------------------------------
 * Surfaces: headless export of a point cloud as a triangle mesh, the GPU
 * counterpart of the reference's MarchingCubesPointCloud
 * (DiffMPMAnimator3D.cpp:488-514) and SphereUnionMarchingCubesSurfaceFromPointCloud
 * (SphereUnionSurfacing.cpp:7-128).  Host arrays; points are float triples;
 * grid arrays hold prod(dims) floats in node order (i * dim_y + j) * dim_z + k,
 * node (i, j, k) at min_point + (i, j, k) * dx.  Each call allocates its device
 * scratch, runs on the default stream and synchronises.
 *
 *   dmpm_surface_grid_dims    ceil((max_x - min_x) / dx) nodes on every axis, as
 *                             both reference functions size their grids
 *   dmpm_surface_p2g_mass     SingleThreadMPM::P2G_Mass (ForwardSimulation.cpp:292-327):
 *                             node masses sum_p w mp_m (float atomics: equal to the
 *                             reference's point-ordered sums up to rounding)
 *   dmpm_surface_g2g_mass     SingleThreadMPM::G2G_Mass (ForwardSimulation.cpp:329-367):
 *                             grid 2's node masses interpolated from grid 1's with
 *                             grid 1's spacing, bit-identical to the reference
 *   dmpm_surface_sphere_field the field of SphereUnionMarchingCubesSurfaceFromPointCloud
 *                             (lines 13-101): max over points of radius - |x - p| inside
 *                             each sphere, then blur_iterations passes of the 27-node sum
 *                             divided by 9 on interior nodes; bit-identical
 *   dmpm_surface_extract      the level set {field = iso} as a triangle mesh (marching
 *                             tetrahedra, one vertex per crossed grid edge, normals toward
 *                             decreasing field); the reference calls libigl's marching
 *                             cubes here, which triangulates the same level set
 *                             differently.  V: 3 floats per vertex, F: 3 vertex indices
 *                             per triangle; *nv, *nf: the counts, DMPM_ERR_TOO_LARGE when
 *                             they exceed the capacities (call with 0 to size).
 * ------------------------------------------------------------------------ */
int dmpm_surface_grid_dims(const float* min_point, const float* max_point, float dx, int* dims);
int dmpm_surface_p2g_mass(const float* points, int64_t n, float mp_m, const int* dims, float dx,
                          const float* min_point, float* mass);
int dmpm_surface_g2g_mass(const float* mass1, const int* dims1, float dx1, const float* min1, const int* dims2,
                          float dx2, const float* min2, float* mass2);
int dmpm_surface_sphere_field(const float* points, int64_t n, float radius, int blur_iterations, const int* dims,
                              float dx, const float* min_point, float* field);
int dmpm_surface_extract(const float* field, const int* dims, float dx, const float* min_point, float iso, float* V,
                         int64_t v_capacity, int* F, int64_t f_capacity, int64_t* nv, int64_t* nf);

#ifdef __cplusplus
}
#endif
#endif /* DMPM_H */
