// CompGraph.h -- the reference's computation graph (CompGraph.h:10-66) over the
// B200 engine.  Same public members and call sequence: the constructor deep
// copies the initial cloud and grid into layers[0], SetUpCompGraph copies
// layer 0 into every layer, ComputeForwardPass / EndLayerMassLoss /
// ComputeBackwardPass run the engine (include/dmpm.h) and leave the host
// layers holding what the reference's would hold (states after the forward
// pass, the last layer's dLdx after the loss, every layer's adjoint after the
// backward pass).
//
// The reference sets dt / drag / f_ext / smoothing_factor only inside
// OptimizeDefGradControlSequence; SetSimulationParameters sets them directly.
// SetEngineOptions selects the engine path (DMPM_FP32_MIXED by default, or
// DMPM_FP64) and the adjoint (DMPM_ADJ_REFCOMPAT by default, or DMPM_ADJ_EXACT).
#pragma once
#include <memory>
#include <vector>
#include "Grid.h"
#include "PointCloud.h"

struct dmpm_ctx;

namespace DiffMPMLib3D {

struct CompGraphLayer {
    std::shared_ptr<PointCloud> point_cloud = nullptr;
    std::shared_ptr<Grid> grid = nullptr;
};

class CompGraph {
   public:
    CompGraph(std::shared_ptr<PointCloud> initial_point_cloud, std::shared_ptr<Grid> grid,
              std::shared_ptr<const Grid> _target_grid);
    ~CompGraph();
    CompGraph(const CompGraph&) = delete;
    CompGraph& operator=(const CompGraph&) = delete;

    void OptimizeDefGradControlSequence(int num_steps, float _dt, float _drag, Vec3 _f_ext, int control_stride,
                                        int max_gd_iters, int max_line_search_iters, float initial_alpha,
                                        float gd_tol, float smoothing_factor);

    void SetUpCompGraph(int num_layers);
    float EndLayerMassLoss();
    void ComputeForwardPass(size_t start_layer);
    void ComputeBackwardPass(size_t control_layer);
    void FiniteDifferencesGradientTest(int num_steps, size_t particle_id);

    std::vector<CompGraphLayer> layers;
    std::shared_ptr<const Grid> target_grid;

    // engine controls (not in the reference)
    void SetSimulationParameters(float dt, float drag, Vec3 f_ext, float smoothing_factor);
    void SetEngineOptions(int precision, int adjoint_mode, int device = 0);
    // FP32-mixed path: integer node sums, so passes repeat bit for bit (dmpm_params::deterministic)
    void SetDeterministic(bool on);
    // FP32-mixed path: store the cloud in cell order on the device (dmpm_params::reorder_particles);
    // every layer's points keep their order here
    void SetReorderParticles(bool on);
    bool sync_grids = true;  // copy every layer's grid and stress P back after each pass

   private:
    void EnsureEngine();
    void PushLayer0AndControls(size_t start_layer);
    void PullStates(size_t first, size_t last);
    void PullGrid(size_t layer);
    void PullAdjoints(size_t first, size_t last);

    Vec3 f_ext = Vec3::Zero();
    float dt = 1.0f / 120.0f;
    float drag = 0.5f;
    float smoothing_factor = 0.1f;
    float alpha_decay = 0.96f;
    float min_alpha = 1e-3f;
    std::vector<float> gradientNormHistory;
    int timestep = 1;

    int precision_ = 1;  // DMPM_FP32_MIXED
    int adjoint_mode_ = 0;
    int device_ = 0;
    bool deterministic_ = false;
    bool reorder_ = false;
    dmpm_ctx* ctx_ = nullptr;
    int ctx_layers_ = 0;
};

}  // namespace DiffMPMLib3D
