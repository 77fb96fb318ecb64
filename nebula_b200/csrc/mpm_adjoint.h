// mpm_adjoint.h -- nebula::AdjointEngine: a differentiable MLS-MPM rollout
// (no counterpart in the reference, which has no adjoint).
//
// Setting: APIC transfer, ELASTIC (Hencky) material with a per-particle
// Young's modulus, uniform rho0 and nu, gravity, the grid wall band; no
// colliders or SDF.  The forward substep is the engine's own (same device
// functions: p2gParticle, gridNode, g2pParticle) on a dense Morton grid in
// particle order.  Loss: |COM(x_T) - target|^2 with COM mass-weighted.
// Backward: reverse-mode adjoint of G2P, grid update and P2G, checkpoints
// every `checkpointEvery` substeps, each segment recomputed with its states
// and grids kept.  The adjoint runs in float32 except the SVD and the
// Hencky-stress derivative, which run in float64.
#pragma once
#include <vector>

#include "mpm_engine.h"

namespace nebula {

// Per-call scalars the graph kernels read from device memory.
struct AdjScalars {
  double com[4];     // sum m x, sum m (accumulated by the forward)
  double target[3];
  float loss;
  float lossGrad;
  uint32_t events;   // 1 J reset, 2 world clamp, 4 speed cap
  uint32_t pad;
};

class AdjointEngine {
 public:
  explicit AdjointEngine(const nebula_mpm_adjoint_config& cfg);
  ~AdjointEngine();
  void forward(const float* dPos4, const float* dVel4, const float* dE, const float target[3], float* dLoss, cudaStream_t s);
  void backward(float lossGrad, float* dGradVel4, float* dGradE, float* dGradPos4, cudaStream_t s);
  void download(int field, float* host, uint64_t count);
  uint32_t events();
  void setGraphs(bool on);
  uint64_t launches() const { return launches_; }

 private:
  void bindDevice() const;
  void forwardBody(cudaStream_t s);
  void backwardBody(cudaStream_t s);
  void substepForward(const float4* const* in, float4* const* out, float4* acc, float4* vel, uint32_t k, bool clear, cudaStream_t s);
  void run(bool fwd, cudaStream_t s);

  nebula_mpm_adjoint_config cfg_;
  int device_ = 0;
  uint32_t n_ = 0, nc_ = 0, segs_ = 0, every_ = 1;
  int finalBuf_ = 0;
  SubstepParams P_{};
  DevBuf forces_, lame_, scal_;
  DevBuf x0_, v0_, E_;             // inputs (engine copies)
  DevBuf gradV_, gradE_, gradX_;   // outputs (engine copies)
  DevBuf ping_[2];                 // forward state: 8 float4 arrays of n
  std::vector<DevBuf> ck_;         // checkpoints: state at substep seg * every
  std::vector<DevBuf> segState_;   // states of the segment being reversed (slots 1..every-1)
  std::vector<DevBuf> segAcc_, segVel_;  // grids of the segment's substeps
  DevBuf acc_, vel_;               // forward grid scratch
  DevBuf adj_[2];                  // adjoint state: x, v ([n] float4), B, F, T ([3n] float4 rows each)
  DevBuf gadj_[2];                 // grid adjoint [nc] float4, alternating by substep
  DevBuf boxes_;                   // per substep: the P2G's node box (NodeBox, mpm_adjoint.cu)
  uint32_t gridBlocks_ = 1;        // CTAs of the grid passes (grid-stride over a node box)
  DevBuf mub_, lamb_;              // per-particle accumulated adjoints of mu, lambda
  bool haveForward_ = false;
  bool useGraphs_ = true;
  cudaGraphExec_t graph_[2] = {nullptr, nullptr};  // [forward, backward]
  uint64_t graphLaunches_[2] = {0, 0};
  uint64_t launches_ = 0;
};

}  // namespace nebula
