// Internal interface of the BF16 MLP surrogate (mlp.cu), used by the surrogate-refined
// map pipeline (ucb_surrogate.cpp). Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/ucb.h"

namespace ucb {

// Rows of a network input. Row r is the point
//   (u[2r], u[2r+1])                                     when u != nullptr, else
//   (cx / (grid_n - 1), cy / (grid_n - 1))               with cell = cells ? cells[r] : r,
//                                                        cx = cell % grid_n, cy = cell / grid_n,
// i.e. kernel-order cells of a square grid mapped to [0, 1]^2.
struct MlpInputs {
    const float* u = nullptr;
    const long long* cells = nullptr;
    long long n = 0;
    int grid_n = 0;
};

struct Mlp;

Mlp* mlp_create(ucb_engine* e, const ucb_mlp_config& cfg, std::string& err);
void mlp_destroy(Mlp* m);
// Re-initialises parameters and the frequency matrix from the configuration's seed
// (buffers are kept).
bool mlp_reinit(Mlp* m, std::string& err);
const ucb_mlp_config& mlp_config(const Mlp* m);
long long mlp_param_count(const Mlp* m);
int mlp_features(const Mlp* m);

// Trains on (inputs, d_y) with Adam for cfg.train_steps mini-batches (one captured CUDA
// graph replayed per step). d_y: n targets (device). Targets are standardised with their
// mean / std, which predictions undo. loss_out: mean loss of the last step.
bool mlp_fit(Mlp* m, const MlpInputs& in, const float* d_y, cudaStream_t st, float* loss_out, std::string& err);

// Mean and standard deviation of the prediction for every input row (device arrays of n).
bool mlp_predict(Mlp* m, const MlpInputs& in, float* d_mean, float* d_std, cudaStream_t st, std::string& err);

}  // namespace ucb
