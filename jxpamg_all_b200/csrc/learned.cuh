// Learned AMG settings: a 16 -> 64 -> 3 MLP (tanh hidden layer, FP32) maps
// cheap statistics of a level operator to that level's strength threshold and
// the interval of its degree-3 Chebyshev smoother.  Inference runs inside the
// setup (one forward pass per level, before the level is coarsened); training
// uses the batch kernels of learned.cu through the C ABI.
#pragma once

#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

constexpr int kMlpIn = 16, kMlpHidden = 64, kMlpOut = 3;
// weight blob (floats): mu[16], sigma[16], W1[64][16], b1[64], W2[3][64], b2[3]
constexpr int kMlpOffMu = 0, kMlpOffSigma = 16, kMlpOffW1 = 32, kMlpOffB1 = kMlpOffW1 + kMlpHidden * kMlpIn,
              kMlpOffW2 = kMlpOffB1 + kMlpHidden, kMlpOffB2 = kMlpOffW2 + kMlpOut * kMlpHidden,
              kMlpWeights = kMlpOffB2 + kMlpOut;

// Output maps (logit y -> setting).
inline double mlp_theta(double y) { return 0.1 + 0.8 / (1.0 + exp(-y)); }
inline double mlp_lower(double y) { return 0.02 + 0.68 / (1.0 + exp(-y)); }
inline double mlp_upper(double y) { return 0.8 + 0.7 / (1.0 + exp(-y)); }

struct LearnedPlan {
    bool active = false;
    bool record = false;     // record features only (no prediction)
    std::vector<double> theta, lower, upper;
    std::vector<double> lambda12;  // lambda_max(D^-1 A) after 12 power steps, per level (the Chebyshev estimate)
    std::vector<std::vector<float>> features;
    int prev_n = 0;
};

// Features of level `level` (kMlpIn floats; prev_n = rows of the previous level, 0 at level 0).
void level_features(const CsrView<double> &A, int level, int prev_n, float *out, cudaStream_t s,
                    double *lambda12 = nullptr);
// Called by the AMG setup before coarsening `level`: records the level's
// features, runs the MLP (when plan.active) and returns the strength threshold.
double learned_predict_level(LearnedPlan &plan, int level, const CsrView<double> &A, double default_theta,
                             cudaStream_t s);
// Current weights (process-wide; defaults compiled in, replaced through the C ABI).
const std::vector<float> &mlp_weights();
void mlp_set_weights(const float *w);
// Host forward pass of one sample (the same arithmetic as the device kernel).
void mlp_forward_host(const float *w, const float *x, float *y);

}  // namespace jxcpr
