// Learned AMG settings: level features, the MLP (inference in the setup,
// batch forward / backward / Adam kernels for training) and its C ABI.
//
// The network and its training are this library's own addition; the
// reference has no learned component.  Features are reductions over the level
// operator in one pass (plus a short power iteration for lambda_max of D^-1 A).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "fast.cuh"
#include "jxcpr_b200.h"
#include "learned.cuh"

namespace jxcpr {

namespace {
#include "learned_weights.inc"  // kDefaultMlpWeights[kMlpWeights] (written by the trainer)

constexpr int kFeatStats = 16;
constexpr int kFeatThreads = 256;

std::mutex g_w_mu;
std::vector<float> &weights_store() {
    static std::vector<float> w(kDefaultMlpWeights, kDefaultMlpWeights + kMlpWeights);
    return w;
}

// Per-row statistics, grid-stride, one partial vector (kFeatStats doubles) per CTA:
// 0 sum nnz, 1 max nnz, 2 sum offsum/|d|, 3 max offsum/|d|, 4 sum rowsum/d, 5 #positive off-diagonals,
// 6 #off-diagonals, 7 sum offmax/offsum, 8..10 #off-diagonals >= {.25,.5,.75} * offmax,
// 11 sum log10|d|, 12 sum log10|d|^2, 13 #rows with a nonzero diagonal, 14 #rows with rowsum/d > 1e-3
__global__ void __launch_bounds__(kFeatThreads) feat_rows_kernel(int n, const int *__restrict__ ia,
                                                                 const int *__restrict__ ja,
                                                                 const double *__restrict__ a,
                                                                 double *__restrict__ partials) {
    double acc[kFeatStats];
#pragma unroll
    for (int k = 0; k < kFeatStats; ++k) acc[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int d = ia[i], e = ia[i + 1];
        const double diag = (d < e && ja[d] == i) ? a[d] : 0.0;
        double offsum = 0.0, offmax = 0.0, rowsum = 0.0;
        int npos = 0, noff = 0;
        for (int k = d; k < e; ++k) {
            const double v = a[k];
            rowsum += v;
            if (ja[k] == i) continue;
            const double av = fabs(v);
            offsum += av;
            offmax = fmax(offmax, av);
            npos += v > 0.0;
            ++noff;
        }
        int s25 = 0, s50 = 0, s75 = 0;
        for (int k = d; k < e; ++k) {
            if (ja[k] == i) continue;
            const double av = fabs(a[k]);
            s25 += av >= 0.25 * offmax;
            s50 += av >= 0.5 * offmax;
            s75 += av >= 0.75 * offmax;
        }
        const double ad = fabs(diag);
        acc[0] += e - d;
        acc[1] = fmax(acc[1], (double)(e - d));
        if (ad > 0.0) {
            const double dom = fmin(offsum / ad, 1e3);
            acc[2] += dom;
            acc[3] = fmax(acc[3], dom);
            acc[4] += rowsum / diag;
            const double l = log10(ad);
            acc[11] += l;
            acc[12] += l * l;
            acc[13] += 1.0;
            acc[14] += rowsum / diag > 1e-3;
        }
        acc[5] += npos;
        acc[6] += noff;
        if (offsum > 0.0) acc[7] += offmax / offsum;
        acc[8] += s25;
        acc[9] += s50;
        acc[10] += s75;
    }
    __shared__ double sh[kFeatThreads / 32][kFeatStats];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kFeatStats; ++k) {
        double v = acc[k];
        const bool is_max = (k == 1 || k == 3);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(0xffffffffu, v, o);
            v = is_max ? fmax(v, w) : v + w;
        }
        if (lane == 0) sh[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < kFeatStats) {
        const int k = threadIdx.x;
        const bool is_max = (k == 1 || k == 3);
        double v = sh[0][k];
        for (int w = 1; w < kFeatThreads / 32; ++w) v = is_max ? fmax(v, sh[w][k]) : v + sh[w][k];
        partials[blockIdx.x * kFeatStats + k] = v;
    }
}

// ---- training kernels -------------------------------------------------------
// X [B][16], H [B][64], Y [B][3], T [B][3]
__global__ void __launch_bounds__(kMlpHidden) mlp_forward_kernel(const float *__restrict__ w,
                                                                 const float *__restrict__ X, int B,
                                                                 float *__restrict__ H, float *__restrict__ Y) {
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= B) return;
    __shared__ float xn[kMlpIn], hs[kMlpHidden];
    if (j < kMlpIn) xn[j] = (X[b * kMlpIn + j] - w[kMlpOffMu + j]) / w[kMlpOffSigma + j];
    __syncthreads();
    float z = w[kMlpOffB1 + j];
    for (int k = 0; k < kMlpIn; ++k) z += w[kMlpOffW1 + j * kMlpIn + k] * xn[k];
    const float h = tanhf(z);
    hs[j] = h;
    if (H) H[b * kMlpHidden + j] = h;
    __syncthreads();
    if (j < kMlpOut) {
        float y = w[kMlpOffB2 + j];
        for (int m = 0; m < kMlpHidden; ++m) y += w[kMlpOffW2 + j * kMlpHidden + m] * hs[m];
        Y[b * kMlpOut + j] = y;
    }
}

// Per sample: dY = 2 (Y - T) / (3 B) (mean squared error over outputs and batch),
// dZ_j = (sum_o dY_o W2[o][j]) (1 - h_j^2).
__global__ void __launch_bounds__(kMlpHidden) mlp_backward_kernel(const float *__restrict__ w,
                                                                  const float *__restrict__ H,
                                                                  const float *__restrict__ Y,
                                                                  const float *__restrict__ T, int B,
                                                                  float *__restrict__ dZ, float *__restrict__ dY) {
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= B) return;
    __shared__ float dy[kMlpOut];
    if (j < kMlpOut) {
        const float g = 2.0f * (Y[b * kMlpOut + j] - T[b * kMlpOut + j]) / (float)(kMlpOut * B);
        dy[j] = g;
        dY[b * kMlpOut + j] = g;
    }
    __syncthreads();
    float s = 0.0f;
    for (int o = 0; o < kMlpOut; ++o) s += dy[o] * w[kMlpOffW2 + o * kMlpHidden + j];
    const float h = H[b * kMlpHidden + j];
    dZ[b * kMlpHidden + j] = s * (1.0f - h * h);
}

// One thread per weight: the gradient summed over the batch in sample order.
__global__ void mlp_weight_grad_kernel(const float *__restrict__ w, const float *__restrict__ X,
                                       const float *__restrict__ H, const float *__restrict__ dZ,
                                       const float *__restrict__ dY, int B, float *__restrict__ grad) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= kMlpWeights) return;
    float g = 0.0f;
    if (idx >= kMlpOffW1 && idx < kMlpOffB1) {
        const int j = (idx - kMlpOffW1) / kMlpIn, k = (idx - kMlpOffW1) % kMlpIn;
        const float mu = w[kMlpOffMu + k], sg = w[kMlpOffSigma + k];
        for (int b = 0; b < B; ++b) g += dZ[b * kMlpHidden + j] * ((X[b * kMlpIn + k] - mu) / sg);
    } else if (idx >= kMlpOffB1 && idx < kMlpOffW2) {
        const int j = idx - kMlpOffB1;
        for (int b = 0; b < B; ++b) g += dZ[b * kMlpHidden + j];
    } else if (idx >= kMlpOffW2 && idx < kMlpOffB2) {
        const int o = (idx - kMlpOffW2) / kMlpHidden, m = (idx - kMlpOffW2) % kMlpHidden;
        for (int b = 0; b < B; ++b) g += dY[b * kMlpOut + o] * H[b * kMlpHidden + m];
    } else if (idx >= kMlpOffB2) {
        const int o = idx - kMlpOffB2;
        for (int b = 0; b < B; ++b) g += dY[b * kMlpOut + o];
    }
    grad[idx] = g;  // the normalisation (mu, sigma) is fixed: zero gradient
}

__global__ void mlp_loss_kernel(const float *__restrict__ Y, const float *__restrict__ T, int B,
                                float *__restrict__ loss) {
    __shared__ float sh[256];
    float s = 0.0f;
    for (int i = threadIdx.x; i < B * kMlpOut; i += blockDim.x) {
        const float d = Y[i] - T[i];
        s += d * d;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = sh[0] / (float)(kMlpOut * B);
}

__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpWeights || i < kMlpOffW1) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}
}  // namespace

const std::vector<float> &mlp_weights() { return weights_store(); }

void mlp_set_weights(const float *w) {
    std::lock_guard<std::mutex> lk(g_w_mu);
    weights_store().assign(w, w + kMlpWeights);
}

void mlp_forward_host(const float *w, const float *x, float *y) {
    float xn[kMlpIn], hs[kMlpHidden];
    for (int k = 0; k < kMlpIn; ++k) xn[k] = (x[k] - w[kMlpOffMu + k]) / w[kMlpOffSigma + k];
    for (int j = 0; j < kMlpHidden; ++j) {
        float z = w[kMlpOffB1 + j];
        for (int k = 0; k < kMlpIn; ++k) z += w[kMlpOffW1 + j * kMlpIn + k] * xn[k];
        hs[j] = tanhf(z);
    }
    for (int o = 0; o < kMlpOut; ++o) {
        float v = w[kMlpOffB2 + o];
        for (int m = 0; m < kMlpHidden; ++m) v += w[kMlpOffW2 + o * kMlpHidden + m] * hs[m];
        y[o] = v;
    }
}

void level_features(const CsrView<double> &A, int level, int prev_n, float *out, cudaStream_t s,
                    double *lambda12) {
    const int n = A.nrows;
    for (int k = 0; k < kMlpIn; ++k) out[k] = 0.0f;
    if (n == 0) return;
    const int grid = std::max(1, std::min(div_up(n, kFeatThreads), 4 * sm_count()));
    DevBuf<double> part((size_t)grid * kFeatStats);
    feat_rows_kernel<<<grid, kFeatThreads, 0, s>>>(n, A.ia, A.ja, A.a, part.get());
    JX_LAUNCH_CHECK();
    std::vector<double> h((size_t)grid * kFeatStats);
    part.download(h.data(), h.size(), s);
    JX_CUDA(cudaStreamSynchronize(s));
    double t[kFeatStats] = {0};
    for (int b = 0; b < grid; ++b)
        for (int k = 0; k < kFeatStats; ++k) {
            const double v = h[(size_t)b * kFeatStats + k];
            t[k] = (k == 1 || k == 3) ? std::max(t[k], v) : t[k] + v;
        }
    // 8 power steps for the feature; on to 12 for the Chebyshev estimate of the fast path
    const double lam = estimate_lambda_max(A, 8, s, lambda12 ? 12 : 0, lambda12);
    const double nd = (double)n, noff = std::max(t[6], 1.0), ndiag = std::max(t[13], 1.0);
    const double mean_nnz = t[0] / nd;
    const double lmean = t[11] / ndiag, lvar = std::max(0.0, t[12] / ndiag - lmean * lmean);
    out[0] = (float)(level / 10.0);
    out[1] = (float)(log10(nd) / 7.0);
    out[2] = (float)(mean_nnz / 32.0);
    out[3] = (float)(t[1] / (4.0 * std::max(mean_nnz, 1.0)));
    out[4] = (float)(t[2] / ndiag);
    out[5] = (float)(std::min(t[3], 10.0) / 10.0);
    out[6] = (float)(t[4] / ndiag);
    out[7] = (float)(t[5] / noff);
    out[8] = (float)(t[7] / nd);
    out[9] = (float)(t[8] / noff);
    out[10] = (float)(t[9] / noff);
    out[11] = (float)(t[10] / noff);
    out[12] = (float)(lam / 2.0);
    out[13] = (float)(sqrt(lvar) / 3.0);
    out[14] = (float)(prev_n > 0 ? nd / prev_n : 1.0);
    out[15] = (float)(t[14] / nd);
}

double learned_predict_level(LearnedPlan &plan, int level, const CsrView<double> &A, double default_theta,
                             cudaStream_t s) {
    std::vector<float> f(kMlpIn);
    double lam12 = 0.0;
    level_features(A, level, plan.prev_n, f.data(), s, &lam12);
    plan.prev_n = A.nrows;
    if ((int)plan.lambda12.size() <= level) plan.lambda12.resize(level + 1, 0.0);
    plan.lambda12[level] = lam12;
    if ((int)plan.features.size() <= level) plan.features.resize(level + 1);
    plan.features[level] = f;
    if (!plan.active) return default_theta;
    std::vector<float> w;
    {
        std::lock_guard<std::mutex> lk(g_w_mu);
        w = weights_store();
    }
    float y[kMlpOut];
    mlp_forward_host(w.data(), f.data(), y);
    // The network is trained on a grid of settings; predictions are snapped to
    // the nearest trained value so that no untrained combination is used.
    const double th_raw = mlp_theta(y[0]), lo_raw = mlp_lower(y[1]), hi_raw = mlp_upper(y[2]);
    static const double kTheta0[] = {0.25, 0.5}, kThetaC[] = {0.25, 0.5, 0.7};
    static const double kLo[] = {0.1, 0.3, 0.5}, kHi[] = {1.2, 1.1, 1.2};
    double th = 0.25, best = 1e30;
    const double *tg = level == 0 ? kTheta0 : kThetaC;
    const int ng = level == 0 ? 2 : 3;
    for (int q = 0; q < ng; ++q)
        if (fabs(tg[q] - th_raw) < best) {
            best = fabs(tg[q] - th_raw);
            th = tg[q];
        }
    double lo = 0.3, hi = 1.1;
    best = 1e30;
    for (int q = 0; q < 3; ++q) {
        const double d = fabs(kLo[q] - lo_raw) / 0.4 + fabs(kHi[q] - hi_raw) / 0.1;
        if (d < best) {
            best = d;
            lo = kLo[q];
            hi = kHi[q];
        }
    }
    if ((int)plan.theta.size() <= level) {
        plan.theta.resize(level + 1, default_theta);
        plan.lower.resize(level + 1, 0.3);
        plan.upper.resize(level + 1, 1.1);
    }
    plan.theta[level] = th;
    plan.lower[level] = lo;
    plan.upper[level] = hi;
    return th;
}

}  // namespace jxcpr

// ---------------------------------------------------------------------------
// C ABI (device pointers for the batch kernels)
// ---------------------------------------------------------------------------
using namespace jxcpr;

extern "C" {

int jxcpr_mlp_num_weights(void) { return kMlpWeights; }

int jxcpr_mlp_set_weights(const float *w_host) {
    if (!w_host) return JXCPR_ERROR_ARG;
    for (int k = 0; k < kMlpIn; ++k)
        if (!(w_host[kMlpOffSigma + k] != 0.0f)) {
            set_error("mlp: sigma[%d] must be nonzero", k);
            return JXCPR_ERROR_ARG;
        }
    mlp_set_weights(w_host);
    return JXCPR_SUCCESS;
}

int jxcpr_mlp_get_weights(float *w_host) {
    if (!w_host) return JXCPR_ERROR_ARG;
    std::lock_guard<std::mutex> lk(g_w_mu);
    memcpy(w_host, weights_store().data(), sizeof(float) * kMlpWeights);
    return JXCPR_SUCCESS;
}

int jxcpr_mlp_forward_host(const float *w_host, const float *x_host, float *y_host) {
    if (!w_host || !x_host || !y_host) return JXCPR_ERROR_ARG;
    mlp_forward_host(w_host, x_host, y_host);
    return JXCPR_SUCCESS;
}

int jxcpr_mlp_forward(const float *w, const float *X, int B, float *H, float *Y, void *stream) {
    if (!w || !X || !Y || B < 0) return JXCPR_ERROR_ARG;
    if (B == 0) return JXCPR_SUCCESS;
    try {
        mlp_forward_kernel<<<B, kMlpHidden, 0, (cudaStream_t)stream>>>(w, X, B, H, Y);
        JX_LAUNCH_CHECK();
        JX_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    } catch (const CudaError &) {
        return JXCPR_ERROR_DEVICE;
    }
    return JXCPR_SUCCESS;
}

int jxcpr_mlp_loss_grad(const float *w, const float *X, const float *T, int B, float *grad, float *loss,
                        float *work, void *stream) {
    if (!w || !X || !T || !grad || !loss || !work || B <= 0) return JXCPR_ERROR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    float *H = work, *dZ = work + (size_t)B * kMlpHidden, *Y = dZ + (size_t)B * kMlpHidden,
          *dY = Y + (size_t)B * kMlpOut;
    try {
        mlp_forward_kernel<<<B, kMlpHidden, 0, s>>>(w, X, B, H, Y);
        JX_LAUNCH_CHECK();
        mlp_backward_kernel<<<B, kMlpHidden, 0, s>>>(w, H, Y, T, B, dZ, dY);
        JX_LAUNCH_CHECK();
        mlp_weight_grad_kernel<<<div_up(kMlpWeights, 128), 128, 0, s>>>(w, X, H, dZ, dY, B, grad);
        JX_LAUNCH_CHECK();
        mlp_loss_kernel<<<1, 256, 0, s>>>(Y, T, B, loss);
        JX_LAUNCH_CHECK();
        JX_CUDA(cudaStreamSynchronize(s));
    } catch (const CudaError &) {
        return JXCPR_ERROR_DEVICE;
    }
    return JXCPR_SUCCESS;
}

int jxcpr_mlp_adam(float *w, const float *grad, float *m, float *v, float lr, float beta1, float beta2, float eps,
                   int step, void *stream) {
    if (!w || !grad || !m || !v || step < 1) return JXCPR_ERROR_ARG;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    try {
        adam_kernel<<<div_up(kMlpWeights, 256), 256, 0, (cudaStream_t)stream>>>(w, grad, m, v, lr, beta1, beta2, eps,
                                                                               c1, c2);
        JX_LAUNCH_CHECK();
    } catch (const CudaError &) {
        return JXCPR_ERROR_DEVICE;
    }
    return JXCPR_SUCCESS;
}

}  // extern "C"
