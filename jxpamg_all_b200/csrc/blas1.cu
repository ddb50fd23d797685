// BLAS-1 kernels for the Krylov loop (jxf_SeqVectorInnerProd / Axpy / Scale /
// Copy, jxfpamg-0220/csrc/operation/vecops/seq_vecop.c:239-260 and par_vecop.c).
// Dot products are deterministic: fixed grid, per-CTA partial sums, then one
// CTA adds the partials in a fixed order, so a run is reproducible bit for bit.
#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

static constexpr int kRedThreads = 512;

int reduce_partials() { return 2 * sm_count(); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int THREADS>
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double ws[THREADS / 32];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < THREADS / 32 ? ws[threadIdx.x] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

__global__ void __launch_bounds__(kRedThreads) dot_partial_kernel(long long n, const double *__restrict__ x,
                                                                   const double *__restrict__ y,
                                                                   double *__restrict__ partials) {
    double acc = 0.0;
    const long long n2 = n / 2;
    const double2 *x2 = reinterpret_cast<const double2 *>(x);
    const double2 *y2 = reinterpret_cast<const double2 *>(y);
    for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < n2;
         i += (long long)gridDim.x * kRedThreads) {
        double2 a = __ldg(x2 + i), b = __ldg(y2 + i);
        acc += a.x * b.x;
        acc += a.y * b.y;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) acc += x[n - 1] * y[n - 1];
    double s = block_sum<kRedThreads>(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads) final_sum_kernel(int np, const double *__restrict__ partials,
                                                                 double *__restrict__ out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += kRedThreads) acc += partials[i];
    double s = block_sum<kRedThreads>(acc);
    if (threadIdx.x == 0) *out = s;
}

void dot_dev(long long n, const double *x, const double *y, double *partials, double *out, cudaStream_t s) {
    int np = reduce_partials();
    dot_partial_kernel<<<np, kRedThreads, 0, s>>>(n, x, y, partials);
    JX_LAUNCH_CHECK();
    final_sum_kernel<<<1, kRedThreads, 0, s>>>(np, partials, out);
    JX_LAUNCH_CHECK();
}

__global__ void axpy_kernel(long long n, double alpha, const double *__restrict__ x, double *__restrict__ y) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = y[i] + alpha * x[i];
}
__global__ void scale_kernel_d(long long n, double alpha, double *__restrict__ x) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = alpha * x[i];
}
__global__ void fill_kernel(long long n, double v, double *__restrict__ x) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = v;
}

void axpy_dev(long long n, double alpha, const double *x, double *y, cudaStream_t s) {
    if (n <= 0) return;
    axpy_kernel<<<div_up(n, 256), 256, 0, s>>>(n, alpha, x, y);
    JX_LAUNCH_CHECK();
}
void scale_dev(long long n, double alpha, double *x, cudaStream_t s) {
    if (n <= 0) return;
    scale_kernel_d<<<div_up(n, 256), 256, 0, s>>>(n, alpha, x);
    JX_LAUNCH_CHECK();
}
void copy_dev(long long n, const double *x, double *y, cudaStream_t s) {
    if (n <= 0 || x == y) return;
    JX_CUDA(cudaMemcpyAsync(y, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
}
void fill_dev(long long n, double v, double *x, cudaStream_t s) {
    if (n <= 0) return;
    fill_kernel<<<div_up(n, 256), 256, 0, s>>>(n, v, x);
    JX_LAUNCH_CHECK();
}

}  // namespace jxcpr
