// Exclusive prefix sums (CUB device scan) used to turn per-row counts into
// CSR row pointers.
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

template <typename T>
static void excl_scan(const T *in, T *out, int n, cudaStream_t s) {
    if (n <= 0) return;
    size_t bytes = 0;
    JX_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    DevBuf<unsigned char> tmp(bytes + 16);
    JX_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in, out, n, s));
    JX_CUDA(cudaStreamSynchronize(s));
}

void exclusive_scan_int(const int *in, int *out, int n, cudaStream_t s) { excl_scan<int>(in, out, n, s); }
void exclusive_scan_ll(const long long *in, long long *out, int n, cudaStream_t s) {
    excl_scan<long long>(in, out, n, s);
}

}  // namespace jxcpr
