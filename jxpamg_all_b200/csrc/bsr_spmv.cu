// BSR sparse matrix-vector product y = alpha*A*x + beta*y for b x b blocks
// (b = 2, 3), the hot kernel of the CPR-GMRES path.
//
// Semantics follow jxf_BSRMatrixMatvec (jxfpamg-0220/csrc/operation/mvops/
// seq_bsr_matvec.c:22-140): y <- (beta/alpha) y (0 if beta/alpha == 0,
// untouched if 1), then for each block of the row in stored order and each
// block column in order  y_i += A_ij x_j, then y <- alpha y.  Each output
// component is accumulated by one thread in exactly that order with separate
// multiply and add (the library is compiled with --fmad=false), so results
// are bit-identical to the reference CPU loop.
//
// B200 mapping: a CTA owns a tile of ROWS consecutive block rows, one thread
// per output component.  The tile's block values and column indices are a
// contiguous slab of global memory [ia[r0], ia[r1]); a single elected thread
// streams each slab into shared memory with the 1-D bulk TMA copy
// (cp.async.bulk, completion on an mbarrier) while the CTA computes the
// previous tile, STAGES slabs deep.  CTAs are persistent (grid = 2 x SMs) and
// walk tiles with a grid stride.  x is gathered through the read-only path
// (it is L2-resident: 18 MB for 1.12 M 2x2 rows).  A tile whose slab does not
// fit a stage, or whose 16-byte-rounded copy would run past the end of the
// arrays, is computed with direct global loads instead; results are the same.
#include "common.cuh"
#include "kernels.cuh"
#include "ptx.cuh"

namespace jxcpr {

template <int BS, typename V>
struct SpmvTileCfg {
    static constexpr int ROWS = (BS == 2) ? 128 : 64;
    static constexpr int THREADS = ROWS * BS;
    static constexpr int STAGES = 3;
    static constexpr int CAP_BLOCKS = ROWS * ((BS == 2) ? 8 : 7);
    static constexpr int VAL_BYTES = CAP_BLOCKS * BS * BS * (int)sizeof(V) + 32;
    static constexpr int COL_BYTES = CAP_BLOCKS * 4 + 32;
    static constexpr int STAGE_BYTES = ((VAL_BYTES + 15) / 16 + (COL_BYTES + 15) / 16) * 16;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 128;
};

struct SlabPlan {
    long long v_src;  // byte offset of the 16-aligned copy start in a[]
    int v_bytes;      // copy size (multiple of 16)
    int v_pre;        // bytes between copy start and the first block of the tile
    long long c_src;
    int c_bytes;
    int c_pre;
    bool staged;
};

template <int BS, typename V>
__device__ __forceinline__ SlabPlan plan_slab(long long k0, long long k1, long long nnzb) {
    using Cfg = SpmvTileCfg<BS, V>;
    SlabPlan p;
    const long long vb = (long long)BS * BS * sizeof(V);
    long long vs = k0 * vb, ve = k1 * vb;
    long long vs16 = vs & ~15LL, ve16 = (ve + 15) & ~15LL;
    long long cs = k0 * 4, ce = k1 * 4;
    long long cs16 = cs & ~15LL, ce16 = (ce + 15) & ~15LL;
    p.v_src = vs16;
    p.v_bytes = (int)(ve16 - vs16);
    p.v_pre = (int)(vs - vs16);
    p.c_src = cs16;
    p.c_bytes = (int)(ce16 - cs16);
    p.c_pre = (int)(cs - cs16);
    p.staged = (k1 > k0) && (p.v_bytes <= Cfg::VAL_BYTES) && (p.c_bytes <= Cfg::COL_BYTES) &&
               (ve16 <= nnzb * vb) && (ce16 <= nnzb * 4);
    return p;
}

template <int BS, typename X>
__device__ __forceinline__ void gather_x(const X *__restrict__ x, int c, X (&xv)[BS]) {
#pragma unroll
    for (int j = 0; j < BS; ++j) xv[j] = __ldg(x + (long long)c * BS + j);
}

template <>
__device__ __forceinline__ void gather_x<2, double>(const double *__restrict__ x, int c, double (&xv)[2]) {
    double2 v = __ldg(reinterpret_cast<const double2 *>(x) + c);
    xv[0] = v.x;
    xv[1] = v.y;
}

// init_mode: 0 -> start from 0, 1 -> start from y, 2 -> start from y*scale_y.
template <int BS, typename V, typename X>
__device__ __forceinline__ X row_init(const X *y, long long idx, int init_mode, X scale_y) {
    if (init_mode == 0) return X(0);
    X v = y[idx];
    return init_mode == 1 ? v : v * scale_y;
}


// Accumulates one output component of a block row in stored block order.
template <int BS, typename V, typename X, bool SMEM>
__device__ __forceinline__ X row_accumulate(X acc, long long kb, long long ke, long long kbase,
                                            const V *__restrict__ vals, const int *__restrict__ cols,
                                            const X *__restrict__ x, int comp) {
    for (long long k = kb; k < ke; ++k) {
        const long long kk = k - kbase;
        const int c = SMEM ? cols[kk] : __ldg(cols + kk);
        X xv[BS];
        gather_x<BS, X>(x, c, xv);
#pragma unroll
        for (int j = 0; j < BS; ++j) {
            const V v = SMEM ? vals[kk * (BS * BS) + comp * BS + j] : __ldg(vals + kk * (BS * BS) + comp * BS + j);
            acc = acc + (X)v * xv[j];
        }
    }
    return acc;
}

template <int BS, typename V, typename X>
__global__ void __launch_bounds__(SpmvTileCfg<BS, V>::THREADS)
    bsr_spmv_tma_kernel(int nb, long long nnzb, const int *__restrict__ ia, const int *__restrict__ ja,
                        const V *__restrict__ a, const X *__restrict__ x, X *__restrict__ y, int init_mode,
                        X scale_y, X alpha, int *__restrict__ err) {
    using Cfg = SpmvTileCfg<BS, V>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    unsigned char *stages = smem_raw + 128;
    const int tid = threadIdx.x;
    const int tiles = (nb + Cfg::ROWS - 1) / Cfg::ROWS;
    const unsigned char *a_bytes = reinterpret_cast<const unsigned char *>(a);
    const unsigned char *j_bytes = reinterpret_cast<const unsigned char *>(ja);

    if (tid == 0) {
        for (int s = 0; s < Cfg::STAGES; ++s) ptx::mbar_init(&bars[s], 1);
        ptx::fence_mbar_init();
    }
    __syncthreads();

    auto issue = [&](int t, int s) {
        long long r0 = (long long)t * Cfg::ROWS;
        long long r1 = min((long long)nb, r0 + Cfg::ROWS);
        long long k0 = ia[r0], k1 = ia[r1];
        SlabPlan p = plan_slab<BS, V>(k0, k1, nnzb);
        unsigned char *st = stages + (size_t)s * Cfg::STAGE_BYTES;
        if (p.staged) {
            ptx::mbar_arrive_expect_tx(&bars[s], (uint32_t)(p.v_bytes + p.c_bytes));
            ptx::bulk_g2s(st, a_bytes + p.v_src, (uint32_t)p.v_bytes, &bars[s]);
            ptx::bulk_g2s(st + ((Cfg::VAL_BYTES + 15) / 16) * 16, j_bytes + p.c_src, (uint32_t)p.c_bytes,
                          &bars[s]);
        } else {
            ptx::mbar_arrive_expect_tx(&bars[s], 0u);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < Cfg::STAGES; ++s) {
            int t = blockIdx.x + s * gridDim.x;
            if (t < tiles) issue(t, s);
        }
    }

    bool aborted = false;
    int iter = 0;
    int t = blockIdx.x;
    for (; t < tiles; t += gridDim.x, ++iter) {
        const int s = iter % Cfg::STAGES;
        const uint32_t parity = (uint32_t)((iter / Cfg::STAGES) & 1);
        const long long r0 = (long long)t * Cfg::ROWS;
        const long long r1 = min((long long)nb, r0 + Cfg::ROWS);
        const long long k0 = ia[r0], k1 = ia[r1];
        const SlabPlan p = plan_slab<BS, V>(k0, k1, nnzb);
        const int failed = ptx::mbar_wait_bounded(&bars[s], parity, 1u << 26) ? 0 : 1;
        if (__syncthreads_or(failed)) {  // uniform decision: every thread leaves together
            if (tid == 0) atomicExch(err, 1);
            aborted = true;
            break;
        }
        const unsigned char *st = stages + (size_t)s * Cfg::STAGE_BYTES;
        const V *vs = reinterpret_cast<const V *>(st + p.v_pre);
        const int *cs = reinterpret_cast<const int *>(st + ((Cfg::VAL_BYTES + 15) / 16) * 16 + p.c_pre);
        const long long row = r0 + tid / BS;
        const int comp = tid % BS;
        if (row < r1) {
            const long long kb = ia[row], ke = ia[row + 1];
            const long long oidx = row * BS + comp;
            X acc = row_init<BS, V, X>(y, oidx, init_mode, scale_y);
            if (p.staged)
                acc = row_accumulate<BS, V, X, true>(acc, kb, ke, k0, vs, cs, x, comp);
            else
                acc = row_accumulate<BS, V, X, false>(acc, kb, ke, 0, a, ja, x, comp);
            y[oidx] = (alpha == X(1)) ? acc : acc * alpha;
        }
        __syncthreads();  // every thread is done with stage s
        if (tid == 0) {
            int nt = t + Cfg::STAGES * gridDim.x;
            if (nt < tiles) issue(nt, s);
        }
    }
    if (aborted && tid == 0) {
        // drain copies still in flight into this CTA's shared memory (bounded)
        int it2 = iter;
        for (int tt = t; tt < tiles && it2 < iter + Cfg::STAGES; tt += gridDim.x, ++it2) {
            int s = it2 % Cfg::STAGES;
            ptx::mbar_wait_bounded(&bars[s], (uint32_t)((it2 / Cfg::STAGES) & 1), 1u << 22);
        }
    }
}

// Direct-load variant (no staging); used for user-provided arrays without the
// guarantees above and as the reference point in tests.
template <int BS, typename V, typename X>
__global__ void __launch_bounds__(256)
    bsr_spmv_direct_kernel(int nb, const int *__restrict__ ia, const int *__restrict__ ja,
                           const V *__restrict__ a, const X *__restrict__ x, X *__restrict__ y, int init_mode,
                           X scale_y, X alpha) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gid / BS;
    const int comp = (int)(gid % BS);
    if (row >= nb) return;
    const long long kb = ia[row], ke = ia[row + 1];
    const long long oidx = row * BS + comp;
    X acc = row_init<BS, V, X>(y, oidx, init_mode, scale_y);
    acc = row_accumulate<BS, V, X, false>(acc, kb, ke, 0, a, ja, x, comp);
    y[oidx] = (alpha == X(1)) ? acc : acc * alpha;
}

template <typename X>
__global__ void scale_kernel(long long n, X beta, X *y) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = y[i] * beta;
}

template <int BS, typename V, typename X>
static void launch_spmv(const BsrView<V> &A, X alpha, const X *x, X beta, X *y, int *err, cudaStream_t stream,
                        bool staged) {
    const long long n = (long long)A.nb * BS;
    if (A.nb == 0) return;
    if (alpha == X(0)) {
        scale_kernel<X><<<div_up(n, 256), 256, 0, stream>>>(n, beta, y);
        JX_LAUNCH_CHECK();
        return;
    }
    X temp = beta / alpha;
    int init_mode = (temp == X(0)) ? 0 : (temp == X(1) ? 1 : 2);
    if (staged && err != nullptr) {
        using Cfg = SpmvTileCfg<BS, V>;
        static bool attr_set[64] = {};
        int dev = 0;
        JX_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64 || !attr_set[dev]) {
            JX_CUDA(cudaFuncSetAttribute(bsr_spmv_tma_kernel<BS, V, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         Cfg::SMEM_BYTES));
            if (dev >= 0 && dev < 64) attr_set[dev] = true;
        }
        int tiles = div_up(A.nb, Cfg::ROWS);
        int grid = std::min(tiles, 2 * sm_count());
        bsr_spmv_tma_kernel<BS, V, X><<<grid, Cfg::THREADS, Cfg::SMEM_BYTES, stream>>>(
            A.nb, A.nnzb, A.ia, A.ja, A.a, x, y, init_mode, temp, alpha, err);
    } else {
        bsr_spmv_direct_kernel<BS, V, X><<<div_up(n, 256), 256, 0, stream>>>(A.nb, A.ia, A.ja, A.a, x, y,
                                                                            init_mode, temp, alpha);
    }
    JX_LAUNCH_CHECK();
}

template <typename V, typename X>
void bsr_spmv(const BsrView<V> &A, X alpha, const X *x, X beta, X *y, int *err, cudaStream_t stream, bool staged) {
    switch (A.bs) {
        case 2: launch_spmv<2, V, X>(A, alpha, x, beta, y, err, stream, staged); break;
        case 3: launch_spmv<3, V, X>(A, alpha, x, beta, y, err, stream, staged); break;
        default:
            set_error("bsr_spmv: unsupported block size %d", A.bs);
            throw CudaError{cudaErrorInvalidValue, "block size"};
    }
}

template void bsr_spmv<double, double>(const BsrView<double> &, double, const double *, double, double *, int *,
                                       cudaStream_t, bool);
template void bsr_spmv<float, double>(const BsrView<float> &, double, const double *, double, double *, int *,
                                      cudaStream_t, bool);
template void bsr_spmv<float, float>(const BsrView<float> &, float, const float *, float, float *, int *,
                                     cudaStream_t, bool);

}  // namespace jxcpr
