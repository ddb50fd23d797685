/*
 * jxcpr_b200.h -- C ABI of the B200 CPR-GMRES library (libjxcpr_b200.so).
 *
 * Plain pointers and sizes only.  Two layers:
 *
 *  1. Device-kernel entry points (jxcpr_*_dev): device pointers, the caller's
 *     CUDA stream passed as void*.  They replace the inner loops the
 *     reference runs on the CPU and are what a solver built on this library
 *     chains together.
 *  2. Host entry points with host arrays (jxcpr_* without _dev), used by the
 *     drop-in layer in jxcpr_dropin.h and by FFI callers.
 *
 * Every function returns a status code: 0 success, 1 generic, 2 memory,
 * 4 argument, 256 not converged (the reference's codes, jxfpamg-0220/include/
 * jxf_util.h:152-159), 512 CUDA failure, 1024 NaN/Inf found on the device.
 * jxcpr_last_error() returns a message for the calling thread's last failure.
 */
#ifndef JXCPR_B200_H
#define JXCPR_B200_H

#if defined(__GNUC__)
#define JXCPR_API __attribute__((visibility("default")))
#else
#define JXCPR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define JXCPR_SUCCESS 0
#define JXCPR_ERROR_GENERIC 1
#define JXCPR_ERROR_MEMORY 2
#define JXCPR_ERROR_ARG 4
#define JXCPR_ERROR_CONV 256
#define JXCPR_ERROR_DEVICE 512
#define JXCPR_ERROR_NUMERIC 1024

/* Library version (major*10000 + minor*100 + patch). */
JXCPR_API int jxcpr_version(void);
/* Message describing the calling thread's last failure ("" if none). */
JXCPR_API const char *jxcpr_last_error(void);

/* ---- BSR SpMV ------------------------------------------------------------
 * y = alpha*A*x + beta*y for a block-CSR matrix with bs x bs row-major blocks
 * (bs = 2 or 3), 0-based ia[nb+1], ja[nnzb], a[nnzb*bs*bs]; x, y have nb*bs
 * entries and must not alias.  Replaces jxf_BSRMatrixMatvec
 * (jxfpamg-0220/csrc/operation/mvops/seq_bsr_matvec.c:22-140) and the local
 * part of jxf_ParBSRMatrixMatvec (par_bsr_matvec.c:21-221), with the same
 * rounding sequence (bit-identical results).  staged != 0 selects the
 * TMA-staged kernel; 0 the direct-load kernel.  x and y must be 16-byte
 * aligned.
 */
JXCPR_API int jxcpr_bsr_matvec_dev(int nb, int bs, long long nnzb, const int *ia, const int *ja, const double *a,
                                   double alpha, const double *x, double beta, double *y, int staged,
                                   void *stream);
/* Same with FP32 block values and FP64 vectors (products formed in FP64). */
JXCPR_API int jxcpr_bsr_matvec_dev_f32(int nb, int bs, long long nnzb, const int *ia, const int *ja,
                                       const float *a, double alpha, const double *x, double beta, double *y,
                                       int staged, void *stream);
/* Reads and clears the per-device flag that the staged kernels raise when a
 * bounded wait on the copy engine gives up (0 = none). */
JXCPR_API int jxcpr_kernel_error_flag(void);

/* ---- BLAS-1 --------------------------------------------------------------
 * <x, y> over n doubles (16-byte aligned), deterministic order; the result is
 * written to *out_host after a stream synchronisation.  Replaces
 * jxf_SeqVectorInnerProd (jxfpamg-0220/csrc/operation/vecops/seq_vecop.c:239).
 */
JXCPR_API int jxcpr_dot_dev(long long n, const double *x, const double *y, double *out_host, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* JXCPR_B200_H */
