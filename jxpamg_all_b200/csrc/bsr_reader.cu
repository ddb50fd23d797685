// BSR files read into device memory (the formats of jxf_BSRMatrixRead / _Binary,
// jxfpamg-0220/csrc/mat_vec_data/seq_bsr_matrix.c:1735-2120, as the host readers in dropin.cu take
// them): the file is read in 64 MB chunks into pinned host memory, each chunk's copy to the device
// starts as soon as it is read (the read of the next one overlaps it), and a text file is then
// tokenised and converted on the device.
//
// Text: every white-space separated token is located by a count pass and a write pass over 64-byte
// chunks (one thread each) around an exclusive scan; the integers of the header, the row pointer and
// the block columns, and the block values are converted by one thread per token (parse_num.cuh: the
// nearest binary64, as the host reader's fscanf("%le") gives; the rare token the device does not
// convert -- more than 19 significant digits, inf, nan -- is converted on the host with strtod).
// Then, as the host reader does: 1-based row pointers and columns become 0-based, the largest column
// must be num_cols - 1, and storage 1 (column-major blocks) is transposed to row-major blocks.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"
#include "jxcpr_b200.h"
#include "kernels.cuh"
#include "parse_num.cuh"

namespace jxcpr {
namespace {

constexpr int kT = 256;
constexpr int kChunk = 64;                     // bytes per tokeniser thread
constexpr size_t kReadChunk = 64ull << 20;     // bytes per file read / upload
constexpr int kMaxToken = 64;                  // longest token accepted
constexpr int kMaxFallback = 1 << 20;          // tokens converted on the host at most

__host__ __device__ inline bool is_space(unsigned char c) { return c == ' ' || (c >= 9 && c <= 13); }

// Token starts in each 64-byte chunk (a byte that is not white space after one that is, or first).
__global__ void count_tokens_kernel(const unsigned char *__restrict__ buf, long long size, int *__restrict__ cnt,
                                    long long nchunks) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const long long b0 = c * kChunk, b1 = min(size, b0 + kChunk);
    int n = 0;
    bool prev_space = b0 == 0 ? true : is_space(buf[b0 - 1]);
    for (long long i = b0; i < b1; ++i) {
        const bool sp = is_space(buf[i]);
        n += (!sp && prev_space) ? 1 : 0;
        prev_space = sp;
    }
    cnt[c] = n;
}

__global__ void write_tokens_kernel(const unsigned char *__restrict__ buf, long long size,
                                    const int *__restrict__ off, long long nchunks, long long ntok,
                                    long long *__restrict__ pos) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const long long b0 = c * kChunk, b1 = min(size, b0 + kChunk);
    long long t = off[c];
    bool prev_space = b0 == 0 ? true : is_space(buf[b0 - 1]);
    for (long long i = b0; i < b1; ++i) {
        const bool sp = is_space(buf[i]);
        if (!sp && prev_space && t < ntok) pos[t++] = i;
        prev_space = sp;
    }
}

// Length of the token starting at p (bounded by the buffer and kMaxToken + 1).
__device__ inline int token_len(const unsigned char *buf, long long size, long long p) {
    int len = 0;
    while (p + len < size && len <= kMaxToken && !is_space(buf[p + len])) ++len;
    return len;
}

// err[0]: a malformed token (its index + 1 in err[1]); err[2]: fallback count
__global__ void parse_ints_kernel(const unsigned char *__restrict__ buf, long long size,
                                  const long long *__restrict__ pos, long long t0, long long n, int *__restrict__ out,
                                  int *__restrict__ err) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const long long p = pos[t0 + k];
    const int len = token_len(buf, size, p);
    int v = 0;
    if (len > kMaxToken || numparse::parse_int(reinterpret_cast<const char *>(buf + p), len, &v) != numparse::kParseOk) {
        atomicExch(err, 1);
        atomicMax(err + 1, (int)min(t0 + k + 1, 2147483647LL));
        return;
    }
    out[k] = v;
}

__global__ void parse_doubles_kernel(const unsigned char *__restrict__ buf, long long size,
                                     const long long *__restrict__ pos, long long t0, long long n,
                                     const unsigned long long *__restrict__ table, double *__restrict__ out,
                                     long long *__restrict__ fallback, int *__restrict__ err) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const long long p = pos[t0 + k];
    const int len = token_len(buf, size, p);
    uint64_t bits = 0;
    const int st = len > kMaxToken ? numparse::kParseFallback
                                   : numparse::parse_double(reinterpret_cast<const char *>(buf + p), len, table, &bits);
    if (st == numparse::kParseOk) {
        out[k] = __longlong_as_double((long long)bits);
    } else if (st == numparse::kParseFallback) {
        const int slot = atomicAdd(err + 2, 1);
        if (slot < kMaxFallback) fallback[slot] = k;
        out[k] = 0.0;
    } else {
        atomicExch(err, 1);
        atomicMax(err + 1, (int)min(t0 + k + 1, 2147483647LL));
    }
}

// 1-based row pointer / columns to 0-based; the largest column into *maxcol
__global__ void rebase_kernel(int *__restrict__ ia, long long nia, int *__restrict__ ja, long long nja, int base,
                              int *__restrict__ maxcol) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nia) ia[k] -= base;
    if (k < nja) {
        const int j = ja[k] - base;
        ja[k] = j;
        atomicMax(maxcol, j);
    }
}

__global__ void blocks_row_major_kernel(double *__restrict__ a, long long nnz, int bs) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    double t[9];
    const int bn = bs * bs;
    double *b = a + k * bn;
    for (int q = 0; q < bn; ++q) t[q] = b[q];
    for (int bi = 0; bi < bs; ++bi)
        for (int bj = 0; bj < bs; ++bj) b[bi * bs + bj] = t[bj * bs + bi];
}

struct Pinned {
    void *p = nullptr;
    explicit Pinned(size_t n) { JX_CUDA(cudaHostAlloc(&p, n > 0 ? n : 1, cudaHostAllocDefault)); }
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};
struct DevRaw {
    void *p = nullptr;
    explicit DevRaw(size_t n) { JX_CUDA(cudaMalloc(&p, n > 0 ? n : 1)); }
    ~DevRaw() {
        if (p) cudaFree(p);
    }
    void *release() {
        void *q = p;
        p = nullptr;
        return q;
    }
};

// Reads `size` bytes of fp into pinned memory and the device buffer, chunk by chunk (the copy of a
// chunk overlaps the read of the next).  False on a short read.
bool read_upload(FILE *fp, size_t size, unsigned char *host, unsigned char *dev, cudaStream_t s) {
    for (size_t off = 0; off < size; off += kReadChunk) {
        const size_t n = std::min(kReadChunk, size - off);
        if (fread(host + off, 1, n, fp) != n) return false;
        JX_CUDA(cudaMemcpyAsync(dev + off, host + off, n, cudaMemcpyHostToDevice, s));
    }
    return true;
}

struct ReadOut {
    int rows = 0, cols = 0, bs = 0;
    long long nnz = 0;
    int *ia = nullptr, *ja = nullptr;
    double *a = nullptr;
};

int fail(const char *fmt, const char *file) {
    set_error(fmt, file);
    return JXCPR_ERROR_ARG;
}

// Shared tail of both formats: 0-based indices, the column check, row-major blocks.
int finish(ReadOut &R, int storage, int *base_probe, const char *file, cudaStream_t s) {
    int first = 0;
    JX_CUDA(cudaMemcpyAsync(&first, R.ia, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    const int base = first == 1 ? 1 : 0;
    JX_CUDA(cudaMemsetAsync(base_probe, 0xff, sizeof(int), s));  // -1: no column yet
    const long long n = std::max<long long>(R.rows + 1, R.nnz);
    if (n > 0) {
        rebase_kernel<<<div_up(n, kT), kT, 0, s>>>(R.ia, R.rows + 1, R.ja, R.nnz, base, base_probe);
        JX_LAUNCH_CHECK();
    }
    int maxcol = -1;
    JX_CUDA(cudaMemcpyAsync(&maxcol, base_probe, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    if (R.nnz > 0 && maxcol + 1 != R.cols) return fail("bsr read: largest column + 1 != num_cols in %s", file);
    if (storage == 1 && R.nnz > 0) {
        blocks_row_major_kernel<<<div_up(R.nnz, kT), kT, 0, s>>>(R.a, R.nnz, R.bs);
        JX_LAUNCH_CHECK();
    }
    JX_CUDA(cudaStreamSynchronize(s));
    return JXCPR_SUCCESS;
}

int read_binary(FILE *fp, const char *file, ReadOut &R, cudaStream_t s) {
    int hdr[5];
    if (fread(hdr, sizeof(int), 5, fp) != 5 || hdr[0] < 0 || hdr[2] < 0 || hdr[3] < 1 || hdr[3] > 3)
        return fail("bsr read: malformed header in %s", file);
    R.rows = hdr[0];
    R.cols = hdr[1];
    R.nnz = hdr[2];
    R.bs = hdr[3];
    const int storage = hdr[4];
    const long long bn = (long long)R.bs * R.bs, nv = R.nnz * bn;
    DevRaw dia((size_t)(R.rows + 1) * 4), dja((size_t)R.nnz * 4), da((size_t)nv * 8), probe(4);
    int n = 0;
    Pinned h(std::max<size_t>((size_t)nv * 8, (size_t)std::max<long long>(R.rows + 1, R.nnz) * 4));
    auto *hb = static_cast<unsigned char *>(h.p);
    // the three arrays one after another through the same pinned buffer (each copy waits for the last)
    const bool ia_ok = fread(&n, 4, 1, fp) == 1 && n == R.rows + 1 &&
                       read_upload(fp, (size_t)n * 4, hb, (unsigned char *)dia.p, s);
    JX_CUDA(cudaStreamSynchronize(s));  // the pinned buffer is reused for the next array
    if (!ia_ok) return fail("bsr read: malformed row pointer in %s", file);
    const bool ja_ok = fread(&n, 4, 1, fp) == 1 && n == R.nnz &&
                       read_upload(fp, (size_t)n * 4, hb, (unsigned char *)dja.p, s);
    JX_CUDA(cudaStreamSynchronize(s));
    if (!ja_ok) return fail("bsr read: malformed columns in %s", file);
    const bool vals_ok = fread(&n, 4, 1, fp) == 1 && (long long)n == nv &&
                         read_upload(fp, (size_t)nv * 8, hb, (unsigned char *)da.p, s);
    JX_CUDA(cudaStreamSynchronize(s));
    if (!vals_ok) return fail("bsr read: malformed values in %s", file);
    R.ia = static_cast<int *>(dia.p);
    R.ja = static_cast<int *>(dja.p);
    R.a = static_cast<double *>(da.p);
    const int st = finish(R, storage, static_cast<int *>(probe.p), file, s);
    if (st != JXCPR_SUCCESS) return st;
    dia.release();
    dja.release();
    da.release();
    return JXCPR_SUCCESS;
}

int read_text(FILE *fp, const char *file, ReadOut &R, cudaStream_t s) {
    if (fseek(fp, 0, SEEK_END) != 0) return fail("bsr read: cannot seek %s", file);
    const long long size = ftell(fp);
    if (size <= 0 || fseek(fp, 0, SEEK_SET) != 0) return fail("bsr read: empty file %s", file);
    Pinned h((size_t)size);
    DevRaw dbuf((size_t)size);
    auto *hb = static_cast<unsigned char *>(h.p);
    auto *db = static_cast<unsigned char *>(dbuf.p);
    const bool read_ok = read_upload(fp, (size_t)size, hb, db, s);
    JX_CUDA(cudaStreamSynchronize(s));  // the pinned buffer is read below and freed on every return
    if (!read_ok) return fail("bsr read: short read of %s", file);
    // header from the pinned copy: rows cols nnz bs storage
    long long hv[5];
    {
        long long p = 0;
        for (int k = 0; k < 5; ++k) {
            while (p < size && is_space(hb[p])) ++p;
            long long e = p;
            while (e < size && !is_space(hb[e])) ++e;
            int v = 0;
            if (e == p || e - p > kMaxToken ||
                numparse::parse_int(reinterpret_cast<const char *>(hb + p), (int)(e - p), &v) != numparse::kParseOk)
                return fail("bsr read: malformed header in %s", file);
            hv[k] = v;
            p = e;
        }
    }
    if (hv[0] < 0 || hv[2] < 0 || hv[3] < 1 || hv[3] > 3) return fail("bsr read: malformed header in %s", file);
    R.rows = (int)hv[0];
    R.cols = (int)hv[1];
    R.nnz = hv[2];
    R.bs = (int)hv[3];
    const int storage = (int)hv[4];
    const long long bn = (long long)R.bs * R.bs, nv = R.nnz * bn;
    // token layout: 5 header, n+1, ia (rows+1), nnz, ja (nnz), nnz*bn, values
    const long long t_ia = 6, t_ja = t_ia + R.rows + 2, t_a = t_ja + R.nnz + 1;
    const long long ntok = t_a + nv;
    const long long nchunks = (size + kChunk - 1) / kChunk;
    if (nchunks >= (1LL << 31) || ntok >= (1LL << 31)) return fail("bsr read: file too large: %s", file);
    DevBuf<int> cnt(nchunks + 1), off(nchunks + 1), err(4), probe(1);
    DevBuf<long long> pos(ntok), fb(std::min<long long>(std::max<long long>(nv, 1), kMaxFallback));
    DevBuf<unsigned long long> table(sizeof(numparse::kPow5Table) / sizeof(unsigned long long));
    table.upload(numparse::kPow5Table, table.n, s);
    err.zero(s);
    JX_CUDA(cudaMemsetAsync(cnt.get() + nchunks, 0, sizeof(int), s));
    count_tokens_kernel<<<div_up(nchunks, kT), kT, 0, s>>>(db, size, cnt.get(), nchunks);
    JX_LAUNCH_CHECK();
    exclusive_scan_int(cnt.get(), off.get(), (int)(nchunks + 1), s);
    int found = 0;
    JX_CUDA(cudaMemcpyAsync(&found, off.get() + nchunks, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    if ((long long)found != ntok) {
        set_error("bsr read: %s holds %d numbers, its header asks for %lld", file, found, ntok);
        return JXCPR_ERROR_ARG;
    }
    write_tokens_kernel<<<div_up(nchunks, kT), kT, 0, s>>>(db, size, off.get(), nchunks, ntok, pos.get());
    JX_LAUNCH_CHECK();
    // the three counts, the row pointer, the columns
    DevBuf<int> counts(3);
    const long long cpos[3] = {5, t_ja - 1, t_a - 1};
    for (int c = 0; c < 3; ++c) {
        parse_ints_kernel<<<1, 1, 0, s>>>(db, size, pos.get(), cpos[c], 1, counts.get() + c, err.get());
        JX_LAUNCH_CHECK();
    }
    DevRaw dia((size_t)(R.rows + 1) * 4), dja((size_t)R.nnz * 4), da((size_t)nv * 8);
    parse_ints_kernel<<<div_up(R.rows + 1, kT), kT, 0, s>>>(db, size, pos.get(), t_ia, R.rows + 1,
                                                           static_cast<int *>(dia.p), err.get());
    JX_LAUNCH_CHECK();
    if (R.nnz > 0) {
        parse_ints_kernel<<<div_up(R.nnz, kT), kT, 0, s>>>(db, size, pos.get(), t_ja, R.nnz,
                                                          static_cast<int *>(dja.p), err.get());
        JX_LAUNCH_CHECK();
    }
    if (nv > 0) {
        parse_doubles_kernel<<<div_up(nv, kT), kT, 0, s>>>(db, size, pos.get(), t_a, nv, table.get(),
                                                           static_cast<double *>(da.p), fb.get(), err.get());
        JX_LAUNCH_CHECK();
    }
    int e[4] = {0, 0, 0, 0}, hc[3] = {0, 0, 0};
    JX_CUDA(cudaMemcpyAsync(e, err.get(), sizeof(e), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaMemcpyAsync(hc, counts.get(), sizeof(hc), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    if (e[0]) {
        set_error("bsr read: malformed number (token %d) in %s", e[1] - 1, file);
        return JXCPR_ERROR_ARG;
    }
    if (hc[0] != R.rows + 1 || hc[1] != R.nnz || (long long)hc[2] != nv)
        return fail("bsr read: array lengths in %s disagree with its header", file);
    if (e[2] > 0) {  // tokens the device did not convert: strtod on the host, from the pinned copy
        std::vector<long long> idx;
        if (e[2] <= kMaxFallback) {
            idx.resize(e[2]);
            JX_CUDA(cudaMemcpyAsync(idx.data(), fb.get(), sizeof(long long) * e[2], cudaMemcpyDeviceToHost, s));
        } else {  // more than the list holds: every value
            idx.resize(nv);
            for (long long k = 0; k < nv; ++k) idx[k] = k;
        }
        std::vector<long long> tp(idx.size());
        std::vector<double> vals(idx.size());
        if ((long long)idx.size() == nv) {  // every value: all positions at once
            JX_CUDA(cudaMemcpyAsync(tp.data(), pos.get() + t_a, sizeof(long long) * nv, cudaMemcpyDeviceToHost, s));
        } else {
            for (size_t q = 0; q < idx.size(); ++q)
                JX_CUDA(cudaMemcpyAsync(&tp[q], pos.get() + t_a + idx[q], sizeof(long long), cudaMemcpyDeviceToHost,
                                        s));
        }
        JX_CUDA(cudaStreamSynchronize(s));
        for (size_t q = 0; q < idx.size(); ++q) {
            const long long p = tp[q];
            long long end = p;
            while (end < size && !is_space(hb[end])) ++end;
            std::string tok(reinterpret_cast<const char *>(hb + p), (size_t)(end - p));
            char *ep = nullptr;
            vals[q] = strtod(tok.c_str(), &ep);
            if (ep != tok.c_str() + tok.size()) return fail("bsr read: malformed number in %s", file);
        }
        if ((long long)idx.size() == nv) {
            JX_CUDA(cudaMemcpyAsync(da.p, vals.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, s));
        } else {
            for (size_t q = 0; q < idx.size(); ++q)
                JX_CUDA(cudaMemcpyAsync(static_cast<double *>(da.p) + idx[q], &vals[q], sizeof(double),
                                        cudaMemcpyHostToDevice, s));
        }
        JX_CUDA(cudaStreamSynchronize(s));
    }
    R.ia = static_cast<int *>(dia.p);
    R.ja = static_cast<int *>(dja.p);
    R.a = static_cast<double *>(da.p);
    const int st = finish(R, storage, probe.get(), file, s);
    if (st != JXCPR_SUCCESS) return st;
    dia.release();
    dja.release();
    da.release();
    return JXCPR_SUCCESS;
}

}  // namespace
}  // namespace jxcpr

using namespace jxcpr;

extern "C" {

JXCPR_API int jxcpr_bsr_read_device(const char *file, int binary, int *rows, int *cols, int *bs, long long *nnzb,
                                    int **ia, int **ja, double **a, void *stream) {
    if (!file || !rows || !cols || !bs || !nnzb || !ia || !ja || !a) return JXCPR_ERROR_ARG;
    FILE *fp = fopen(file, binary ? "rb" : "r");
    if (!fp) {
        set_error("bsr read: cannot open %s", file);
        return JXCPR_ERROR_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ReadOut R;
    int st;
    try {
        st = binary ? read_binary(fp, file, R, s) : read_text(fp, file, R, s);
    } catch (const CudaError &) {
        st = JXCPR_ERROR_DEVICE;
    }
    fclose(fp);
    if (st != JXCPR_SUCCESS) return st;
    *rows = R.rows;
    *cols = R.cols;
    *bs = R.bs;
    *nnzb = R.nnz;
    *ia = R.ia;
    *ja = R.ja;
    *a = R.a;
    return JXCPR_SUCCESS;
}

JXCPR_API int jxcpr_bsr_free_device(int *ia, int *ja, double *a) {
    if (ia) cudaFree(ia);
    if (ja) cudaFree(ja);
    if (a) cudaFree(a);
    return JXCPR_SUCCESS;
}

JXCPR_API int jxcpr_parse_double_host(const char *token, int len, double *out) {
    if (!token || !out || len < 0) return JXCPR_ERROR_ARG;
    uint64_t bits = 0;
    const int st = numparse::parse_double(token, len, numparse::kPow5Table, &bits);
    if (st == numparse::kParseOk) memcpy(out, &bits, sizeof(double));
    return st;
}

}  // extern "C"
