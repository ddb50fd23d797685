// Setup of the pressure AMG hierarchy as CPR configures it
// (jxfpamg-0220/csrc/cpr/jxf_cpr.c:319-377): classical strength, HMIS
// coarsening, extended+i interpolation, Galerkin coarse operator.
//
// Every numeric and ordering decision follows the reference so that the CF
// splitting, the interpolation pattern and values and the coarse operators
// are bit-identical (checked against the oracle and the golden fixtures):
//
// * strength      -- jxf_PAMGCreateS, amg/par_strength.c:20-415; one thread
//                    per row, S keeps A's column order without the diagonal.
// * HMIS          -- amg/par_coarsen_hmis.c:20-37: the Ruge-Stueben first
//                    pass (par_coarsen_ruge.c:249-420) is a sequential greedy
//                    on a bucket list and runs on the host (rs_first_pass in
//                    setup_host.cpp); the PMIS completion
//                    (par_coarsen_pmis.c:27-719) runs here.  Its result does
//                    not depend on the order points are visited, so a
//                    parallel sweep per round reproduces it; the random
//                    tie-breaks are the reference's Park-Miller sequence from
//                    seed 2747 (par_indepset.c:19-55), computed per point by
//                    jumping ahead a^(i+1) mod (2^31-1).
// * ext+i         -- jxf_PAMGBuildExtPIInterp, amg/par_interp_6.c:19-790; one
//                    thread per fine row runs the reference's row procedure,
//                    with the row's interpolation set kept in a scratch list
//                    (discovery order) instead of the global marker array.
// * Galerkin      -- jxf_PAMGBuildCoarseOperatorKT,
//                    operation/matops/par_rap.c:185: one thread per coarse
//                    row walks R row -> A row -> P row, diagonal first, new
//                    columns appended in discovery order, products (r*a)*p
//                    accumulated in traversal order, with a per-row open-
//                    addressing table mapping column -> slot.
#include <algorithm>
#include <vector>

#include "amg.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

// ---------------------------------------------------------------------------
// Strength of connection
// ---------------------------------------------------------------------------
__global__ void strength_mark_kernel(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                     const double *__restrict__ a, double theta, double max_row_sum,
                                     unsigned char *__restrict__ mark, int *__restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int d = ia[i], e = ia[i + 1];
    if (d == e) {  // empty row: no connections (the reference assumes a stored diagonal)
        cnt[i] = 0;
        return;
    }
    const double diag = a[d];
    double row_scale = 0.0, row_sum = diag;
    if (diag < 0) {
        for (int k = d + 1; k < e; ++k) {
            const double v = a[k];
            row_scale = row_scale < v ? v : row_scale;
            row_sum += v;
        }
    } else {
        for (int k = d + 1; k < e; ++k) {
            const double v = a[k];
            row_scale = row_scale < v ? row_scale : v;
            row_sum += v;
        }
    }
    row_sum = fabs(row_sum / diag);
    int c = 0;
    mark[d] = 0;
    if ((row_sum > max_row_sum) && (max_row_sum < 1.0)) {
        for (int k = d + 1; k < e; ++k) mark[k] = 0;
    } else if (diag < 0) {
        for (int k = d + 1; k < e; ++k) {
            const unsigned char m = !(a[k] <= theta * row_scale);
            mark[k] = m;
            c += m;
        }
    } else {
        for (int k = d + 1; k < e; ++k) {
            const unsigned char m = !(a[k] >= theta * row_scale);
            mark[k] = m;
            c += m;
        }
    }
    cnt[i] = c;
}

__global__ void strength_fill_kernel(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                     const unsigned char *__restrict__ mark, const int *__restrict__ sia,
                                     int *__restrict__ sja) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = sia[i];
    for (int k = ia[i]; k < ia[i + 1]; ++k)
        if (mark[k]) sja[p++] = ja[k];
}

void amg_strength(const CsrView<double> &A, double theta, double max_row_sum, DevPattern &S, cudaStream_t s) {
    const int n = A.nrows;
    DevBuf<unsigned char> mark(A.nnz > 0 ? A.nnz : 1);
    DevBuf<int> cnt(n + 1);
    cnt.zero(s);
    strength_mark_kernel<<<div_up(n, 256), 256, 0, s>>>(n, A.ia, A.ja, A.a, theta, max_row_sum, mark.get(),
                                                        cnt.get());
    JX_LAUNCH_CHECK();
    S.n = n;
    S.ia.alloc(n + 1);
    exclusive_scan_int(cnt.get(), S.ia.get(), n + 1, s);
    int nnz = 0;
    JX_CUDA(cudaMemcpyAsync(&nnz, S.ia.get() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    S.nnz = nnz;
    S.ja.alloc(nnz > 0 ? nnz : 1);
    strength_fill_kernel<<<div_up(n, 256), 256, 0, s>>>(n, A.ia, A.ja, mark.get(), S.ia.get(), S.ja.get());
    JX_LAUNCH_CHECK();
    JX_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------------------
// PMIS completion of HMIS
// ---------------------------------------------------------------------------
#define CF_C 1
#define CF_F (-1)
#define CF_Z (-2)
#define CF_SF (-3)

__global__ void col_count_kernel(long long nnz, const int *__restrict__ ja, int *__restrict__ cnt) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnz) atomicAdd(cnt + ja[k], 1);
}

// Park-Miller: seed_{i+1} = 16807 * seed_i mod (2^31 - 1); the i-th draw after
// seeding with s0 is s0 * 16807^(i+1) mod m, divided by m.
__device__ __forceinline__ unsigned long long pm_pow(unsigned long long e) {
    const unsigned long long m = 2147483647ULL;
    unsigned long long r = 1, b = 16807ULL;
    while (e) {
        if (e & 1ULL) r = (r * b) % m;
        b = (b * b) % m;
        e >>= 1;
    }
    return r;
}

__global__ void pmis_init_kernel(int n, const int *__restrict__ sia, const int *__restrict__ colcnt,
                                 double *__restrict__ measure, int *__restrict__ cf,
                                 unsigned char *__restrict__ in_graph) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long m = 2147483647ULL;
    const unsigned long long seed = (2747ULL * pm_pow((unsigned long long)i + 1ULL)) % m;
    double meas = (double)colcnt[i];
    meas += (double)(int)seed / 2147483647.0;
    int c = cf[i];
    unsigned char g = 0;
    if (c == -1) c = 0;
    if (c == CF_Z) {
        if (meas >= 1.0 || (sia[i + 1] - sia[i]) > 0) {
            c = 0;
            g = 1;
        } else {
            c = CF_F;
        }
    } else if (c == CF_SF) {
        meas = 0.0;
    } else {
        g = 1;
    }
    cf[i] = c;
    measure[i] = meas;
    in_graph[i] = g;
}

__global__ void pmis_is_init_kernel(int n, const double *__restrict__ measure, const unsigned char *__restrict__ g,
                                    int *__restrict__ cf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && g[i] && measure[i] > 1) cf[i] = 1;
}

__global__ void pmis_is_remove_kernel(int n, const int *__restrict__ sia, const int *__restrict__ sja,
                                      const double *__restrict__ measure, const unsigned char *__restrict__ g,
                                      int *__restrict__ cf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !g[i]) return;
    const double mi = measure[i];
    if (!(mi > 1)) return;
    for (int k = sia[i]; k < sia[i + 1]; ++k) {
        int j = sja[k];
        if (j < 0) j = -j - 1;
        const double mj = measure[j];
        if (mj > 1) {
            if (mi > mj) cf[j] = 0;
            else if (mj > mi) cf[i] = 0;
        }
    }
}

__global__ void pmis_set_cf_kernel(int n, const int *__restrict__ sia, int *__restrict__ sja,
                                   const double *__restrict__ measure, const unsigned char *__restrict__ g,
                                   int *__restrict__ cf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !g[i]) return;
    const int kb = sia[i], ke = sia[i + 1];
    int c = cf[i];
    bool remove = false;
    if (measure[i] < 1.0) {
        c = CF_F;
        remove = true;
    }
    if (c > 0) {
        c = CF_C;
        remove = true;
    } else {
        for (int k = kb; k < ke; ++k) {
            int j = sja[k];
            if (j < 0) j = -j - 1;
            if (j != i && cf[j] > 0) c = CF_F;  // a neighbour's own entry is never i (S has no diagonal)
        }
        if (c == CF_F) remove = true;
    }
    cf[i] = c;
    if (remove)
        for (int k = kb; k < ke; ++k)
            if (sja[k] > -1) sja[k] = -sja[k] - 1;
}

__global__ void pmis_remove_edges_kernel(int n, const int *__restrict__ sia, int *__restrict__ sja,
                                         const unsigned char *__restrict__ g, const int *__restrict__ cf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !g[i] || cf[i] != 0) return;
    for (int k = sia[i]; k < sia[i + 1]; ++k) {
        int j = sja[k];
        if (j < 0) j = -j - 1;
        if (cf[j] != 0 && sja[k] > -1) sja[k] = -sja[k] - 1;
    }
}

__global__ void pmis_update_graph_kernel(int n, double *__restrict__ measure, unsigned char *__restrict__ g,
                                         const int *__restrict__ cf, int *__restrict__ remaining) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !g[i]) return;
    if (cf[i] != 0) {
        measure[i] = 0.0;
        g[i] = 0;
    } else {
        atomicAdd(remaining, 1);
    }
}

__global__ void count_flag_kernel(int n, const unsigned char *__restrict__ g, int *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && g[i]) atomicAdd(out, 1);
}

void amg_pmis(const DevPattern &S, int *cf_dev, cudaStream_t s) {
    const int n = S.n;
    DevBuf<int> sja(S.nnz > 0 ? S.nnz : 1), colcnt(n), counter(1);
    DevBuf<double> measure(n);
    DevBuf<unsigned char> g(n);
    if (S.nnz) JX_CUDA(cudaMemcpyAsync(sja.get(), S.ja.get(), sizeof(int) * S.nnz, cudaMemcpyDeviceToDevice, s));
    colcnt.zero(s);
    if (S.nnz) {
        col_count_kernel<<<div_up(S.nnz, 256), 256, 0, s>>>(S.nnz, S.ja.get(), colcnt.get());
        JX_LAUNCH_CHECK();
    }
    const int grid = div_up(n, 256);
    pmis_init_kernel<<<grid, 256, 0, s>>>(n, S.ia.get(), colcnt.get(), measure.get(), cf_dev, g.get());
    JX_LAUNCH_CHECK();
    counter.zero(s);
    count_flag_kernel<<<grid, 256, 0, s>>>(n, g.get(), counter.get());
    JX_LAUNCH_CHECK();
    int remaining = 0;
    JX_CUDA(cudaMemcpyAsync(&remaining, counter.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    int iter = 0;
    while (remaining > 0) {
        if (iter > 20000) {
            set_error("pmis: no progress");
            throw CudaError{cudaErrorUnknown, "pmis"};
        }
        if (iter) {
            pmis_is_init_kernel<<<grid, 256, 0, s>>>(n, measure.get(), g.get(), cf_dev);
            JX_LAUNCH_CHECK();
            pmis_is_remove_kernel<<<grid, 256, 0, s>>>(n, S.ia.get(), sja.get(), measure.get(), g.get(), cf_dev);
            JX_LAUNCH_CHECK();
        }
        ++iter;
        pmis_set_cf_kernel<<<grid, 256, 0, s>>>(n, S.ia.get(), sja.get(), measure.get(), g.get(), cf_dev);
        JX_LAUNCH_CHECK();
        pmis_remove_edges_kernel<<<grid, 256, 0, s>>>(n, S.ia.get(), sja.get(), g.get(), cf_dev);
        JX_LAUNCH_CHECK();
        counter.zero(s);
        pmis_update_graph_kernel<<<grid, 256, 0, s>>>(n, measure.get(), g.get(), cf_dev, counter.get());
        JX_LAUNCH_CHECK();
        JX_CUDA(cudaMemcpyAsync(&remaining, counter.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        JX_CUDA(cudaStreamSynchronize(s));
    }
}

// ---------------------------------------------------------------------------
// Extended+i interpolation
// ---------------------------------------------------------------------------
__global__ void c_flag_kernel(int n, const int *__restrict__ cf, int *__restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = cf[i] >= 0 ? 1 : 0;
}

// Upper bound of the interpolation set size of each fine row.
__global__ void interp_bound_kernel(int n, const int *__restrict__ sia, const int *__restrict__ sja,
                                    const int *__restrict__ cf, long long *__restrict__ bound) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long b = 0;
    const int ci = cf[i];
    if (ci >= 0) {
        b = 1;
    } else if (ci != CF_SF) {
        for (int k = sia[i]; k < sia[i + 1]; ++k) {
            const int i1 = sja[k];
            const int c1 = cf[i1];
            if (c1 >= 0) b += 1;
            else if (c1 != CF_SF) b += sia[i1 + 1] - sia[i1];
        }
    }
    bound[i] = b;
}

// Lowest t < len with list[t] == v, or -1: the whole warp searches (v uniform).
__device__ __forceinline__ int warp_find(const int *list, int len, int v) {
    const int lane = threadIdx.x & 31;
    for (int t0 = 0; t0 < len; t0 += 32) {
        const int t = t0 + lane;
        const unsigned hit = __ballot_sync(0xffffffffu, t < len && list[t] == v);
        if (hit) return t0 + __ffs(hit) - 1;
    }
    return -1;
}

// One lane's own search (lanes look for different values).
__device__ __forceinline__ int lane_find(const int *list, int len, int v) {
    for (int t = 0; t < len; ++t)
        if (list[t] == v) return t;
    return -1;
}

// Discovery-ordered interpolation set of each F row (fine indices, deduped),
// one warp per row: the candidates are taken in order, each one searched for
// by the whole warp in the set built so far.
__global__ void interp_list_kernel(int n, const int *__restrict__ sia, const int *__restrict__ sja,
                                   const int *__restrict__ cf, const long long *__restrict__ boff,
                                   int *__restrict__ scratch, int *__restrict__ cnt) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= n) return;  // whole warps
    const int i = (int)gw;
    const int ci = cf[i];
    if (ci >= 0 || ci == CF_SF) {
        if (lane == 0) cnt[i] = ci >= 0 ? 1 : 0;
        return;
    }
    int *list = scratch + boff[i];
    int len = 0;
    auto add = [&](int v) {
        if (warp_find(list, len, v) < 0) {
            if (lane == 0) list[len] = v;
            __syncwarp();
            ++len;
        }
    };
    for (int k = sia[i]; k < sia[i + 1]; ++k) {
        const int i1 = sja[k];
        const int c1 = cf[i1];
        if (c1 >= 0) {
            add(i1);
        } else if (c1 != CF_SF) {
            for (int q = sia[i1]; q < sia[i1 + 1]; ++q) {
                const int k1 = sja[q];
                if (cf[k1] >= 0) add(k1);
            }
        }
    }
    if (lane == 0) cnt[i] = len;
}

// i1 a strong F neighbour of i (whole warp)
__device__ __forceinline__ bool warp_is_strong_f(const int *__restrict__ sia, const int *__restrict__ sja,
                                                 const int *__restrict__ cf, int i, int i1) {
    const int c1 = cf[i1];
    if (c1 >= 0 || c1 == CF_SF) return false;
    return warp_find(sja + sia[i], sia[i + 1] - sia[i], i1) >= 0;
}

// Weights of each F row, one warp per row.  Every floating-point operation is
// the sequential row algorithm's, in its order: the entries of row i are
// taken one after another (the warp only searches the interpolation set in
// parallel); the sum over a strong F neighbour's row is accumulated in column
// order from flags computed 32 entries at a time; the distribution adds to
// distinct weights (distinct columns), so its lanes may run side by side.
__global__ void interp_fill_kernel(int n, const int *__restrict__ aia, const int *__restrict__ aja,
                                   const double *__restrict__ aa, const int *__restrict__ sia,
                                   const int *__restrict__ sja, const int *__restrict__ cf,
                                   const int *__restrict__ f2c, const long long *__restrict__ boff,
                                   const int *__restrict__ scratch, const int *__restrict__ pia,
                                   int *__restrict__ pja, double *__restrict__ pa) {
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= n) return;  // whole warps
    const int i = (int)gw;
    const int ci = cf[i];
    const int jb = pia[i];
    if (ci >= 0) {
        if (lane == 0) {
            pja[jb] = f2c[i];
            pa[jb] = 1.0;
        }
        return;
    }
    if (ci == CF_SF) return;
    const int *list = scratch + boff[i];
    const int len = pia[i + 1] - jb;
    for (int t = lane; t < len; t += 32) {
        pja[jb + t] = f2c[list[t]];
        pa[jb + t] = 0.0;
    }
    __syncwarp();
    if (aia[i] == aia[i + 1]) return;  // empty row
    double diagonal = aa[aia[i]];
    for (int k = aia[i] + 1; k < aia[i + 1]; ++k) {
        const int i1 = aja[k];
        const int slot = warp_find(list, len, i1);
        if (slot >= 0) {
            if (lane == 0) pa[jb + slot] += aa[k];
        } else if (warp_is_strong_f(sia, sja, cf, i, i1)) {
            double sum = 0.0;
            int sgn = 1;
            if (aia[i1] < aia[i1 + 1] && aa[aia[i1]] < 0) sgn = -1;
            const int qb = aia[i1] + 1, qe = aia[i1 + 1];
            for (int q0 = qb; q0 < qe; q0 += 32) {
                const int q = q0 + lane;
                double v = 0.0;
                int f = 0;
                if (q < qe) {
                    const int i2 = aja[q];
                    v = aa[q];
                    f = ((i2 == i || lane_find(list, len, i2) >= 0) && (sgn * v) < 0) ? 1 : 0;
                }
                const int m = min(32, qe - q0);
                for (int u = 0; u < m; ++u) {
                    const double vu = __shfl_sync(0xffffffffu, v, u);
                    if (__shfl_sync(0xffffffffu, f, u)) sum += vu;
                }
            }
            if (sum != 0) {
                const double distribute = aa[k] / sum;
                double dadd = 0.0;
                int has = 0;
                for (int q = qb + lane; q < qe; q += 32) {
                    const int i2 = aja[q];
                    const double v = aa[q];
                    if ((sgn * v) < 0) {
                        const int s2 = lane_find(list, len, i2);
                        if (s2 >= 0) pa[jb + s2] += distribute * v;
                        if (i2 == i) {
                            dadd = distribute * v;
                            has = 1;
                        }
                    }
                }
                const unsigned hb = __ballot_sync(0xffffffffu, has);
                if (hb) diagonal += __shfl_sync(0xffffffffu, dadd, __ffs(hb) - 1);
            } else {
                diagonal += aa[k];
            }
        } else if (cf[i1] != CF_SF) {
            diagonal += aa[k];
        }
        __syncwarp();
    }
    for (int t = lane; t < len; t += 32) pa[jb + t] /= -diagonal;
}

int amg_extpi_interp(const CsrView<double> &A, const DevPattern &S, const int *cf_dev, DeviceCsr &P,
                     cudaStream_t s) {
    const int n = A.nrows;
    const int grid = div_up(n, 256);
    DevBuf<int> flag(n + 1), f2c(n + 1), cnt(n + 1);
    c_flag_kernel<<<grid, 256, 0, s>>>(n, cf_dev, flag.get());
    JX_LAUNCH_CHECK();
    exclusive_scan_int(flag.get(), f2c.get(), n + 1, s);
    int nc = 0;
    JX_CUDA(cudaMemcpyAsync(&nc, f2c.get() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    DevBuf<long long> bound(n + 1), boff(n + 1);
    bound.zero(s);
    interp_bound_kernel<<<grid, 256, 0, s>>>(n, S.ia.get(), S.ja.get(), cf_dev, bound.get());
    JX_LAUNCH_CHECK();
    exclusive_scan_ll(bound.get(), boff.get(), n + 1, s);
    long long total = 0;
    JX_CUDA(cudaMemcpyAsync(&total, boff.get() + n, sizeof(long long), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    DevBuf<int> scratch(total > 0 ? total : 1);
    cnt.zero(s);
    const int wgrid = (int)div_up((long long)n * 32, 256);  // one warp per row
    interp_list_kernel<<<wgrid, 256, 0, s>>>(n, S.ia.get(), S.ja.get(), cf_dev, boff.get(), scratch.get(),
                                            cnt.get());
    JX_LAUNCH_CHECK();
    DevBuf<int> pia(n + 1);
    exclusive_scan_int(cnt.get(), pia.get(), n + 1, s);
    int nnz = 0;
    JX_CUDA(cudaMemcpyAsync(&nnz, pia.get() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    P.nrows = n;
    P.ncols = nc;
    P.nnz = nnz;
    P.ia = std::move(pia);
    P.ja.alloc(nnz > 0 ? nnz : 1);
    P.a.alloc(nnz > 0 ? nnz : 1);
    interp_fill_kernel<<<wgrid, 256, 0, s>>>(n, A.ia, A.ja, A.a, S.ia.get(), S.ja.get(), cf_dev, f2c.get(),
                                            boff.get(), scratch.get(), P.ia.get(), P.ja.get(), P.a.get());
    JX_LAUNCH_CHECK();
    JX_CUDA(cudaStreamSynchronize(s));
    return nc;
}

// ---------------------------------------------------------------------------
// Galerkin coarse operator A_c = R A P (R = P^T, stable transpose)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned hash_col(int c) { return (unsigned)c * 2654435761u; }

// Returns the slot of column J (inserting it with slot `next` if absent).
__device__ __forceinline__ int table_slot(int *keys, int *vals, long long tsz, int J, int &next, bool &fresh) {
    unsigned h = hash_col(J) & (unsigned)(tsz - 1);
    while (true) {
        const int k = keys[h];
        if (k == J) {
            fresh = false;
            return vals[h];
        }
        if (k < 0) {
            keys[h] = J;
            vals[h] = next;
            fresh = true;
            return next++;
        }
        h = (h + 1) & (unsigned)(tsz - 1);
    }
}

// Warp-cooperative Galerkin product with the same discovery and accumulation
// order as the sequential traversal (R row I -> A row i -> P row j): the 32
// lanes take 32 consecutive products of the traversal; lanes with the same
// coarse column are grouped (__match_any_sync) and the group's lowest lane adds
// the members' products to the column's sum one by one in lane order, so
// every column's sum is formed in traversal order.  New columns get slots in
// order of first occurrence.  The row's column table lives in shared memory,
// in two sizes: every row is first tried with a 256-entry table (8 warps per
// block, many blocks per SM: the rows of the fine levels are short), a row
// with more than 128 columns again with a 2,048-entry table (2 warps per
// block), and a row with more than 1,024 columns is redone by
// rap_fallback_kernel (one thread, table in global memory).  The table only
// indexes the columns: a row's result does not depend on which size held it.
// overflow[I]: 0 small table, 1 large table, 2 fallback.
static constexpr int kRapTableS = 256, kRapWarpsS = 8;   // small tier: entries per warp, warps per block
static constexpr int kRapTableL = 2048, kRapWarpsL = 2;  // large tier

template <int TBL>
__device__ __forceinline__ int rap_find(const int *keys, int J) {
    unsigned h = hash_col(J) & (TBL - 1);
    while (true) {
        const int k = keys[h];
        if (k == J) return (int)h;
        if (k < 0) return -1;
        h = (h + 1) & (TBL - 1);
    }
}

template <int TBL>
__device__ __forceinline__ int rap_insert(int *keys, int J) {
    unsigned h = hash_col(J) & (TBL - 1);
    while (true) {
        const int prev = atomicCAS(keys + h, -1, J);
        if (prev == -1 || prev == J) return (int)h;
        h = (h + 1) & (TBL - 1);
    }
}

template <bool FILL, int TBL, int WARPS>
__global__ void __launch_bounds__(32 * WARPS)
    rap_warp_kernel(int nrows, const int *__restrict__ ria, const int *__restrict__ rja,
                    const double *__restrict__ ra, const int *__restrict__ aia, const int *__restrict__ aja,
                    const double *__restrict__ aa, const int *__restrict__ pia, const int *__restrict__ pja,
                    const double *__restrict__ pa, int *__restrict__ cnt, unsigned char *__restrict__ overflow,
                    const int *__restrict__ cia, int *__restrict__ cja, double *__restrict__ ca) {
    constexpr int kMaxCols = TBL / 2;  // columns a warp row may hold
    constexpr unsigned char kTier = TBL == kRapTableS ? 0 : 1;
    extern __shared__ __align__(16) unsigned char rap_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *keys = reinterpret_cast<int *>(rap_smem) + warp * TBL;
    int *slots = reinterpret_cast<int *>(rap_smem) + WARPS * TBL + warp * TBL;
    double *vals = reinterpret_cast<double *>(rap_smem + (size_t)2 * WARPS * TBL * sizeof(int)) + warp * TBL;
    const unsigned FULL = 0xffffffffu;
    for (int I = blockIdx.x * WARPS + warp; I < nrows; I += gridDim.x * WARPS) {
        // the small tier counts every row; every other pass takes the rows of its own tier
        if ((FILL || kTier == 1) && overflow[I] != kTier) continue;
        for (int t = lane; t < TBL; t += 32) keys[t] = -1;
        __syncwarp();
        int next = 1;
        if (lane == 0) {
            const int h = rap_insert<TBL>(keys, I);  // diagonal first, starting from zero
            slots[h] = 0;
            if (FILL) vals[h] = 0.0;
        }
        __syncwarp();
        bool over = false;
        for (int r = ria[I]; r < ria[I + 1] && !over; ++r) {
            const int i = rja[r];
            const double rv = FILL ? ra[r] : 0.0;
            const int kb = aia[i], ke = aia[i + 1];
            for (int kc = kb; kc < ke && !over; kc += 32) {
                const int k = kc + lane;
                int len = 0, j = 0;
                double av = 0.0;
                if (k < ke) {
                    j = aja[k];
                    av = FILL ? aa[k] : 0.0;
                    len = pia[j + 1] - pia[j];
                }
                int incl = len;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += v;
                }
                const int pre = incl - len;
                const int total = __shfl_sync(FULL, incl, 31);
                for (int pb = 0; pb < total; pb += 32) {
                    const int p = pb + lane;
                    const bool valid = p < total;
                    // owner: the last lane whose prefix is <= p
                    int lo = 0, hi = 31;
#pragma unroll
                    for (int it = 0; it < 5; ++it) {
                        const int mid = (lo + hi + 1) >> 1;
                        const int pm = __shfl_sync(FULL, pre, mid);
                        if (pm <= p) lo = mid; else hi = mid - 1;
                    }
                    const int o = lo;
                    const int jo = __shfl_sync(FULL, j, o);
                    const double ao = __shfl_sync(FULL, av, o);
                    const int preo = __shfl_sync(FULL, pre, o);
                    int J = -1 - lane;  // unique dummy key for idle lanes
                    double prod = 0.0;
                    if (valid) {
                        const int q = pia[jo] + (p - preo);
                        J = pja[q];
                        if (FILL) prod = (rv * ao) * pa[q];
                    }
                    const unsigned grp = __match_any_sync(FULL, J);
                    const int leader = __ffs(grp) - 1;
                    const bool is_leader = valid && lane == leader;
                    int h = -1;
                    if (is_leader) h = rap_find<TBL>(keys, J);
                    const bool fresh = is_leader && h < 0;
                    const unsigned fresh_mask = __ballot_sync(FULL, fresh);
                    if (next + __popc(fresh_mask) > kMaxCols) {
                        over = true;  // warp-uniform
                        break;
                    }
                    if (fresh) {
                        h = rap_insert<TBL>(keys, J);
                        slots[h] = next + __popc(fresh_mask & ((1u << lane) - 1u));
                    }
                    next += __popc(fresh_mask);
                    if (FILL) {
                        // each leader adds its group's products in lane order (the discovery order);
                        // the warp takes as many shuffle steps as the largest group has members
                        double acc = 0.0;
                        bool first = fresh;
                        if (is_leader && !fresh) acc = vals[h];
                        unsigned rem = is_leader ? grp : 0u;
                        const unsigned steps = __reduce_max_sync(FULL, (unsigned)__popc(rem));
                        for (unsigned it = 0; it < steps; ++it) {
                            const int src = rem ? __ffs(rem) - 1 : lane;
                            const double v = __shfl_sync(FULL, prod, src);
                            if (rem) {
                                if (first) {
                                    acc = v;
                                    first = false;
                                } else {
                                    acc += v;
                                }
                                rem &= rem - 1u;
                            }
                        }
                        if (is_leader) vals[h] = acc;
                    }
                    __syncwarp();
                }
            }
        }
        if (over) {
            if (!FILL && lane == 0) overflow[I] = kTier + 1;  // to the next tier
            __syncwarp();
            continue;
        }
        if (!FILL) {
            if (lane == 0) cnt[I] = next;
        } else {
            const int base = cia[I];
            for (int t = lane; t < TBL; t += 32) {
                const int key = keys[t];
                if (key >= 0) {
                    cja[base + slots[t]] = key;
                    ca[base + slots[t]] = vals[t];
                }
            }
        }
        __syncwarp();
    }
}

// Thread-per-row fallback for the rows the warp kernel could not hold.
template <bool FILL>
__global__ void rap_fallback_kernel(int nlist, const int *__restrict__ list, const int *__restrict__ ria,
                                    const int *__restrict__ rja, const double *__restrict__ ra,
                                    const int *__restrict__ aia, const int *__restrict__ aja,
                                    const double *__restrict__ aa, const int *__restrict__ pia,
                                    const int *__restrict__ pja, const double *__restrict__ pa,
                                    const long long *__restrict__ toff, int *__restrict__ tkeys,
                                    int *__restrict__ tvals, int *__restrict__ cnt, const int *__restrict__ cia,
                                    int *__restrict__ cja, double *__restrict__ ca) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nlist) return;
    const int I = list[t];
    const long long tsz = toff[t + 1] - toff[t];
    int *keys = tkeys + toff[t];
    int *vals = tvals + toff[t];
    for (long long q = 0; q < tsz; ++q) keys[q] = -1;
    int next = 0;
    bool fresh;
    const int base = FILL ? cia[I] : 0;
    table_slot(keys, vals, tsz, I, next, fresh);
    if (FILL) {
        cja[base] = I;
        ca[base] = 0.0;
    }
    for (int r = ria[I]; r < ria[I + 1]; ++r) {
        const int i = rja[r];
        const double pr = FILL ? ra[r] : 0.0;
        for (int k = aia[i]; k < aia[i + 1]; ++k) {
            const int j = aja[k];
            const double pav = FILL ? pr * aa[k] : 0.0;
            for (int q = pia[j]; q < pia[j + 1]; ++q) {
                const int J = pja[q];
                const int slot = table_slot(keys, vals, tsz, J, next, fresh);
                if (FILL) {
                    if (fresh) {
                        cja[base + slot] = J;
                        ca[base + slot] = pav * pa[q];
                    } else {
                        ca[base + slot] += pav * pa[q];
                    }
                }
            }
        }
    }
    if (!FILL) cnt[I] = next;
}

void amg_rap(const CsrView<double> &A, const DeviceCsr &P, const DeviceCsr &R, DeviceCsr &Ac, cudaStream_t s,
             long long table_budget_entries) {
    (void)table_budget_entries;
    const int nc = P.ncols;
    const size_t smemS = (size_t)kRapWarpsS * kRapTableS * (2 * sizeof(int) + sizeof(double));
    const size_t smemL = (size_t)kRapWarpsL * kRapTableL * (2 * sizeof(int) + sizeof(double));
    static bool attr[64] = {};
    int dev = 0;
    JX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !attr[dev]) {
        JX_CUDA(cudaFuncSetAttribute(rap_warp_kernel<false, kRapTableL, kRapWarpsL>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemL));
        JX_CUDA(cudaFuncSetAttribute(rap_warp_kernel<true, kRapTableL, kRapWarpsL>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemL));
        if (dev >= 0 && dev < 64) attr[dev] = true;
    }
    DevBuf<int> cnt(nc + 1);
    DevBuf<unsigned char> over(nc + 1);
    cnt.zero(s);
    over.zero(s);
    const int gridS = std::max(1, std::min(div_up(nc, kRapWarpsS), 64 * sm_count()));
    const int gridL = std::max(1, std::min(div_up(nc, kRapWarpsL), 64 * sm_count()));
    if (nc > 0) {
        rap_warp_kernel<false, kRapTableS, kRapWarpsS><<<gridS, 32 * kRapWarpsS, smemS, s>>>(
            nc, R.ia.get(), R.ja.get(), R.a.get(), A.ia, A.ja, A.a, P.ia.get(), P.ja.get(), P.a.get(), cnt.get(),
            over.get(), nullptr, nullptr, nullptr);
        JX_LAUNCH_CHECK();
        rap_warp_kernel<false, kRapTableL, kRapWarpsL><<<gridL, 32 * kRapWarpsL, smemL, s>>>(
            nc, R.ia.get(), R.ja.get(), R.a.get(), A.ia, A.ja, A.a, P.ia.get(), P.ja.get(), P.a.get(), cnt.get(),
            over.get(), nullptr, nullptr, nullptr);
        JX_LAUNCH_CHECK();
    }
    // rows that overflowed the shared table: thread-per-row with a global table
    std::vector<unsigned char> h_over(nc > 0 ? nc : 1);
    over.download(h_over.data(), nc, s);
    JX_CUDA(cudaStreamSynchronize(s));
    std::vector<int> list;
    for (int I = 0; I < nc; ++I)
        if (h_over[I] == 2) list.push_back(I);
    const int nl = (int)list.size();
    DevBuf<int> d_list(nl > 0 ? nl : 1);
    DevBuf<long long> toff(nl + 1);
    DevBuf<int> tkeys, tvals;
    if (nl > 0) {
        d_list.upload(list.data(), nl, s);
        // table per listed row: 2 x (columns reachable) <= 2 x nc, power of two
        long long t = 16;
        while (t < 2LL * nc) t <<= 1;
        std::vector<long long> h_off(nl + 1);
        for (int q = 0; q <= nl; ++q) h_off[q] = (long long)q * t;
        toff.upload(h_off.data(), nl + 1, s);
        tkeys.alloc((size_t)nl * t);
        tvals.alloc((size_t)nl * t);
        rap_fallback_kernel<false><<<div_up(nl, 64), 64, 0, s>>>(
            nl, d_list.get(), R.ia.get(), R.ja.get(), R.a.get(), A.ia, A.ja, A.a, P.ia.get(), P.ja.get(), P.a.get(),
            toff.get(), tkeys.get(), tvals.get(), cnt.get(), nullptr, nullptr, nullptr);
        JX_LAUNCH_CHECK();
    }
    DevBuf<int> cia(nc + 1);
    exclusive_scan_int(cnt.get(), cia.get(), nc + 1, s);
    int nnz = 0;
    JX_CUDA(cudaMemcpyAsync(&nnz, cia.get() + nc, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    Ac.nrows = nc;
    Ac.ncols = nc;
    Ac.nnz = nnz;
    Ac.ia = std::move(cia);
    Ac.ja.alloc(nnz > 0 ? nnz : 1);
    Ac.a.alloc(nnz > 0 ? nnz : 1);
    if (nc > 0) {
        rap_warp_kernel<true, kRapTableS, kRapWarpsS><<<gridS, 32 * kRapWarpsS, smemS, s>>>(
            nc, R.ia.get(), R.ja.get(), R.a.get(), A.ia, A.ja, A.a, P.ia.get(), P.ja.get(), P.a.get(), nullptr,
            over.get(), Ac.ia.get(), Ac.ja.get(), Ac.a.get());
        JX_LAUNCH_CHECK();
        rap_warp_kernel<true, kRapTableL, kRapWarpsL><<<gridL, 32 * kRapWarpsL, smemL, s>>>(
            nc, R.ia.get(), R.ja.get(), R.a.get(), A.ia, A.ja, A.a, P.ia.get(), P.ja.get(), P.a.get(), nullptr,
            over.get(), Ac.ia.get(), Ac.ja.get(), Ac.a.get());
        JX_LAUNCH_CHECK();
    }
    if (nl > 0) {
        rap_fallback_kernel<true><<<div_up(nl, 64), 64, 0, s>>>(
            nl, d_list.get(), R.ia.get(), R.ja.get(), R.a.get(), A.ia, A.ja, A.a, P.ia.get(), P.ja.get(), P.a.get(),
            toff.get(), tkeys.get(), tvals.get(), nullptr, Ac.ia.get(), Ac.ja.get(), Ac.a.get());
        JX_LAUNCH_CHECK();
    }
    JX_CUDA(cudaStreamSynchronize(s));
}

}  // namespace jxcpr
