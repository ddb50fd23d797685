// The two inherently sequential graph passes of the setup, run on the host:
//
// * rs_first_pass_host -- the Ruge-Stueben first coloring pass used by HMIS
//   (jxfpamg-0220/csrc/amg/par_coarsen_ruge.c:249-420 with the bucket lists
//   of amg/amg_linklist.c).  It is a greedy that always takes the head of the
//   highest non-empty measure bucket, so its result depends on the exact
//   insertion order; it is reproduced here with O(1) bucket operations:
//   buckets indexed by measure, points appended at the tail, the highest
//   non-empty bucket tracked.
//   rs_first_pass_ranges runs the pass on row ranges of a fixed size, each on
//   the diagonal block of S for its rows (strong connections to other ranges
//   are not seen), as every process of a distributed run of the reference does
//   (par_coarsen_ruge.c:37-44 take S_diag, :197 and :212 count the measures in
//   it alone for the HMIS first pass, :261 marks SF_PT only when the row is
//   empty in the diagonal and the off-diagonal block).  The ranges depend
//   on n and the range size only, so the splitting is the same on any host;
//   the ranges run on host threads.
// * build_schedule_host -- grouping of rows for the Gauss-Seidel sweeps on
//   the device: either the level schedule of the natural ordering (row i
//   waits for every j < i of its row in a forward sweep, j > i backward) or a
//   greedy multicolouring.
// * build_chunk_order_host -- the stage-2 sweep order of the throughput path:
//   chunks of `chunk` consecutive rows, greedily coloured so that no two
//   chunks of one colour are coupled; the sweep visits the colours in turn
//   and, inside each chunk, its rows in natural order.
//
// All read the pattern once (O(nnz)); everything numeric stays on the GPU.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "amg.cuh"

namespace jxcpr {

namespace {
struct Buckets {
    std::vector<int> next, prev, head, tail;
    int maxm = 0;
    Buckets(int n, int cap) : next(n, -1), prev(n, -1), head(cap, -1), tail(cap, -1) {}
    void enter(int m, int i) {
        next[i] = -1;
        prev[i] = tail[m];
        if (tail[m] >= 0) next[tail[m]] = i; else head[m] = i;
        tail[m] = i;
        if (m > maxm) maxm = m;
    }
    void remove(int m, int i) {
        if (prev[i] >= 0) next[prev[i]] = next[i]; else head[m] = next[i];
        if (next[i] >= 0) prev[next[i]] = prev[i]; else tail[m] = prev[i];
        while (maxm > 0 && head[maxm] < 0) --maxm;
    }
};
}  // namespace

void rs_first_pass_host(int n, const int *Si, const int *Sj, int *CF, const int *gia) {
    const int nnz = Si[n];
    std::vector<int> STi(n + 1, 0), STj(nnz > 0 ? nnz : 1);
    for (int k = 0; k < nnz; ++k) STi[Sj[k] + 1]++;
    for (int i = 0; i < n; ++i) STi[i + 1] += STi[i];
    {
        std::vector<int> pos(STi.begin(), STi.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int k = Si[i]; k < Si[i + 1]; ++k) STj[pos[Sj[k]]++] = i;
    }
    rs_first_pass_host(n, Si, Sj, STi.data(), STj.data(), CF, gia);
}

// STi/STj: the transpose of S with the rows of each column in ascending order.
// gia (optional): the row offsets of the whole strength pattern when S is the
// diagonal block of a row range; a point is SF_PT only when that row is empty.
void rs_first_pass_host(int n, const int *Si, const int *Sj, const int *STi, const int *STj, int *CF,
                        const int *gia) {
    const int C_PT = 1, F_PT = -1, Z_PT = -2, SF_PT = -3, UNDEC = 0;
    std::vector<int> measure(n);
    int maxmeasure = 0;
    for (int i = 0; i < n; ++i) {
        measure[i] = STi[i + 1] - STi[i];
        maxmeasure = std::max(maxmeasure, measure[i]);
    }
    Buckets B(n, maxmeasure + n + 2);
    int num_left = 0;
    const int *rows = gia ? gia : Si;
    for (int j = 0; j < n; ++j) {
        if (rows[j + 1] - rows[j] == 0) {
            CF[j] = SF_PT;
            measure[j] = 0;
        } else {
            CF[j] = UNDEC;
            ++num_left;
        }
    }
    for (int j = 0; j < n; ++j) {
        const int m = measure[j];
        if (CF[j] == SF_PT) continue;
        if (m > 0) {
            B.enter(m, j);
        } else {
            CF[j] = Z_PT;
            for (int k = Si[j]; k < Si[j + 1]; ++k) {
                const int nb = Sj[k];
                if (CF[nb] != SF_PT) {
                    if (nb < j) {
                        int nm = measure[nb];
                        if (nm > 0) B.remove(nm, nb);
                        nm = ++measure[nb];
                        B.enter(nm, nb);
                    } else {
                        ++measure[nb];
                    }
                }
            }
            --num_left;
        }
    }
    while (num_left > 0) {
        const int index = B.head[B.maxm];
        CF[index] = C_PT;
        const int m = measure[index];
        measure[index] = 0;
        --num_left;
        B.remove(m, index);
        for (int k = STi[index]; k < STi[index + 1]; ++k) {
            const int nb = STj[k];
            if (CF[nb] == UNDEC) {
                CF[nb] = F_PT;
                B.remove(measure[nb], nb);
                --num_left;
                for (int q = Si[nb]; q < Si[nb + 1]; ++q) {
                    const int n2 = Sj[q];
                    if (CF[n2] == UNDEC) {
                        B.remove(measure[n2], n2);
                        B.enter(++measure[n2], n2);
                    }
                }
            }
        }
        for (int k = Si[index]; k < Si[index + 1]; ++k) {
            const int nb = Sj[k];
            if (CF[nb] == UNDEC) {
                int mm = measure[nb];
                B.remove(mm, nb);
                measure[nb] = --mm;
                if (mm > 0) {
                    B.enter(mm, nb);
                } else {
                    CF[nb] = F_PT;
                    --num_left;
                    for (int q = Si[nb]; q < Si[nb + 1]; ++q) {
                        const int n2 = Sj[q];
                        if (CF[n2] == UNDEC) {
                            B.remove(measure[n2], n2);
                            B.enter(++measure[n2], n2);
                        }
                    }
                }
            }
        }
    }
}

void rs_first_pass_ranges(int n, const int *Si, const int *Sj, int range_rows, int *CF) {
    const int nr = range_rows > 0 ? std::max(1, n / range_rows) : 1;
    if (nr == 1) {
        rs_first_pass_host(n, Si, Sj, CF, nullptr);
        return;
    }
    auto one = [&](int r) {
        const int r0 = (int)((long long)n * r / nr), r1 = (int)((long long)n * (r + 1) / nr), m = r1 - r0;
        std::vector<int> li(m + 1, 0), lj;
        lj.reserve((size_t)(Si[r1] - Si[r0]) + 1);
        for (int i = r0; i < r1; ++i) {
            for (int k = Si[i]; k < Si[i + 1]; ++k) {
                const int j = Sj[k];
                if (j >= r0 && j < r1) lj.push_back(j - r0);
            }
            li[i - r0 + 1] = (int)lj.size();
        }
        rs_first_pass_host(m, li.data(), lj.data(), CF + r0, Si + r0);
    };
    const int threads = std::max(1, std::min(nr, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next{0};
    auto worker = [&]() {
        for (int r = next.fetch_add(1); r < nr; r = next.fetch_add(1)) one(r);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
}

void build_schedule_host(int n, const int *ia, const int *ja, int order, bool forward, std::vector<int> &perm,
                         std::vector<int> &group_ptr, std::vector<int> &rank) {
    std::vector<int> grp(n, 0);
    int ng = 0;
    if (order == ORDER_EXACT) {
        if (forward) {
            for (int i = 0; i < n; ++i) {
                int g = 0;
                for (int k = ia[i]; k < ia[i + 1]; ++k) {
                    const int j = ja[k];
                    if (j < i) g = std::max(g, grp[j] + 1);
                }
                grp[i] = g;
                ng = std::max(ng, g + 1);
            }
        } else {
            for (int i = n - 1; i >= 0; --i) {
                int g = 0;
                for (int k = ia[i]; k < ia[i + 1]; ++k) {
                    const int j = ja[k];
                    if (j > i) g = std::max(g, grp[j] + 1);
                }
                grp[i] = g;
                ng = std::max(ng, g + 1);
            }
        }
    } else {
        // greedy colouring of the symmetrised pattern, natural order
        std::vector<int> ti(n + 1, 0), tj(ia[n] > 0 ? ia[n] : 1);
        for (int k = 0; k < ia[n]; ++k) ti[ja[k] + 1]++;
        for (int i = 0; i < n; ++i) ti[i + 1] += ti[i];
        {
            std::vector<int> pos(ti.begin(), ti.end() - 1);
            for (int i = 0; i < n; ++i)
                for (int k = ia[i]; k < ia[i + 1]; ++k) tj[pos[ja[k]]++] = i;
        }
        std::vector<int> color(n, -1), mark(64, -1);
        for (int i = 0; i < n; ++i) {
            auto note = [&](int j) {
                if (j != i && color[j] >= 0) {
                    if (color[j] >= (int)mark.size()) mark.resize(2 * color[j] + 2, -1);
                    mark[color[j]] = i;
                }
            };
            for (int k = ia[i]; k < ia[i + 1]; ++k) note(ja[k]);
            for (int k = ti[i]; k < ti[i + 1]; ++k) note(tj[k]);
            int c = 0;
            while (c < (int)mark.size() && mark[c] == i) ++c;
            color[i] = c;
            ng = std::max(ng, c + 1);
        }
        for (int i = 0; i < n; ++i) grp[i] = forward ? color[i] : (ng - 1 - color[i]);
    }
    if (n == 0) ng = 0;
    group_ptr.assign(ng + 1, 0);
    for (int i = 0; i < n; ++i) group_ptr[grp[i] + 1]++;
    for (int g = 0; g < ng; ++g) group_ptr[g + 1] += group_ptr[g];
    perm.assign(n > 0 ? n : 1, 0);
    std::vector<int> pos(group_ptr.begin(), group_ptr.end());
    for (int i = 0; i < n; ++i) perm[pos[grp[i]]++] = i;
    // rank: the position of a row in the sequential order the sweep emulates
    rank.assign(n > 0 ? n : 1, 0);
    if (order == ORDER_EXACT) {
        for (int i = 0; i < n; ++i) rank[i] = forward ? i : (n - 1 - i);
    } else {
        for (int i = 0; i < n; ++i) rank[i] = grp[i];
    }
}

void upload_schedule(const std::vector<int> &perm, const std::vector<int> &gptr, const std::vector<int> &rank,
                     Schedule &S, cudaStream_t s) {
    S.ngroups = (int)gptr.size() - 1;
    S.h_group_ptr = gptr;
    S.max_group = 0;
    for (int g = 0; g < S.ngroups; ++g) S.max_group = std::max(S.max_group, gptr[g + 1] - gptr[g]);
    S.perm.alloc(perm.size());
    S.perm.upload(perm.data(), perm.size(), s);
    S.group_ptr.alloc(gptr.size());
    S.group_ptr.upload(gptr.data(), gptr.size(), s);
    S.rank.alloc(rank.size());
    S.rank.upload(rank.data(), rank.size(), s);
    JX_CUDA(cudaStreamSynchronize(s));
}

// Stage-2 order of the throughput path.  The reference sweeps the block rows in natural order
// (jxf_ParBSRHGSRelax, jxfpamg-0220/csrc/amg/par_relax_bsr.c:193-573).  On the upwinded reservoir
// Jacobians that order carries information along the grid's fastest index within one sweep, and a
// plain multicolouring loses it (C1: 57 GMRES iterations instead of 51).  Chunks of `chunk`
// consecutive rows keep that coupling: chunk c = rows [c*chunk, (c+1)*chunk), chunks coloured in
// natural order with the smallest colour no coupled chunk (symmetrised pattern) has taken.  Output:
// order = stored rows, colour by colour, chunks ascending, each chunk's rows ascending, every chunk
// padded to `chunk` entries and every colour to a multiple of 32 entries with -1; seg = the colour
// segments' stored-row offsets.  chunk must divide 32.
void build_chunk_order_host(int n, const int *ia, const int *ja, int chunk, std::vector<int> &order,
                            std::vector<int> &seg) {
    order.clear();
    seg.assign(1, 0);
    if (n <= 0) return;
    const int nc = (n + chunk - 1) / chunk;
    // transpose pattern (column -> rows) for the symmetrised coupling
    std::vector<int> ti(n + 1, 0), tj(ia[n] > 0 ? ia[n] : 1);
    for (int k = 0; k < ia[n]; ++k) ti[ja[k] + 1]++;
    for (int i = 0; i < n; ++i) ti[i + 1] += ti[i];
    {
        std::vector<int> pos(ti.begin(), ti.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int k = ia[i]; k < ia[i + 1]; ++k) tj[pos[ja[k]]++] = i;
    }
    std::vector<int> color(nc, -1), mark(64, -1);
    int ncol = 0;
    for (int c = 0; c < nc; ++c) {
        auto note = [&](int j) {
            const int d = j / chunk;
            if (d != c && color[d] >= 0) {
                if (color[d] >= (int)mark.size()) mark.resize(2 * color[d] + 2, -1);
                mark[color[d]] = c;
            }
        };
        const int i1 = std::min(n, (c + 1) * chunk);
        for (int i = c * chunk; i < i1; ++i) {
            for (int k = ia[i]; k < ia[i + 1]; ++k) note(ja[k]);
            for (int k = ti[i]; k < ti[i + 1]; ++k) note(tj[k]);
        }
        int q = 0;
        while (q < (int)mark.size() && mark[q] == c) ++q;
        color[c] = q;
        ncol = std::max(ncol, q + 1);
    }
    std::vector<int> cnt(ncol + 1, 0);
    for (int c = 0; c < nc; ++c) cnt[color[c] + 1]++;
    std::vector<int> cstart(ncol + 1, 0);
    for (int q = 0; q < ncol; ++q) cstart[q + 1] = cstart[q] + cnt[q + 1];
    std::vector<int> corder(nc);
    {
        std::vector<int> pos(cstart.begin(), cstart.end() - 1);
        for (int c = 0; c < nc; ++c) corder[pos[color[c]]++] = c;
    }
    for (int q = 0; q < ncol; ++q) {
        for (int t = cstart[q]; t < cstart[q + 1]; ++t) {
            const int c = corder[t];
            for (int r = 0; r < chunk; ++r) order.push_back(c * chunk + r < n ? c * chunk + r : -1);
        }
        while (order.size() % 32) order.push_back(-1);
        seg.push_back((int)order.size());
    }
}

}  // namespace jxcpr
