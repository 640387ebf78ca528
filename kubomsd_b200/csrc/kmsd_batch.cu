// Ragged batches: KPM moments of many independent orthogonal-basis
// Hamiltonians of uneven size in one launch per Chebyshev step.
//
// The instances are concatenated into one block-diagonal operator (global
// CSR, and ELL when every instance has the same short width).  Their rows are
// cut into tiles that never cross an instance.  One step kernel walks the tile
// list with per-tile spectral scaling (center_i, half_i) and writes per-tile
// column partial sums; a second kernel (one CTA per instance) combines an
// instance's tiles in a fixed order and writes its moments.  The sequence of
// all steps of a call is captured once into a CUDA graph and replayed on later
// calls with the same buffers and shape.  `kmsd_batch_tune` times candidate
// tile sizes and keeps the fastest.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "kmsd.h"
#include "kmsd_impl.h"
#include "kmsd_kernels.cuh"

using namespace kmsd;

namespace {

struct Tiles {
    int *seg = nullptr;       // instance of each tile
    int64_t *r0 = nullptr;    // first row
    int64_t *r1 = nullptr;    // one past the last row
    int *seg_tile0 = nullptr; // first tile of each instance (ninst+1)
    int64_t ntiles = 0;
    int64_t tile_rows = 0;
};

template <class T> struct BatchArgs {
    using V = typename Unit<T>::vec;
    RowMap mp;
    CsrView<T> H;
    EllView<T> E;
    const int *tseg;
    const int64_t *tr0, *tr1;
    int64_t ntiles;
    const double *center, *half;  // per instance
    const V *curr, *prev;
    V *next;
    const V *bra;
    const V *hx;  // HSRC_SOLVED: the operator already applied (S^-1 H T_k)
    int first;
    int exact_sums;    // MODE_DOUBLING: FP64 row products (mu_0, mu_1 of a direct-moments call)
    double2 *partial;  // [ntiles][ncol] (x2 for doubling)
};

// One Chebyshev step over the tile list; per-tile column sums.
template <class T, int MU, int MODE, int HSRC>
__global__ void __launch_bounds__(256) batch_step_kernel(const BatchArgs<T> a) {
    using V = typename Unit<T>::vec;
    constexpr int C = Unit<T>::C;
    extern __shared__ double2 smem[];
    const RowMap mp = a.mp;
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const int ncol = mp.U * C;
    for (int64_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int s = a.tseg[tile];
        const double cen64 = a.center[s], hal64 = a.half[s];
        const T cen = (T)cen64, hal = (T)hal64, inv = (T)(1. / hal64);
        double2 acc0[MU][C], acc1[MU][C];
#pragma unroll
        for (int m = 0; m < MU; ++m)
#pragma unroll
            for (int c = 0; c < C; ++c) {
                acc0[m][c] = make_double2(0., 0.);
                acc1[m][c] = make_double2(0., 0.);
            }
        for (int64_t row = a.tr0[tile] + g; row < a.tr1[tile]; row += mp.gpc) {
            Pk<T> xo[MU], po[MU], h[MU];
#pragma unroll
            for (int m = 0; m < MU; ++m) {
                const int u = lane + m * mp.G;
                h[m] = pk_zero<T>();
                if (u < mp.U) {
                    const size_t o = (size_t)row * mp.U + u;
                    xo[m] = ld(a.curr + o);
                    po[m] = a.first ? pk_zero<T>() : ld(a.prev + o);
                }
            }
            if (HSRC == HSRC_SOLVED) {
#pragma unroll
                for (int m = 0; m < MU; ++m) {
                    const int u = lane + m * mp.G;
                    if (u < mp.U) h[m] = ld(a.hx + (size_t)row * mp.U + u);
                }
            } else if (HSRC == HSRC_ELL) {
                gather_row_ell<T, MU>(a.E, a.curr, row, mp.U, mp.G, lane, h);
            } else {
                gather_row<T, MU>(a.H, a.curr, row, mp.U, mp.G, lane, h);
            }
#pragma unroll
            for (int m = 0; m < MU; ++m) {
                const int u = lane + m * mp.G;
                if (u >= mp.U) continue;
                const size_t o = (size_t)row * mp.U + u;
                Pk<T> nx;
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const T tr = rdiv(h[m].re[c] - cen * xo[m].re[c], hal, inv);
                    const T ti = rdiv(h[m].im[c] - cen * xo[m].im[c], hal, inv);
                    nx.re[c] = a.first ? tr : T(2) * tr - po[m].re[c];
                    nx.im[c] = a.first ? ti : T(2) * ti - po[m].im[c];
                }
                st(a.next + o, nx);
                if (MODE == MODE_DIRECT) {
                    const Pk<T> br = ld(a.bra + o);
#pragma unroll
                    for (int c = 0; c < C; ++c)
                        acc0[m][c].x += (double)br.re[c] * nx.re[c] + (double)br.im[c] * nx.im[c];
                } else {
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        const Pk<T> &x = xo[m];
                        doubling_sums<T>(acc0[m][c].x, acc1[m][c].x, x.re[c], x.im[c], nx.re[c], nx.im[c], a.exact_sums);
                    }
                }
            }
        }
        // this tile's partial sums: [tile][even | odd][ncol]
        cta_column_sums_at<MU, C>(acc0, mp, ncol, smem, a.partial + (size_t)tile * ncol * 2);
        if (MODE == MODE_DOUBLING)
            cta_column_sums_at<MU, C>(acc1, mp, ncol, smem, a.partial + (size_t)tile * ncol * 2 + ncol);
    }
}

// Per tile: Re sum_rows conj(bra) x per column (mu_0 = Re<S B, B> of the
// nonorthogonal path), laid out as batch_step_kernel's MODE_DIRECT partials.
template <int MU>
__global__ void __launch_bounds__(256) batch_dot_kernel(const BatchArgs<double> a, const double2 *x) {
    extern __shared__ double2 smem[];
    const RowMap mp = a.mp;
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const int ncol = mp.U;
    for (int64_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        double2 acc[MU][1];
#pragma unroll
        for (int m = 0; m < MU; ++m) acc[m][0] = make_double2(0., 0.);
        for (int64_t row = a.tr0[tile] + g; row < a.tr1[tile]; row += mp.gpc) {
#pragma unroll
            for (int m = 0; m < MU; ++m) {
                const int u = lane + m * mp.G;
                if (u < mp.U) {
                    const size_t o = (size_t)row * mp.U + u;
                    const double2 br = a.bra[o], xv = x[o];
                    acc[m][0].x += br.x * xv.x + br.y * xv.y;
                }
            }
        }
        cta_column_sums_at<MU, 1>(acc, mp, ncol, smem, a.partial + (size_t)tile * ncol * 2);
    }
}

// Per instance: combine its tiles' partial sums in tile order, write moments.
template <int MODE>
__global__ void batch_finalize_kernel(const double2 *partial, const int *seg_tile0, int ncol, int bcols,
                                      double *mu, int64_t length, int64_t kmom) {
    const int s = blockIdx.x;
    const int t0 = seg_tile0[s], t1 = seg_tile0[s + 1];
    double *mus = mu + (size_t)s * length * bcols;
    for (int j = threadIdx.x; j < bcols; j += blockDim.x) {
        double se = 0., so = 0.;
        for (int t = t0; t < t1; ++t) {
            se += partial[(size_t)t * ncol * 2 + j].x;
            if (MODE == MODE_DOUBLING) so += partial[(size_t)t * ncol * 2 + ncol + j].x;
        }
        if (MODE == MODE_DIRECT) {
            mus[(size_t)kmom * bcols + j] = se;
        } else if (kmom == 0) {
            mus[j] = se;
            if (length > 1) mus[(size_t)bcols + j] = so;
        } else {
            const double mu0 = mus[j], mu1 = mus[(size_t)bcols + j];
            if (2 * kmom < length) mus[(size_t)(2 * kmom) * bcols + j] = 2. * se - mu0;
            if (2 * kmom + 1 < length) mus[(size_t)(2 * kmom + 1) * bcols + j] = 2. * so - mu1;
        }
    }
}

__global__ void offset_csr_kernel(const int *ptr, const int *idx, int64_t n, int64_t nnz, int row_off, int nnz_off,
                                  int *gptr, int *gidx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x)
        gidx[nnz_off + i] = idx[i] + row_off;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        gptr[row_off + r] = ptr[r] + nnz_off;
}
__global__ void offset_ell_kernel(const int *idx, int64_t m, int row_off, int *gidx, int64_t goff) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        gidx[goff + i] = idx[i] + row_off;
}

}  // namespace

struct kmsd_batch_s {
    int64_t ninst = 0, n = 0, nnz = 0;
    std::vector<int64_t> row_off, nnz_off;
    std::vector<kmsd_csr_s *> parts;
    int precision = KMSD_FP64;
    kmsd_csr_s G;  // global block-diagonal operator (owns its arrays)
    Tiles tiles;
    DevBuf dcenter, dhalf, ta, tb, bra, partial, tilemem;
    std::vector<double> last_center, last_half;
    // graph cache: (input, mu, b, length, flags, tile_rows) -> executable graph
    std::map<std::tuple<const void *, const void *, int64_t, int64_t, int, int64_t>, cudaGraphExec_t> graphs;
    int64_t kernels_per_graph = 0;
    cudaStream_t cap = nullptr;  // capture stream
    // Nonorthogonal instances: the block-diagonal H (any storage form) and a
    // metric over the block-diagonal S, segmented by instance.
    kmsd_csr_s *gh = nullptr;
    kmsd_metric_s *gm = nullptr;
    double rtol = 1e-10, atol = 0.;
    int maxiter = 1000;
    DevBuf hx, t1, status, report;
    int64_t general_kernels = 0;  // host-side kernels recorded in the nonorthogonal graph
};

namespace {

int build_tiles(kmsd_batch_s *bt, int64_t tile_rows) {
    std::vector<int> seg, first(bt->ninst + 1);
    std::vector<int64_t> r0, r1;
    for (int64_t s = 0; s < bt->ninst; ++s) {
        first[s] = (int)seg.size();
        for (int64_t r = bt->row_off[s]; r < bt->row_off[s + 1]; r += tile_rows) {
            seg.push_back((int)s);
            r0.push_back(r);
            r1.push_back(std::min(r + tile_rows, bt->row_off[s + 1]));
        }
    }
    first[bt->ninst] = (int)seg.size();
    const int64_t nt = (int64_t)seg.size();
    const size_t bytes = nt * (sizeof(int) + 2 * sizeof(int64_t)) + (bt->ninst + 1) * sizeof(int) + 256;
    if (bt->tilemem.ensure(bytes)) return KMSD_ECUDA;
    char *p = bt->tilemem.as<char>();
    bt->tiles.r0 = reinterpret_cast<int64_t *>(p);
    bt->tiles.r1 = bt->tiles.r0 + nt;
    bt->tiles.seg = reinterpret_cast<int *>(bt->tiles.r1 + nt);
    bt->tiles.seg_tile0 = bt->tiles.seg + nt;
    KMSD_CUDA(cudaMemcpy(bt->tiles.r0, r0.data(), nt * sizeof(int64_t), cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemcpy(bt->tiles.r1, r1.data(), nt * sizeof(int64_t), cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemcpy(bt->tiles.seg, seg.data(), nt * sizeof(int), cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemcpy(bt->tiles.seg_tile0, first.data(), (bt->ninst + 1) * sizeof(int), cudaMemcpyHostToDevice));
    bt->tiles.ntiles = nt;
    bt->tiles.tile_rows = tile_rows;
    for (auto &kv : bt->graphs) cudaGraphExecDestroy(kv.second);
    bt->graphs.clear();
    return KMSD_OK;
}

template <class T, int MU, int MODE>
int launch_batch_step(kmsd_batch_s *bt, BatchArgs<T> &a, cudaStream_t s) {
    const size_t sm = reduce_smem(a.mp, Unit<T>::C);
    const bool ell = a.E.w > 0;
    const void *kern = ell ? (const void *)batch_step_kernel<T, MU, MODE, HSRC_ELL>
                           : (const void *)batch_step_kernel<T, MU, MODE, HSRC_CSR>;
    int per_sm = 0;
    KMSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, sm));
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(a.ntiles, (int64_t)sm_count() * std::max(per_sm, 1)));
    if (ell) batch_step_kernel<T, MU, MODE, HSRC_ELL><<<grid, kThreads, sm, s>>>(a);
    else batch_step_kernel<T, MU, MODE, HSRC_CSR><<<grid, kThreads, sm, s>>>(a);
    return KMSD_OK;
}

template <class T, int MU>
int record(kmsd_batch_s *bt, const double2 *B, double *mu, int64_t b, int64_t length, bool doubling,
           cudaStream_t s, int64_t *kernels) {
    using V = typename Unit<T>::vec;
    constexpr int C = Unit<T>::C;
    const int64_t n = bt->n;
    const int U = (int)((b + C - 1) / C);
    const RowMap mp = make_map(U, kThreads);
    const int ncol = U * C;
    V *ta = bt->ta.as<V>(), *tb = bt->tb.as<V>();
    BatchArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.mp = mp;
    if constexpr (C == 2) {
        a.H = bt->G.view32();
        a.E = bt->G.ell32();
    } else {
        a.H = bt->G.view64();
        a.E = bt->G.ell64();
    }
    a.tseg = bt->tiles.seg;
    a.tr0 = bt->tiles.r0;
    a.tr1 = bt->tiles.r1;
    a.ntiles = bt->tiles.ntiles;
    a.center = bt->dcenter.as<double>();
    a.half = bt->dhalf.as<double>();
    a.partial = bt->partial.as<double2>();
    int64_t k_count = 0;
    const V *t0;
    if (C == 2) {
        const int64_t total = n * U;
        const int eg = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16));
        to_f32_kernel<<<eg, 256, 0, s>>>(B, reinterpret_cast<float4 *>(tb), n, (int)b, U);
        ++k_count;
        if (!doubling) {
            to_f32_kernel<<<eg, 256, 0, s>>>(B, reinterpret_cast<float4 *>(bt->bra.as<V>()), n, (int)b, U);
            ++k_count;
        }
        t0 = tb;
        a.bra = bt->bra.as<V>();
    } else {
        t0 = reinterpret_cast<const V *>(B);
        a.bra = reinterpret_cast<const V *>(B);
    }
    const int64_t steps = length == 1 ? 1 : doubling ? (length + 1) / 2 : length - 1;
    const V *curr = t0, *prev = nullptr;
    V *second = C == 2 ? nullptr : tb;
    for (int64_t k = 1; k <= steps; ++k) {
        V *next = k == 1 ? ta : (k == 2 && second != nullptr) ? second : const_cast<V *>(prev);
        a.curr = curr;
        a.prev = prev;
        a.next = next;
        a.first = k == 1;
        int rc;
        if (k == 1 || doubling) {
            a.exact_sums = !doubling;
            rc = launch_batch_step<T, MU, MODE_DOUBLING>(bt, a, s);
            batch_finalize_kernel<MODE_DOUBLING><<<(int)bt->ninst, 128, 0, s>>>(
                a.partial, bt->tiles.seg_tile0, ncol, (int)b, mu, length, k - 1);
        } else {
            rc = launch_batch_step<T, MU, MODE_DIRECT>(bt, a, s);
            batch_finalize_kernel<MODE_DIRECT><<<(int)bt->ninst, 128, 0, s>>>(a.partial, bt->tiles.seg_tile0, ncol,
                                                                              (int)b, mu, length, k);
        }
        if (rc) return rc;
        k_count += 2;
        prev = curr;
        curr = next;
    }
    *kernels = k_count;
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

template <class T, int MU, int MODE, int HSRC>
void launch_tiles(const BatchArgs<T> &a, int64_t ntiles, cudaStream_t s) {
    const size_t sm = reduce_smem(a.mp, Unit<T>::C);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_step_kernel<T, MU, MODE, HSRC>, kThreads, sm) !=
        cudaSuccess)
        per_sm = 1;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)sm_count() * std::max(per_sm, 1)));
    batch_step_kernel<T, MU, MODE, HSRC><<<grid, kThreads, sm, s>>>(a);
}

// Nonorthogonal batch (FP64): per step one SpMM of the block-diagonal H, one
// segmented PCG over every instance's S (one CG per instance and column),
// and one tile step kernel on the solved operand; mu_k = Re<S B, T_k> per
// instance (Engine::moments, cpp/native.cpp:590-609, for each instance).
// Everything the nonorthogonal sequence allocates, done before any capture.
int prepare_general(kmsd_batch_s *bt, const double2 *B, int64_t b, cudaStream_t s) {
    const size_t vb = (size_t)bt->n * b * sizeof(double2);
    if (bt->ta.ensure(vb) || bt->tb.ensure(vb) || bt->bra.ensure(vb) || bt->hx.ensure(vb) || bt->t1.ensure(vb) ||
        bt->partial.ensure((size_t)bt->tiles.ntiles * b * 2 * sizeof(double2) + 256) ||
        bt->status.ensure(4 * sizeof(int)) || bt->report.ensure(sizeof(FailReportFull)))
        return KMSD_ECUDA;
    return bt->gm->prepare_dev(b);
}

// The launches of a nonorthogonal moments call (recorded into a graph, or
// run as they are); the status word is read by the caller.
template <int MU>
int record_general(kmsd_batch_s *bt, const double2 *B, double *mu, int64_t b, int64_t length, cudaStream_t s) {
    const RowMap mp = make_map((int)b, kThreads);
    const int ncol = (int)b;
    int *status = bt->status.as<int>();
    KMSD_CUDA(cudaMemsetAsync(status, 0, 4 * sizeof(int), s));
    double2 *ta = bt->ta.as<double2>(), *tb = bt->tb.as<double2>(), *sb = bt->bra.as<double2>();
    double2 *hx = bt->hx.as<double2>(), *t1 = bt->t1.as<double2>();
    BatchArgs<double> a;
    std::memset(&a, 0, sizeof(a));
    a.mp = mp;
    a.tseg = bt->tiles.seg;
    a.tr0 = bt->tiles.r0;
    a.tr1 = bt->tiles.r1;
    a.ntiles = bt->tiles.ntiles;
    a.center = bt->dcenter.as<double>();
    a.half = bt->dhalf.as<double>();
    a.partial = bt->partial.as<double2>();
    a.bra = sb;
    a.hx = hx;
    int rc = spmm64(bt->gm->S, B, sb, b, s);  // S B, the bra of every moment
    if (rc) return rc;
    {
        const size_t sm = reduce_smem(mp, 1);
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(a.ntiles, (int64_t)sm_count() * 4));
        batch_dot_kernel<MU><<<grid, kThreads, sm, s>>>(a, B);
        batch_finalize_kernel<MODE_DIRECT><<<(int)bt->ninst, 128, 0, s>>>(a.partial, bt->tiles.seg_tile0, ncol,
                                                                          (int)b, mu, length, 0);
        count_launch(2);
    }
    const double2 *curr = B, *prev = nullptr;
    for (int64_t k = 1; k < length; ++k) {
        double2 *next = k == 1 ? ta : k == 2 ? tb : const_cast<double2 *>(prev);
        if ((rc = spmm64(bt->gh, curr, t1, b, s))) return rc;
        if ((rc = bt->gm->solve_dev(t1, hx, b, bt->rtol, bt->atol, bt->maxiter, s, status, bt->report.p)))
            return rc;
        a.curr = curr;
        a.prev = prev;
        a.next = next;
        a.first = k == 1;
        launch_tiles<double, MU, MODE_DIRECT, HSRC_SOLVED>(a, a.ntiles, s);
        batch_finalize_kernel<MODE_DIRECT><<<(int)bt->ninst, 128, 0, s>>>(a.partial, bt->tiles.seg_tile0, ncol,
                                                                          (int)b, mu, length, k);
        count_launch(2);
        prev = curr;
        curr = next;
    }
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

// A failed solve of any instance fails the call with the reference's message.
int general_status(kmsd_batch_s *bt, cudaStream_t s) {
    int st[4];
    KMSD_CUDA(cudaMemcpyAsync(st, bt->status.as<int>(), sizeof(st), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaStreamSynchronize(s));
    if (st[0] != 0) {
        FailReportFull fr;
        KMSD_CUDA(cudaMemcpy(&fr, bt->report.p, sizeof(fr), cudaMemcpyDeviceToHost));
        switch (fr.head.reason) {
            case 3: return fail(KMSD_EINVAL, "metric RHS must be finite");
            case 2:
                return fail(KMSD_EMETRIC,
                            "S solve solution is nonfinite or not representable in complex128 after rescaling");
            case 1: return fail(KMSD_EMETRIC, "PCG non-positive/complex curvature breakdown");
            default: return fail(KMSD_EMETRIC, "S solve failed true-residual acceptance");
        }
    }
    return KMSD_OK;
}

template <class T>
int run_batch(kmsd_batch_s *bt, const double2 *B, double *mu, int64_t b, int64_t length, bool doubling,
              cudaStream_t s, bool use_graph) {
    constexpr int C = Unit<T>::C;
    const int U = (int)((b + C - 1) / C);
    const RowMap mp = make_map(U, kThreads);
    const int mu_n = mu_for(mp);
    if (!mu_n) return fail(KMSD_EINVAL, "too many columns for one batch call");
    using V = typename Unit<T>::vec;
    const size_t vb = (size_t)bt->n * U * sizeof(V);
    const void *before[4] = {bt->ta.p, bt->tb.p, bt->bra.p, bt->partial.p};
    if (bt->ta.ensure(vb) || bt->tb.ensure(vb) || (C == 2 && !doubling && bt->bra.ensure(vb)) ||
        bt->partial.ensure((size_t)bt->tiles.ntiles * U * C * 2 * sizeof(double2) + 256))
        return KMSD_ECUDA;
    const void *after[4] = {bt->ta.p, bt->tb.p, bt->bra.p, bt->partial.p};
    if (!std::equal(before, before + 4, after)) {  // recorded graphs point at the old buffers
        for (auto &kv : bt->graphs) cudaGraphExecDestroy(kv.second);
        bt->graphs.clear();
    }
    auto rec = [&](int64_t *k) -> int {
        switch (mu_n) {
            case 1: return record<T, 1>(bt, B, mu, b, length, doubling, s, k);
            case 2: return record<T, 2>(bt, B, mu, b, length, doubling, s, k);
        }
        return fail(KMSD_EINVAL, "too many columns for one batch call");
    };
    if (!use_graph) {
        int64_t k = 0;
        int rc = rec(&k);
        if (!rc) count_launch(k);
        return rc;
    }
    const auto key = std::make_tuple((const void *)B, (const void *)mu, b, length, (int)doubling, bt->tiles.tile_rows);
    auto it = bt->graphs.find(key);
    if (it == bt->graphs.end()) {
        // Capture on a private stream (the legacy default stream cannot be
        // captured); the graph is launched on the caller's stream.
        cudaGraph_t graph;
        if (!bt->cap) KMSD_CUDA(cudaStreamCreateWithFlags(&bt->cap, cudaStreamNonBlocking));
        KMSD_CUDA(cudaStreamSynchronize(s));
        KMSD_CUDA(cudaStreamBeginCapture(bt->cap, cudaStreamCaptureModeThreadLocal));
        int64_t k = 0;
        int rc;
        {
            cudaStream_t caller = s;
            s = bt->cap;
            rc = rec(&k);
            s = caller;
        }
        cudaGraph_t g2 = nullptr;
        const cudaError_t e = cudaStreamEndCapture(bt->cap, &g2);
        if (rc) {
            if (g2) cudaGraphDestroy(g2);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (batch moments)");
        graph = g2;
        cudaGraphExec_t exec;
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate (batch moments)");
        it = bt->graphs.emplace(key, exec).first;
        bt->kernels_per_graph = k;
    }
    KMSD_CUDA(cudaGraphLaunch(it->second, s));
    count_launch(bt->kernels_per_graph);
    return KMSD_OK;
}

int batch_call(kmsd_batch_s *bt, const void *b_in, double *mu, int64_t b, int64_t length, const double *center,
               const double *half, int flags, cudaStream_t s, bool use_graph) {
    if (!bt || !b_in || !mu || b < 1) return fail(KMSD_EINVAL, "expected nonempty finite (N,batch) array");
    if (length < 1) return fail(KMSD_EINVAL, "moment count must be positive");
    if (!center || !half) return fail(KMSD_EINVAL, "per-instance spectral window required");
    for (int64_t i = 0; i < bt->ninst; ++i)
        if (length > 1 && !(half[i] > 0)) return fail(KMSD_EINVAL, "spectral half-width must be positive");
    const bool doubling = (flags & KMSD_MOMENTS_DOUBLING) != 0;
    // per-instance window: uploaded only when it changed (a graph reads the buffers)
    if (bt->last_center.size() != (size_t)bt->ninst ||
        !std::equal(center, center + bt->ninst, bt->last_center.begin()) ||
        !std::equal(half, half + bt->ninst, bt->last_half.begin())) {
        std::vector<double> h1(half, half + bt->ninst);
        for (auto &x : h1)
            if (!(x > 0)) x = 1.;  // a single moment never applies the operator
        KMSD_CUDA(cudaMemcpyAsync(bt->dcenter.p, center, bt->ninst * sizeof(double), cudaMemcpyHostToDevice, s));
        KMSD_CUDA(cudaMemcpyAsync(bt->dhalf.p, h1.data(), bt->ninst * sizeof(double), cudaMemcpyHostToDevice, s));
        KMSD_CUDA(cudaStreamSynchronize(s));
        bt->last_center.assign(center, center + bt->ninst);
        bt->last_half.assign(half, half + bt->ninst);
    }
    if (bt->gm) {
        if (doubling) return fail(KMSD_EINVAL, "moment doubling needs an orthogonal basis (S = I)");
        const RowMap mp = make_map((int)b, kThreads);
        const int m = mu_for(mp);
        if (!m || b > 256) return fail(KMSD_EINVAL, "too many columns for one batch call");
        const double2 *B = static_cast<const double2 *>(b_in);
        const void *before[3] = {bt->ta.p, bt->partial.p, bt->hx.p};
        int rc = prepare_general(bt, B, b, s);
        if (rc) return rc;
        const void *after[3] = {bt->ta.p, bt->partial.p, bt->hx.p};
        if (!std::equal(before, before + 3, after)) {  // recorded graphs point at the old buffers
            for (auto &kv : bt->graphs) cudaGraphExecDestroy(kv.second);
            bt->graphs.clear();
        }
        auto rec = [&](cudaStream_t st) {
            return m == 1 ? record_general<1>(bt, B, mu, b, length, st) : record_general<2>(bt, B, mu, b, length, st);
        };
        if (!use_graph) {
            if ((rc = rec(s))) return rc;
            return general_status(bt, s);
        }
        // one graph for the whole call: every solve is a WHILE node inside it
        const auto key = std::make_tuple((const void *)B, (const void *)mu, b, length, 2, bt->tiles.tile_rows);
        auto it = bt->graphs.find(key);
        if (it == bt->graphs.end()) {
            if (!bt->cap) KMSD_CUDA(cudaStreamCreateWithFlags(&bt->cap, cudaStreamNonBlocking));
            // the SpMMs size this thread's reduction buffers on first use:
            // run them once outside the capture
            if ((rc = spmm64(bt->gm->S, B, bt->t1.as<double2>(), b, s))) return rc;
            if ((rc = spmm64(bt->gh, B, bt->t1.as<double2>(), b, s))) return rc;
            KMSD_CUDA(cudaStreamSynchronize(s));
            cudaGraph_t g = nullptr;
            int64_t recorded = 0;
            {
                CountOff off;
                KMSD_CUDA(cudaStreamBeginCapture(bt->cap, cudaStreamCaptureModeThreadLocal));
                rc = rec(bt->cap);
                const cudaError_t e = cudaStreamEndCapture(bt->cap, &g);
                recorded = off.recorded();
                if (rc) {
                    if (g) cudaGraphDestroy(g);
                    return rc;
                }
                if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (nonorthogonal batch)");
            }
            cudaGraphExec_t exec;
            const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate (nonorthogonal batch)");
            it = bt->graphs.emplace(key, exec).first;
            bt->general_kernels = recorded;
        }
        KMSD_CUDA(cudaGraphLaunch(it->second, s));
        count_launch(bt->general_kernels);  // the PCG loop bodies are counted on the device
        return general_status(bt, s);
    }
    int rc = bt->precision == KMSD_MIXED
                 ? run_batch<float>(bt, static_cast<const double2 *>(b_in), mu, b, length, doubling, s, use_graph)
                 : run_batch<double>(bt, static_cast<const double2 *>(b_in), mu, b, length, doubling, s, use_graph);
    if (rc) return rc;
    KMSD_CUDA(cudaStreamSynchronize(s));
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

}  // namespace

extern "C" {

int kmsd_batch_create(int64_t ninst, const kmsd_csr *H, int precision, int64_t tile_rows, kmsd_batch *out) {
    if (ninst < 1 || !H || !out) return fail(KMSD_EINVAL, "invalid batch");
    if (precision != KMSD_FP64 && precision != KMSD_MIXED) return fail(KMSD_EINVAL, "invalid batch precision");
    auto *bt = new kmsd_batch_s();
    bt->ninst = ninst;
    bt->precision = precision;
    bt->row_off.assign(ninst + 1, 0);
    bt->nnz_off.assign(ninst + 1, 0);
    bool cplx = false;
    int w = H[0] ? H[0]->ell_w : 0;
    for (int64_t i = 0; i < ninst; ++i) {
        if (!H[i]) {
            delete bt;
            return fail(KMSD_EINVAL, "invalid batch");
        }
        if (precision == KMSD_MIXED && H[i]->ensure_f32()) {
            delete bt;
            return KMSD_ECUDA;
        }
        bt->parts.push_back(H[i]);
        bt->row_off[i + 1] = bt->row_off[i] + H[i]->n;
        bt->nnz_off[i + 1] = bt->nnz_off[i] + H[i]->nnz;
        cplx = cplx || H[i]->complex_values;
        if (H[i]->ell_w != w) w = 0;
    }
    bt->n = bt->row_off[ninst];
    bt->nnz = bt->nnz_off[ninst];
    if (bt->n >= INT32_MAX || bt->nnz >= INT32_MAX) {
        delete bt;
        return fail(KMSD_EINVAL, "batch too large for 32-bit indices");
    }
    kmsd_csr_s &G = bt->G;
    G.n = bt->n;
    G.nnz = bt->nnz;
    G.complex_values = cplx;
    auto mal = [](void **p, size_t bytes) -> int {
        KMSD_CUDA(cudaMalloc(p, std::max<size_t>(bytes, 16)));
        return KMSD_OK;
    };
    int rc = mal((void **)&G.ptr, (G.n + 1) * sizeof(int));
    if (!rc) rc = mal((void **)&G.idx, G.nnz * sizeof(int));
    if (!rc) rc = mal((void **)&G.re64, G.nnz * sizeof(double));
    if (!rc && cplx) rc = mal((void **)&G.im64, G.nnz * sizeof(double));
    if (!rc && precision == KMSD_MIXED) rc = mal((void **)&G.re32, G.nnz * sizeof(float));
    if (!rc && precision == KMSD_MIXED && cplx) rc = mal((void **)&G.im32, G.nnz * sizeof(float));
    if (!rc && w > 0) {
        rc = mal((void **)&G.ell_idx, G.n * w * sizeof(int));
        if (!rc) rc = mal((void **)&G.ell_re64, G.n * w * sizeof(double));
        if (!rc && cplx) rc = mal((void **)&G.ell_im64, G.n * w * sizeof(double));
        if (!rc && precision == KMSD_MIXED) rc = mal((void **)&G.ell_re32, G.n * w * sizeof(float));
        if (!rc && precision == KMSD_MIXED && cplx) rc = mal((void **)&G.ell_im32, G.n * w * sizeof(float));
        if (!rc) G.ell_w = w;
    }
    for (int64_t i = 0; i < ninst && !rc; ++i) {
        const kmsd_csr_s *A = H[i];
        const int ro = (int)bt->row_off[i], no = (int)bt->nnz_off[i];
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((std::max(A->nnz, A->n + 1) + 255) / 256, 4096));
        offset_csr_kernel<<<grid, 256>>>(A->ptr, A->idx, A->n, A->nnz, ro, no, G.ptr, G.idx);
        count_launch();
        auto cp = [&](void *dst, const void *src, size_t bytes) -> int {
            if (bytes) KMSD_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToDevice));
            return KMSD_OK;
        };
        rc = cp(G.re64 + no, A->re64, A->nnz * sizeof(double));
        if (!rc && cplx) {
            if (A->complex_values) rc = cp(G.im64 + no, A->im64, A->nnz * sizeof(double));
            else KMSD_CUDA(cudaMemset(G.im64 + no, 0, A->nnz * sizeof(double)));
        }
        if (!rc && precision == KMSD_MIXED) rc = cp(G.re32 + no, A->re32, A->nnz * sizeof(float));
        if (!rc && precision == KMSD_MIXED && cplx) {
            if (A->complex_values) rc = cp(G.im32 + no, A->im32, A->nnz * sizeof(float));
            else KMSD_CUDA(cudaMemset(G.im32 + no, 0, A->nnz * sizeof(float)));
        }
        if (!rc && G.ell_w > 0) {
            const int64_t m = A->n * w;
            offset_ell_kernel<<<grid, 256>>>(A->ell_idx, m, ro, G.ell_idx, (int64_t)ro * w);
            count_launch();
            rc = cp(G.ell_re64 + (int64_t)ro * w, A->ell_re64, m * sizeof(double));
            if (!rc && cplx) {
                if (A->complex_values) rc = cp(G.ell_im64 + (int64_t)ro * w, A->ell_im64, m * sizeof(double));
                else KMSD_CUDA(cudaMemset(G.ell_im64 + (int64_t)ro * w, 0, m * sizeof(double)));
            }
            if (!rc && precision == KMSD_MIXED) rc = cp(G.ell_re32 + (int64_t)ro * w, A->ell_re32, m * sizeof(float));
            if (!rc && precision == KMSD_MIXED && cplx) {
                if (A->complex_values) rc = cp(G.ell_im32 + (int64_t)ro * w, A->ell_im32, m * sizeof(float));
                else KMSD_CUDA(cudaMemset(G.ell_im32 + (int64_t)ro * w, 0, m * sizeof(float)));
            }
        }
    }
    if (!rc) {
        const int last = (int)bt->nnz;  // closing row pointer
        rc = cudaMemcpy(G.ptr + G.n, &last, sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess ? KMSD_OK
                                                                                               : KMSD_ECUDA;
    }
    if (!rc && (bt->dcenter.ensure(ninst * sizeof(double)) || bt->dhalf.ensure(ninst * sizeof(double))))
        rc = KMSD_ECUDA;
    if (!rc) rc = build_tiles(bt, tile_rows > 0 ? tile_rows : 2048);
    if (!rc) rc = cudaDeviceSynchronize() == cudaSuccess ? KMSD_OK : KMSD_ECUDA;
    if (rc) {
        kmsd_batch_destroy(bt);
        return rc;
    }
    *out = bt;
    return KMSD_OK;
}

void kmsd_batch_destroy(kmsd_batch bt) {
    if (!bt) return;
    for (auto &kv : bt->graphs) cudaGraphExecDestroy(kv.second);
    if (bt->cap) cudaStreamDestroy(bt->cap);
    kmsd_csr_s &G = bt->G;
    for (void *p : {(void *)G.ptr, (void *)G.idx, (void *)G.re64, (void *)G.im64, (void *)G.re32, (void *)G.im32,
                    (void *)G.ell_idx, (void *)G.ell_re64, (void *)G.ell_im64, (void *)G.ell_re32,
                    (void *)G.ell_im32})
        cudaFree(p);
    G = kmsd_csr_s();
    for (DevBuf *d : {&bt->dcenter, &bt->dhalf, &bt->ta, &bt->tb, &bt->bra, &bt->partial, &bt->tilemem, &bt->hx,
                      &bt->t1, &bt->status, &bt->report})
        d->release();
    delete bt;
}

int kmsd_batch_attach_metric(kmsd_batch bt, kmsd_csr h, kmsd_metric m, double rtol, double atol, int maxiter) {
    if (!bt || !h || !m) return fail(KMSD_EINVAL, "invalid batch metric");
    if (h->n != bt->n || m->n != bt->n)
        return fail(KMSD_EINVAL, "the block-diagonal H and S must have the batch's rows");
    if (bt->precision != KMSD_FP64) return fail(KMSD_EINVAL, "a batch with a metric runs in FP64");
    if (!(rtol >= 0) || !(atol >= 0) || !std::isfinite(rtol) || !std::isfinite(atol) || maxiter < 1)
        return fail(KMSD_EINVAL, "invalid metric RHS shape/tolerances");
    const int rc = kmsd_metric_set_segments(m, bt->ninst, bt->row_off.data());
    if (rc) return rc;
    bt->gh = h;
    bt->gm = m;
    bt->rtol = rtol;
    bt->atol = atol;
    bt->maxiter = maxiter;
    return KMSD_OK;
}

int kmsd_batch_rows(kmsd_batch bt, int64_t *offsets) {
    if (!bt || !offsets) return fail(KMSD_EINVAL, "invalid batch");
    std::copy(bt->row_off.begin(), bt->row_off.end(), offsets);
    return KMSD_OK;
}

int kmsd_batch_moments(kmsd_batch bt, const void *b_in, double *mu, int64_t b, int64_t length, const double *center,
                       const double *half, int flags, int use_graph, void *stream) {
    return batch_call(bt, b_in, mu, b, length, center, half, flags, static_cast<cudaStream_t>(stream),
                      use_graph != 0);
}

int kmsd_batch_set_tile_rows(kmsd_batch bt, int64_t tile_rows) {
    if (!bt || tile_rows < 1) return fail(KMSD_EINVAL, "invalid batch");
    return build_tiles(bt, tile_rows);
}

int kmsd_batch_tune(kmsd_batch bt, const void *b_in, double *mu, int64_t b, int64_t length, const double *center,
                    const double *half, int flags, int64_t *chosen_tile_rows, void *stream) {
    if (!bt) return fail(KMSD_EINVAL, "invalid batch");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t candidates[] = {512, 1024, 2048, 4096, 8192};
    double best = 1e300;
    int64_t best_rows = bt->tiles.tile_rows;
    cudaEvent_t e0, e1;
    KMSD_CUDA(cudaEventCreate(&e0));
    KMSD_CUDA(cudaEventCreate(&e1));
    for (int64_t rows : candidates) {
        int rc = build_tiles(bt, rows);
        if (!rc) rc = batch_call(bt, b_in, mu, b, length, center, half, flags, s, false);  // warm
        if (rc) return rc;
        KMSD_CUDA(cudaEventRecord(e0, s));
        rc = batch_call(bt, b_in, mu, b, length, center, half, flags, s, false);
        if (rc) return rc;
        KMSD_CUDA(cudaEventRecord(e1, s));
        KMSD_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        KMSD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            best_rows = rows;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc = build_tiles(bt, best_rows);
    if (rc) return rc;
    if (chosen_tile_rows) *chosen_tile_rows = best_rows;
    return KMSD_OK;
}

}  // extern "C"
