// Two Chebyshev steps per launch for the doubling moments over a real ELL
// operator of width 4 or 8 (the lattice Hamiltonians of the precision form):
//   phase A of tile t:  X = T_{k+1} = 2 Ht T_k - T_{k-1}        (rows of t)
//   phase B of tile t:  Y = T_{k+2} = 2 Ht T_{k+1} - T_k         (rows of t)
// with the four sums <T_k,T_k>, <T_k,T_{k+1}>, <T_{k+1},T_{k+1}>,
// <T_{k+1},T_{k+2}> giving moments 2k..2k+3.  Phase B needs T_{k+1} on the
// rows its rows couple to, so a tile publishes an epoch-tagged flag after its
// phase A, and phase B of tile t waits for the flags of the tiles
// [dep_lo[t], dep_hi[t]] (from the operator's pattern).  T_{k+1} and the
// T_k rows re-read in phase B are recent and come from L2: per two steps the
// DRAM traffic is T_{k-1} and T_k read, T_{k+1} and T_{k+2} written — four
// vector passes instead of six.
//
// Scheduling: CTA c owns tiles c, c + G, c + 2G, ... and runs A(t0), A(t1),
// B(t0), A(t2), B(t1), ..., B(t_last).  A never waits.  B(t) waits only on
// tiles within W = G - 1 of t; a tile whose pattern reaches further (the
// periodic wrap of a lattice) is deferred until every tile's phase A is done.
// With every CTA resident (a cooperative launch), the phase A of wave i
// completes once the B phases of wave i - 2 have, which wait only on waves up
// to i - 1, so by induction every wait ends.  Each wait is also bounded by
// wall-clock time: a wait that runs out sets *timeout, and the kernel
// continues without hanging (the host then reports an error).
#pragma once

#include "kmsd_tile.cuh"

namespace kmsd {

#ifndef KMSD_WAVE
#define KMSD_WAVE 1  // two steps per launch for the doubling moments where it applies
#endif
#ifndef KMSD_WAVE_TILE_ROWS
#define KMSD_WAVE_TILE_ROWS 64
#endif
#ifndef KMSD_WAVE_MINB
#define KMSD_WAVE_MINB 2
#endif

template <class T> struct WaveArgs {
    using V = typename Unit<T>::vec;
    int64_t n;
    RowMap mp;
    EllView<T> E;
    const V *curr;   // T_k
    const V *prev;   // T_{k-1}; nullptr when k == 0
    V *X;            // T_{k+1}
    V *next;         // T_{k+2}; may alias prev
    double center, half;
    T inv_half;
    int tr;          // rows per tile
    int64_t ntiles;
    const int *dep_lo, *dep_hi;  // per tile: range of tiles its rows couple to
    int *flags;      // per tile: epoch of its finished phase A
    unsigned *a_done;  // phase-A tiles finished in this launch
    int epoch;
    int *timeout;
    double2 *partial;  // 4 x [grid][ncol]
    Ticket *ticket;
    double *mu;
    int64_t kmom;    // moments 2 kmom .. 2 kmom + 3
    int64_t mlen;
    int bcols;
};

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One step on row r for this lane's unit: nx = 2 (Ht x) - p (or Ht x when p is
// absent), stored to dst; adds |x|^2 and Re<x, nx> to the sums.  CG: src was
// written earlier in this launch, so it is read through L2 (bypassing L1).
template <class T, int PF, bool CG>
__device__ __forceinline__ void wave_rows(const WaveArgs<T> &a, const typename Unit<T>::vec *src,
                                          const typename Unit<T>::vec *pv, typename Unit<T>::vec *dst, int64_t r,
                                          bool has_p, int u, double2 (&e)[Unit<T>::C], double2 (&o)[Unit<T>::C]) {
    using V = typename Unit<T>::vec;
    constexpr int C = Unit<T>::C;
    const int U = a.mp.U;
    EllRow<T, PF> er;
    ell_row_load<T, PF>(a.E, r, er);
    const size_t o_ = (size_t)r * U + u;
    const Pk<T> x = CG ? ldcg_pk(src + o_) : ld(src + o_);
    const Pk<T> p = has_p ? ld(pv + o_) : pk_zero<T>();
    Pk<T> h = pk_zero<T>();
#pragma unroll
    for (int q = 0; q < PF; ++q) {
        const int col[4] = {er.idx[q].x, er.idx[q].y, er.idx[q].z, er.idx[q].w};
        Pk<T> xs[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) xs[j] = CG ? ldcg_pk(src + (size_t)col[j] * U + u) : ldg(src + (size_t)col[j] * U + u);
#pragma unroll
        for (int j = 0; j < 4; ++j) cmac_real(h, er.val[q][j], xs[j]);
    }
    const T cen = (T)a.center, hal = (T)a.half;
    Pk<T> nx;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const T tr_ = rdiv(h.re[c] - cen * x.re[c], hal, a.inv_half);
        const T ti_ = rdiv(h.im[c] - cen * x.im[c], hal, a.inv_half);
        nx.re[c] = has_p ? T(2) * tr_ - p.re[c] : tr_;
        nx.im[c] = has_p ? T(2) * ti_ - p.im[c] : ti_;
        e[c].x += (double)x.re[c] * (double)x.re[c] + (double)x.im[c] * (double)x.im[c];
        o[c].x += (double)x.re[c] * (double)nx.re[c] + (double)x.im[c] * (double)nx.im[c];
    }
    st(dst + o_, nx);
}

template <class T, int PF>
__global__ void __launch_bounds__(256, KMSD_WAVE_MINB) cheb_wave_kernel(const WaveArgs<T> a) {
    constexpr int C = Unit<T>::C;
    extern __shared__ double2 smem[];
    __shared__ int stop;
    const RowMap mp = a.mp;
    const int g = threadIdx.x / mp.G, u = threadIdx.x % mp.G;
    const int G = gridDim.x;
    const int64_t W = G - 1;
    double2 e0[C], o0[C], e1[C], o1[C];
#pragma unroll
    for (int c = 0; c < C; ++c) e0[c] = o0[c] = e1[c] = o1[c] = make_double2(0., 0.);
    // a wait that ran out earlier in this call: skip every wait (the call fails)
    if (threadIdx.x == 0) stop = *(volatile int *)a.timeout != 0;
    __syncthreads();
    const int64_t mine = (int64_t)blockIdx.x < a.ntiles ? (a.ntiles - 1 - blockIdx.x) / G + 1 : 0;
    auto tile_of = [&](int64_t i) { return (int64_t)blockIdx.x + i * G; };
    auto is_far = [&](int64_t t) { return (int64_t)a.dep_hi[t] - t > W || t - (int64_t)a.dep_lo[t] > W; };
    auto rows_of = [&](int64_t t) { return (int)(a.n - t * a.tr < a.tr ? a.n - t * a.tr : a.tr); };

    auto phase_a = [&](int64_t t) {
        const int64_t r0 = t * a.tr;
        const int rows = rows_of(t);
        if (u < mp.U)
            for (int r = g; r < rows; r += mp.gpc)
                wave_rows<T, PF, false>(a, a.curr, a.prev, a.X, r0 + r, a.prev != nullptr, u, e0, o0);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            st_release(a.flags + t, a.epoch);
            atomicAdd(a.a_done, 1u);
        }
    };
    // waits (warp 0) for the phase-A flags of tiles [lo, hi], or for every
    // tile when `all`; bounded by wall-clock time
    auto wait_for = [&](int64_t lo, int64_t hi, bool all) {
        if (threadIdx.x < 32) {
            const uint64_t t0 = global_ns();
            bool ok = false;
            for (unsigned it = 0; it < (1u << 30) && !ok; ++it) {
                bool mine_ok = true;
                if (all) {
                    if (threadIdx.x == 0) {
                        unsigned v;
                        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a.a_done) : "memory");
                        mine_ok = v >= (unsigned)a.ntiles;
                    }
                } else {
                    for (int64_t q = lo + threadIdx.x; q <= hi; q += 32) mine_ok &= ld_acquire(a.flags + q) == a.epoch;
                }
                ok = __all_sync(0xffffffffu, mine_ok);
                if (!ok && (it & 63u) == 63u && global_ns() - t0 > KMSD_TILE_WAIT_NS) break;
            }
            if (!ok && threadIdx.x == 0) {
                atomicOr(a.timeout, 1);
                stop = 1;
            }
        }
        __syncthreads();
    };
    auto phase_b = [&](int64_t t) {
        const int64_t r0 = t * a.tr;
        const int rows = rows_of(t);
        if (u < mp.U)
            for (int r = g; r < rows; r += mp.gpc)
                wave_rows<T, PF, true>(a, a.X, a.curr, a.next, r0 + r, true, u, e1, o1);
    };

    for (int64_t i = 0; i < mine; ++i) {
        phase_a(tile_of(i));
        if (i >= 1 && !stop) {
            const int64_t t = tile_of(i - 1);
            if (!is_far(t)) {
                wait_for(a.dep_lo[t], a.dep_hi[t], false);
                if (!stop) phase_b(t);
            }
        }
    }
    if (mine > 0 && !stop) {
        const int64_t t = tile_of(mine - 1);
        if (!is_far(t)) {
            wait_for(a.dep_lo[t], a.dep_hi[t], false);
            if (!stop) phase_b(t);
        }
    }
    bool any_far = false;
    for (int64_t i = 0; i < mine; ++i) any_far |= is_far(tile_of(i));
    if (any_far && !stop) {
        wait_for(0, 0, true);
        for (int64_t i = 0; i < mine && !stop; ++i)
            if (is_far(tile_of(i))) phase_b(tile_of(i));
    }
    // ---- the four column sums, then the moments from the last CTA
    const int ncol = mp.U * C;
    double2 acc[4][1][C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        acc[0][0][c] = e0[c];
        acc[1][0][c] = o0[c];
        acc[2][0][c] = e1[c];
        acc[3][0][c] = o1[c];
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) cta_column_sums<1, C>(acc[s], mp, ncol, smem, a.partial + (size_t)s * G * ncol);
    if (!last_cta(a.ticket)) return;
    if (threadIdx.x == 0) *a.a_done = 0;  // every CTA has passed its waits
    double2 *tot = smem;
    __shared__ double2 outbuf[512];
    __shared__ double sums[4][256];
    for (int s = 0; s < 4; ++s) {
        final_column_sums(a.partial + (size_t)s * G * ncol, G, ncol, tot, outbuf);
        for (int j = threadIdx.x; j < ncol && j < 256; j += blockDim.x) sums[s][j] = outbuf[j].x;
        __syncthreads();
    }
    const int64_t nn = a.kmom;
    for (int j = threadIdx.x; j < a.bcols; j += blockDim.x) {
        const double se0 = sums[0][j], so0 = sums[1][j], se1 = sums[2][j], so1 = sums[3][j];
        double mu0, mu1;
        if (nn == 0) {
            mu0 = se0;
            mu1 = so0;
            a.mu[j] = se0;
            if (a.mlen > 1) a.mu[(size_t)a.bcols + j] = so0;
        } else {
            mu0 = a.mu[j];
            mu1 = a.mu[(size_t)a.bcols + j];
            if (2 * nn < a.mlen) a.mu[(size_t)(2 * nn) * a.bcols + j] = 2. * se0 - mu0;
            if (2 * nn + 1 < a.mlen) a.mu[(size_t)(2 * nn + 1) * a.bcols + j] = 2. * so0 - mu1;
        }
        if (2 * nn + 2 < a.mlen) a.mu[(size_t)(2 * nn + 2) * a.bcols + j] = 2. * se1 - mu0;
        if (2 * nn + 3 < a.mlen) a.mu[(size_t)(2 * nn + 3) * a.bcols + j] = 2. * so1 - mu1;
    }
}

}  // namespace kmsd
