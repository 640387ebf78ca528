// Tile-pipelined Chebyshev moment step for the identity metric over a real
// ELL operator of width 4 or 8 (the lattice Hamiltonians of the precision
// form): the same arithmetic as cheb_step_kernel in MODE_DOUBLING /
// MODE_DIRECT, with the streaming operands moved by the copy engine.
//
// Each CTA is persistent and owns the row tiles blockIdx.x, blockIdx.x +
// gridDim.x, ...  One producer warp copies a tile's T_{k-1} rows, T_{k-2}
// rows (and the bra rows for direct moments) and its ELL indices and values
// into a ring of KMSD_TILE_STAGES shared-memory stages with cp.async.bulk;
// a full/empty mbarrier pair per stage hands stages between the producer and
// the eight consumer warps.  The consumers read x and prev from shared
// memory, take the neighbour rows that fall inside the tile from shared memory
// too, and gather only the others from global memory (L2), so the DRAM
// stream in flight per SM is set by the ring depth instead of by registers.
//
// Every wait is bounded by wall-clock time (KMSD_TILE_WAIT_NS); a wait that
// runs out sets *timeout and the CTA drains the copies it issued before it
// returns, so the host reports an error instead of the GPU hanging.
#pragma once

#include "kmsd_kernels.cuh"

namespace kmsd {

#ifndef KMSD_TILE
#define KMSD_TILE 1  // use the tile kernel where it applies
#endif
#ifndef KMSD_TILE_STAGES
#define KMSD_TILE_STAGES 3
#endif
#ifndef KMSD_TILE_RING
#define KMSD_TILE_RING 101376  // bytes of the stage ring of one CTA (two CTAs per SM)
#endif
#ifndef KMSD_TILE_MINB
#define KMSD_TILE_MINB 2  // resident CTAs per SM asked of the compiler
#endif
#ifndef KMSD_TILE_F32_DOUBLING
#define KMSD_TILE_F32_DOUBLING 0  // the mixed doubling step keeps the paired-row step kernel
#endif
#ifndef KMSD_TILE_RB
#define KMSD_TILE_RB 2  // rows of a row group whose neighbour loads are issued together
#endif
#ifndef KMSD_TILE_WAIT_NS
#define KMSD_TILE_WAIT_NS 2000000000ull  // 2 s
#endif

// Vector loads of a row's ELL entries from the stage and 32-bit in-tile
// offsets: on the 4.19M-site honeycomb at R=64 this took FP64 direct moments
// from 7.92e10 to 8.91e10, FP64 doubling from 1.60e11 to 1.95e11 and mixed
// direct from 1.78e11 to 1.93e11 orbital*moment*vec/s (one GPU, 1800 MHz).
#ifndef KMSD_TILE_VEC
#define KMSD_TILE_VEC 1
#endif

// W ELL values of one row from the stage (16-byte aligned: the values region
// starts on a 16-byte boundary and a row holds 4 or 8 entries).
template <class T, int W>
__device__ __forceinline__ void tile_vals(const T *p, T (&v)[W]) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int k = 0; k < W / 4; ++k) {
            const float4 q = reinterpret_cast<const float4 *>(p)[k];
            v[4 * k] = q.x; v[4 * k + 1] = q.y; v[4 * k + 2] = q.z; v[4 * k + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < W / 2; ++k) {
            const double2 q = reinterpret_cast<const double2 *>(p)[k];
            v[2 * k] = q.x; v[2 * k + 1] = q.y;
        }
    }
}

constexpr int kTileConsumers = 256;                    // eight consumer warps
constexpr int kTileThreads = kTileConsumers + 32;      // plus one producer warp
constexpr int kTileMaxRows = 256;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Waits until the phase of `bar` with parity `parity` has completed; false
// when KMSD_TILE_WAIT_NS pass first.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (unsigned it = 1; it < (1u << 30); ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255u) == 0 && global_ns() - t0 > KMSD_TILE_WAIT_NS) return false;
    }
    return false;
}
// Bulk global -> shared copy completing on `bar` (both addresses 16-byte
// aligned, bytes a multiple of 16).  No multicast.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void async_proxy_fence() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Shared-memory layout of one stage for tiles of `tr` rows of `U` units.
struct TileLayout {
    int tr;       // rows per tile
    int w;        // ELL width
    int nvec;     // vector operands per stage: x, prev (+ bra)
    int vbytes;   // one vector operand
    int ibytes;   // ELL indices
    int rbytes;   // ELL values
    int sbytes;   // one stage, rounded to 128 bytes
};
__host__ __device__ inline TileLayout tile_layout(int tr, int U, int w, int nvec, int val_size) {
    TileLayout L;
    L.tr = tr;
    L.w = w;
    L.nvec = nvec;
    L.vbytes = tr * U * 16;
    L.ibytes = tr * w * 4;
    L.rbytes = tr * w * val_size;
    L.sbytes = (L.vbytes * nvec + L.ibytes + L.rbytes + 127) / 128 * 128;
    return L;
}
// Bytes of dynamic shared memory of a launch: the stages, or the epilogue's
// scratch if that is larger.
__host__ inline size_t tile_smem(const TileLayout &L, const RowMap &mp, int C) {
    const size_t ring = (size_t)L.sbytes * KMSD_TILE_STAGES;
    const size_t red = ((size_t)mp.gpc * mp.U * C + kTileThreads + 2 * 512) * sizeof(double2);
    return ring > red ? ring : red;
}

// MODE_DOUBLING or MODE_DIRECT; W = 4 or 8 (real ELL values).
template <class T, int MODE, int W>
__global__ void __launch_bounds__(kTileThreads, KMSD_TILE_MINB)
    cheb_tile_kernel(const StepArgs<T> a, const TileLayout L, int *timeout) {
    using V = typename Unit<T>::vec;
    constexpr int C = Unit<T>::C;
    constexpr int NS = KMSD_TILE_STAGES;
    extern __shared__ __align__(128) unsigned char tsm[];
    __shared__ uint64_t full[NS], empty[NS];
    __shared__ int abort_flag;
    const RowMap mp = a.mp;
    const int U = mp.U;
    const int tid = threadIdx.x;
    const int TR = L.tr;
    const int64_t n = a.n;
    const bool has_prev = !a.first;
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kTileConsumers / 32);
        }
        abort_flag = 0;
        mbar_init_fence();
    }
    __syncthreads();
    const int64_t ntiles = (n + TR - 1) / TR;
    const int64_t mine = (int64_t)blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    double2 acc0[1][C], acc1[1][C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        acc0[0][c] = make_double2(0., 0.);
        acc1[0][c] = make_double2(0., 0.);
    }
    if (tid >= kTileConsumers) {
        // ---------------------------------------------------------- producer
        if (tid == kTileConsumers) {
            int64_t issued = 0;
            for (int64_t i = 0; i < mine; ++i) {
                const int s = (int)(i % NS);
                if (i >= NS && !mbar_wait(&empty[s], (unsigned)((i / NS - 1) & 1))) {
                    atomicOr(timeout, 1);
                    abort_flag = 1;
                    break;
                }
                if (*(volatile int *)&abort_flag) break;
                async_proxy_fence();
                const int64_t t0 = ((int64_t)blockIdx.x + i * gridDim.x) * TR;
                const int rows = (int)(n - t0 < TR ? n - t0 : TR);
                unsigned char *stg = tsm + (size_t)s * L.sbytes;
                const unsigned vb = (unsigned)rows * U * 16, ib = (unsigned)rows * W * 4,
                               rb = (unsigned)rows * W * (unsigned)sizeof(T);
                const unsigned tx = vb * (1 + (has_prev ? 1 : 0) + (MODE == MODE_DIRECT ? 1 : 0)) + ib + rb;
                mbar_expect_tx(&full[s], tx);
                bulk_load(stg, a.curr + t0 * U, vb, &full[s]);
                if (has_prev) bulk_load(stg + L.vbytes, a.prev + t0 * U, vb, &full[s]);
                if (MODE == MODE_DIRECT) bulk_load(stg + 2 * L.vbytes, a.bra + t0 * U, vb, &full[s]);
                unsigned char *ell = stg + (size_t)L.vbytes * L.nvec;
                bulk_load(ell, a.E.idx + t0 * W, ib, &full[s]);
                bulk_load(ell + L.ibytes, a.E.re + t0 * W, rb, &full[s]);
                ++issued;
            }
            // copies issued and not yet seen complete by a consumer: wait for
            // them (bounded) so no copy lands after the CTA has exited
            for (int64_t j = issued > NS ? issued - NS : 0; j < issued; ++j)
                if (!mbar_wait(&full[j % NS], (unsigned)((j / NS) & 1))) atomicOr(timeout, 1);
        }
    } else {
        // ---------------------------------------------------------- consumers
        const int g = tid / mp.G, u = tid % mp.G;
        const T cen = (T)a.center, hal = (T)a.half;
        for (int64_t i = 0; i < mine; ++i) {
            const int s = (int)(i % NS);
            if (!mbar_wait(&full[s], (unsigned)((i / NS) & 1))) {
                atomicOr(timeout, 1);
                abort_flag = 1;
                break;
            }
            const int64_t t0 = ((int64_t)blockIdx.x + i * gridDim.x) * TR;
            const int rows = (int)(n - t0 < TR ? n - t0 : TR);
            const unsigned char *stg = tsm + (size_t)s * L.sbytes;
            const V *xs = reinterpret_cast<const V *>(stg);
            const V *ps = reinterpret_cast<const V *>(stg + L.vbytes);
            const V *bs = reinterpret_cast<const V *>(stg + 2 * L.vbytes);
            const int *is = reinterpret_cast<const int *>(stg + (size_t)L.vbytes * L.nvec);
            const T *vs = reinterpret_cast<const T *>(stg + (size_t)L.vbytes * L.nvec + L.ibytes);
            if (g < mp.gpc && u < U) {
                // KMSD_TILE_RB rows of this row group at a time: all their
                // neighbour loads are issued before any of them is computed
                constexpr int RB = KMSD_TILE_RB;
                const int t0i = (int)t0;  // rows and column indices are int32
                for (int r = g; r < rows; r += RB * mp.gpc) {
                    Pk<T> xg[RB][W];
#pragma unroll
                    for (int q = 0; q < RB; ++q) {
                        const int rr = r + q * mp.gpc;
                        if (rr >= rows) break;
                        if (KMSD_TILE_VEC) {
                            // the row's indices as int4 (16-byte aligned in the stage);
                            // in-tile offsets in 32 bits
                            int cols[W];
#pragma unroll
                            for (int j4 = 0; j4 < W / 4; ++j4) {
                                const int4 c4 = reinterpret_cast<const int4 *>(is + rr * W)[j4];
                                cols[4 * j4] = c4.x;
                                cols[4 * j4 + 1] = c4.y;
                                cols[4 * j4 + 2] = c4.z;
                                cols[4 * j4 + 3] = c4.w;
                            }
#pragma unroll
                            for (int j = 0; j < W; ++j) {
                                const unsigned lc = (unsigned)(cols[j] - t0i);
                                xg[q][j] = lc < (unsigned)rows ? ld(xs + (int)lc * U + u)
                                                               : ldg(a.curr + (int64_t)cols[j] * U + u);
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < W; ++j) {
                                const int col = is[rr * W + j];
                                const int64_t lc = (int64_t)col - t0;
                                const V *src = (uint64_t)lc < (uint64_t)rows ? xs + lc * U + u
                                                                              : a.curr + (int64_t)col * U + u;
                                xg[q][j] = ld(src);
                            }
                        }
                    }
#pragma unroll
                    for (int q = 0; q < RB; ++q) {
                        const int rr = r + q * mp.gpc;
                        if (rr >= rows) break;
                        Pk<T> h = pk_zero<T>();
                        if (KMSD_TILE_VEC) {
                            T vals[W];
                            tile_vals<T, W>(vs + rr * W, vals);
#pragma unroll
                            for (int j = 0; j < W; ++j) cmac_real(h, vals[j], xg[q][j]);
                        } else {
#pragma unroll
                            for (int j = 0; j < W; ++j) cmac_real(h, vs[rr * W + j], xg[q][j]);
                        }
                        const Pk<T> x = ld(xs + rr * U + u);
                        const Pk<T> pv = has_prev ? ld(ps + rr * U + u) : pk_zero<T>();
                        Pk<T> nx;
#pragma unroll
                        for (int c = 0; c < C; ++c) {
                            const T tr_ = rdiv(h.re[c] - cen * x.re[c], hal, a.inv_half);
                            const T ti_ = rdiv(h.im[c] - cen * x.im[c], hal, a.inv_half);
                            nx.re[c] = has_prev ? T(2) * tr_ - pv.re[c] : tr_;
                            nx.im[c] = has_prev ? T(2) * ti_ - pv.im[c] : ti_;
                        }
                        st(a.next + (t0 + rr) * U + u, nx);
                        if (MODE == MODE_DIRECT) {
                            const Pk<T> br = ld(bs + rr * U + u);
#pragma unroll
                            for (int c = 0; c < C; ++c)
                                acc0[0][c].x += (double)br.re[c] * (double)nx.re[c] +
                                                (double)br.im[c] * (double)nx.im[c];
                        } else {
#pragma unroll
                            for (int c = 0; c < C; ++c)
                                doubling_sums<T>(acc0[0][c].x, acc1[0][c].x, x.re[c], x.im[c], nx.re[c], nx.im[c], a.exact_sums);
                        }
                    }
                }
            }
            __syncwarp();
            if ((tid & 31) == 0) mbar_arrive(&empty[s]);
            if (*(volatile int *)&abort_flag) break;
        }
    }
    __syncthreads();  // every copy has landed: the ring is free for the epilogue
    const int ncol = U * C;
    double2 *red = reinterpret_cast<double2 *>(tsm);
    double2 *tot = red + (size_t)mp.gpc * U * C;
    double2 *outbuf = tot + kTileThreads;
    double *even = reinterpret_cast<double *>(outbuf + 512);
    cta_column_sums<1, C>(acc0, mp, ncol, red, a.partial);
    if (MODE == MODE_DOUBLING) cta_column_sums<1, C>(acc1, mp, ncol, red, a.partial + (size_t)gridDim.x * ncol);
    if (!last_cta(a.ticket)) return;
    final_column_sums(a.partial, gridDim.x, ncol, tot, outbuf);
    if (MODE == MODE_DIRECT) {
        for (int j = threadIdx.x; j < a.bcols; j += blockDim.x) a.mu[(size_t)a.kmom * a.bcols + j] = outbuf[j].x;
        return;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < ncol; j += blockDim.x) even[j] = outbuf[j].x;
    __syncthreads();
    final_column_sums(a.partial + (size_t)gridDim.x * ncol, gridDim.x, ncol, tot, outbuf);
    const int64_t nn = a.kmom;
    for (int j = threadIdx.x; j < a.bcols; j += blockDim.x) {
        const double se = even[j], so = outbuf[j].x;
        if (nn == 0) {
            a.mu[j] = se;
            if (a.mlen > 1) a.mu[(size_t)a.bcols + j] = so;
        } else {
            const double mu0 = a.mu[j], mu1 = a.mu[(size_t)a.bcols + j];
            if (2 * nn < a.mlen) a.mu[(size_t)(2 * nn) * a.bcols + j] = 2. * se - mu0;
            if (2 * nn + 1 < a.mlen) a.mu[(size_t)(2 * nn + 1) * a.bcols + j] = 2. * so - mu1;
        }
    }
}

}  // namespace kmsd
