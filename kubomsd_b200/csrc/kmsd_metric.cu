// Overlap metric of the B200 engine: batched preconditioned CG for S^-1 and
// the Chebyshev (Clenshaw) sampler for S^-1/2.
//
// The solve follows Metric::solve of the reference (cpp/native.cpp:313-452)
// column by column: RHS scaling by safe_j = max_i max(|Re|,|Im|)
// (native.cpp:320-329), thresholds max(rtol*||q_j||, atol/safe_j) (333),
// curvature breakdown test (363-371), fixed / adaptive true-residual refresh
// with restart (379-402), beta with the rz == 0 guard (405-408), final
// true-residual acceptance (413-423) and representability checks (424-444).
// All columns advance together; per-column scalars (alpha, beta, active, ...)
// live on the device and are updated by the last CTA of each reduction
// kernel, so an iteration needs no host round trip.  The host polls a single
// halt word once per chunk of iterations to stop launching.
#include <math.h>
#include <float.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <type_traits>
#include <utility>

#include "kmsd.h"
#include "kmsd_impl.h"
#include "kmsd_kernels.cuh"

using namespace kmsd;

namespace {

struct ColPtr {
    double *safe, *bn, *thr, *rz, *alpha, *beta, *rn, *tn, *newrz, *gap, *relative, *residual;
    double *rsn;  // residual norm at the last (re)start (mixed form)
    int *active, *restart, *brk, *conv, *finp, *fino;
    long long *iters;
    int *flags;  // [0] halt, [1] check, [2] nonfinite rhs, [3] breakdown, [4] n_active
};
constexpr int kDoubles = 13, kInts = 6;
size_t col_bytes(int64_t b) { return (size_t)b * (kDoubles * 8 + kInts * 4 + 8) + 64; }
ColPtr col_ptr(void *base, int64_t b) {
    ColPtr c;
    double *d = static_cast<double *>(base);
    double **dp[kDoubles] = {&c.safe, &c.bn, &c.thr, &c.rz, &c.alpha, &c.beta,       &c.rn,
                             &c.tn,   &c.newrz, &c.gap, &c.relative, &c.residual, &c.rsn};
    for (int i = 0; i < kDoubles; ++i) *dp[i] = d + (size_t)i * b;
    long long *l = reinterpret_cast<long long *>(d + (size_t)kDoubles * b);
    c.iters = l;
    int *ip = reinterpret_cast<int *>(l + b);
    int **ipp[kInts] = {&c.active, &c.restart, &c.brk, &c.conv, &c.finp, &c.fino};
    for (int i = 0; i < kInts; ++i) *ipp[i] = ip + (size_t)i * b;
    c.flags = ip + (size_t)kInts * b;
    return c;
}
// device counters: [0] refreshes [1] checks [2] restarts [3] iterations sum; [4] max relative (double bits)
struct Counters {
    long long v[4];
    double max_rel;
};

struct Pre {
    const double *diag;
    const int *bstart;
    const int64_t *foff;
    const double2 *factors;
    int ub;    // uniform block size, or 0: rows and factors are then found without lookups
    int real;  // every block inverse is real
};

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, den = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    }
    const double r = b.x / b.y, den = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}

// Rows of preconditioner block bi: [r0, r0+m).
template <int MAXB>
__device__ __forceinline__ void block_rows(const Pre &P, int64_t bi, int64_t &r0, int &m) {
    if (MAXB == 1) {
        r0 = bi;
        m = 1;
    } else if (P.ub) {
        r0 = bi * P.ub;
        m = P.ub;
    } else {
        r0 = P.bstart[bi];
        m = P.bstart[bi + 1] - (int)r0;
    }
}

// Blocks of at most this many rows apply the preconditioner as the dense
// Hermitian inverse (L L^H)^-1, formed once on the host from the Cholesky
// factor; larger blocks keep the two triangular substitutions.
#ifndef KMSD_BLOCK_INVERSE
#define KMSD_BLOCK_INVERSE 8
#endif

// z = M^-1 r on one block for one column: the diagonal and block-Jacobi
// preconditioners of native.cpp:259-277.  The reference runs the forward and
// back substitution with the lower Cholesky factor L; blocks of up to
// KMSD_BLOCK_INVERSE rows multiply by the stored inverse instead, which is
// the same operator without divisions or a dependent chain of rows.
template <int MAXB>
__device__ __forceinline__ void precond(const Pre &P, int64_t bi, int64_t r0, int m, const double2 (&r)[MAXB],
                                        double2 (&z)[MAXB]) {
    if (MAXB == 1) {
        const double d = P.diag[r0];
        z[0] = make_double2(r[0].x / d, r[0].y / d);
        return;
    }
    const double2 *L = P.factors + (P.ub ? bi * P.ub * P.ub : P.foff[bi]);
    if constexpr (MAXB <= KMSD_BLOCK_INVERSE) {
        // L holds the inverse, row-major; real when every factor is
        if (P.real) {
            const double *Q = reinterpret_cast<const double *>(L);
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                if (i < m) {
                    double2 v = make_double2(0., 0.);
#pragma unroll
                    for (int k = 0; k < MAXB; ++k) {
                        if (k < m) {
                            const double q = __ldg(Q + 2 * (i * m + k));
                            v.x += q * r[k].x;
                            v.y += q * r[k].y;
                        }
                    }
                    z[i] = v;
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                if (i < m) {
                    double2 v = make_double2(0., 0.);
#pragma unroll
                    for (int k = 0; k < MAXB; ++k) {
                        if (k < m) {
                            const double2 q = __ldg(L + i * m + k);
                            v.x += q.x * r[k].x - q.y * r[k].y;
                            v.y += q.x * r[k].y + q.y * r[k].x;
                        }
                    }
                    z[i] = v;
                }
            }
        }
    } else {
        // Large blocks: plain loops (registers spill to local memory).
        for (int i = 0; i < m; ++i) {
            double2 v = r[i];
            for (int k = 0; k < i; ++k) {
                const double2 l = L[i * m + k];
                v.x -= l.x * z[k].x - l.y * z[k].y;
                v.y -= l.x * z[k].y + l.y * z[k].x;
            }
            z[i] = cdiv(v, L[i * m + i]);
        }
        for (int i = m - 1; i >= 0; --i) {
            double2 v = z[i];
            for (int k = i + 1; k < m; ++k) {
                const double2 l = L[k * m + i];
                v.x -= l.x * z[k].x + l.y * z[k].y;
                v.y -= l.x * z[k].y - l.y * z[k].x;
            }
            const double2 d = L[i * m + i];
            z[i] = cdiv(v, make_double2(d.x, -d.y));
        }
    }
}

// CTAs per SM the block kernels (init, update, restart) are compiled for
// when blocks have at most four rows; they are latency bound, so occupancy
// is traded against a few bytes of register spill.
#ifndef KMSD_PCG_MINB4
#define KMSD_PCG_MINB4 4
#endif
#define KMSD_PCG_MINB(maxb) ((maxb) <= 4 ? KMSD_PCG_MINB4 : 1)

#define ZERO_ACC(acc)                                   \
    _Pragma("unroll") for (int m_ = 0; m_ < MU; ++m_) { \
        acc[m_][0] = make_double2(0., 0.);              \
    }

// ---- segments
// A segmented solve treats the operator as block-diagonal over nseg row
// ranges (independent systems: the instances of a ragged batch) and runs one
// CG per (segment, column), with its column state at index s * b + j.  Every
// CTA belongs to one segment and walks only that segment's rows, 4x4 block
// rows and preconditioner blocks; column sums combine per segment (its own
// tickets and level-2 rows), and a last-segment ticket aggregates the flags
// that every segment contributes to.  A plain solve is the SEG = false
// instantiation: one segment over the whole grid.
struct SegView {
    int nseg;
    const int *cta_seg;   // [grid] segment of each CTA
    const int *cta0;      // [nseg + 1] first CTA of each segment
    const int64_t *row0;  // [nseg + 1] first row
    const int64_t *blk0;  // [nseg + 1] first preconditioner block
    const int *tk0;       // [nseg + 1] first ticket of each segment; tk0[nseg]: the last-segment ticket
    const int *l2;        // [nseg] first level-2 partial row, counted after the grid's rows
    int *segn;            // [nseg] active columns of each segment
    int *segchk;          // [nseg] a true-residual check is due in the segment
};

// This CTA's segment, its place among the segment's CTAs, and the segment's
// rows [r0, r1) and preconditioner blocks [b0, b1).
struct Ctx {
    int s, lc, nct;
    int64_t r0, r1, b0, b1;
};

template <bool SEG>
__device__ __forceinline__ Ctx seg_ctx(const SegView &sv, int64_t n, int64_t nb) {
    if constexpr (!SEG) {
        return Ctx{0, (int)blockIdx.x, (int)gridDim.x, 0, n, 0, nb};
    } else {
        const int s = sv.cta_seg[blockIdx.x], c0 = sv.cta0[s];
        return Ctx{s, (int)blockIdx.x - c0, sv.cta0[s + 1] - c0, sv.row0[s], sv.row0[s + 1], sv.blk0[s],
                   sv.blk0[s + 1]};
    }
}

// True in the CTA that holds this segment's column sums in out.
template <bool SEG>
__device__ __forceinline__ bool seg_sums(double2 *partial, int ncol, Ticket *tk, double2 *smem, double2 *out,
                                         const SegView &sv, const Ctx &x) {
    if constexpr (!SEG) {
        return tree_column_sums(partial, ncol, tk, smem, out);
    } else {
        return range_column_sums(partial, ncol, (int)blockIdx.x - x.lc, x.nct, x.lc, tk + sv.tk0[x.s],
                                 partial + (size_t)(gridDim.x + sv.l2[x.s]) * ncol, smem, out);
    }
}
template <bool SEG>
__device__ __forceinline__ bool seg_max(double *partial, int ncol, Ticket *tk, double *out, const SegView &sv,
                                        const Ctx &x) {
    if constexpr (!SEG) {
        return tree_column_max(partial, ncol, tk, out);
    } else {
        return range_column_max(partial, ncol, (int)blockIdx.x - x.lc, x.nct, x.lc, tk + sv.tk0[x.s],
                                partial + (size_t)(gridDim.x + sv.l2[x.s]) * ncol, out);
    }
}

// Called by every CTA that closed its segment: true in the last of them (a
// plain solve has one segment, so there it is always true).
template <bool SEG>
__device__ __forceinline__ bool last_segment(Ticket *tk, const SegView &sv) {
    if constexpr (!SEG) {
        return true;
    } else {
        return arrive_last(tk + sv.tk0[sv.nseg], sv.nseg);
    }
}

// Sum of segn over the segments (thread 0's result), in segment order.
__device__ __forceinline__ int total_active(const SegView &sv) {
    int t = 0;
    for (int s = 0; s < sv.nseg; ++s) t += __ldcg(sv.segn + s);
    return t;
}

// ---- column scale: safe_j = max_i max(|Re|,|Im|), nonfinite detection
template <int MU, bool SEG>
__global__ void __launch_bounds__(256) pcg_scale_kernel(const double2 *B, int64_t n, RowMap mp, ColPtr c,
                                                        double *partial, Ticket *tk, SegView sv) {
    extern __shared__ double2 smem2[];
    double *smem = reinterpret_cast<double *>(smem2);
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const Ctx x = seg_ctx<SEG>(sv, n, 0);
    double acc[MU][1];
#pragma unroll
    for (int m = 0; m < MU; ++m) acc[m][0] = 0.;
    bool bad = false;
    for (int64_t row = x.r0 + (int64_t)x.lc * mp.gpc + g; row < x.r1; row += (int64_t)x.nct * mp.gpc) {
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
                const double2 v = B[(size_t)row * mp.U + u];
                bad |= !isfinite(v.x) || !isfinite(v.y);
                acc[m][0] = fmax(acc[m][0], fmax(fabs(v.x), fabs(v.y)));
            }
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(c.flags + 2, 1);
    cta_column_max<MU, 1>(acc, mp, mp.U, smem, partial);
    double *safe = c.safe + (size_t)x.s * mp.U;
    if (seg_max<SEG>(partial, mp.U, tk, safe, sv, x)) {
        __syncthreads();
        for (int j = threadIdx.x; j < mp.U; j += blockDim.x)
            if (safe[j] == 0.) safe[j] = 1.;
    }
}

// ---- init: q = B/safe, r = q, y = 0, z = M^-1 r; sums |q|^2 and Re<r,z>
template <int MU, int MAXB, bool SEG, class W>
__global__ void __launch_bounds__(256, KMSD_PCG_MINB(MAXB))
    pcg_init_kernel(const double2 *B, double2 *q, double2 *y, W *r, W *z, Pre P, int64_t nb, RowMap mp,
                    ColPtr c, double rtol, double atol, double2 *partial, Ticket *tk, SegView sv) {
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const int U = mp.U;
    const Ctx x = seg_ctx<SEG>(sv, 0, nb);
    const size_t cs0 = (size_t)x.s * U;
    double2 acc[MU][1];
    ZERO_ACC(acc);
    for (int64_t bi = x.b0 + (int64_t)x.lc * mp.gpc + g; bi < x.b1; bi += (int64_t)x.nct * mp.gpc) {
        int64_t r0;
        int m;
        block_rows<MAXB>(P, bi, r0, m);
#pragma unroll
        for (int mm = 0; mm < MU; ++mm) {
            const int u = lane + mm * mp.G;
            if (u >= U) continue;
            const double sf = c.safe[cs0 + u];
            double2 rr[MAXB], zz[MAXB];
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                if (i < m) {
                    const size_t o = (size_t)(r0 + i) * U + u;
                    const double2 v = B[o];
                    const double2 qq = make_double2(v.x / sf, v.y / sf);
                    q[o] = qq;
                    stw(r + o, qq);
                    y[o] = make_double2(0., 0.);
                    rr[i] = stored<W>(qq);
                    acc[mm][0].x += qq.x * qq.x + qq.y * qq.y;
                }
            }
            precond<MAXB>(P, bi, r0, m, rr, zz);
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                if (i < m) {
                    stw(z + (size_t)(r0 + i) * U + u, zz[i]);
                    const double2 zs = stored<W>(zz[i]);
                    acc[mm][0].y += rr[i].x * zs.x + rr[i].y * zs.y;
                }
            }
        }
    }
    cta_column_sums<MU, 1>(acc, mp, U, smem, partial);
    __shared__ double2 tot[256];
    if (seg_sums<SEG>(partial, U, tk, smem, tot, sv, x)) {
        __syncthreads();
        const int j = threadIdx.x;
        bool act = false;
        if (j < U) {
            const size_t cj = cs0 + j;
            const double bn = sqrt(tot[j].x);
            const double thr = fmax(rtol * bn, atol / c.safe[cj]);
            act = bn > thr;
            c.bn[cj] = bn;
            c.thr[cj] = thr;
            c.rsn[cj] = bn;
            c.active[cj] = act;
            c.rz[cj] = tot[j].y;
            c.iters[cj] = 0;
            c.brk[cj] = 0;
            c.restart[cj] = 0;
            c.alpha[cj] = 0.;
            c.beta[cj] = 0.;
        }
        const int nact = __syncthreads_count(act);
        if constexpr (SEG) {
            if (threadIdx.x == 0) {
                sv.segn[x.s] = nact;
                sv.segchk[x.s] = 0;
            }
        }
        if (last_segment<SEG>(tk, sv) && threadIdx.x == 0) {
            const int total = SEG ? total_active(sv) : nact;
            c.flags[0] = total == 0;  // halt: nothing to iterate
            c.flags[1] = 0;
            c.flags[3] = 0;
            c.flags[4] = total;
        }
    }
}

// p = active ? z : 0
template <bool SEG, class W>
__global__ void pcg_pinit_kernel(const W *z, W *p, int64_t len, RowMap mp, ColPtr c, SegView sv) {
    if constexpr (!SEG) {
        const int U = mp.U;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
             i += (int64_t)gridDim.x * blockDim.x) {
            const int j = (int)(i % U);
            p[i] = c.active[j] ? z[i] : W{};
        }
    } else {
        const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
        const Ctx x = seg_ctx<SEG>(sv, 0, 0);
        for (int64_t row = x.r0 + (int64_t)x.lc * mp.gpc + g; row < x.r1; row += (int64_t)x.nct * mp.gpc)
            for (int u = lane; u < mp.U; u += mp.G) {
                const size_t o = (size_t)row * mp.U + u;
                p[o] = c.active[(size_t)x.s * mp.U + u] ? z[o] : W{};
            }
    }
}

// Storage form of S in the S products: CSR, or 4x4 blocks with real or
// complex values.
enum { S_CSR = 0, S_BSR_REAL = 1, S_BSR_CPLX = 2 };

// Calls f(row, yv) for every row of rows [x.r0, x.r1) owned by this thread's
// row group, with yv[m] = (S X)[row, unit lane + m*G], from CSR or from 4x4
// blocks (a block row's four rows share every gathered input row).
//
// Small operators (few block rows for the resident row groups) split each
// block row over ks row groups of the CTA: group g takes every ks-th block,
// which divides the chain of dependent gathers by ks, and the partials are
// summed in shared memory in a fixed order before f.  Every thread of the CTA
// calls this when ks > 1 (the split synchronises the CTA); the dynamic shared
// memory then holds split_smem_units(MU) double2.
__host__ __device__ constexpr int split_smem_units(int mu) { return 1024 * mu; }
// CTAs per SM assumed when the split factor is chosen (block rows x ks up to
// the row groups of that many CTAs on every SM).
#ifndef KMSD_SPLIT_CTAS
#define KMSD_SPLIT_CTAS 4
#endif

template <int MU, int SF, class XV, class F>
__device__ __forceinline__ void for_rows_spmv(const CsrView<double> &S, const BsrView<double> &SB, const XV *X,
                                              const Ctx &x, const RowMap &mp, int g, int lane, int ks, F &&f) {
    if (SF != S_CSR && ks > 1) {
        extern __shared__ double2 part_sums[];  // [group][4 rows][MU][G lanes]
        const int spc = mp.gpc / ks, slot = g / ks, part = g % ks;
        const int64_t end = x.r1 / 4;
        for (int64_t base = x.r0 / 4 + (int64_t)x.lc * spc; base < end; base += (int64_t)x.nct * spc) {
            const int64_t I = base + slot;
            Pk<double> acc4[4][MU];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int m = 0; m < MU; ++m) acc4[i][m] = pk_zero<double>();
            if (I < end) gather_block_row<MU, SF == S_BSR_CPLX>(SB, X, I, mp.U, mp.G, lane, acc4, part, ks);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int m = 0; m < MU; ++m)
                    part_sums[((g * 4 + i) * MU + m) * mp.G + lane] = make_double2(acc4[i][m].re[0], acc4[i][m].im[0]);
            __syncthreads();
            if (part == 0 && I < end) {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    Pk<double> yv[MU];
#pragma unroll
                    for (int m = 0; m < MU; ++m) {
                        double re = 0., im = 0.;
                        for (int q = 0; q < ks; ++q) {
                            const double2 v = part_sums[(((g + q) * 4 + i) * MU + m) * mp.G + lane];
                            re += v.x;
                            im += v.y;
                        }
                        yv[m].re[0] = re;
                        yv[m].im[0] = im;
                    }
                    f(4 * I + i, yv);
                }
            }
            __syncthreads();
        }
    } else if constexpr (SF != S_CSR) {
        for (int64_t I = x.r0 / 4 + (int64_t)x.lc * mp.gpc + g; I < x.r1 / 4; I += (int64_t)x.nct * mp.gpc) {
            Pk<double> acc4[4][MU];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int m = 0; m < MU; ++m) acc4[i][m] = pk_zero<double>();
            gather_block_row<MU, SF == S_BSR_CPLX>(SB, X, I, mp.U, mp.G, lane, acc4);
#pragma unroll
            for (int i = 0; i < 4; ++i) f(4 * I + i, acc4[i]);
        }
    } else {
        for (int64_t row = x.r0 + (int64_t)x.lc * mp.gpc + g; row < x.r1; row += (int64_t)x.nct * mp.gpc) {
            Pk<double> yv[MU];
#pragma unroll
            for (int m = 0; m < MU; ++m) yv[m] = pk_zero<double>();
            if constexpr (std::is_same<XV, double2>::value) gather_row<double, MU>(S, X, row, mp.U, mp.G, lane, yv);
            else gather_row_d<MU>(S, X, row, mp.U, mp.G, lane, yv);
            f(row, yv);
        }
    }
}

// Device-driven iterations: the solve is captured with its iterations as a
// WHILE node (`again`) whose body holds an IF node (`check`) around the
// true-residual and restart kernels.  The update kernel's last CTA counts
// the iteration in flags[5] and sets both conditions; the restart kernel's
// last CTA decides `again` after a check; an update that finds the halt
// word stops the loop.  on == 0: iterations driven by the host.
struct Loop {
    int on, maxiter;
    cudaGraphConditionalHandle again, check;
    int has_check;  // the check kernels sit in an IF node driven by `check`
};

// Launch options of the device-driven loop body: KMSD_PCG_PDL chains the
// body's kernels with programmatic dependent launch (a kernel's CTAs are
// scheduled while its predecessor drains and wait in griddepcontrol.wait
// until it has completed); KMSD_PCG_IFNODE = 0 runs the true-residual and
// restart kernels in every iteration (they return at once unless a check is
// due) instead of behind an IF node.
#ifndef KMSD_PCG_PDL
#define KMSD_PCG_PDL 1
#endif
#ifndef KMSD_PCG_IFNODE
#define KMSD_PCG_IFNODE 1
#endif

// Kernels launched inside device-driven loops, counted on the device (the
// host does not see those launches).
__device__ unsigned long long g_loop_launches;

__device__ __forceinline__ void loop_count(const Loop &lp) {
    if (lp.on && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&g_loop_launches, 1ull);
    // (no-ops unless launched as a programmatic dependent)
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// ---- sp = S p, curvature <p, sp>, alpha, breakdown
// CTAs per SM the S-product kernel is compiled for (one unit per lane); 0:
// left to the compiler.
#ifndef KMSD_SPMV_MINB
#define KMSD_SPMV_MINB 4
#endif
#if KMSD_SPMV_MINB > 0
#define KMSD_SPMV_BOUNDS(mu) __launch_bounds__(256, (mu) == 1 ? KMSD_SPMV_MINB : 1)
#else
#define KMSD_SPMV_BOUNDS(mu) __launch_bounds__(256)
#endif

template <int MU, int SF, bool SEG, class W>
__global__ void KMSD_SPMV_BOUNDS(MU)
    pcg_spmv_kernel(CsrView<double> S, BsrView<double> SB, const W *p, W *sp, int64_t n, RowMap mp,
                    ColPtr c, double2 *partial, Ticket *tk, SegView sv, Loop lp, int ks) {
    loop_count(lp);
    if (*(volatile int *)c.flags) return;
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const Ctx x = seg_ctx<SEG>(sv, n, 0);
    double2 acc[MU][1];
    ZERO_ACC(acc);
    for_rows_spmv<MU, SF>(S, SB, p, x, mp, g, lane, ks, [&](int64_t row, const Pk<double>(&yv)[MU]) {
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
                const size_t o = (size_t)row * mp.U + u;
                // <p, S p> from the stored p and the exact FP64 product
                stw(sp + o, make_double2(yv[m].re[0], yv[m].im[0]));
                const double2 xv = ldw(p + o);
                acc[m][0].x += xv.x * yv[m].re[0] + xv.y * yv[m].im[0];
                acc[m][0].y += xv.x * yv[m].im[0] - xv.y * yv[m].re[0];
            }
        }
    });
    cta_column_sums<MU, 1>(acc, mp, mp.U, smem, partial);
    __shared__ double2 tot[256];
    if (seg_sums<SEG>(partial, mp.U, tk, smem, tot, sv, x)) {
        __syncthreads();
        const int j = threadIdx.x;
        bool b = false;
        if (j < mp.U) {
            const size_t cj = (size_t)x.s * mp.U + j;
            const double cr = tot[j].x, ci = tot[j].y;
            const bool act = c.active[cj];
            if (act && (!(cr > 0.) || !isfinite(cr) || !isfinite(ci) || fabs(ci) > 1e-10 * fmax(fabs(cr), DBL_MIN))) {
                c.brk[cj] = 1;
                b = true;
            }
            c.alpha[cj] = act ? c.rz[cj] / cr : 0.;
        }
        const bool any_brk = __syncthreads_or(b);
        if constexpr (!SEG) {
            if (any_brk && threadIdx.x == 0) {
                c.flags[3] = 1;
                c.flags[0] = 1;
            }
        } else {
            // Segments halt together, and only once every CTA of this launch
            // has passed its entry check (a CTA that saw the halt word early
            // would skip its segment's tickets): the last segment raises it.
            if (any_brk && threadIdx.x == 0) c.flags[3] = 1;
            if (last_segment<SEG>(tk, sv) && threadIdx.x == 0 && __ldcg(c.flags + 3)) c.flags[0] = 1;
        }
    }
}

// ---- y += alpha p, r -= alpha sp, z = M^-1 r; sums |r|^2, Re<r,z>
template <int MU, int MAXB, bool SEG, class W>
__global__ void __launch_bounds__(256, KMSD_PCG_MINB(MAXB))
    pcg_update_kernel(double2 *y, W *r, W *z, const W *p, const W *sp, Pre P, int64_t nb,
                      RowMap mp, ColPtr c, int refresh, int interval, int adaptive, double2 *partial, Ticket *tk,
                      SegView sv, Loop lp) {
    loop_count(lp);
    if (*(volatile int *)c.flags) {
        if (lp.on && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(lp.again, 0u);
        return;
    }
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const int U = mp.U;
    const Ctx x = seg_ctx<SEG>(sv, 0, nb);
    const size_t cs0 = (size_t)x.s * U;
    double2 acc[MU][1];
    ZERO_ACC(acc);
    for (int64_t bi = x.b0 + (int64_t)x.lc * mp.gpc + g; bi < x.b1; bi += (int64_t)x.nct * mp.gpc) {
        int64_t r0;
        int m;
        block_rows<MAXB>(P, bi, r0, m);
#pragma unroll
        for (int mm = 0; mm < MU; ++mm) {
            const int u = lane + mm * mp.G;
            if (u >= U) continue;
            const double al = c.alpha[cs0 + u];
            double2 rr[MAXB], zz[MAXB];
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                if (i < m) {
                    const size_t o = (size_t)(r0 + i) * U + u;
                    const double2 pv = ldw(p + o), sv2 = ldw(sp + o);
                    double2 yv = y[o], rv = ldw(r + o);
                    yv.x += pv.x * al;
                    yv.y += pv.y * al;
                    rv.x -= sv2.x * al;
                    rv.y -= sv2.y * al;
                    y[o] = yv;
                    stw(r + o, rv);
                    rr[i] = stored<W>(rv);
                    acc[mm][0].x += rr[i].x * rr[i].x + rr[i].y * rr[i].y;
                }
            }
            precond<MAXB>(P, bi, r0, m, rr, zz);
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                if (i < m) {
                    stw(z + (size_t)(r0 + i) * U + u, zz[i]);
                    const double2 zs = stored<W>(zz[i]);
                    acc[mm][0].y += rr[i].x * zs.x + rr[i].y * zs.y;
                }
            }
        }
    }
    cta_column_sums<MU, 1>(acc, mp, U, smem, partial);
    __shared__ double2 tot[256];
    if (seg_sums<SEG>(partial, U, tk, smem, tot, sv, x)) {
        __syncthreads();
        const int j = threadIdx.x;
        const size_t cj = cs0 + j;
        // Mixed form: complex64 work vectors let the recursive residual drift
        // from the true one by at most ~4e-6 x the residual at the last
        // (re)start.  A column whose drift bound is below a tenth of its
        // threshold stops on its recursive residual with a 10 % margin; any
        // other column that reaches the threshold is checked in FP64 (as the
        // adaptive policy does) and restarted from its true residual.
        constexpr bool kMixed = sizeof(W) == sizeof(float2);
        constexpr double kTrust = 2.5e4, kMargin = .9;
        bool cand = false, cand_mixed = false;
        if (j < U) {
            const int act = c.active[cj];
            c.iters[cj] += act;
            const double rn = sqrt(tot[j].x);
            c.rn[cj] = rn;
            c.newrz[cj] = tot[j].y;
            cand = act && rn <= c.thr[cj];
            if (kMixed) cand_mixed = cand && c.rsn[cj] > kTrust * c.thr[cj];
        }
        const bool candidate = __syncthreads_or(cand);
        const bool candidate_mixed = __syncthreads_or(cand_mixed);
        // in a device-driven loop the iteration index lives in flags[5]
        if (interval > 0) refresh = ((*(volatile int *)(c.flags + 5) + 1) % interval) == 0;
        const bool check = refresh || (adaptive && candidate) || (kMixed && candidate_mixed);
        bool act_now = false;
        if (j < U) {
            if (!check) {
                int act = c.active[cj];
                if (!adaptive) act = act && c.rn[cj] > (kMixed ? kMargin : 1.) * c.thr[cj];
                c.active[cj] = act;
                c.restart[cj] = 0;
                const double rz = c.rz[cj], nrz = c.newrz[cj];
                c.beta[cj] = act ? nrz / (rz != 0. ? rz : 1.) : 0.;
                c.rz[cj] = nrz;
                act_now = act;
            }
        }
        const int nact = __syncthreads_count(act_now);
        if constexpr (SEG) {
            if (threadIdx.x == 0) {
                sv.segchk[x.s] = check;
                if (!check) sv.segn[x.s] = nact;
            }
        }
        if (last_segment<SEG>(tk, sv) && threadIdx.x == 0) {
            if constexpr (!SEG) {
                c.flags[1] = check;
                if (!check) {
                    c.flags[4] = nact;
                    if (nact == 0) c.flags[0] = 1;
                }
            } else {
                int any = 0;
                for (int s = 0; s < sv.nseg; ++s) any |= __ldcg(sv.segchk + s);
                const int total = total_active(sv);
                c.flags[1] = any;
                c.flags[4] = total;
                if (!any && total == 0) c.flags[0] = 1;
            }
            if (lp.on) {
                const int k = c.flags[5] + 1;
                c.flags[5] = k;
                if (lp.has_check) cudaGraphSetConditional(lp.check, c.flags[1] ? 1u : 0u);
                cudaGraphSetConditional(lp.again, (c.flags[0] == 0 && k < lp.maxiter) ? 1u : 0u);
            }
        }
    }
}

// ---- true residual t = q - S y; sums |t|^2 and |t - r|^2; refresh decision
template <int MU, int SF, bool SEG, class W>
__global__ void __launch_bounds__(256)
    pcg_true_residual_kernel(CsrView<double> S, BsrView<double> SB, const double2 *q, const double2 *y,
                             const W *r, W *t, int64_t n, RowMap mp, ColPtr c, int adaptive,
                             double gap_ratio, double2 *partial, Ticket *tk, Counters *cnt, SegView sv, Loop lp,
                             int ks) {
    loop_count(lp);
    if (*(volatile int *)c.flags || !*(volatile int *)(c.flags + 1)) return;
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const Ctx x = seg_ctx<SEG>(sv, n, 0);
    // a segment without a due check only takes part in the combine
    const bool due = SEG ? sv.segchk[x.s] != 0 : true;
    double2 acc[MU][1];
    ZERO_ACC(acc);
    if (due) {
        for_rows_spmv<MU, SF>(S, SB, y, x, mp, g, lane, ks, [&](int64_t row, const Pk<double>(&sy)[MU]) {
#pragma unroll
            for (int m = 0; m < MU; ++m) {
                const int u = lane + m * mp.G;
                if (u < mp.U) {
                    const size_t o = (size_t)row * mp.U + u;
                    const double2 qv = q[o], rv = ldw(r + o);
                    const double2 tv = make_double2(qv.x - sy[m].re[0], qv.y - sy[m].im[0]);
                    stw(t + o, tv);
                    acc[m][0].x += tv.x * tv.x + tv.y * tv.y;
                    const double dx = tv.x - rv.x, dy = tv.y - rv.y;
                    acc[m][0].y += dx * dx + dy * dy;
                }
            }
        });
    }
    cta_column_sums<MU, 1>(acc, mp, mp.U, smem, partial);
    __shared__ double2 tot[256];
    if (seg_sums<SEG>(partial, mp.U, tk, smem, tot, sv, x)) {
        __syncthreads();
        const int j = threadIdx.x;
        bool rs = false;
        if (due && j < mp.U) {
            const size_t cj = (size_t)x.s * mp.U + j;
            int act = c.active[cj];
            int restart = 0;
            if (act) {
                const double tn = sqrt(tot[j].x), thr = c.thr[cj];
                if (adaptive) {
                    const double gap = sqrt(tot[j].y);
                    restart = tn > thr && (gap > gap_ratio * fmax(tn, thr) || c.rn[cj] <= thr);
                } else {
                    restart = 1;
                }
                act = tn > thr;
                c.tn[cj] = tn;
            }
            c.active[cj] = act;
            c.restart[cj] = restart;
            if (restart) c.rsn[cj] = c.tn[cj];
            rs = restart;
        }
        const int nrs = __syncthreads_count(rs);
        if constexpr (SEG) {
            if (threadIdx.x == 0 && nrs) atomicAdd(reinterpret_cast<unsigned long long *>(&cnt->v[2]),
                                                   (unsigned long long)nrs);
        }
        if (last_segment<SEG>(tk, sv) && threadIdx.x == 0) {
            cnt->v[0] += 1;  // true_residual_refreshes
            cnt->v[1] += 1;  // true_residual_checks
            if constexpr (!SEG) cnt->v[2] += nrs;
        }
    }
}

// ---- after a check: r <- t on restarted columns, z = M^-1 r, beta
template <int MU, int MAXB, bool SEG, class W>
__global__ void __launch_bounds__(256, KMSD_PCG_MINB(MAXB))
    pcg_restart_kernel(W *r, W *z, const W *t, Pre P, int64_t nb, RowMap mp, ColPtr c,
                       double2 *partial, Ticket *tk, SegView sv, Loop lp) {
    loop_count(lp);
    if (*(volatile int *)c.flags || !*(volatile int *)(c.flags + 1)) return;
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const int U = mp.U;
    const Ctx x = seg_ctx<SEG>(sv, 0, nb);
    const size_t cs0 = (size_t)x.s * U;
    const bool due = SEG ? sv.segchk[x.s] != 0 : true;
    double2 acc[MU][1];
    ZERO_ACC(acc);
    for (int64_t bi = x.b0 + (int64_t)x.lc * mp.gpc + g; due && bi < x.b1; bi += (int64_t)x.nct * mp.gpc) {
        int64_t r0;
        int m;
        block_rows<MAXB>(P, bi, r0, m);
#pragma unroll
        for (int mm = 0; mm < MU; ++mm) {
            const int u = lane + mm * mp.G;
            if (u >= U) continue;
            const int rs = c.restart[cs0 + u];
            double2 rr[MAXB], zz[MAXB];
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                if (i < m) {
                    const size_t o = (size_t)(r0 + i) * U + u;
                    double2 rv = ldw(r + o);
                    if (rs) {
                        rv = ldw(t + o);
                        stw(r + o, rv);
                    }
                    rr[i] = rv;
                }
            }
            precond<MAXB>(P, bi, r0, m, rr, zz);
#pragma unroll
            for (int i = 0; i < MAXB; ++i) {
                if (i < m) {
                    stw(z + (size_t)(r0 + i) * U + u, zz[i]);
                    const double2 zs = stored<W>(zz[i]);
                    acc[mm][0].y += rr[i].x * zs.x + rr[i].y * zs.y;
                }
            }
        }
    }
    cta_column_sums<MU, 1>(acc, mp, U, smem, partial);
    __shared__ double2 tot[256];
    if (seg_sums<SEG>(partial, U, tk, smem, tot, sv, x)) {
        __syncthreads();
        const int j = threadIdx.x;
        bool act = false;
        if (due && j < U) {
            const size_t cj = cs0 + j;
            act = c.active[cj];
            const double rz = c.rz[cj], nrz = tot[j].y;
            c.beta[cj] = act ? nrz / (rz != 0. ? rz : 1.) : 0.;
            c.rz[cj] = nrz;
        }
        const int nact = __syncthreads_count(act);
        if constexpr (SEG) {
            if (threadIdx.x == 0 && due) {
                sv.segn[x.s] = nact;
                sv.segchk[x.s] = 0;
            }
        }
        if (last_segment<SEG>(tk, sv) && threadIdx.x == 0) {
            const int total = SEG ? total_active(sv) : nact;
            c.flags[1] = 0;
            c.flags[4] = total;
            if (total == 0) c.flags[0] = 1;
            if (lp.on) cudaGraphSetConditional(lp.again, (c.flags[0] == 0 && c.flags[5] < lp.maxiter) ? 1u : 0u);
        }
    }
}

// p = active ? z + (restart ? 0 : beta p) : 0
__device__ __forceinline__ double2 direction(const ColPtr &c, size_t cj, double2 zv, double2 pv) {
    if (!c.active[cj]) return make_double2(0., 0.);
    if (c.restart[cj]) return zv;
    const double be = c.beta[cj];
    return make_double2(zv.x + pv.x * be, zv.y + pv.y * be);
}
template <bool SEG, class W>
__global__ void pcg_direction_kernel(const W *z, W *p, int64_t len, RowMap mp, ColPtr c, SegView sv,
                                     Loop lp) {
    loop_count(lp);
    if (*(volatile int *)c.flags) return;
    if constexpr (!SEG) {
        const int U = mp.U;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
             i += (int64_t)gridDim.x * blockDim.x) {
            const int j = (int)(i % U);
            if (!c.active[j]) {
                stw(p + i, make_double2(0., 0.));
            } else {
                const double2 zv = ldw(z + i);
                stw(p + i, c.restart[j] ? zv : direction(c, j, zv, ldw(p + i)));
            }
        }
    } else {
        const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
        const Ctx x = seg_ctx<SEG>(sv, 0, 0);
        for (int64_t row = x.r0 + (int64_t)x.lc * mp.gpc + g; row < x.r1; row += (int64_t)x.nct * mp.gpc)
            for (int u = lane; u < mp.U; u += mp.G) {
                const size_t o = (size_t)row * mp.U + u;
                stw(p + o, direction(c, (size_t)x.s * mp.U + u, ldw(z + o), ldw(p + o)));
            }
    }
}

// ---- final acceptance: t = q - S y; converged, relative, residual
template <int MU, int SF, bool SEG>
__global__ void __launch_bounds__(256)
    pcg_final_kernel(CsrView<double> S, BsrView<double> SB, const double2 *q, const double2 *y, int64_t n,
                     RowMap mp, ColPtr c, double2 *partial, Ticket *tk, Counters *cnt, SegView sv, int ks) {
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const Ctx x = seg_ctx<SEG>(sv, n, 0);
    double2 acc[MU][1];
    ZERO_ACC(acc);
    for_rows_spmv<MU, SF>(S, SB, y, x, mp, g, lane, ks, [&](int64_t row, const Pk<double>(&sy)[MU]) {
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
                const double2 qv = q[(size_t)row * mp.U + u];
                const double tx = qv.x - sy[m].re[0], ty = qv.y - sy[m].im[0];
                acc[m][0].x += tx * tx + ty * ty;
            }
        }
    });
    cta_column_sums<MU, 1>(acc, mp, mp.U, smem, partial);
    __shared__ double2 tot[256];
    if (seg_sums<SEG>(partial, mp.U, tk, smem, tot, sv, x)) {
        __syncthreads();
        const int j = threadIdx.x;
        if (j < mp.U) {
            const size_t cj = (size_t)x.s * mp.U + j;
            const double rn = sqrt(tot[j].x), bn = c.bn[cj];
            c.conv[cj] = rn <= c.thr[cj] && !c.brk[cj];
            c.relative[cj] = bn > 0. ? rn / bn : 0.;
            c.residual[cj] = rn * c.safe[cj];
            c.rn[cj] = rn;
        }
        if (last_segment<SEG>(tk, sv) && threadIdx.x == 0) cnt->v[1] += 1;
    }
}

// ---- output: Y = y * safe with representability checks; status
template <int MU, bool SEG>
__global__ void __launch_bounds__(256) pcg_out_kernel(const double2 *y, double2 *Y, int64_t n, RowMap mp,
                                                      ColPtr c, double2 *partial, Ticket *tk, Counters *cnt,
                                                      int *status, FailReportFull *fr, SegView sv) {
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    const Ctx x = seg_ctx<SEG>(sv, n, 0);
    const size_t cs0 = (size_t)x.s * mp.U;
    double2 acc[MU][1];
    ZERO_ACC(acc);
    for (int64_t row = x.r0 + (int64_t)x.lc * mp.gpc + g; row < x.r1; row += (int64_t)x.nct * mp.gpc) {
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
                const size_t o = (size_t)row * mp.U + u;
                const double2 v = y[o];
                const double sf = c.safe[cs0 + u];
                const double2 w = make_double2(v.x * sf, v.y * sf);
                Y[o] = w;
                acc[m][0].x += (!isfinite(v.x) || !isfinite(v.y)) ? 1. : 0.;
                acc[m][0].y += (!isfinite(w.x) || !isfinite(w.y)) ? 1. : 0.;
            }
        }
    }
    cta_column_sums<MU, 1>(acc, mp, mp.U, smem, partial);
    __shared__ double2 tot[256];
    if (seg_sums<SEG>(partial, mp.U, tk, smem, tot, sv, x)) {
        __syncthreads();
        const int j = threadIdx.x;
        if (j < mp.U) {
            const size_t cj = cs0 + j;
            const int fin = tot[j].x == 0. && tot[j].y == 0.;
            c.finp[cj] = tot[j].x == 0.;
            c.fino[cj] = fin;
            c.conv[cj] = c.conv[cj] && fin;
        }
        if (last_segment<SEG>(tk, sv)) {
            // every column's state is final: reduce over all of them
            __syncthreads();
            const int ncols = (SEG ? sv.nseg : 1) * mp.U;
            bool notconv = false, unrep = false;
            long long it = 0;
            double rel = 0.;
            for (int k = threadIdx.x; k < ncols; k += blockDim.x) {
                notconv |= !__ldcg(c.conv + k);
                unrep |= !__ldcg(c.fino + k);
                it = max(it, __ldcg(c.iters + k));
                rel = fmax(rel, __ldcg(c.relative + k));
            }
            const bool any_nc = __syncthreads_or(notconv);
            const bool any_unrep = __syncthreads_or(unrep);
            __shared__ long long imax[256];
            __shared__ double rmax[256];
            imax[threadIdx.x] = it;
            rmax[threadIdx.x] = rel;
            __syncthreads();
            if (threadIdx.x == 0) {
                long long mi = 0;
                double mr = cnt->max_rel;
                for (int k = 0; k < (int)blockDim.x; ++k) {
                    mi = imax[k] > mi ? imax[k] : mi;
                    mr = fmax(mr, rmax[k]);
                }
                cnt->v[3] += mi;
                cnt->max_rel = mr;
                const bool nonfinite_rhs = c.flags[2] != 0;
                const bool brk = c.flags[3] != 0;
                if ((any_nc || brk || nonfinite_rhs) && status != nullptr && *status == 0) {
                    *status = nonfinite_rhs ? KMSD_EINVAL : KMSD_EMETRIC;
                    status[1] = 2;  // this solve owns the failure report
                    if (fr != nullptr) {
                        fr->head.ncols = ncols;
                        fr->head.code = *status;
                        fr->head.reason = nonfinite_rhs ? 3 : any_unrep ? 2 : brk ? 1 : 0;
                    }
                }
            }
        }
    }
}

// Copy the per-column report of a failed asynchronous solve (first failure).
__global__ void pcg_copy_report_kernel(ColPtr c, int ncols, int *status, int *claimed, FailReportFull *fr) {
    // Runs after pcg_out_kernel; only the solve that raised the status fills
    // the report (claimed == 2), later ones leave it unchanged.
    if (*claimed != 2) return;
    __syncthreads();
    for (int j = threadIdx.x; j < ncols && j < kMaxReportCols; j += blockDim.x) {
        fr->converged[j] = (uint8_t)c.conv[j];
        fr->breakdown[j] = (uint8_t)c.brk[j];
        fr->iterations[j] = c.iters[j];
        fr->true_residual[j] = c.residual[j];
        fr->relative_residual[j] = c.relative[j];
    }
    __syncthreads();
    if (threadIdx.x == 0) *claimed = 1;
}

}  // namespace

// ------------------------------------------------------------------ host side
int kmsd_metric_s::ensure(int64_t b, int64_t state_cols) {
    if (cols.ensure(col_bytes(std::max(b, state_cols)))) return KMSD_ECUDA;
    if (b <= wb && q.p) return KMSD_OK;
    const size_t bytes = (size_t)n * b * sizeof(double2);
    for (DevBuf *d : {&q, &y, &r, &z, &p, &sp, &t})
        if (d->ensure(bytes)) return KMSD_ECUDA;
    if (!dcount.p) {
        if (dcount.ensure(sizeof(Counters))) return KMSD_ECUDA;
        KMSD_CUDA(cudaMemset(dcount.p, 0, sizeof(Counters)));
    }
    if (!host_pinned.p) {
        void *h = nullptr;
        KMSD_CUDA(cudaMallocHost(&h, 64));
        host_pinned.p = h;
        host_pinned.bytes = 64;
        KMSD_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
        KMSD_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    }
    wb = b;
    return KMSD_OK;
}

// Device descriptor of the segments for row groups of `gpc` per CTA: CTAs
// are shared out in proportion to each segment's rows (at least one each,
// about one wave in total); tickets and level-2 partial rows per segment.
int kmsd_metric_s::seg_plan(int gpc, SegPlan **out) {
    auto it = seg_plans.find(gpc);
    if (it != seg_plans.end()) {
        *out = &it->second;
        return KMSD_OK;
    }
    const int64_t ns = nseg;
    std::vector<int64_t> want(ns);
    int64_t total = 0;
    for (int64_t s = 0; s < ns; ++s) {
        const int64_t rows = seg_row0[s + 1] - seg_row0[s];
        want[s] = std::max<int64_t>(1, (rows + 4 * gpc - 1) / (4 * gpc));
        total += want[s];
    }
    const int64_t cap = (int64_t)sm_count() * 8;
    std::vector<int> cta0(ns + 1, 0), tk0(ns + 1, 0), l2(ns, 0), cta_seg;
    int l2rows = 0;
    for (int64_t s = 0; s < ns; ++s) {
        const int64_t k = total > cap ? std::max<int64_t>(1, want[s] * cap / total) : want[s];
        cta0[s + 1] = cta0[s] + (int)k;
        tk0[s + 1] = tk0[s] + range_tickets((int)k);
        l2[s] = l2rows;
        const int groups = ((int)k + kTreeFan - 1) / kTreeFan;
        if (groups > 1) l2rows += groups;
        for (int64_t q = 0; q < k; ++q) cta_seg.push_back((int)s);
    }
    const int grid = cta0[ns];
    const int ntk = tk0[ns] + 1;  // plus the last-segment ticket
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t o_row = 0, o_blk = o_row + al((ns + 1) * 8), o_cseg = o_blk + al((ns + 1) * 8);
    const size_t o_cta0 = o_cseg + al((size_t)grid * 4), o_tk0 = o_cta0 + al((ns + 1) * 4);
    const size_t o_l2 = o_tk0 + al((ns + 1) * 4), o_segn = o_l2 + al(ns * 4), o_chk = o_segn + al(ns * 4);
    const size_t o_tick = o_chk + al(ns * 4), bytes = o_tick + al((size_t)ntk * sizeof(Ticket));
    SegPlan pl;
    if (pl.mem.ensure(bytes)) return KMSD_ECUDA;
    char *base = pl.mem.as<char>();
    KMSD_CUDA(cudaMemset(base, 0, bytes));
    KMSD_CUDA(cudaMemcpy(base + o_row, seg_row0.data(), (ns + 1) * 8, cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemcpy(base + o_blk, seg_blk0.data(), (ns + 1) * 8, cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemcpy(base + o_cseg, cta_seg.data(), (size_t)grid * 4, cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemcpy(base + o_cta0, cta0.data(), (ns + 1) * 4, cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemcpy(base + o_tk0, tk0.data(), (ns + 1) * 4, cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemcpy(base + o_l2, l2.data(), ns * 4, cudaMemcpyHostToDevice));
    pl.row0 = reinterpret_cast<int64_t *>(base + o_row);
    pl.blk0 = reinterpret_cast<int64_t *>(base + o_blk);
    pl.cta_seg = reinterpret_cast<int *>(base + o_cseg);
    pl.cta0 = reinterpret_cast<int *>(base + o_cta0);
    pl.tk0 = reinterpret_cast<int *>(base + o_tk0);
    pl.l2 = reinterpret_cast<int *>(base + o_l2);
    pl.segn = reinterpret_cast<int *>(base + o_segn);
    pl.segchk = reinterpret_cast<int *>(base + o_chk);
    pl.tickets = reinterpret_cast<Ticket *>(base + o_tick);
    pl.grid = grid;
    pl.l2rows = l2rows;
    auto ins = seg_plans.emplace(gpc, pl);
    pl.mem.p = nullptr;  // owned by the map entry now
    *out = &ins.first->second;
    return KMSD_OK;
}

namespace {

// How run_pcg drives the iterations: from the host (polling the halt word),
// not at all (only the workspace is prepared, so that a capture allocates
// nothing), or from the device as the WHILE node of a capturing stream.
enum { kHostLoop = 0, kPrepare = 1, kDeviceLoop = 2 };

// A kernel launch, as a programmatic dependent of the stream's previous
// kernel when `pdl` is set.
template <class... KArgs, class... Args>
cudaError_t launch_k(bool pdl, void (*kernel)(KArgs...), int grid, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

template <int MU, int MAXB, int SF, bool SEG, class W>
int run_pcg(kmsd_metric_s *M, const double2 *B, double2 *Y, int64_t b, double rtol, double atol, int maxiter,
            cudaStream_t s, int *status, FailReportFull *fr, int *claimed, int mode) {
    const int64_t n = M->n;
    const RowMap mp = make_map((int)b, kThreads);
    const int64_t nb = MAXB == 1 ? n : M->nblocks;
    const BsrView<double> SB = M->S->bsr64();
    const size_t sm = reduce_smem(mp, 1);
    // split each 4x4 block row over ks row groups while there are few block
    // rows for the resident row groups (four CTAs per SM)
    int ks = 1;
    if constexpr (SF != S_CSR) {
        const int64_t resident = (int64_t)sm_count() * KMSD_SPLIT_CTAS * mp.gpc;
        const int kmax = std::min(8, mp.gpc);
        while (ks * 2 <= kmax && M->S->bsr_nb * ks * 2 <= resident) ks *= 2;
    }
    const size_t sm_s = ks > 1 ? std::max(sm, (size_t)split_smem_units(MU) * sizeof(double2)) : sm;
    const int64_t len = n * b;
    int grid_r, grid_b, grid_s, egrid;
    SegView sv{};
    sv.nseg = 1;
    Ticket *tk;
    if constexpr (SEG) {
        // one grid for every kernel: each CTA belongs to one segment
        kmsd_metric_s::SegPlan *pl = nullptr;
        if (int rc = M->seg_plan(mp.gpc, &pl)) return rc;
        grid_r = grid_b = grid_s = egrid = pl->grid;
        if (M->red.ensure(pl->grid + pl->l2rows, (int)b)) return KMSD_ECUDA;
        sv = SegView{(int)M->nseg, pl->cta_seg, pl->cta0, pl->row0, pl->blk0, pl->tk0, pl->l2, pl->segn, pl->segchk};
        tk = pl->tickets;
    } else {
        grid_r = grid_for(n, mp);
        grid_b = grid_for(nb, mp);
        // S products walk block rows when S is stored as 4x4 blocks
        if constexpr (SF != S_CSR) {
            const int64_t spc = mp.gpc / ks;  // block rows per CTA and pass
            grid_s = (int)std::max<int64_t>(1, std::min<int64_t>((M->S->bsr_nb + spc - 1) / spc,
                                                                 (int64_t)sm_count() * 8));
        } else {
            grid_s = grid_r;
        }
        egrid = (int)std::min<int64_t>((len + 255) / 256, (int64_t)sm_count() * 16);
        if (M->red.ensure(std::max(grid_r, std::max(grid_b, grid_s)), (int)b)) return KMSD_ECUDA;
        tk = M->red.tick();
    }
    if (mode == kPrepare) return KMSD_OK;
    const int64_t ncols = (int64_t)sv.nseg * b;
    ColPtr c = col_ptr(M->cols.p, ncols);
    Pre P{M->diag, M->bstart, M->foff, M->factors, M->ub, M->inv_real};
    const CsrView<double> S = M->S->view64();
    Counters *cnt = M->dcount.as<Counters>();
    double2 *q = M->q.as<double2>(), *y = M->y.as<double2>();
    W *r = M->r.as<W>(), *z = M->z.as<W>(), *p = M->p.as<W>(), *sp = M->sp.as<W>(), *t = M->t.as<W>();
    double2 *part = M->red.part();

    KMSD_CUDA(cudaMemsetAsync(c.flags, 0, 8 * sizeof(int), s));
    pcg_scale_kernel<MU, SEG><<<grid_r, kThreads, sm, s>>>(B, n, mp, c, reinterpret_cast<double *>(part), tk, sv);
    count_launch();
    pcg_init_kernel<MU, MAXB, SEG><<<grid_b, kThreads, sm, s>>>(B, q, y, r, z, P, nb, mp, c, rtol, atol, part, tk,
                                                                sv);
    count_launch();
    pcg_pinit_kernel<SEG><<<egrid, 256, 0, s>>>(z, p, len, mp, c, sv);
    count_launch();
    if (mode == kDeviceLoop) {
        // The iterations as a WHILE node of the capture on s.  Its body is
        // captured on the metric's loop stream: spmv, update, an IF node
        // (captured on the check stream) around the true residual and the
        // restart, and the direction.
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        KMSD_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
        if (cs != cudaStreamCaptureStatusActive) return fail(KMSD_ERUNTIME, "a device-driven PCG loop must be captured");
        // (the node parameters' union has no default constructor)
        alignas(cudaGraphNodeParams) unsigned char w_store[sizeof(cudaGraphNodeParams)] = {};
        alignas(cudaGraphNodeParams) unsigned char i_store[sizeof(cudaGraphNodeParams)] = {};
        cudaGraphNodeParams &wp = *reinterpret_cast<cudaGraphNodeParams *>(w_store);
        cudaGraphNodeParams &ip = *reinterpret_cast<cudaGraphNodeParams *>(i_store);
        Loop lp{1, maxiter, 0, 0};
        KMSD_CUDA(cudaGraphConditionalHandleCreate(&lp.again, g, 1, cudaGraphCondAssignDefault));
        wp.type = cudaGraphNodeTypeConditional;
        wp.conditional.handle = lp.again;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        cudaGraphNode_t wnode;
        KMSD_CUDA(cudaGraphAddNode(&wnode, g, deps, nd, &wp));
        KMSD_CUDA(cudaStreamUpdateCaptureDependencies(s, &wnode, 1, cudaStreamSetCaptureDependencies));
        cudaGraph_t body = wp.conditional.phGraph_out[0];
        // (the IF handle goes into the update kernel's arguments, so it is made first)
        lp.has_check = KMSD_PCG_IFNODE;
        if (KMSD_PCG_IFNODE) KMSD_CUDA(cudaGraphConditionalHandleCreate(&lp.check, body, 0, cudaGraphCondAssignDefault));
        cudaStream_t bs = M->loop_stream, cs2 = M->check_stream;
        KMSD_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        cudaError_t le = launch_k(false, pcg_spmv_kernel<MU, SF, SEG, W>, grid_s, sm_s, bs, S, SB, (const W *)p, sp,
                                  n, mp, c, part, tk, sv, lp, ks);
        if (le == cudaSuccess)
            le = launch_k(KMSD_PCG_PDL, pcg_update_kernel<MU, MAXB, SEG, W>, grid_b, sm, bs, y, r, z, (const W *)p,
                          (const W *)sp, P, nb, mp, c, 0, M->interval, M->adaptive, part, tk, sv, lp);
        cudaError_t ae = cudaSuccess;
        if (KMSD_PCG_IFNODE) {
            cudaStreamCaptureStatus bcs;
            cudaGraph_t bg = nullptr;
            const cudaGraphNode_t *bdeps = nullptr;
            size_t bnd = 0;
            cudaGraphNode_t inode = nullptr;
            ae = cudaStreamGetCaptureInfo(bs, &bcs, nullptr, &bg, &bdeps, &bnd);
            if (ae == cudaSuccess) {
                ip.type = cudaGraphNodeTypeConditional;
                ip.conditional.handle = lp.check;
                ip.conditional.type = cudaGraphCondTypeIf;
                ip.conditional.size = 1;
                ae = cudaGraphAddNode(&inode, bg, bdeps, bnd, &ip);
            }
            if (ae == cudaSuccess)
                ae = cudaStreamUpdateCaptureDependencies(bs, &inode, 1, cudaStreamSetCaptureDependencies);
            if (ae == cudaSuccess)
                ae = cudaStreamBeginCaptureToGraph(cs2, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal);
            if (ae == cudaSuccess) {
                pcg_true_residual_kernel<MU, SF, SEG><<<grid_s, kThreads, sm_s, cs2>>>(
                    S, SB, q, y, r, t, n, mp, c, M->adaptive, M->gap_ratio, part, tk, cnt, sv, lp, ks);
                pcg_restart_kernel<MU, MAXB, SEG><<<grid_b, kThreads, sm, cs2>>>(r, z, t, P, nb, mp, c, part, tk, sv,
                                                                                lp);
                if (le == cudaSuccess) le = cudaGetLastError();
                cudaGraph_t ib = nullptr;
                ae = cudaStreamEndCapture(cs2, &ib);
            }
        } else {
            if (le == cudaSuccess)
                le = launch_k(KMSD_PCG_PDL, pcg_true_residual_kernel<MU, SF, SEG, W>, grid_s, sm_s, bs, S, SB,
                              (const double2 *)q, (const double2 *)y, (const W *)r, t, n, mp, c, M->adaptive,
                              M->gap_ratio, part, tk, cnt, sv, lp, ks);
            if (le == cudaSuccess)
                le = launch_k(KMSD_PCG_PDL, pcg_restart_kernel<MU, MAXB, SEG, W>, grid_b, sm, bs, r, z,
                              (const W *)t, P, nb, mp, c, part, tk, sv, lp);
        }
        if (le == cudaSuccess)
            le = launch_k(KMSD_PCG_PDL && !KMSD_PCG_IFNODE, pcg_direction_kernel<SEG, W>, egrid, 0, bs, z, p, len,
                          mp, c, sv, lp);
        cudaGraph_t bout = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(bs, &bout);
        if (ae != cudaSuccess) return cuda_fail(ae, "device PCG loop (check branch)");
        if (le != cudaSuccess) return cuda_fail(le, "device PCG loop body");
        if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture (device PCG loop body)");
    } else {
        volatile int *hflag = static_cast<volatile int *>(M->host_pinned.p);
        const int chunk = 4;
        int slot = 0, pending = 0;
        for (int k = 0; k < maxiter; ++k) {
            const int refresh = ((k + 1) % M->interval) == 0;
            pcg_spmv_kernel<MU, SF, SEG><<<grid_s, kThreads, sm_s, s>>>(S, SB, p, sp, n, mp, c, part, tk, sv, Loop{},
                                                                          ks);
            count_launch();
            pcg_update_kernel<MU, MAXB, SEG><<<grid_b, kThreads, sm, s>>>(y, r, z, p, sp, P, nb, mp, c, refresh, 0,
                                                                          M->adaptive, part, tk, sv, Loop{});
            count_launch();
            if (refresh || M->adaptive || M->store32) {
                pcg_true_residual_kernel<MU, SF, SEG><<<grid_s, kThreads, sm_s, s>>>(
                    S, SB, q, y, r, t, n, mp, c, M->adaptive, M->gap_ratio, part, tk, cnt, sv, Loop{}, ks);
                count_launch();
                pcg_restart_kernel<MU, MAXB, SEG><<<grid_b, kThreads, sm, s>>>(r, z, t, P, nb, mp, c, part, tk, sv,
                                                                               Loop{});
                count_launch();
            }
            pcg_direction_kernel<SEG><<<egrid, 256, 0, s>>>(z, p, len, mp, c, sv, Loop{});
            count_launch();
            if ((k + 1) % chunk == 0) {
                KMSD_CUDA(cudaMemcpyAsync((void *)(hflag + slot), c.flags, sizeof(int), cudaMemcpyDeviceToHost, s));
                KMSD_CUDA(cudaEventRecord(M->ev[slot], s));
                ++pending;
                const int other = slot ^ 1;
                if (pending >= 2) {
                    KMSD_CUDA(cudaEventSynchronize(M->ev[other]));
                    if (hflag[other]) break;
                }
                slot = other;
            }
        }
    }
    KMSD_CUDA(cudaGetLastError());
    pcg_final_kernel<MU, SF, SEG><<<grid_s, kThreads, sm_s, s>>>(S, SB, q, y, n, mp, c, part, tk, cnt, sv, ks);
    count_launch();
    pcg_out_kernel<MU, SEG><<<grid_r, kThreads, sm, s>>>(y, Y, n, mp, c, part, tk, cnt, status, fr, sv);
    count_launch();
    if (status != nullptr && fr != nullptr) {
        pcg_copy_report_kernel<<<1, 256, 0, s>>>(c, (int)ncols, status, claimed, fr);
        count_launch();
    }
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

using PcgFn = int (*)(kmsd_metric_s *, const double2 *, double2 *, int64_t, double, double, int, cudaStream_t,
                      int *, FailReportFull *, int *, int);

template <int MAXB, int SF, bool SEG, class W>
PcgFn pick_mu(int mu) {
    switch (mu) {
        case 1: return run_pcg<1, MAXB, SF, SEG, W>;
        case 2: return run_pcg<2, MAXB, SF, SEG, W>;
    }
    return nullptr;
}
template <int SF, bool SEG, class W>
PcgFn pick_b(int mu, int maxb) {
    if (maxb <= 1) return pick_mu<1, SF, SEG, W>(mu);
    if (maxb <= 4) return pick_mu<4, SF, SEG, W>(mu);
    if (maxb <= 8) return pick_mu<8, SF, SEG, W>(mu);
    if (maxb <= 32) return pick_mu<32, SF, SEG, W>(mu);
    return nullptr;
}
template <bool SEG, class W>
PcgFn pick_s(int mu, int maxb, int sf) {
    switch (sf) {
        case S_BSR_REAL: return pick_b<S_BSR_REAL, SEG, W>(mu, maxb);
        case S_BSR_CPLX: return pick_b<S_BSR_CPLX, SEG, W>(mu, maxb);
    }
    return pick_b<S_CSR, SEG, W>(mu, maxb);
}
// store32: the CG work vectors in complex64 (the mixed form)
PcgFn pick(int mu, int maxb, int sf, bool seg, bool store32) {
    if (store32) return seg ? pick_s<true, float2>(mu, maxb, sf) : pick_s<false, float2>(mu, maxb, sf);
    return seg ? pick_s<true, double2>(mu, maxb, sf) : pick_s<false, double2>(mu, maxb, sf);
}

}  // namespace

int kmsd_metric_s::solve(const double2 *B, double2 *Y, int64_t b, double rtol, double atol, int maxiter,
                         kmsd_solve_report *report, cudaStream_t s, int *status, void *fail_report) {
    if (b < 1 || !std::isfinite(rtol) || !std::isfinite(atol) || rtol < 0 || atol < 0 || maxiter < 1)
        return fail(KMSD_EINVAL, "invalid metric RHS shape/tolerances");
    if (b > 256) return fail(KMSD_EINVAL, "metric solve supports at most 256 columns per call");
    const auto start = std::chrono::steady_clock::now();
    const bool seg = nseg > 1;
    const int64_t ncols = seg ? nseg * b : b;
    if (ensure(b, ncols)) return KMSD_ECUDA;
    const RowMap mp = make_map((int)b, kThreads);
    // 4x4 block rows may not straddle two segments
    const bool bsr = S->bsr_nb > 0 && (!seg || seg_aligned4);
    const int sf = bsr ? (S->bsr64().im ? S_BSR_CPLX : S_BSR_REAL) : S_CSR;
    PcgFn fn = pick(mu_for(mp), nblocks ? maxb : 1, sf, seg, store32 != 0);
    if (!fn) return fail(KMSD_EINVAL, "unsupported metric block size / column count");
    const bool sync = status == nullptr;
    // Synchronous calls use a private status word and report.
    static thread_local DevBuf own_status, own_report;
    int *st = status;
    FailReportFull *fr = static_cast<FailReportFull *>(fail_report);
    int *claimed = nullptr;
    if (sync) {
        if (own_status.ensure(2 * sizeof(int))) return KMSD_ECUDA;
        if (own_report.ensure(sizeof(FailReportFull))) return KMSD_ECUDA;
        st = own_status.as<int>();
        fr = own_report.as<FailReportFull>();
        KMSD_CUDA(cudaMemsetAsync(st, 0, 2 * sizeof(int), s));
    }
    claimed = st + 1;
    int rc = fn(this, B, Y, b, rtol, atol, maxiter, s, st, fr, claimed, kHostLoop);
    if (rc) return rc;
    ++calls;
    if (!sync) return KMSD_OK;
    // Read status + per-column report (segment-major for a segmented solve).
    ColPtr c = col_ptr(cols.p, ncols);
    std::vector<int> conv(ncols), brk(ncols), flags(8);
    std::vector<long long> it(ncols);
    std::vector<double> res(ncols), rel(ncols);
    int hst[2];
    KMSD_CUDA(cudaMemcpyAsync(conv.data(), c.conv, ncols * sizeof(int), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaMemcpyAsync(brk.data(), c.brk, ncols * sizeof(int), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaMemcpyAsync(it.data(), c.iters, ncols * sizeof(long long), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaMemcpyAsync(res.data(), c.residual, ncols * sizeof(double), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaMemcpyAsync(rel.data(), c.relative, ncols * sizeof(double), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaMemcpyAsync(flags.data(), c.flags, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaMemcpyAsync(hst, st, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaStreamSynchronize(s));
    seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    if (report) {
        for (int64_t j = 0; j < ncols; ++j) {
            report->converged[j] = (uint8_t)conv[j];
            report->breakdown[j] = (uint8_t)brk[j];
            report->iterations[j] = it[j];
            report->true_residual[j] = res[j];
            report->relative_residual[j] = rel[j];
        }
    }
    if (flags[2]) return fail(KMSD_EINVAL, "metric RHS must be finite");
    if (hst[0]) {
        // Reproduce the reference's message precedence (native.cpp:447-450).
        std::vector<int> fino(ncols);
        KMSD_CUDA(cudaMemcpy(fino.data(), c.fino, ncols * sizeof(int), cudaMemcpyDeviceToHost));
        bool representable = true;
        for (int64_t j = 0; j < ncols; ++j) representable = representable && fino[j];
        if (!representable)
            return fail(KMSD_EMETRIC,
                        "S solve solution is nonfinite or not representable in complex128 after rescaling");
        if (flags[3]) return fail(KMSD_EMETRIC, "PCG non-positive/complex curvature breakdown");
        return fail(KMSD_EMETRIC, "S solve failed true-residual acceptance");
    }
    return KMSD_OK;
}

namespace kmsd {
int64_t device_loop_launches() {
    unsigned long long v = 0;
    if (cudaMemcpyFromSymbol(&v, g_loop_launches, sizeof(v)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (int64_t)v;
}
}  // namespace kmsd

int kmsd_metric_s::prepare_dev(int64_t b) {
    if (b < 1 || b > 256) return fail(KMSD_EINVAL, "metric solve supports at most 256 columns per call");
    const bool seg = nseg > 1;
    if (ensure(b, seg ? nseg * b : b)) return KMSD_ECUDA;
    const RowMap mp = make_map((int)b, kThreads);
    const bool bsr = S->bsr_nb > 0 && (!seg || seg_aligned4);
    const int sf = bsr ? (S->bsr64().im ? S_BSR_CPLX : S_BSR_REAL) : S_CSR;
    PcgFn fn = pick(mu_for(mp), nblocks ? maxb : 1, sf, seg, store32 != 0);
    if (!fn) return fail(KMSD_EINVAL, "unsupported metric block size / column count");
    if (!loop_stream) KMSD_CUDA(cudaStreamCreateWithFlags(&loop_stream, cudaStreamNonBlocking));
    if (!check_stream) KMSD_CUDA(cudaStreamCreateWithFlags(&check_stream, cudaStreamNonBlocking));
    return fn(this, nullptr, nullptr, b, 0., 0., 1, nullptr, nullptr, nullptr, nullptr, kPrepare);
}

int kmsd_metric_s::solve_dev(const double2 *B, double2 *Y, int64_t b, double rtol, double atol, int maxiter,
                             cudaStream_t s, int *status, void *fail_report) {
    if (b < 1 || !std::isfinite(rtol) || !std::isfinite(atol) || rtol < 0 || atol < 0 || maxiter < 1)
        return fail(KMSD_EINVAL, "invalid metric RHS shape/tolerances");
    if (b > 256) return fail(KMSD_EINVAL, "metric solve supports at most 256 columns per call");
    if (!status || !fail_report) return fail(KMSD_EINVAL, "a device-driven solve reports through a status word");
    const bool seg = nseg > 1;
    const int64_t ncols = seg ? nseg * b : b;
    if (ensure(b, ncols)) return KMSD_ECUDA;
    const RowMap mp = make_map((int)b, kThreads);
    const bool bsr = S->bsr_nb > 0 && (!seg || seg_aligned4);
    const int sf = bsr ? (S->bsr64().im ? S_BSR_CPLX : S_BSR_REAL) : S_CSR;
    PcgFn fn = pick(mu_for(mp), nblocks ? maxb : 1, sf, seg, store32 != 0);
    if (!fn) return fail(KMSD_EINVAL, "unsupported metric block size / column count");
    if (!loop_stream) KMSD_CUDA(cudaStreamCreateWithFlags(&loop_stream, cudaStreamNonBlocking));
    if (!check_stream) KMSD_CUDA(cudaStreamCreateWithFlags(&check_stream, cudaStreamNonBlocking));
    FailReportFull *fr = static_cast<FailReportFull *>(fail_report);
    int *claimed = status + 1;
    // every allocation happens here, outside any capture
    int rc = fn(this, B, Y, b, rtol, atol, maxiter, s, status, fr, claimed, kPrepare);
    if (rc) return rc;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    KMSD_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusActive) {  // part of the caller's graph
        CountOff off;
        rc = fn(this, B, Y, b, rtol, atol, maxiter, s, status, fr, claimed, kDeviceLoop);
        if (!rc) ++calls;
        return rc;
    }
    // the workspace the cached graphs point into
    std::vector<const void *> ws = {q.p, y.p, r.p, z.p, p.p, sp.p, t.p, cols.p, dcount.p, red.partial.p, red.ticket.p};
    for (auto &kv : seg_plans) ws.push_back(kv.second.mem.p);
    if (ws != graph_ws) {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second.first);
        graphs.clear();
        graph_ws = ws;
    }
    auto bits = [](double x) {
        uint64_t u;
        std::memcpy(&u, &x, sizeof(u));
        return u;
    };
    const std::vector<uint64_t> key = {(uint64_t)(uintptr_t)B, (uint64_t)(uintptr_t)Y, (uint64_t)b, bits(rtol),
                                       bits(atol), (uint64_t)maxiter, (uint64_t)(uintptr_t)status,
                                       (uint64_t)(uintptr_t)fail_report, (uint64_t)adaptive, (uint64_t)interval,
                                       bits(gap_ratio), (uint64_t)store32};
    auto it = graphs.find(key);
    if (it == graphs.end()) {
        if (graphs.size() >= 32) {  // bounded cache
            for (auto &kv : graphs) cudaGraphExecDestroy(kv.second.first);
            graphs.clear();
        }
        if (!cap_stream) KMSD_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        int64_t recorded = 0;
        {
            CountOff off;
            KMSD_CUDA(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
            rc = fn(this, B, Y, b, rtol, atol, maxiter, cap_stream, status, fr, claimed, kDeviceLoop);
            const cudaError_t e = cudaStreamEndCapture(cap_stream, &g);
            recorded = off.recorded();
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (device PCG solve)");
        }
        cudaGraphExec_t exec;
        const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate (device PCG solve)");
        it = graphs.emplace(key, std::make_pair(exec, recorded)).first;
    }
    KMSD_CUDA(cudaGraphLaunch(it->second.first, s));
    count_launch(it->second.second);  // the loop body's kernels are counted on the device
    ++calls;
    return KMSD_OK;
}

// ------------------------------------------------------------------ sampling
namespace {
int sample_impl(kmsd_metric_s *M, const double2 *xi, double2 *out, int64_t b, const double *coeff,
                int64_t ncoeff, double center, double half, cudaStream_t s) {
    const int64_t n = M->n;
    if (M->ensure(b)) return KMSD_ECUDA;
    const RowMap mp = make_map((int)b, kThreads);
    const int grid = grid_for(n, mp);
    double2 *b1 = M->q.as<double2>(), *b2 = M->r.as<double2>();
    const size_t bytes = (size_t)n * b * sizeof(double2);
    const CsrView<double> S = M->S->view64();
    if (ncoeff == 1) {
        // out = z .* (0 + c0 xi)
        KMSD_CUDA(cudaMemsetAsync(b1, 0, bytes, s));
        KMSD_CUDA(cudaMemsetAsync(b2, 0, bytes, s));
        // act(b1 = 0) = 0, so FINAL gives z .* (0 - 0 + c0 xi)
        clenshaw_kernel<1><<<grid, kThreads, 0, s>>>(S, M->zinv, b1, b2, xi, out, coeff[0], center, 1.0, n, mp);
        count_launch();
        KMSD_CUDA(cudaGetLastError());
        return KMSD_OK;
    }
    KMSD_CUDA(cudaMemsetAsync(b1, 0, bytes, s));
    KMSD_CUDA(cudaMemsetAsync(b2, 0, bytes, s));
    for (int64_t k = ncoeff - 1; k > 0; --k) {
        // b0 = 2 act(b1) - b2 + c_k xi, written over b2; then swap roles.
        clenshaw_kernel<0><<<grid, kThreads, 0, s>>>(S, M->zinv, b1, b2, xi, nullptr, coeff[k], center, half, n,
                                                    mp);
        count_launch();
        std::swap(b1, b2);
    }
    clenshaw_kernel<1><<<grid, kThreads, 0, s>>>(S, M->zinv, b1, b2, xi, out, coeff[0], center, half, n, mp);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}
// The Hermitian inverse (L L^H)^-1 of one m x m block from its lower
// Cholesky factor L (row-major): W = L^-1 by forward substitution, then the
// lower triangle of W^H W, mirrored so that the result is exactly Hermitian
// with a real diagonal.
void block_inverse(const double2 *L, int64_t m, double2 *out) {
    using cd = std::complex<double>;
    std::vector<cd> W(m * m, cd(0., 0.));
    auto l = [&](int64_t i, int64_t k) { return cd(L[i * m + k].x, L[i * m + k].y); };
    for (int64_t j = 0; j < m; ++j) {
        W[j * m + j] = 1. / l(j, j);
        for (int64_t i = j + 1; i < m; ++i) {
            cd v(0., 0.);
            for (int64_t k = j; k < i; ++k) v += l(i, k) * W[k * m + j];
            W[i * m + j] = -v / l(i, i);
        }
    }
    for (int64_t i = 0; i < m; ++i)
        for (int64_t k = 0; k <= i; ++k) {
            cd v(0., 0.);
            for (int64_t q = i; q < m; ++q) v += std::conj(W[q * m + i]) * W[q * m + k];
            if (k == i) v = cd(v.real(), 0.);
            out[i * m + k] = make_double2(v.real(), v.imag());
            out[k * m + i] = make_double2(v.real(), -v.imag());
        }
}
}  // namespace

// ------------------------------------------------------------------ ABI
extern "C" {

int kmsd_metric_create(kmsd_csr s, const double *diag, int64_t nblocks, const int64_t *block_start,
                       const int64_t *factor_offset, const double *factor_re, const double *factor_im,
                       kmsd_metric *out) {
    if (!s || !diag || !out) return fail(KMSD_EINVAL, "invalid metric diagonal/threads");
    const int64_t n = s->n;
    for (int64_t i = 0; i < n; ++i)
        if (!(diag[i] > 0) || !std::isfinite(diag[i])) return fail(KMSD_EINVAL, "invalid metric diagonal");
    int maxb = 1;
    std::vector<int> bs;
    std::vector<double2> fac;
    std::vector<int64_t> offs;
    if (nblocks > 0) {
        if (!block_start || !factor_offset || !factor_re)
            return fail(KMSD_EINVAL, "invalid block-Jacobi factor partition");
        if (block_start[0] != 0) return fail(KMSD_EINVAL, "invalid block-Jacobi factor partition");
        int64_t total = 0;
        for (int64_t i = 0; i < nblocks; ++i) {
            const int64_t a = block_start[i], bnd = block_start[i + 1];
            if (bnd <= a || bnd > n) return fail(KMSD_EINVAL, "invalid block-Jacobi factor partition");
            const int64_t m = bnd - a;
            if (m > 32) return fail(KMSD_EINVAL, "block-Jacobi blocks larger than 32 rows are not supported");
            if (m > maxb) maxb = (int)m;
            total = std::max(total, factor_offset[i] + m * m);
        }
        if (block_start[nblocks] != n) return fail(KMSD_EINVAL, "incomplete block-Jacobi partition");
        if (n > INT32_MAX) return fail(KMSD_EINVAL, "metric too large");
        bs.assign(block_start, block_start + nblocks + 1);
        offs.assign(factor_offset, factor_offset + nblocks);
        fac.resize(total);
        for (int64_t i = 0; i < total; ++i)
            fac[i] = make_double2(factor_re[i], factor_im ? factor_im[i] : 0.);
        for (int64_t i = 0; i < nblocks; ++i) {
            const int64_t m = block_start[i + 1] - block_start[i];
            for (int64_t d = 0; d < m; ++d) {
                const double2 v = fac[offs[i] + d * m + d];
                if (!(v.x != 0 || v.y != 0) || !std::isfinite(v.x) || !std::isfinite(v.y))
                    return fail(KMSD_EINVAL, "invalid block-Jacobi factor partition");
            }
        }
    }
    // Kernels for blocks of up to KMSD_BLOCK_INVERSE rows (the 4- and 8-row
    // instantiations) multiply by the block inverses.
    const int bucket = maxb <= 1 ? 1 : maxb <= 4 ? 4 : maxb <= 8 ? 8 : 32;
    bool inv_real = false;
    if (nblocks > 0 && bucket > 1 && bucket <= KMSD_BLOCK_INVERSE) {
        std::vector<double2> inv(fac.size(), make_double2(0., 0.));
        for (int64_t i = 0; i < nblocks; ++i)
            block_inverse(fac.data() + offs[i], block_start[i + 1] - block_start[i], inv.data() + offs[i]);
        for (const double2 &v : inv)
            if (!std::isfinite(v.x) || !std::isfinite(v.y))
                return fail(KMSD_EINVAL, "invalid block-Jacobi factor partition");
        inv_real = std::all_of(inv.begin(), inv.end(), [](const double2 &v) { return v.y == 0.; });
        fac.swap(inv);
    }
    auto *M = new kmsd_metric_s();
    M->S = s;
    M->n = n;
    M->nblocks = nblocks;
    M->maxb = maxb;
    M->inv_real = inv_real;
    M->bstart_host.assign(bs.begin(), bs.end());
    // Uniform partition with factors packed in block order (atom blocks of
    // one size): the kernels then compute rows and factor offsets directly.
    if (nblocks > 0) {
        bool uni = n % nblocks == 0;
        const int64_t m0 = uni ? n / nblocks : 0;
        for (int64_t i = 0; i < nblocks && uni; ++i)
            uni = block_start[i] == i * m0 && factor_offset[i] == i * m0 * m0;
        M->ub = uni ? (int)m0 : 0;
    }
    std::vector<double> zinv(n);
    for (int64_t i = 0; i < n; ++i) zinv[i] = 1. / std::sqrt(diag[i]);
    bool unit_diag = true;
    for (int64_t i = 0; i < n; ++i) unit_diag = unit_diag && diag[i] == 1.;
    M->identity = s->identity && nblocks == 0 && unit_diag;
    auto up = [&](void **dst, const void *src, size_t bytes) -> int {
        KMSD_CUDA(cudaMalloc(dst, bytes));
        KMSD_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
        return KMSD_OK;
    };
    int rc = up((void **)&M->diag, diag, n * sizeof(double));
    if (!rc) rc = up((void **)&M->zinv, zinv.data(), n * sizeof(double));
    if (!rc && nblocks > 0) {
        rc = up((void **)&M->bstart, bs.data(), bs.size() * sizeof(int));
        if (!rc) rc = up((void **)&M->foff, offs.data(), offs.size() * sizeof(int64_t));
        if (!rc) rc = up((void **)&M->factors, fac.data(), fac.size() * sizeof(double2));
    }
    if (rc) {
        kmsd_metric_destroy(M);
        return rc;
    }
    *out = M;
    return KMSD_OK;
}

void kmsd_metric_destroy(kmsd_metric m) {
    if (!m) return;
    cudaFree(m->diag);
    cudaFree(m->zinv);
    cudaFree(m->bstart);
    cudaFree(m->foff);
    cudaFree(m->factors);
    for (DevBuf *d : {&m->q, &m->y, &m->r, &m->z, &m->p, &m->sp, &m->t, &m->cols, &m->dcount}) d->release();
    m->red.partial.release();
    m->red.ticket.release();
    if (m->host_pinned.p) cudaFreeHost(m->host_pinned.p);
    for (auto &kv : m->seg_plans) kv.second.mem.release();
    for (auto &kv : m->graphs) cudaGraphExecDestroy(kv.second.first);
    if (m->loop_stream) cudaStreamDestroy(m->loop_stream);
    if (m->check_stream) cudaStreamDestroy(m->check_stream);
    if (m->cap_stream) cudaStreamDestroy(m->cap_stream);
    for (auto &e : m->ev)
        if (e) cudaEventDestroy(e);
    delete m;
}

namespace {
// bad[0] = 1 when a row of S has an entry outside its segment's rows.
__global__ void seg_coupling_kernel(const int *ptr, const int *idx, int64_t n, const int64_t *row0, int nseg,
                                    int *bad) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = nseg - 1;  // segment of row r: row0[lo] <= r < row0[lo + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (row0[mid] <= r) lo = mid;
            else hi = mid - 1;
        }
        const int64_t a = row0[lo], b = row0[lo + 1];
        for (int k = ptr[r]; k < ptr[r + 1]; ++k)
            if (idx[k] < a || idx[k] >= b) bad[0] = 1;
    }
}
}  // namespace

int kmsd_metric_set_segments(kmsd_metric m, int64_t nseg, const int64_t *row_offsets) {
    if (!m) return fail(KMSD_EINVAL, "invalid metric segments");
    for (auto &kv : m->seg_plans) kv.second.mem.release();
    m->seg_plans.clear();
    m->nseg = 0;
    m->seg_row0.clear();
    m->seg_blk0.clear();
    if (nseg <= 1) return KMSD_OK;
    if (!row_offsets || row_offsets[0] != 0 || row_offsets[nseg] != m->n)
        return fail(KMSD_EINVAL, "segment offsets must run from 0 to the metric size");
    for (int64_t s = 0; s < nseg; ++s)
        if (row_offsets[s + 1] <= row_offsets[s]) return fail(KMSD_EINVAL, "segment offsets must increase");
    std::vector<int64_t> blk(nseg + 1);
    if (m->nblocks > 0) {
        int64_t k = 0;
        for (int64_t s = 0; s <= nseg; ++s) {
            while (k < m->nblocks && m->bstart_host[k] < row_offsets[s]) ++k;
            if (m->bstart_host[k] != row_offsets[s])
                return fail(KMSD_EINVAL, "block-Jacobi blocks cross a segment boundary");
            blk[s] = k;
        }
    } else {
        blk.assign(row_offsets, row_offsets + nseg + 1);
    }
    // S must be block-diagonal over the segments
    DevBuf chk;
    if (chk.ensure((size_t)(nseg + 1) * 8 + 256)) return KMSD_ECUDA;
    int64_t *d_row0 = chk.as<int64_t>();
    int *d_bad = reinterpret_cast<int *>(reinterpret_cast<char *>(chk.p) + (size_t)(nseg + 1) * 8 + 128);
    int bad = 0;
    KMSD_CUDA(cudaMemcpy(d_row0, row_offsets, (size_t)(nseg + 1) * 8, cudaMemcpyHostToDevice));
    KMSD_CUDA(cudaMemset(d_bad, 0, sizeof(int)));
    const int grid = (int)std::min<int64_t>((m->n + 255) / 256, (int64_t)sm_count() * 8);
    seg_coupling_kernel<<<grid, 256>>>(m->S->ptr, m->S->idx, m->n, d_row0, (int)nseg, d_bad);
    count_launch();
    KMSD_CUDA(cudaMemcpy(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost));
    chk.release();
    if (bad) return fail(KMSD_EINVAL, "S couples two segments; a segmented solve needs a block-diagonal S");
    m->nseg = nseg;
    m->seg_row0.assign(row_offsets, row_offsets + nseg + 1);
    m->seg_blk0 = blk;
    m->seg_aligned4 = true;
    for (int64_t s = 0; s <= nseg; ++s) m->seg_aligned4 = m->seg_aligned4 && row_offsets[s] % 4 == 0;
    return KMSD_OK;
}

int kmsd_metric_set_storage(kmsd_metric m, int precision) {
    if (!m || (precision != KMSD_FP64 && precision != KMSD_MIXED)) return fail(KMSD_EINVAL, "invalid metric storage");
    m->store32 = precision == KMSD_MIXED;
    return KMSD_OK;
}

int kmsd_metric_set_residual_policy(kmsd_metric m, int policy, int interval, double gap_ratio) {
    if (!m || (policy != 0 && policy != 1) || interval < 1 || !(gap_ratio > 0 && gap_ratio < 1))
        return fail(KMSD_EINVAL, "invalid residual policy");
    m->adaptive = policy;
    m->interval = interval;
    m->gap_ratio = gap_ratio;
    return KMSD_OK;
}

int kmsd_metric_solve(kmsd_metric m, const void *b_in, void *y_out, int64_t b, double rtol, double atol,
                      int maxiter, kmsd_solve_report *report, void *stream) {
    if (!m || !b_in || !y_out) return fail(KMSD_EINVAL, "invalid metric RHS shape/tolerances");
    return m->solve(static_cast<const double2 *>(b_in), static_cast<double2 *>(y_out), b, rtol, atol, maxiter,
                    report, static_cast<cudaStream_t>(stream));
}

int kmsd_metric_sample(kmsd_metric m, const void *xi, void *out, int64_t b, const double *coeff, int64_t ncoeff,
                       double center, double half, void *stream) {
    if (!m || !xi || !out || b < 1 || ncoeff < 1 || !coeff) return fail(KMSD_EINVAL, "invalid sampling dimensions");
    if (b > 256) return fail(KMSD_EINVAL, "sampling supports at most 256 columns per call");
    if (ncoeff > 1 && !(half > 0)) return fail(KMSD_EINVAL, "sampling half-width must be positive");
    return sample_impl(m, static_cast<const double2 *>(xi), static_cast<double2 *>(out), b, coeff, ncoeff, center,
                       half, static_cast<cudaStream_t>(stream));
}

int kmsd_metric_stats_get(kmsd_metric m, kmsd_metric_stats *out) {
    if (!m || !out) return fail(KMSD_EINVAL, "invalid metric");
    Counters c{};
    if (m->dcount.p) {
        KMSD_CUDA(cudaDeviceSynchronize());
        KMSD_CUDA(cudaMemcpy(&c, m->dcount.p, sizeof(Counters), cudaMemcpyDeviceToHost));
    }
    out->calls = m->calls;
    out->max_iterations_sum = c.v[3];
    out->seconds = m->seconds;
    out->max_relative_residual = c.max_rel;
    out->true_residual_refreshes = c.v[0];
    out->true_residual_checks = c.v[1];
    out->residual_restarts = c.v[2];
    out->refinement_steps = 0;
    return KMSD_OK;
}

int kmsd_metric_is_identity(kmsd_metric m) { return m && m->identity ? 1 : 0; }

}  // extern "C"
