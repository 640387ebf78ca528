// Device kernels of the B200 stochastic-KPM engine: CSR SpMM, the fused
// Chebyshev step (moments / chain / augmented series), the Clenshaw sampling
// step, and small elementwise helpers.  Every kernel is a grid-stride loop
// over row groups (RowMap) with 128-bit unit accesses; reductions go through
// the deterministic two-stage column sums of kmsd_common.cuh.
#pragma once

#include "kmsd_common.cuh"

namespace kmsd {

// ------------------------------------------------------------ complex helpers
template <class T>
__device__ __forceinline__ void cmac_real(Pk<T> &acc, T v, const Pk<T> &x) {
#pragma unroll
    for (int c = 0; c < Pk<T>::C; ++c) {
        acc.re[c] = fma(v, x.re[c], acc.re[c]);
        acc.im[c] = fma(v, x.im[c], acc.im[c]);
    }
}
template <class T>
__device__ __forceinline__ void cmac_cplx(Pk<T> &acc, T vr, T vi, const Pk<T> &x) {
#pragma unroll
    for (int c = 0; c < Pk<T>::C; ++c) {
        acc.re[c] = fma(vr, x.re[c], fma(-vi, x.im[c], acc.re[c]));
        acc.im[c] = fma(vr, x.im[c], fma(vi, x.re[c], acc.im[c]));
    }
}
// The spectral rescaling (h - c x) / half.  The reference's Engine::scaled
// divides (native.cpp:534-538); here both precisions multiply by the rounded
// reciprocal, one rounding apart per element and step (the FP64 results stay
// within 1e-10 of the reference's).  On the 4.19M-site honeycomb at R=64 the
// FP64 tile step ran 2.57 ms per doubling launch against 2.76 ms dividing (ncu:
// 155.7M against 195.8M instructions per 524,288-row launch).
// KMSD_F64_RECIP=0 restores the division.
#ifndef KMSD_F64_RECIP
#define KMSD_F64_RECIP 1
#endif
__device__ __forceinline__ double rdiv(double a, double s, double inv) { return KMSD_F64_RECIP ? a * inv : a / s; }
__device__ __forceinline__ float rdiv(float a, float, float inv) { return a * inv; }

// The two product-identity sums of one row element: |x|^2 and Re(conj(x) next),
// added to FP64 column sums.  Every complex64 doubling step (paired, generic,
// tiled, batched) forms the two products in FP32 with one FMA each
// (KMSD_PAIR_SUM32), so all entry points compute the same mixed form;
// complex128 rows form them in FP64.  Against converting the four factors
// to FP64 first, the paired step on the 4.19M-site honeycomb at R=64 measured
// 4.159e11 / 4.152e11 against 4.050e11 / 4.077e11 orbital*moment*vec/s
// (1690 MHz), and the moments' error against the FP64 path went from 8.9e-8
// to 9.8e-8 (norm-wise).
#ifndef KMSD_PAIR_SUM32
#define KMSD_PAIR_SUM32 1
#endif
// `exact` forms the products in FP64 in every precision: the first launch of
// a direct-moments call that takes mu_0 and mu_1 from these sums (the batch and
// the allocation-free entry point) matches the direct path's FP64 products.
template <class T>
__device__ __forceinline__ void doubling_sums(double &s0, double &s1, T xr, T xi, T nr, T ni, bool exact = false) {
    if (KMSD_PAIR_SUM32 && sizeof(T) == 4 && !exact) {
        s0 += (double)fma(xr, xr, xi * xi);
        s1 += (double)fma(xr, nr, xi * ni);
    } else {
        s0 += (double)xr * (double)xr + (double)xi * (double)xi;
        s1 += (double)xr * (double)nr + (double)xi * (double)ni;
    }
}

// acc[m] += sum_k A[row,k] X[k, unit u_m]   for the MU units of this lane.
template <class T, int MU>
__device__ __forceinline__ void gather_row(const CsrView<T> &A, const typename Unit<T>::vec *X,
                                           int64_t row, int U, int G, int lane, Pk<T> (&acc)[MU]) {
    const int k0 = __ldg(A.ptr + row), k1 = __ldg(A.ptr + row + 1);
    if (A.im == nullptr) {
        for (int k = k0; k < k1; ++k) {
            const int col = __ldg(A.idx + k);
            const T v = __ldg(A.re + k);
            const typename Unit<T>::vec *src = X + (size_t)col * U;
#pragma unroll
            for (int m = 0; m < MU; ++m) {
                const int u = lane + m * G;
                if (u < U) cmac_real(acc[m], v, ldg(src + u));
            }
        }
    } else {
        for (int k = k0; k < k1; ++k) {
            const int col = __ldg(A.idx + k);
            const T vr = __ldg(A.re + k), vi = __ldg(A.im + k);
            const typename Unit<T>::vec *src = X + (size_t)col * U;
#pragma unroll
            for (int m = 0; m < MU; ++m) {
                const int u = lane + m * G;
                if (u < U) cmac_cplx(acc[m], vr, vi, ldg(src + u));
            }
        }
    }
}

// gather_row for a complex128 matrix over complex128 or complex64 X, with
// FP64 accumulation (the S products of the metric solve).
template <int MU, class XV>
__device__ __forceinline__ void gather_row_d(const CsrView<double> &A, const XV *X, int64_t row, int U, int G,
                                             int lane, Pk<double> (&acc)[MU]) {
    const int k0 = __ldg(A.ptr + row), k1 = __ldg(A.ptr + row + 1);
    for (int k = k0; k < k1; ++k) {
        const int col = __ldg(A.idx + k);
        const double vr = __ldg(A.re + k), vi = A.im ? __ldg(A.im + k) : 0.;
        const XV *src = X + (size_t)col * U;
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * G;
            if (u < U) {
                if (A.im) cmac_cplx(acc[m], vr, vi, ldg_d(src + u));
                else cmac_real(acc[m], vr, ldg_d(src + u));
            }
        }
    }
}

// Four matrix values starting at a 16-byte aligned element.
__device__ __forceinline__ void ld4(const float *p, float (&v)[4]) {
    const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double *p, double (&v)[4]) {
    const double2 q0 = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 q1 = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
}

// acc[m] += sum_k A[row,k] X[k, unit u_m] over the ELL row: one int4 of
// column indices and one 16-byte load of values per four entries, all four
// gathers of a chunk issued before their multiply-adds.
template <class T, int MU>
__device__ __forceinline__ void gather_row_ell(const EllView<T> &A, const typename Unit<T>::vec *X, int64_t row,
                                               int U, int G, int lane, Pk<T> (&acc)[MU]) {
    const int4 *ip = reinterpret_cast<const int4 *>(A.idx + row * A.w);
    const T *rp = A.re + row * A.w;
    const T *jp = A.im ? A.im + row * A.w : nullptr;
    for (int k4 = 0; k4 < A.w / 4; ++k4) {
        const int4 c = __ldg(ip + k4);
        T vr[4], vi[4];
        ld4(rp + 4 * k4, vr);
        if (jp) ld4(jp + 4 * k4, vi);
        const int col[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * G;
            if (u < U) {
                Pk<T> xs[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) xs[j] = ldg(X + (size_t)col[j] * U + u);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (jp) cmac_cplx(acc[m], vr[j], vi[j], xs[j]);
                    else cmac_real(acc[m], vr[j], xs[j]);
                }
            }
        }
    }
}

// acc[i][m] += sum over the 4x4 blocks of block row I of A[4I+i, 4J+j] X[4J+j, u_m]:
// each gathered input row serves four output rows from registers.  CPLX
// selects complex block values at compile time, so a real matrix (the usual
// tight-binding S and H) carries no registers for imaginary parts; block
// values are loaded one block row at a time.
// With ks > 1 this call takes only the blocks part, part + ks, ... of the
// block row (a split of one block row over ks row groups).
template <int MU, bool CPLX, class XV = double2>
__device__ __forceinline__ void gather_block_row(const BsrView<double> &A, const XV *X, int64_t I, int U,
                                                 int G, int lane, Pk<double> (&acc)[4][MU], int part = 0,
                                                 int ks = 1) {
    const int k0 = __ldg(A.bptr + I) + part, k1 = __ldg(A.bptr + I + 1);
    // Lanes past the last unit read the last unit instead: their sums are
    // never stored, and the gathers need no per-load select.
    const XV *xl[MU];
#pragma unroll
    for (int m = 0; m < MU; ++m) {
        const int u = lane + m * G;
        xl[m] = X + (u < U ? u : U - 1);
    }
    const unsigned U4 = 4u * (unsigned)U;
    const size_t Us = (size_t)U;
    // the next block's column index is loaded one block ahead, so each
    // block's gathers wait for one memory round trip, not two
    int Jn = k0 < k1 ? __ldg(A.bidx + k0) : 0;
    for (int k = k0; k < k1; k += ks) {
        const unsigned J = (unsigned)Jn;
        if (k + ks < k1) Jn = __ldg(A.bidx + k + ks);
        Pk<double> x[MU][4];
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const XV *xr = xl[m] + (size_t)J * U4;  // block column J: rows 4J .. 4J+3
#pragma unroll
            for (int j = 0; j < 4; ++j) x[m][j] = ldg_d(xr + j * Us);
        }
        const double2 *pr = reinterpret_cast<const double2 *>(A.re + (size_t)k * 16);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double2 r01 = __ldg(pr + 2 * i), r23 = __ldg(pr + 2 * i + 1);
            const double vr[4] = {r01.x, r01.y, r23.x, r23.y};
            if constexpr (CPLX) {
                const double2 *pi = reinterpret_cast<const double2 *>(A.im + (size_t)k * 16);
                const double2 i01 = __ldg(pi + 2 * i), i23 = __ldg(pi + 2 * i + 1);
                const double vi[4] = {i01.x, i01.y, i23.x, i23.y};
#pragma unroll
                for (int m = 0; m < MU; ++m)
#pragma unroll
                    for (int j = 0; j < 4; ++j) cmac_cplx(acc[i][m], vr[j], vi[j], x[m][j]);
            } else {
#pragma unroll
                for (int m = 0; m < MU; ++m)
#pragma unroll
                    for (int j = 0; j < 4; ++j) cmac_real(acc[i][m], vr[j], x[m][j]);
            }
        }
    }
}

// Y = A X over the block rows of a 4x4 BSR matrix (optionally with the
// conj(X_row) * Y_row column sums, as spmm_kernel).
template <int MU, bool DOT, bool CPLX>
__global__ void __launch_bounds__(256) spmm_bsr_kernel(BsrView<double> A, const double2 *X, double2 *Y, RowMap mp,
                                                       double2 *partial, Ticket *ticket, double2 *dot_out) {
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    double2 acc[MU][1];
#pragma unroll
    for (int m = 0; m < MU; ++m) acc[m][0] = make_double2(0., 0.);
    for (int64_t I = (int64_t)blockIdx.x * mp.gpc + g; I < A.nbrows; I += (int64_t)gridDim.x * mp.gpc) {
        Pk<double> y[4][MU];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int m = 0; m < MU; ++m) y[i][m] = pk_zero<double>();
        gather_block_row<MU, CPLX>(A, X, I, mp.U, mp.G, lane, y);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int m = 0; m < MU; ++m) {
                const int u = lane + m * mp.G;
                if (u < mp.U) {
                    const size_t o = (size_t)(4 * I + i) * mp.U + u;
                    st(Y + o, y[i][m]);
                    if (DOT) {
                        const Pk<double> x = ld(X + o);
                        acc[m][0].x += x.re[0] * y[i][m].re[0] + x.im[0] * y[i][m].im[0];
                        acc[m][0].y += x.re[0] * y[i][m].im[0] - x.im[0] * y[i][m].re[0];
                    }
                }
            }
    }
    if (DOT) {
        cta_column_sums<MU, 1>(acc, mp, mp.U, smem, partial);
        tree_column_sums(partial, mp.U, ticket, smem, dot_out);
    }
}

// Same for one unit (runtime loop callers).
template <class T>
__device__ __forceinline__ Pk<T> gather_unit(const CsrView<T> &A, const typename Unit<T>::vec *X,
                                             int64_t row, int U, int u) {
    Pk<T> acc = pk_zero<T>();
    const int k0 = __ldg(A.ptr + row), k1 = __ldg(A.ptr + row + 1);
    if (A.im == nullptr) {
        for (int k = k0; k < k1; ++k)
            cmac_real(acc, __ldg(A.re + k), ldg(X + (size_t)__ldg(A.idx + k) * U + u));
    } else {
        for (int k = k0; k < k1; ++k)
            cmac_cplx(acc, __ldg(A.re + k), __ldg(A.im + k), ldg(X + (size_t)__ldg(A.idx + k) * U + u));
    }
    return acc;
}

// sum_j H_ij (x_j - x_i) X[j, unit u]: the commutator [H, X] with the
// diagonal X = diag(x) applied to one unit of the row, from H's CSR row.
// The coordinate difference is formed in FP64 before it meets H_ij, so
// large absolute coordinates lose no precision in the mixed form.
template <class T>
__device__ __forceinline__ Pk<T> gather_commutator(const CsrView<T> &A, const double *x,
                                                   const typename Unit<T>::vec *X, int64_t row, int U, int u) {
    Pk<T> acc = pk_zero<T>();
    const int k0 = __ldg(A.ptr + row), k1 = __ldg(A.ptr + row + 1);
    const double xi = __ldg(x + row);
    for (int k = k0; k < k1; ++k) {
        const int col = __ldg(A.idx + k);
        const T d = (T)(__ldg(x + col) - xi);
        const Pk<T> xv = ldg(X + (size_t)col * U + u);
        if (A.im == nullptr) cmac_real(acc, d * __ldg(A.re + k), xv);
        else cmac_cplx(acc, d * __ldg(A.re + k), d * __ldg(A.im + k), xv);
    }
    return acc;
}

// ------------------------------------------------------------ SpMM
// Y = A X (optionally with per-column partial sums of conj(X_row) * Y_row,
// the curvature <p, S p> of the metric solve).
template <class T, int MU, bool DOT>
__global__ void __launch_bounds__(256) spmm_kernel(CsrView<T> A, const typename Unit<T>::vec *X,
                                                   typename Unit<T>::vec *Y, int64_t n, RowMap mp,
                                                   double2 *partial, Ticket *ticket, double2 *dot_out) {
    using V = typename Unit<T>::vec;
    constexpr int C = Unit<T>::C;
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    double2 acc[MU][C];
#pragma unroll
    for (int m = 0; m < MU; ++m)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[m][c] = make_double2(0., 0.);
    for (int64_t row = (int64_t)blockIdx.x * mp.gpc + g; row < n; row += (int64_t)gridDim.x * mp.gpc) {
        Pk<T> y[MU];
#pragma unroll
        for (int m = 0; m < MU; ++m) y[m] = pk_zero<T>();
        gather_row<T, MU>(A, X, row, mp.U, mp.G, lane, y);
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
                const size_t o = (size_t)row * mp.U + u;
                st(Y + o, y[m]);
                if (DOT) {
                    const Pk<T> x = ld(X + o);
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        // conj(x) * y
                        acc[m][c].x += (double)x.re[c] * y[m].re[c] + (double)x.im[c] * y[m].im[c];
                        acc[m][c].y += (double)x.re[c] * y[m].im[c] - (double)x.im[c] * y[m].re[c];
                    }
                }
            }
        }
    }
    if (DOT) {
        const int ncol = mp.U * C;
        cta_column_sums<MU, C>(acc, mp, ncol, smem, partial);
        tree_column_sums(partial, ncol, ticket, smem, dot_out);
    }
}

// ------------------------------------------------------------ Chebyshev step
// next = first ? t : 2 t - prev,  t = (h - center x)/half  [+ injection],
// h = S^-1 H x: computed inline from H when the metric is the identity
// (h_inline) or read from a precomputed buffer `hx` (general metric).
// MODE selects the epilogue:
//   MODE_CHAIN    store next (and optionally a complex128 copy)
//   MODE_DIRECT   moment mu_k[j] = Re sum_i conj(bra_ij) next_ij
//   MODE_DOUBLING s_even = <x,x>, s_odd = <x,next>  (mu_2n, mu_2n+1)
//   MODE_SERIES   out = first ? c0 x + c1 next : out + ck next, with the
//                 augmented velocity injection on the phi columns
enum { MODE_CHAIN = 0, MODE_DIRECT = 1, MODE_DOUBLING = 2, MODE_SERIES = 3 };

template <class T> struct StepArgs {
    using V = typename Unit<T>::vec;
    int64_t n;
    RowMap mp;
    CsrView<T> H;          // inline operator (identity metric)
    EllView<T> E;          // the same operator in ELL form (HSRC_ELL)
    const V *hx;           // precomputed S^-1 H x (general metric), or nullptr
    const V *curr;         // T_{k-1} (= x)
    const V *prev;         // T_{k-2}; may alias `next`
    V *next;               // T_k
    int first;             // k == 1
    int exact_sums;        // MODE_DOUBLING: FP64 row products in every precision
    double center, half;
    T inv_half;
    // moments
    const V *bra;          // S B (MODE_DIRECT)
    double2 *partial;      // [grid][ncol] (x2 for doubling)
    Ticket *ticket;
    double *mu;            // moment array (length, bcols)
    int64_t kmom;          // MODE_DIRECT: row of mu; MODE_DOUBLING: n
    int64_t mlen;          // number of moments
    int bcols;             // real columns (<= U*C)
    // chain copy-out (complex128), MODE_CHAIN
    double2 *store64;
    // series
    V *out;
    T c0r, c0i, ckr, cki;  // coefficients (c0 used when first)
    int UR;                // units of the psi block (0: no augmentation)
    int nphi;              // number of phi blocks
    // inline velocity: for each axis, CSR and weight w[a][axis] (complex).
    // vform[v] = 0: Vm[v] is the velocity matrix; 1: the velocity is the
    // commutator i [H, X] / hbar with X = diag(xdiag[v]), applied from H's
    // row (the i / hbar is folded into the weights)
    CsrView<T> Vm[3];
    int vform[3];
    const double *xdiag[3];
    // vform[v] = 2: the velocity's values aligned with H's ELL columns
    // (vel_re/vel_im[row * w + j] pairs with H's ELL index [row * w + j]),
    // applied from the ELL row the step already holds
    const T *vel_re[3], *vel_im[3];
    int nvel;              // number of velocity matrices in use
    int share_v;           // every velocity in use has vform 2: psi lanes share V psi (see gather_share_v)
    int vel_axis[3];
    T wr[4][3], wi[4][3];  // injection weights per phi block and velocity matrix
    // precomputed injection (general path): inj[a] of shape (n, UR units), FP64 complex
    const V *inj[4];
    T injr, inji;          // injection scale (-i hbar / half)
    int *status;           // nonfinite flag for series output
};

// Where h = S^-1 H x comes from: a solved operand (general metric), CSR,
// ELL of any width, or real ELL of width 4 / 8 whose next row's indices and
// values are prefetched one grid-stride iteration ahead, so each row waits on
// one memory latency (its gathers) instead of three.
enum { HSRC_SOLVED = 0, HSRC_CSR = 1, HSRC_ELL = 2, HSRC_ELL4 = 3, HSRC_ELL8 = 4 };

// Minimum resident CTAs per SM asked of the compiler for the one-unit-per-lane
// step kernels.  The kernel is latency bound; on B200 four CTAs of 256
// threads (<= 64 registers) measured best for the moment steps.
// Moment steps over a 4- or 8-wide real ELL form take two rows per row group
// and iteration (all loads of both rows issued before either row is
// computed), at KMSD_STEP_PAIR_MINB CTAs per SM.  On the 4.19M-site
// honeycomb moment step this measured 1.5 % faster than one row at four CTAs
// per SM, and two rows at three CTAs per SM were slower.  0 disables it.
#ifndef KMSD_STEP_PAIR
#define KMSD_STEP_PAIR 1
#endif
#ifndef KMSD_STEP_PAIR_MINB
#define KMSD_STEP_PAIR_MINB 2
#endif
#ifndef KMSD_STEP_MINB
#define KMSD_STEP_MINB 4
#endif

template <class T, int PF> struct EllRow {
    int4 idx[PF];
    T val[PF][4];
};
template <class T, int PF>
__device__ __forceinline__ void ell_row_load(const EllView<T> &A, int64_t row, EllRow<T, PF> &r) {
    const int4 *ip = reinterpret_cast<const int4 *>(A.idx + row * (4 * PF));
    const T *vp = A.re + row * (4 * PF);
#pragma unroll
    for (int q = 0; q < PF; ++q) {
        r.idx[q] = __ldg(ip + q);
        ld4(vp + 4 * q, r.val[q]);
    }
}
// acc[m] += sum over the prefetched ELL row (real values).
template <class T, int MU, int PF>
__device__ __forceinline__ void gather_prefetched(const EllRow<T, PF> &r, const typename Unit<T>::vec *X, int U,
                                                  int G, int lane, Pk<T> (&acc)[MU]) {
#pragma unroll
    for (int m = 0; m < MU; ++m) {
        const int u = lane + m * G;
        if (u < U) {
#pragma unroll
            for (int q = 0; q < PF; ++q) {
                const int col[4] = {r.idx[q].x, r.idx[q].y, r.idx[q].z, r.idx[q].w};
                Pk<T> xs[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) xs[j] = ldg(X + (size_t)col[j] * U + u);
#pragma unroll
                for (int j = 0; j < 4; ++j) cmac_real(acc[m], r.val[q][j], xs[j]);
            }
        }
    }
}

#ifndef KMSD_STEP_PAIR_F64
#define KMSD_STEP_PAIR_F64 1  // the paired form for FP64 vectors too
#endif

#ifndef KMSD_STEP_PAIR_PREFETCH
#define KMSD_STEP_PAIR_PREFETCH 0  // rows of the next pair loaded ahead: 0 ELL, 1 + T_{k-2}, 2 + T_{k-1}
#endif
template <class T, int MU, int MODE, int HSRC>
constexpr bool step_pairs() {
    return KMSD_STEP_PAIR && (KMSD_STEP_PAIR_F64 || sizeof(T) == 4) && MU == 1 && MODE == MODE_DOUBLING &&
           (HSRC == HSRC_ELL4 || HSRC == HSRC_ELL8);
}

// Resident CTAs per SM asked for the one-unit series step.  On the
// 4,194,304-site honeycomb with [psi | phi] of 2 x 64 (complex64) or 2 x 32
// (complex128) columns, 3 (80 registers, no spill) measured 6.04 / 6.41 ms per
// step against 8.13 / 16.1 ms unbounded and 8.14 / 8.78 ms at 2.
#ifndef KMSD_SERIES_MINB
#define KMSD_SERIES_MINB 3
#endif
#ifndef KMSD_SERIES_MINB_F64
#define KMSD_SERIES_MINB_F64 KMSD_SERIES_MINB
#endif
// The series step loads a row's Bessel accumulator with its other row-local
// operands, before the gathers, instead of after the row's arithmetic.
#ifndef KMSD_SERIES_EARLY_OUT
#define KMSD_SERIES_EARLY_OUT 1
#endif
// Series step over a 4- or 8-wide ELL operator with every velocity aligned to
// H's ELL columns: the psi lanes form the velocity products V_v psi from the
// neighbour values they gather for H anyway and leave them in shared memory
// (two parity slices of nvel x blockDim.x units) for the phi lanes of their
// row group, which then gather only their own H row.
// On the 4,194,304-site honeycomb with [psi | phi] of 2 x 64 complex64 columns
// the series step took 5.08 ms with the shared products against 5.44 ms
// without (6.04 ms before the early accumulator load); with 2 x 32 complex128
// columns it took 6.46 against 6.41 ms (a 68-byte spill under the register
// bound), so the FP64 step keeps its own gathers.
#ifndef KMSD_SERIES_SHARE_V
#define KMSD_SERIES_SHARE_V 1
#endif
#ifndef KMSD_SERIES_SHARE_V_F64
#define KMSD_SERIES_SHARE_V_F64 0
#endif
template <class T> constexpr bool series_shares_v() {
    return KMSD_SERIES_SHARE_V && (sizeof(T) == 4 || KMSD_SERIES_SHARE_V_F64);
}
template <class T, int PF>
__device__ __forceinline__ void gather_share_v(const StepArgs<T> &a, const EllRow<T, PF> &r, int64_t row, int u,
                                               Pk<T> &acc, typename Unit<T>::vec *slot) {
    const int U = a.mp.U;
    if (u >= U) return;
    Pk<T> xs[PF][4];
#pragma unroll
    for (int q = 0; q < PF; ++q) {
        const int col[4] = {r.idx[q].x, r.idx[q].y, r.idx[q].z, r.idx[q].w};
#pragma unroll
        for (int j = 0; j < 4; ++j) xs[q][j] = ldg(a.curr + (size_t)col[j] * U + u);
    }
#pragma unroll
    for (int q = 0; q < PF; ++q)
#pragma unroll
        for (int j = 0; j < 4; ++j) cmac_real(acc, r.val[q][j], xs[q][j]);
    if (u >= a.UR) return;
#pragma unroll 1
    for (int v = 0; v < a.nvel; ++v) {
        Pk<T> vp = pk_zero<T>();
        const T *vr = a.vel_re[v] + row * (4 * PF), *vi = a.vel_im[v] + row * (4 * PF);
#pragma unroll
        for (int q = 0; q < PF; ++q) {
            T r4[4], i4[4];
            ld4(vr + 4 * q, r4);
            ld4(vi + 4 * q, i4);
#pragma unroll
            for (int j = 0; j < 4; ++j) cmac_cplx(vp, r4[j], i4[j], xs[q][j]);
        }
        st(slot + (size_t)v * blockDim.x, vp);
    }
}
// Barrier over one row group: a named barrier for groups of several warps,
// the group's lanes of the warp otherwise (a group shares its trip count).
__device__ __forceinline__ void group_sync(const RowMap &mp, int g) {
    if (mp.G > 32) {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(mp.G) : "memory");
    } else {
        const unsigned lanes =
            mp.G == 32 ? 0xffffffffu : ((1u << mp.G) - 1u) << ((threadIdx.x & 31) / mp.G * mp.G);
        __syncwarp(lanes);
    }
}

template <class T, int MU, int MODE, int HSRC, bool INLINE_V>
__global__ void __launch_bounds__(256, (step_pairs<T, MU, MODE, HSRC>() ? KMSD_STEP_PAIR_MINB
                                        : MU == 1 && MODE != MODE_SERIES ? KMSD_STEP_MINB
                                        : MU == 1 ? (sizeof(T) == 8 ? KMSD_SERIES_MINB_F64 : KMSD_SERIES_MINB)
                                                  : 1))
    cheb_step_kernel(const StepArgs<T> a) {
    using V = typename Unit<T>::vec;
    constexpr int C = Unit<T>::C;
    extern __shared__ double2 smem[];
    const RowMap mp = a.mp;
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    double2 acc0[MU][C], acc1[MU][C];
#pragma unroll
    for (int m = 0; m < MU; ++m)
#pragma unroll
        for (int c = 0; c < C; ++c) {
            acc0[m][c] = make_double2(0., 0.);
            acc1[m][c] = make_double2(0., 0.);
        }
    const T cen = (T)a.center, hal = (T)a.half;
    bool bad = false;
    constexpr int PF = HSRC == HSRC_ELL4 ? 1 : HSRC == HSRC_ELL8 ? 2 : 1;
    const int64_t stride = (int64_t)gridDim.x * mp.gpc;
    if constexpr (step_pairs<T, MU, MODE, HSRC>()) {
        // Rows `row` and `row + stride` per iteration; the ELL rows of the
        // next pair are loaded one iteration ahead.
        // With KMSD_STEP_PAIR_PREFETCH >= 1 the T_{k-2} rows of the next pair
        // are loaded one iteration ahead too (>= 2: and its T_{k-1} rows).
        // The next pair's rows are written only in their own iteration, so the
        // in-place update is unaffected.
        const int u = lane;
        const int64_t first = (int64_t)blockIdx.x * mp.gpc + g;
        constexpr int PRE = KMSD_STEP_PAIR_PREFETCH;
        const bool lane_on = u < mp.U;
        EllRow<T, PF> aheadA, aheadB;
        Pk<T> pnA = pk_zero<T>(), pnB = pk_zero<T>(), xnA = pk_zero<T>(), xnB = pk_zero<T>();
        auto rows_ahead = [&](int64_t rA) {
            const int64_t rB = rA + stride;
            if (rA < a.n) ell_row_load<T, PF>(a.E, rA, aheadA);
            if (rB < a.n) ell_row_load<T, PF>(a.E, rB, aheadB);
            if (PRE >= 1 && lane_on && !a.first) {
                if (rA < a.n) pnA = ld(a.prev + (size_t)rA * mp.U + u);
                if (rB < a.n) pnB = ld(a.prev + (size_t)rB * mp.U + u);
            }
            if (PRE >= 2 && lane_on) {
                if (rA < a.n) xnA = ld(a.curr + (size_t)rA * mp.U + u);
                if (rB < a.n) xnB = ld(a.curr + (size_t)rB * mp.U + u);
            }
        };
        rows_ahead(first);
        for (int64_t row = first; row < a.n; row += 2 * stride) {
            const int64_t rowB = row + stride;
            const bool hasB = rowB < a.n;
            const EllRow<T, PF> curA = aheadA, curB = aheadB;
            const Pk<T> pcA = pnA, pcB = pnB, xcA = xnA, xcB = xnB;
            rows_ahead(row + 2 * stride);
            if (!lane_on) continue;
            const size_t oA = (size_t)row * mp.U + u, oB = (size_t)rowB * mp.U + u;
            const Pk<T> xA = PRE >= 2 ? xcA : ld(a.curr + oA);
            const Pk<T> pA = a.first ? pk_zero<T>() : PRE >= 1 ? pcA : ld(a.prev + oA);
            Pk<T> xB = pk_zero<T>(), pB = pk_zero<T>();
            if (hasB) {
                xB = PRE >= 2 ? xcB : ld(a.curr + oB);
                if (!a.first) pB = PRE >= 1 ? pcB : ld(a.prev + oB);
            }
            Pk<T> hA[1] = {pk_zero<T>()}, hB[1] = {pk_zero<T>()};
            gather_prefetched<T, 1, PF>(curA, a.curr, mp.U, mp.G, lane, hA);
            if (hasB) gather_prefetched<T, 1, PF>(curB, a.curr, mp.U, mp.G, lane, hB);
#pragma unroll
            for (int r2 = 0; r2 < 2; ++r2) {
                if (r2 == 1 && !hasB) break;
                const Pk<T> &x = r2 ? xB : xA;
                const Pk<T> &pv = r2 ? pB : pA;
                const Pk<T> &hv = r2 ? hB[0] : hA[0];
                Pk<T> nx;
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const T tr = rdiv(hv.re[c] - cen * x.re[c], hal, a.inv_half);
                    const T ti = rdiv(hv.im[c] - cen * x.im[c], hal, a.inv_half);
                    nx.re[c] = a.first ? tr : T(2) * tr - pv.re[c];
                    nx.im[c] = a.first ? ti : T(2) * ti - pv.im[c];
                    doubling_sums<T>(acc0[0][c].x, acc1[0][c].x, x.re[c], x.im[c], nx.re[c], nx.im[c], a.exact_sums);
                }
                st(a.next + (r2 ? oB : oA), nx);
            }
        }
    }
    constexpr bool SHARE = series_shares_v<T>() && MODE == MODE_SERIES && INLINE_V && MU == 1 &&
                           (HSRC == HSRC_ELL4 || HSRC == HSRC_ELL8);
    const bool share = SHARE && a.share_v;
    V *const vshare = reinterpret_cast<V *>(smem);
    int parity = 0;
    EllRow<T, PF> ahead;
    if (!step_pairs<T, MU, MODE, HSRC>() && (HSRC == HSRC_ELL4 || HSRC == HSRC_ELL8) &&
        (int64_t)blockIdx.x * mp.gpc + g < a.n)
        ell_row_load<T, PF>(a.E, (int64_t)blockIdx.x * mp.gpc + g, ahead);
    for (int64_t row = (int64_t)blockIdx.x * mp.gpc + g; !step_pairs<T, MU, MODE, HSRC>() && row < a.n; row += stride) {
        EllRow<T, PF> cur;
        if (HSRC == HSRC_ELL4 || HSRC == HSRC_ELL8) {
            cur = ahead;
            if (row + stride < a.n) ell_row_load<T, PF>(a.E, row + stride, ahead);
        }
        // Row-local operands first, so their latency overlaps the gathers
        // (the series accumulator too, when this row adds to it).
        Pk<T> xo[MU], po[MU], oo[MODE == MODE_SERIES ? MU : 1];
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
                const size_t o = (size_t)row * mp.U + u;
                xo[m] = ld(a.curr + o);
                po[m] = a.first ? pk_zero<T>() : ld(a.prev + o);
                if (MODE == MODE_SERIES && KMSD_SERIES_EARLY_OUT) oo[m] = a.first ? pk_zero<T>() : ld(a.out + o);
            }
        }
        Pk<T> h[MU];
        if (HSRC != HSRC_SOLVED) {
#pragma unroll
            for (int m = 0; m < MU; ++m) h[m] = pk_zero<T>();
            if constexpr (SHARE) {
                if (share)
                    gather_share_v<T, PF>(a, cur, row, lane, h[0],
                                          vshare + (size_t)parity * a.nvel * blockDim.x + threadIdx.x);
                else
                    gather_prefetched<T, MU, PF>(cur, a.curr, mp.U, mp.G, lane, h);
            } else if (HSRC == HSRC_ELL4 || HSRC == HSRC_ELL8) {
                gather_prefetched<T, MU, PF>(cur, a.curr, mp.U, mp.G, lane, h);
            } else if (HSRC == HSRC_ELL) {
                gather_row_ell<T, MU>(a.E, a.curr, row, mp.U, mp.G, lane, h);
            } else {
                gather_row<T, MU>(a.H, a.curr, row, mp.U, mp.G, lane, h);
            }
        }
        if (SHARE && share) group_sync(mp, g);
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u >= mp.U) continue;
            const size_t o = (size_t)row * mp.U + u;
            const Pk<T> x = xo[m];
            const Pk<T> hv = HSRC != HSRC_SOLVED ? h[m] : ld(a.hx + o);
            Pk<T> t;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                t.re[c] = rdiv(hv.re[c] - cen * x.re[c], hal, a.inv_half);
                t.im[c] = rdiv(hv.im[c] - cen * x.im[c], hal, a.inv_half);
            }
            if (MODE == MODE_SERIES && a.UR > 0 && u >= a.UR) {
                const int blk = u / a.UR - 1;  // phi block
                const int upsi = u - (blk + 1) * a.UR;
                if (INLINE_V) {
                    for (int v = 0; v < a.nvel; ++v) {
                        const T wr = a.wr[blk][v], wi = a.wi[blk][v];
                        if (wr == T(0) && wi == T(0)) continue;
                        Pk<T> vp;
                        if (SHARE && share) {
                            vp = ld(vshare + ((size_t)parity * a.nvel + v) * blockDim.x + g * mp.G + upsi);
                        } else if ((HSRC == HSRC_ELL4 || HSRC == HSRC_ELL8) && a.vform[v] == 2) {
                            vp = pk_zero<T>();
                            const T *vr = a.vel_re[v] + row * (4 * PF), *vi = a.vel_im[v] + row * (4 * PF);
#pragma unroll
                            for (int q = 0; q < PF; ++q) {
                                T r4[4], i4[4];
                                ld4(vr + 4 * q, r4);
                                ld4(vi + 4 * q, i4);
                                const int col[4] = {cur.idx[q].x, cur.idx[q].y, cur.idx[q].z, cur.idx[q].w};
#pragma unroll
                                for (int j = 0; j < 4; ++j)
                                    cmac_cplx(vp, r4[j], i4[j], ldg(a.curr + (size_t)col[j] * mp.U + upsi));
                            }
                        } else if (a.vform[v] == 1) {
                            vp = gather_commutator<T>(a.H, a.xdiag[v], a.curr, row, mp.U, upsi);
                        } else {
                            vp = gather_unit<T>(a.Vm[v], a.curr, row, mp.U, upsi);
                        }
#pragma unroll
                        for (int c = 0; c < C; ++c) {
                            t.re[c] += wr * vp.re[c] - wi * vp.im[c];
                            t.im[c] += wr * vp.im[c] + wi * vp.re[c];
                        }
                    }
                } else {
                    const Pk<T> v = ld(a.inj[blk] + (size_t)row * a.UR + upsi);
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        t.re[c] += a.injr * v.re[c] - a.inji * v.im[c];
                        t.im[c] += a.injr * v.im[c] + a.inji * v.re[c];
                    }
                }
            }
            Pk<T> nx;
            if (a.first) {
                nx = t;
            } else {
                const Pk<T> p = po[m];
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    nx.re[c] = T(2) * t.re[c] - p.re[c];
                    nx.im[c] = T(2) * t.im[c] - p.im[c];
                }
            }
            st(a.next + o, nx);
            if (MODE == MODE_CHAIN && a.store64 != nullptr) {
#pragma unroll
                for (int c = 0; c < C; ++c)
                    a.store64[o * C + c] = make_double2((double)nx.re[c], (double)nx.im[c]);
            }
            if (MODE == MODE_DIRECT) {
                const Pk<T> br = ld(a.bra + o);
#pragma unroll
                for (int c = 0; c < C; ++c)
                    acc0[m][c].x += (double)br.re[c] * (double)nx.re[c] + (double)br.im[c] * (double)nx.im[c];
            }
            if (MODE == MODE_DOUBLING) {
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    doubling_sums<T>(acc0[m][c].x, acc1[m][c].x, x.re[c], x.im[c], nx.re[c], nx.im[c], a.exact_sums);
                }
            }
            if (MODE == MODE_SERIES) {
                Pk<T> ov;
                if (a.first) {
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        ov.re[c] = a.c0r * x.re[c] - a.c0i * x.im[c] + a.ckr * nx.re[c] - a.cki * nx.im[c];
                        ov.im[c] = a.c0r * x.im[c] + a.c0i * x.re[c] + a.ckr * nx.im[c] + a.cki * nx.re[c];
                    }
                } else {
                    ov = KMSD_SERIES_EARLY_OUT ? oo[MODE == MODE_SERIES ? m : 0] : ld(a.out + o);
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        ov.re[c] += a.ckr * nx.re[c] - a.cki * nx.im[c];
                        ov.im[c] += a.ckr * nx.im[c] + a.cki * nx.re[c];
                    }
                }
#pragma unroll
                for (int c = 0; c < C; ++c) bad |= !isfinite(ov.re[c]) || !isfinite(ov.im[c]);
                st(a.out + o, ov);
            }
        }
        // the next row writes the other slice; this row's readers are done
        // with it once they reach the next row's barrier
        if (SHARE) parity ^= 1;
    }
    if (MODE == MODE_SERIES) {
        if (bad) atomicOr(a.status, 1);
    }
    if (MODE == MODE_DIRECT || MODE == MODE_DOUBLING) {
        const int ncol = mp.U * C;
        cta_column_sums<MU, C>(acc0, mp, ncol, smem, a.partial);
        if (MODE == MODE_DOUBLING)
            cta_column_sums<MU, C>(acc1, mp, ncol, smem, a.partial + (size_t)gridDim.x * ncol);
        if (last_cta(a.ticket)) {
            double2 *tot = smem;  // scratch of blockDim.x entries for the final combine
            __shared__ double2 outbuf[512];  // ncol <= 8 units * 32 lanes * 2 columns
            final_column_sums(a.partial, gridDim.x, ncol, tot, outbuf);
            if (MODE == MODE_DIRECT) {
                for (int j = threadIdx.x; j < a.bcols; j += blockDim.x)
                    a.mu[(size_t)a.kmom * a.bcols + j] = outbuf[j].x;
            } else {
                __syncthreads();
                // outbuf holds the even sums; stage them before computing odd sums
                __shared__ double even[512];
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
        }
    }
}

// ------------------------------------------------------------ sampling
// One Clenshaw step of the metric sampler (Metric::sample, native.cpp:453-479):
//   act = (z .* S (z .* b1) - center b1) / half
//   FINAL = 0: b0 = 2 act - b2 + c xi   (written over b2)
//   FINAL = 1: out = z .* (act - b2 + c xi)
template <int FINAL>
__global__ void __launch_bounds__(256) clenshaw_kernel(CsrView<double> S, const double *z, const double2 *b1,
                                                       double2 *b2, const double2 *xi, double2 *out,
                                                       double coef, double center, double half,
                                                       int64_t n, RowMap mp) {
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    for (int64_t row = (int64_t)blockIdx.x * mp.gpc + g; row < n; row += (int64_t)gridDim.x * mp.gpc) {
        const int k0 = __ldg(S.ptr + row), k1 = __ldg(S.ptr + row + 1);
        const double zr = __ldg(z + row);
        for (int u = lane; u < mp.U; u += mp.G) {
            double sr = 0., si = 0.;
            for (int k = k0; k < k1; ++k) {
                const int col = __ldg(S.idx + k);
                const double zc = __ldg(z + col);
                const double2 bv = __ldg(b1 + (size_t)col * mp.U + u);
                const double xr = bv.x * zc, xi_ = bv.y * zc;
                const double vr = __ldg(S.re + k), vi = S.im ? __ldg(S.im + k) : 0.;
                sr += vr * xr - vi * xi_;
                si += vr * xi_ + vi * xr;
            }
            const size_t o = (size_t)row * mp.U + u;
            const double2 b = b1[o];
            const double ar = (zr * sr - center * b.x) / half;
            const double ai = (zr * si - center * b.y) / half;
            const double2 p2 = b2[o];
            const double2 x = xi[o];
            if (FINAL == 0) {
                b2[o] = make_double2(2. * ar - p2.x + coef * x.x, 2. * ai - p2.y + coef * x.y);
            } else {
                out[o] = make_double2(zr * (ar - p2.x + coef * x.x), zr * (ai - p2.y + coef * x.y));
            }
        }
    }
}

// ------------------------------------------------------------ conversions
static __global__ void to_f32_kernel(const double2 *src, float4 *dst, int64_t n, int bsrc, int upad) {
    // src: (n, bsrc) complex128; dst: (n, upad) float4 units (2 complex each),
    // zero-padding columns >= bsrc.
    const int64_t total = n * upad;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = i / upad;
        const int u = (int)(i - row * upad);
        const int j0 = 2 * u, j1 = 2 * u + 1;
        const double2 a = j0 < bsrc ? src[row * bsrc + j0] : make_double2(0., 0.);
        const double2 b = j1 < bsrc ? src[row * bsrc + j1] : make_double2(0., 0.);
        dst[i] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
    }
}
static __global__ void to_f64_kernel(const float4 *src, double2 *dst, int64_t n, int bdst, int upad) {
    const int64_t total = n * (int64_t)bdst;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = i / bdst;
        const int j = (int)(i - row * bdst);
        const float4 v = src[row * upad + j / 2];
        dst[i] = (j & 1) ? make_double2(v.z, v.w) : make_double2(v.x, v.y);
    }
}

// Strided column-slice copy: dst(n, bd) = src(n, bs)[:, off:off+bd] (complex128).
static __global__ void slice_kernel(const double2 *src, double2 *dst, int64_t n, int bs, int off, int bd) {
    const int64_t total = n * (int64_t)bd;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = i / bd;
        const int j = (int)(i - row * bd);
        dst[i] = src[row * bs + off + j];
    }
}

// y = sum_m coef_m * x_m over complex128 arrays of `len` elements (up to 4 terms;
// y may alias one of the inputs only if it is read at the same index).
struct Lincomb {
    const double2 *x[4];
    double cr[4], ci[4];
    int terms;
    int accumulate;  // y += ... instead of y = ...
};
static __global__ void lincomb_kernel(Lincomb L, double2 *y, int64_t len) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
         i += (int64_t)gridDim.x * blockDim.x) {
        double sr = 0., si = 0.;
        if (L.accumulate) {
            const double2 v = y[i];
            sr = v.x;
            si = v.y;
        }
        for (int t = 0; t < L.terms; ++t) {
            const double2 v = L.x[t][i];
            sr += L.cr[t] * v.x - L.ci[t] * v.y;
            si += L.cr[t] * v.y + L.ci[t] * v.x;
        }
        y[i] = make_double2(sr, si);
    }
}

// Nonfinite scan: status |= 1 if any element is nonfinite.
static __global__ void finite_scan_kernel(const double2 *x, int64_t len, int *status) {
    bool bad = false;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = x[i];
        bad |= !isfinite(v.x) || !isfinite(v.y);
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, 1);
}

}  // namespace kmsd
