// Shared device/host definitions of the B200 stochastic-KPM engine.
//
// Vector blocks are row-major (N, b) complex arrays (the layout of the
// reference's Dense, cpp/native.cpp:26-41).  Device code moves them in
// 16-byte "units": one complex128 (double2) or two complex64 (float4), so
// every global access is a 128-bit load or store.  A row of b columns is
// U = b / C units; a "row group" of G threads (G = next power of two >= U,
// at most 128) walks rows with a grid stride, each lane owning the units
// lane, lane + G, ... of the row.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

namespace kmsd {

// ---------------------------------------------------------------- units
template <class T> struct Unit;
template <> struct Unit<double> {
    using vec = double2;
    static constexpr int C = 1;  // complex numbers per unit
};
template <> struct Unit<float> {
    using vec = float4;
    static constexpr int C = 2;
};

// C complex numbers of precision T held in registers.
template <class T> struct Pk {
    static constexpr int C = Unit<T>::C;
    T re[C], im[C];
};

__device__ __forceinline__ Pk<double> ld(const double2 *p) {
    double2 v = *p;
    Pk<double> r;
    r.re[0] = v.x; r.im[0] = v.y;
    return r;
}
__device__ __forceinline__ Pk<float> ld(const float4 *p) {
    float4 v = *p;
    Pk<float> r;
    r.re[0] = v.x; r.im[0] = v.y; r.re[1] = v.z; r.im[1] = v.w;
    return r;
}
// Read-only (non-coherent) path for gathered operands.
__device__ __forceinline__ Pk<double> ldg(const double2 *p) {
    double2 v = __ldg(p);
    Pk<double> r;
    r.re[0] = v.x; r.im[0] = v.y;
    return r;
}
__device__ __forceinline__ Pk<float> ldg(const float4 *p) {
    float4 v = __ldg(p);
    Pk<float> r;
    r.re[0] = v.x; r.im[0] = v.y; r.re[1] = v.z; r.im[1] = v.w;
    return r;
}
__device__ __forceinline__ void st(double2 *p, const Pk<double> &a) {
    *p = make_double2(a.re[0], a.im[0]);
}
__device__ __forceinline__ void st(float4 *p, const Pk<float> &a) {
    *p = make_float4(a.re[0], a.im[0], a.re[1], a.im[1]);
}

// ------------------------------------------------------- CG work-vector storage
// The work vectors of the metric solve (r, z, p, S p, t) are stored as
// complex128 or, in the mixed form, complex64; every operation on them is
// FP64.  stored<W>(v) is v as it reads back after stw into W.
__device__ __forceinline__ double2 ldw(const double2 *p) { return *p; }
__device__ __forceinline__ double2 ldw(const float2 *p) {
    const float2 v = *p;
    return make_double2(v.x, v.y);
}
__device__ __forceinline__ void stw(double2 *p, double2 v) { *p = v; }
__device__ __forceinline__ void stw(float2 *p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }
template <class W> __device__ __forceinline__ double2 stored(double2 v) {
    if constexpr (sizeof(W) == sizeof(float2)) return make_double2((double)(float)v.x, (double)(float)v.y);
    else return v;
}
// Read-only gathers of either storage into FP64 registers.
__device__ __forceinline__ Pk<double> ldg_d(const double2 *p) { return ldg(p); }
__device__ __forceinline__ Pk<double> ldg_d(const float2 *p) {
    const float2 v = __ldg(p);
    Pk<double> r;
    r.re[0] = v.x;
    r.im[0] = v.y;
    return r;
}

template <class T> __device__ __forceinline__ Pk<T> pk_zero() {
    Pk<T> r;
#pragma unroll
    for (int c = 0; c < Pk<T>::C; ++c) { r.re[c] = T(0); r.im[c] = T(0); }
    return r;
}

// CSR matrix on the device with values in the vector precision T.
template <class T> struct CsrView {
    const int *ptr;
    const int *idx;
    const T *re;
    const T *im;  // nullptr for a real matrix
};

// The same matrix as a row-major ELL block [n][w] (w a multiple of 4; short
// rows padded with zero values pointing at their own row), so a row's
// indices and values are 16-byte vector loads and no row pointer is read.
template <class T> struct EllView {
    const int *idx;
    const T *re;
    const T *im;  // nullptr for a real matrix
    int w;        // 0: no ELL form
};

// The same matrix as block CSR with dense 4x4 blocks (the atom blocks of an
// sp3 basis): block row I covers rows 4I..4I+3; each block's 16 values are
// stored row-major, absent entries as zeros.  nbrows == 0 when not built.
template <class T> struct BsrView {
    const int *bptr;  // nbrows + 1
    const int *bidx;  // block column of each block
    const T *re;      // 16 values per block
    const T *im;      // nullptr for a real matrix
    int64_t nbrows;
};

// ---------------------------------------------------------------- mapping
struct RowMap {
    int G;      // threads per row group (power of two, <= 128)
    int gpc;    // row groups per CTA
    int U;      // units per row
};

inline int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}
// Row groups span up to four warps (G <= 128), so rows of up to 128 units
// keep one unit per lane; wider rows give each lane several units.
inline RowMap make_map(int U, int threads) {
    RowMap m;
    m.U = U;
    m.G = U >= 128 ? 128 : next_pow2(U < 1 ? 1 : U);
    m.gpc = threads / m.G;
    return m;
}

// ---------------------------------------------------------------- reductions
// Column reductions are deterministic: a fixed grid, fixed row ownership, a
// fixed-order shared-memory combination inside each CTA, and a fixed-order
// combination of the per-CTA partials by the last CTA to finish (found with
// an atomic ticket; no spinning on other CTAs).
struct Ticket {
    unsigned int count;
};

// Each thread holds `acc[m][c]` for its units u = lane + m*G (m < MU) and the
// C columns of each unit.  Writes the CTA's per-column sums to dst[col]
// (the CTA's row of a partial-sum array).  smem needs gpc * U * C double2.
template <int MU, int C>
__device__ __forceinline__ void cta_column_sums_at(const double2 (&acc)[MU][C], const RowMap &mp,
                                                   int ncol, double2 *smem, double2 *dst) {
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    if (g < mp.gpc) {
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
#pragma unroll
                for (int c = 0; c < C; ++c) smem[(g * mp.U + u) * C + c] = acc[m][c];
            }
        }
    }
    __syncthreads();
    for (int col = threadIdx.x; col < ncol; col += blockDim.x) {
        double sx = 0., sy = 0.;
        for (int gg = 0; gg < mp.gpc; ++gg) {
            const double2 v = smem[gg * mp.U * C + col];
            sx += v.x;
            sy += v.y;
        }
        dst[col] = make_double2(sx, sy);
    }
    __syncthreads();
}

// The same, written to partial[blockIdx.x * ncol + col].
template <int MU, int C>
__device__ __forceinline__ void cta_column_sums(const double2 (&acc)[MU][C], const RowMap &mp,
                                                int ncol, double2 *smem, double2 *partial) {
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    if (g < mp.gpc) {
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
#pragma unroll
                for (int c = 0; c < C; ++c) smem[(g * mp.U + u) * C + c] = acc[m][c];
            }
        }
    }
    __syncthreads();
    for (int col = threadIdx.x; col < ncol; col += blockDim.x) {
        double sx = 0., sy = 0.;
        for (int gg = 0; gg < mp.gpc; ++gg) {
            const double2 v = smem[gg * mp.U * C + col];
            sx += v.x;
            sy += v.y;
        }
        partial[(size_t)blockIdx.x * ncol + col] = make_double2(sx, sy);
    }
    __syncthreads();
}

// Same for a max reduction of one double per column.
template <int MU, int C>
__device__ __forceinline__ void cta_column_max(const double (&acc)[MU][C], const RowMap &mp, int ncol,
                                               double *smem, double *partial) {
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    if (g < mp.gpc) {
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
#pragma unroll
                for (int c = 0; c < C; ++c) smem[(g * mp.U + u) * C + c] = acc[m][c];
            }
        }
    }
    __syncthreads();
    for (int col = threadIdx.x; col < ncol; col += blockDim.x) {
        double s = 0.;
        for (int gg = 0; gg < mp.gpc; ++gg) s = fmax(s, smem[gg * mp.U * C + col]);
        partial[(size_t)blockIdx.x * ncol + col] = s;
    }
    __syncthreads();
}

// Returns true in exactly one CTA (the last to arrive), after all other CTAs'
// partials are visible.  Resets the ticket for the next launch.
__device__ __forceinline__ bool last_cta(Ticket *t) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned prev = atomicAdd(&t->count, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        if (threadIdx.x == 0) t->count = 0;
    }
    return is_last;
}

// Inside the last CTA: out[col] = sum over CTAs (fixed order) of partial.
// Uses all threads: the CTAs are split into `split` fixed contiguous ranges
// per column, combined in a fixed order through shared memory.
__device__ __forceinline__ void final_column_sums(const double2 *partial, int nparts, int ncol,
                                                  double2 *smem /* blockDim.x */, double2 *out) {
    // Process columns in chunks of at most blockDim.x.
    for (int c0 = 0; c0 < ncol; c0 += blockDim.x) {
        const int cols = min((int)blockDim.x, ncol - c0);
        const int split = max(1, (int)blockDim.x / cols);
        const int col = threadIdx.x % cols, part = threadIdx.x / cols;
        double sx = 0., sy = 0.;
        if (part < split) {
            const int per = (nparts + split - 1) / split;
            const int lo = part * per, hi = min(nparts, lo + per);
            // four independent chains keep four loads in flight; they are
            // combined in a fixed order, so the sum does not depend on timing
            double ax[4] = {0., 0., 0., 0.}, ay[4] = {0., 0., 0., 0.};
            int p = lo;
            for (; p + 4 <= hi; p += 4) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double2 v = __ldcg(partial + (size_t)(p + q) * ncol + c0 + col);
                    ax[q] += v.x;
                    ay[q] += v.y;
                }
            }
            for (; p < hi; ++p) {
                const double2 v = __ldcg(partial + (size_t)p * ncol + c0 + col);
                ax[0] += v.x;
                ay[0] += v.y;
            }
            sx = (ax[0] + ax[1]) + (ax[2] + ax[3]);
            sy = (ay[0] + ay[1]) + (ay[2] + ay[3]);
        }
        __syncthreads();
        if (part < split) smem[part * cols + col] = make_double2(sx, sy);
        __syncthreads();
        if (threadIdx.x < cols) {
            double tx = 0., ty = 0.;
            for (int p = 0; p < split; ++p) {
                const double2 v = smem[p * cols + threadIdx.x];
                tx += v.x;
                ty += v.y;
            }
            out[c0 + threadIdx.x] = make_double2(tx, ty);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void final_column_max(const double *partial, int nparts, int ncol,
                                                 double *out) {
    for (int col = threadIdx.x; col < ncol; col += blockDim.x) {
        double s = 0.;
#pragma unroll 8
        for (int p = 0; p < nparts; ++p) s = fmax(s, __ldcg(partial + (size_t)p * ncol + col));
        out[col] = s;
    }
}

// ------------------------------------------------------- two-level combination
// In a short kernel (one PCG iteration on a few 10^4 rows takes
// microseconds) a last CTA that reads all ~10^3 partial rows is the critical
// path.  Instead the CTAs form groups of kTreeFan consecutive CTAs: the last
// CTA of a group to arrive combines the group's rows in a fixed order into a
// level-2 row partial[(gridDim.x + group) * ncol + col], and the last group
// to arrive combines the level-2 rows in a fixed order into out.  The result
// is the same in every run, and each step reads at most kTreeFan rows per
// column.  Tickets: tk[0] for the root, tk[1 + group] per group; all are
// left at zero.  The partial array needs tree_rows(gridDim.x) rows.
constexpr int kTreeFan = 32;
constexpr int kTreeTickets = 1024;  // tickets in a reduction's ticket array
__host__ __device__ inline int tree_rows(int grid) { return grid + (grid + kTreeFan - 1) / kTreeFan; }

// True in the CTA that is the `expected`-th to arrive at ticket t; its reads
// after the return see every arrived CTA's writes.  Resets the ticket.
__device__ __forceinline__ bool arrive_last(Ticket *t, unsigned expected) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(&t->count, 1u) == expected - 1;
    __syncthreads();
    if (is_last) {
        __threadfence();
        if (threadIdx.x == 0) t->count = 0;
    }
    return is_last;
}

// The same over the consecutive CTAs [c0, c0 + nct) of one range (a segment
// of a segmented solve), this CTA being c0 + lc: tickets tks[0] (root) and
// tks[1 + group], level-2 rows level2[group * ncol].  Returns true in the CTA
// that holds the range's totals in out.
__device__ __forceinline__ bool range_column_sums(double2 *partial, int ncol, int c0, int nct, int lc, Ticket *tks,
                                                  double2 *level2, double2 *smem, double2 *out) {
    const int ngroups = (nct + kTreeFan - 1) / kTreeFan;
    if (ngroups == 1) {
        if (!arrive_last(tks, nct)) return false;
        final_column_sums(partial + (size_t)c0 * ncol, nct, ncol, smem, out);
        return true;
    }
    const int group = lc / kTreeFan, lo = group * kTreeFan, cnt = min(kTreeFan, nct - lo);
    if (!arrive_last(tks + 1 + group, cnt)) return false;
    final_column_sums(partial + (size_t)(c0 + lo) * ncol, cnt, ncol, smem, level2 + (size_t)group * ncol);
    if (!arrive_last(tks, ngroups)) return false;
    final_column_sums(level2, ngroups, ncol, smem, out);
    return true;
}

__device__ __forceinline__ bool range_column_max(double *partial, int ncol, int c0, int nct, int lc, Ticket *tks,
                                                 double *level2, double *out) {
    const int ngroups = (nct + kTreeFan - 1) / kTreeFan;
    if (ngroups == 1) {
        if (!arrive_last(tks, nct)) return false;
        final_column_max(partial + (size_t)c0 * ncol, nct, ncol, out);
        return true;
    }
    const int group = lc / kTreeFan, lo = group * kTreeFan, cnt = min(kTreeFan, nct - lo);
    if (!arrive_last(tks + 1 + group, cnt)) return false;
    final_column_max(partial + (size_t)(c0 + lo) * ncol, cnt, ncol, level2 + (size_t)group * ncol);
    __syncthreads();
    if (!arrive_last(tks, ngroups)) return false;
    final_column_max(level2, ngroups, ncol, out);
    return true;
}

// Tickets a range of nct CTAs uses.
__host__ __device__ inline int range_tickets(int nct) {
    const int ngroups = (nct + kTreeFan - 1) / kTreeFan;
    return ngroups == 1 ? 1 : 1 + ngroups;
}

__device__ __forceinline__ bool tree_column_sums(double2 *partial, int ncol, Ticket *tk, double2 *smem,
                                                 double2 *out) {
    return range_column_sums(partial, ncol, 0, gridDim.x, blockIdx.x, tk, partial + (size_t)gridDim.x * ncol, smem,
                             out);
}

__device__ __forceinline__ bool tree_column_max(double *partial, int ncol, Ticket *tk, double *out) {
    return range_column_max(partial, ncol, 0, gridDim.x, blockIdx.x, tk, partial + (size_t)gridDim.x * ncol, out);
}

// ---------------------------------------------------------------- host errors
struct Error {
    int code;
    std::string msg;
};

}  // namespace kmsd
