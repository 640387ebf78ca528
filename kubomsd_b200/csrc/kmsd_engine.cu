// Transport engine of the B200 stochastic-KPM backend: sparse matrices, the
// operator applications of the reference Engine (cpp/native.cpp:488-610) and
// the C ABI around them.
//
// Two execution paths:
//  * identity metric (orthogonal basis, S = I with unit diagonal): every
//    Chebyshev step is ONE fused kernel (cheb_step_kernel) that streams the
//    vector block once — SpMM of H, spectral rescaling, three-term recurrence,
//    velocity injection and the moment / series epilogue — in FP64 or in the
//    mixed form (complex64 vectors, FP64 accumulations);
//  * general metric: H X (SpMM), S^-1 by the batched PCG of kmsd_metric.cu,
//    then the same step kernel reading the solved operand (FP64 only).
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <utility>
#include <vector>

#include "kmsd.h"
#include "kmsd_impl.h"
#include "kmsd_kernels.cuh"

using namespace kmsd;

// ------------------------------------------------------------------ errors
namespace {
thread_local std::string g_last_error;
}
namespace kmsd {
int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char *what) {
    g_last_error = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " + what;
    return KMSD_ECUDA;
}
int DevBuf::ensure(size_t want) {
    if (want <= bytes && p) return 0;
    release();
    if (want == 0) want = 16;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        cuda_fail(e, "cudaMalloc (workspace)");
        return 1;
    }
    bytes = want;
    return 0;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}
static std::atomic<int64_t> g_launches{0};
static thread_local int g_count_off = 0;
static thread_local int64_t g_recorded = 0;
void count_launch(int64_t n) {
    if (g_count_off) g_recorded += n;
    else g_launches.fetch_add(n, std::memory_order_relaxed);
}
CountOff::CountOff() : start(g_recorded) { ++g_count_off; }
CountOff::~CountOff() { --g_count_off; }
int64_t CountOff::recorded() const { return g_recorded - start; }
int64_t launches() { return g_launches.load(std::memory_order_relaxed); }
int sm_count() {
    // initialised once, thread-safely, on the first call
    static const int cached = [] {
        int dev = 0, count = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        return count > 0 ? count : 148;
    }();
    return cached;
}
int grid_for(int64_t rows, const RowMap &mp) {
    const int64_t need = (rows + mp.gpc - 1) / mp.gpc;
    const int64_t cap = (int64_t)sm_count() * 8;  // 8 CTAs of 256 threads per SM
    return (int)std::max<int64_t>(1, std::min(need, cap));
}
int wave_grid(const void *kernel, size_t smem, int64_t rows, const RowMap &mp) {
    static std::mutex lock;
    static std::map<std::pair<const void *, size_t>, int> cache;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> g(lock);
        auto it = cache.find({kernel, smem});
        if (it != cache.end()) {
            per_sm = it->second;
        } else {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem) != cudaSuccess ||
                per_sm < 1)
                per_sm = 1;
            cache[{kernel, smem}] = per_sm;
        }
    }
    const int64_t need = (rows + mp.gpc - 1) / mp.gpc;
    return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sm_count() * per_sm));
}
int mu_for(const RowMap &mp) {
    // At most 256 units (512 reduction columns) per launch: the fixed-size
    // shared buffers of the reductions are sized for that.  Row groups are up
    // to 128 lanes wide, so a lane holds one or two units.
    if (mp.U > 256) return 0;
    const int per = (mp.U + mp.G - 1) / mp.G;
    if (per <= 1) return 1;
    if (per <= 2) return 2;
    return 0;
}
size_t reduce_smem(const RowMap &mp, int C) {
    const size_t a = (size_t)mp.gpc * mp.U * C, b = kThreads;
    return std::max(a, b) * sizeof(double2);
}
int Reducer::ensure(int grid, int ncol, int copies) {
    if (partial.ensure((size_t)tree_rows(grid) * ncol * copies * sizeof(double2) + 64)) return KMSD_ECUDA;
    if (!ticket.p) {
        if (ticket.ensure(kTreeTickets * sizeof(Ticket))) return KMSD_ECUDA;
        KMSD_CUDA(cudaMemset(ticket.p, 0, kTreeTickets * sizeof(Ticket)));
    }
    return KMSD_OK;
}
}  // namespace kmsd

// ------------------------------------------------------------------ CSR
// The complex64 copies of an uploaded matrix, built on first use.  Engine
// replicas on several host threads share one matrix, so the build runs under
// one lock and the pointers are published only once their values are on the
// device: a second caller never sees an allocated but unfilled copy.
int kmsd_csr_s::ensure_f32() {
    static std::mutex lock;
    std::lock_guard<std::mutex> guard(lock);
    if (re32) return KMSD_OK;
    float *dre = nullptr, *dim = nullptr, *dere = nullptr, *deim = nullptr;
    auto fail_free = [&](cudaError_t err) {
        for (float *q : {dre, dim, dere, deim})
            if (q) cudaFree(q);
        return fail(KMSD_ECUDA, cudaGetErrorString(err));
    };
    // d = (float) src for `count` values of a device FP64 array
    auto convert = [&](const double *src, int64_t count, float **d) -> cudaError_t {
        std::vector<double> h(std::max<int64_t>(count, 1));
        std::vector<float> f(h.size());
        cudaError_t err = cudaMemcpy(h.data(), src, count * sizeof(double), cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) return err;
        for (int64_t i = 0; i < count; ++i) f[i] = (float)h[i];
        if ((err = cudaMalloc(d, f.size() * sizeof(float))) != cudaSuccess) return err;
        return cudaMemcpy(*d, f.data(), count * sizeof(float), cudaMemcpyHostToDevice);
    };
    cudaError_t err = convert(re64, nnz, &dre);
    if (err == cudaSuccess && complex_values) err = convert(im64, nnz, &dim);
    if (err == cudaSuccess && ell_w > 0) {
        err = convert(ell_re64, n * ell_w, &dere);
        if (err == cudaSuccess && complex_values) err = convert(ell_im64, n * ell_w, &deim);
    }
    if (err != cudaSuccess) return fail_free(err);
    im32 = dim;
    ell_re32 = dere;
    ell_im32 = deim;
    re32 = dre;  // last: the copy counts as built once re32 is set
    return KMSD_OK;
}

namespace {
template <class T, int MU, bool DOT>
void launch_spmm(CsrView<T> A, const typename Unit<T>::vec *X, typename Unit<T>::vec *Y, int64_t n, RowMap mp,
                 Reducer &red, double2 *dot, cudaStream_t s) {
    const int grid = grid_for(n, mp);
    spmm_kernel<T, MU, DOT><<<grid, kThreads, reduce_smem(mp, Unit<T>::C), s>>>(A, X, Y, n, mp, red.part(),
                                                                               red.tick(), dot);
    count_launch();
}
template <class T>
int spmm_any(CsrView<T> A, const typename Unit<T>::vec *X, typename Unit<T>::vec *Y, int64_t n, int U,
             cudaStream_t s, double2 *dot) {
    static thread_local Reducer red;
    const RowMap mp = make_map(U, kThreads);
    const int mu = mu_for(mp);
    if (!mu) return fail(KMSD_EINVAL, "too many columns for one SpMM call");
    if (red.ensure(grid_for(n, mp), U * Unit<T>::C)) return KMSD_ECUDA;
#define KMSD_SPMM_CASE(M)                                                      \
    case M:                                                                    \
        if (dot) launch_spmm<T, M, true>(A, X, Y, n, mp, red, dot, s);         \
        else launch_spmm<T, M, false>(A, X, Y, n, mp, red, nullptr, s);        \
        break;
    switch (mu) {
        KMSD_SPMM_CASE(1)
        KMSD_SPMM_CASE(2)
    }
#undef KMSD_SPMM_CASE
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}
}  // namespace

namespace kmsd {
int spmm64(const kmsd_csr_s *A, const double2 *X, double2 *Y, int64_t b, cudaStream_t s, double2 *dot_out) {
    if (A->bsr_nb > 0) {
        static thread_local Reducer red;
        const RowMap mp = make_map((int)b, kThreads);
        const int mu = mu_for(mp);
        if (!mu) return fail(KMSD_EINVAL, "too many columns for one SpMM call");
        const int grid = grid_for(A->bsr_nb, mp);
        if (red.ensure(grid, (int)b)) return KMSD_ECUDA;
        const size_t sm = reduce_smem(mp, 1);
        const BsrView<double> v = A->bsr64();
        const bool cplx = v.im != nullptr;
#define KMSD_BSR_LAUNCH(M, D, Z) \
    spmm_bsr_kernel<M, D, Z><<<grid, kThreads, sm, s>>>(v, X, Y, mp, red.part(), red.tick(), D ? dot_out : nullptr)
#define KMSD_BSR_CASE(M)                              \
    case M:                                           \
        if (dot_out) {                                \
            if (cplx) KMSD_BSR_LAUNCH(M, true, true); \
            else KMSD_BSR_LAUNCH(M, true, false);     \
        } else {                                      \
            if (cplx) KMSD_BSR_LAUNCH(M, false, true); \
            else KMSD_BSR_LAUNCH(M, false, false);    \
        }                                             \
        break;
        switch (mu) {
            KMSD_BSR_CASE(1)
            KMSD_BSR_CASE(2)
        }
#undef KMSD_BSR_CASE
#undef KMSD_BSR_LAUNCH
        count_launch();
        KMSD_CUDA(cudaGetLastError());
        return KMSD_OK;
    }
    return spmm_any<double>(A->view64(), X, Y, A->n, (int)b, s, dot_out);
}
int spmm32(const kmsd_csr_s *A, const float4 *X, float4 *Y, int64_t U, cudaStream_t s, double2 *dot_out) {
    return spmm_any<float>(A->view32(), X, Y, A->n, (int)U, s, dot_out);
}
int lincomb(cudaStream_t s, double2 *y, int64_t len, int accumulate, int terms, const double2 *const *x,
            const double *cr, const double *ci) {
    Lincomb L{};
    L.terms = terms;
    L.accumulate = accumulate;
    for (int t = 0; t < terms; ++t) {
        L.x[t] = x[t];
        L.cr[t] = cr[t];
        L.ci[t] = ci[t];
    }
    const int grid = (int)std::min<int64_t>((len + 255) / 256, (int64_t)sm_count() * 16);
    lincomb_kernel<<<std::max(grid, 1), 256, 0, s>>>(L, y, len);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}
}  // namespace kmsd

// ------------------------------------------------------------------ column dot
namespace {
// out[j] = sum_i conj(x_ij) y_ij (complex, double2), deterministic.
template <class T, int MU>
__global__ void __launch_bounds__(256) coldot_kernel(const typename Unit<T>::vec *x, const typename Unit<T>::vec *y,
                                                     int64_t n, RowMap mp, double2 *partial, Ticket *tk,
                                                     double2 *out) {
    constexpr int C = Unit<T>::C;
    extern __shared__ double2 smem[];
    const int g = threadIdx.x / mp.G, lane = threadIdx.x % mp.G;
    double2 acc[MU][C];
#pragma unroll
    for (int m = 0; m < MU; ++m)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[m][c] = make_double2(0., 0.);
    for (int64_t row = (int64_t)blockIdx.x * mp.gpc + g; row < n; row += (int64_t)gridDim.x * mp.gpc) {
#pragma unroll
        for (int m = 0; m < MU; ++m) {
            const int u = lane + m * mp.G;
            if (u < mp.U) {
                const size_t o = (size_t)row * mp.U + u;
                const Pk<T> a = ld(x + o), b = ld(y + o);
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    acc[m][c].x += (double)a.re[c] * b.re[c] + (double)a.im[c] * b.im[c];
                    acc[m][c].y += (double)a.re[c] * b.im[c] - (double)a.im[c] * b.re[c];
                }
            }
        }
    }
    const int ncol = mp.U * C;
    cta_column_sums<MU, C>(acc, mp, ncol, smem, partial);
    tree_column_sums(partial, ncol, tk, smem, out);
}

template <class T>
int coldot_any(const typename Unit<T>::vec *x, const typename Unit<T>::vec *y, int64_t n, int U, double2 *out,
               cudaStream_t s) {
    static thread_local Reducer red;
    const RowMap mp = make_map(U, kThreads);
    const int mu = mu_for(mp);
    if (!mu) return fail(KMSD_EINVAL, "too many columns for one reduction");
    const int grid = grid_for(n, mp);
    if (red.ensure(grid, U * Unit<T>::C)) return KMSD_ECUDA;
    const size_t sm = reduce_smem(mp, Unit<T>::C);
    switch (mu) {
        case 1: coldot_kernel<T, 1><<<grid, kThreads, sm, s>>>(x, y, n, mp, red.part(), red.tick(), out); break;
        case 2: coldot_kernel<T, 2><<<grid, kThreads, sm, s>>>(x, y, n, mp, red.part(), red.tick(), out); break;
    }
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

__global__ void take_real_kernel(const double2 *src, double *dst, int n) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) dst[j] = src[j].x;
}
}  // namespace

namespace kmsd {
int coldot64(const double2 *x, const double2 *y, int64_t n, int64_t b, double2 *out, cudaStream_t s) {
    return coldot_any<double>(x, y, n, (int)b, out, s);
}
int coldot32(const float4 *x, const float4 *y, int64_t n, int64_t U, double2 *out, cudaStream_t s) {
    return coldot_any<float>(x, y, n, (int)U, out, s);
}
int take_real(const double2 *src, double *dst, int64_t b, cudaStream_t s) {
    take_real_kernel<<<1, 256, 0, s>>>(src, dst, (int)b);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}
}  // namespace kmsd

// ------------------------------------------------------------------ CSR ABI
extern "C" {

const char *kmsd_last_error(void) { return g_last_error.c_str(); }

int64_t kmsd_kernel_launches(void) { return launches() + device_loop_launches(); }

const char *kmsd_build_info(void) {
    return "{\"language\": \"C++17/CUDA\", \"architecture\": \"sm_100a\", "
           "\"precision\": \"complex128/float64 (FP64) or complex64 vectors with float64 accumulation (MIXED)\", "
           "\"implementation\": \"fused CSR SpMM + Chebyshev recurrence kernels, batched device PCG\"}";
}

int kmsd_device(int *device) {
    if (!device) return fail(KMSD_EINVAL, "null device pointer");
    KMSD_CUDA(cudaGetDevice(device));
    return KMSD_OK;
}

int kmsd_csr_create(int64_t n, const int64_t *indptr, const int64_t *indices, const double *val_re,
                    const double *val_im, kmsd_csr *out) {
    if (!out || n < 1 || !indptr) return fail(KMSD_EINVAL, "invalid CSR dimensions/threads");
    const int64_t nnz = indptr[n];
    if (indptr[0] != 0 || nnz < 0) return fail(KMSD_EINVAL, "invalid CSR row pointers");
    if (nnz > 0 && (!indices || !val_re)) return fail(KMSD_EINVAL, "invalid CSR dimensions/threads");
    for (int64_t r = 0; r < n; ++r)
        if (indptr[r] > indptr[r + 1]) return fail(KMSD_EINVAL, "nonmonotone CSR row pointers");
    for (int64_t k = 0; k < nnz; ++k)
        if (indices[k] < 0 || indices[k] >= n || !std::isfinite(val_re[k]) ||
            (val_im && !std::isfinite(val_im[k])))
            return fail(KMSD_EINVAL, "invalid CSR index or nonfinite entry");
    if (n >= INT32_MAX || nnz >= INT32_MAX) return fail(KMSD_EINVAL, "CSR too large for 32-bit indices");
    bool cplx = false;
    if (val_im)
        for (int64_t k = 0; k < nnz && !cplx; ++k) cplx = val_im[k] != 0.;
    bool ident = nnz == n;
    for (int64_t r = 0; r < n && ident; ++r)
        ident = indptr[r] == r && indices[r] == r && val_re[r] == 1. && (!val_im || val_im[r] == 0.);
    std::vector<int> p32(n + 1), i32(std::max<int64_t>(nnz, 1));
    for (int64_t r = 0; r <= n; ++r) p32[r] = (int)indptr[r];
    for (int64_t k = 0; k < nnz; ++k) i32[k] = (int)indices[k];
    auto *A = new kmsd_csr_s();
    A->n = n;
    A->nnz = nnz;
    A->complex_values = cplx;
    A->identity = ident;
    bool diag = nnz == n && !cplx;
    for (int64_t r = 0; r < n && diag; ++r) diag = indptr[r] == r && indices[r] == r;
    A->diagonal = diag;
    cudaGetDevice(&A->device);
    auto up = [&](void **dst, const void *src, size_t bytes) -> int {
        KMSD_CUDA(cudaMalloc(dst, std::max<size_t>(bytes, 16)));
        if (bytes) KMSD_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
        return KMSD_OK;
    };
    int rc = up((void **)&A->ptr, p32.data(), (n + 1) * sizeof(int));
    if (!rc) rc = up((void **)&A->idx, i32.data(), nnz * sizeof(int));
    if (!rc) rc = up((void **)&A->re64, val_re, nnz * sizeof(double));
    if (!rc && cplx) rc = up((void **)&A->im64, val_im, nnz * sizeof(double));
    // ELL form when rows are short and padding costs at most a quarter of the
    // index/value bytes (lattice Hamiltonians: every row has the same length).
    int64_t lmax = 0;
    for (int64_t r = 0; r < n; ++r) lmax = std::max<int64_t>(lmax, indptr[r + 1] - indptr[r]);
    const int64_t w = std::max<int64_t>(4, (lmax + 3) / 4 * 4);
    if (!rc && lmax > 0 && w <= 32 && n * w <= nnz + nnz / 4 + 4) {
        const int64_t m = n * w;
        std::vector<int> ei(m);
        std::vector<double> er(m, 0.), eim(cplx ? m : 0, 0.);
        for (int64_t r = 0; r < n; ++r) {
            int64_t j = 0;
            for (int64_t k = indptr[r]; k < indptr[r + 1]; ++k, ++j) {
                ei[r * w + j] = (int)indices[k];
                er[r * w + j] = val_re[k];
                if (cplx) eim[r * w + j] = val_im[k];
            }
            for (; j < w; ++j) ei[r * w + j] = (int)r;  // zero-valued padding on the own row
        }
        rc = up((void **)&A->ell_idx, ei.data(), m * sizeof(int));
        if (!rc) rc = up((void **)&A->ell_re64, er.data(), m * sizeof(double));
        if (!rc && cplx) rc = up((void **)&A->ell_im64, eim.data(), m * sizeof(double));
        if (!rc) A->ell_w = (int)w;
    }
    // 4x4 block-CSR form when the pattern tiles into aligned 4x4 blocks (the
    // atom blocks of an sp3 basis) with at most a quarter of zero fill over
    // the matrix, and no block row more than doubled: each gathered input row
    // then serves four output rows.
    if (!rc && !ident && n % 4 == 0 && nnz >= 16) {
        const int64_t nbr = n / 4;
        std::vector<int> bptr(nbr + 1, 0), bcols;
        std::vector<int64_t> mark(nbr, -1);
        bool ok = true;
        for (int64_t I = 0; I < nbr && ok; ++I) {
            const size_t start = bcols.size();
            for (int64_t r = 4 * I; r < 4 * I + 4; ++r)
                for (int64_t k = indptr[r]; k < indptr[r + 1]; ++k) {
                    const int64_t J = indices[k] / 4;
                    if (mark[J] != I) {
                        mark[J] = I;
                        bcols.push_back((int)J);
                    }
                }
            std::sort(bcols.begin() + start, bcols.end());
            const int64_t row_nnz = indptr[4 * I + 4] - indptr[4 * I];
            ok = (int64_t)(bcols.size() - start) * 16 <= 2 * row_nnz + 16 && bcols.size() < (size_t)INT32_MAX / 16;
            bptr[I + 1] = (int)bcols.size();
        }
        const int64_t nblk = (int64_t)bcols.size();
        if (ok && nblk * 16 <= nnz + nnz / 4) {
            std::vector<double> br((size_t)nblk * 16, 0.), bi(cplx ? (size_t)nblk * 16 : 0, 0.);
            for (int64_t I = 0; I < nbr; ++I) {
                const int *b0 = bcols.data() + bptr[I], *b1 = bcols.data() + bptr[I + 1];
                for (int64_t r = 4 * I; r < 4 * I + 4; ++r)
                    for (int64_t k = indptr[r]; k < indptr[r + 1]; ++k) {
                        const int J = (int)(indices[k] / 4);
                        const int64_t q = std::lower_bound(b0, b1, J) - bcols.data();
                        const size_t e = (size_t)q * 16 + (size_t)(r - 4 * I) * 4 + (size_t)(indices[k] - 4 * J);
                        br[e] += val_re[k];
                        if (cplx) bi[e] += val_im[k];
                    }
            }
            rc = up((void **)&A->bsr_ptr, bptr.data(), (nbr + 1) * sizeof(int));
            if (!rc) rc = up((void **)&A->bsr_idx, bcols.data(), nblk * sizeof(int));
            if (!rc) rc = up((void **)&A->bsr_re, br.data(), br.size() * sizeof(double));
            if (!rc && cplx) rc = up((void **)&A->bsr_im, bi.data(), bi.size() * sizeof(double));
            if (!rc) A->bsr_nb = nbr;
        }
    }
    if (rc) {
        kmsd_csr_destroy(A);
        return rc;
    }
    *out = A;
    return KMSD_OK;
}

void kmsd_csr_destroy(kmsd_csr a) {
    if (!a) return;
    cudaFree(a->ptr);
    cudaFree(a->idx);
    cudaFree(a->re64);
    cudaFree(a->im64);
    cudaFree(a->re32);
    cudaFree(a->im32);
    cudaFree(a->ell_idx);
    cudaFree(a->ell_re64);
    cudaFree(a->ell_im64);
    cudaFree(a->ell_re32);
    cudaFree(a->ell_im32);
    cudaFree(a->bsr_ptr);
    cudaFree(a->bsr_idx);
    cudaFree(a->bsr_re);
    cudaFree(a->bsr_im);
    delete a;
}

int64_t kmsd_csr_rows(kmsd_csr a) { return a ? a->n : -1; }
int64_t kmsd_csr_nnz(kmsd_csr a) { return a ? a->nnz : -1; }
int kmsd_csr_forms(kmsd_csr a) {
    if (!a) return -1;
    return (a->ell_w > 0 ? KMSD_FORM_ELL : 0) | (a->bsr_nb > 0 ? KMSD_FORM_BSR4 : 0);
}

int kmsd_csr_matmul(kmsd_csr a, const void *x, void *y, int64_t b, void *stream) {
    if (!a || !x || !y || b < 1) return fail(KMSD_EINVAL, "CSR input dimension mismatch");
    return spmm64(a, static_cast<const double2 *>(x), static_cast<double2 *>(y), b,
                  static_cast<cudaStream_t>(stream));
}

int kmsd_column_dot(const void *x, const void *y, int64_t n, int64_t b, void *out, void *stream) {
    if (!x || !y || !out || n < 1 || b < 1) return fail(KMSD_EINVAL, "invalid column dot dimensions");
    return coldot64(static_cast<const double2 *>(x), static_cast<const double2 *>(y), n, b,
                    static_cast<double2 *>(out), static_cast<cudaStream_t>(stream));
}

}  // extern "C"

