// Engine operations of the B200 stochastic-KPM backend (replaces Engine of
// the reference, cpp/native.cpp:488-610).
//
// Identity metric (S = I, unit diagonal): one fused cheb_step_kernel launch
// per Chebyshev step, FP64 or mixed.  General metric: SpMM + batched PCG +
// the same step kernel on the solved operand (FP64).  Every public call ends
// with one stream synchronisation that reads the device status word, so a
// failure inside any operator application (failed PCG acceptance, nonfinite
// propagation) is reported with the reference's error class and message.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "kmsd.h"
#include "kmsd_impl.h"
#include "kmsd_kernels.cuh"
#include "kmsd_tile.cuh"

using namespace kmsd;

namespace {
using E = kmsd_engine_s;

struct Ctl {  // solve controls of one call
    double rtol, atol;
    int maxiter;
};

int ensure_vec(DevBuf &d, int64_t n, int64_t cols, size_t elem = sizeof(double2)) {
    return d.ensure((size_t)n * cols * elem) ? KMSD_ECUDA : KMSD_OK;
}

int begin(E *e, cudaStream_t s) {
    if (e->status.ensure(4 * sizeof(int)) || e->report.ensure(sizeof(FailReportFull)) ||
        e->dots.ensure(512 * sizeof(double2)))
        return KMSD_ECUDA;
    KMSD_CUDA(cudaMemsetAsync(e->status.p, 0, 4 * sizeof(int), s));
    return KMSD_OK;
}

int finish(E *e, cudaStream_t s) {
    int st[4];
    KMSD_CUDA(cudaMemcpyAsync(st, e->status.p, sizeof(st), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaStreamSynchronize(s));
    KMSD_CUDA(cudaGetLastError());
    if (st[0] != 0) {
        KMSD_CUDA(cudaMemcpy(&e->last, e->report.p, sizeof(FailReportFull), cudaMemcpyDeviceToHost));
        switch (e->last.head.reason) {
            case 3: return fail(KMSD_EINVAL, "metric RHS must be finite");
            case 2:
                return fail(KMSD_EMETRIC,
                            "S solve solution is nonfinite or not representable in complex128 after rescaling");
            case 1: return fail(KMSD_EMETRIC, "PCG non-positive/complex curvature breakdown");
            default: return fail(KMSD_EMETRIC, "S solve failed true-residual acceptance");
        }
    }
    if (st[2] != 0) return fail(KMSD_ERUNTIME, "nonfinite Chebyshev propagation; check bounds and solves");
    if (st[3] != 0) return fail(KMSD_ERUNTIME, "a bounded device wait of the tiled Chebyshev step ran out");
    return KMSD_OK;
}

int *status_ptr(E *e) { return e->status.as<int>(); }

// Y = S^-1 B (asynchronous; failures land in the status word).
int solve(E *e, const double2 *B, double2 *Y, int64_t b, const Ctl &c, cudaStream_t s) {
    const int64_t n = e->H->n;
    if (e->identity) {
        // S = I with unit diagonal: PCG converges in one exact step (alpha = 1),
        // the solution is the right-hand side itself.
        if (B != Y) KMSD_CUDA(cudaMemcpyAsync(Y, B, (size_t)n * b * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        e->M->calls += 1;
        return KMSD_OK;
    }
    return e->M->solve_dev(B, Y, b, c.rtol, c.atol, c.maxiter, s, status_ptr(e), e->report.p);
}

// out = S^-1 H B
int h_action(E *e, const double2 *B, double2 *out, int64_t b, const Ctl &c, cudaStream_t s) {
    ++e->h_calls;
    if (e->identity) return spmm64(e->H, B, out, b, s);
    if (ensure_vec(e->t1, e->H->n, b)) return KMSD_ECUDA;
    int rc = spmm64(e->H, B, e->t1.as<double2>(), b, s);
    if (rc) return rc;
    return solve(e, e->t1.as<double2>(), out, b, c, s);
}

// out += coef * v_axis B (Engine::v_cart, native.cpp:506-523); coef real.
int v_cart_acc(E *e, int axis, const double2 *B, double2 *out, int64_t b, double coef, const Ctl &c,
               cudaStream_t s) {
    const int64_t n = e->H->n, len = n * b;
    const int kind = e->vel_kind[axis];
    kmsd_csr_s **m = e->vel + 3 * axis;
    for (DevBuf *d : {&e->t2, &e->t3, &e->t4, &e->t5})
        if (ensure_vec(*d, n, b)) return KMSD_ECUDA;
    double2 *t2 = e->t2.as<double2>(), *t3 = e->t3.as<double2>(), *t4 = e->t4.as<double2>(),
            *t5 = e->t5.as<double2>();
    const double k = coef / e->hbar;  // i * coef / hbar
    int rc;
    if (kind == 0 && m[0]) {
        if ((rc = spmm64(m[0], B, t2, b, s))) return rc;
        const double2 *x[1] = {t2};
        const double cr[1] = {coef}, ci[1] = {0.};
        return lincomb(s, out, len, 1, 1, x, cr, ci);
    }
    if (kind == 1 && m[0]) {
        // i (H S^-1 X B - X S^-1 H B) / hbar
        if ((rc = spmm64(m[0], B, t2, b, s))) return rc;
        if ((rc = solve(e, t2, t3, b, c, s))) return rc;
        if ((rc = spmm64(e->H, t3, t4, b, s))) return rc;
        if ((rc = spmm64(e->H, B, t2, b, s))) return rc;
        if ((rc = solve(e, t2, t3, b, c, s))) return rc;
        if ((rc = spmm64(m[0], t3, t5, b, s))) return rc;
        const double2 *x[2] = {t4, t5};
        const double cr[2] = {0., 0.}, ci[2] = {k, -k};
        return lincomb(s, out, len, 1, 2, x, cr, ci);
    }
    if (kind == 2 && m[0] && m[1] && m[2]) {
        // i (bond B - xbar S^-1 H B + H S^-1 delta B) / hbar
        if ((rc = spmm64(m[0], B, t2, b, s))) return rc;
        if ((rc = spmm64(e->H, B, t3, b, s))) return rc;
        if ((rc = solve(e, t3, t4, b, c, s))) return rc;
        if ((rc = spmm64(m[1], t4, t5, b, s))) return rc;
        if ((rc = spmm64(m[2], B, t3, b, s))) return rc;
        if ((rc = solve(e, t3, t4, b, c, s))) return rc;
        if ((rc = spmm64(e->H, t4, t3, b, s))) return rc;
        const double2 *x[3] = {t2, t5, t3};
        const double cr[3] = {0., 0., 0.}, ci[3] = {k, -k, k};
        return lincomb(s, out, len, 1, 3, x, cr, ci);
    }
    return fail(KMSD_EINVAL, "missing Cartesian velocity");
}

// out = sum_a dir[a] v_a B (Engine::v_cov, native.cpp:524-533)
int v_cov(E *e, const double *dir, const double2 *B, double2 *out, int64_t b, const Ctl &c, cudaStream_t s) {
    ++e->v_calls;
    KMSD_CUDA(cudaMemsetAsync(out, 0, (size_t)e->H->n * b * sizeof(double2), s));
    for (int a = 0; a < 3; ++a)
        if (dir[a] != 0.) {
            int rc = v_cart_acc(e, a, B, out, b, dir[a], c, s);
            if (rc) return rc;
        }
    return KMSD_OK;
}

// ---------------------------------------------------------------- step launch
// One resident wave: the grid is the number of CTAs the SMs hold at once for
// this kernel (occupancy API), capped by the rows to cover.  Fixed per kernel
// and shape, so row ownership — and with it every reduction order — is
// reproducible run to run.
template <class T, int MU, int MODE, int HSRC, bool IV>
int launch_step_mu(E *e, StepArgs<T> &a, cudaStream_t s) {
    const auto kern = cheb_step_kernel<T, MU, MODE, HSRC, IV>;
    size_t sm = reduce_smem(a.mp, Unit<T>::C);
    if (MODE == MODE_SERIES && a.share_v)  // two parity slices of the shared velocity products
        sm = std::max(sm, (size_t)2 * a.nvel * kThreads * sizeof(typename Unit<T>::vec));
    const int grid = wave_grid((const void *)kern, sm, a.n, a.mp);
    if (MODE == MODE_DIRECT || MODE == MODE_DOUBLING) {
        if (e->red.ensure(grid, a.mp.U * Unit<T>::C, 2)) return KMSD_ECUDA;
        a.partial = e->red.part();
        a.ticket = e->red.tick();
    }
    kern<<<grid, kThreads, sm, s>>>(a);
    return KMSD_OK;
}

template <class T, int MODE, int HSRC, bool IV>
int launch_step_h(E *e, StepArgs<T> &a, cudaStream_t s) {
    switch (mu_for(a.mp)) {
        case 1: return launch_step_mu<T, 1, MODE, HSRC, IV>(e, a, s);
        case 2: return launch_step_mu<T, 2, MODE, HSRC, IV>(e, a, s);
    }
    return fail(KMSD_EINVAL, "too many columns for one engine call");
}

// Tile-pipelined moment step (kmsd_tile.cuh): persistent grid of one
// resident wave; tiles sized so the stage ring of a CTA is about
// KMSD_TILE_RING bytes, a whole number of rows per row group.
template <class T, int MODE, int W>
int launch_tile(E *e, StepArgs<T> &a, cudaStream_t s) {
    const auto kern = cheb_tile_kernel<T, MODE, W>;
    // per instantiation, shared by every calling thread
    static std::mutex lock;
    static int smem_cap = 0;
    static std::map<size_t, int> per_sm_cache;  // shared bytes -> CTAs per SM
    std::unique_lock<std::mutex> guard(lock);
    if (!smem_cap) {
        int dev = 0, optin = 0;
        KMSD_CUDA(cudaGetDevice(&dev));
        KMSD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        KMSD_CUDA(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       optin - 1024));
        smem_cap = optin - 1024;
    }
    const RowMap &mp = a.mp;
    const int nvec = MODE == MODE_DIRECT ? 3 : 2;
    const int row_bytes = nvec * mp.U * 16 + W * (4 + (int)sizeof(T));
    int tr = KMSD_TILE_RING / KMSD_TILE_STAGES / row_bytes / mp.gpc * mp.gpc;
    tr = std::max(mp.gpc, std::min(kTileMaxRows / mp.gpc * mp.gpc, tr));
    const TileLayout L = tile_layout(tr, mp.U, W, nvec, (int)sizeof(T));
    const size_t sm = tile_smem(L, mp, Unit<T>::C);
    if (sm > (size_t)smem_cap) return fail(KMSD_EINVAL, "tile step does not fit in shared memory");
    int per_sm = 0;
    auto it = per_sm_cache.find(sm);
    if (it != per_sm_cache.end()) {
        per_sm = it->second;
    } else {
        KMSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)kern, kTileThreads, sm));
        per_sm = std::max(per_sm, 1);
        per_sm_cache[sm] = per_sm;
    }
    guard.unlock();
    const int64_t ntiles = (a.n + tr - 1) / tr;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)sm_count() * per_sm));
    if (e->red.ensure(grid, mp.U * Unit<T>::C, 2)) return KMSD_ECUDA;
    a.partial = e->red.part();
    a.ticket = e->red.tick();
    kern<<<grid, kTileThreads, sm, s>>>(a, L, status_ptr(e) + 3);
    return KMSD_OK;
}

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// The tile step applies to moment steps over a real ELL form of width 4 or 8
// with one unit per lane, on 16-byte aligned operands.
template <class T, int MODE, bool IH>
bool tile_applies(const StepArgs<T> &a) {
    if (!KMSD_TILE || !IH || (MODE != MODE_DOUBLING && MODE != MODE_DIRECT)) return false;
    if (std::is_same<T, float>::value && MODE == MODE_DOUBLING && !KMSD_TILE_F32_DOUBLING) return false;
    if (a.E.im != nullptr || (a.E.w != 4 && a.E.w != 8) || a.mp.U > 128 || mu_for(a.mp) != 1) return false;
    return aligned16(a.curr) && aligned16(a.prev) && aligned16(a.next) &&
           (MODE != MODE_DIRECT || aligned16(a.bra));
}

// IH: the operator is applied inline (identity metric), from the ELL form
// when the matrix has one, else from CSR; otherwise the step reads the solved
// operand a.hx.
template <class T, int MODE, bool IH, bool IV>
int launch_step(E *e, StepArgs<T> &a, cudaStream_t s) {
    int rc;
    if constexpr (MODE == MODE_DOUBLING || MODE == MODE_DIRECT) {
        if (tile_applies<T, MODE, IH>(a)) {
            rc = a.E.w == 4 ? launch_tile<T, MODE, 4>(e, a, s) : launch_tile<T, MODE, 8>(e, a, s);
            if (rc) return rc;
            count_launch();
            KMSD_CUDA(cudaGetLastError());
            return KMSD_OK;
        }
    }
    if (!IH) rc = launch_step_h<T, MODE, HSRC_SOLVED, IV>(e, a, s);
    else if (a.E.w == 4 && a.E.im == nullptr) rc = launch_step_h<T, MODE, HSRC_ELL4, IV>(e, a, s);
    else if (a.E.w == 8 && a.E.im == nullptr) rc = launch_step_h<T, MODE, HSRC_ELL8, IV>(e, a, s);
    else if (a.E.w > 0) rc = launch_step_h<T, MODE, HSRC_ELL, IV>(e, a, s);
    else rc = launch_step_h<T, MODE, HSRC_CSR, IV>(e, a, s);
    if (rc) return rc;
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

template <class T> CsrView<T> view_of(kmsd_csr_s *A);
template <> CsrView<double> view_of<double>(kmsd_csr_s *A) { return A->view64(); }
template <> CsrView<float> view_of<float>(kmsd_csr_s *A) { return A->view32(); }
template <class T> EllView<T> ell_of(kmsd_csr_s *A);
template <> EllView<double> ell_of<double>(kmsd_csr_s *A) { return A->ell64(); }
template <> EllView<float> ell_of<float>(kmsd_csr_s *A) {
    EllView<float> v = A->ell32();
    if (v.re == nullptr) v.w = 0;  // no complex64 ELL values yet: use CSR
    return v;
}

template <class T> StepArgs<T> base_args(E *e, int U, double center, double half) {
    StepArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.n = e->H->n;
    a.mp = make_map(U, kThreads);
    a.H = view_of<T>(e->H);
    a.E = ell_of<T>(e->H);
    a.center = center;
    a.half = half;
    a.inv_half = (T)(1. / half);
    a.status = status_ptr(e) + 2;
    return a;
}

int to_f32(const double2 *src, float4 *dst, int64_t n, int64_t b, int U, cudaStream_t s) {
    const int64_t total = n * U;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16));
    to_f32_kernel<<<grid, 256, 0, s>>>(src, dst, n, (int)b, U);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}
int to_f64(const float4 *src, double2 *dst, int64_t n, int64_t b, int U, cudaStream_t s) {
    const int64_t total = n * b;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16));
    to_f64_kernel<<<grid, 256, 0, s>>>(src, dst, n, (int)b, U);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

// ---------------------------------------------------------------- Lanczos
// w <- w - alpha v - beta v_prev with alpha = Re dot->x, beta from the device.
__global__ void lanczos_update_kernel(double2 *w, const double2 *v, const double2 *vp, int64_t n, const double2 *dot,
                                      const double *beta_prev) {
    const double al = dot->x, be = beta_prev ? *beta_prev : 0.;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = w[i], x = v[i], y = vp[i];
        w[i] = make_double2(a.x - al * x.x - be * y.x, a.y - al * x.y - be * y.y);
    }
}
// v <- w / beta with beta = sqrt(max(Re dot->x, 0)), recorded in beta_out.
__global__ void lanczos_scale_kernel(const double2 *w, double2 *v, int64_t n, const double2 *dot, double *beta_out) {
    const double be = sqrt(fmax(dot->x, 0.));
    if (beta_out && blockIdx.x == 0 && threadIdx.x == 0) *beta_out = be;
    const double inv = be > 0. ? 1. / be : 0.;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = w[i];
        v[i] = make_double2(a.x * inv, a.y * inv);
    }
}

// ---------------------------------------------------------------- moments
int moments_impl(E *e, const double2 *B, double *mu, int64_t b, int64_t len, double center, double half, int flags,
                 cudaStream_t s) {
    const int64_t n = e->H->n;
    const Ctl c{e->rtol, e->atol, e->maxiter};
    const bool doubling = (flags & KMSD_MOMENTS_DOUBLING) != 0;
    if (doubling && !e->identity)
        return fail(KMSD_EINVAL, "moment doubling requires an identity metric (orthogonal basis)");
    double2 *dots = e->dots.as<double2>();
    int rc;
    if (e->precision == KMSD_FP64) {
        const double2 *bra = B;
        if (e->identity) {
            if ((rc = coldot64(B, B, n, b, dots, s))) return rc;
        } else {
            if (ensure_vec(e->bra, n, b)) return KMSD_ECUDA;
            if ((rc = spmm64(e->M->S, B, e->bra.as<double2>(), b, s, dots))) return rc;
            bra = e->bra.as<double2>();
        }
        if ((rc = take_real(dots, mu, b, s))) return rc;
        if (len == 1) return KMSD_OK;
        if (ensure_vec(e->ta, n, b) || ensure_vec(e->tb, n, b)) return KMSD_ECUDA;
        double2 *ta = e->ta.as<double2>(), *tb = e->tb.as<double2>();
        if (e->identity) {
            StepArgs<double> a = base_args<double>(e, (int)b, center, half);
            a.bra = bra;
            a.mu = mu;
            a.mlen = len;
            a.bcols = (int)b;
            // T0 = B (read only), T1 -> ta, T2 -> tb, then in place over T_{k-2}.
            const double2 *curr = B, *prev = nullptr;
            double2 *bufs[2] = {ta, tb};
            const int64_t steps = doubling ? (len + 1) / 2 : len - 1;
            for (int64_t k = 1; k <= steps; ++k) {
                double2 *next = k <= 2 ? bufs[k - 1] : const_cast<double2 *>(prev);
                a.curr = curr;
                a.prev = prev;
                a.next = next;
                a.first = k == 1;
                if (doubling) {
                    a.kmom = k - 1;
                    if ((rc = launch_step<double, MODE_DOUBLING, true, false>(e, a, s))) return rc;
                } else {
                    a.kmom = k;
                    if ((rc = launch_step<double, MODE_DIRECT, true, false>(e, a, s))) return rc;
                }
                prev = curr;
                curr = next;
            }
            e->h_calls += steps;
            return KMSD_OK;
        }
        // General metric: S^-1 H T_{k-1} by SpMM + PCG, then the fused epilogue.
        if (ensure_vec(e->hx, n, b)) return KMSD_ECUDA;
        double2 *hx = e->hx.as<double2>();
        KMSD_CUDA(cudaMemcpyAsync(tb, B, (size_t)n * b * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        StepArgs<double> a = base_args<double>(e, (int)b, center, half);
        a.bra = bra;
        a.mu = mu;
        a.mlen = len;
        a.bcols = (int)b;
        a.hx = hx;
        double2 *curr = tb, *prev = nullptr, *spare = ta;
        for (int64_t k = 1; k < len; ++k) {
            if ((rc = h_action(e, curr, hx, b, c, s))) return rc;
            double2 *next = k == 1 ? spare : prev;
            a.curr = curr;
            a.prev = prev;
            a.next = next;
            a.first = k == 1;
            a.kmom = k;
            if ((rc = launch_step<double, MODE_DIRECT, false, false>(e, a, s))) return rc;
            prev = curr;
            curr = next;
        }
        return KMSD_OK;
    }
    // Mixed: identity metric only.
    if (!e->identity) return fail(KMSD_EINVAL, "mixed precision requires an identity metric (orthogonal basis)");
    const int U = (int)((b + 1) / 2);
    if (ensure_vec(e->ta, n, U, sizeof(float4)) || ensure_vec(e->tb, n, U, sizeof(float4)) ||
        ensure_vec(e->bra, n, U, sizeof(float4)) || e->H->ensure_f32())
        return KMSD_ECUDA;
    float4 *ta = e->ta.as<float4>(), *tb = e->tb.as<float4>(), *bra = e->bra.as<float4>();
    if ((rc = to_f32(B, tb, n, b, U, s))) return rc;
    if (!doubling) KMSD_CUDA(cudaMemcpyAsync(bra, tb, (size_t)n * U * sizeof(float4), cudaMemcpyDeviceToDevice, s));
    if ((rc = coldot32(tb, tb, n, U, dots, s))) return rc;
    if ((rc = take_real(dots, mu, b, s))) return rc;
    if (len == 1) return KMSD_OK;
    StepArgs<float> a = base_args<float>(e, U, center, half);
    a.bra = bra;
    a.mu = mu;
    a.mlen = len;
    a.bcols = (int)b;
    float4 *curr = tb, *prev = nullptr, *spare = ta;
    const int64_t steps = doubling ? (len + 1) / 2 : len - 1;
    for (int64_t k = 1; k <= steps; ++k) {
        float4 *next = k == 1 ? spare : prev;
        a.curr = curr;
        a.prev = prev;
        a.next = next;
        a.first = k == 1;
        if (doubling) {
            a.kmom = k - 1;
            if ((rc = launch_step<float, MODE_DOUBLING, true, false>(e, a, s))) return rc;
        } else {
            a.kmom = k;
            if ((rc = launch_step<float, MODE_DIRECT, true, false>(e, a, s))) return rc;
        }
        prev = curr;
        curr = next;
    }
    e->h_calls += steps;
    return KMSD_OK;
}

// ---------------------------------------------------------------- chain
int chain_impl(E *e, const double2 *B, double2 *out, int64_t b, int64_t len, double center, double half,
               cudaStream_t s) {
    const int64_t n = e->H->n;
    const size_t slab = (size_t)n * b;
    const Ctl c{e->rtol, e->atol, e->maxiter};
    int rc;
    KMSD_CUDA(cudaMemcpyAsync(out, B, slab * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    if (len == 1) return KMSD_OK;
    if (e->precision == KMSD_FP64) {
        StepArgs<double> a = base_args<double>(e, (int)b, center, half);
        if (!e->identity) {
            if (ensure_vec(e->hx, n, b)) return KMSD_ECUDA;
            a.hx = e->hx.as<double2>();
        }
        for (int64_t k = 1; k < len; ++k) {
            a.curr = out + (k - 1) * slab;
            a.prev = k >= 2 ? out + (k - 2) * slab : nullptr;
            a.next = out + k * slab;
            a.first = k == 1;
            if (e->identity) {
                ++e->h_calls;
                if ((rc = launch_step<double, MODE_CHAIN, true, false>(e, a, s))) return rc;
            } else {
                if ((rc = h_action(e, a.curr, e->hx.as<double2>(), b, c, s))) return rc;
                if ((rc = launch_step<double, MODE_CHAIN, false, false>(e, a, s))) return rc;
            }
        }
        return KMSD_OK;
    }
    if (!e->identity) return fail(KMSD_EINVAL, "mixed precision requires an identity metric (orthogonal basis)");
    if (b % 2) return fail(KMSD_EINVAL, "mixed-precision chain needs an even number of columns");
    const int U = (int)(b / 2);
    if (ensure_vec(e->ta, n, U, sizeof(float4)) || ensure_vec(e->tb, n, U, sizeof(float4)) || e->H->ensure_f32())
        return KMSD_ECUDA;
    float4 *ta = e->ta.as<float4>(), *tb = e->tb.as<float4>();
    if ((rc = to_f32(B, tb, n, b, U, s))) return rc;
    StepArgs<float> a = base_args<float>(e, U, center, half);
    float4 *curr = tb, *prev = nullptr;
    for (int64_t k = 1; k < len; ++k) {
        float4 *next = k == 1 ? ta : prev;
        a.curr = curr;
        a.prev = prev;
        a.next = next;
        a.first = k == 1;
        a.store64 = out + k * slab;
        if ((rc = launch_step<float, MODE_CHAIN, true, false>(e, a, s))) return rc;
        prev = curr;
        curr = next;
    }
    e->h_calls += len - 1;
    return KMSD_OK;
}

// ---------------------------------------------------------------- correlate
// tables[b, j, k] = <T_j(Ht) B[:, b], cov[:, k, b]> for j < len, k < k1,
// with the chain generated into a ring of ring_slots() vector blocks and
// contracted every ring_slots() steps (kmsd_corr.cu), never stored whole.
// Step k writes slot k % J, which held T_{k-J}: the contraction that read it
// was queued on the same stream before this step.
int correlate_impl(E *e, const double2 *B, const double2 *cov, int64_t b, int64_t len, int64_t k1, double center,
                   double half, double2 *tables, cudaStream_t s) {
    const int64_t n = e->H->n;
    const int64_t slab = n * b;
    const int J = ring_slots();
    const Ctl c{e->rtol, e->atol, e->maxiter};
    if (ensure_vec(e->ring, n, b * J)) return KMSD_ECUDA;
    double2 *ring = e->ring.as<double2>();
    auto slot = [&](int64_t k) { return ring + (k % J) * slab; };
    int rc;
    auto contract_after = [&](int64_t k) -> int {  // chain index k was just written
        if ((k + 1) % J != 0 && k != len - 1) return KMSD_OK;
        const int64_t j0 = k - k % J;
        return corr_ring(ring, n, (int)b, cov, (int)k1, j0, (int)(k - j0 + 1), len, tables, e->corr_partial, s);
    };
    KMSD_CUDA(cudaMemcpyAsync(slot(0), B, slab * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    if ((rc = contract_after(0))) return rc;
    if (len == 1) return KMSD_OK;
    if (e->precision == KMSD_FP64) {
        StepArgs<double> a = base_args<double>(e, (int)b, center, half);
        if (!e->identity) {
            if (ensure_vec(e->hx, n, b)) return KMSD_ECUDA;
            a.hx = e->hx.as<double2>();
        }
        for (int64_t k = 1; k < len; ++k) {
            a.curr = slot(k - 1);
            a.prev = k >= 2 ? slot(k - 2) : nullptr;
            a.next = slot(k);
            a.first = k == 1;
            if (e->identity) {
                ++e->h_calls;
                if ((rc = launch_step<double, MODE_CHAIN, true, false>(e, a, s))) return rc;
            } else {
                if ((rc = h_action(e, a.curr, e->hx.as<double2>(), b, c, s))) return rc;
                if ((rc = launch_step<double, MODE_CHAIN, false, false>(e, a, s))) return rc;
            }
            if ((rc = contract_after(k))) return rc;
        }
        return KMSD_OK;
    }
    if (!e->identity) return fail(KMSD_EINVAL, "mixed precision requires an identity metric (orthogonal basis)");
    if (b % 2) return fail(KMSD_EINVAL, "mixed-precision chain needs an even number of columns");
    const int U = (int)(b / 2);
    if (ensure_vec(e->ta, n, U, sizeof(float4)) || ensure_vec(e->tb, n, U, sizeof(float4)) || e->H->ensure_f32())
        return KMSD_ECUDA;
    float4 *ta = e->ta.as<float4>(), *tb = e->tb.as<float4>();
    if ((rc = to_f32(B, tb, n, b, U, s))) return rc;
    StepArgs<float> a = base_args<float>(e, U, center, half);
    float4 *curr = tb, *prev = nullptr;
    for (int64_t k = 1; k < len; ++k) {
        float4 *next = k == 1 ? ta : prev;
        a.curr = curr;
        a.prev = prev;
        a.next = next;
        a.first = k == 1;
        a.store64 = slot(k);
        if ((rc = launch_step<float, MODE_CHAIN, true, false>(e, a, s))) return rc;
        if ((rc = contract_after(k))) return rc;
        prev = curr;
        curr = next;
    }
    e->h_calls += len - 1;
    return KMSD_OK;
}

// ---------------------------------------------------------------- series
struct Aug {
    int64_t nb = 0, ndir = 0;
    const double *dirs = nullptr;  // ndir x 3
    bool inline_v = false;
    int nvel = 0, vel_axis[3] = {0, 0, 0};
};

// Position operator of axis x given by site coordinates (a diagonal X) on an
// orthogonal basis: its velocity i [H, X] / hbar is applied inside the step
// kernel from H's rows.
bool commutator_inline(const E *e, int x) {
    return e->vel_kind[x] == 1 && e->identity && e->vel[3 * x] && e->vel[3 * x]->diagonal;
}

// Can every velocity contribution be applied inside the step kernel: an
// explicit matrix (kind 0), or a position commutator with coordinates?
int plan_aug(E *e, Aug &g) {
    g.inline_v = true;
    for (int64_t a = 0; a < g.ndir; ++a)
        for (int x = 0; x < 3; ++x)
            if (g.dirs[3 * a + x] != 0.) {
                if (e->vel_kind[x] < 0) return fail(KMSD_EINVAL, "missing Cartesian velocity");
                if (e->vel_kind[x] != 0 && !commutator_inline(e, x)) g.inline_v = false;
            }
    g.nvel = 0;
    for (int x = 0; x < 3; ++x) {
        bool used = false;
        for (int64_t a = 0; a < g.ndir; ++a) used |= g.dirs[3 * a + x] != 0.;
        if (used) g.vel_axis[g.nvel++] = x;
    }
    return KMSD_OK;
}

// The inline velocity of axis x with its values laid out like H's ELL form:
// entry [r * w + j] is V[r, c] for c = H's ELL column [r * w + j] (zero for
// padding).  V is the explicit matrix (kind 0) or i [H, X] / hbar for
// coordinates X (kind 1), formed in FP64 on the host.  Returns false when V
// has an entry outside H's pattern (the step then gathers V's own rows).
bool aligned_velocity(E *e, int x) {
    if (e->vell_state[x]) return e->vell_state[x] > 0;
    e->vell_state[x] = -1;
    const kmsd_csr_s *H = e->H, *V = e->vel[3 * x];
    const int64_t n = H->n, w = H->ell_w;
    if (w != 4 && w != 8) return false;
    if (H->complex_values || !V) return false;
    std::vector<int> eidx(n * w);
    std::vector<double> eval(n * w);
    if (cudaMemcpy(eidx.data(), H->ell_idx, eidx.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(eval.data(), H->ell_re64, eval.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    std::vector<double> re(n * w, 0.), im(n * w, 0.);
    const bool comm = commutator_inline(e, x);
    if (comm) {
        std::vector<double> xs(n);
        if (cudaMemcpy(xs.data(), V->re64, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
        for (int64_t r = 0; r < n; ++r)
            for (int64_t j = 0; j < w; ++j) {
                const int c = eidx[r * w + j];
                im[r * w + j] = eval[r * w + j] * (xs[c] - xs[r]) / e->hbar;  // i H_rc (x_c - x_r) / hbar
            }
    } else {
        std::vector<int> vp(n + 1), vi(std::max<int64_t>(V->nnz, 1));
        std::vector<double> vr(std::max<int64_t>(V->nnz, 1)), vim(std::max<int64_t>(V->nnz, 1), 0.);
        if (cudaMemcpy(vp.data(), V->ptr, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(vi.data(), V->idx, V->nnz * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(vr.data(), V->re64, V->nnz * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return false;
        if (V->complex_values &&
            cudaMemcpy(vim.data(), V->im64, V->nnz * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return false;
        for (int64_t r = 0; r < n; ++r)
            for (int k = vp[r]; k < vp[r + 1]; ++k) {
                int64_t j = 0;
                // the first ELL slot of this column that is still unused (a padding
                // slot points at its own row with a zero value)
                while (j < w && (eidx[r * w + j] != vi[k] || re[r * w + j] != 0. || im[r * w + j] != 0.)) ++j;
                if (j == w) return false;
                re[r * w + j] += vr[k];
                im[r * w + j] += vim[k];
            }
    }
    std::vector<float> re32(re.begin(), re.end()), im32(im.begin(), im.end());
    const size_t m = (size_t)n * w;
    if (e->vell64[x].ensure(2 * m * sizeof(double)) || e->vell32[x].ensure(2 * m * sizeof(float))) return false;
    double *d64 = e->vell64[x].as<double>();
    float *d32 = e->vell32[x].as<float>();
    if (cudaMemcpy(d64, re.data(), m * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d64 + m, im.data(), m * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d32, re32.data(), m * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d32 + m, im32.data(), m * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    e->vell_state[x] = 1;
    return true;
}

template <class T> const T *vell_of(E *e, int x);
template <> const double *vell_of<double>(E *e, int x) { return e->vell64[x].as<double>(); }
template <> const float *vell_of<float>(E *e, int x) { return e->vell32[x].as<float>(); }

template <class T> void set_inline_v(E *e, StepArgs<T> &a, const Aug &g, double half) {
    a.nvel = g.nvel;
    for (int v = 0; v < g.nvel; ++v) {
        const int x = g.vel_axis[v];
        const bool comm = commutator_inline(e, x);
        const bool aligned = e->identity && aligned_velocity(e, x);
        a.vform[v] = aligned ? 2 : comm ? 1 : 0;
        a.xdiag[v] = comm ? e->vel[3 * x]->re64 : nullptr;
        if (!comm) a.Vm[v] = view_of<T>(e->vel[3 * x]);
        if (aligned) {
            const size_t m = (size_t)e->H->n * e->H->ell_w;
            a.vel_re[v] = vell_of<T>(e, x);
            a.vel_im[v] = vell_of<T>(e, x) + m;
        }
        a.vel_axis[v] = x;
        for (int64_t blk = 0; blk < g.ndir; ++blk) {
            if (comm && !aligned) {
                // (-i hbar / half) * dir * (i / hbar) on sum_j H_ij (x_j - x_i) psi_j
                a.wr[blk][v] = (T)(g.dirs[3 * blk + x] / half);
                a.wi[blk][v] = (T)0;
            } else {
                // (-i hbar / half) * dir on V psi
                a.wr[blk][v] = (T)0;
                a.wi[blk][v] = (T)(-e->hbar / half * g.dirs[3 * blk + x]);
            }
        }
    }
    a.share_v = series_shares_v<T>() && a.nvel > 0;
    for (int v = 0; v < a.nvel; ++v) a.share_v &= a.vform[v] == 2;
}

// Injection buffers inj[a] = S^-1 v_cov(dir_a, psi) for the general path.
int compute_inj(E *e, const double2 *X, int64_t W, const Aug &g, const Ctl &c, cudaStream_t s) {
    const int64_t n = e->H->n;
    if (ensure_vec(e->psi, n, g.nb) || ensure_vec(e->vc, n, g.nb)) return KMSD_ECUDA;
    const int64_t total = n * g.nb;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16));
    slice_kernel<<<grid, 256, 0, s>>>(X, e->psi.as<double2>(), n, (int)W, 0, (int)g.nb);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    for (int64_t a = 0; a < g.ndir; ++a) {
        if (ensure_vec(e->inj[a], n, g.nb)) return KMSD_ECUDA;
        int rc = v_cov(e, g.dirs + 3 * a, e->psi.as<double2>(), e->vc.as<double2>(), g.nb, c, s);
        if (rc) return rc;
        rc = solve(e, e->vc.as<double2>(), e->inj[a].as<double2>(), g.nb, c, s);
        if (rc) return rc;
    }
    return KMSD_OK;
}

int series_impl(E *e, const double2 *B, double2 *out, int64_t b, const double *coeff, int64_t nc, double center,
                double half, const double *dirs, int64_t ndir, cudaStream_t s) {
    const int64_t n = e->H->n;
    const size_t bytes = (size_t)n * b * sizeof(double2);
    const Ctl c{e->rtol, e->atol, e->maxiter};
    int rc;
    if (nc == 1) {
        const double2 *x[1] = {B};
        const double cr[1] = {coeff[0]}, ci[1] = {coeff[1]};
        return lincomb(s, out, n * b, 0, 1, x, cr, ci);
    }
    Aug g;
    g.ndir = ndir;
    g.dirs = dirs;
    g.nb = ndir ? b / (ndir + 1) : b;
    if (ndir && (rc = plan_aug(e, g))) return rc;
    if (e->precision == KMSD_MIXED) {
        if (!e->identity) return fail(KMSD_EINVAL, "mixed precision requires an identity metric (orthogonal basis)");
        if (ndir && !g.inline_v)
            return fail(KMSD_EINVAL, "mixed precision requires explicit velocity matrices (kind 0) or a position "
                                     "operator given by site coordinates (kind 1, diagonal)");
        if (ndir && g.nb % 2)
            return fail(KMSD_EINVAL, "mixed-precision propagation needs an even number of vectors per block");
        const int U = (int)((b + 1) / 2);
        if (ensure_vec(e->ta, n, U, sizeof(float4)) || ensure_vec(e->tb, n, U, sizeof(float4)) ||
            ensure_vec(e->outw, n, U, sizeof(float4)) || e->H->ensure_f32())
            return KMSD_ECUDA;
        for (int v = 0; v < g.nvel; ++v)
            if (!commutator_inline(e, g.vel_axis[v]) && e->vel[3 * g.vel_axis[v]]->ensure_f32()) return KMSD_ECUDA;
        float4 *ta = e->ta.as<float4>(), *tb = e->tb.as<float4>(), *ow = e->outw.as<float4>();
        if ((rc = to_f32(B, tb, n, b, U, s))) return rc;
        StepArgs<float> a = base_args<float>(e, U, center, half);
        a.out = ow;
        a.UR = ndir ? (int)(g.nb / 2) : 0;
        a.nphi = (int)ndir;
        if (ndir) set_inline_v(e, a, g, half);
        a.c0r = (float)coeff[0];
        a.c0i = (float)coeff[1];
        float4 *curr = tb, *prev = nullptr;
        for (int64_t k = 1; k < nc; ++k) {
            float4 *next = k == 1 ? ta : prev;
            a.curr = curr;
            a.prev = prev;
            a.next = next;
            a.first = k == 1;
            a.ckr = (float)coeff[2 * k];
            a.cki = (float)coeff[2 * k + 1];
            if ((rc = launch_step<float, MODE_SERIES, true, true>(e, a, s))) return rc;
            prev = curr;
            curr = next;
        }
        e->h_calls += nc - 1;
        e->v_calls += (nc - 1) * ndir;
        return to_f64(ow, out, n, b, U, s);
    }
    if (ensure_vec(e->ta, n, b) || ensure_vec(e->tb, n, b)) return KMSD_ECUDA;
    double2 *ta = e->ta.as<double2>(), *tb = e->tb.as<double2>();
    StepArgs<double> a = base_args<double>(e, (int)b, center, half);
    a.out = out;
    a.UR = ndir ? (int)g.nb : 0;
    a.nphi = (int)ndir;
    a.c0r = coeff[0];
    a.c0i = coeff[1];
    a.injr = 0.;
    a.inji = -e->hbar / half;
    const bool fused = e->identity && (ndir == 0 || g.inline_v);
    if (fused && ndir) set_inline_v(e, a, g, half);
    if (!e->identity) {
        if (ensure_vec(e->hx, n, b)) return KMSD_ECUDA;
        a.hx = e->hx.as<double2>();
    }
    KMSD_CUDA(cudaMemcpyAsync(tb, B, bytes, cudaMemcpyDeviceToDevice, s));
    double2 *curr = tb, *prev = nullptr;
    for (int64_t k = 1; k < nc; ++k) {
        double2 *next = k == 1 ? ta : prev;
        a.curr = curr;
        a.prev = prev;
        a.next = next;
        a.first = k == 1;
        a.ckr = coeff[2 * k];
        a.cki = coeff[2 * k + 1];
        if (fused) {
            ++e->h_calls;
            e->v_calls += ndir;
            if ((rc = launch_step<double, MODE_SERIES, true, true>(e, a, s))) return rc;
        } else {
            if (ndir) {
                if ((rc = compute_inj(e, curr, b, g, c, s))) return rc;
                for (int64_t d = 0; d < ndir; ++d) a.inj[d] = e->inj[d].as<double2>();
            }
            if (e->identity) {
                ++e->h_calls;
                if ((rc = launch_step<double, MODE_SERIES, true, false>(e, a, s))) return rc;
            } else {
                if ((rc = h_action(e, curr, e->hx.as<double2>(), b, c, s))) return rc;
                if ((rc = launch_step<double, MODE_SERIES, false, false>(e, a, s))) return rc;
            }
        }
        prev = curr;
        curr = next;
    }
    return KMSD_OK;
}

int fill_report(const FailReportFull &f, kmsd_solve_report *r, int64_t cap) {
    if (!r) return 0;
    const int64_t m = std::min<int64_t>(std::min<int64_t>(f.head.ncols, cap), kMaxReportCols);
    for (int64_t j = 0; j < m; ++j) {
        r->converged[j] = f.converged[j];
        r->breakdown[j] = f.breakdown[j];
        r->iterations[j] = f.iterations[j];
        r->true_residual[j] = f.true_residual[j];
        r->relative_residual[j] = f.relative_residual[j];
    }
    return (int)m;
}

bool bad_engine(E *e) { return !e || !e->H; }

}  // namespace

// ------------------------------------------------------------------ ABI
extern "C" {

int kmsd_engine_create(kmsd_csr h, kmsd_metric m, const int *vel_kind, const kmsd_csr *vel, double rtol,
                       double atol, int maxiter, double hbar, int precision, kmsd_engine *out) {
    if (!h || !m || !out || !vel_kind || h->n != m->n) return fail(KMSD_EINVAL, "invalid engine operators");
    if (precision != KMSD_FP64 && precision != KMSD_MIXED) return fail(KMSD_EINVAL, "invalid engine precision");
    for (int a = 0; a < 3; ++a) {
        const int k = vel_kind[a];
        const int need = k == 0 || k == 1 ? 1 : k == 2 ? 3 : 0;
        if (k < -1 || k > 2) return fail(KMSD_EINVAL, "invalid engine operators");
        for (int j = 0; j < need; ++j)
            if (!vel || !vel[3 * a + j] || vel[3 * a + j]->n != h->n)
                return fail(KMSD_EINVAL, "invalid engine operators");
    }
    auto *e = new kmsd_engine_s();
    e->H = h;
    e->M = m;
    for (int a = 0; a < 3; ++a) {
        e->vel_kind[a] = vel_kind[a];
        for (int j = 0; j < 3; ++j) e->vel[3 * a + j] = vel ? vel[3 * a + j] : nullptr;
    }
    e->rtol = rtol;
    e->atol = atol;
    e->maxiter = maxiter;
    e->hbar = hbar;
    e->precision = precision;
    e->identity = m->identity;
    *out = e;
    return KMSD_OK;
}

void kmsd_engine_destroy(kmsd_engine e) {
    if (!e) return;
    for (DevBuf *d : {&e->ta, &e->tb, &e->bra, &e->hx, &e->t1, &e->t2, &e->t3, &e->t4, &e->t5, &e->psi, &e->vc,
                      &e->inj[0], &e->inj[1], &e->inj[2], &e->outw, &e->status, &e->report, &e->dots})
        d->release();
    e->red.partial.release();
    e->red.ticket.release();
    delete e;
}

int kmsd_engine_h_action(kmsd_engine e, const void *b_in, void *out, int64_t b, void *stream) {
    if (bad_engine(e) || !b_in || !out || b < 1) return fail(KMSD_EINVAL, "expected nonempty finite (N,batch) array");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = begin(e, s);
    if (rc) return rc;
    const Ctl c{e->rtol, e->atol, e->maxiter};
    rc = h_action(e, static_cast<const double2 *>(b_in), static_cast<double2 *>(out), b, c, s);
    if (rc) return rc;
    return finish(e, s);
}

int kmsd_engine_v_cov(kmsd_engine e, const double *direction, const void *b_in, void *out, int64_t b, double rtol,
                      double atol, int maxiter, void *stream) {
    if (bad_engine(e) || !b_in || !out || b < 1) return fail(KMSD_EINVAL, "expected nonempty finite (N,batch) array");
    if (!direction) return fail(KMSD_EINVAL, "direction must have three components");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = begin(e, s);
    if (rc) return rc;
    const Ctl c = maxiter >= 1 ? Ctl{rtol, atol, maxiter} : Ctl{e->rtol, e->atol, e->maxiter};
    rc = v_cov(e, direction, static_cast<const double2 *>(b_in), static_cast<double2 *>(out), b, c, s);
    if (rc) return rc;
    return finish(e, s);
}

int kmsd_engine_series(kmsd_engine e, const void *b_in, void *out, int64_t b, const double *coeff, int64_t ncoeff,
                       double center, double half, const double *directions, int64_t ndir, void *stream) {
    if (bad_engine(e) || !b_in || !out || b < 1) return fail(KMSD_EINVAL, "expected nonempty finite (N,batch) array");
    if (!coeff || ncoeff < 1) return fail(KMSD_EINVAL, "empty Chebyshev coefficients");
    if (ndir < 0 || ndir > 3 || (ndir && !directions)) return fail(KMSD_EINVAL, "invalid augmented block columns");
    if (ncoeff > 1 && !(half > 0)) return fail(KMSD_EINVAL, "spectral half-width must be positive");
    if (ndir && b % (ndir + 1)) return fail(KMSD_EINVAL, "invalid augmented block columns");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = begin(e, s);
    if (rc) return rc;
    rc = series_impl(e, static_cast<const double2 *>(b_in), static_cast<double2 *>(out), b, coeff, ncoeff, center,
                     half, directions, ndir, s);
    if (rc) return rc;
    return finish(e, s);
}

int kmsd_engine_chain_correlate(kmsd_engine e, const void *b_in, const void *cov, int64_t b, int64_t length,
                                int64_t kcols, double center, double half, void *tables, void *stream) {
    if (bad_engine(e) || !b_in || !cov || !tables || b < 1 || kcols < 1)
        return fail(KMSD_EINVAL, "expected nonempty finite (N,batch) array");
    if (length < 1) return fail(KMSD_EINVAL, "Chebyshev chain must be nonempty");
    if (length > 1 && !(half > 0)) return fail(KMSD_EINVAL, "spectral half-width must be positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = begin(e, s);
    if (rc) return rc;
    rc = correlate_impl(e, static_cast<const double2 *>(b_in), static_cast<const double2 *>(cov), b, length, kcols,
                        center, half, static_cast<double2 *>(tables), s);
    if (rc) return rc;
    return finish(e, s);
}

int kmsd_engine_chain(kmsd_engine e, const void *b_in, void *out, int64_t b, int64_t length, double center,
                      double half, void *stream) {
    if (bad_engine(e) || !b_in || !out || b < 1) return fail(KMSD_EINVAL, "expected nonempty finite (N,batch) array");
    if (length < 1) return fail(KMSD_EINVAL, "Chebyshev chain must be nonempty");
    if (length > 1 && !(half > 0)) return fail(KMSD_EINVAL, "spectral half-width must be positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = begin(e, s);
    if (rc) return rc;
    rc = chain_impl(e, static_cast<const double2 *>(b_in), static_cast<double2 *>(out), b, length, center, half, s);
    if (rc) return rc;
    return finish(e, s);
}

int kmsd_engine_moments(kmsd_engine e, const void *b_in, double *mu, int64_t b, int64_t length, double center,
                        double half, int flags, void *stream) {
    if (bad_engine(e) || !b_in || !mu || b < 1) return fail(KMSD_EINVAL, "expected nonempty finite (N,batch) array");
    if (length < 1) return fail(KMSD_EINVAL, "moment count must be positive");
    if (length > 1 && !(half > 0)) return fail(KMSD_EINVAL, "spectral half-width must be positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = begin(e, s);
    if (rc) return rc;
    rc = moments_impl(e, static_cast<const double2 *>(b_in), mu, b, length, center, half, flags, s);
    if (rc) return rc;
    return finish(e, s);
}

int kmsd_engine_inner(kmsd_engine e, const void *a, const void *b_in, void *out, int64_t b, void *stream) {
    if (bad_engine(e) || !a || !b_in || !out || b < 1) return fail(KMSD_EINVAL, "invalid inner product operands");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = e->H->n;
    if (e->identity)
        return coldot64(static_cast<const double2 *>(a), static_cast<const double2 *>(b_in), n, b,
                        static_cast<double2 *>(out), s);
    if (ensure_vec(e->t1, n, b)) return KMSD_ECUDA;
    int rc = spmm64(e->M->S, static_cast<const double2 *>(b_in), e->t1.as<double2>(), b, s);
    if (rc) return rc;
    return coldot64(static_cast<const double2 *>(a), e->t1.as<double2>(), n, b, static_cast<double2 *>(out), s);
}

int kmsd_engine_lanczos(kmsd_engine e, const void *v0, int64_t steps, double *alpha, double *beta, void *stream) {
    if (bad_engine(e) || !v0 || !alpha || !beta || steps < 1) return fail(KMSD_EINVAL, "invalid Lanczos arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t n = e->H->n;
    int rc = begin(e, s);
    if (rc) return rc;
    // v, v_prev, H v, w, S w, then the (alpha, beta^2) dots and betas; freed
    // when the call returns (after its synchronisation on success)
    DevBuf work;
    struct Release {
        DevBuf &b;
        cudaStream_t s;
        ~Release() {
            cudaStreamSynchronize(s);
            b.release();
        }
    } release_work{work, s};
    if (work.ensure((size_t)5 * n * sizeof(double2) + (size_t)steps * (2 * sizeof(double2) + sizeof(double))))
        return KMSD_ECUDA;
    double2 *v = work.as<double2>(), *vp = v + n, *hv = vp + n, *w = hv + n, *sw = w + n;
    double2 *dots = sw + n;  // [2 steps]: <v, H v>, <w, S w>
    double *bet = reinterpret_cast<double *>(dots + 2 * steps);
    const Ctl c{e->rtol, e->atol, e->maxiter};
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8));
    // S-normalise the start vector
    KMSD_CUDA(cudaMemcpyAsync(w, v0, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    KMSD_CUDA(cudaMemsetAsync(vp, 0, n * sizeof(double2), s));
    const double2 *swp = w;
    if (!e->identity) {
        if ((rc = spmm64(e->M->S, w, sw, 1, s))) return rc;
        swp = sw;
    }
    if ((rc = coldot64(w, swp, n, 1, dots + 2 * steps - 1, s))) return rc;  // (scratch slot, overwritten later)
    lanczos_scale_kernel<<<grid, 256, 0, s>>>(w, v, n, dots + 2 * steps - 1, nullptr);
    count_launch();
    for (int64_t j = 0; j < steps; ++j) {
        // H v; alpha_j = <v, S w> = <v, H v> for w = S^-1 H v
        if ((rc = spmm64(e->H, v, hv, 1, s))) return rc;
        if ((rc = coldot64(v, hv, n, 1, dots + 2 * j, s))) return rc;
        if (e->identity) {
            KMSD_CUDA(cudaMemcpyAsync(w, hv, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        } else if ((rc = solve(e, hv, w, 1, c, s))) {
            return rc;
        }
        ++e->h_calls;
        lanczos_update_kernel<<<grid, 256, 0, s>>>(w, v, vp, n, dots + 2 * j, j ? bet + j - 1 : nullptr);
        count_launch();
        swp = w;
        if (!e->identity) {
            if ((rc = spmm64(e->M->S, w, sw, 1, s))) return rc;
            swp = sw;
        }
        if ((rc = coldot64(w, swp, n, 1, dots + 2 * j + 1, s))) return rc;
        // v_prev <- v, v <- w / beta_j
        KMSD_CUDA(cudaMemcpyAsync(vp, v, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        lanczos_scale_kernel<<<grid, 256, 0, s>>>(w, v, n, dots + 2 * j + 1, bet + j);
        count_launch();
    }
    KMSD_CUDA(cudaGetLastError());
    std::vector<double2> hd(2 * steps);
    KMSD_CUDA(cudaMemcpyAsync(hd.data(), dots, 2 * steps * sizeof(double2), cudaMemcpyDeviceToHost, s));
    KMSD_CUDA(cudaMemcpyAsync(beta, bet, steps * sizeof(double), cudaMemcpyDeviceToHost, s));
    if ((rc = finish(e, s))) return rc;
    for (int64_t j = 0; j < steps; ++j) alpha[j] = hd[2 * j].x;
    return KMSD_OK;
}

int kmsd_engine_counters(kmsd_engine e, int64_t *h_calls, int64_t *v_calls) {
    if (bad_engine(e)) return fail(KMSD_EINVAL, "invalid engine");
    if (h_calls) *h_calls = e->h_calls;
    if (v_calls) *v_calls = e->v_calls;
    return KMSD_OK;
}

int kmsd_engine_failure_report(kmsd_engine e, kmsd_solve_report *report, int64_t capacity, int64_t *ncols) {
    if (bad_engine(e)) return fail(KMSD_EINVAL, "invalid engine");
    const int m = fill_report(e->last, report, capacity);
    if (ncols) *ncols = m;
    return KMSD_OK;
}

}  // extern "C"
