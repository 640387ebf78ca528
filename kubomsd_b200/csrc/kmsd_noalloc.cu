// KPM moments without any device allocation.
//
// Some callers cannot call cudaMalloc at the point where they need moments.
// Examples: a serving loop that must not stall other streams on the implicit
// device synchronisation of cudaMalloc/cudaFree; a host framework that owns
// every byte of device memory through its own pool and budget; code that must
// not hit an out-of-memory failure halfway through a run.  For them,
// kmsd_engine_moments_noalloc computes the same moments as
// kmsd_engine_moments on an orthogonal-basis engine (S = I).  Its workspace is
// a fixed block of device memory that is part of the library image: the
// vector buffers of the Chebyshev recurrence, the reduction partials and the
// reduction ticket all live in `g_moments_scratch` below.
//
// Properties a caller must know:
//  * the block is 64 MiB per GPU and is held until the process exits.  It is
//    reserved when the runtime loads the library's device code on that GPU.
//    Under CUDA's lazy module loading (the default since CUDA 12) that
//    happens at the first call on each GPU, and that first call may then
//    synchronise the device or fail with out-of-memory.  Callers that rely on
//    "no stall, no out-of-memory" make one warm-up call per GPU at start-up;
//  * calls whose buffers would not fit are rejected with KMSD_EINVAL and a
//    message naming the bytes needed; kmsd_engine_moments has no such limit;
//  * the block's device address is looked up with cudaGetSymbolAddress the
//    first time a CUDA context calls (once per context, under a lock) and is
//    cached per context.  Make that first call before any stream capture.
//    cudaDeviceReset invalidates the cache together with every engine handle,
//    whose device buffers the reset frees: no handle is usable after a reset;
//  * every call on a GPU uses the same block and leaves its contents
//    behind.  The call clears what must start at zero, so the contents left by
//    an earlier call are harmless.  Two calls that overlap on the GPU, on
//    different streams or from different threads, race on the block: order
//    them on one stream or serialise them;
//  * the call is asynchronous on `stream`: mu is complete when the stream
//    reaches the end of the call's work;
//  * a mixed-precision engine needs the complex64 copy of H, which the first
//    allocating call (kmsd_engine_moments / series / chain) creates; without
//    it the call is rejected rather than allocating.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "kmsd.h"
#include "kmsd_impl.h"
#include "kmsd_kernels.cuh"

using namespace kmsd;

// The workspace of kmsd_engine_moments_noalloc (see the file comment).
static constexpr size_t kMomentsScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_moments_scratch[kMomentsScratchBytes];

namespace {

std::mutex g_scratch_lock;
std::map<void *, void *> g_scratch_address;  // CUDA context -> device address of the block

// The current CUDA context, or null when none is current on this thread (the
// driver's cuCtxGetCurrent, reached through the runtime so the library needs
// no link-time dependency on libcuda).
int current_context(void **ctx) {
    using GetCurrent = int (*)(void **);
    // looked up once, thread-safely, on the first call
    static const GetCurrent fn = []() -> GetCurrent {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<GetCurrent>(p);
    }();
    if (fn == nullptr) return fail(KMSD_ECUDA, "cuCtxGetCurrent is not available from the driver");
    *ctx = nullptr;
    if (fn(ctx) != 0) return fail(KMSD_ECUDA, "cuCtxGetCurrent failed");
    return KMSD_OK;
}

// Device address of g_moments_scratch in the current context.  In host code
// the symbol names a host-side stand-in, not device memory, so its address is
// looked up with cudaGetSymbolAddress once per context and cached.
int scratch_address(void **out) {
    void *ctx = nullptr;
    if (int rc = current_context(&ctx)) return rc;
    if (ctx == nullptr) {
        // no context current on this thread yet: make the current device's
        // primary context current, as the runtime would on its first call
        int dev = 0;
        KMSD_CUDA(cudaGetDevice(&dev));
        KMSD_CUDA(cudaSetDevice(dev));
        if (int rc = current_context(&ctx)) return rc;
        if (ctx == nullptr) return fail(KMSD_ECUDA, "no current CUDA context for the moments scratch");
    }
    std::lock_guard<std::mutex> guard(g_scratch_lock);
    auto it = g_scratch_address.find(ctx);
    if (it == g_scratch_address.end()) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_moments_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_moments_scratch)");
        it = g_scratch_address.emplace(ctx, p).first;
    }
    *out = it->second;
    return KMSD_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

template <class T, int MU, int MODE>
int occupancy_grid(int64_t n, const RowMap &mp, size_t smem, int *grid) {
    int per_sm = 0;
    KMSD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, cheb_step_kernel<T, MU, MODE, HSRC_CSR, false>, kThreads, smem));
    if (per_sm < 1) per_sm = 1;
    const int64_t need = (n + mp.gpc - 1) / mp.gpc;
    *grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sm_count() * per_sm));
    return KMSD_OK;
}

template <class T, int MU>
int run(kmsd_engine_s *e, const double2 *B, double *mu, int64_t b, int64_t length, double center, double half,
        bool doubling, cudaStream_t s) {
    using V = typename Unit<T>::vec;
    constexpr int C = Unit<T>::C;
    const int64_t n = e->H->n;
    const int U = (int)((b + C - 1) / C);
    const RowMap mp = make_map(U, kThreads);
    const size_t smem = reduce_smem(mp, C);
    const int ncol = U * C;
    int g_first = 0, g_rest = 0;
    int rc = occupancy_grid<T, MU, MODE_DOUBLING>(n, mp, smem, &g_first);
    if (!rc) rc = occupancy_grid<T, MU, MODE_DIRECT>(n, mp, smem, &g_rest);
    if (rc) return rc;
    const int grid = std::max(g_first, g_rest);
    // scratch layout: ticket | T buffer A | T buffer B | bra (mixed, direct) | partials
    const size_t vec_bytes = align256((size_t)n * U * sizeof(V));
    const bool need_bra = C == 2 && !doubling;
    const size_t off_a = 256, off_b = off_a + vec_bytes, off_bra = off_b + vec_bytes;
    const size_t off_part = off_bra + (need_bra ? vec_bytes : 0);
    const size_t need = off_part + align256((size_t)grid * ncol * 2 * sizeof(double2));
    if (need > kMomentsScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "kmsd_engine_moments_noalloc: this call needs %zu bytes of scratch but the static block holds "
                 "%zu bytes (64 MiB); use kmsd_engine_moments for larger blocks",
                 need, kMomentsScratchBytes);
        return fail(KMSD_EINVAL, msg);
    }
    void *base = nullptr;
    if ((rc = scratch_address(&base))) return rc;
    unsigned char *sc = static_cast<unsigned char *>(base);
    Ticket *ticket = reinterpret_cast<Ticket *>(sc);
    V *ta = reinterpret_cast<V *>(sc + off_a), *tb = reinterpret_cast<V *>(sc + off_b);
    V *bra = need_bra ? reinterpret_cast<V *>(sc + off_bra) : nullptr;
    double2 *partial = reinterpret_cast<double2 *>(sc + off_part);
    KMSD_CUDA(cudaMemsetAsync(ticket, 0, 256, s));  // the ticket must start at zero

    StepArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.mp = mp;
    if constexpr (C == 2) {
        a.H = CsrView<T>{e->H->ptr, e->H->idx, reinterpret_cast<const T *>(e->H->re32),
                         e->H->complex_values ? reinterpret_cast<const T *>(e->H->im32) : nullptr};
    } else {
        a.H = CsrView<T>{e->H->ptr, e->H->idx, reinterpret_cast<const T *>(e->H->re64),
                         e->H->complex_values ? reinterpret_cast<const T *>(e->H->im64) : nullptr};
    }
    const double hw = length > 1 ? half : 1.;  // a single moment never applies the operator
    a.center = center;
    a.half = hw;
    a.inv_half = (T)(1. / hw);
    a.partial = partial;
    a.ticket = ticket;
    a.mu = mu;
    a.mlen = length;
    a.bcols = (int)b;
    const V *t0;
    if (C == 2) {
        const int64_t total = n * U;
        const int eg = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16));
        to_f32_kernel<<<eg, 256, 0, s>>>(B, reinterpret_cast<float4 *>(tb), n, (int)b, U);
        count_launch();
        if (need_bra) {
            to_f32_kernel<<<eg, 256, 0, s>>>(B, reinterpret_cast<float4 *>(bra), n, (int)b, U);
            count_launch();
        }
        t0 = tb;
        a.bra = bra;
    } else {
        t0 = reinterpret_cast<const V *>(B);
        a.bra = reinterpret_cast<const V *>(B);
    }
    // Step 1 (always in the product form): mu_0 = <T0,T0>, mu_1 = <T0,T1>.
    // Then T_k over two rotating buffers; in FP64 the read-only input is T0.
    const int64_t steps = length == 1 ? 1 : doubling ? (length + 1) / 2 : length - 1;
    const V *curr = t0, *prev = nullptr;
    V *spare = ta, *second = C == 2 ? nullptr : tb;
    for (int64_t k = 1; k <= steps; ++k) {
        V *next = k == 1 ? spare : (k == 2 && second != nullptr) ? second : const_cast<V *>(prev);
        a.curr = curr;
        a.prev = prev;
        a.next = next;
        a.first = k == 1;
        if (k == 1 || doubling) {
            a.kmom = k - 1;
            a.exact_sums = !doubling;
            cheb_step_kernel<T, MU, MODE_DOUBLING, HSRC_CSR, false><<<g_first, kThreads, smem, s>>>(a);
        } else {
            a.kmom = k;
            cheb_step_kernel<T, MU, MODE_DIRECT, HSRC_CSR, false><<<g_rest, kThreads, smem, s>>>(a);
        }
        count_launch();
        prev = curr;
        curr = next;
    }
    e->h_calls += length > 1 ? steps : 0;
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

template <class T>
int dispatch(kmsd_engine_s *e, const double2 *B, double *mu, int64_t b, int64_t length, double center, double half,
             bool doubling, cudaStream_t s) {
    constexpr int C = Unit<T>::C;
    const RowMap mp = make_map((int)((b + C - 1) / C), kThreads);
    switch (mu_for(mp)) {
        case 1: return run<T, 1>(e, B, mu, b, length, center, half, doubling, s);
        case 2: return run<T, 2>(e, B, mu, b, length, center, half, doubling, s);
    }
    return fail(KMSD_EINVAL, "too many columns for one engine call");
}

}  // namespace

extern "C" int kmsd_engine_moments_noalloc(kmsd_engine e, const void *b_in, double *mu, int64_t b, int64_t length,
                                           double center, double half, int flags, void *stream) {
    if (!e || !e->H || !b_in || !mu || b < 1) return fail(KMSD_EINVAL, "expected nonempty finite (N,batch) array");
    if (length < 1) return fail(KMSD_EINVAL, "moment count must be positive");
    if (length > 1 && !(half > 0)) return fail(KMSD_EINVAL, "spectral half-width must be positive");
    if (!e->identity)
        return fail(KMSD_EINVAL, "kmsd_engine_moments_noalloc supports orthogonal-basis engines (S = I) only");
    const bool doubling = (flags & KMSD_MOMENTS_DOUBLING) != 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double2 *B = static_cast<const double2 *>(b_in);
    if (e->precision == KMSD_MIXED) {
        if (e->H->re32 == nullptr)
            return fail(KMSD_EINVAL, "kmsd_engine_moments_noalloc: the mixed-precision engine has no complex64 copy "
                                     "of H yet; one allocating call (kmsd_engine_moments) creates it");
        return dispatch<float>(e, B, mu, b, length, center, half, doubling, s);
    }
    return dispatch<double>(e, B, mu, b, length, center, half, doubling, s);
}
