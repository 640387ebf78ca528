// Device statistics of the stochastic transport driver: the Jackson-KPM
// projection of moments onto the energy grid and the paired block bootstrap
// of ratio estimators, so block sums stay in device memory until the
// normalised results are read back once.
//
// kmsd_project_moments: out[c][e] = sum_l G[e][l] mu[l][c] (the (G mu)^T of
//   src/kubo_msd/solvers/chebyshev.py:50-54), one warp per (c, e), lanes over l
//   in a fixed order.
// kmsd_bootstrap_ratio: the paired block bootstrap of sums of
//   src/kubo_msd/observables/statistics.py:5-23 (device form:
//   kubo_msd_gpu/.../observables/statistics_gpu.py:6-28): value = sum_k A_k /
//   sum_k D_k and stderr = std over resamples r (ddof 1) of
//   (sum_k w_rk A_k) / (sum_k w_rk D_k), a ratio with a zero denominator being
//   NaN, as in the reference.  The resampling weights w (counts of each block
//   in each resample) are drawn on the host from the reference's seed and
//   passed in.  One thread per output element; two passes over the
//   resamples (mean, then squared deviations).
#include <algorithm>
#include <cmath>

#include "kmsd.h"
#include "kmsd_impl.h"

using namespace kmsd;

namespace {

__global__ void project_kernel(const double *mu, int64_t M, int64_t b, const double *G, int64_t ne, double *out) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t w = blockIdx.x * (int64_t)(blockDim.x / 32) + threadIdx.x / 32; w < b * ne; w += warps) {
        const int64_t c = w / ne, e = w % ne;
        const double *gr = G + e * M;
        double s = 0.;
        for (int64_t l = lane; l < M; l += 32) s = fma(gr[l], mu[l * b + c], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[w] = s;
    }
}

__device__ __forceinline__ double resampled_ratio(const double *A, const double *D, const double *w, int nb,
                                                  int64_t P, int64_t ne, int64_t p) {
    double ra = 0., rd = 0.;
    for (int k = 0; k < nb; ++k) {
        const double wk = w[k];
        ra = fma(wk, A[(int64_t)k * P + p], ra);
        rd = fma(wk, D[(int64_t)k * ne + p % ne], rd);
    }
    return rd != 0. ? ra / rd : NAN;
}

// A: (nb, P) block numerators; D: (nb, ne) block denominators, broadcast over
// the leading dimensions of P (the energy axis is last); w: (nres, nb).
__global__ void bootstrap_kernel(const double *A, const double *D, int nb, int64_t P, int64_t ne, const double *w,
                                 int nres, double *value, double *stderr_out) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
        double ta = 0., td = 0.;
        for (int k = 0; k < nb; ++k) {
            ta += A[(int64_t)k * P + p];
            td += D[(int64_t)k * ne + p % ne];
        }
        value[p] = td != 0. ? ta / td : NAN;
        if (stderr_out == nullptr) continue;
        double mean = 0.;
        for (int r = 0; r < nres; ++r) mean += resampled_ratio(A, D, w + (int64_t)r * nb, nb, P, ne, p);
        mean /= nres;
        double ss = 0.;
        for (int r = 0; r < nres; ++r) {
            const double d = resampled_ratio(A, D, w + (int64_t)r * nb, nb, P, ne, p) - mean;
            ss = fma(d, d, ss);
        }
        stderr_out[p] = sqrt(ss / (nres - 1));
    }
}

// ---------------------------------------------------------------- phases
// The random phases of the reference's sampler, exp(2 pi i u) with u the
// doubles of NumPy's Generator(PCG64(SeedSequence([seed, id]))).random(n)
// (src/kubo_msd/metric/sampling.py:8-9), generated on the device.  PCG64 is
// the published PCG XSL-RR 128/64 generator (O'Neill 2014): a 128-bit LCG,
// state <- state * A + inc, whose output is rotr64(hi ^ lo, state >> 122) of
// the new state; a double is (output >> 11) * 2^-53.  The per-column seeding
// (SeedSequence) is done by the caller, which passes each column's 128-bit
// state and increment.  A thread jumps its column's stream to the first row
// of its chunk (LCG jump-ahead by repeated squaring) and then steps through
// the chunk, so every u is bit-identical to NumPy's.
using u128 = unsigned __int128;
__device__ __forceinline__ u128 pcg_mult() {
    return ((u128)0x2360ED051FC65DA4ull << 64) | (u128)0x4385DF649FCCF645ull;
}
__device__ __forceinline__ u128 pcg_advance(u128 state, u128 inc, uint64_t delta) {
    u128 am = 1, ap = 0, cm = pcg_mult(), cp = inc;
    while (delta) {
        if (delta & 1) {
            am *= cm;
            ap = ap * cm + cp;
        }
        cp = (cm + 1) * cp;
        cm *= cm;
        delta >>= 1;
    }
    return am * state + ap;
}
__device__ __forceinline__ uint64_t pcg_output(u128 state) {
    const unsigned rot = (unsigned)(state >> 122);
    const uint64_t x = (uint64_t)(state >> 64) ^ (uint64_t)state;
    return (x >> rot) | (x << ((64u - rot) & 63u));
}

constexpr int kPhaseChunk = 256;

// st: per column {state_lo, state_hi, inc_lo, inc_hi}; out (n, b) complex128.
__global__ void phases_kernel(int64_t n, int b, const uint64_t *st, double2 *out) {
    const int64_t chunks = (n + kPhaseChunk - 1) / kPhaseChunk;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < chunks * b;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(t % b);
        const int64_t r0 = (t / b) * kPhaseChunk, r1 = min(n, r0 + kPhaseChunk);
        const u128 inc = ((u128)st[4 * c + 3] << 64) | st[4 * c + 2];
        u128 state = pcg_advance(((u128)st[4 * c + 1] << 64) | st[4 * c], inc, (uint64_t)r0);
        const u128 A = pcg_mult();
        const double two_pi = 2. * 3.141592653589793;
        for (int64_t r = r0; r < r1; ++r) {
            state = state * A + inc;
            const double u = (double)(pcg_output(state) >> 11) * (1. / 9007199254740992.);
            double sn, cs;
            sincos(two_pi * u, &sn, &cs);
            out[r * b + c] = make_double2(cs, sn);
        }
    }
}

int grid_for_elems(int64_t total) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 8));
}

}  // namespace

extern "C" int kmsd_project_moments(const double *mu, int64_t length, int64_t b, const double *G, int64_t n_energy,
                                    double *out, void *stream) {
    if (!mu || !G || !out || length < 1 || b < 1 || n_energy < 1)
        return fail(KMSD_EINVAL, "invalid moment projection arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t warps = b * n_energy;
    project_kernel<<<(int)std::max<int64_t>(1, std::min<int64_t>((warps + 7) / 8, (int64_t)sm_count() * 8)), 256, 0,
                     s>>>(mu, length, b, G, n_energy, out);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

extern "C" int kmsd_random_phases(int64_t n, int64_t b, const uint64_t *pcg_state, void *out, void *stream) {
    if (n < 1 || b < 1 || !pcg_state || !out) return fail(KMSD_EINVAL, "invalid random phase arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t threads = (n + kPhaseChunk - 1) / kPhaseChunk * b;
    phases_kernel<<<grid_for_elems(threads), 256, 0, s>>>(n, (int)b, pcg_state, static_cast<double2 *>(out));
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

extern "C" int kmsd_bootstrap_ratio(const double *A, const double *D, int64_t nblocks, int64_t P, int64_t n_energy,
                                    const double *weights, int64_t n_resamples, double *value, double *stderr_out,
                                    void *stream) {
    if (!A || !D || !value || nblocks < 1 || P < 1 || n_energy < 1 || P % n_energy)
        return fail(KMSD_EINVAL, "inconsistent statistical blocks/counts");
    if (stderr_out && (!weights || n_resamples < 2)) return fail(KMSD_EINVAL, "bootstrap needs two or more resamples");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bootstrap_kernel<<<grid_for_elems(P), 256, 0, s>>>(A, D, (int)nblocks, P, n_energy, weights, (int)n_resamples,
                                                       value, stderr_out);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}
