// Spectral velocity-autocorrelation tables without the stored left chain
// (the correlation reduction of src/kubo_msd/solvers/spectral.py:33-38) and
// the per-node Bessel / product-rule tail (spectral.py:39-51) on the device.
//
// tables[b, j, k] = sum_n conj(T_j(Ht) c)[n, b] * cov[n, k, b] for j < length
// and k < kcols, where cov holds the velocity applied to the right chain
// T_k(Ht) v.  The left chain is generated into a ring of kRing vector blocks
// by the engine's fused Chebyshev step; every kRing steps one contraction
// launch reduces the ring against cov:
//   * corr_partial_kernel: CTA (row chunk, tile of kJT chain vectors); each
//     thread owns one column b and up to KPT values of k for all kJT chain
//     vectors, and walks the rows of its chunk; partial sums per chunk;
//   * corr_reduce_kernel: tables = sum over chunks in chunk order.
// Row ownership and the chunk order are fixed, so the tables are the same in
// every run.  HBM per ring: the ring written once by the steps and read once
// here, and cov read once (the kRing / kJT tiles of a chunk are neighbouring
// CTAs and meet cov in L2).
#include <algorithm>
#include <cstring>
#include <vector>

#include "kmsd.h"
#include "kmsd_impl.h"
#include "kmsd_kernels.cuh"

using namespace kmsd;

namespace {

constexpr int kRing = 32;  // left-chain vector blocks held at once
constexpr int kJT = 8;     // chain vectors per contraction tile
constexpr int kCorrThreads = 256;

// partial[chunk][jj][k][b] for the ring's chain vectors jj < jn (ring slot
// (j0 + jj) % kRing), rows [chunk * rows_per, ...).
template <int KPT>
__global__ void __launch_bounds__(kCorrThreads) corr_partial_kernel(const double2 *ring, int64_t slab,
                                                                   const double2 *cov, int64_t n, int nb, int nbp,
                                                                   int k1, int64_t j0, int jn, int64_t rows_per,
                                                                   int ntiles, double2 *partial) {
    const int chunk = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
    const int t = threadIdx.x;
    const int b = t % nbp, kg = t / nbp, kgroups = kCorrThreads / nbp;
    const int jt0 = tile * kJT;
    const int64_t r0 = (int64_t)chunk * rows_per, r1 = min(n, r0 + rows_per);
    double2 acc[kJT][KPT];
#pragma unroll
    for (int jj = 0; jj < kJT; ++jj)
#pragma unroll
        for (int i = 0; i < KPT; ++i) acc[jj][i] = make_double2(0., 0.);
    const bool active = b < nb;
    const double2 *slot[kJT];
#pragma unroll
    for (int jj = 0; jj < kJT; ++jj) {
        const int jr = jt0 + jj < jn ? jt0 + jj : jn - 1;  // (clamped: never accumulated)
        slot[jj] = ring + (size_t)((j0 + jr) % kRing) * slab;
    }
    if (active) {
        for (int64_t r = r0; r < r1; ++r) {
            double2 cv[kJT], kv[KPT];
#pragma unroll
            for (int jj = 0; jj < kJT; ++jj) cv[jj] = __ldg(slot[jj] + r * nb + b);
#pragma unroll
            for (int i = 0; i < KPT; ++i) {
                const int k = kg + i * kgroups;
                kv[i] = k < k1 ? __ldg(cov + (r * k1 + k) * nb + b) : make_double2(0., 0.);
            }
#pragma unroll
            for (int jj = 0; jj < kJT; ++jj)
#pragma unroll
                for (int i = 0; i < KPT; ++i) {
                    // conj(cv) * kv
                    acc[jj][i].x = fma(cv[jj].x, kv[i].x, fma(cv[jj].y, kv[i].y, acc[jj][i].x));
                    acc[jj][i].y = fma(cv[jj].x, kv[i].y, fma(-cv[jj].y, kv[i].x, acc[jj][i].y));
                }
        }
        double2 *out = partial + (size_t)chunk * kRing * k1 * nb;
#pragma unroll
        for (int jj = 0; jj < kJT; ++jj) {
            if (jt0 + jj >= jn) break;
#pragma unroll
            for (int i = 0; i < KPT; ++i) {
                const int k = kg + i * kgroups;
                if (k < k1) out[((size_t)(jt0 + jj) * k1 + k) * nb + b] = acc[jj][i];
            }
        }
    }
}

// tables[b][j0 + jj][k] = sum over chunks (in chunk order) of partial.
__global__ void corr_reduce_kernel(const double2 *partial, int nchunks, int jn, int k1, int nb, int64_t j0,
                                   int64_t length, double2 *tables) {
    const int64_t total = (int64_t)jn * k1 * nb;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(e % nb);
        const int64_t jk = e / nb;
        const int k = (int)(jk % k1), jj = (int)(jk / k1);
        double sx = 0., sy = 0.;
        const size_t stride = (size_t)kRing * k1 * nb;
        for (int c = 0; c < nchunks; ++c) {
            const double2 v = partial[c * stride + ((size_t)jj * k1 + k) * nb + b];
            sx += v.x;
            sy += v.y;
        }
        tables[((size_t)b * length + j0 + jj) * k1 + k] = make_double2(sx, sy);
    }
}

using PartialFn = void (*)(const double2 *, int64_t, const double2 *, int64_t, int, int, int, int64_t, int, int64_t,
                           int, double2 *);

PartialFn partial_kernel(int kpt) {
    switch (kpt) {
        case 1: return corr_partial_kernel<1>;
        case 2: return corr_partial_kernel<2>;
        case 3: return corr_partial_kernel<3>;
        case 4: return corr_partial_kernel<4>;
    }
    return nullptr;
}

// ------------------------------------------------------------------ node tail
// For the spectral nodes t_m of one segment, with Bessel coefficients
// coef[m][p] (p <= kt[m]):
//   q[m][b][j]   = sum_{k <= kt[m]} tables[b][j][k] coef[m][k]          (j < L + kt[m])
//   mom[m][b][l] = Re sum_{p <= kt[m]} (q[l + p] + q[|l - p|]) / 2 conj(coef[m][p])   (l < L)
//   vac[m][b][e] = sum_l G[e][l] mom[m][b][l]
// (the product rule T_l T_p = (T_{l+p} + T_|l-p|) / 2 of spectral.py:43-49).
__global__ void node_q_kernel(const double2 *tables, int nb, int64_t length, int k1, const double2 *coef,
                              const int *kt, int m, int64_t L, double2 *q) {
    const int64_t total = (int64_t)m * nb * length;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e % length;
        const int64_t mb = e / length;
        const int b = (int)(mb % nb), node = (int)(mb / nb);
        const int K = kt[node];
        double sx = 0., sy = 0.;
        if (j < L + K) {
            const double2 *tr = tables + ((size_t)b * length + j) * k1;
            const double2 *cr = coef + (size_t)node * k1;
            for (int k = 0; k <= K; ++k) {
                const double2 tv = tr[k], cv = cr[k];
                sx = fma(tv.x, cv.x, fma(-tv.y, cv.y, sx));
                sy = fma(tv.x, cv.y, fma(tv.y, cv.x, sy));
            }
        }
        q[e] = make_double2(sx, sy);
    }
}

__global__ void node_moments_kernel(const double2 *q, int nb, int64_t length, int k1, const double2 *coef,
                                    const int *kt, int m, int64_t L, double *mom) {
    const int64_t total = (int64_t)m * nb * L;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t l = e % L;
        const int64_t mb = e / L;
        const int node = (int)(mb / nb);
        const int K = kt[node];
        const double2 *qr = q + mb * length;
        const double2 *cr = coef + (size_t)node * k1;
        double s = 0.;
        for (int p = 0; p <= K; ++p) {
            const double2 a = qr[l + p], c = qr[l >= p ? l - p : p - l], cv = cr[p];
            // Re((a + c) / 2 * conj(cv))
            s += .5 * ((a.x + c.x) * cv.x + (a.y + c.y) * cv.y);
        }
        mom[e] = s;
    }
}

// vac[row][e] = sum_l G[e][l] mom[row][l]; one warp per (row, e).
__global__ void node_project_kernel(const double *mom, int64_t rows, int64_t L, const double *G, int ne,
                                    double *vac) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t w = blockIdx.x * (int64_t)(blockDim.x / 32) + threadIdx.x / 32; w < rows * ne; w += warps) {
        const int64_t row = w / ne;
        const int e = (int)(w % ne);
        const double *mr = mom + row * L, *gr = G + (size_t)e * L;
        double s = 0.;
        for (int64_t l = lane; l < L; l += 32) s = fma(gr[l], mr[l], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) vac[w] = s;
    }
}

}  // namespace

namespace kmsd {

// One contraction of the ring's chain vectors [j0, j0 + jn) against cov.
int corr_ring(const double2 *ring, int64_t n, int nb, const double2 *cov, int k1, int64_t j0, int jn,
              int64_t length, double2 *tables, DevBuf &partial, cudaStream_t s) {
    const int nbp = nb <= 1 ? 1 : nb <= 2 ? 2 : nb <= 4 ? 4 : 8;
    const int kgroups = kCorrThreads / nbp;
    const int kpt = (k1 + kgroups - 1) / kgroups;
    const PartialFn fn = partial_kernel(kpt);
    if (nb > 8 || fn == nullptr)
        return fail(KMSD_EINVAL, "correlation tables take at most 8 vectors and 1024/vectors right-chain terms per call");
    const int ntiles = (jn + kJT - 1) / kJT;
    int nchunks = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sm_count() * 4 / ntiles, n));
    const int64_t rows_per = (n + nchunks - 1) / nchunks;
    nchunks = (int)((n + rows_per - 1) / rows_per);
    if (partial.ensure((size_t)nchunks * kRing * k1 * nb * sizeof(double2))) return KMSD_ECUDA;
    fn<<<nchunks * ntiles, kCorrThreads, 0, s>>>(ring, n * nb, cov, n, nb, nbp, k1, j0, jn, rows_per, ntiles,
                                                 partial.as<double2>());
    count_launch();
    const int64_t total = (int64_t)jn * k1 * nb;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 8));
    corr_reduce_kernel<<<grid, 256, 0, s>>>(partial.as<double2>(), nchunks, jn, k1, nb, j0, length, tables);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}

int ring_slots() { return kRing; }

}  // namespace kmsd

extern "C" int kmsd_vac_nodes(const void *tables, int64_t b, int64_t length, int64_t kcols, int64_t n_moments,
                              const void *coeff, const int *orders, int64_t nodes, const double *G,
                              int64_t n_energy, void *work, int64_t work_bytes, double *vac, void *stream) {
    if (!tables || !coeff || !orders || !G || !vac || b < 1 || nodes < 1 || n_energy < 1 || n_moments < 1 ||
        kcols < 1 || length < n_moments)
        return fail(KMSD_EINVAL, "invalid spectral node arguments");
    const int64_t need = nodes * b * length * (int64_t)sizeof(double2) + nodes * b * n_moments * 8;
    if (!work || work_bytes < need) return fail(KMSD_EINVAL, "spectral node workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double2 *q = static_cast<double2 *>(work);
    double *mom = reinterpret_cast<double *>(q + nodes * b * length);
    auto grid_of = [](int64_t total) {
        return (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 8));
    };
    node_q_kernel<<<grid_of(nodes * b * length), 256, 0, s>>>(static_cast<const double2 *>(tables), (int)b, length,
                                                              (int)kcols, static_cast<const double2 *>(coeff), orders,
                                                              (int)nodes, n_moments, q);
    count_launch();
    node_moments_kernel<<<grid_of(nodes * b * n_moments), 256, 0, s>>>(q, (int)b, length, (int)kcols,
                                                                       static_cast<const double2 *>(coeff), orders,
                                                                       (int)nodes, n_moments, mom);
    count_launch();
    const int64_t warps = nodes * b * n_energy;
    node_project_kernel<<<(int)std::max<int64_t>(1, std::min<int64_t>((warps + 7) / 8, (int64_t)sm_count() * 8)),
                          256, 0, s>>>(mom, nodes * b, n_moments, G, (int)n_energy, vac);
    count_launch();
    KMSD_CUDA(cudaGetLastError());
    return KMSD_OK;
}
