/*
 * kmsd.h — C ABI of the B200 stochastic-KPM transport engine (libkmsd_b200.so).
 *
 * The library replaces the compiled CPU engine of KuboMSD (`kubo_msd._native`,
 * cpp/native.cpp) behind the same three objects — a sparse matrix (CSR), an
 * overlap metric (Metric) and a transport engine (Engine) — with the same
 * operations, argument meaning and error classes.  Every operation works on
 * DEVICE buffers that the caller owns: vector blocks are row-major (N, b)
 * arrays of complex128 (interleaved re/im doubles, b contiguous per row),
 * exactly the layout of the reference's `Dense` (cpp/native.cpp:26-41).
 * Matrices are passed once, as host CSR arrays, and are uploaded and owned by
 * the library.  Work is queued on the caller's CUDA stream (`stream` is a
 * cudaStream_t passed as void*; NULL = legacy default stream).  The engine
 * operations and kmsd_metric_solve end with ONE synchronisation of that
 * stream to read the device status word (failed solve acceptance, nonfinite
 * propagation), so they return only when their results are ready; the
 * functions documented as asynchronous do not synchronise.
 *
 * Return value of every int function: KMSD_OK or an error class.  The message
 * of the last error on the calling thread is returned by kmsd_last_error().
 * Error classes mirror the reference's exceptions:
 *   KMSD_EINVAL   std::invalid_argument  -> ValueError        (native.cpp:33,63,316,...)
 *   KMSD_ERUNTIME std::runtime_error     -> RuntimeError      (native.cpp:571)
 *   KMSD_EMETRIC  MetricFailure          -> RuntimeError with per-column
 *                                           diagnostics       (native.cpp:139-143,447-450)
 *   KMSD_ECUDA    CUDA runtime failure (no reference counterpart)
 *
 * Handles are not thread-safe: one call at a time per handle (each handle owns
 * its device workspace).  Different handles may be used concurrently.
 */
#ifndef KMSD_H
#define KMSD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KMSD_OK 0
#define KMSD_EINVAL 1
#define KMSD_ERUNTIME 2
#define KMSD_EMETRIC 3
#define KMSD_ECUDA 4

/* Arithmetic of an engine (kmsd_engine_create).  FP64: complex128 vectors and
 * SpMM, the reference's precision.  MIXED: complex64 vectors and SpMM inside
 * the Chebyshev recurrences; moment/correlation accumulation, metric solves,
 * inner products and norms stay FP64.  Inputs and outputs are complex128 in
 * both modes. */
#define KMSD_FP64 0
#define KMSD_MIXED 1

/* kmsd_engine_moments flags. */
#define KMSD_MOMENTS_DIRECT 0   /* mu_k = Re<S B, T_k B>, one operator application per moment */
#define KMSD_MOMENTS_DOUBLING 1 /* mu_2n = 2<T_n,S T_n>-mu_0, mu_2n+1 = 2<T_n+1,S T_n>-mu_1 (S = I only) */

typedef struct kmsd_csr_s *kmsd_csr;
typedef struct kmsd_metric_s *kmsd_metric;
typedef struct kmsd_engine_s *kmsd_engine;

/* Per-column report of one metric solve; arrays of length b, caller-allocated
 * HOST memory.  Mirrors SolveReport (cpp/native.cpp:123-129) and the Python
 * MetricSolveReport (src/kubo_msd/contracts.py:33-39). */
typedef struct {
    uint8_t *converged;
    uint8_t *breakdown;
    int64_t *iterations;
    double *true_residual;
    double *relative_residual;
} kmsd_solve_report;

/* Cumulative metric counters; mirrors Metric::diagnostics
 * (cpp/native.cpp:666-675). */
typedef struct {
    int64_t calls;
    int64_t max_iterations_sum;
    double seconds;
    double max_relative_residual;
    int64_t true_residual_refreshes;
    int64_t true_residual_checks;
    int64_t residual_restarts;
    int64_t refinement_steps;
} kmsd_metric_stats;

/* ---- library ---------------------------------------------------------- */

/* Thread-local message of the last failed call ("" if none). */
const char *kmsd_last_error(void);

/* Static description (language, precision, architecture); mirrors
 * `_native.build_info()` (cpp/native.cpp:631-639). */
const char *kmsd_build_info(void);

/* Device ordinal the library will use (the caller's current device). */
int kmsd_device(int *device);

/* Number of kernels this library has launched in the process so far (all
 * devices).  No counterpart in the reference; used to account the work of a
 * timed region. */
int64_t kmsd_kernel_launches(void);

/* ---- CSR: replaces `_native.CSR` (cpp/native.cpp:54-90, 640-646) -------- */

/* n rows, n columns; indptr[n+1], indices[nnz] (int64, host, 0-based);
 * values: val_re[nnz] and val_im[nnz] (val_im NULL for a real matrix).
 * Validation follows the reference constructor (cpp/native.cpp:59-74):
 * monotone pointers starting at 0 and ending at nnz, indices in [0,n),
 * finite entries; otherwise KMSD_EINVAL "invalid CSR ...".  Rows need not be
 * sorted; entries are applied in the given order. */
int kmsd_csr_create(int64_t n, const int64_t *indptr, const int64_t *indices,
                    const double *val_re, const double *val_im, kmsd_csr *out);
void kmsd_csr_destroy(kmsd_csr a);
int64_t kmsd_csr_rows(kmsd_csr a);
int64_t kmsd_csr_nnz(kmsd_csr a);
/* Device storage forms built at upload besides CSR, as a bit mask:
 * KMSD_FORM_ELL (padded rows of width <= 32, padding <= 25%) and
 * KMSD_FORM_BSR4 (dense 4x4 blocks, zero fill <= 25%).  No counterpart in the
 * reference, which keeps CSR only; -1 for a null handle. */
#define KMSD_FORM_ELL 1
#define KMSD_FORM_BSR4 2
int kmsd_csr_forms(kmsd_csr a);

/* Y = A X for device complex128 X, Y of shape (n, b).  Replaces CSR::mul /
 * `CSR.matmul` (cpp/native.cpp:75-89, 642-646).  X and Y must not overlap. */
int kmsd_csr_matmul(kmsd_csr a, const void *x, void *y, int64_t b, void *stream);

/* ---- Metric: replaces `_native.Metric` (cpp/native.cpp:150-480, 647-675) */

/* S: overlap (kept by reference; destroy the metric before S).
 * diag[n] > 0: the preconditioner diagonal (positive, finite).
 * Block-Jacobi factors (optional, nblocks = 0 for the diagonal
 * preconditioner): block i covers rows [block_start[i], block_start[i+1]),
 * block_start[0] = 0, block_start[nblocks] = n, each block at most 32 rows;
 * its lower Cholesky factor is stored row-major at factor_offset[i] in
 * factor_re/factor_im (m*m entries).  Mirrors Metric(S, diagonal, blocks)
 * (cpp/native.cpp:212-236) and its "invalid block-Jacobi factor partition" /
 * "incomplete block-Jacobi partition" checks. */
int kmsd_metric_create(kmsd_csr s, const double *diag, int64_t nblocks,
                       const int64_t *block_start, const int64_t *factor_offset,
                       const double *factor_re, const double *factor_im,
                       kmsd_metric *out);
void kmsd_metric_destroy(kmsd_metric m);

/* policy 0 = fixed, 1 = adaptive; interval >= 1; 0 < gap_ratio < 1.
 * Replaces Metric::set_residual_policy (cpp/native.cpp:206-210). */
int kmsd_metric_set_residual_policy(kmsd_metric m, int policy, int interval,
                                    double gap_ratio);

/* Y = S^-1 B by batched preconditioned CG, one independent recurrence per
 * column, with the reference's per-column RHS scaling, thresholds
 * max(rtol*||q||, atol/safe), curvature-breakdown test, true-residual refresh
 * every `interval` iterations, final true-residual acceptance and
 * representability checks (Metric::solve, cpp/native.cpp:313-452).
 * Synchronises the stream once to read the per-column status.  On failure
 * returns KMSD_EMETRIC with the reference's message and fills `report`
 * (which may be NULL when not wanted). */
int kmsd_metric_solve(kmsd_metric m, const void *b_in, void *y_out, int64_t b,
                      double rtol, double atol, int maxiter,
                      kmsd_solve_report *report, void *stream);

/* Declare S block-diagonal over the row ranges [row_offsets[s],
 * row_offsets[s+1]), s < nseg (row_offsets[0] = 0, row_offsets[nseg] = n): a
 * later kmsd_metric_solve then runs one CG per (segment, column), each with
 * the reference's per-column semantics (thresholds, breakdown, refresh,
 * acceptance), all segments in the same launches.  This solves the metric
 * systems of many independent instances (a ragged batch) at once.  The
 * report arrays then hold nseg * b entries, segment-major.  Fails with
 * KMSD_EINVAL when S couples two segments or a block-Jacobi block crosses a
 * boundary; nseg <= 1 restores the single system.  No counterpart in the
 * reference, which solves one system per metric. */
int kmsd_metric_set_segments(kmsd_metric m, int64_t nseg, const int64_t *row_offsets);

/* Storage of the CG work vectors (r, z, p, S p and the true residual):
 * KMSD_FP64 (default) or KMSD_MIXED (complex64).  Every operation on them
 * stays FP64, and so do the right-hand side, the solution, every inner
 * product and norm, the breakdown test and the true-residual acceptance; the
 * mixed form halves the solve's vector traffic.  No counterpart in the
 * reference, whose solve is complex128 throughout. */
int kmsd_metric_set_storage(kmsd_metric m, int precision);

/* out = D^-1/2 p(W) xi with W = (D^-1/2 S D^-1/2 - center)/half and p the
 * Chebyshev series `coeff` (Clenshaw).  Replaces Metric::sample
 * (cpp/native.cpp:453-479). */
int kmsd_metric_sample(kmsd_metric m, const void *xi, void *out, int64_t b,
                       const double *coeff, int64_t ncoeff, double center,
                       double half, void *stream);

/* Read the cumulative counters (synchronises the device). */
int kmsd_metric_stats_get(kmsd_metric m, kmsd_metric_stats *out);

/* 1 when S is exactly the identity and the preconditioner is the unit
 * diagonal: solves are then exact copies and the engine skips them. */
int kmsd_metric_is_identity(kmsd_metric m);

/* ---- Engine: replaces `_native.Engine` (cpp/native.cpp:488-610, 676-719) */

/* h: Hamiltonian; m: metric (same n).  vel_kind[3] for axes x,y,z:
 * -1 absent, 0 explicit covariant velocity (1 matrix), 1 position
 * (1 matrix), 2 composite bond/xbar/delta (3 matrices); vel[3*axis+j] are
 * the matrices (NULL where unused).  rtol/atol/maxiter: metric-solve
 * controls used inside every operator application; hbar in eV*fs.
 * precision: KMSD_FP64 or KMSD_MIXED.  Mirrors the Engine constructor
 * (cpp/native.cpp:495-503). */
int kmsd_engine_create(kmsd_csr h, kmsd_metric m, const int *vel_kind,
                       const kmsd_csr *vel, double rtol, double atol,
                       int maxiter, double hbar, int precision,
                       kmsd_engine *out);
void kmsd_engine_destroy(kmsd_engine e);

/* out = S^-1 H B.  Engine::h_action (cpp/native.cpp:505). */
int kmsd_engine_h_action(kmsd_engine e, const void *b_in, void *out, int64_t b,
                         void *stream);

/* out = sum_a direction[a] v_a B with v_a the covariant Cartesian velocity of
 * kind 0/1/2.  maxiter < 1 uses the engine's solve controls; otherwise
 * rtol/atol/maxiter override them for this call only (v_cov_with_controls).
 * Engine::v_cart / v_cov (cpp/native.cpp:506-533, 683-697). */
int kmsd_engine_v_cov(kmsd_engine e, const double *direction, const void *b_in,
                      void *out, int64_t b, double rtol, double atol,
                      int maxiter, void *stream);

/* out = sum_k coeff[k] T_k(A) B, A the augmented scaled operator of
 * Engine::augmented: for ndir direction rows (ndir*3 doubles), B has
 * b = nb*(1+ndir) columns [psi | phi_1..phi_ndir] and
 * A[psi; phi_a] = [Ht psi; Ht phi_a + (-i hbar/half) S^-1 v_cov(dir_a, psi)],
 * Ht = (S^-1 H - center)/half.  coeff: ncoeff complex values as interleaved
 * (re, im) doubles.  Engine::series (cpp/native.cpp:540-573); fails with
 * KMSD_ERUNTIME "nonfinite Chebyshev propagation; check bounds and solves". */
int kmsd_engine_series(kmsd_engine e, const void *b_in, void *out, int64_t b,
                       const double *coeff, int64_t ncoeff, double center,
                       double half, const double *directions, int64_t ndir,
                       void *stream);

/* out[k] = T_k(Ht) B for k < length; out is (length, n, b) complex128.
 * Engine::chain (cpp/native.cpp:574-589). */
int kmsd_engine_chain(kmsd_engine e, const void *b_in, void *out, int64_t b,
                      int64_t length, double center, double half, void *stream);

/* The correlation tables of the spectral VAC without storing the chain:
 * tables[c, j, k] = sum_n conj(T_j(Ht) B)[n, c] * cov[n, k, c]
 * for j < length, k < kcols and column c < b, written as a (b, length, kcols)
 * complex128 device array (tables[(c*length + j)*kcols + k]).  cov is the
 * (n, kcols, b) complex128 device array of the velocity applied to the right
 * chain T_k(Ht) v.  Replaces the reference's stored left chain
 * (Engine::chain, cpp/native.cpp:574-589) followed by the contraction
 * `np.einsum` of src/kubo_msd/solvers/spectral.py:33-38: the chain is
 * generated into a ring of 32 vector blocks and contracted as it goes.
 * b <= 8 and kcols <= 1024 / b per call. */
int kmsd_engine_chain_correlate(kmsd_engine e, const void *b_in, const void *cov,
                                int64_t b, int64_t length, int64_t kcols,
                                double center, double half, void *tables,
                                void *stream);

/* The per-node tail of the spectral VAC (src/kubo_msd/solvers/spectral.py:
 * 39-51) for `nodes` time nodes at once, on the device: with Bessel
 * coefficients coeff[m][p] (complex128, (nodes, kcols), device; p <= orders[m],
 * orders an int32 device array) and tables from
 * kmsd_engine_chain_correlate,
 *   q[m][c][j]   = sum_k tables[c][j][k] coeff[m][k],
 *   mom[m][c][l] = Re sum_p (q[m][c][l+p] + q[m][c][|l-p|]) / 2 conj(coeff[m][p]),
 *   vac[m][c][e] = sum_l G[e][l] mom[m][c][l]   (l < n_moments),
 * with G the (n_energy, n_moments) reconstruction matrix (float64, device)
 * and vac a (nodes, b, n_energy) float64 device array.  `work` is device
 * scratch of at least nodes*b*(16*length + 8*n_moments) bytes.  Asynchronous. */
/* The reference sampler's random phases on the device: out[r*b + c] =
 * exp(2 pi i u_rc), u_rc the r-th double of NumPy's
 * Generator(PCG64(SeedSequence([seed, id_c]))).random(n)
 * (src/kubo_msd/metric/sampling.py:8-9).  pcg_state is a device array of b x
 * 4 uint64: each column's PCG64 state (low, high 64 bits) and increment (low,
 * high) as SeedSequence sets them up.  The u are bit-identical to NumPy's;
 * the phases agree to a few ulp (device sincos).  out is (n, b) complex128 on
 * the device.  Asynchronous. */
int kmsd_random_phases(int64_t n, int64_t b, const uint64_t *pcg_state,
                       void *out, void *stream);

/* out[c*n_energy + e] = sum_l G[e*length + l] mu[l*b + c]: the projection
 * (G mu)^T of moments onto the energy grid (src/kubo_msd/solvers/
 * chebyshev.py:50-54), all arrays float64 on the device.  Asynchronous. */
int kmsd_project_moments(const double *mu, int64_t length, int64_t b,
                         const double *G, int64_t n_energy, double *out,
                         void *stream);

/* Paired block bootstrap of a ratio of block sums on the device
 * (src/kubo_msd/observables/statistics.py:5-23; the reference's device form
 * kubo_msd_gpu/src/kubo_msd/observables/statistics_gpu.py:6-28): A is the
 * (nblocks, P) block numerators and D the (nblocks, n_energy) block
 * denominators, broadcast over P = (...) x n_energy; value[p] = sum A / sum D
 * (NaN where the sum of D is zero) and, when stderr_out is not NULL,
 * stderr_out[p] = standard deviation (ddof 1) over the n_resamples rows of
 * `weights` (nres, nblocks; the count of each block in each resample, drawn
 * by the caller) of the resampled ratios.  Float64 device arrays.
 * Asynchronous. */
int kmsd_bootstrap_ratio(const double *A, const double *D, int64_t nblocks,
                         int64_t P, int64_t n_energy, const double *weights,
                         int64_t n_resamples, double *value, double *stderr_out,
                         void *stream);

int kmsd_vac_nodes(const void *tables, int64_t b, int64_t length, int64_t kcols,
                   int64_t n_moments, const void *coeff, const int *orders,
                   int64_t nodes, const double *G, int64_t n_energy, void *work,
                   int64_t work_bytes, double *vac, void *stream);

/* mu[k*b + j] = Re sum_i conj((S B)_ij) (T_k(Ht) B)_ij for k < length, on the
 * device (float64, (length, b)).  Engine::moments (cpp/native.cpp:590-609).
 * flags: KMSD_MOMENTS_DIRECT or KMSD_MOMENTS_DOUBLING (S = I only). */
int kmsd_engine_moments(kmsd_engine e, const void *b_in, double *mu, int64_t b,
                        int64_t length, double center, double half, int flags,
                        void *stream);

/* The moments of kmsd_engine_moments, computed without allocating device
 * memory; no counterpart in the reference.  For callers that cannot call
 * cudaMalloc where they need moments: serving loops that must not stall on
 * the device synchronisation of cudaMalloc/cudaFree, frameworks that keep
 * all device memory in their own pool, code that must not fail with
 * out-of-memory mid-run.  Orthogonal-basis engines (S = I) only; FP64, or
 * MIXED once an allocating call has created the complex64 copy of H.  The
 * workspace is one static 64 MiB device block per GPU (part of the library
 * image, held until exit); calls that need more are rejected with
 * KMSD_EINVAL.  Under CUDA's lazy module loading (the default) the block is
 * reserved at the first call on each GPU, which may then synchronise or fail
 * with out-of-memory: callers that need the no-stall, no-out-of-memory
 * promise make one warm-up call per GPU at start-up.  The first call in a
 * CUDA context also looks up the block's address; make it before any stream
 * capture.  No handle survives cudaDeviceReset.  All calls on a GPU share the
 * block: calls that overlap on the GPU race, so keep them on one stream.
 * Asynchronous on `stream`; mu is device memory (length, b). */
int kmsd_engine_moments_noalloc(kmsd_engine e, const void *b_in, double *mu,
                                int64_t b, int64_t length, double center,
                                double half, int flags, void *stream);

/* `steps` Lanczos iterations of the pencil (H, S) in the S inner product,
 * started from the (n, 1) complex128 device vector v0 (S-normalised here):
 * w = S^-1 H v_j, alpha_j = <v_j, H v_j>, w -= alpha_j v_j + beta_{j-1}
 * v_{j-1}, beta_j = |w|_S, v_{j+1} = w / beta_j.  alpha and beta are HOST
 * arrays of `steps` doubles, filled at the end; every step runs on the
 * device with the scalars kept there, and the call synchronises once.  The
 * device replacement of the host ARPACK spectral-bound estimate
 * (src/kubo_msd/metric/bounds.py:26-58); the caller forms the tridiagonal
 * matrix and truncates at the first negligible beta. */
int kmsd_engine_lanczos(kmsd_engine e, const void *v0, int64_t steps, double *alpha,
                        double *beta, void *stream);

/* Reference counters h_calls / v_calls (cpp/native.cpp:718-719). */
int kmsd_engine_counters(kmsd_engine e, int64_t *h_calls, int64_t *v_calls);

/* Per-column diagnostics of the metric solve that made the last engine call
 * fail with KMSD_EMETRIC (the first failing solve of that call); the
 * reference attaches the same dict to its MetricFailure
 * (cpp/native.cpp:622-629, src/kubo_msd/backends/native.py:32-39).  Writes
 * at most `capacity` columns and their count to *ncols (host memory). */
int kmsd_engine_failure_report(kmsd_engine e, kmsd_solve_report *report,
                               int64_t capacity, int64_t *ncols);

/* out[j] = sum_i conj(A_ij) (S B)_ij, complex, into device memory as b
 * interleaved (re, im) doubles; asynchronous.  The device form of
 * OperatorBundle.inner (src/kubo_msd/operators/velocity.py:117), which the
 * reference evaluates with NumPy on the host. */
int kmsd_engine_inner(kmsd_engine e, const void *a, const void *b_in, void *out,
                      int64_t b, void *stream);

/* out[j] = sum_i conj(x_ij) y_ij for device complex128 (n, b) arrays, into
 * device memory (b complex values); deterministic order; asynchronous.  No
 * counterpart in the reference (its column sums run in NumPy). */
int kmsd_column_dot(const void *x, const void *y, int64_t n, int64_t b,
                    void *out, void *stream);

/* ---- Ragged batches (the batching form; no counterpart in the reference) */

/* A batch of `ninst` independent orthogonal-basis Hamiltonians of any sizes,
 * concatenated block-diagonally and cut into row tiles of `tile_rows` rows
 * (0: 2048) that never cross an instance.  The reference runs independent
 * disorder realisations one after another (src/kubo_msd/solvers/stochastic.py
 * per statistics block); here one kernel per Chebyshev step covers all
 * instances.  precision: KMSD_FP64 or KMSD_MIXED. */
typedef struct kmsd_batch_s *kmsd_batch;
int kmsd_batch_create(int64_t ninst, const kmsd_csr *h, int precision,
                      int64_t tile_rows, kmsd_batch *out);
void kmsd_batch_destroy(kmsd_batch bt);

/* Make the batch nonorthogonal: `h` is the block-diagonal H of all
 * instances (any storage form; 4x4 blocks pay for atom-block models) and `m`
 * a metric over the block-diagonal S with its preconditioner; the batch
 * declares m's segments to be its instances (kmsd_metric_set_segments).
 * kmsd_batch_moments then computes, per instance, mu_k = Re<S B, T_k(H~) B>
 * with T_k advanced by S^-1 H through one segmented PCG per step, in FP64,
 * with direct moments (KMSD_MOMENTS_DOUBLING is rejected) and without a
 * CUDA graph (the PCG loop stops on a polled device flag).  The handles stay
 * owned by the caller and must outlive the batch's use of them. */
int kmsd_batch_attach_metric(kmsd_batch bt, kmsd_csr h, kmsd_metric m, double rtol,
                             double atol, int maxiter);

/* Row offsets of the instances in the concatenated vector block (ninst+1
 * values, host). */
int kmsd_batch_rows(kmsd_batch bt, int64_t *offsets);

/* mu[(i*length + k)*b + j] = moment k of column j of instance i, the moments
 * of kmsd_engine_moments for each instance with its own window
 * (center[i], half[i]; host arrays).  b_in: the concatenated (sum N_i, b)
 * complex128 block (device); mu: (ninst, length, b) float64 (device).
 * use_graph = 1: the whole sequence of step and reduction kernels is
 * captured once into a CUDA graph per (buffers, shape) and replayed.
 * Synchronises the stream at the end. */
int kmsd_batch_moments(kmsd_batch bt, const void *b_in, double *mu, int64_t b,
                       int64_t length, const double *center, const double *half,
                       int flags, int use_graph, void *stream);

/* Sets the row-tile size of the batch step kernels (as chosen by
 * kmsd_batch_tune).  No counterpart in the reference. */
int kmsd_batch_set_tile_rows(kmsd_batch bt, int64_t tile_rows);

/* Autotuner: times the tile sizes 512..8192 rows on this call's shape and
 * keeps the fastest (written to *chosen_tile_rows). */
int kmsd_batch_tune(kmsd_batch bt, const void *b_in, double *mu, int64_t b,
                    int64_t length, const double *center, const double *half,
                    int flags, int64_t *chosen_tile_rows, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* KMSD_H */
