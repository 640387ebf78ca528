// Host-side objects of libkmsd_b200.so shared by the metric and engine
// translation units.  Not part of the public ABI (include/kmsd.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "kmsd.h"
#include "kmsd_common.cuh"

namespace kmsd {

constexpr int kThreads = 256;

// Last-error state (thread local) and status helpers.
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
#define KMSD_CUDA(call)                                      \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
    } while (0)

// Grow-only device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t want);
    void release();
    template <class X> X *as() const { return static_cast<X *>(p); }
};

int sm_count();
// Process-wide count of kernels launched by the library.
void count_launch(int64_t n = 1);
// While a CountOff lives, this thread's launches are tallied instead of
// counted: launches recorded into a graph during capture are counted each
// time the graph runs (recorded() of them per launch).
struct CountOff {
    CountOff();
    ~CountOff();
    int64_t recorded() const;
    int64_t start;
};
// Kernels launched by device-driven loops on the current device (read from
// the device; synchronises it).
int64_t device_loop_launches();
// Grid for a row-group kernel over `rows` rows.
int grid_for(int64_t rows, const RowMap &mp);
// Grid of one resident wave of `kernel` (occupancy API; cached per kernel and
// shared-memory size), capped by the row groups needed.
int wave_grid(const void *kernel, size_t smem, int64_t rows, const RowMap &mp);
// Units per lane: 1 or 2 (row groups are up to 128 lanes, rows up to 256
// units); 0 when too wide.
int mu_for(const RowMap &mp);
size_t reduce_smem(const RowMap &mp, int C);

}  // namespace kmsd

// ------------------------------------------------------------------ CSR
struct kmsd_csr_s {
    int64_t n = 0, nnz = 0;
    int *ptr = nullptr, *idx = nullptr;
    double *re64 = nullptr, *im64 = nullptr;
    float *re32 = nullptr, *im32 = nullptr;  // created on first mixed use
    bool complex_values = false;
    bool identity = false;
    // one real entry per row, on the diagonal (a position operator given by
    // site coordinates): re64 then holds the coordinates in row order
    bool diagonal = false;
    int device = 0;
    // ELL copy for short rows (see EllView); ell_w == 0 when not built.
    int ell_w = 0;
    int *ell_idx = nullptr;
    double *ell_re64 = nullptr, *ell_im64 = nullptr;
    float *ell_re32 = nullptr, *ell_im32 = nullptr;
    // 4x4 block-CSR copy (see BsrView); bsr_nb == 0 when not built.
    int64_t bsr_nb = 0;
    int *bsr_ptr = nullptr, *bsr_idx = nullptr;
    double *bsr_re = nullptr, *bsr_im = nullptr;
    int ensure_f32();
    kmsd::CsrView<double> view64() const { return {ptr, idx, re64, complex_values ? im64 : nullptr}; }
    kmsd::CsrView<float> view32() const { return {ptr, idx, re32, complex_values ? im32 : nullptr}; }
    kmsd::EllView<double> ell64() const { return {ell_idx, ell_re64, complex_values ? ell_im64 : nullptr, ell_w}; }
    kmsd::EllView<float> ell32() const { return {ell_idx, ell_re32, complex_values ? ell_im32 : nullptr, ell_w}; }
    kmsd::BsrView<double> bsr64() const {
        return {bsr_ptr, bsr_idx, bsr_re, complex_values ? bsr_im : nullptr, bsr_nb};
    }
};

namespace kmsd {
// Y = A X over complex128 (n, b); optional curvature dot into dot_out (double2[b]).
int spmm64(const kmsd_csr_s *A, const double2 *X, double2 *Y, int64_t b, cudaStream_t s,
           double2 *dot_out = nullptr);
int spmm32(const kmsd_csr_s *A, const float4 *X, float4 *Y, int64_t U, cudaStream_t s,
           double2 *dot_out = nullptr);
// out[j] = sum_i conj(x_ij) y_ij into device double2[ncol] (deterministic).
int coldot64(const double2 *x, const double2 *y, int64_t n, int64_t b, double2 *out, cudaStream_t s);
int coldot32(const float4 *x, const float4 *y, int64_t n, int64_t U, double2 *out, cudaStream_t s);
int take_real(const double2 *src, double *dst, int64_t b, cudaStream_t s);
// y = sum coef_m x_m  (or y += ...).
int lincomb(cudaStream_t s, double2 *y, int64_t len, int accumulate, int terms, const double2 *const *x,
            const double *cr, const double *ci);
// Correlation tables of ring slots [j0, j0 + jn) against cov (kmsd_corr.cu).
int corr_ring(const double2 *ring, int64_t n, int nb, const double2 *cov, int k1, int64_t j0, int jn,
              int64_t length, double2 *tables, DevBuf &partial, cudaStream_t s);
int ring_slots();
// Shared scratch for reductions (partials + tickets), grown per call site.
struct Reducer {
    DevBuf partial;
    DevBuf ticket;
    int ensure(int grid, int ncol, int copies = 1);
    double2 *part() const { return partial.as<double2>(); }
    Ticket *tick() const { return ticket.as<Ticket>(); }
};
}  // namespace kmsd

// ------------------------------------------------------------------ metric
struct PcgCols;
struct kmsd_metric_s {
    kmsd_csr_s *S = nullptr;
    int64_t n = 0;
    double *diag = nullptr;   // device
    double *zinv = nullptr;   // 1/sqrt(diag), device (sampling)
    int64_t nblocks = 0;      // 0: diagonal preconditioner
    int *bstart = nullptr;    // device, nblocks+1
    int64_t *foff = nullptr;  // device
    double2 *factors = nullptr;  // Cholesky factors, or the block inverses (kernels with small blocks)
    int inv_real = 0;            // factors hold real block inverses
    int maxb = 1;
    int ub = 0;               // uniform block size (block i = rows [i*ub, (i+1)*ub)), else 0
    int store32 = 0;          // CG work vectors stored as complex64 (the mixed form)
    bool identity = false;
    int adaptive = 0, interval = 32;
    double gap_ratio = .1;
    // workspace
    int64_t wb = 0;  // columns the workspace is sized for
    kmsd::DevBuf q, y, r, z, p, sp, t;
    kmsd::DevBuf cols;       // per-column state (PcgCols layout)
    kmsd::DevBuf host_pinned;  // pinned host flags
    kmsd::Reducer red;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // counters (host side, plus device counters folded in on read)
    int64_t calls = 0;
    double seconds = 0.;
    kmsd::DevBuf dcount;  // device counters: refreshes, checks, restarts, iters_sum, max_rel(bits)
    // Segments: S is block-diagonal over the row ranges [seg_row0[s],
    // seg_row0[s+1]), each an independent system with its own CG per column
    // (nseg <= 1: one system).  Device descriptors per row-group width.
    struct SegPlan {
        kmsd::DevBuf mem;
        int grid = 0, l2rows = 0;
        int *cta_seg = nullptr, *cta0 = nullptr, *tk0 = nullptr, *l2 = nullptr, *segn = nullptr,
            *segchk = nullptr;
        int64_t *row0 = nullptr, *blk0 = nullptr;
        kmsd::Ticket *tickets = nullptr;
    };
    int64_t nseg = 0;
    std::vector<int64_t> seg_row0, seg_blk0;
    std::vector<int64_t> bstart_host;  // block-Jacobi partition (host copy)
    bool seg_aligned4 = false;  // every segment starts on a multiple of 4 rows
    std::map<int, SegPlan> seg_plans;
    int seg_plan(int gpc, SegPlan **out);
    // Whole solves captured as graphs with a device-driven iteration loop,
    // per argument set; valid while the workspace pointers in graph_ws hold.
    cudaStream_t loop_stream = nullptr, check_stream = nullptr, cap_stream = nullptr;
    std::map<std::vector<uint64_t>, std::pair<cudaGraphExec_t, int64_t>> graphs;  // exec, kernels recorded
    std::vector<const void *> graph_ws;
    // The same solve as `solve` (asynchronous form), with the iterations
    // driven by the device: one graph launch per call, no host polling.
    // When `s` is capturing, the solve is recorded into that capture.
    int solve_dev(const double2 *B, double2 *Y, int64_t b, double rtol, double atol, int maxiter, cudaStream_t s,
                  int *status, void *fail_report);
    // Allocates everything a device-driven solve of b columns needs, so that
    // a later capture allocates nothing.
    int prepare_dev(int64_t b);
    // state_cols: per-column state entries (nseg * b for a segmented solve)
    int ensure(int64_t b, int64_t state_cols = 0);
    // Batched PCG on device buffers (complex128).  When `report` is null and
    // `status` non-null, the call is asynchronous: a failure is recorded in
    // *status (first failure wins) together with the per-column report in
    // `fail_report`.
    int solve(const double2 *B, double2 *Y, int64_t b, double rtol, double atol, int maxiter,
              kmsd_solve_report *report, cudaStream_t s, int *status = nullptr, void *fail_report = nullptr);
};

struct FailReportFull;

// Per-column device failure report for asynchronous solves.
struct FailReport {
    int64_t ncols;
    int code;  // KMSD_EMETRIC / KMSD_EINVAL
    int reason;  // 0 acceptance, 1 breakdown, 2 not representable, 3 nonfinite RHS
};
constexpr int kMaxReportCols = 512;
struct FailReportFull {
    FailReport head;
    uint8_t converged[kMaxReportCols];
    uint8_t breakdown[kMaxReportCols];
    int64_t iterations[kMaxReportCols];
    double true_residual[kMaxReportCols];
    double relative_residual[kMaxReportCols];
};

// ------------------------------------------------------------------ engine
struct kmsd_engine_s {
    kmsd_csr_s *H = nullptr;
    kmsd_metric_s *M = nullptr;
    int vel_kind[3] = {-1, -1, -1};
    kmsd_csr_s *vel[9] = {};
    double rtol = 1e-10, atol = 0., hbar = 0.6582119569509067;
    int maxiter = 1000;
    int precision = KMSD_FP64;
    int64_t h_calls = 0, v_calls = 0;
    bool identity = false;
    kmsd::DevBuf ta, tb, bra, hx, t1, t2, t3, t4, t5, psi, vc, inj[3], outw;
    kmsd::DevBuf ring, corr_partial;  // left-chain ring and partial sums of the correlation tables
    // per axis, the inline velocity's values aligned with H's ELL columns
    // (complex, FP64 and FP32 copies); built on first use, -1: cannot align
    kmsd::DevBuf vell64[3], vell32[3];
    int vell_state[3] = {0, 0, 0};
    kmsd::DevBuf status;  // int[4]: [0] code, [1] report claim, [2] series nonfinite
    kmsd::DevBuf report;  // FailReportFull
    kmsd::DevBuf dots;    // double2[512]
    kmsd::Reducer red;
    FailReportFull last{};
};
