// GpuAbsorber: the B200 implementation of the reference's `Absorber` trait
// (crates/fereg-core/src/absorber.rs:62-97) over the cell structure of `FeSolver`
// (crates/fereg-core/src/solve.rs:351-1344).
#pragma once

#include <cuda_runtime.h>

#include <memory>

#include "common.h"
#include "device.cuh"

namespace fereg {

struct Ctx {
    int (*interrupt)(void*) = nullptr;
    void* interrupt_data = nullptr;
    void (*log)(void*, const char*) = nullptr;
    void* log_data = nullptr;
    int verbose = 0;
    // Scheduling level of the absorber's stream: 0 the device's highest stream priority, each step
    // one lower (clamped above the lowest, which side passes take); -1 a stream of the default
    // priority. The serving engine gives small requests the high levels, so that their short
    // kernels are not queued behind the large requests' passes.
    int priority_level = -1;
    // The S·P grid autotuner may time the passes (off in the serving engine: concurrent requests
    // make the timings meaningless, and every grid gives the same bits).
    bool autotune = true;
    void check() const {
        if (interrupt && interrupt(interrupt_data)) throw Error(RC_INTERRUPTED, "--Break--");
    }
    void logf(const std::string& s) const {
        if (log && verbose >= 2) log(log_data, s.c_str());
    }
};

// absorber.rs:27-37 SolveInfo (coefficients returned through a caller buffer).
struct SolveInfo {
    u64 iterations = 0;
    bool escalated = false;
    bool exact = false;
};

// Precision of the inner PCG: FP64 throughout, or FP32 iterations inside FP64 refinement.
enum class Precision : int { F64 = 0, F32_REFINED = 1 };

struct Scratch;

// The device absorber behind a session and the C ABI (the reference's `Absorber` trait,
// absorber.rs:62-97): the intercept-only solver (GpuAbsorber, solve.rs FeSolver) or the
// heterogeneous-slope solver (GpuSlopeSolver, slopes.rs SlopeSolver), chosen as solve.rs:338
// `build` chooses. Rows are in the absorber's row order; coefficient blocks are
// coefs_len() x R row-major.
class DeviceAbsorber {
   public:
    virtual ~DeviceAbsorber() = default;
    virtual size_t n() const = 0;
    virtual size_t coefs_len() const = 0;
    // Values term_values writes: sum over terms of levels x (intercept + slopes).
    virtual size_t term_values_len() const = 0;
    virtual const std::vector<u32>& row_order() const = 0;
    virtual bool weights(double* out) const = 0;
    virtual void set_weights(const double* w_rows) = 0;
    virtual void set_weights_device(const double* w_rows_dev) = 0;
    virtual SolveInfo residualize(double* z, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                                  double* coefs, Precision prec = Precision::F64) = 0;
    virtual SolveInfo residualize_device(double* z_dev, size_t r, double tol, size_t maxiter, bool want_coefs,
                                         const double* warm, double* coefs, Precision prec = Precision::F64) = 0;
    virtual SolveInfo residualize_device_warm_last(double* z_dev, size_t r, double tol, size_t maxiter,
                                                   Precision prec = Precision::F64) = 0;
    virtual void fit_rows(const double* coefs, size_t r, size_t col, double* out) const = 0;
    virtual void term_values(const double* coefs, size_t r, size_t col, double* out) const = 0;
    virtual cudaStream_t stream() const = 0;
    virtual void set_profiling(bool on) = 0;
    virtual void phase_times(double* ms, u64* counts) const = 0;
    virtual u64 launches() const = 0;
    virtual void solver_stats(u64* out4) const = 0;
    virtual const Ctx& ctx() const = 0;
    virtual void set_ctx(const Ctx& c) = 0;
    virtual size_t escalated_blocks() const { return 0; }
    virtual u64 escalations() const { return 0; }
    // Exact leverage of the FE columns per row (leverage.rs:128 fe_hat), row order, into device
    // memory (n values).
    virtual void fe_leverage_device(double* h_dev) = 0;
    // The next residualize call makes its stream wait for `ev` (recorded on another stream) before
    // it writes the rows, so that work still reading the raw rows runs beside the solve.
    void set_write_fence(cudaEvent_t ev) { write_fence_ = ev; }

   protected:
    void wait_write_fence(cudaStream_t st) {
        if (write_fence_) CK(cudaStreamWaitEvent(st, write_fence_, 0));
        write_fence_ = nullptr;
    }
    cudaEvent_t write_fence_ = nullptr;
};

class GpuAbsorber : public DeviceAbsorber {
   public:
    // `codes[q]` are the kept-order codes of term q (< g[q]); `w` kept-order weights or null.
    // The cell structure is built on the device; `dev_codes`, when given, are device copies of
    // `codes` (the caller's session keeps them), otherwise the codes are uploaded for the build.
    GpuAbsorber(const std::vector<const u32*>& codes, const std::vector<u32>& g, const double* w, size_t n, const Ctx& ctx,
                const std::vector<const u32*>* dev_codes = nullptr);
    ~GpuAbsorber() override;

    size_t n() const override { return hs_.n; }
    size_t m() const { return hs_.m; }
    size_t g1() const { return hs_.g1; }
    size_t coefs_len() const override { return hs_.m + hs_.g1; }
    size_t term_values_len() const override;
    const std::vector<u32>& row_order() const override { return hs_.pi; }
    const HostStructure& structure() const { return hs_; }
    // Row-order weights (false: all ones).
    bool weights(double* out) const override;
    // Row-order weights (null = ones), strictly positive and finite (solve.rs:1010-1139).
    void set_weights(const double* w_rows) override;
    // The same for row-order weights in device memory; the weight state is computed on the
    // device (the host mirrors follow when a host-side reader needs them).
    void set_weights_device(const double* w_rows_dev) override;

    // Residualizes the N x R row-major block `z` in place (rows in row order). `z` is host
    // memory for `residualize`, device memory for `residualize_device`. `warm` and `coefs` are
    // (m + g1) x R row-major host buffers ([x; alpha1], solve.rs:7-9) or null.
    SolveInfo residualize(double* z, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                          double* coefs, Precision prec = Precision::F64) override;
    SolveInfo residualize_device(double* z_dev, size_t r, double tol, size_t maxiter, bool want_coefs,
                                 const double* warm, double* coefs, Precision prec = Precision::F64) override;
    // The same, warm-started from the reduced solution the previous solve left on the device
    // (the IRLS warm start without the host round trip); the previous solve must have had the
    // same column count.
    SolveInfo residualize_device_warm_last(double* z_dev, size_t r, double tol, size_t maxiter,
                                           Precision prec = Precision::F64) override;

    // FE fit of coefficient column `col` per row (row order) (absorber.rs:88).
    void fit_rows(const double* coefs, size_t r, size_t col, double* out) const override;
    // Values per session term, normalized as solve.rs:1319-1343; `out` holds sum_q g_q values.
    void term_values(const double* coefs, size_t r, size_t col, double* out) const override;

    cudaStream_t stream() const override { return stream_; }

    // Phase timing with CUDA events on the solver's stream (the reference's PhaseTimer,
    // timing.rs): per-slot milliseconds and launch counts, accumulated while enabled.
    // P_APPLY is the segment pass of S*P, P_APPLY_PULL its coordinate-list pass.
    enum Slot {
        P_RHS_SEG = 0,
        P_RHS_PULL,
        P_APPLY,
        P_PRECOND,
        P_VECTOR,
        P_RESID,
        P_H2D,
        P_D2H,
        P_APPLY_PULL,
        P_ESCALATE,
        P_NSLOTS
    };
    void set_profiling(bool on) override;
    void phase_times(double* ms, u64* counts) const override;
    u64 launches() const override;
    // [graphs captured, graph launches, host us of the captures, FP32-refined solves finished in FP64]
    void solver_stats(u64* out4) const override;
    // Large blocks currently preconditioned by a multigrid V-cycle, and the escalations so far.
    size_t escalated_blocks() const override;
    u64 escalations() const override;
    void set_ctx(const Ctx& c) override { ctx_ = c; }
    const Ctx& ctx() const override { return ctx_; }

    // Kernel-level entry points for the parity tests (device work, host buffers).
    void apply_host(const double* p, size_t r, double* y);
    void rhs_host(const double* rows, size_t r, double* y, double* b1, double* wsq, double* wsum);
    void precond_host(const double* rr, size_t r, double* z);
    // The right-hand side pass on caller device buffers with caller-provided scratch: queues the
    // pass on the solver's stream and allocates nothing. rows: n x r; rhs: m x r; b1: g1 x r;
    // colsum: 3 x r ([sum w v^2; sum w v; sum b1^2 / n1]). scratch holds `cap` doubles (256-byte
    // aligned); a call that needs more is rejected (198).
    void rhs_device_scratch(const double* rows, size_t r, double* rhs, double* b1, double* colsum, double* scratch,
                            size_t cap);
    // The reduced system must be held by the dense small factor (at most 1024 coordinates, or
    // none); larger systems are rejected (198) rather than approximated.
    void fe_leverage_device(double* h_dev) override;
    // Weight state (n1, nr, diag, redundant) as held for the kernels.
    void weight_state(double* n1, double* nr, double* diag, uint8_t* red, double* sw) const;

   private:
    // the host copy: scalars, row order, seg_off, cell_row; coord fetched on demand (ensure_host_coord)
    mutable HostStructure hs_;
    std::vector<u32> g_;
    int norm_fe1_ = -1;
    Ctx ctx_;
    cudaStream_t stream_ = nullptr;
    // host weight state (operator.rs:44-63); after set_weights_device these mirrors are copied
    // back from the device on first use (host_stale_)
    mutable std::vector<double> w_rows_, cell_w_, n1_, nr_, diag_;
    mutable std::vector<uint8_t> red_;
    mutable bool host_stale_ = false;
    mutable bool coord_stale_ = false;  // nr / diag / Jacobi on the device are of earlier weights
    double sw_ = 0;
    bool weighted_ = false;
    bool pre_fresh_ = false;
    bool small_ok_ = false;  // the dense small factor exists
    bool amg_wanted_ = false;  // blocks were escalated (their hierarchies are kept across weights)
    bool amg_stale_ = false;   // the hierarchies were built for earlier weights
    std::unique_ptr<Scratch> d_;

    // Escalation (cg.rs:24-37 probe, solve.rs:838 escalate_block): multigrid hierarchies of the
    // large blocks; true when a stronger preconditioner now exists.
    bool escalate(double rho_hat);
    void build_amg();
    void refresh_small();
    void refresh_coord() const;
    void build_small_device();

    void unit_weights_device();
    void build_srow();
    void sync_host_weights() const;
    void ensure_host_coord() const;
    void ensure_precond();
    SolveInfo solve(double* z_dev, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                    double* coefs, Precision prec, bool warm_last = false);
    size_t last_r_ = 0;        // column count of the solution left in the solve scratch
    bool small_stale_ = false;  // the dense small factor was built for earlier weights
};

}  // namespace fereg
