// GpuSlopeSolver: the absorber of terms with heterogeneous slopes (`fe#c.x`, `fe##c.x`, terms
// without an intercept), the B200 form of the reference's SlopeSolver
// (crates/fereg-core/src/slopes.rs:2183-2475) behind the same Absorber contract.
//
// Structure (slopes.rs:354-501): rows sorted stably by the eliminated term E (FE1 when an
// intercept-only term exists, else the term with the most levels); every row owns k design
// slots, one per (block, intercept or slope), each a reduced coordinate and a value. Level l of a
// block of width b owns the b consecutive coordinates off + l b ... The blocks are ordered small
// first by the reference's cost model, so the coefficient layout [x (m x R); alpha_E (G_E b_E x
// R)] is the reference's.
//
// Device passes per PCG iteration, every sum in a fixed order:
//   segment pass: per (level s of E, column j) one thread loads u_i = sum_slots v P[c] over the
//     segment's rows, forms t = M_s^+ sum_i w_i h_E,i u_i and writes z_i = w_i (u_i - h_E,i' t);
//   coordinate pass: per (coordinate, column) Y = sum over the coordinate's rows of v z_i, from a
//     coordinate-sorted list of (row, slot value) built once;
//   preconditioner: per-level b x b block-Jacobi inverses of every block (the reference factors
//     the small blocks densely and escalates large ones to a sparse Cholesky; both change the
//     iterations to the same tolerance, not the solution).
// The PCG is the device loop of PcgDriver (cg.rs:132-292).
#pragma once

#include <memory>
#include <vector>

#include "absorber.h"
#include "common.h"

namespace fereg {

// One absorb term (session.rs:20-42 Term): kept-order codes below g, intercept flag and slope
// variables (kept order, n values each).
struct SlopeTermIn {
    const u32* codes = nullptr;
    u32 g = 0;
    bool intercept = true;
    std::vector<const double*> slopes;
};

// slopes.rs:163-182 SBlock.
struct SlopeBlock {
    size_t term = 0;
    u32 g = 0;
    bool icpt = false;
    u32 ns = 0, b = 0, s0 = 0, off = 0;
    bool small = false;
};

// slopes.rs:195-211 SlopeStructure (host side) and the device lists built from it.
struct SlopeHost {
    size_t n = 0;
    std::vector<u32> pi;  // kept observation of each row
    size_t e = 0;
    u32 ge = 0, e_ns = 0, be = 0;
    bool e_icpt = false;
    std::vector<u32> seg_off;  // ge + 1
    u32 k = 0;                 // design slots per row
    std::vector<u32> sc;       // n x k coordinates
    std::vector<double> sv;    // n x k values
    std::vector<double> he;    // n x e_ns slopes of E
    std::vector<SlopeBlock> blocks;
    u32 nsmall = 0, m = 0, m_small = 0;
    // coordinate-sorted (row, value) lists of the slots (m + 1 offsets)
    std::vector<u32> pl_off, pl_row;
    std::vector<double> pl_val;
    // block-Jacobi units: first coordinate, width and offset into the inverses of every level
    std::vector<u32> un_c0, un_b, un_joff;
    u32 jlen = 0;
};

// Builds the structure (slopes.rs:354-501; the small-block cost model of slopes.rs:62-78 and
// 347-352 with small_limit = 4096, structure.rs:23).
SlopeHost build_slope_structure(const std::vector<SlopeTermIn>& terms, size_t n);

// slopes.rs:102-132 sweep_ginv: generalized inverse of the symmetric PSD k x k `a` in place.
void sweep_ginv(double* a, size_t k, const double* refd, double tol);

struct SlopeDevBufs;

class GpuSlopeSolver : public DeviceAbsorber {
   public:
    // terms as the session holds them; w: kept-order weights or null (validated: positive, finite).
    GpuSlopeSolver(const std::vector<SlopeTermIn>& terms, const double* w, size_t n, const Ctx& ctx);
    ~GpuSlopeSolver() override;

    size_t n() const override { return hs_.n; }
    size_t coefs_len() const override { return size_t(hs_.m) + size_t(hs_.ge) * hs_.be; }
    size_t term_values_len() const override;
    const std::vector<u32>& row_order() const override { return hs_.pi; }
    bool weights(double* out) const override;
    void set_weights(const double* w_rows) override;
    void set_weights_device(const double* w_rows_dev) override;
    SolveInfo residualize(double* z, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                          double* coefs, Precision prec = Precision::F64) override;
    SolveInfo residualize_device(double* z_dev, size_t r, double tol, size_t maxiter, bool want_coefs,
                                 const double* warm, double* coefs, Precision prec = Precision::F64) override;
    SolveInfo residualize_device_warm_last(double* z_dev, size_t r, double tol, size_t maxiter,
                                           Precision prec = Precision::F64) override;
    void fit_rows(const double* coefs, size_t r, size_t col, double* out) const override;
    void term_values(const double* coefs, size_t r, size_t col, double* out) const override;
    cudaStream_t stream() const override { return stream_; }
    void set_profiling(bool on) override { prof_ = on; }
    void phase_times(double* ms, u64* counts) const override;
    u64 launches() const override;
    void solver_stats(u64* out4) const override;
    const Ctx& ctx() const override { return ctx_; }
    void set_ctx(const Ctx& c) override { ctx_ = c; }
    void fe_leverage_device(double*) override {
        throw Error(RC_INVALID_INPUT, "fereg: the exact FE leverage (HC2/HC3) of slope terms is not built");
    }

    const SlopeHost& structure() const { return hs_; }
    // The weight state: M_s^+ of every level of E (ge x be^2), the block-Jacobi inverses and
    // the redundant coordinates (m).
    void weight_state(double* minv, double* jinv, uint8_t* red) const;
    // One application of S and of the preconditioner to host m x r blocks (parity tests).
    void apply_host(const double* p, size_t r, double* y);
    void precond_host(const double* rr, size_t r, double* z);
    // The reduced right-hand side of the n x r host block and [sum w v^2; sum w v; sum w e^2].
    void rhs_host(const double* rows, size_t r, double* y, double* stats);

   private:
    SlopeHost hs_;
    std::vector<bool> t_icpt_;
    std::vector<u32> t_ns_, t_g_;
    int fe1_ = -1;
    Ctx ctx_;
    cudaStream_t stream_ = nullptr;
    bool prof_ = false;
    // weight state (slopes.rs:527-697), host copies
    std::vector<double> w_rows_, minv_, jinv_;
    std::vector<uint8_t> red_;
    double sw_ = 0;
    std::unique_ptr<SlopeDevBufs> d_;
    size_t last_r_ = 0;

    void refresh_weights();
    SolveInfo solve(double* z_dev, size_t r, double tol, size_t maxiter, bool want_coefs, const double* warm,
                    double* coefs, bool warm_last);
};

}  // namespace fereg
