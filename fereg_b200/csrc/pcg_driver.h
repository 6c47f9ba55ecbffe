// The PCG of cg.rs:132-292 for an absorber other than the intercept-only one: the same device
// loop (fused vector kernels, the stopping rule on the device, iteration bodies replayed as
// captured CUDA graphs under a WHILE node) around an operator the caller supplies.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "common.h"

namespace fereg {

// q = S p and z = M^-1 r on m x R row-major FP64 blocks in device memory (R a multiple of 4;
// columns past the caller's are zero). key() appends every device address the two launch
// sequences read or write: a captured iteration is replayed only while the key is unchanged.
struct DevOperator {
    virtual ~DevOperator() = default;
    virtual u32 m() const = 0;
    virtual void apply(double* p, int R, double* q, cudaStream_t st) = 0;
    virtual void precond(double* r, double* z, int R, cudaStream_t st) = 0;
    virtual void key(std::vector<u64>& k) const = 0;
};

struct Scratch;

class PcgDriver {
   public:
    PcgDriver();
    ~PcgDriver();
    PcgDriver(const PcgDriver&) = delete;
    PcgDriver& operator=(const PcgDriver&) = delete;

    // PCG on op x = b (m x R, device memory), from x when x_is_start, else from 0, under the
    // reference's stopping rule per column (ss0 > 0: the column is solved; ss1: the FP64
    // quantity of the rule, cg.rs:132-170); tol and maxiter as cg::pcg (a column still active
    // after maxiter iterations throws RC_CONVERGENCE). Returns the iterations run.
    u64 run(DevOperator& op, double* x, const double* b, int R, const std::vector<double>& ss0,
            const std::vector<double>& ss1, double tol, size_t maxiter, bool x_is_start, const Ctx& ctx,
            cudaStream_t st);
    // Column sums of `nparts` rows of `ncols` partials (fixed order) into out (device memory).
    void col_sums(const double* part, int nparts, int ncols, double* out, cudaStream_t st);

    u64 launches() const;
    // graph captures, graph launches, host microseconds of the captures, 0
    void stats(u64* out4) const;

   private:
    std::unique_ptr<Scratch> d_;
};

}  // namespace fereg
