// aem_design.h -- gradient of a probe figure of merit with respect to the
// permittivity and conductivity of every cell of a design box.
//
// The reference's optimisation workflow
// (optimization_scripts/adjoint_optimization/adjoint_optimization.py)
// runs the solver twice per iteration, a forward run and an "adjoint" run
// with a rescaled, delayed source, and forms the gradient from the overlap
// of the two runs' field spectra (:121-134).  Here the gradient is the exact
// derivative of the discrete time loop instead: a forward run of the
// reference's update (bulk Yee, CPML, lumped ports: fdtd_solver.f90
// :4442-5375, :5667-6670) with per-cell eps_r / sigma inside the design box,
// then the transposed update run backwards in time from the last step.  The
// forward state is kept at checkpoints every K steps; each K-step segment is
// recomputed from its checkpoint while the adjoint sweeps it, so device
// memory holds one segment of design-box field history, not the whole run.
//
// Figure of merit: F = |D|^2, D = sum_n c^n exp(-i 2 pi f n dt), c^n the
// probe E component after step n.
#pragma once
#include <memory>
#include <string>
#include <vector>

namespace aem {

class DesignRun {
   public:
    // `inputs_path` names a deck of the standard solver without periodic
    // axes, plane-wave source, sheets, Drude poles or gridded ports (a lumped
    // port drives it); the design box is the cells lo..lo+n-1 (reference
    // indices) and must keep its edges out of the CPML slabs and off the
    // ports.  precision 4: FP32 state (the reference's arithmetic); 8: FP64.
    static DesignRun* create(const std::string& inputs_path, const std::string& outdir, const int lo[3],
                             const int n[3], int precision);
    virtual ~DesignRun() {}
    // probe: E component `comp` (0..2) at reference edge (i, j, k), frequency
    virtual void set_probe(int comp, int i, int j, int k, double freq_hz) = 0;
    // design values, n0*n1*n2 float32 each, x fastest; host or device
    // pointers; sig null keeps the deck's conductivity
    virtual void set_design(const float* eps, const float* sig) = 0;
    // Forward run of the deck's full step count.  checkpoint_every < 1: no
    // state kept (a plain forward run); otherwise checkpoints every that many
    // steps, ready for gradient().  Returns F; dft (may be null) gets D.
    virtual double forward(int checkpoint_every, double dft[2]) = 0;
    // dF/d eps_r and dF/d sigma per design cell (n0*n1*n2 float32 each, x
    // fastest; host or device pointers, either may be null), scaled by
    // `scale`; needs a forward() with checkpoints since the last set_design
    virtual void gradient(float* geps, float* gsig, double scale) = 0;
    // Overlap check: with it on, gradient() also accumulates the DFTs at the
    // probe frequency of the forward E and of the adjoint field on every
    // design edge; gradient_overlap() then returns dF/d eps_r and dF/d sigma
    // estimated from those two spectra alone (the frequency-domain overlap
    // of adjoint_optimization.py:121-134, which assumes the adjoint field is
    // a tone at that frequency), in gradient()'s layout and scale
    virtual void set_overlap(bool on) = 0;
    virtual void gradient_overlap(float* geps, float* gsig, double scale) = 0;
    // device time (ms) of the last forward() and gradient() calls, and the
    // kernel launches of each
    virtual void timing(double ms[2], long long launches[2]) const = 0;
    // current field component comp (0..5 = Ex..Hz) in the reference layout
    // (as Solver::get_field); dims gets its extents
    virtual void get_field(int comp, std::vector<double>& out, int dims[3]) = 0;
    virtual void* stream() const = 0;
    virtual size_t device_bytes() const = 0;
};

}  // namespace aem
