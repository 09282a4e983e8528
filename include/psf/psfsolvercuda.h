// PSFSolverCUDA: the B200 implementation of the reference's solver plug-in.
//
// Drop-in sibling of PSFSolver (CPU, Solver/SolverImpl/psfsolver.h:8-19) and
// PSFSolverGPU (OpenCL, Solver/SolverImpl/psfsolvergpu.h:10-88): the same
// AbstractSolver overrides (integrate, buildLaplace, buildAdvection,
// drawParticles), with the per-step work done by the CUDA engine behind the
// C ABI of psf_b200.h.  Host mirrors (basisCoeff, velocityField, particles)
// are refreshed lazily when a getter asks for them.
#pragma once

#include <stdexcept>
#include <string>

#include "psf/abstractsolver.h"
#include "psf_b200.h"

class PSFSolverCUDA : public AbstractSolver {
public:
    explicit PSFSolverCUDA(int device = 0);
    ~PSFSolverCUDA() override;

    void integrate() override;
    void drawParticles(ShaderProgram *program, const glm::mat4 &pvm) override;

    // Particle integrator (PSF_RK1 as the reference, or PSF_RK4).
    void setIntegrator(int integrator);
    // Decay exp(-nu lam dt) as the OpenCL kernel instead of exp(+nu lam dt).
    void setDecayNegative(bool neg);
    // Replace the forcing vector (defaults to the projected gravity).
    void setForcing(const psf::VectorXd &f);
    void setRespawnSeed(uint64_t seed);
    // Run `n` steps without refreshing host mirrors in between.
    void integrateSteps(int n);
    psf_ctx *context() { return ctx; }

protected:
    void buildLaplace() override;
    void buildAdvection() override;
    void stateChanged() override;
    void particlesChanged() override;
    void paramsChanged() override { pushParams(); }

private:
    void check(int rc, const char *what);
    psf_params params() const;
    void pushParams();
    void pullState();

    int device;
    int integrator = PSF_RK1;
    bool decayNegative = false;
    uint64_t seed = 0;
    psf_ctx *ctx = nullptr;
    psf::BasisFile active;  // basis truncated to nEigenFunctions
    psf::VectorXd forcing;
    bool hostStale = false;
};
