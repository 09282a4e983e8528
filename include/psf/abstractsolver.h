// Headless re-declaration of the reference's solver plug-in interface.
//
// Same class name, virtual methods, setters and getters as
// Solver/abstractsolver.h:13-127.  Differences, all forced by the build
// environment or the scope:
//   - Eigen is not available, so the getters return the small dense types of
//     psf/dense.h (column-major MatrixXd, VectorXd, VectorXf) instead of
//     Eigen::MatrixXd / VectorXd / VectorXf.
//   - There is no GL/Qt: setMesh takes a precomputed domain basis (the
//     output of voxelisation + buildLaplace + buildAdvection, written by the
//     Python precompute as a .psfb file) instead of a Model*, and the draw
//     calls take opaque handles and do nothing in the headless build.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "psf/basis_file.h"
#include "psf/dense.h"

class ShaderProgram;  // graphics types of the reference; unused headless
namespace glm {
struct mat4;
}

// Graphics/Particle/Particle.h:14 -- glm::vec4(pos.xyz, lifetime), 16 bytes.
struct Particle {
    float x, y, z, w;
};

class AbstractSolver {
public:
    AbstractSolver();
    virtual ~AbstractSolver();

    virtual void integrate() = 0;
    void setMesh(const std::string &basis_path);
    void setMesh(const psf::BasisFile &basis);

    void setInitialVelocityField(const psf::VectorXf &field);
    void setInitialVorticityField(const psf::VectorXf &field);
    // Headless additions: set the coefficient state or the particle set directly.
    void setBasisCoefficients(const std::vector<double> &w);
    void setParticles(const std::vector<Particle> &p);

    void setNumberEigenFunctions(unsigned int n);
    void changeNumParticles(unsigned int n);
    void setViscosity(double visc);
    void setTimestep(double timestep);
    void setGravityActive(bool state);
    void setLifeTime(float lt);
    void startBenchmark(bool benchmark);

    unsigned int getNumEigenFunctions();
    double getTimestep();
    const psf::VectorXd &getEigenFunction(unsigned int n);
    const psf::MatrixXd &getVelocityBasisField();
    const psf::VectorXd &getBasisCoefficients();
    const psf::VectorXf &getVelocityField();

    const std::vector<Particle> &getParticles();
    void clearParticles();
    void addParticle(Particle particle);
    unsigned int getNumParticles();

    virtual void drawParticles(ShaderProgram *program, const glm::mat4 &pvm) = 0;

    // Benchmark sums (t_advect_ms, t_particles_ms) as in abstractsolver.cpp:252-302.
    const std::vector<double> &getBenchmarkSums() const { return benchmarkSums; }

    bool gpu = false;

protected:
    unsigned int maxFramesBenchmark = 1000;
    bool isBenchmark = false;
    unsigned int benchmarkFrameNo = 0;
    std::vector<double> benchmarkSums;

    unsigned int maxParticles = 1000;
    unsigned int particlePointer = 0;
    double simTime = 0.0;

    virtual void buildLaplace() = 0;
    virtual void buildAdvection() = 0;
    // Called after the coefficient state or the particles were changed on the host.
    virtual void stateChanged() {}
    virtual void particlesChanged() {}
    // Called after dt, viscosity, gravity or lifetime changed.
    virtual void paramsChanged() {}

    float lifeTime = 60.0f;
    unsigned int nEigenFunctions = 16;
    double timeStep = 1.0 / 60.0;
    double viscosity = 0.0;
    bool gravityActive = false;

    psf::BasisFile basis;  // full precomputed basis of the current domain

    std::vector<psf::VectorXd> eigenFunctions;
    psf::VectorXf velocityField;
    psf::VectorXd gravity;
    psf::VectorXd eigenValues;
    psf::VectorXd basisCoeff;
    psf::MatrixXd velBasisField;
    std::vector<Particle> particles;
};
