// Headless AbstractSolver (include/psf/abstractsolver.h), restating the
// non-virtual parts of Solver/abstractsolver.cpp.
#include "psf/abstractsolver.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

AbstractSolver::AbstractSolver()
{
    // Defaults of Solver/abstractsolver.cpp:7-46.
    maxFramesBenchmark = 1000;
    maxParticles = 1000;
    gravityActive = false;
    nEigenFunctions = 16;
    viscosity = 0.0;
    timeStep = 1.0 / 60.0;
    lifeTime = 1.0f * 60.0f;
    particles.assign(maxParticles, Particle{0.f, 0.f, 0.f, 0.f});
}

AbstractSolver::~AbstractSolver() = default;

void AbstractSolver::setMesh(const std::string &basis_path)
{
    psf::BasisFile b;
    std::string err = b.load(basis_path);
    if (!err.empty()) throw std::runtime_error(err);
    setMesh(b);
}

void AbstractSolver::setMesh(const psf::BasisFile &b)
{
    // Solver/abstractsolver.cpp:92-166: clear, voxelise, build the basis and tensor.
    clearParticles();
    basis = b;
    nEigenFunctions = std::min<unsigned int>(nEigenFunctions, (unsigned int)b.n_modes);
    buildLaplace();
    buildAdvection();
}

void AbstractSolver::setInitialVelocityField(const psf::VectorXf &field)
{
    // basisCoeff = Phi^T field (Solver/abstractsolver.cpp:168-171).
    const size_t N = velBasisField.cols();
    basisCoeff.resize(N);
    for (size_t i = 0; i < N; ++i) {
        double acc = 0.0;
        for (size_t f = 0; f < velBasisField.rows(); ++f) acc += velBasisField(f, i) * (double)field[f];
        basisCoeff[i] = acc;
    }
    stateChanged();
}

void AbstractSolver::setBasisCoefficients(const std::vector<double> &w)
{
    if (w.size() != nEigenFunctions) throw std::runtime_error("state length must equal the mode count");
    basisCoeff.resize(w.size());
    for (size_t i = 0; i < w.size(); ++i) basisCoeff[i] = w[i];
    stateChanged();
}

void AbstractSolver::setParticles(const std::vector<Particle> &p)
{
    particles = p;
    maxParticles = (unsigned int)p.size();
    particlePointer = 0;
    particlesChanged();
}

void AbstractSolver::setInitialVorticityField(const psf::VectorXf &)
{
    throw std::runtime_error("the basis file holds no vorticity basis; use setInitialVelocityField");
}

void AbstractSolver::setNumberEigenFunctions(unsigned int n)
{
    // Solver/abstractsolver.cpp:173-179.
    clearParticles();
    nEigenFunctions = n;
    if (!basis.empty()) {
        if (n > (unsigned int)basis.n_modes) throw std::runtime_error("more modes than the basis holds");
        buildLaplace();
        buildAdvection();
    }
}

void AbstractSolver::changeNumParticles(unsigned int n)
{
    maxParticles = n;
    clearParticles();
}

void AbstractSolver::setViscosity(double visc)
{
    viscosity = visc;
    paramsChanged();
}

void AbstractSolver::setTimestep(double t)
{
    timeStep = t;
    paramsChanged();
}

void AbstractSolver::setGravityActive(bool state)
{
    gravityActive = state;
    paramsChanged();
}

void AbstractSolver::setLifeTime(float lt)
{
    lifeTime = lt * 60.0f;
    paramsChanged();
}

void AbstractSolver::startBenchmark(bool benchmark)
{
    isBenchmark = benchmark;
    if (benchmark) {
        benchmarkSums.assign(2, 0.0);
        benchmarkFrameNo = 0;
    }
}

unsigned int AbstractSolver::getNumEigenFunctions() { return nEigenFunctions; }
double AbstractSolver::getTimestep() { return timeStep; }
const psf::VectorXd &AbstractSolver::getEigenFunction(unsigned int n) { return eigenFunctions.at(n); }
const psf::MatrixXd &AbstractSolver::getVelocityBasisField() { return velBasisField; }
const psf::VectorXd &AbstractSolver::getBasisCoefficients() { return basisCoeff; }
const psf::VectorXf &AbstractSolver::getVelocityField() { return velocityField; }
const std::vector<Particle> &AbstractSolver::getParticles() { return particles; }
unsigned int AbstractSolver::getNumParticles() { return (unsigned int)particles.size(); }

void AbstractSolver::clearParticles()
{
    // Solver/abstractsolver.cpp:377-385 with ParticleBuffer::reserve: maxParticles
    // zeroed particles, which respawn on their first step.
    simTime = 0.0;
    particlePointer = 0;
    particles.assign(maxParticles, Particle{0.f, 0.f, 0.f, 0.f});
    particlesChanged();
}

void AbstractSolver::addParticle(Particle p)
{
    // Solver/abstractsolver.cpp:387-397 with DECMesh3D::isPointInside
    // (DEC/decmesh3d.cpp:1799-1806, which offsets by one voxel and uses min.x
    // for z).
    if (basis.empty() || particles.empty()) return;
    const double h = basis.h;
    const unsigned yO = (unsigned)((-basis.aabb_min[1] + p.y) / h) + 1;
    const unsigned xO = (unsigned)((-basis.aabb_min[0] + p.x) / h) + 1;
    const unsigned zO = (unsigned)((-basis.aabb_min[0] + p.z) / h) + 1;
    const uint64_t vid = (uint64_t)zO * basis.dims[0] * basis.dims[1] + (uint64_t)yO * basis.dims[0] + xO;
    const bool inside = vid < basis.inside.size() && basis.inside[vid] != 0;
    if (inside && simTime >= particles[particlePointer].w) {
        Particle &q = particles[particlePointer];
        q.x = p.x;
        q.y = p.y;
        q.z = p.z;
        q.w = (float)(simTime + p.w);
        particlePointer = (particlePointer + 1) % maxParticles;
        particlesChanged();
    }
}
