// Headless driver for PSFSolverCUDA (the role of the reference's GUI timer
// loop, Widgets/glcanvas.cpp:143-156): load a basis, set the state and the
// particles, integrate, write the results.
//
//   psf_run <basis.psfb> <n_modes> <steps> <dt> <integrator 1|4> <w0.f64> <particles.f32> <out_prefix>
//
// Inputs are raw little-endian arrays; writes <out_prefix>.w.f64 and
// <out_prefix>.p.f32.  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "psf/psfsolvercuda.h"

template <class T>
static std::vector<T> read_raw(const std::string &path)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<T> v((size_t)n / sizeof(T));
    if (std::fread(v.data(), sizeof(T), v.size(), f) != v.size()) throw std::runtime_error("short read " + path);
    std::fclose(f);
    return v;
}

template <class T>
static void write_raw(const std::string &path, const T *data, size_t n)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(data, sizeof(T), n, f) != n) throw std::runtime_error("cannot write " + path);
    std::fclose(f);
}

int main(int argc, char **argv)
{
    if (argc != 9) {
        std::fprintf(stderr, "usage: %s basis.psfb n_modes steps dt integrator w0.f64 particles.f32 out_prefix\n",
                     argv[0]);
        return 2;
    }
    try {
        PSFSolverCUDA solver(0);
        solver.setNumberEigenFunctions((unsigned)std::atoi(argv[2]));
        auto parts = read_raw<float>(argv[7]);
        solver.changeNumParticles((unsigned)(parts.size() / 4));
        solver.setTimestep(std::atof(argv[4]));
        solver.setIntegrator(std::atoi(argv[5]));
        solver.setMesh(std::string(argv[1]));
        auto w0 = read_raw<double>(argv[6]);
        solver.setBasisCoefficients(w0);
        std::vector<Particle> ps(parts.size() / 4);
        for (size_t i = 0; i < ps.size(); ++i) ps[i] = {parts[4 * i], parts[4 * i + 1], parts[4 * i + 2], parts[4 * i + 3]};
        solver.setParticles(ps);
        solver.integrateSteps(std::atoi(argv[3]));
        const auto &w = solver.getBasisCoefficients();
        const auto &p = solver.getParticles();
        std::string out = argv[8];
        write_raw(out + ".w.f64", w.data(), w.size());
        write_raw(out + ".p.f32", reinterpret_cast<const float *>(p.data()), p.size() * 4);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "psf_run: %s\n", e.what());
        return 1;
    }
    return 0;
}
