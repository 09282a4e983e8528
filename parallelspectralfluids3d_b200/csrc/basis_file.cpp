// Reader of the .psfb domain-basis file (include/psf/basis_file.h).
#include "psf/basis_file.h"

#include <cstdio>
#include <cstring>

namespace psf {

namespace {

template <class T>
T rd(const std::vector<unsigned char> &buf, size_t off)
{
    T v;
    std::memcpy(&v, buf.data() + off, sizeof(T));
    return v;
}

}  // namespace

std::string BasisFile::load(const std::string &path)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    std::vector<unsigned char> buf;
    unsigned char chunk[1 << 16];
    size_t n;
    while ((n = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf.insert(buf.end(), chunk, chunk + n);
    std::fclose(f);
    if (buf.size() < 148 || std::memcmp(buf.data(), "PSFBASIS", 8) != 0) return path + ": not a basis file";
    if (rd<uint32_t>(buf, 8) != 1) return path + ": unsupported basis file version";
    for (int i = 0; i < 3; ++i) dims[i] = rd<uint32_t>(buf, 12 + 4 * i);
    h = rd<double>(buf, 24);
    for (int i = 0; i < 3; ++i) aabb_min[i] = rd<float>(buf, 32 + 4 * i);
    for (int i = 0; i < 3; ++i) aabb_max[i] = rd<float>(buf, 44 + 4 * i);
    n_modes = rd<int32_t>(buf, 56);
    n_faces = rd<int64_t>(buf, 60);
    const int64_t n_active = rd<int64_t>(buf, 68);
    const int64_t n_voxels = rd<int64_t>(buf, 76);
    const int64_t n_words = rd<int64_t>(buf, 84);
    uint64_t off[7];
    for (int i = 0; i < 7; ++i) off[i] = rd<uint64_t>(buf, 92 + 8 * i);
    const int64_t N = n_modes;
    const uint64_t sizes[7] = {(uint64_t)n_active * 4, (uint64_t)N * 8, (uint64_t)N * 8,
                               (uint64_t)(n_active * N) * 8, (uint64_t)(N * N * N) * 8, (uint64_t)n_words * 4,
                               (uint64_t)n_voxels};
    for (int i = 0; i < 7; ++i)
        if (off[i] + sizes[i] > buf.size()) return path + ": truncated basis file";
    auto grab = [&](auto &vec, int i, size_t count) {
        vec.resize(count);
        std::memcpy(vec.data(), buf.data() + off[i], sizes[i]);
    };
    grab(active_faces, 0, (size_t)n_active);
    grab(lam, 1, (size_t)N);
    grab(gravity, 2, (size_t)N);
    grab(phi, 3, (size_t)(n_active * N));
    grab(C, 4, (size_t)(N * N * N));
    grab(sign_bits, 5, (size_t)n_words);
    grab(inside, 6, (size_t)n_voxels);
    return "";
}

BasisFile BasisFile::truncated(int32_t n) const
{
    BasisFile t;
    std::memcpy(t.dims, dims, sizeof dims);
    t.h = h;
    std::memcpy(t.aabb_min, aabb_min, sizeof aabb_min);
    std::memcpy(t.aabb_max, aabb_max, sizeof aabb_max);
    t.n_modes = n;
    t.n_faces = n_faces;
    t.active_faces = active_faces;
    t.sign_bits = sign_bits;
    t.inside = inside;
    t.lam.assign(lam.begin(), lam.begin() + n);
    t.gravity.assign(gravity.begin(), gravity.begin() + n);
    const size_t Fa = active_faces.size(), N = (size_t)n_modes;
    t.phi.resize(Fa * n);
    for (size_t r = 0; r < Fa; ++r)
        for (int32_t i = 0; i < n; ++i) t.phi[r * n + i] = phi[r * N + i];
    t.C.resize((size_t)n * n * n);
    for (int32_t k = 0; k < n; ++k)
        for (int32_t a = 0; a < n; ++a)
            for (int32_t j = 0; j < n; ++j)
                t.C[((size_t)k * n + a) * n + j] = C[((size_t)k * N + a) * N + j];
    return t;
}

psf_basis_desc BasisFile::desc() const
{
    psf_basis_desc d{};
    for (int i = 0; i < 3; ++i) {
        d.grid.dims[i] = dims[i];
        d.grid.aabb_min[i] = aabb_min[i];
        d.grid.aabb_max[i] = aabb_max[i];
    }
    d.grid.resolution = h;
    d.n_modes = n_modes;
    d.n_active = (int64_t)active_faces.size();
    d.active_faces = active_faces.data();
    d.phi = phi.data();
    d.advection = C.data();
    d.eigenvalues = lam.data();
    d.sign_bits = sign_bits.data();
    return d;
}

}  // namespace psf
