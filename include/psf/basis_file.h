// Reader of the .psfb domain-basis file written by
// parallelspectralfluids3d_b200/fixture.py (Basis.save).
//
// Layout (little endian): a 256-byte header
//   char magic[8] = "PSFBASIS"; u32 version = 1; u32 dims[3]; f64 h;
//   f32 aabb_min[3]; f32 aabb_max[3]; i32 n_modes; i64 n_faces; i64 n_active;
//   i64 n_voxels; i64 n_sign_words; u64 offset[7]
// (packed, no padding) followed by the arrays at the given byte offsets:
//   active_faces i32[n_active], lam f64[N], gravity f64[N],
//   phi f64[n_active][N], C f64[N][N][N], sign_bits u32[n_sign_words],
//   inside u8[n_voxels].
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "psf_b200.h"

namespace psf {

struct BasisFile {
    uint32_t dims[3] = {0, 0, 0};
    double h = 0.0;
    float aabb_min[3] = {0, 0, 0};
    float aabb_max[3] = {0, 0, 0};
    int32_t n_modes = 0;
    int64_t n_faces = 0;
    std::vector<int32_t> active_faces;
    std::vector<double> lam, gravity;
    std::vector<double> phi;  // [n_active][n_modes]
    std::vector<double> C;    // [n_modes]^3
    std::vector<uint32_t> sign_bits;
    std::vector<uint8_t> inside;

    // Returns an empty string on success, else the reason.
    std::string load(const std::string &path);
    // Exact prefix slice to the lowest n modes.
    BasisFile truncated(int32_t n) const;
    // Descriptor pointing into this object's arrays (valid while it lives).
    psf_basis_desc desc() const;
    bool empty() const { return n_modes == 0; }
};

}  // namespace psf
