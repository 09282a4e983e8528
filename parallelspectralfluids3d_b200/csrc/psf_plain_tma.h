// Coefficient half of a single-instance step (FP32 basis): one cooperative,
// TMA-staged kernel for contraction, FP64 state update and reconstruction.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "psf_internal.h"

namespace psf {

// Tensor maps of C ([k][a][j], tiles of 32 rows x 64 columns) and Phi
// ([tile][i][64 faces], boxes of 64 modes of one tile), FP32, no swizzle.
int make_plain_tma_maps(const PlainDev &d, CUtensorMap *tmC, CUtensorMap *tmP);
// Row chunks per mode of the contraction (dwpart holds N x this many partials).
int contract_tma_row_chunks(int N);
int coeff_tma_smem_bytes(int N);
// One launch per step: `grid_bar` is zeroed on `st` first; one CTA per SM.
int launch_coeff_tma(const PlainDev &d, const CUtensorMap &tmC, const CUtensorMap &tmP, int num_sms,
                     unsigned int *grid_bar, int *err, cudaStream_t st);

// FP32 tiled tensor map without swizzle (zero fill outside the tensor).
int encode_tensor_map_f32(CUtensorMap *map, void *base, int rank, const uint64_t *dims, const uint64_t *strides_bytes,
                          const uint32_t *box);

}  // namespace psf
