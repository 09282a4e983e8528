// Internal types of the batched engine (include/psf_batch.h), shared by the
// kernels (psf_batch.cu) and the C ABI implementation (psf_batch_api.cpp).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "psf_internal.h"

namespace psf {

constexpr int BATCH_MAX_GROUPS = 6;   // distinct bases in one batch
constexpr int BATCH_MAX_SLOTS = 256;  // instance slots per basis (one MMA N tile)
constexpr int BATCH_MAX_ALL_SLOTS = BATCH_MAX_GROUPS * BATCH_MAX_SLOTS;
constexpr int GEMM_THREADS = 192;     // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int GEMM_MAX_KSPLIT = 4;

// One basis inside a GEMM launch: A operand (C or Phi) and B operand (the
// slots' coefficient vectors), both BF16 hi/lo pairs, K-major, 128-byte
// swizzled by TMA.
struct SlotDev;

struct alignas(64) GemmGroup {
    CUtensorMap tmA;        // 4D (k inner 64, rows 128, hi/lo 2, outer 1)
    CUtensorMap tmB;        // 3D (k inner 64, bn rows, hi/lo 2)
    int tiles;              // work units of this basis: 128-row tiles x K splits
    int m_inner;            // row tiles per outer index (contraction: a-tiles per mode k)
    int k_chunks;           // K / 64
    int ksplit;             // K ranges per row tile (each writes its own partial sums)
    int kc_per;             // K chunks per range
    int bn;                 // MMA N: slots rounded up to 16
    uint32_t tx_bytes;      // bytes one pipeline stage receives
    int cap;                // slots in use (columns)
    int n_rows;             // valid rows: N (contraction) or F_act (reconstruction)
    int ldw;                // row stride of w (= the basis' N)
    const float *wf;        // contraction: FP32 copy of the state [cap][ldw]
    double *dwpart;         // contraction: partials [k][nparts (a-tile, K range, warp)][slot]
    int nparts;             // contraction: partials per (slot, k)
    long long n_faces;
    const int32_t *pair_dst;  // reconstruction: [n_rows][2] float slots in a slot's face pairs
    float *pairs;           // reconstruction: per-voxel face pairs [cap][3V] (float2)
    long long pair_floats;  // 6V: floats per slot in pairs
    const SlotDev *slot_of; // reconstruction: the group's slots (column b is slot_of[b]); pairs are
                            // written only for slots that stepped (the tracer reads no others)
};

struct GroupDev;

// Arguments of one tensor-core launch: contraction units [0, c_tiles) over
// g[0 .. n_groups), reconstruction units over g[n_groups .. 2 n_groups).
// A fused launch (cooperative) runs the state update between the two.
struct StepArgs {
    GemmGroup g[2 * BATCH_MAX_GROUPS];
    int n_groups;
    int c_tiles;
    int r_tiles;
    int fused;
    int *err;                 // device error word (bounded waits)
    unsigned int *grid_bar;   // grid barrier counter, zeroed before each fused launch
    const GroupDev *groups;   // state update of a fused launch
    SlotDev *slots;
    int n_slots;
};

// Per-slot parameters and counters, in device memory.
struct SlotDev {
    int active;
    int n_modes;
    int rk4;
    int group;
    int slot;
    unsigned int flags;
    double dt;
    double visc_signed;
    float lifetime;
    float pad0;
    unsigned long long seed;
    unsigned long long step;  // steps taken since the slot was set (device counter)
    long long n_particles;
    long long poff;           // first particle of the slot in the particle pool
    unsigned long long target;  // stop after this many steps (0: no limit)
    int stepped;              // 1 if the slot advanced in the current step (set by the state kernel)
    int pad1;
};

// Per-basis device view used by the state kernel and the tracer.
struct GroupDev {
    GridDev grid;
    int N, Nj, cap, bn, a_tiles, slot_base;
    int nparts;           // contraction partials per mode: a_tiles x ksplit x 4
    long long n_faces, pmax;
    double *w;            // [cap][N]
    float *wf;            // [cap][N] FP32 copy of w (contraction epilogue)
    double *force;        // [cap][N]
    const double *lam;    // [N]
    double *dwpart;       // see GemmGroup
    uint16_t *W;          // BF16 [2][bn][Nj]
    float2 *pairs;        // [cap][3V] per-voxel face pairs of each slot
    long long V;
    float4 *parts;        // particle pool (all slots of the batch)
    int32_t *perm;        // caller index of each pooled particle
};


// Launchers (psf_batch.cu).  `bn_max` selects the kernel variant (64, 128 or
// 256 MMA columns per accumulator); `grid` the number of persistent CTAs.
int batch_gemm_smem_bytes(int bn_max);
int launch_batch_step_tc(const StepArgs &args, int bn_max, int grid, cudaStream_t st);
int max_fused_grid(int bn_max, int num_sms);
int launch_batch_state(const GroupDev *groups, SlotDev *slots, int n_slots, cudaStream_t st);
// prefix[s] = particles of slots 0..s-1 (occupied slots only); n_slots + 1 entries.
int launch_batch_trace(const GroupDev *groups, const SlotDev *slots, const long long *prefix, int n_slots, int grid,
                       cudaStream_t st);
int launch_batch_pack(const GroupDev *groups, const SlotDev *slots, int slot_global, cudaStream_t st);
int batch_trace_grid(int num_sms);

// Host helpers.
int encode_tensor_map(CUtensorMap *map, void *base, int rank, const uint64_t *dims, const uint64_t *strides_bytes,
                      const uint32_t *box);
void split_bf16_host(double x, uint16_t *hi, uint16_t *lo);

}  // namespace psf

// Entry points of psf_batch_api.cpp used by the serving engine
// (psf_engine.cpp); not part of the C ABI.
struct psf_batch;
struct psf_instance_desc;
namespace psf {
// psf_batch_set_instances without the closing synchronisation: the copies,
// orderings and the priming contraction stay queued on the batch's stream.
// Host rows the copies read are kept until the next psf_batch_sync.
int batch_place_async(psf_batch *B, int32_t n, const int32_t *basis, const int32_t *slot,
                      const psf_instance_desc *const *inst, int32_t *status);
// Second stream and pinned buffers for batch_read_frozen (once, before use).
int batch_prepare_reads(psf_batch *B);
// State and caller-order particles of occupied slots that the work queued on
// the batch's stream does not step (their step target is reached), read on a
// second stream while that work runs.  The caller-order scatter runs on the
// host.
int batch_read_frozen(psf_batch *B, int32_t n, const int32_t *basis, const int32_t *slot, double *const *w,
                      float *const *xyzw);
}  // namespace psf
