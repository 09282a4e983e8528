// Allocation-free coefficient step: psf_coeff_step_static (include/psf_b200.h).
//
// Some hosts cannot let a library call cudaMalloc.  An interactive frame loop
// like the reference's 60 Hz GUI timer (Widgets/glcanvas.cpp:36-39) cannot
// afford the device-wide synchronisation that cudaMalloc/cudaFree may imply in
// the middle of a frame; an embedding application that carves all device
// memory out of its own fixed pool, or hands this library only device
// pointers over an FFI, has no allocator to offer and must not see the
// library grow its footprint behind its back.  For those callers this file
// runs the same contraction + FP64 state-update kernel as a context's step,
// on buffers the caller already owns, with the kernel's scratch (per-block
// partial sums, the completion ticket, a step counter) taken from a fixed
// array in the library's own device data segment instead of from cudaMalloc.
//
// That array is a file-scope __device__ variable, so every GPU that loads the
// library holds its PSF_STATIC_SCRATCH_BYTES until the process exits.  All
// calls on a device share it: it keeps whatever the previous call left, the
// ticket that must start at zero is cleared on the caller's stream before
// every launch, and two calls whose kernels overlap on the GPU (different
// streams, or different host threads, without ordering between them) race on
// the partial sums and give wrong results.

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "psf_b200.h"
#include "psf_internal.h"

namespace {

// Partial sums of the contraction: one double per (mode, row slice).
constexpr int kStaticPartials = 4096;
constexpr size_t kTicketOffset = sizeof(double) * kStaticPartials;  // u32 ticket
constexpr size_t kCounterOffset = kTicketOffset + 64;                 // u64 step counter
constexpr size_t kScratchBytes = kCounterOffset + 64;
static_assert(kScratchBytes == PSF_STATIC_SCRATCH_BYTES, "header and implementation disagree on the size");

// The scratch itself.  Host code may not use this name as a device address:
// on the host it names a shadow variable, so its address is looked up with
// cudaGetSymbolAddress once per CUDA context (with that context current).
static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_dev[kMaxDevices] = {};
void *g_scratch_ctx[kMaxDevices] = {};  // the context the address above belongs to
int g_num_sms[kMaxDevices] = {};

// cuCtxGetCurrent through the runtime's driver entry point (no link against
// libcuda).  The module holding the scratch array is loaded once per context,
// so a device address is valid only while the context it was resolved in is
// current: after cudaDeviceReset, or with another context made current on
// the same GPU, the array lives at a new address.
using CtxGetCurrentFn = int (*)(void **);

int current_context(void **ctx)
{
    static CtxGetCurrentFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
    });
    *ctx = nullptr;
    if (!fn) return psf::fail(PSF_ERR_CUDA, "cuCtxGetCurrent is not available from the CUDA driver");
    if (fn(ctx) != 0) return psf::fail(PSF_ERR_CUDA, "cuCtxGetCurrent failed");
    return PSF_OK;
}

// Resolve the device address of the scratch array and the SM count for the
// current device.  Done on the first call in each context; a lookup needs
// the module loaded, which a stream capture cannot do, so a first call made
// while `stream` is capturing is refused with PSF_ERR_STATE.
int setup_current_device(cudaStream_t stream, int *device_out, unsigned char **scratch, int *num_sms)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return psf::cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices)
        return psf::fail(PSF_ERR_UNSUPPORTED, "device ordinal beyond the static scratch table");
    void *ctx = nullptr;
    int rc = current_context(&ctx);
    if (rc != PSF_OK) return rc;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!ctx || !g_scratch_dev[dev] || g_scratch_ctx[dev] != ctx) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        e = cudaStreamIsCapturing(stream, &cs);
        if (e != cudaSuccess) return psf::cuda_fail(e, "cudaStreamIsCapturing");
        if (cs != cudaStreamCaptureStatusNone)
            return psf::fail(PSF_ERR_STATE, "psf_coeff_step_static: the first call in a CUDA context must not be "
                                            "made during stream capture (it looks up the scratch array)");
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return psf::cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
        // The lookup made the runtime's context current if none was: record that one.
        rc = current_context(&ctx);
        if (rc != PSF_OK) return rc;
        if (!ctx) return psf::fail(PSF_ERR_CUDA, "no current CUDA context");
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return psf::cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
        g_num_sms[dev] = sms;
        g_scratch_dev[dev] = static_cast<unsigned char *>(p);
        g_scratch_ctx[dev] = ctx;
    }
    *device_out = dev;
    *scratch = g_scratch_dev[dev];
    *num_sms = g_num_sms[dev];
    return PSF_OK;
}

}  // namespace

extern "C" int psf_coeff_step_static(const float *advection_f32, int32_t n_modes, double *w,
                                     const double *eigenvalues, const double *forcing,
                                     const psf_params *params, void *stream)
{
    if (!advection_f32 || !w || !eigenvalues || !params) return psf::fail(PSF_ERR_INVALID, "null argument");
    if (n_modes < 1 || n_modes > PSF_STATIC_MAX_MODES)
        return psf::fail(PSF_ERR_UNSUPPORTED, "psf_coeff_step_static: n_modes must be in [1, PSF_STATIC_MAX_MODES]");
    if (!(params->timestep > 0.0)) return psf::fail(PSF_ERR_INVALID, "timestep must be positive");
    if ((params->flags & PSF_FLAG_FORCING) && !forcing)
        return psf::fail(PSF_ERR_INVALID, "PSF_FLAG_FORCING is set but forcing is null");

    int dev = 0, num_sms = 0;
    unsigned char *scratch = nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = setup_current_device(st, &dev, &scratch, &num_sms);
    if (rc != PSF_OK) return rc;

    // Same work split as a context's step (psf_create), so the result is the
    // same as psf_step's on the same inputs.
    const int N = n_modes;
    const int S = std::max(1, std::min(N, (2 * num_sms + N - 1) / N));
    if ((long long)N * S > kStaticPartials)
        return psf::fail(PSF_ERR_UNSUPPORTED, "psf_coeff_step_static: partial sums exceed the static scratch");

    psf::PlainDev d{};
    d.N = N;
    d.Np = (N + 3) / 4 * 4;
    d.S = S;
    d.C = advection_f32;
    d.w = w;
    d.w_next = w;  // in place
    d.lam = eigenvalues;
    d.force = forcing;
    d.dwpart = reinterpret_cast<double *>(scratch);
    d.ticket = reinterpret_cast<unsigned int *>(scratch + kTicketOffset);
    d.step_ctr = reinterpret_cast<unsigned long long *>(scratch + kCounterOffset);
    d.step_ctr_next = d.step_ctr;
    d.sp.dt = params->timestep;
    d.sp.visc_signed = (params->flags & PSF_FLAG_DECAY_NEG) ? -params->viscosity : params->viscosity;
    d.sp.flags = params->flags;

    cudaError_t e = cudaMemsetAsync(d.ticket, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return psf::cuda_fail(e, "clearing the static ticket");
    return psf::launch_contract_state(d, st);
}
