"""The allocation-free coefficient step (psf_coeff_step_static) against a context's step.

psf_coeff_step_static exists for hosts that cannot let a library call
cudaMalloc: a real-time frame loop that cannot take an allocation's
device-wide stall, or an application that owns all device memory in its own
pool and hands the library only device pointers.  It runs the same kernel as
psf_step's coefficient half with its scratch in a fixed array of the
library's device data.  Here the test (not the library) allocates the inputs
with torch, then two calls in a row must reproduce what the existing entry
point gives after one and after two steps, within the plain path's state
tolerance.  This file is named to be collected last.
"""
import ctypes as ct

import numpy as np
import pytest

from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200.fixture import initial_coefficients
from parallelspectralfluids3d_b200.solver import Context

from conftest import rel_err

pytestmark = pytest.mark.gpu

W_TOL = 1e-5  # relative L2 error of w, as in the plain-path parity tests


def _device_inputs(torch, b, w0, forcing):
    N = b.n_modes
    Np = (N + 3) // 4 * 4
    C = np.zeros((N, N, Np), dtype=np.float32)
    C[:, :, :N] = b.C
    dev = torch.device("cuda", 0)
    return (torch.from_numpy(C).to(dev), torch.from_numpy(np.array(w0, dtype=np.float64)).to(dev),
            torch.from_numpy(np.ascontiguousarray(b.lam, dtype=np.float64)).to(dev),
            torch.from_numpy(np.ascontiguousarray(forcing, dtype=np.float64)).to(dev))


@pytest.fixture(params=["box16_n64", "box16_n4", "box12_n160"])
def static_basis(request, c1_basis, medium_basis):
    """Mode counts that reach the kernel's one- and two-chunk templates and its
    smallest and largest row splits (N = 4 splits each mode over 4 blocks)."""
    return {"box16_n64": lambda: c1_basis, "box16_n4": lambda: c1_basis.truncate(4),
            "box12_n160": lambda: medium_basis}[request.param]()


@pytest.mark.parametrize("flags", [L.PSF_FLAG_RENORM, L.PSF_FLAG_RENORM | L.PSF_FLAG_FORCING])
def test_static_scratch_step_matches_context_step(static_basis, flags):
    import torch

    lib = L.load()
    b = static_basis
    w0 = initial_coefficients(b.n_modes, 11)
    forcing = np.zeros(b.n_modes)
    forcing[0] = 0.1 / 0.01
    params = L.make_params(dt=0.01, viscosity=0.02, flags=flags)

    ctx = Context(b, params)
    ctx.set_forcing(forcing)
    ctx.set_state(w0)
    expected = []
    for _ in range(2):
        ctx.step(1)
        expected.append(ctx.get_state())
    ctx.close()

    C, w, lam, f = _device_inputs(torch, b, w0, forcing)
    stream = torch.cuda.Stream()
    for call in range(2):
        rc = lib.psf_coeff_step_static(C.data_ptr(), b.n_modes, w.data_ptr(), lam.data_ptr(), f.data_ptr(),
                                       ct.byref(params), ct.c_void_p(stream.cuda_stream))
        L.check(rc)
        stream.synchronize()
        got = w.cpu().numpy()
        assert rel_err(got, expected[call]) <= W_TOL, f"call {call + 1}"


def test_static_scratch_rejects_sizes_beyond_its_limit():
    lib = L.load()
    params = L.make_params(dt=0.01)
    dummy = ct.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.psf_coeff_step_static(dummy, 4096, dummy, dummy, None, ct.byref(params), None)
    assert rc == -6 and b"PSF_STATIC_MAX_MODES" in lib.psf_last_error()
