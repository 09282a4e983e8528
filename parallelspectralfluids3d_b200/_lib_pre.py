"""ctypes declarations of the precompute kernels (``include/psf_precompute.h``)."""

from __future__ import annotations

import ctypes as ct

PRE_EXPORTS = ("psf_pre_csr_cheb", "psf_pre_advection_workspace", "psf_pre_advection_tensor")


class WedgeDesc(ct.Structure):
    _fields_ = [
        ("n_edges", ct.c_int64),
        ("n_modes", ct.c_int32),
        ("ldn", ct.c_int32),
        ("edge_faces", ct.c_void_p),
        ("edge_S", ct.c_void_p),
        ("psi", ct.c_void_p),
        ("phi", ct.c_void_p),
        ("phi_zero_row", ct.c_int64),
        ("eigenvalues", ct.c_void_p),
    ]


def declare(lib) -> None:
    vp = ct.c_void_p
    d = ct.c_double
    lib.psf_pre_csr_cheb.argtypes = [ct.c_int64, ct.c_int64, ct.c_int32, ct.c_int64, vp, vp, vp, vp, vp, vp,
                                     d, d, d, vp]
    lib.psf_pre_advection_workspace.argtypes = [ct.POINTER(WedgeDesc), ct.c_int32, ct.POINTER(ct.c_int64)]
    lib.psf_pre_advection_tensor.argtypes = [ct.POINTER(WedgeDesc), ct.c_int32, vp, ct.c_int64, vp, vp]
