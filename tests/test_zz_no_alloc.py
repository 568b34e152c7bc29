"""The allocation-free synthesis entry point (ps_synthesis_noalloc).

It serves callers that cannot allocate device memory when they transform: its
scratch is a static device array inside the library instead of a workspace the
caller allocates.  Called through the C ABI, it must reproduce the workspace
entry point ps_synthesis, call after call (the static scratch keeps the previous
call's contents), and refuse requests larger than its 16 MiB scratch on the host.
This file is collected last so that a failure here stops a run only after every
other test has run.
"""
import ctypes

import numpy as np
import pytest

TOL = 1e-10


def _rel(x, ref):
    return float((x - ref).abs().max() / ref.abs().max())


@pytest.mark.gpu
def test_noalloc_synthesis_matches_workspace_entry_point():
    import torch
    from polyspec_b200 import _lib
    from polyspec_b200.sht import SHTPlan

    L = _lib.lib()
    plan = SHTPlan(32, 95)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):  # two calls in a row with different inputs
        for spin, batch in ((0, 3), (2, 2), (1, 1)):
            g = torch.Generator(device="cuda").manual_seed(100 * call + 10 * spin + batch)
            shape = (batch, plan.nalm) if spin == 0 else (batch, 2, plan.nalm)
            alm = torch.randn(shape, dtype=torch.complex128, device="cuda", generator=g)
            ref = plan.synthesis(alm, spin)
            out = torch.full_like(ref, float("nan"))
            rc = L.ps_synthesis_noalloc(plan._h, ctypes.c_void_p(alm.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                        batch, spin, stream)
            assert rc == 0, _lib.lib().ps_error_string(rc)
            torch.cuda.synchronize()
            assert _rel(out, ref) < TOL, (call, spin, batch)


@pytest.mark.gpu
def test_noalloc_mixed_precision_matches_workspace_entry_point():
    """The mixed-precision plan puts FP32 ring phases and the tensor-core Legendre stage's
    inputs in the same static scratch: compare with ps_synthesis on the same plan handle and a
    workspace the caller allocates (same kernels, so the results agree to rounding)."""
    import torch
    from polyspec_b200 import _lib
    from polyspec_b200.sht import SHTPlan

    L = _lib.lib()
    plan = SHTPlan(32, 95, prec="mixed", autotune=False)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        for spin, batch in ((0, 8), (2, 4), (3, 1)):
            need = ctypes.c_size_t()
            _lib.call("ps_sht_workspace_bytes", plan._h, batch, spin, 0, ctypes.byref(need))
            assert need.value <= 16 * 1024 * 1024
            g = torch.Generator(device="cuda").manual_seed(1000 + 100 * call + 10 * spin + batch)
            shape = (batch, plan.nalm) if spin == 0 else (batch, 2, plan.nalm)
            alm = torch.randn(shape, dtype=torch.complex128, device="cuda", generator=g)
            npix_shape = (batch, plan.npix) if spin == 0 else (batch, 2, plan.npix)
            ref = torch.empty(npix_shape, dtype=torch.float64, device="cuda")
            ws = torch.empty(max(need.value, 256), dtype=torch.uint8, device="cuda")
            _lib.call("ps_synthesis", plan._h, ctypes.c_void_p(alm.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                      batch, spin, ctypes.c_void_p(ws.data_ptr()), need.value, stream)
            out = torch.full_like(ref, float("nan"))
            rc = L.ps_synthesis_noalloc(plan._h, ctypes.c_void_p(alm.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                        batch, spin, stream)
            assert rc == 0, _lib.lib().ps_error_string(rc)
            torch.cuda.synchronize()
            assert plan.error_flag() == 0
            assert _rel(out, ref) < TOL, (call, spin, batch)


@pytest.mark.gpu
def test_noalloc_rejects_requests_beyond_its_scratch():
    import torch
    from polyspec_b200 import _lib
    from polyspec_b200.sht import SHTPlan

    L = _lib.lib()
    plan = SHTPlan(256, 767)
    need = ctypes.c_size_t()
    _lib.call("ps_sht_workspace_bytes", plan._h, 4, 0, 0, ctypes.byref(need))
    assert need.value > 16 * 1024 * 1024
    alm = torch.zeros((4, plan.nalm), dtype=torch.complex128, device="cuda")
    out = torch.zeros((4, plan.npix), dtype=torch.float64, device="cuda")
    rc = L.ps_synthesis_noalloc(plan._h, ctypes.c_void_p(alm.data_ptr()), ctypes.c_void_p(out.data_ptr()), 4, 0,
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -5  # PS_ERR_WORKSPACE, refused before any launch
    torch.cuda.synchronize()
    assert float(out.abs().max()) == 0.0
