"""The reference-side binding shown in INTEGRATION.md section 2: a maintainer's ctypes.CDLL of
libpscuda.so with argtypes declared by hand (not this package's _lib), plan creation, and
the spin-0 to_lm / to_map calls of polyspec/base.py:145-151, 169-176 routed through
ps_adjoint / ps_synthesis, checked against the package's PolySpec (FP64, 1e-12)."""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_reference_side_ctypes_binding():
    import torch
    from polyspec_b200 import PolySpec
    from polyspec_b200 import workloads as W
    Nside = 32
    lmax = 3 * Nside - 1
    nalm = (lmax + 1) * (lmax + 2) // 2
    ps = ctypes.CDLL(os.path.join(ROOT, "polyspec_b200", "libpscuda.so"))
    ps.ps_plan_create.argtypes = [ctypes.c_int] * 5 + [ctypes.POINTER(ctypes.c_void_p)]
    ps.ps_synthesis.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 2 + [ctypes.c_void_p, ctypes.c_size_t,
                                                                              ctypes.c_void_p]
    ps.ps_adjoint.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 2 + [ctypes.c_double, ctypes.c_void_p,
                                                                            ctypes.c_size_t, ctypes.c_void_p]
    ps.ps_sht_workspace_bytes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_size_t)]
    ps.ps_plan_destroy.argtypes = [ctypes.c_void_p]
    plan = ctypes.c_void_p()
    assert ps.ps_plan_create(Nside, lmax, lmax, 0b1111, 0, ctypes.byref(plan)) == 0
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    input_map = rng.normal(size=(1, 12 * Nside ** 2))
    # to_lm (spin-0 part)
    m = torch.as_tensor(input_map[:1], device='cuda')
    a = torch.empty((1, nalm), dtype=torch.complex128, device='cuda')
    n = ctypes.c_size_t()
    assert ps.ps_sht_workspace_bytes(plan, 1, 0, 1, ctypes.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device='cuda')
    assert ps.ps_adjoint(plan, m.data_ptr(), a.data_ptr(), 1, 0, np.pi / (3. * Nside ** 2), ws.data_ptr(), n.value,
                         stream) == 0
    # to_map of those harmonics
    mp = torch.empty((1, 12 * Nside ** 2), dtype=torch.float64, device='cuda')
    assert ps.ps_sht_workspace_bytes(plan, 1, 0, 0, ctypes.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device='cuda')
    assert ps.ps_synthesis(plan, a.data_ptr(), mp.data_ptr(), 1, 0, ws.data_ptr(), n.value, stream) == 0
    torch.cuda.synchronize()
    cl = W.fiducial_cl(lmax, False)
    base = PolySpec(Nside, {'TT': cl['TT']}, beam=[np.ones(lmax + 1)], pol=False, backend="cuda")
    ref_a = base.to_lm(input_map)
    ref_m = base.to_map(ref_a)
    got_a, got_m = a.cpu().numpy(), mp.cpu().numpy()
    assert np.abs(got_a - ref_a).max() <= 1e-12 * np.abs(ref_a).max()
    assert np.abs(got_m - ref_m).max() <= 1e-12 * np.abs(ref_m).max()
    assert ps.ps_plan_destroy(plan) == 0
