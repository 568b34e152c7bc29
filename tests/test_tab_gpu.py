"""Table-driven tensor-core Legendre stages (ps_plan_build_table) against the FP64
backend: batches that fill several map groups (up to 32 maps of spin 0 or 16 of
spin s per CTA), orders with several l groups, and band plans (ps_plan_band) that
read the parent's table at their ring offset.  Tolerances as for the mixed
backend: 1e-5 relative (max-norm) per transform at these sizes (the FP32 phases
and FFTs, TF32x3 or BF16x3 products and the tensor core's truncating accumulation
over 32-term stages), for both table formats."""
import ctypes

import numpy as np
import pytest

TOL = 1e-5


def _alm(P, B, spin, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    shape = (B, P.nalm) if spin == 0 else (B, 2, P.nalm)
    l = torch.as_tensor(np.concatenate([np.arange(m, P.lmax + 1) for m in range(P.lmax + 1)]), device="cuda")
    return torch.randn(shape, dtype=torch.complex128, device="cuda", generator=g) / (l + 10.0)


def _rel(x, ref):
    return float((x - ref).abs().max() / ref.abs().max())


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["tf32x3", "bf16x3"])
@pytest.mark.parametrize("nside,lmax", [(16, 47), (64, 200), (256, 511)])
@pytest.mark.parametrize("spin", [0, 1, 2])
@pytest.mark.parametrize("batch", [2, 33, 70])
def test_table_transforms_vs_fp64(nside, lmax, spin, batch, fmt):
    import torch
    from polyspec_b200.sht import SHTPlan
    if nside == 256 and batch == 70:
        batch = 34
    p64 = SHTPlan(nside, lmax, prec="fp64", autotune=False)
    pmx = SHTPlan(nside, lmax, prec="mixed", autotune=False, tables=True, table_format=fmt)
    alm = _alm(p64, batch, spin, 10 * nside + spin + batch)
    out = pmx.synthesis(alm, spin)
    ref = p64.synthesis(alm, spin)
    torch.cuda.synchronize()
    assert pmx.has_table(spin) and pmx.error_flag() == 0
    assert max(_rel(out[i], ref[i]) for i in range(batch)) < TOL
    g = torch.Generator(device="cuda").manual_seed(nside + spin + batch)
    mp = torch.randn(ref.shape, dtype=torch.float64, device="cuda", generator=g)
    out_a = pmx.adjoint(mp, spin, 0.25)
    ref_a = p64.adjoint(mp, spin, 0.25)
    torch.cuda.synchronize()
    assert pmx.error_flag() == 0
    assert max(_rel(out_a[i], ref_a[i]) for i in range(batch)) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["tf32x3", "bf16x3"])
@pytest.mark.parametrize("nside,lmax,k", [(16, 40, 5), (64, 150, 13), (128, 256, 64)])
@pytest.mark.parametrize("spin", [0, 2])
def test_table_band_plan_vs_fp64(nside, lmax, k, spin, fmt):
    """Legendre stages of a band plan (the k ring pairs nearest the equator) of a mixed plan
    with a table, against the band plan of an FP64 plan: ps_legendre_synthesis and the adjoint."""
    import torch
    from polyspec_b200 import _lib
    from polyspec_b200.sht import SHTPlan
    p64 = SHTPlan(nside, lmax, prec="fp64", autotune=False)
    pmx = SHTPlan(nside, lmax, prec="mixed", autotune=False, tables=True, table_format=fmt)
    assert pmx.build_table(spin, force=True)
    bands = {}
    for name, P in (("fp64", p64), ("mixed", pmx)):
        h = ctypes.c_void_p()
        _lib.call("ps_plan_band", P._h, k, ctypes.byref(h))
        bands[name] = h
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    B, nc = 5, 1 if spin == 0 else 2
    alm = _alm(p64, B, spin, 77 + spin)
    Rb = 2 * k - 1
    outs = {}
    for name, h in bands.items():
        n = ctypes.c_size_t()
        _lib.call("ps_legendre_workspace_bytes", h, B, spin, 0, ctypes.byref(n))
        ws = torch.empty(max(n.value, 256), dtype=torch.uint8, device="cuda")
        ph = torch.empty((Rb, lmax + 1, B, nc), dtype=torch.complex128, device="cuda")
        _lib.call("ps_legendre_synthesis", h, ctypes.c_void_p(alm.data_ptr()), ctypes.c_void_p(ph.data_ptr()), B,
                  spin, ctypes.c_void_p(ws.data_ptr()), n.value, st)
        outs[name] = ph
    torch.cuda.synchronize()
    assert _rel(outs["mixed"], outs["fp64"]) < TOL
    g = torch.Generator(device="cuda").manual_seed(5 + spin)
    ph = torch.randn((Rb, lmax + 1, B, nc), dtype=torch.complex128, device="cuda", generator=g)
    back = {}
    for name, h in bands.items():
        n = ctypes.c_size_t()
        _lib.call("ps_legendre_workspace_bytes", h, B, spin, 1, ctypes.byref(n))
        ws = torch.empty(max(n.value, 256), dtype=torch.uint8, device="cuda")
        a = torch.empty_like(alm)
        _lib.call("ps_legendre_adjoint", h, ctypes.c_void_p(ph.data_ptr()), ctypes.c_void_p(a.data_ptr()), B, spin,
                  1.0, ctypes.c_void_p(ws.data_ptr()), n.value, st)
        back[name] = a
    torch.cuda.synchronize()
    assert pmx.error_flag() == 0
    assert _rel(back["mixed"], back["fp64"]) < TOL
    for h in bands.values():
        _lib.call("ps_plan_destroy", h)


@pytest.mark.gpu
def test_table_sizes_and_refusals():
    """Table bytes: per table block and quad of rings (Rh rounded up to 128), two half-block units of
    (ncomp x 2 parities x 16 positions x 4 rings) FP32 values plus 16 bytes of padding; FP64 plans refuse
    a table; dropping the tables returns the transforms to the on-the-fly kernels."""
    import torch
    from polyspec_b200 import _lib
    from polyspec_b200.sht import SHTPlan
    nside, lmax = 32, 70
    pmx = SHTPlan(nside, lmax, prec="mixed", autotune=False, tables=False)
    nblk = sum((lmax - m) // 64 + 1 for m in range(lmax + 1))
    nquads = 128 // 4
    assert pmx.table_bytes(0) == nblk * nquads * 2 * (1 * 128 + 4) * 4
    assert pmx.table_bytes(2) == nblk * nquads * 2 * (2 * 128 + 4) * 4
    # BF16x3: per block and slab of 16 rings, 3 planes of (ncomp x 2 parities x 32 positions x 16 rings)
    p3 = SHTPlan(nside, lmax, prec="mixed", autotune=False, tables=False, table_format="bf16x3")
    assert p3.table_bytes(0) == nblk * (128 // 16) * 3 * 2 * 32 * 16 * 2
    assert p3.table_bytes(2) == nblk * (128 // 16) * 3 * 2 * 2 * 32 * 16 * 2
    p64 = SHTPlan(nside, lmax, prec="fp64", autotune=False)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert _lib.lib().ps_plan_build_table(p64._h, 0, st) == _lib.PS_ERR_UNSUPPORTED
    alm = _alm(p64, 3, 0, 1)
    ref = p64.synthesis(alm, 0)
    assert pmx.build_table(0, force=True) and pmx.has_table(0)
    a = pmx.synthesis(alm, 0)
    pmx.drop_tables()
    assert not pmx.has_table(0)
    b = pmx.synthesis(alm, 0)
    torch.cuda.synchronize()
    assert _rel(a, ref) < TOL and _rel(b, ref) < TOL
