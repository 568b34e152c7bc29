"""Mixed-precision SHT (tensor-core Legendre stage, FP32 ring transforms)
against the FP64 backend, with the Legendre tables (streaming tensor-core GEMMs)
and without them (on-the-fly recurrences).  Tolerance: 1e-5 relative (max-norm over every
pixel of the map) for the synthesis of random a_lm up to lmax 383; the TF32 x3
products carry ~2^-21 relative error, the FP32 accumulation over l and the
FP32 ring FFTs ~1e-6 each.  (The 1e-6 requirement of the mixed backend is on
binned spectra and Fisher matrices, where these per-pixel errors average out;
the pipeline tests check it there.)"""
import numpy as np
import pytest

TOL = 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("nside,lmax", [(8, 23), (16, 32), (32, 95), (64, 128), (128, 383)])
@pytest.mark.parametrize("spin", [0, 1, 2, 3])
@pytest.mark.parametrize("batch", [1, 3, 20])
@pytest.mark.parametrize("tables", [False, True])
def test_mixed_synthesis_vs_fp64(nside, lmax, spin, batch, tables):
    import torch
    from polyspec_b200.sht import SHTPlan
    p64 = SHTPlan(nside, lmax, prec="fp64")
    pmx = SHTPlan(nside, lmax, prec="mixed", autotune=False, tables=tables)
    g = torch.Generator(device="cuda").manual_seed(nside * 100 + spin * 10 + batch)
    shape = (batch, p64.nalm) if spin == 0 else (batch, 2, p64.nalm)
    alm = torch.randn(shape, dtype=torch.complex128, device="cuda", generator=g)
    # CMB-like spectrum: a_lm ~ 1/(l+10)
    l = torch.as_tensor(np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)]), device="cuda")
    alm = alm / (l + 10.0)
    ref = p64.synthesis(alm, spin)
    out = pmx.synthesis(alm, spin)
    torch.cuda.synchronize()
    assert pmx.error_flag() == 0
    assert pmx.has_table(spin) == tables
    err = float((out - ref).abs().max() / ref.abs().max())
    assert err < TOL, err


@pytest.mark.gpu
@pytest.mark.parametrize("nside,lmax", [(8, 23), (32, 95), (128, 383)])
@pytest.mark.parametrize("spin", [0, 1, 2, 3])
@pytest.mark.parametrize("batch", [1, 3, 9, 40])
@pytest.mark.parametrize("tables", [False, True])
def test_mixed_adjoint_vs_fp64(nside, lmax, spin, batch, tables):
    import torch
    from polyspec_b200.sht import SHTPlan
    p64 = SHTPlan(nside, lmax, prec="fp64")
    pmx = SHTPlan(nside, lmax, prec="mixed", autotune=False, tables=tables)
    g = torch.Generator(device="cuda").manual_seed(nside * 1000 + spin * 10 + batch)
    shape = (batch, 12 * nside * nside) if spin == 0 else (batch, 2, 12 * nside * nside)
    mp = torch.randn(shape, dtype=torch.float64, device="cuda", generator=g)
    ref = p64.adjoint(mp, spin, 0.5)
    out = pmx.adjoint(mp, spin, 0.5)
    torch.cuda.synchronize()
    assert pmx.error_flag() == 0
    assert pmx.has_table(spin) == tables
    err = float((out - ref).abs().max() / ref.abs().max())
    assert err < TOL, err
