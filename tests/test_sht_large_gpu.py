"""SHT parity at the benchmarked sizes.

* FP64 backend against the FP64 oracle at Nside 1024, lmax 2048 (the masked-CG
  Fisher workload): spin 0 and spin 2, one map each way, 1e-10 relative
  (max-norm), as at small Nside.  The log-scaled recurrence seeds matter here:
  sin^m(theta) of the polar rings underflows FP64 for m above ~1000.
* Mixed backend against the FP64 backend at the same size, spin 0 and 2,
  batches of 1 and 3 (every map compared).
* Mixed backend against the oracle at Nside 2048, lmax 4096 (the largest size
  of the mixed-size serving mix), one map each way.  The FP64 backend does not
  run there (its Bluestein work arrays exceed shared memory), so the oracle is
  the reference.

Mixed tolerances: synthesis 2e-6 and adjoint 1e-6 relative (max-norm over the
whole map or alm set).  The error budget: FP32 Legendre values and phases
(2^-24 each), TF32x3 products (~2^-22), the tensor core's truncating FP32
accumulation over short l chunks, FP32 ring FFTs (~log2(n) 2^-24); a
CMB-like a_lm spectrum 1/(l+10) puts the largest contributions at low l.
"""
import numpy as np
import pytest

from oracle import sht as osht

TOL64 = 1e-10
TOL_SYN = 2e-6
TOL_ADJ = 1e-6


def _cmb_alm(rng, lmax, lead):
    n = osht.nalm(lmax)
    a = rng.normal(size=lead + (n,)) + 1j * rng.normal(size=lead + (n,))
    l, m = osht.getlm(lmax)
    a[..., m == 0] = a[..., m == 0].real
    return a / (l + 10.0)


def _rel(x, ref):
    return float(np.abs(x - ref).max() / np.abs(ref).max())


def _as_gpu(a, spin):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a if spin > 0 else a[:, 0])).cuda()


def _as_np(t, spin):
    out = t.cpu().numpy()
    return out if spin > 0 else out[:, None]


@pytest.mark.gpu
@pytest.mark.parametrize("spin", [0, 2])
def test_fp64_vs_oracle_nside1024(spin):
    from polyspec_b200.sht import SHTPlan
    nside, lmax = 1024, 2048
    ncomp = 1 if spin == 0 else 2
    rng = np.random.default_rng(7000 + spin)
    alm = _cmb_alm(rng, lmax, (1, ncomp))
    plan = SHTPlan(nside, lmax, spins=(0, spin), prec="fp64", autotune=False)
    out = _as_np(plan.synthesis(_as_gpu(alm, spin), spin), spin)
    ref = osht.synthesis(alm, lmax, spin, nside)
    assert _rel(out, ref) < TOL64
    mp = rng.normal(size=(1, ncomp, 12 * nside * nside))
    scale = np.pi / (3.0 * nside ** 2)
    out_a = _as_np(plan.adjoint(_as_gpu(mp, spin), spin, scale), spin)
    ref_a = osht.adjoint_synthesis(mp, lmax, spin, nside) * scale
    assert _rel(out_a, ref_a) < TOL64


@pytest.mark.gpu
@pytest.mark.parametrize("spin", [0, 2])
@pytest.mark.parametrize("batch", [1, 3])
def test_mixed_vs_fp64_nside1024(spin, batch):
    import torch
    from polyspec_b200.sht import SHTPlan
    nside, lmax = 1024, 2048
    ncomp = 1 if spin == 0 else 2
    rng = np.random.default_rng(7100 + 10 * spin + batch)
    p64 = SHTPlan(nside, lmax, spins=(0, spin), prec="fp64", autotune=False)
    pmx = SHTPlan(nside, lmax, spins=(0, spin), prec="mixed", autotune=False)
    alm = _as_gpu(_cmb_alm(rng, lmax, (batch, ncomp)), spin)
    ref = p64.synthesis(alm, spin)
    out = pmx.synthesis(alm, spin)
    torch.cuda.synchronize()
    assert pmx.error_flag() == 0
    err = [float((out[i] - ref[i]).abs().max() / ref[i].abs().max()) for i in range(batch)]
    assert max(err) < TOL_SYN, err
    g = torch.Generator(device="cuda").manual_seed(7200 + 10 * spin + batch)
    shape = (batch, 12 * nside ** 2) if spin == 0 else (batch, 2, 12 * nside ** 2)
    mp = torch.randn(shape, dtype=torch.float64, device="cuda", generator=g)
    scale = np.pi / (3.0 * nside ** 2)
    ref_a = p64.adjoint(mp, spin, scale)
    out_a = pmx.adjoint(mp, spin, scale)
    torch.cuda.synchronize()
    assert pmx.error_flag() == 0
    err = [float((out_a[i] - ref_a[i]).abs().max() / ref_a[i].abs().max()) for i in range(batch)]
    assert max(err) < TOL_ADJ, err


@pytest.mark.gpu
@pytest.mark.parametrize("spin", [0, 2])
def test_mixed_vs_oracle_nside2048(spin):
    import torch
    from polyspec_b200.sht import SHTPlan
    nside, lmax = 2048, 4096
    ncomp = 1 if spin == 0 else 2
    rng = np.random.default_rng(7300 + spin)
    alm = _cmb_alm(rng, lmax, (1, ncomp))
    pmx = SHTPlan(nside, lmax, spins=(0, spin), prec="mixed", autotune=False)
    out = _as_np(pmx.synthesis(_as_gpu(alm, spin), spin), spin)
    assert pmx.error_flag() == 0
    ref = osht.synthesis(alm, lmax, spin, nside)
    assert _rel(out, ref) < TOL_SYN
    del out, ref
    mp = rng.normal(size=(1, ncomp, 12 * nside * nside))
    scale = np.pi / (3.0 * nside ** 2)
    out_a = _as_np(pmx.adjoint(_as_gpu(mp, spin), spin, scale), spin)
    torch.cuda.synchronize()
    assert pmx.error_flag() == 0
    ref_a = osht.adjoint_synthesis(mp, lmax, spin, nside) * scale
    assert _rel(out_a, ref_a) < TOL_ADJ
