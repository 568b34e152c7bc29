"""Fused weighted round trip (ps_sht_weighted_roundtrip): scale * beam * Y^H W Y (beam * alm)
for T (spin 0) and E, B (spin 2) of [B, 3, nalm] harmonics in place, against the same
operator composed from the plan's synthesis, a pixel weight and the adjoint (the CG's
_apply_A before fusion).  Mixed precision: 1e-5 relative (max-norm) per map."""
import numpy as np
import pytest

TOL = 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("nside,lmax,B", [(16, 40, 3), (64, 128, 20), (128, 256, 35)])
@pytest.mark.parametrize("nf", [1, 3])
def test_roundtrip_vs_composed(nside, lmax, B, nf):
    import torch
    from polyspec_b200.sht import SHTPlan
    P = SHTPlan(nside, lmax, prec="mixed", autotune=False, tables=True)
    g = torch.Generator(device="cuda").manual_seed(nside + B + nf)
    nalm, npix = P.nalm, P.npix
    l = torch.as_tensor(np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)]), device="cuda")
    alm = torch.randn((B, nf, nalm), dtype=torch.complex128, device="cuda", generator=g) / (l + 10.0)
    w = torch.rand((nf, npix), dtype=torch.float64, device="cuda", generator=g)
    w[:, :npix // 7] = 0.0
    beam = torch.exp(-l * (l + 1.0) * 1e-4).to(torch.float64)[None].expand(nf, -1).contiguous()
    scale = 4 * np.pi / npix
    out = P.weighted_roundtrip(alm, w, beam, scale)
    assert out is not None and P.has_table(0) and (nf == 1 or P.has_table(2))
    # composed: synthesis of beam * alm, weight, adjoint, beam
    ref = torch.empty_like(alm)
    x = alm * beam
    m0 = P.synthesis(x[:, 0].contiguous(), 0) * w[0]
    ref[:, 0] = P.adjoint(m0, 0, scale) * beam[0]
    if nf == 3:
        m2 = P.synthesis(x[:, 1:].contiguous(), 2) * w[1:]
        ref[:, 1:] = P.adjoint(m2, 2, scale) * beam[1:]
    torch.cuda.synchronize()
    assert P.error_flag() == 0
    err = max(float((out[i] - ref[i]).abs().max() / ref[i].abs().max()) for i in range(B))
    assert err < TOL, err


@pytest.mark.gpu
def test_batched_cg_fused_matches_unfused():
    """The batched CG's A operator with and without fusion (PS_FUSED_A=0): 12 steps of a masked TEB
    solve at Nside 32 give the same iterate to 1e-5 (both mixed precision; the two operators
    differ by FP32 rounding, which the CG steps amplify a little)."""
    import os
    import torch
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200 import workloads as Wl
    nside, lmax = 32, 64
    cl, cltot, beam, mask, noise, l_bins = Wl.cg_fisher_setup(nside, lmax, n_holes=30, fwhm_arcmin=60.0, nbins=4)
    base = PolySpec(nside, dict(cltot), beam=list(beam), pol=True, lmax=lmax, prec="mixed")
    base.plan().tables = True
    wts = Weightings(base, mask, dict(cl), noise_cov=noise)
    d = torch.as_tensor(np.asarray(mask), device="cuda") * base.generate_data(seed=3, output_type="map", rng="device")
    outs, iters = {}, {}
    for fused in ("1", "0"):
        os.environ["PS_FUSED_A"] = fused
        try:
            wts._rt_ops = None
            outs[fused] = wts.batched_applySinv_optimal(d[None], preconditioner="harmonic", nstep=12, thresh=0.0)
            iters[fused] = int(wts.last_cgd.iters[0])
        finally:
            os.environ.pop("PS_FUSED_A", None)
    assert iters["1"] == iters["0"] == 12
    err = float((outs["1"] - outs["0"]).abs().max() / outs["0"].abs().max())
    assert err < 1e-5, err
