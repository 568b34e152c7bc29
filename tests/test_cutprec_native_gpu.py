"""Native masked-band preconditioner (ps_cutprec_apply) against its torch composition
(CutPreconditioner with native=False: band stages, torch.bmm with complex64 K_m^-1, Sigma
products) on the same right-hand sides.

Both compute s + c with s = Sigma r; they differ in the per-m GEMM of the correction c:
the native path rounds K_m^-1 and the band vector to BF16 (planes=1) or to BF16 hi + lo
(planes=2) for the tensor cores.  Bars on ||out_native - out_torch|| / ||c||: 3e-2
for planes=1 (BF16 has 8 significant bits), 1e-4 for planes=2; a layout error in the
GEMM's operands or epilogue would give O(1).  The preconditioned CG with the native
path must still reach its tolerance (true residual) in fewer steps than the harmonic CG."""
import pytest


def _setup():
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200 import workloads as W
    nside, lmax = 32, 64
    cl, cltot, beam, mask, noise, _ = W.cg_fisher_setup(nside, lmax, n_holes=40)
    base = PolySpec(nside, dict(cltot), beam=list(beam), pol=True, lmax=lmax, prec="mixed")
    wts = Weightings(base, mask, dict(cl), noise_cov=noise)
    return base, wts, mask


@pytest.mark.gpu
@pytest.mark.parametrize("planes,tol", [(1, 3e-2), (2, 1e-4)])
def test_native_cut_apply_matches_torch(planes, tol):
    import torch
    from polyspec_b200.cutprec import CutPreconditioner
    base, wts, _ = _setup()
    ref = CutPreconditioner(wts, native=False)
    nat = CutPreconditioner(wts, native=True, planes=planes)
    assert ref.enabled and nat._native is not None and nat.Kinv is None
    g = torch.Generator(device="cuda").manual_seed(planes)
    nlm = base.plan().nalm
    for B in (1, 5):
        r = torch.randn((B, 3, nlm), dtype=torch.complex128, device="cuda", generator=g)
        s = ref._sigma(r)
        out_r = ref.apply(r)
        out_n = nat.apply(r)
        torch.cuda.synchronize()
        c = out_r - s
        for b in range(B):
            d = float(torch.linalg.norm(out_n[b] - out_r[b]) / torch.linalg.norm(c[b]))
            assert d < tol, (planes, B, b, d)
        # the m = 0 correction is real
        m0 = torch.as_tensor(base.m_arr == 0, device="cuda")
        assert float((out_n - s)[:, :, m0].imag.abs().max()) == 0.0


@pytest.mark.gpu
def test_native_cut_preconditioned_cg_converges():
    import torch
    base, wts, mask = _setup()
    cut = wts.cut_preconditioner()
    assert cut._native is not None
    dmask = torch.as_tensor(mask, device="cuda")
    maps = []
    for i in range(4):
        a = base.generate_data(seed=90 + i, output_type="harmonic", rng="device")
        if i >= 2:
            a[0] = 0.0
            a[1] = 0.0
        maps.append(dmask * base.to_map(a))
    maps = torch.stack(maps)
    its = {}
    for pre in ("harmonic", "cut"):
        wts.batched_applySinv_optimal(maps, preconditioner=pre, nstep=500, thresh=1e-8)
        cg = wts.last_cgd
        its[pre] = int(cg.iters.sum())
        b0 = cg._get_b(maps)
        r = b0 - cg._apply_A(cg.x0 + cg.x)
        true_err = cg.dot(r, cg._sigma(r)) / cg.dot(b0, cg._sigma(b0))
        assert bool((true_err < 1e-7).all()), (pre, true_err)
    assert its["cut"] < its["harmonic"], its
