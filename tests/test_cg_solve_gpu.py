"""Native masked CG (ps_cg_solve through polyspec_b200.cgsolve.NativeCG) against the
batched Python CG (BatchedCGD, the reference's CGD at polyspec/weighting.py:217-367
run per right-hand side) on the same right-hand sides, harmonic preconditioner.

Both drive the same operator kernels; they differ only in the reduction order of the
dot products.  Two CG runs stopped at err < thresh differ by up to their remaining
error, so the solutions must agree to 1e-6 (relative, per system; measured 2.2e-8 at
thresh 1e-8 on the mixed plan) and the step counts to one step; over three fixed
steps the iterates agree to 1e-10.  The native solution also passes the reference's stopping test
on the recomputed true residual b - A x.  Cases: TEB on a mixed plan with Legendre
tables (fused round trip), TEB and T on FP64 plans (synthesis -> weight -> adjoint), a
step limit (PS_ERR_NOT_CONVERGED with the last iterate) and a zero right-hand side
(solved at step 0, as x = x0)."""
import numpy as np
import pytest

NSIDE, LMAX = 32, 64


def _setup(pol, prec):
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200 import workloads as W
    cl, cltot, beam, mask, noise, _ = W.cg_fisher_setup(NSIDE, LMAX, n_holes=40)
    if pol:
        base = PolySpec(NSIDE, dict(cltot), beam=list(beam), pol=True, lmax=LMAX, prec=prec)
        wts = Weightings(base, mask, dict(cl), noise_cov=noise)
    else:
        base = PolySpec(NSIDE, {'TT': cltot['TT']}, beam=[beam[0]], pol=False, lmax=LMAX, prec=prec)
        wts = Weightings(base, mask[:1], {'TT': cl['TT']}, noise_cov=noise[:1])
    return base, wts, mask


def _maps(base, mask, n, pol):
    import torch
    dmask = torch.as_tensor(mask if pol else mask[:1], device="cuda")
    out = []
    for i in range(n):
        a = base.generate_data(seed=70 + i, output_type="harmonic", rng="device")
        if pol and i == n - 1:  # a B-mode-only sky: a slow system
            a[0] = 0.0
            a[1] = 0.0
        out.append(dmask * base.to_map(a))
    return torch.stack(out)


@pytest.mark.gpu
@pytest.mark.parametrize("pol,prec", [(True, "mixed"), (True, "fp64"), (False, "fp64")])
def test_native_cg_matches_batched_cg(pol, prec):
    import torch
    from polyspec_b200.cgsolve import NativeCG
    base, wts, mask = _setup(pol, prec)
    maps = _maps(base, mask, 4, pol)
    thresh, nstep = 1e-8, 400
    wts.batched_applySinv_optimal(maps, preconditioner="harmonic", nstep=nstep, thresh=thresh)
    cg = wts.last_cgd
    ref_x = cg.x0 + cg.x
    ref_it = cg.iters.cpu().numpy()
    b0 = cg._get_b(maps)
    ncg = NativeCG(wts)
    fused = base.prec != "fp64"
    if fused:  # the fused round trip needs the plan's Legendre tables
        assert ncg.plan.has_table(0) and ncg.plan.has_table(2)
    x, its, err, ok = ncg.solve(b0, cg.x0, nstep=nstep, thresh=thresh)
    torch.cuda.synchronize()
    assert ok and bool((err < thresh).all()), (its, err)
    assert np.abs(its - ref_it).max() <= 1, (its, ref_it, fused)
    for n in range(x.shape[0]):
        d = float(torch.linalg.norm(x[n] - ref_x[n]) / torch.linalg.norm(ref_x[n]))
        assert d < 1e-6, (n, d)
    # the true residual meets the stopping test
    r = b0 - cg._apply_A(x)
    sig = cg._sigma
    true_err = (cg.dot(r, sig(r)) / cg.dot(b0, sig(b0))).cpu().numpy()
    assert (true_err < 10 * thresh).all(), true_err


@pytest.mark.gpu
def test_native_cg_step_limit_and_zero_rhs():
    import torch
    from polyspec_b200.cgsolve import NativeCG
    base, wts, mask = _setup(True, "mixed")
    maps = _maps(base, mask, 2, True)
    from polyspec_b200.weighting import BatchedCGD
    x0 = torch.zeros((3, 3, base.plan().nalm), dtype=torch.complex128, device="cuda")
    cg = BatchedCGD(wts, maps, x0[:2], preconditioner="harmonic")
    b0 = torch.cat([cg._get_b(maps), torch.zeros_like(x0[:1])])
    x0[2] = 1.5  # the zero system returns its x0
    ncg = NativeCG(wts)
    x, its, err, ok = ncg.solve(b0, x0, nstep=3, thresh=1e-12)
    assert not ok
    assert list(its) == [3, 3, 0], its
    assert err[2] == 0.0 and bool((err[:2] > 1e-12).all()), err
    assert bool(torch.equal(x[2], x0[2]))
    # three steps of the Python CG from the same start give the same iterate
    cg.run(nstep=3, thresh=1e-12)
    for n in range(2):
        d = float(torch.linalg.norm(x[n] - (cg.x0[n] + cg.x[n])) / torch.linalg.norm(cg.x0[n] + cg.x[n]))
        assert d < 1e-10, (n, d)
