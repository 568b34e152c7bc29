"""Mixed-precision backend against the FP64 backend through the whole
PSpecBin pipeline (masked CG S^-1, batched solves, Fisher contribution).

Both backends run the same CG steps (fixed step count, so the comparison
isolates arithmetic error from the stopping rule).  Tolerance: 1e-6 relative
on each binned spectrum (the norm of its error over the bins against the norm
of the spectrum, per field) and on the Fisher contribution (Frobenius norm),
the accuracy target of the mixed backend; the largest single-bin relative
error is bounded at 2e-6."""
import numpy as np
import pytest

TOL = 1e-6


def _setup(prec, nside=32, lmax=64):
    from polyspec_b200 import PolySpec, Weightings, PSpecBin
    from polyspec_b200 import workloads as W
    cl, cltot, beam, mask, noise, l_bins = W.cg_fisher_setup(nside, lmax, n_holes=40, fwhm_arcmin=40.0, nbins=4)
    # autotune off: every transform of the mixed backend runs the mixed-precision kernels
    base = PolySpec(nside, dict(cltot), beam=list(beam), pol=True, lmax=lmax, prec=prec, autotune=False)
    wts = Weightings(base, mask, dict(cl), noise_cov=noise)
    app = wts.make_applySinv("optimal", preconditioner="harmonic", nstep=8, thresh=0.0)
    psb = PSpecBin(base, mask, app, l_bins, fields=["TT", "TE", "EE", "BB"])
    return base, psb, mask


@pytest.mark.gpu
def test_mixed_pipeline_matches_fp64():
    import torch
    b64, p64, mask = _setup("fp64")
    bmx, pmx, _ = _setup("mixed")
    a = b64.generate_data(seed=123, output_type="harmonic", deconvolve_beam=True)
    data = b64.to_map(b64.generate_data(seed=7, output_type="harmonic")) * mask
    n64 = p64.Cl_numerator(data)
    nmx = pmx.Cl_numerator(data)
    for f in range(n64.shape[0]):
        assert np.linalg.norm(nmx[f] - n64[f]) / np.linalg.norm(n64[f]) < TOL
    assert np.max(np.abs(nmx - n64) / np.abs(n64)) < 2 * TOL
    f64 = p64.compute_fisher_contribution(1, a_lm=a, batched=True)
    fmx = pmx.compute_fisher_contribution(1, a_lm=a, batched=True)
    assert np.linalg.norm(fmx - f64) / np.linalg.norm(f64) < TOL
    # the batched solves reproduce the one-at-a-time solves of the reference structure
    f64s = p64.compute_fisher_contribution(1, a_lm=a, batched=False)
    assert np.linalg.norm(f64s - f64) / np.linalg.norm(f64) < 1e-10
    torch.cuda.synchronize()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,precond", [("mixed", "cut"), ("fp64", "harmonic")])
def test_fisher_contributions_of_several_simulations(prec, precond):
    """compute_fisher_contributions solves the K (N_p + 1) systems of K simulations as one batch; each
    system keeps its own stopping test, so every contribution equals compute_fisher_contribution of its
    simulation (to 1e-8 of sqrt(F_ii F_jj): only the reduction order of the batch's dot products differs)."""
    from polyspec_b200 import PolySpec, Weightings, PSpecBin
    from polyspec_b200 import workloads as W
    nside, lmax = 32, 64
    cl, cltot, beam, mask, noise, l_bins = W.cg_fisher_setup(nside, lmax, n_holes=40, fwhm_arcmin=40.0, nbins=4)
    base = PolySpec(nside, dict(cltot), beam=list(beam), pol=True, lmax=lmax, prec=prec, autotune=False)
    wts = Weightings(base, mask, dict(cl), noise_cov=noise)
    app = wts.make_applySinv("optimal", preconditioner=precond, nstep=300, thresh=1e-10)
    psb = PSpecBin(base, mask, app, l_bins, fields=["TT", "TE", "EE", "BB"])
    a_lms = [base.generate_data(seed=200 + k, output_type="harmonic", deconvolve_beam=True) for k in range(3)]
    many = psb.compute_fisher_contributions(None, a_lms=a_lms)
    assert many.shape == (3, psb.N_p, psb.N_p)
    for k in range(3):
        one = psb.compute_fisher_contribution(0, a_lm=a_lms[k], batched=True)
        scale = np.sqrt(np.outer(np.abs(np.diag(one)), np.abs(np.diag(one))))
        assert np.max(np.abs(many[k] - one) / scale) < 1e-8, k
