"""CUDA backend against golden fixtures produced by the unmodified reference
(tests/golden/make_golden.py): SHT wrappers, S^-1 filters, CG and PSpecBin.

Tolerance: 1e-10 relative (max-norm) for the FP64 backend; CG trajectories
of 8-12 steps and the Fisher matrices built on them: 1e-9.
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-10
TOL_CG = 1e-9


def rel(x, ref):
    x = np.asarray(x)
    ref = np.asarray(ref)
    return np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300)


def load(pol):
    return dict(np.load(os.path.join(GOLD, "pspec_nside16_%s.npz" % ("teb" if pol else "t"))))


def build(d, pol):
    from polyspec_b200 import PolySpec, Weightings
    cltot = {k[6:]: d[k] for k in d if k.startswith("cltot_")}
    clraw = {k[6:]: d[k] for k in d if k.startswith("clraw_")}
    beam = d["beam"]
    base = PolySpec(int(d["nside"]), dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="cuda")
    wts = Weightings(base, d["mask"], dict(clraw), noise_cov=d["noise"])
    return base, wts


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_sht_wrappers(pol):
    d = load(pol)
    base, _ = build(d, pol)
    assert rel(base.to_map(d["in_alm"]), d["to_map"]) < TOL
    assert rel(base.to_lm(d["in_map"]), d["to_lm"]) < TOL
    for s in (1, 2, 3):
        ap, am = d["in_spin%d_alm" % s]
        assert rel(np.stack(base.to_map_spin(ap, am, s)), d["to_map_spin%d" % s]) < TOL
        mp, mm = d["in_spin%d_map" % s]
        assert rel(base.to_lm_spin(mp, mm, s), d["to_lm_spin%d" % s]) < TOL
    assert rel(base.to_map_vec(d["in_vec_alm"]), d["to_map_vec0"]) < TOL
    assert rel(base.to_map_vec(d["in_vec_alm"], output_spin=1), d["to_map_vec1"]) < TOL
    assert rel(base.to_map_vec(d["in_vec_alm"], output_spin=2), d["to_map_vec2"]) < TOL
    assert rel(base.to_lm_vec(d["in_vec_map"]), d["to_lm_vec0"]) < TOL
    assert rel(np.asarray(base.compute_spin_transform_map([d["in_vec_alm"][0]], 1)), d["spin_transform_p1"]) < TOL
    assert rel(np.asarray(base.compute_spin_transform_map([d["in_vec_alm"][1]], -2)), d["spin_transform_m2"]) < TOL
    assert rel(base.applyAinv(d["in_alm"], input_type="harmonic"), d["applyAinv"]) < TOL
    # counters follow the reference
    assert base.n_SHTs_forward > 0 and base.n_SHTs_reverse > 0


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_sinv_filters(pol):
    d = load(pol)
    base, wts = build(d, pol)
    assert rel(wts.applySinv_ideal(d["data"] * d["mask"]), d["sinv_ideal"]) < TOL
    for pre in ("harmonic", "pseudo_inverse"):
        out = wts.applySinv_optimal(d["data"], preconditioner=pre, nstep=12, thresh=0.0)
        assert rel(out, d["sinv_opt_%s" % pre]) < TOL_CG, pre


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_cg_test_mode(pol):
    import torch
    from polyspec_b200.weighting import CGD
    d = load(pol)
    base, wts = build(d, pol)
    xk = torch.as_tensor(d["cg_test_x"], device="cuda")
    A = CGD(wts, torch.as_tensor(d["data"], device="cuda"), preconditioner="harmonic")._apply_A(xk)
    cg = CGD(wts, [], test_b=A, preconditioner="harmonic")
    cg.run(nstep=60, thresh=1e-20)
    sol = cg.x.cpu().numpy()
    assert rel(sol, d["cg_test_sol"]) < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_pspec_bin(pol):
    from polyspec_b200 import PSpecBin
    d = load(pol)
    base, wts = build(d, pol)
    mask = d["mask"]
    fields = ["TT", "TE", "EE", "BB"] if pol else ["TT"]
    ideal = lambda x, input_type="map", lmax=None: wts.applySinv_ideal(x * base._in(mask, x.dtype)[0] if input_type == "map" else x,
                                                                          input_type=input_type, lmax=lmax)
    psb = PSpecBin(base, mask, ideal, d["l_bins"], fields=fields)
    assert rel(psb.Cl_numerator(d["data"]), d["cl_num_ideal_filter"]) < TOL
    # the GRF of seed 1 through the documented host generator
    g = base.generate_data(seed=1 + int(1e7), output_type="harmonic", deconvolve_beam=True)
    assert rel(g, d["grf_seed1"]) < 1e-14
    assert rel(psb.compute_fisher_contribution(1), d["fisher_ideal_filter_seed1"]) < TOL
    opt = lambda x, input_type="map", lmax=None: wts.applySinv_optimal(x, preconditioner="harmonic", nstep=8,
                                                                        thresh=0.0, lmax=lmax)
    psb2 = PSpecBin(base, mask, opt, d["l_bins"], fields=fields)
    assert rel(psb2.compute_fisher_contribution(2), d["fisher_opt_filter_seed2"]) < TOL_CG
    assert rel(psb.compute_fisher_ideal(), d["fisher_ideal_analytic"]) < TOL
    assert rel(psb.Cl_numerator_ideal(d["data"]), d["cl_num_ideal"]) < TOL
