"""TSpecTemplate (gNL-loc, lensing, point-source) against golden fixtures made by
the unmodified reference (tests/golden/make_golden_tspec.py).

Tolerances: the k-space integrals q_l^X(r), p_l^X(r) agree with the reference's
(whose spherical Bessel table is the oracle's scipy restatement of GSL's) to 1e-10
of their largest value; filtered maps, numerators and Fisher entries to 1e-9,
relative per entry (the templates' amplitudes differ by up to 60 decades; a Fisher
entry is compared with sqrt(F_ii F_jj)).
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9


def load(pol):
    return dict(np.load(os.path.join(GOLD, "tspec_nside16_%s.npz" % ("teb" if pol else "t"))))


def rel_max(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    return np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300)


def rel_each(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    return (np.abs(x - ref) / np.maximum(np.abs(ref), 1e-300)).max()


def fisher_err(f, ref):
    d = np.sqrt(np.abs(np.outer(np.diag(ref), np.diag(ref))))
    return (np.abs(f - ref) / d).max()


def _build(d, pol, inject=True):
    import torch
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200.tspec_template import TSpecTemplate
    cltot = {k[6:]: d[k] for k in d if k.startswith("cltot_")}
    clraw = {k[6:]: d[k] for k in d if k.startswith("clraw_")}
    clens = {k[6:]: d[k] for k in d if k.startswith("clens_")}
    beam = d["beam"]
    base = PolySpec(int(d["nside"]), dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="cuda")
    wts = Weightings(base, d["mask"], dict(clraw), noise_cov=d["noise"])
    mask = torch.as_tensor(d["mask"], device="cuda")

    class Ideal:  # the fixture's filter: mask, then the ideal S^-1
        def __call__(self, x, input_type='map', lmax=None):
            return wts.applySinv_ideal(x * mask if input_type == 'map' else x, input_type=input_type, lmax=lmax)

        def batched(self, maps, lmax=None):
            return wts.batched_applySinv_ideal(maps * mask[None], lmax=lmax)

    tst = TSpecTemplate(base, d["mask"], Ideal(), [str(t) for t in d["templates"]], d["k_arr"], d["Tl_arr"],
                        int(d["lmin_t"]), int(d["lmax_t"]), r_values=d["r_values"],
                        r_weights={'gNL-loc': d["r_weights_gNL_loc"]}, C_phi=d["C_phi"], C_lens_weight=clens)
    if inject:
        tst.set_radial_integrals(d["qlXs"], d["plLXs"])
    return base, tst


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_k_integrals(pol):
    d = load(pol)
    _, tst = _build(d, pol, inject=False)
    assert tst.qlXs.shape == d["qlXs"].shape and tst.plLXs.shape == d["plLXs"].shape
    assert rel_max(tst.qlXs, d["qlXs"]) < 1e-10
    assert rel_max(tst.plLXs, d["plLXs"]) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_filtered_maps(pol):
    d = load(pol)
    base, tst = _build(d, pol)
    h = tst._sinv_filt(base._in(d["data"], __import__("torch").float64)[0])
    proc = tst._apply_all_filters(h)
    for k in ("q", "p00", "u", "v"):
        assert rel_max(proc[k].cpu().numpy(), d["proc_" + k]) < TOL, k
    assert rel_max(tst._compute_lensing_Phi(proc, proc).cpu().numpy(), d["phi_dd"]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_numerator(pol):
    d = load(pol)
    _, tst = _build(d, pol)
    tst.generate_sims(1)
    assert rel_each(tst.Tl_numerator(d["data"], include_disconnected_term=False), d["tl_num_4"]) < TOL
    assert rel_each(tst.Tl_numerator(d["data"], include_disconnected_term=True), d["tl_num_full"]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_fisher_contribution(pol):
    d = load(pol)
    base, tst = _build(d, pol)
    a0 = base.generate_data(seed=1 + int(1e9), output_type='harmonic', deconvolve_beam=True)
    assert rel_max(a0, d["fisher_grf_a0"]) < 1e-12
    f = tst.compute_fisher_contribution(1)
    assert fisher_err(f, d["fisher_seed1"]) < TOL
