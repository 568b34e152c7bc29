"""TSpecTemplate for the local tauNL template (beside gNL-loc) against golden
fixtures made by the unmodified reference (tests/golden/make_golden_tspec_tauloc.py).

The reference evaluates F_L(r, r') with GSL's 2F1; the fixtures carry the oracle's
scipy evaluation, which the GPU's series / connection-formula evaluation matches to
1e-11 of the largest entry here (both are checked against mpmath on the CPU in
tests/test_kint_oracle.py).  (P Q)_LM maps to 1e-9 of their largest value;
numerators and Fisher entries to 1e-9, relative per entry (a Fisher entry is
compared with sqrt(F_ii F_jj)).
"""
import os

import numpy as np
import pytest

from test_tspec import rel_max, rel_each, fisher_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9


def load(pol):
    return dict(np.load(os.path.join(GOLD, "tspec_tauloc_nside16_%s.npz" % ("teb" if pol else "t"))))


def _build(d, pol, inject=True):
    import torch
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200.tspec_template import TSpecTemplate
    cltot = {k[6:]: d[k] for k in d if k.startswith("cltot_")}
    clraw = {k[6:]: d[k] for k in d if k.startswith("clraw_")}
    beam = d["beam"]
    base = PolySpec(int(d["nside"]), dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="cuda")
    wts = Weightings(base, d["mask"], dict(clraw), noise_cov=d["noise"])
    mask = torch.as_tensor(d["mask"], device="cuda")

    class Ideal:  # the fixture's filter: mask, then the ideal S^-1
        def __call__(self, x, input_type='map', lmax=None):
            return wts.applySinv_ideal(x * mask if input_type == 'map' else x, input_type=input_type, lmax=lmax)

        def batched(self, maps, lmax=None):
            return wts.batched_applySinv_ideal(maps * mask[None], lmax=lmax)

    templates = [str(t) for t in d["templates"]]
    r_weights = {t: d["r_weights_" + t.replace('-', '_')] for t in templates}
    tst = TSpecTemplate(base, d["mask"], Ideal(), templates, d["k_arr"], d["Tl_arr"], int(d["lmin_t"]),
                        int(d["lmax_t"]), r_values=d["r_values"], r_weights=r_weights)
    if inject:
        tst.set_radial_integrals(d["qlXs"], d["plLXs"], FLLs=d["FLLs"])
    return base, tst


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_F_integrals(pol):
    d = load(pol)
    _, tst = _build(d, pol, inject=False)
    assert tst.FLLs.shape == d["FLLs"].shape
    assert rel_max(tst.FLLs, d["FLLs"]) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_PQ_maps(pol):
    import torch
    d = load(pol)
    base, tst = _build(d, pol)
    h = tst._sinv_filt(base._in(d["data"], torch.float64)[0])
    proc = tst._apply_all_filters(h)
    A = tst._A_maps(proc, proc, 0)[0][:, torch.as_tensor(np.nonzero(tst.nLminfilt)[0], device="cuda")]
    assert rel_max(A.T.cpu().numpy(), d["A_dd"]) < TOL


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
    _, tst = _build(d, pol)
    assert fisher_err(tst.compute_fisher_contribution(1), d["fisher_seed1"]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_gaunt_maps(pol):
    """The direction-dependent P_{n,mu} maps (n = 1, 2) of _compute_weighted_gaunt_maps against the
    reference's (tests/golden/make_golden_tspec_gaunt.py; its Gaunt coefficients from the compiled
    wignerSymbols): 1e-12 of the largest magnitude."""
    import torch
    d = load(pol)
    g = dict(np.load(os.path.join(GOLD, "tspec_gaunt_nside16_%s.npz" % ("teb" if pol else "t"))))
    _, tst = _build(d, pol)
    tst.set_radial_integrals(plLXs=g["plLXs"])
    h = torch.as_tensor(g["h_filt"], device="cuda")
    for n in (1, 2):
        for mu in range(n + 1):
            got = tst._compute_weighted_gaunt_maps(h, tst.d_plLXs, n, mu).cpu().numpy()
            assert rel_max(got, g["p%d%d" % (n, mu)]) < 1e-12, (n, mu)
