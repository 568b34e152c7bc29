"""TSpecTemplate for gNL-con and the EFTI shapes (gNL-dotdot, gNL-dotdel,
gNL-deldel) against golden fixtures made by the unmodified reference
(tests/golden/make_golden_tspec_efti.py).

Tolerances as for the other TSpecTemplate templates: the k-space integrals r, a,
b, c to 1e-10 of their largest value; filtered maps to 1e-9 of theirs; numerators
and Fisher entries to 1e-9, relative per entry (a Fisher entry is compared with
sqrt(F_ii F_jj)).
"""
import os

import numpy as np
import pytest

from test_tspec import rel_max, rel_each, fisher_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9


def load(pol):
    return dict(np.load(os.path.join(GOLD, "tspec_efti_nside16_%s.npz" % ("teb" if pol else "t"))))


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
    rtau_weights = {t: d["rtau_weights_" + t.replace('-', '_')] for t in templates if t != 'gNL-con'}
    tst = TSpecTemplate(base, d["mask"], Ideal(), templates, d["k_arr"], d["Tl_arr"], int(d["lmin_t"]),
                        int(d["lmax_t"]), r_values=d["r_values"], r_weights={'gNL-con': d["r_weights_gNL_con"]},
                        rtau_values=d["rtau_values"], rtau_weights=rtau_weights)
    if inject:
        tst.set_radial_integrals(rlXs=d["rlXs"], alXs=d["alXs"], blXs=d["blXs"], clXs=d["clXs"])
    return base, tst


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_k_integrals(pol):
    d = load(pol)
    _, tst = _build(d, pol, inject=False)
    for k in ("rlXs", "alXs", "blXs", "clXs"):
        assert getattr(tst, k).shape == d[k].shape, k
        assert rel_max(getattr(tst, k), d[k]) < 1e-10, k


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_filtered_maps(pol):
    import torch
    d = load(pol)
    base, tst = _build(d, pol)
    h = tst._sinv_filt(base._in(d["data"], torch.float64)[0])
    proc = tst._apply_all_filters(h)
    for k in ("r", "a", "b", "c"):
        assert rel_max(proc[k].cpu().numpy(), d["proc_" + k]) < TOL, k


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
