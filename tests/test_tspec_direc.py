"""TSpecTemplate for the direction-dependent tauNL templates with n = 0
(tauNL-direc:1,1,0 and tauNL-direc:2,2,0, together) against golden fixtures made by
the unmodified reference (tests/golden/make_golden_tspec_gaunt.py; its Gaunt and 3j
symbols from the compiled wignerSymbols).  The k-space and F integrals are injected
from the fixture.  Numerators and Fisher entries to 1e-9, relative per entry (a
Fisher entry is compared with sqrt(F_ii F_jj))."""
import os

import numpy as np
import pytest

from test_tspec import rel_each, fisher_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9


def load(pol):
    return dict(np.load(os.path.join(GOLD, "tspec_gaunt_nside16_%s.npz" % ("teb" if pol else "t"))))


def _build(pol):
    import torch
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200.tspec_template import TSpecTemplate
    d = load(pol)
    base_d = dict(np.load(os.path.join(GOLD, "tspec_tauloc_nside16_%s.npz" % ("teb" if pol else "t"))))
    cltot = {k[6:]: base_d[k] for k in base_d if k.startswith("cltot_")}
    clraw = {k[6:]: base_d[k] for k in base_d if k.startswith("clraw_")}
    beam = base_d["beam"]
    base = PolySpec(int(base_d["nside"]), dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="cuda")
    wts = Weightings(base, base_d["mask"], dict(clraw), noise_cov=base_d["noise"])
    mask = torch.as_tensor(base_d["mask"], device="cuda")

    class Ideal:  # the fixture's filter: mask, then the ideal S^-1
        def __call__(self, x, input_type='map', lmax=None):
            return wts.applySinv_ideal(x * mask if input_type == 'map' else x, input_type=input_type, lmax=lmax)

        def batched(self, maps, lmax=None):
            return wts.batched_applySinv_ideal(maps * mask[None], lmax=lmax)

    templates = [str(t) for t in d["templates"]]
    r_weights = {t: d["r_weights_" + t] for t in templates}
    tst = TSpecTemplate(base, base_d["mask"], Ideal(), templates, d["k_arr"], d["Tl_arr"], int(base_d["lmin_t"]),
                        int(base_d["lmax_t"]), r_values=d["r_values"], r_weights=r_weights)
    tst.set_radial_integrals(d["qlXs"], d["plLXs"], FLLs=d["FLLs"])
    return d, tst


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_numerator(pol):
    d, tst = _build(pol)
    tst.generate_sims(1)
    assert rel_each(tst.Tl_numerator(d["data"], include_disconnected_term=False), d["tl_num_4"]) < TOL
    assert rel_each(tst.Tl_numerator(d["data"], include_disconnected_term=True), d["tl_num_full"]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_fisher_contribution(pol):
    d, tst = _build(pol)
    assert fisher_err(tst.compute_fisher_contribution(1), d["fisher_seed1"]) < TOL


def test_unsupported_direc_raises():
    """Direction-dependent templates with n > 0 are refused while the templates are parsed."""
    from polyspec_b200.tspec_template import TSpecTemplate
    t = TSpecTemplate.__new__(TSpecTemplate)
    t.templates = ['tauNL-direc:1,1,1']
    with pytest.raises(NotImplementedError):
        t._configure_templates(t.templates, [], {})
