"""TSpecTemplate for the direction-dependent tauNL templates against golden fixtures made
by the unmodified reference (its Gaunt and 3j symbols from the compiled wignerSymbols):
n = 0 (tauNL-direc:1,1,0 and tauNL-direc:2,2,0 together, make_golden_tspec_gaunt.py) and
general (n1, n3, n) (tauNL-direc:1,1,2, tauNL-direc:1,2,1 and tauNL-direc:0,1,1 together,
L in [2, 40]) and the tauNL-even:0, tauNL-even:1 and tauNL-odd:1 combinations
(make_golden_tspec_direc.py).  The k-space and F integrals are injected from
the fixture.  Numerators and Fisher entries to 1e-9, relative per entry (a Fisher entry is
compared with sqrt(F_ii F_jj))."""
import os

import numpy as np
import pytest

from test_tspec import rel_each, fisher_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9


FIXTURES = {"n0": ("tspec_gaunt", {}), "general": ("tspec_direc", {"Lmin": 2, "Lmax": 40}),
            "evenodd": ("tspec_evenodd", {"Lmin": 2, "Lmax": 40})}


def load(pol, kind="n0"):
    return dict(np.load(os.path.join(GOLD, "%s_nside16_%s.npz" % (FIXTURES[kind][0], "teb" if pol else "t"))))


def _build(pol, kind="n0"):
    import torch
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200.tspec_template import TSpecTemplate
    d = load(pol, kind)
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
                        int(base_d["lmax_t"]), r_values=d["r_values"], r_weights=r_weights, **FIXTURES[kind][1])
    tst.set_radial_integrals(d["qlXs"], d["plLXs"], FLLs=d["FLLs"])
    return d, tst


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["n0", "general", "evenodd"])
@pytest.mark.parametrize("pol", [False, True])
def test_numerator(pol, kind):
    d, tst = _build(pol, kind)
    tst.generate_sims(1)
    assert rel_each(tst.Tl_numerator(d["data"], include_disconnected_term=False), d["tl_num_4"]) < TOL
    assert rel_each(tst.Tl_numerator(d["data"], include_disconnected_term=True), d["tl_num_full"]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["n0", "general", "evenodd"])
@pytest.mark.parametrize("pol", [False, True])
def test_fisher_contribution(pol, kind):
    d, tst = _build(pol, kind)
    assert fisher_err(tst.compute_fisher_contribution(1), d["fisher_seed1"]) < TOL


def _configured(templates):
    from polyspec_b200.tspec_template import TSpecTemplate
    t = TSpecTemplate.__new__(TSpecTemplate)
    t.templates = list(templates)
    t.Lmin, t.Lmax, t.lmin, t.lmax = 2, 40, 2, 30

    class _Base:
        l_arr = np.concatenate([np.arange(m, 48) for m in range(48)])
        m_arr = np.concatenate([np.full(48 - m, m) for m in range(48)])
    t.base = _Base()
    t._configure_templates(t.templates, [], {})
    return t


def test_direc_configuration():
    """General (n1, n3, n) parse as the reference does: P_{n} maps for n1 and n3, the triangle
    condition and the n1 <-> n3 degeneracy check; an unknown template is refused."""
    t = _configured(['tauNL-direc:1,2,1', 'tauNL-direc:0,1,1'])
    assert [list(x) for x in t.n1n3n] == [[1, 2, 1], [0, 1, 1]] and t.p_inds == [0, 1, 2]
    with pytest.raises(AssertionError):
        _configured(['tauNL-direc:1,1,3'])
    with pytest.raises(Exception, match="degenerate"):
        _configured(['tauNL-direc:1,2,1', 'tauNL-direc:2,1,1'])
    with pytest.raises(AssertionError, match="Unknown"):
        _configured(['tauNL-medium:1,1.5'])


@pytest.mark.gpu
def test_F_integrals_shifted():
    """F_{L,L+n}(r, r') for n = -2..2 computed on the GPU (ps_tau_F_integral, not injected)
    against the fixture's: 1e-11 of the largest magnitude."""
    import torch
    from polyspec_b200 import PolySpec
    from polyspec_b200.tspec_template import TSpecTemplate
    d = load(False, "general")
    base_d = dict(np.load(os.path.join(GOLD, "tspec_tauloc_nside16_t.npz")))
    base = PolySpec(int(base_d["nside"]), {k[6:]: base_d[k] for k in base_d if k.startswith("cltot_")},
                    beam=base_d["beam"][:1], pol=False, backend="cuda")
    templates = [str(t) for t in d["templates"]]
    tst = TSpecTemplate(base, base_d["mask"], lambda x, input_type='map', lmax=None: x, templates, d["k_arr"],
                        d["Tl_arr"], int(base_d["lmin_t"]), int(base_d["lmax_t"]), r_values=d["r_values"],
                        r_weights={t: d["r_weights_" + t] for t in templates}, Lmin=2, Lmax=40)
    assert tst.FLLs.shape == d["FLLs"].shape
    assert np.abs(tst.FLLs - d["FLLs"]).max() <= 1e-11 * np.abs(d["FLLs"]).max()
    del torch


def test_small_wigner_symbols():
    """The package's wig3zero / wig6 (host-side, for the tauNL-odd weights) and the oracle shim's
    wig6jj against sympy's exact symbols: 1e-14 relative."""
    from sympy.physics.wigner import wigner_3j, wigner_6j
    from polyspec_b200.tspec_template import wig3zero, wig6
    from oracle.shims import pywigxjpf as pw
    for l1 in range(7):
        for l2 in range(7):
            for l3 in range(9):
                e = float(wigner_3j(l1, l2, l3, 0, 0, 0))
                assert abs(wig3zero(l1, l2, l3) - e) <= 1e-14 * abs(e)
    for js in [(1, 1, 1, 1, 1, 1), (2, 1, 2, 1, 3, 1), (0, 1, 1, 1, 1, 1), (3, 1, 4, 1, 3, 1), (2, 1, 1, 1, 2, 1),
               (4, 1, 4, 1, 5, 1), (5, 1, 6, 1, 5, 1), (1, 2, 3, 2, 1, 2), (3, 3, 3, 3, 3, 3), (2, 1, 4, 1, 3, 1)]:
        e = float(wigner_6j(*js))
        assert abs(wig6(*js) - e) <= 1e-14 * max(abs(e), 1e-300), js
        assert abs(pw.wig6jj(*(2 * j for j in js)) - e) <= 1e-14 * max(abs(e), 1e-300), js


def test_odd_even_decompositions():
    """tauNL-even/odd decompositions: the pieces satisfy the triangle conditions and appear in the
    parsed (n1, n3, n) list, and the even weights are (-1)^n (4 pi)^(3/2) / (3 sqrt(2n+1)) times 1, 2."""
    t = _configured(['tauNL-even:2', 'tauNL-odd:1'])
    got = {tuple(x) for x in t.n1n3n}
    for tt in ('tauNL-even:2', 'tauNL-odd:1'):
        for n1, n3, n, w in t._direc_parts(tt):
            assert (n1, n3, n) in got and abs(n1 - n3) <= n <= n1 + n3 and np.isfinite(w)
    pe = (4. * np.pi) ** 1.5 / 3. / np.sqrt(5.)
    assert np.allclose([w for *_, w in t._direc_parts('tauNL-even:2')], [pe, 2 * pe], rtol=1e-15)


def test_lmax_too_large_for_shifts():
    """Lmax + n beyond the maps' lmax is refused while the templates are parsed."""
    from polyspec_b200.tspec_template import TSpecTemplate
    t = TSpecTemplate.__new__(TSpecTemplate)
    t.templates = ['tauNL-direc:1,1,2']
    t.Lmin, t.Lmax, t.lmin, t.lmax = 2, 47, 2, 30

    class _Base:
        l_arr = np.concatenate([np.arange(m, 48) for m in range(48)])
        m_arr = np.concatenate([np.full(48 - m, m) for m in range(48)])
    t.base = _Base()
    with pytest.raises(ValueError, match="Lmax"):
        t._configure_templates(t.templates, [], {})
