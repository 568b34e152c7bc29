"""TSpecTemplate for the collider templates (tauNL-light:s,nu_s and tauNL-heavy:s,mu_s) against
golden fixtures made by the unmodified reference (make_golden_tspec_collider.py: light:0,0.7,
light:1,0.3, light:1,0.0, heavy:0,0.5 and heavy:1,0.8 together, L in [2, 40], k_coll = K_coll =
0.01), which exercise the reference's tau_sum_n0_collider, tau_sum_nu0_collider and
tau_sum_general_collider (polyspec/cython/tauNL_utils.pyx:723-964) and its collider p and F
integrals (k_integrals.pyx:399-545, restated by the oracle shim).

The collider p^beta and F^beta integrals computed on the GPU are compared with the fixture's
(1e-9 of the largest magnitude per beta); the numerators (4-field, and with the 2- and 0-field
terms of one simulation pair) and the Fisher contribution of seed 1 with the fixture's integrals
injected, to 1e-9 relative per entry (Fisher entries relative to sqrt(F_ii F_jj)), and the
numerator with the GPU's own integrals to 1e-7."""
import os

import numpy as np
import pytest

from test_tspec import rel_each, fisher_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9


def load(pol):
    return dict(np.load(os.path.join(GOLD, "tspec_collider_nside16_%s.npz" % ("teb" if pol else "t"))))


def beta_key(beta):
    return "%.8f,%.8f" % (np.real(beta), np.imag(beta))


def _build(pol, inject=True):
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
                        int(base_d["lmax_t"]), r_values=d["r_values"], r_weights=r_weights, Lmin=2, Lmax=40,
                        K_coll=0.01, k_coll=0.01)
    if inject:
        tst.set_radial_integrals(d["qlXs"])
        tst.set_collider_integrals({b: d["coll_plLXs_" + beta_key(b)] for b in tst.coll_plLXs},
                                   {b: d["coll_FLLs_" + beta_key(b)] for b in tst.coll_FLLs})
    return d, tst


@pytest.mark.gpu
def test_collider_integrals():
    """p^beta_{lL}^X(r) and F^beta_{L,L+n}(r, r') for the five betas (two complex) against the fixture."""
    d, tst = _build(True, inject=False)
    assert len(tst.coll_plLXs) == 5 and len(tst.coll_FLLs) == 5
    for b, arr in tst.coll_plLXs.items():
        ref = d["coll_plLXs_" + beta_key(b)]
        assert arr.shape == ref.shape
        assert np.abs(arr - ref).max() <= TOL * np.abs(ref).max(), b
    for b, arr in tst.coll_FLLs.items():
        ref = d["coll_FLLs_" + beta_key(b)]
        assert arr.shape == ref.shape
        assert np.abs(arr - ref).max() <= TOL * np.abs(ref).max(), b


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
    """compute_fisher_contribution(1): the collider Q-derivatives (convolve_F_general_collider,
    convolve_F_n000_real, compute_pF_map_complex / _real of tauNL_utils.pyx:997-1446) against the fixture,
    each entry to 1e-9 of sqrt(F_ii F_jj)."""
    d, tst = _build(pol)
    assert fisher_err(tst.compute_fisher_contribution(1), d["fisher_seed1"]) < TOL


@pytest.mark.gpu
def test_numerator_own_integrals():
    d, tst = _build(False, inject=False)
    assert rel_each(tst.Tl_numerator(d["data"], include_disconnected_term=False), d["tl_num_4"]) < 1e-7


def _configured(templates):
    from polyspec_b200.tspec_template import TSpecTemplate
    t = TSpecTemplate.__new__(TSpecTemplate)
    t.templates = list(templates)
    t.Lmin, t.Lmax, t.lmin, t.lmax = 2, 40, 2, 30
    t.K_coll, t.k_coll = 0.01, 0.01

    class _Base:
        l_arr = np.concatenate([np.arange(m, 48) for m in range(48)])
        m_arr = np.concatenate([np.full(48 - m, m) for m in range(48)])
    t.base = _Base()
    t._configure_templates(t.templates, [], {})
    return t


def test_collider_configuration():
    """Collider templates parse as the reference's (polyspec/tspec_template.py:347-389, 415-442): beta = nu_s - 3/2
    or -3/2 +- i mu_s with the (s, S) pairs S = 0, 2, .., 2s, the widened L range and the bounds checks."""
    t = _configured(['tauNL-light:1,0.3', 'tauNL-heavy:2,1.0', 'tauNL-light:0,0.7'])
    keys = list(t.coll_params)
    assert keys[0] == -1.2 and keys[1] == -1.5 + 1.0j and keys[2] == -1.5 - 1.0j and keys[3] == -0.8
    assert [list(x) for x in t.coll_params[-1.5 + 1.0j]] == [[2, 0], [2, 2], [2, 4]]
    assert t.nmax_coll == 2 and t.nmax_coll_F == 4 and t.nLmax == 44 and t.nLmin == -2
    assert t.ints_coll and t.ints_1d and 'q' in t.to_compute
    with pytest.raises(AssertionError):
        _configured(['tauNL-light:1,1.5'])  # nu_s > s - 1/2
    with pytest.raises(Exception, match="degenerate"):
        _configured(['tauNL-light:0,1.5', 'tauNL-loc'])
    with pytest.raises(ValueError, match="Lmax"):
        _configured(['tauNL-heavy:5,1.0'])  # Lmax + 2s beyond the maps' lmax


def test_wig3_small():
    """The host 3j symbol of the collider couplings against sympy's exact values: 1e-14 relative."""
    from sympy.physics.wigner import wigner_3j
    from polyspec_b200.tspec_template import wig3
    for j1 in range(4):
        for j2 in range(4):
            for j3 in range(7):
                for m1 in range(-j1, j1 + 1):
                    for m2 in range(-j2, j2 + 1):
                        m3 = -m1 - m2
                        e = float(wigner_3j(j1, j2, j3, m1, m2, m3))
                        assert abs(wig3(j1, j2, j3, m1, m2, m3) - e) <= 1e-14 * max(abs(e), 1e-300)


def test_collider_couplings():
    """C_s(S, mu_s) for mu_s = 0 is delta_S0 (4 pi)^(3/2) (-1)^s / sqrt(2s+1); for a light particle it is real and,
    at nu_s -> 0, tends to the mu_s = 0 value; omega' vanishes for light particles."""
    from polyspec_b200.tspec_template import TSpecTemplate
    t = TSpecTemplate.__new__(TSpecTemplate)
    for s in range(3):
        for S in range(0, 2 * s + 1, 2):
            exp = (S == 0) * (4. * np.pi) ** 1.5 * (-1.) ** s / np.sqrt(2. * s + 1.)
            assert t._calC(s, S, 0.) == exp
            light = t._calC(s, S, 1e-9j)
            assert np.isrealobj(light) and abs(light - exp) < 1e-6 * (4. * np.pi) ** 1.5
    assert t._omega_prime(1, 0.3j) == 0. and np.isfinite(t._omega_prime(1, 0.8))
