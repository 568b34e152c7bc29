"""TSpecBin (binned trispectrum) against golden fixtures made by the unmodified
reference (tests/golden/make_golden_tspecbin.py): symmetry factors, the numerator
without and with the disconnected terms, and the Fisher contribution.

Tolerances: numerators 1e-10 relative to their largest entry; Fisher entries 1e-9
relative to sqrt(F_ii F_jj) (the bins' amplitudes span many decades).
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    return np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300)


def fisher_err(f, ref):
    d = np.sqrt(np.abs(np.outer(np.diag(ref), np.diag(ref))))
    return (np.abs(f - ref) / np.where(d > 0, d, 1.0)).max()


def load(pol):
    return dict(np.load(os.path.join(GOLD, "tspecbin_nside16_%s.npz" % ("teb" if pol else "t"))))


class _HostBase:
    """The attributes TSpecBin reads from its base class, on the CPU (binning logic only)."""

    def __init__(self, d, pol):
        import torch
        from polyspec_b200.base import getlm
        self.pol = pol
        self.lmax = int(d["lmax"])
        self.l_arr, self.m_arr = getlm(self.lmax)
        self.indices = {'T': 0, 'E': 1, 'B': 2}
        self.parities = {'T': 1, 'E': 1, 'B': -1}
        self.beam = d["beam"]
        self.beam_lm = np.stack([b[self.l_arr] for b in d["beam"]])
        self.device = torch.device("cpu")
        self.m_weight = np.where(self.m_arr == 0, 1.0, 2.0)

    def dev(self, name, lmax=None):
        import torch
        return torch.as_tensor({'beam_lm': self.beam_lm, 'm_weight': self.m_weight}[name])


@pytest.mark.parametrize("pol", [False, True])
def test_symmetry_factors(pol):
    from polyspec_b200.tspec_bin import TSpecBin
    d = load(pol)
    t = TSpecBin(_HostBase(d, pol), d["mask"][0], None, d["l_bins"], fields=[str(f) for f in d["fields"]],
                 parity=str(d["parity"]))
    t._compute_symmetry_factor()
    assert np.array_equal(t.sym_factor, d["sym_factor"])


def _build(d, pol):
    import torch
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200.tspec_bin import TSpecBin
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

    t = TSpecBin(base, d["mask"][0], Ideal(), d["l_bins"], fields=[str(f) for f in d["fields"]],
                 parity=str(d["parity"]))
    return base, t


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_numerator(pol):
    d = load(pol)
    _, t = _build(d, pol)
    assert rel(t.Tl_numerator(d["data"], include_disconnected_term=False), d["tl_num_4"]) < 1e-10
    t.generate_sims(1)
    assert rel(t.Tl_numerator(d["data"], include_disconnected_term=True), d["tl_num_full"]) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_fisher_contribution(pol):
    d = load(pol)
    _, t = _build(d, pol)
    assert fisher_err(t.compute_fisher_contribution(1), d["fisher_seed1"]) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_numerator_ideal(pol):
    """Tl_numerator_ideal against the reference's (exact 3j symbols for the 0- and 2-field terms,
    tests/golden/make_golden_tspecbin_ideal.py): 1e-10 relative, max-norm."""
    d = load(pol)
    g = np.load(os.path.join(GOLD, "tspecbin_ideal_nside16_%s.npz" % ("teb" if pol else "t")))
    _, tsb = _build(d, pol)
    assert rel(tsb.Tl_numerator_ideal(d["data"], include_disconnected_term=False), g["tl_num_ideal_4"]) < 1e-10
    assert rel(tsb.Tl_numerator_ideal(d["data"], include_disconnected_term=True), g["tl_num_ideal_full"]) < 1e-10
