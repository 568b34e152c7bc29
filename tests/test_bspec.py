"""BSpecBin (binned bispectrum) against golden fixtures made by the unmodified
reference (tests/golden/make_golden_bspec.py): bin list, symmetry factors,
numerators (cubic, with the linear term, ideal) and the Fisher contribution.

Tolerances (relative, max-norm over the vector / matrix): 1e-10 for the
numerators and 1e-9 for the Fisher contribution on the FP64 backend.
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-10
TOL_F = 1e-9


def rel(x, ref):
    x = np.asarray(x)
    ref = np.asarray(ref)
    return np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300)


def load(pol):
    return dict(np.load(os.path.join(GOLD, "bspec_nside16_%s.npz" % ("teb" if pol else "t"))))


class _HostBase:
    """The attributes BSpecBin reads from its base class, on the CPU (binning logic only)."""

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
def test_bin_list_and_symmetry(pol):
    from polyspec_b200.bspec_bin import BSpecBin
    d = load(pol)
    base = _HostBase(d, pol)
    b = BSpecBin(base, d["mask"][0], None, d["l_bins"], fields=[str(f) for f in d["fields"]],
                 parity=str(d["parity"]))
    b._compute_symmetry_factor()
    assert np.array_equal(b.all_bins, d["all_bins"])
    assert np.array_equal(b.sym_factor, d["sym_factor"])
    # every triplet feeds three (pair, field, bin) contributions into each of its Q3 rows
    assert len(b.all_bins) * len(b.chi_arr) == b.N_b


def _build(d, pol):
    import torch
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200.bspec_bin import BSpecBin
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

    bsb = BSpecBin(base, d["mask"][0], Ideal(), d["l_bins"], fields=[str(f) for f in d["fields"]],
                   parity=str(d["parity"]))
    return base, bsb


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_numerators(pol):
    d = load(pol)
    base, bsb = _build(d, pol)
    assert rel(bsb.Bl_numerator(d["data"], include_linear_term=False), d["bl_num_cubic"]) < TOL
    bsb.generate_sims(2)
    assert rel(bsb.Bl_numerator(d["data"], include_linear_term=True), d["bl_num_full"]) < TOL
    assert rel(bsb.Bl_numerator_ideal(d["data"]), d["bl_num_ideal"]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_fisher_contribution(pol):
    d = load(pol)
    base, bsb = _build(d, pol)
    a0 = base.generate_data(seed=1 + int(1e8), deconvolve_beam=True, output_type="harmonic")
    assert rel(a0, d["fisher_grf_a0"]) < 1e-12
    f = bsb.compute_fisher_contribution(1)
    assert rel(f, d["fisher_seed1"]) < TOL_F


@pytest.mark.gpu
def test_fisher_contribution_unbatched_filter():
    """The same contribution through an applySinv without a batched method."""
    d = load(False)
    base, bsb = _build(d, False)
    f = bsb.applySinv

    class Plain:
        def __call__(self, *a, **k):
            return f(*a, **k)
    bsb.applySinv = Plain()
    assert rel(bsb.compute_fisher_contribution(1), d["fisher_seed1"]) < TOL_F


@pytest.mark.gpu
@pytest.mark.parametrize("pol", [False, True])
def test_fisher_ideal(pol):
    """The analytic ideal Fisher matrix against the reference's (exact 3j symbols,
    tests/golden/make_golden_bspec_ideal.py): 1e-12 relative, max-norm."""
    d = load(pol)
    g = np.load(os.path.join(GOLD, "bspec_ideal_nside16_%s.npz" % ("teb" if pol else "t")))["fisher_ideal"]
    _, bsb = _build(d, pol)
    assert rel(bsb.compute_fisher_ideal(), g) < 1e-12


@pytest.mark.gpu
def test_mc_fisher_converges_to_ideal():
    """With a unit mask and the ideal filter the Monte Carlo Fisher matrix converges to
    the analytic ideal one (the consistency check the reference's ideal estimators
    provide): 160 seeds, diagonal within 5 %, every entry within 3 % of the largest."""
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200.bspec_bin import BSpecBin
    d = load(False)
    cltot = {k[6:]: d[k] for k in d if k.startswith("cltot_")}
    clraw = {k[6:]: d[k] for k in d if k.startswith("clraw_")}
    base = PolySpec(int(d["nside"]), dict(cltot), beam=d["beam"][:1], pol=False, backend="cuda")
    ones = np.ones_like(d["mask"])
    wts = Weightings(base, ones, dict(clraw), noise_cov=d["noise"])
    bsb = BSpecBin(base, ones[0], wts.make_applySinv('ideal'), d["l_bins"], fields=['TTT'], parity='even')
    Fi = bsb.compute_fisher_ideal()
    F = np.mean([bsb.compute_fisher_contribution(s) for s in range(160)], axis=0)
    assert np.abs(np.diag(F) / np.diag(Fi) - 1.).max() < 0.05
    assert np.abs(F - Fi).max() < 0.03 * np.abs(Fi).max()
