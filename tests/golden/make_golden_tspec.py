"""Generate the TSpecTemplate golden fixtures of tests/golden from the UNMODIFIED reference.

    python tests/golden/make_golden_tspec.py [/path/to/reference]

Runs polyspec/tspec_template.py of the reference as-is, for the templates
gNL-loc, lensing and point-source, over the oracle shims: ducc0's SHTs are the
FP64 restatement of oracle/sht_oracle.cpp; the reference's Cython modules are its
own tauNL_utils and ideal_fisher compiled by oracle/build_ref.sh, and the numpy
restatement oracle/shims/k_integrals.py stands in for k_integrals (GSL is absent).
Two compatibility aliases are installed first: ``np.product`` (removed in numpy 2)
-> ``np.prod``, and ``scipy.special.lpmn`` (removed in scipy 1.15; the reference
uses it only in its radial-sampling optimiser) -> a function that raises.

Inputs (Nside 16, base lmax 47; l in [2, 30]): seeded smooth transfer functions
T_l^X(k) on 160 log-spaced k in [1e-4, 0.12] Mpc^-1, 6 radial points around
recombination with seeded weights, C_phi = 1e-7 / (L (L+1))^2, the fiducial
spectra as the lensing weights, the latitude mask and the ideal S^-1 filter.

Fixtures: the q_l^X(r) and p_l^X(r) integrals, the data's filtered maps, the
numerator with and without the disconnected terms (one simulation pair), and
compute_fisher_contribution(seed=1), for T only and for T, E, B.

Only this script reads the reference checkout; the committed .npz files are
what the tests use.
"""
import importlib.util
import os
import sys

import numpy as np
import scipy.special

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

if not hasattr(np, "product"):
    np.product = np.prod
if not hasattr(scipy.special, "lpmn"):
    def _lpmn(*a, **k):
        raise NotImplementedError("lpmn is not available in this scipy")
    scipy.special.lpmn = _lpmn

from oracle import reference_harness  # noqa: E402
from make_golden import inputs, NSIDE  # noqa: E402

TEMPLATES = ['gNL-loc', 'lensing', 'point-source']
LMIN, LMAX = 2, 30


def transfer(pol, k_arr, lmax_t, seed=3):
    """Seeded smooth transfer functions: sums of Gaussian bumps in (log k, l), zero at l = 0, 1."""
    rng = np.random.default_rng(seed)
    npol = 2 if pol else 1
    l = np.arange(lmax_t + 1)[:, None]
    lk = np.log(k_arr)[None, :]
    T = np.zeros((npol, lmax_t + 1, len(k_arr)))
    for X in range(npol):
        for _ in range(6):
            a = rng.normal() * (0.3 if X else 1.0)
            lc = rng.uniform(np.log(2e-4), np.log(0.08))
            sl = rng.uniform(0.4, 1.2)
            l0 = rng.uniform(0, lmax_t)
            s0 = rng.uniform(5, 20)
            T[X] += a * np.exp(-(lk - lc) ** 2 / (2 * sl ** 2) - (l - l0) ** 2 / (2 * s0 ** 2))
    T[:, :2] = 0.
    return T


def make(pol, ref):
    base_mod, wt_mod, ts_mod = ref["base"], ref["weighting"], ref["tspec_template"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    out = {"nside": NSIDE, "lmax": lmax, "pol": int(pol), "mask": mask, "noise": noise, "beam": beam,
           "lmin_t": LMIN, "lmax_t": LMAX, "templates": np.asarray(TEMPLATES)}
    for k, v in cltot.items():
        out["cltot_" + k] = v
    for k, v in cl.items():
        out["clraw_" + k] = v
    base = base_mod.PolySpec(NSIDE, dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="ducc",
                             nthreads=2)
    wts = wt_mod.Weightings(base, mask, dict(cl), noise_cov=noise)
    ideal = lambda x, input_type="map", lmax=None: wts.applySinv_ideal(x * mask if input_type == "map" else x,
                                                                          input_type=input_type, lmax=lmax)
    k_arr = np.geomspace(1e-4, 0.12, 160)
    Tl = transfer(pol, k_arr, lmax + 1)
    rng = np.random.default_rng(11)
    r_values = np.linspace(13300., 14400., 6)
    r_weights = {'gNL-loc': rng.uniform(0.5, 1.5, 6) * 200.}
    L = np.arange(lmax + 1, dtype=np.float64)
    C_phi = np.zeros(lmax + 1)
    C_phi[1:] = 1e-7 / (L[1:] * (L[1:] + 1.)) ** 2
    C_lens = {k: cl[k].copy() for k in (['TT', 'TE', 'EE', 'BB'] if pol else ['TT'])}
    out.update(k_arr=k_arr, Tl_arr=Tl, r_values=r_values, r_weights_gNL_loc=r_weights['gNL-loc'], C_phi=C_phi)
    for k, v in C_lens.items():
        out["clens_" + k] = v
    tst = ts_mod.TSpecTemplate(base, mask, ideal, list(TEMPLATES), k_arr, Tl, LMIN, LMAX, r_values=r_values,
                               r_weights=r_weights, C_phi=C_phi, C_lens_weight=C_lens)
    out["qlXs"] = tst.qlXs
    out["plLXs"] = tst.plLXs
    data = base.to_map(base.generate_data(seed=5, output_type="harmonic"))
    out["data"] = data
    h = np.asarray(tst.applySinv(data, input_type='map', lmax=tst.lmax)[:, tst.lminfilt], order='C')
    proc = tst._apply_all_filters(h)
    for k in ('q', 'p00', 'u', 'v'):
        out["proc_" + k] = proc[k]
    out["phi_dd"] = tst._compute_lensing_Phi(proc, proc)
    tst.generate_sims(1)
    out["tl_num_4"] = tst.Tl_numerator(data, include_disconnected_term=False)
    out["tl_num_full"] = tst.Tl_numerator(data, include_disconnected_term=True)
    out["fisher_seed1"] = tst.compute_fisher_contribution(1)
    for ii in range(2):
        out["fisher_grf_a%d" % ii] = base.generate_data(seed=1 + int((1 + ii) * 1e9), output_type='harmonic',
                                                        deconvolve_beam=True)
    return out


def load_reference(refroot):
    """The reference's base, weighting and tspec_template modules over the oracle shims."""
    ref = reference_harness.load(refroot, modules=("base", "weighting"))
    reference_harness.load_cython()
    spec = importlib.util.spec_from_file_location("refpolyspec.tspec_template",
                                                  os.path.join(refroot, "polyspec", "tspec_template.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["refpolyspec.tspec_template"] = mod
    spec.loader.exec_module(mod)
    ref["tspec_template"] = mod
    return ref


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PS_REFERENCE_ROOT", "")
    if not refroot:
        sys.exit("usage: %s <reference checkout> (or set PS_REFERENCE_ROOT)" % sys.argv[0])
    ref = load_reference(refroot)
    for pol in (False, True):
        d = make(pol, ref)
        path = os.path.join(HERE, "tspec_nside16_%s.npz" % ("teb" if pol else "t"))
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
