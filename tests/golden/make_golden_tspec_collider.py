"""Generate the collider tauNL fixtures (tauNL-light:s,nu_s and tauNL-heavy:s,mu_s) of
tests/golden from the UNMODIFIED reference.

    python tests/golden/make_golden_tspec_collider.py [/path/to/reference]

Builds polyspec/tspec_template.py's TSpecTemplate as-is with the templates
tauNL-light:0,0.7 (s = 0, real beta: tau_sum_n0_collider), tauNL-light:1,0.3 (s = 1,
real beta: tau_sum_general_collider), tauNL-light:1,0.0 (nu_s = 0: tau_sum_nu0_collider),
tauNL-heavy:0,0.5 (s = 0, complex beta) and tauNL-heavy:1,0.8 (s = 1, complex beta, with
the m -> -m piece), over the oracle shims of make_golden_tspec.py (2 <= L <= 40,
k_coll = K_coll = 0.01 so that the collider integrals see many k points).  It saves the
collider p^beta_lL^X(r) and F^beta_{L,L+n}(r, r') integrals (oracle/shims/k_integrals.py
restates k_integrals.pyx:399-545), the numerator with and without the disconnected
terms (one simulation pair) and compute_fisher_contribution(1), for T only and for
T, E, B.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden_tspec as mgt  # noqa: E402  (installs the numpy / scipy aliases)
from make_golden import inputs, NSIDE  # noqa: E402

TEMPLATES = ['tauNL-light:0,0.7', 'tauNL-light:1,0.3', 'tauNL-light:1,0.0', 'tauNL-heavy:0,0.5',
             'tauNL-heavy:1,0.8']
LMIN, LMAX = mgt.LMIN, mgt.LMAX
L_MIN, L_MAX = 2, 40
K_COLL = 0.01


def beta_key(beta):
    return "%.8f,%.8f" % (np.real(beta), np.imag(beta))


def make(pol, ref, with_fisher=True):
    base_mod, wt_mod, ts_mod = ref["base"], ref["weighting"], ref["tspec_template"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    base = base_mod.PolySpec(NSIDE, dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="ducc",
                             nthreads=2)
    wts = wt_mod.Weightings(base, mask, dict(cl), noise_cov=noise)
    ideal = lambda x, input_type="map", lmax=None: wts.applySinv_ideal(x * mask if input_type == "map" else x,
                                                                          input_type=input_type, lmax=lmax)
    k_arr = np.geomspace(1e-4, 0.12, 160)
    Tl = mgt.transfer(pol, k_arr, lmax + 1)
    rng = np.random.default_rng(37)
    r_values = np.linspace(13300., 14400., 5)
    r_weights = {t: rng.uniform(0.5, 1.5, 5) * 200. for t in TEMPLATES}
    tst = ts_mod.TSpecTemplate(base, mask, ideal, list(TEMPLATES), k_arr, Tl, LMIN, LMAX, r_values=r_values,
                               r_weights=r_weights, Lmin=L_MIN, Lmax=L_MAX, K_coll=K_COLL, k_coll=K_COLL)
    data = base.to_map(base.generate_data(seed=11, output_type="harmonic"))
    out = {"qlXs": tst.qlXs, "data": data, "r_values": r_values, "k_arr": k_arr, "Tl_arr": Tl,
           "templates": np.asarray(TEMPLATES)}
    for beta, arr in tst.coll_plLXs.items():
        out["coll_plLXs_" + beta_key(beta)] = arr
    for beta, arr in tst.coll_FLLs.items():
        out["coll_FLLs_" + beta_key(beta)] = arr
    for t, w in r_weights.items():
        out["r_weights_" + t] = w
    tst.generate_sims(1)
    out["tl_num_4"] = tst.Tl_numerator(data, include_disconnected_term=False)
    out["tl_num_full"] = tst.Tl_numerator(data, include_disconnected_term=True)
    if with_fisher:
        out["fisher_seed1"] = tst.compute_fisher_contribution(1)
    return out


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PS_REFERENCE_ROOT", "")
    if not refroot:
        sys.exit("usage: %s <reference checkout> (or set PS_REFERENCE_ROOT)" % sys.argv[0])
    ref = mgt.load_reference(refroot)
    for pol in (False, True):
        d = make(pol, ref)
        path = os.path.join(HERE, "tspec_collider_nside16_%s.npz" % ("teb" if pol else "t"))
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
