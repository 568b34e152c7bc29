"""Generate the direction-dependent tauNL fixtures (P_{n,mu} maps; the tauNL-direc:1,1,0 and
tauNL-direc:2,2,0 numerators and Fisher contribution) of tests/golden from the
UNMODIFIED reference.

    python tests/golden/make_golden_tspec_gaunt.py [/path/to/reference]

Builds polyspec/tspec_template.py's TSpecTemplate as-is with the templates
tauNL-direc:1,1,0 and tauNL-direc:2,2,0 over the oracle shims of make_golden_tspec.py
(so p_lL^X(r) is computed for the shifts -2..2) and saves its p_lL^X(r) integrals
and the filtered maps P_{n,mu} (n = 1, 2; 0 <= mu <= n) of the S^-1-filtered data
(_compute_weighted_gaunt_maps, whose Gaunt coefficients come from the reference's
compiled wignerSymbols), the q_l^X(r) and F_L(r, r') integrals, the numerator with and
without the disconnected terms (one simulation pair) and compute_fisher_contribution(1),
for T only and for T, E, B.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden_tspec as mgt  # noqa: E402  (installs the numpy / scipy aliases)
from make_golden import inputs, NSIDE  # noqa: E402

TEMPLATES = ['tauNL-direc:1,1,0', 'tauNL-direc:2,2,0']
LMIN, LMAX = mgt.LMIN, mgt.LMAX


def make(pol, ref):
    base_mod, wt_mod, ts_mod = ref["base"], ref["weighting"], ref["tspec_template"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    base = base_mod.PolySpec(NSIDE, dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="ducc",
                             nthreads=2)
    wts = wt_mod.Weightings(base, mask, dict(cl), noise_cov=noise)
    ideal = lambda x, input_type="map", lmax=None: wts.applySinv_ideal(x * mask if input_type == "map" else x,
                                                                          input_type=input_type, lmax=lmax)
    k_arr = np.geomspace(1e-4, 0.12, 160)
    Tl = mgt.transfer(pol, k_arr, lmax + 1)
    rng = np.random.default_rng(29)
    r_values = np.linspace(13300., 14400., 6)
    r_weights = {t: rng.uniform(0.5, 1.5, 6) * 200. for t in TEMPLATES}
    tst = ts_mod.TSpecTemplate(base, mask, ideal, list(TEMPLATES), k_arr, Tl, LMIN, LMAX, r_values=r_values,
                               r_weights=r_weights)
    data = base.to_map(base.generate_data(seed=5, output_type="harmonic"))
    h = np.asarray(tst.applySinv(data, input_type='map', lmax=tst.lmax)[:, tst.lminfilt], order='C')
    out = {"plLXs": tst.plLXs, "h_filt": h, "qlXs": tst.qlXs, "FLLs": tst.FLLs, "data": data,
           "r_values": r_values, "k_arr": k_arr, "Tl_arr": Tl, "templates": np.asarray(TEMPLATES)}
    for t, w in r_weights.items():
        out["r_weights_" + t] = w
    for n in (1, 2):
        for mu in range(n + 1):
            out["p%d%d" % (n, mu)] = tst._compute_weighted_gaunt_maps(h, tst.plLXs, n, mu)
    tst.generate_sims(1)
    out["tl_num_4"] = tst.Tl_numerator(data, include_disconnected_term=False)
    out["tl_num_full"] = tst.Tl_numerator(data, include_disconnected_term=True)
    out["fisher_seed1"] = tst.compute_fisher_contribution(1)
    return out


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PS_REFERENCE_ROOT", "")
    if not refroot:
        sys.exit("usage: %s <reference checkout> (or set PS_REFERENCE_ROOT)" % sys.argv[0])
    ref = mgt.load_reference(refroot)
    for pol in (False, True):
        d = make(pol, ref)
        path = os.path.join(HERE, "tspec_gaunt_nside16_%s.npz" % ("teb" if pol else "t"))
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
