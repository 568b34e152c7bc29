"""Generate the general direction-dependent tauNL fixtures (n > 0 or n1 != n3, and the
tauNL-even / tauNL-odd combinations) of tests/golden from the UNMODIFIED reference.

    python tests/golden/make_golden_tspec_direc.py [/path/to/reference]

Builds polyspec/tspec_template.py's TSpecTemplate as-is, once with the templates
tauNL-direc:1,1,2, tauNL-direc:1,2,1 and tauNL-direc:0,1,1 (tspec_direc_*) and once with
tauNL-even:0, tauNL-even:1 and tauNL-odd:1 (tspec_evenodd_*; the odd weights use the shim's
exact 6j symbols), over the oracle shims of make_golden_tspec.py (with 2 <= L <= 40) and saves its q_l^X(r), p_lL^X(r) and F_{L,L+Delta}(r, r') integrals,
the numerator with and without the disconnected terms (one simulation pair) and
compute_fisher_contribution(1), for T only and for T, E, B.  These exercise the reference's
tau_sum_general and convolve_F_general (tauNL_utils.pyx:650-715, :1069-1190), the n1 != n3
symmetrisation of the Fisher derivative and its n1 = 0 / n3 = 0 rows.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden_tspec as mgt  # noqa: E402  (installs the numpy / scipy aliases)
from make_golden import inputs, NSIDE  # noqa: E402

TEMPLATE_SETS = {"direc": ['tauNL-direc:1,1,2', 'tauNL-direc:1,2,1', 'tauNL-direc:0,1,1'],
                 "evenodd": ['tauNL-even:0', 'tauNL-even:1', 'tauNL-odd:1']}
LMIN, LMAX = mgt.LMIN, mgt.LMAX
# L range of the exchanged momentum: L_MAX + max(n) must stay within the maps' lmax (3 Nside - 1)
L_MIN, L_MAX = 2, 40


def make(pol, ref, TEMPLATES):
    base_mod, wt_mod, ts_mod = ref["base"], ref["weighting"], ref["tspec_template"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    base = base_mod.PolySpec(NSIDE, dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="ducc",
                             nthreads=2)
    wts = wt_mod.Weightings(base, mask, dict(cl), noise_cov=noise)
    ideal = lambda x, input_type="map", lmax=None: wts.applySinv_ideal(x * mask if input_type == "map" else x,
                                                                          input_type=input_type, lmax=lmax)
    k_arr = np.geomspace(1e-4, 0.12, 160)
    Tl = mgt.transfer(pol, k_arr, lmax + 1)
    rng = np.random.default_rng(31)
    r_values = np.linspace(13300., 14400., 5)
    r_weights = {t: rng.uniform(0.5, 1.5, 5) * 200. for t in TEMPLATES}
    tst = ts_mod.TSpecTemplate(base, mask, ideal, list(TEMPLATES), k_arr, Tl, LMIN, LMAX, r_values=r_values,
                               r_weights=r_weights, Lmin=L_MIN, Lmax=L_MAX)
    data = base.to_map(base.generate_data(seed=7, output_type="harmonic"))
    out = {"plLXs": tst.plLXs, "qlXs": tst.qlXs, "FLLs": tst.FLLs, "data": data, "r_values": r_values,
           "k_arr": k_arr, "Tl_arr": Tl, "templates": np.asarray(TEMPLATES)}
    for t, w in r_weights.items():
        out["r_weights_" + t] = w
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
    for name, templates in TEMPLATE_SETS.items():
        for pol in (False, True):
            d = make(pol, ref, templates)
            path = os.path.join(HERE, "tspec_%s_nside16_%s.npz" % (name, "teb" if pol else "t"))
            np.savez_compressed(path, **d)
            print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
