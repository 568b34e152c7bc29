"""Generate the TSpecBin golden fixtures of tests/golden from the UNMODIFIED reference.

    python tests/golden/make_golden_tspecbin.py [/path/to/reference]

Runs polyspec/tspec_bin.py of the reference as-is over the oracle shims (ducc0's
SHTs are the FP64 restatement of oracle/sht_oracle.cpp; healpy and pywigxjpf are
import-time stand-ins: the optimal estimator uses no Wigner symbols), with the
numpy 2 alias ``np.product`` -> ``np.prod``.

Fixtures (Nside 16, lmax = 3 Nside - 1, ideal S^-1 filter = mask, then the
harmonic C^-1 and the beam): symmetry factors, ``Tl_numerator`` of a seeded data
map without and with the disconnected terms (one simulation pair) and
``compute_fisher_contribution(seed=1)``, for temperature only (TTTT) and for a
set of T, E, B field quadruplets with both parities.

Only this script reads the reference checkout; the committed .npz files are
what the tests use.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

if not hasattr(np, "product"):
    np.product = np.prod

from oracle import reference_harness  # noqa: E402
from make_golden import inputs, NSIDE  # noqa: E402

POL_FIELDS = ['TTTT', 'TTTE', 'TTEE', 'TETE', 'TEEE', 'EEEE', 'TTBB', 'TBTB', 'TTTB', 'TEEB']


def make(pol, ref, l_bins, fields, parity):
    base_mod, wt_mod, ts_mod = ref["base"], ref["weighting"], ref["tspec_bin"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    out = {"nside": NSIDE, "lmax": lmax, "pol": int(pol), "mask": mask, "noise": noise, "beam": beam,
           "l_bins": np.asarray(l_bins), "fields": np.asarray(fields), "parity": parity}
    for k, v in cltot.items():
        out["cltot_" + k] = v
    for k, v in cl.items():
        out["clraw_" + k] = v
    base = base_mod.PolySpec(NSIDE, dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="ducc",
                             nthreads=2)
    wts = wt_mod.Weightings(base, mask, dict(cl), noise_cov=noise)
    ideal = lambda x, input_type="map", lmax=None: wts.applySinv_ideal(x * mask if input_type == "map" else x,
                                                                          input_type=input_type, lmax=lmax)
    data = base.to_map(base.generate_data(seed=5, output_type="harmonic"))
    out["data"] = data
    tsb = ts_mod.TSpecBin(base, mask[0], ideal, np.asarray(l_bins), fields=list(fields), parity=parity)
    tsb._compute_symmetry_factor()
    out["sym_factor"] = np.asarray(tsb.sym_factor)
    out["tl_num_4"] = tsb.Tl_numerator(data, include_disconnected_term=False)
    tsb.generate_sims(1)
    out["tl_num_full"] = tsb.Tl_numerator(data, include_disconnected_term=True)
    out["fisher_seed1"] = tsb.compute_fisher_contribution(1)
    return out


CASES = [
    (False, [2, 8, 14, 23], ['TTTT'], 'even', "tspecbin_nside16_t.npz"),
    (True, [2, 10, 23], POL_FIELDS, 'both', "tspecbin_nside16_teb.npz"),
]


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PS_REFERENCE_ROOT", "")
    if not refroot:
        sys.exit("usage: %s <reference checkout> (or set PS_REFERENCE_ROOT)" % sys.argv[0])
    ref = reference_harness.load(refroot, modules=("base", "weighting", "tspec_bin"))
    for pol, l_bins, fields, parity, name in CASES:
        d = make(pol, ref, l_bins, fields, parity)
        path = os.path.join(HERE, name)
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes", "N_t", len(d["sym_factor"]))


if __name__ == "__main__":
    main()
