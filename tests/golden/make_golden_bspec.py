"""Generate the BSpecBin golden fixtures of tests/golden from the UNMODIFIED reference.

    python tests/golden/make_golden_bspec.py [/path/to/reference]

Runs polyspec/bspec_bin.py of the reference as-is over the oracle shims (ducc0's
SHTs are the FP64 restatement of oracle/sht_oracle.cpp; healpy and pywigxjpf
are import-time stand-ins).  One compatibility alias is installed first: the
reference calls ``np.product``, which numpy 2 removed; it is bound to
``np.prod`` (the same function under its current name).

Fixtures (Nside 16, lmax = 3 Nside - 1, ideal S^-1 filter = mask, then the
harmonic C^-1 and the beam):
  * the bin list (``all_bins``) and symmetry factors;
  * ``Bl_numerator`` of a seeded data map, cubic term alone and with the linear
    term over two generated simulations;
  * ``Bl_numerator_ideal`` of the same map;
  * ``compute_fisher_contribution(seed=1)``;
for temperature only (TTT) and for T, E, B with all ten field triplets and both
parities.  The GRF harmonics the Fisher contribution draws internally are saved
too, so a test can check the draw separately from the estimator.

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

ALL_FIELDS = ['TTT', 'TTE', 'TEE', 'EEE', 'TBB', 'EBB', 'TTB', 'TEB', 'EEB', 'BBB']


def make(pol, ref, l_bins, fields, parity):
    base_mod, wt_mod, bs_mod = ref["base"], ref["weighting"], ref["bspec_bin"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    nf = 3 if pol else 1
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
    bsb = bs_mod.BSpecBin(base, mask[0], ideal, np.asarray(l_bins), fields=list(fields), parity=parity)
    bsb._compute_symmetry_factor()
    out["all_bins"] = np.asarray(bsb.all_bins)
    out["sym_factor"] = np.asarray(bsb.sym_factor)
    out["bl_num_cubic"] = bsb.Bl_numerator(data, include_linear_term=False)
    bsb.generate_sims(2)
    out["bl_num_full"] = bsb.Bl_numerator(data, include_linear_term=True)
    out["bl_num_ideal"] = bsb.Bl_numerator_ideal(data)
    out["fisher_seed1"] = bsb.compute_fisher_contribution(1)
    out["fisher_grf_a0"] = base.generate_data(seed=1 + int(1e8), deconvolve_beam=True, output_type="harmonic")
    out["fisher_grf_a1"] = base.generate_data(seed=1 + int(2e8), deconvolve_beam=True, output_type="harmonic")
    return out


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PS_REFERENCE_ROOT", "")
    if not refroot:
        sys.exit("usage: %s <reference checkout> (or set PS_REFERENCE_ROOT)" % sys.argv[0])
    ref = reference_harness.load(refroot, modules=("base", "weighting", "bspec_bin"))
    cases = [
        (False, [2, 6, 10, 16, 23], ['TTT'], 'even', "bspec_nside16_t.npz"),
        (True, [2, 7, 13, 23], ALL_FIELDS, 'both', "bspec_nside16_teb.npz"),
    ]
    for pol, l_bins, fields, parity, name in cases:
        d = make(pol, ref, l_bins, fields, parity)
        path = os.path.join(HERE, name)
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes", "N_b", len(d["sym_factor"]))


if __name__ == "__main__":
    main()
