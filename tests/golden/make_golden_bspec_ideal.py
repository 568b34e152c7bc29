"""Generate the ideal BSpecBin Fisher fixtures of tests/golden from the UNMODIFIED
reference.

    python tests/golden/make_golden_bspec_ideal.py [/path/to/reference]

Runs BSpecBin.compute_fisher_ideal of polyspec/bspec_bin.py as-is over the oracle
shims, on the two cases of make_golden_bspec.py (TTT with even parity; the ten
T, E, B triplets with both parities).  Its Wigner 3j symbols come from the
pywigxjpf stand-in oracle/shims/pywigxjpf (exact Racah sums).  The fixtures hold
the ideal Fisher matrix only; the inputs are those of bspec_nside16_*.npz.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden_bspec as mgb  # noqa: E402  (installs the numpy alias)
from make_golden import inputs, NSIDE  # noqa: E402


def make(pol, ref, l_bins, fields, parity):
    base_mod, bs_mod = ref["base"], ref["bspec_bin"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    base = base_mod.PolySpec(NSIDE, dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="ducc",
                             nthreads=2)
    bsb = bs_mod.BSpecBin(base, mask[0], None, np.asarray(l_bins), fields=list(fields), parity=parity)
    return {"fisher_ideal": bsb.compute_fisher_ideal(N_cpus=1)}


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PS_REFERENCE_ROOT", "")
    if not refroot:
        sys.exit("usage: %s <reference checkout> (or set PS_REFERENCE_ROOT)" % sys.argv[0])
    ref = mgb.reference_harness.load(refroot, modules=("base", "weighting", "bspec_bin"))
    cases = [
        (False, [2, 6, 10, 16, 23], ['TTT'], 'even', "bspec_ideal_nside16_t.npz"),
        (True, [2, 7, 13, 23], mgb.ALL_FIELDS, 'both', "bspec_ideal_nside16_teb.npz"),
    ]
    for pol, l_bins, fields, parity, name in cases:
        d = make(pol, ref, l_bins, fields, parity)
        path = os.path.join(HERE, name)
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes", d["fisher_ideal"].shape)


if __name__ == "__main__":
    main()
