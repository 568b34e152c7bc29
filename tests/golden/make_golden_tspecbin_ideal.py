"""Generate the ideal TSpecBin numerator fixtures of tests/golden from the UNMODIFIED
reference.

    python tests/golden/make_golden_tspecbin_ideal.py [/path/to/reference]

Runs TSpecBin.Tl_numerator_ideal of polyspec/tspec_bin.py as-is over the oracle
shims, on the two cases of make_golden_tspecbin.py, without and with the 0- and
2-field terms (whose 3j symbols come from the exact-3j pywigxjpf stand-in
oracle/shims/pywigxjpf).  The inputs are those of tspecbin_nside16_*.npz.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden_tspecbin as mgt  # noqa: E402  (installs the numpy alias)
from make_golden import inputs, NSIDE  # noqa: E402


def make(pol, ref, l_bins, fields, parity):
    base_mod, ts_mod = ref["base"], ref["tspec_bin"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    base = base_mod.PolySpec(NSIDE, dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="ducc",
                             nthreads=2)
    data = base.to_map(base.generate_data(seed=5, output_type="harmonic"))
    tsb = ts_mod.TSpecBin(base, mask[0], None, np.asarray(l_bins), fields=list(fields), parity=parity)
    out = {"tl_num_ideal_4": tsb.Tl_numerator_ideal(data, include_disconnected_term=False, N_cpus=1)}
    out["tl_num_ideal_full"] = tsb.Tl_numerator_ideal(data, include_disconnected_term=True, N_cpus=1)
    return out


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PS_REFERENCE_ROOT", "")
    if not refroot:
        sys.exit("usage: %s <reference checkout> (or set PS_REFERENCE_ROOT)" % sys.argv[0])
    ref = mgt.reference_harness.load(refroot, modules=("base", "weighting", "tspec_bin"))
    for pol, l_bins, fields, parity, name in mgt.CASES:
        d = make(pol, ref, l_bins, fields, parity)
        path = os.path.join(HERE, name.replace("tspecbin_", "tspecbin_ideal_"))
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
