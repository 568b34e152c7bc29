"""The numpy restatement of the reference's S^-1 / PSpecBin path (oracle/polyspec_port.py)
against the fixtures the unmodified reference produced (tests/golden)."""
import os

import numpy as np
import pytest

from oracle import polyspec_port as P

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(x, ref):
    return np.abs(np.asarray(x) - np.asarray(ref)).max() / np.abs(np.asarray(ref)).max()


@pytest.mark.parametrize("pol", [False, True])
def test_port_matches_reference_fixtures(pol):
    d = dict(np.load(os.path.join(GOLD, "pspec_nside16_%s.npz" % ("teb" if pol else "t"))))
    cltot = {k[6:]: d[k] for k in d if k.startswith("cltot_")}
    clraw = {k[6:]: d[k] for k in d if k.startswith("clraw_")}
    base = P.PortBase(int(d["nside"]), cltot, d["beam"], pol=pol, nthreads=2)
    W = P.PortWeightings(base, d["mask"], clraw, d["noise"])
    assert rel(base.to_map(d["in_alm"]), d["to_map"]) < 1e-13
    assert rel(base.to_lm(d["in_map"]), d["to_lm"]) < 1e-13
    assert rel(base.applyAinv(d["in_alm"]), d["applyAinv"]) < 1e-13
    assert rel(W.applySinv_ideal(d["data"] * d["mask"]), d["sinv_ideal"]) < 1e-13
    for pre in ("harmonic", "pseudo_inverse"):
        assert rel(W.applySinv_optimal(d["data"], pre, nstep=12, thresh=0.0), d["sinv_opt_%s" % pre]) < 1e-11
    assert rel(base.generate_data(1 + int(1e7)), d["grf_seed1"]) < 1e-14
    fields = ["TT", "TE", "EE", "BB"] if pol else ["TT"]
    ideal = P.PortPSpecBin(base, d["mask"], lambda x: W.applySinv_ideal(x * d["mask"]), d["l_bins"], fields)
    assert rel(ideal.Cl_numerator(d["data"]), d["cl_num_ideal_filter"]) < 1e-12
    assert rel(ideal.compute_fisher_contribution(1), d["fisher_ideal_filter_seed1"]) < 1e-12
    opt = P.PortPSpecBin(base, d["mask"], lambda x: W.applySinv_optimal(x, "harmonic", nstep=8, thresh=0.0),
                         d["l_bins"], fields)
    assert rel(opt.compute_fisher_contribution(2), d["fisher_opt_filter_seed2"]) < 1e-11
