"""Generate the TSpecTemplate golden fixtures for the gNL-con template and the three
EFTI shapes (gNL-dotdot, gNL-dotdel, gNL-deldel) from the UNMODIFIED reference.

    python tests/golden/make_golden_tspec_efti.py [/path/to/reference]

Runs polyspec/tspec_template.py of the reference as-is over the same oracle shims
as make_golden_tspec.py (FP64 restatement of ducc0's SHTs, the reference's own
tauNL_utils compiled by oracle/build_ref.sh, and the numpy restatement
oracle/shims/k_integrals.py of k_integrals, which now includes the r, a, b, c
integrals and j_l').

Inputs: those of make_golden_tspec.py (Nside 16, l in [2, 30], seeded transfer
functions on 160 log-spaced k), 6 radial points for gNL-con and a 3 x 3 grid of
(r, tau) points (r in [13400, 14200] Mpc, tau in [-2000, -50] Mpc) for the EFTI
shapes, each with seeded weights per template.

Fixtures: the r_l^X(r), a_l^X(r,tau), b_l^X(r,tau), c_l^X(r,tau) integrals, the
data's filtered maps r, a, b, c, the numerator with and without the disconnected
terms (one simulation pair), and compute_fisher_contribution(seed=1), for T only
and for T, E, B.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden_tspec as mgt  # noqa: E402  (installs the numpy / scipy aliases)
from make_golden import inputs, NSIDE  # noqa: E402

TEMPLATES = ['gNL-con', 'gNL-dotdot', 'gNL-dotdel', 'gNL-deldel']
LMIN, LMAX = mgt.LMIN, mgt.LMAX


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
    Tl = mgt.transfer(pol, k_arr, lmax + 1)
    rng = np.random.default_rng(17)
    r_values = np.linspace(13300., 14400., 6)
    r_weights = {'gNL-con': rng.uniform(0.5, 1.5, 6) * 200.}
    rr, tt = np.meshgrid(np.linspace(13400., 14200., 3), -np.geomspace(50., 2000., 3), indexing='ij')
    rtau_values = np.stack([rr.ravel(), tt.ravel()], axis=1)
    rtau_weights = {t: rng.uniform(0.5, 1.5, len(rtau_values)) * 100. for t in TEMPLATES[1:]}
    out.update(k_arr=k_arr, Tl_arr=Tl, r_values=r_values, rtau_values=rtau_values,
               r_weights_gNL_con=r_weights['gNL-con'])
    for t, w in rtau_weights.items():
        out["rtau_weights_" + t.replace('-', '_')] = w
    tst = ts_mod.TSpecTemplate(base, mask, ideal, list(TEMPLATES), k_arr, Tl, LMIN, LMAX, r_values=r_values,
                               r_weights=r_weights, rtau_values=rtau_values, rtau_weights=rtau_weights)
    for k in ("rlXs", "alXs", "blXs", "clXs"):
        out[k] = getattr(tst, k)
    data = base.to_map(base.generate_data(seed=5, output_type="harmonic"))
    out["data"] = data
    h = np.asarray(tst.applySinv(data, input_type='map', lmax=tst.lmax)[:, tst.lminfilt], order='C')
    proc = tst._apply_all_filters(h)
    for k in ('r', 'a', 'b', 'c'):
        out["proc_" + k] = proc[k]
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
        path = os.path.join(HERE, "tspec_efti_nside16_%s.npz" % ("teb" if pol else "t"))
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
