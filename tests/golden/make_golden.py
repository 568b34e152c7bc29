"""Generate the golden fixtures of tests/golden from the UNMODIFIED reference.

    python tests/golden/make_golden.py [/path/to/reference]

The reference package (polyspec/base.py, weighting.py, pspec_bin.py) is run
as-is; the third-party modules it imports and that are absent here (ducc0,
healpy, pywigxjpf) are the oracle shims under oracle/shims (ducc0's SHTs are
the FP64 restatement of oracle/sht_oracle.cpp).  The fixtures pin the product
against the reference's own wrapper logic (spin conventions, scalings,
recombinations), its S^-1 filters (ideal and conjugate gradient) and its
PSpecBin numerator and Fisher contribution, on seeded small inputs
(Nside 16, lmax = 3 Nside - 1 as the reference fixes it).

Only this script reads the reference checkout; the committed .npz files are
what the tests use.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import reference_harness  # noqa: E402
from polyspec_b200 import workloads as W  # noqa: E402

NSIDE = 16


def rand_alm(rng, lmax, lead):
    l = np.concatenate([np.arange(mm, lmax + 1) for mm in range(lmax + 1)])
    m = np.concatenate([np.full(lmax + 1 - mm, mm) for mm in range(lmax + 1)])
    a = rng.normal(size=lead + (len(l),)) + 1j * rng.normal(size=lead + (len(l),))
    a[..., m == 0] = a[..., m == 0].real
    return a


def inputs(pol):
    lmax = 3 * NSIDE - 1
    cl = W.fiducial_cl(lmax, pol)
    beam1 = W.gaussian_beam(lmax, 120.0)
    nl = W.noise_cl(NSIDE, lmax, 30.0, pol)
    beam = np.stack([beam1] * (3 if pol else 1))
    cltot = W.total_cl(cl, beam, nl)
    nf = 3 if pol else 1
    mask = np.stack([W.latitude_mask(NSIDE, 15.0, 5.0)] * nf)
    noise = W.white_noise_cov(NSIDE, 30.0, pol)
    return lmax, cl, beam, cltot, mask, noise


def make(pol, ref):
    base_mod, wt_mod, ps_mod = ref["base"], ref["weighting"], ref["pspec_bin"]
    lmax, cl, beam, cltot, mask, noise = inputs(pol)
    nf = 3 if pol else 1
    out = {"nside": NSIDE, "lmax": lmax, "pol": int(pol), "mask": mask, "noise": noise, "beam": beam}
    for k, v in cltot.items():
        out["cltot_" + k] = v
    for k, v in cl.items():
        out["clraw_" + k] = v
    base = base_mod.PolySpec(NSIDE, dict(cltot), beam=list(beam) if pol else beam[:1], pol=pol, backend="ducc",
                             nthreads=2)
    rng = np.random.default_rng(7 + pol)
    npix = 12 * NSIDE ** 2
    # ---- SHT wrappers
    alm = rand_alm(rng, lmax, (nf,))
    out["in_alm"] = alm
    out["to_map"] = base.to_map(alm)
    mp = rng.normal(size=(nf, npix))
    out["in_map"] = mp
    out["to_lm"] = base.to_lm(mp)
    for s in (1, 2, 3):
        ap, am = rand_alm(rng, lmax, (2,))
        out["in_spin%d_alm" % s] = np.stack([ap, am])
        p, mi = base.to_map_spin(ap, am, s)
        out["to_map_spin%d" % s] = np.stack([p, mi])
        mpp = rng.normal(size=npix) + 1j * rng.normal(size=npix)
        mpm = np.conj(mpp)
        out["in_spin%d_map" % s] = np.stack([mpp, mpm])
        out["to_lm_spin%d" % s] = base.to_lm_spin(mpp, mpm, s)
    vec = rand_alm(rng, lmax, (3,))
    out["in_vec_alm"] = vec
    out["to_map_vec0"] = base.to_map_vec(vec)
    out["to_map_vec1"] = base.to_map_vec(vec, output_spin=1)
    out["to_map_vec2"] = base.to_map_vec(vec, output_spin=2)
    vmap = rng.normal(size=(3, npix))
    out["in_vec_map"] = vmap
    out["to_lm_vec0"] = base.to_lm_vec(vmap)
    out["spin_transform_p1"] = np.asarray(base.compute_spin_transform_map([vec[0]], 1))
    out["spin_transform_m2"] = np.asarray(base.compute_spin_transform_map([vec[1]], -2))
    out["applyAinv"] = base.applyAinv(alm, input_type="harmonic")

    # ---- S^-1 filters
    wts = wt_mod.Weightings(base, mask, dict(cl), noise_cov=noise)
    data = base.to_map(base.generate_data(seed=3, output_type="harmonic"))
    out["data"] = data
    out["sinv_ideal"] = wts.applySinv_ideal(data * mask)
    for pre in ("harmonic", "pseudo_inverse"):
        out["sinv_opt_%s" % pre] = wts.applySinv_optimal(data, preconditioner=pre, nstep=12, thresh=0.0)
    # CG test mode: b = A x for a known x
    xk = rand_alm(rng, lmax, (nf,))
    cg = wt_mod.CGD(wts, [], test_b=wt_mod.CGD(wts, data, preconditioner="harmonic")._apply_A(xk),
                    preconditioner="harmonic")
    cg.run(nstep=60, thresh=1e-20)
    out["cg_test_x"] = xk
    out["cg_test_sol"] = cg.x

    # ---- PSpecBin
    fields = ["TT", "TE", "EE", "BB"] if pol else ["TT"]
    l_bins = np.array([2, 6, 10, 14, 18, 22])
    out["l_bins"] = l_bins
    ideal = lambda x, input_type="map", lmax=None: wts.applySinv_ideal(x * mask if input_type == "map" else x,
                                                                          input_type=input_type, lmax=lmax)
    psb = ps_mod.PSpecBin(base, mask, ideal, l_bins, fields=fields)
    out["cl_num_ideal_filter"] = psb.Cl_numerator(data)
    out["fisher_ideal_filter_seed1"] = psb.compute_fisher_contribution(1)
    out["grf_seed1"] = base.generate_data(seed=1 + int(1e7), output_type="harmonic", deconvolve_beam=True)
    out["grf_seed2"] = base.generate_data(seed=2 + int(1e7), output_type="harmonic", deconvolve_beam=True)
    opt = lambda x, input_type="map", lmax=None: wts.applySinv_optimal(x, preconditioner="harmonic", nstep=8,
                                                                        thresh=0.0, lmax=lmax)
    psb2 = ps_mod.PSpecBin(base, mask, opt, l_bins, fields=fields)
    out["fisher_opt_filter_seed2"] = psb2.compute_fisher_contribution(2)
    out["fisher_ideal_analytic"] = psb.compute_fisher_ideal()
    out["cl_num_ideal"] = psb.Cl_numerator_ideal(data)
    return out


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PS_REFERENCE_ROOT", "")
    if not refroot:
        sys.exit("usage: %s <reference checkout> (or set PS_REFERENCE_ROOT)" % sys.argv[0])
    ref = reference_harness.load(refroot)
    for pol in (False, True):
        d = make(pol, ref)
        path = os.path.join(HERE, "pspec_nside16_%s.npz" % ("teb" if pol else "t"))
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
