"""Small fixed workloads for profiling the kernels under ncu.

    python -m polyspec_b200.profile_cli sht --nside 1024 --lmax 2048 --ops s0,a0,s2,a2 [--batch 1] [--tables on]

Each op runs once (no warm-up) so that a launch list or an ncu capture of
``-k <kernel> -c 1`` sees exactly one launch per transform stage.
ops: s0/a0 = spin-0 synthesis/adjoint, s2/a2 = spin-2 synthesis/adjoint; only the
spins of the ops are planned (and, for a mixed plan, tabulated).

    python -m polyspec_b200.profile_cli pix --nside 512 --nr 24 [--reps 3]

runs the pixel-product / radial-sum kernels on [nr, Npix] maps (config-3
sizes by default) and prints each one's device time and achieved HBM GB/s
(algorithmic bytes / CUDA-event time, best of --reps).

    python -m polyspec_b200.profile_cli serve --n 64 [--reps 3] [--prec mixed]

the mixed-size serving workload (n = 64 keeps the FP64 maps and alm of all
requests, about 15 GB per 16 requests, well inside HBM): n requests with Nside drawn uniformly from
{256, 512, 1024, 2048}, lmax = 2 Nside, spin 0 or 2, half alm2map and half
map2alm (seeded), grouped and replayed as one CUDA graph; prints maps/s
(requests per second, both directions counted).

    python -m polyspec_b200.profile_cli bspec [--nside 256 --lmax 511 --nbins 10] [--precs fp64,mixed]

one binned-bispectrum Fisher contribution (T+E, log bins, both parities, ideal
S^-1 filter) per precision: device time, kernel time per kind, the numerator
with two simulations, and the mixed-vs-FP64 Fisher difference.

    python -m polyspec_b200.profile_cli tspecbin [--nside 128 --lmax 255 --nbins 6]
    python -m polyspec_b200.profile_cli tspec [--nside 512 --lmax 1000 --nr 24 --templates gNL-loc,...
                                               --K-coll 0.1]

the binned trispectrum (T+E) and the template trispectrum (gNL-loc, lensing,
point source): Fisher contribution and numerator times, FP64 and mixed.

    python -m polyspec_b200.profile_cli inpaint [--nside 1024 --holes 2000 --layers 2]

inpainting of a T, Q, U map: --holes seeded point-source holes grown by --layers
neighbour rings, fill passes plus 50 smoothing passes; prints the neighbour-table
build time and the inpaint_map time.

    python -m polyspec_b200.profile_cli tauconv [--Lmax 600 --nr 24 --n1 1 --n3 2 --n 2 --launches 4]

one direction-dependent tauNL F convolution (tauNL_utils.convolve_F_general, mu1 = 0) over the
(L, M) rows with L <= Lmax + 2 and random [P Q] vectors and F: --launches calls, the last timed
with CUDA events (the first three are warm-ups).
"""
import argparse
import re
import sys

import torch


def inpaint(a):
    """Weightings.inpaint_map on a T, Q, U map with seeded point-source holes."""
    import time
    import numpy as np
    from polyspec_b200 import PolySpec, Weightings, healpix
    from polyspec_b200 import workloads as W
    n = a.nside
    npix = 12 * n * n
    dev = torch.device("cuda")
    t0 = time.time()
    nb = healpix.neighbours(n, dev)
    torch.cuda.synchronize()
    t_nb = time.time() - t0
    g = torch.Generator(device=dev).manual_seed(1)
    hole = torch.zeros(npix, dtype=torch.bool, device=dev)
    hole[torch.randint(0, npix, (a.holes,), generator=g, device=dev)] = True
    for _ in range(a.layers):
        idx = nb[hole].flatten().long()
        hole[idx[idx >= 0]] = True
    imask = torch.stack([hole] * 3).to(torch.float64).cpu().numpy()
    lmax = 3 * n - 1
    cl = W.fiducial_cl(lmax, True)
    beam = np.stack([W.gaussian_beam(lmax, 10.)] * 3)
    base = PolySpec(n, dict(W.total_cl(cl, beam, W.noise_cl(n, lmax, 30.0, True))), beam=list(beam), pol=True)
    wts = Weightings(base, np.ones((3, npix)), dict(cl), inpainting_mask=imask)
    m = (1. + torch.randn((3, npix), generator=g, device=dev, dtype=torch.float64)) * (1. - torch.as_tensor(imask,
                                                                                                    device=dev))
    wts.inpaint_map(m)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    wts.inpaint_map(m)
    e1.record()
    torch.cuda.synchronize()
    print("inpaint: Nside %d, %d holes (%d pixels, %.3f%% of the sky): neighbour table %.1f ms (first call); "
          "inpaint_map (T, Q, U; 50 smoothing passes) %.1f ms" % (n, a.holes, int(hole.sum()),
                                                                    100. * float(hole.sum()) / npix, 1e3 * t_nb,
                                                                    e0.elapsed_time(e1)))


def sht(a):
    from polyspec_b200.sht import SHTPlan
    ops = a.ops.split(",")
    spins = sorted({0} | {int(op[1]) for op in ops if op[1:].isdigit()})
    P = SHTPlan(a.nside, a.lmax, spins=spins, prec=a.prec, autotune=False,
                tables={"auto": "auto", "on": True, "off": False}[a.tables])
    B = a.batch
    need0 = any(op in ("s0", "a0") for op in ops)
    need2 = any(op in ("s2", "a2") for op in ops)
    alm0 = torch.randn(B, P.nalm, dtype=torch.complex128, device="cuda") if need0 else None
    map0 = torch.randn(B, P.npix, dtype=torch.float64, device="cuda") if need0 else None
    alm2 = torch.randn(B, 2, P.nalm, dtype=torch.complex128, device="cuda") if need2 else None
    map2 = torch.randn(B, 2, P.npix, dtype=torch.float64, device="cuda") if need2 else None
    for op in ops:
        if op == "s0":
            P.synthesis(alm0, 0)
        elif op == "a0":
            P.adjoint(map0, 0)
        elif op == "s2":
            P.synthesis(alm2, 2)
        elif op == "a2":
            P.adjoint(map2, 2)
        else:
            raise SystemExit("unknown op " + op)
    torch.cuda.synchronize()
    print("done", a.ops, "tables", {s: P.has_table(s) for s in spins} if a.prec != "fp64" else None)


def pix(a):
    from polyspec_b200 import pixel as P
    npix = 12 * a.nside ** 2
    nr = a.nr
    g = torch.Generator(device="cuda").manual_seed(0)
    R = [torch.randn(nr, npix, dtype=torch.float64, device="cuda", generator=g) for _ in range(3)]
    Cx = torch.randn(nr, npix, dtype=torch.complex128, device="cuda", generator=g)
    w = torch.rand(nr, dtype=torch.float64, device="cuda", generator=g)
    t = P.tauNL_utils(1, nr, [0, 1], [0, 0], 0, 1, [0, 1], [0, 0], [0, 1], [0, 0], 1)
    lmax = 2 * a.nside
    nlm = (lmax + 1) * (lmax + 2) // 2
    Q = torch.randn(4, 16, 3 * nlm, dtype=torch.complex128, device="cuda", generator=g)
    n = nr * npix
    cases = [
        ("multiply", lambda: t.multiply(R[0], R[1], R[2]), 32.0 * n),
        ("multiplyRC", lambda: P.multiplyRC(R[0], Cx), 40.0 * n),
        ("multiplyCC", lambda: t.multiplyCC(R[0], R[1], Cx), 40.0 * n),
        ("gnl_loc_sum", lambda: t.gnl_loc_sum(w, R[0], R[1]), 16.0 * n),
        ("gnl_dotdel_sum", lambda: t.gnl_dotdel_sum(w, w, R[0], R[1], Cx), 32.0 * n),
        ("outer_product", lambda: P.outer_product(Q, Q, 0, True), 16.0 * Q.numel()),
    ]
    for name, f, nbytes in cases:
        best = None
        for _ in range(a.reps):
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record()
            f()
            s1.record()
            torch.cuda.synchronize()
            ms = s0.elapsed_time(s1)
            best = ms if best is None else min(best, ms)
        print("%-16s %8.3f ms  %7.1f GB/s (algorithmic %.2f GB)" % (name, best, nbytes / best / 1e6, nbytes / 1e9),
              flush=True)


def serve(a):
    import numpy as np
    from polyspec_b200.serve import SHTServer
    rng = np.random.default_rng(0)
    reqs = []
    for i in range(a.n):
        nside = int(rng.choice([256, 512, 1024, 2048]))
        reqs.append(dict(nside=nside, lmax=2 * nside, spin=int(rng.choice([0, 2])),
                         direction="alm2map" if i % 2 == 0 else "map2alm"))
    srv = SHTServer(reqs, prec=a.prec)
    for x in srv.inputs:
        x.normal_()
    best = None
    for _ in range(a.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        srv.run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    groups = ", ".join("%d x (Nside %d, spin %d, %s)" % (len(idx), k[0], k[2], k[3]) for k, idx in srv.groups)
    print("serve: %d requests in %d groups, graph replay %.1f ms -> %.1f maps/s" % (len(reqs), len(srv.groups), best,
                                                                                  1e3 * len(reqs) / best))
    print("groups:", groups)


def bspec(a):
    """Binned-bispectrum Fisher contributions (T+E, log bins, ideal filter) per second."""
    import numpy as np
    from polyspec_b200 import PolySpec, Weightings, _lib
    from polyspec_b200 import workloads as W
    from polyspec_b200.bspec_bin import BSpecBin
    cltot, cl, beam, mask, l_bins, fields = W.bispec_setup(a.nside, a.lmax, a.nbins)
    res = {}
    for prec in a.precs.split(","):
        base = PolySpec(a.nside, dict(cltot), beam=list(beam), pol=True, lmax=a.lmax, prec=prec)
        wts = Weightings(base, np.stack([mask] * 3), dict(cl), noise_cov=W.white_noise_cov(a.nside))
        bsb = BSpecBin(base, mask, wts.make_applySinv('ideal'), l_bins, fields=fields, parity='both')
        bsb._compute_symmetry_factor()
        if a.numerator_only:
            data = base.to_map(base.generate_data(seed=3, output_type='harmonic', rng='device'))
            bsb.generate_sims(2)
            bsb.Bl_numerator(data)
            torch.cuda.synchronize()
            print("bspec %s numerator done (N_b %d)" % (prec, bsb.N_b), flush=True)
            continue
        a_lms = [base.generate_data(seed=11 + i, deconvolve_beam=True, output_type='harmonic', rng='device')
                 for i in range(2)]
        f = bsb.compute_fisher_contribution(0, a_lms=a_lms)  # warm-up (autotuning, lazy set-up)
        torch.cuda.synchronize()
        best = None
        for _ in range(a.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            f = bsb.compute_fisher_contribution(0, a_lms=a_lms)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        res[prec] = f
        _lib.call("ps_stats_reset")
        _lib.call("ps_stats_enable_timing", 1)
        bsb.compute_fisher_contribution(0, a_lms=a_lms)
        torch.cuda.synchronize()
        _lib.call("ps_stats_enable_timing", 0)
        st = {k: _lib.stats(k) for k in _lib.KERNEL_KINDS}
        print("bspec %s kernel ms: %s" % (prec, ", ".join("%s %.1f" % (k, v[1]) for k, v in st.items() if v[0])))
        data = base.to_map(base.generate_data(seed=3, output_type='harmonic', rng='device'))
        bsb.generate_sims(2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        bsb.Bl_numerator(data)
        e1.record()
        torch.cuda.synchronize()
        print("bspec %s: Nside %d lmax %d, %d bins, N_b %d, %d Q3 pairs: Fisher contribution %.1f ms -> %.3f sims/s;"
              " numerator with 2 sims %.1f ms" % (prec, a.nside, a.lmax, len(l_bins) - 1, bsb.N_b,
                                                  bsb._tables['npair'], best, 1e3 / best, e0.elapsed_time(e1)),
              flush=True)
        del bsb, wts, base
        torch.cuda.empty_cache()
    if "fp64" in res and "mixed" in res:
        r = np.abs(res["mixed"] - res["fp64"]).max() / np.abs(res["fp64"]).max()
        d = np.abs(np.diag(res["mixed"]) / np.diag(res["fp64"]) - 1).max()
        print("bspec mixed vs fp64 Fisher: max rel (of max) %.2e, diagonal max rel %.2e" % (r, d))


def tspec(a):
    """Template trispectrum (--templates, default gNL-loc, lensing, point-source): set-up, numerator and one
    Fisher contribution."""
    import time
    import numpy as np
    from polyspec_b200 import PolySpec, Weightings, _lib
    from polyspec_b200 import workloads as W
    from polyspec_b200.tspec_template import TSpecTemplate
    w = W.tspec_setup(a.nside, a.lmax, a.nr)
    res = {}
    for prec in a.precs.split(","):
        base = PolySpec(a.nside, dict(w['cltot']), beam=list(w['beam']), pol=True, prec=prec)
        wts = Weightings(base, np.stack([w['mask']] * 3), dict(w['cl']), noise_cov=W.white_noise_cov(a.nside))
        t0 = time.time()
        templates = re.split(r",(?=[A-Za-z])", a.templates)  # tauNL-direc:1,1,2 keeps its commas
        r_weights = dict(w['r_weights'])
        for t in templates:  # direction-dependent templates take the tauNL-loc radial weights
            r_weights.setdefault(t, w['r_weights']['tauNL-loc'])
        tst = TSpecTemplate(base, w['mask'], wts.make_applySinv('ideal'), templates,
                            w['k_arr'], w['Tl_arr'], w['lmin'], w['lmax'], r_values=w['r_values'],
                            r_weights=r_weights, rtau_values=w['rtau_values'], rtau_weights=w['rtau_weights'],
                            C_phi=w['C_phi'], C_lens_weight=w['C_lens_weight'], Lmax=a.Lmax,
                            K_coll=a.K_coll, k_coll=a.K_coll)
        torch.cuda.synchronize()
        t_setup = time.time() - t0
        a_lms = [base.generate_data(seed=21 + i, deconvolve_beam=True, output_type='harmonic', rng='device')
                 for i in range(2)]
        f = tst.compute_fisher_contribution(0, a_lms=a_lms)  # warm-up
        best = None
        for _ in range(a.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            f = tst.compute_fisher_contribution(0, a_lms=a_lms)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        res[prec] = f
        _lib.call("ps_stats_reset")
        _lib.call("ps_stats_enable_timing", 1)
        tst.compute_fisher_contribution(0, a_lms=a_lms)
        torch.cuda.synchronize()
        _lib.call("ps_stats_enable_timing", 0)
        st = {k: _lib.stats(k) for k in _lib.KERNEL_KINDS}
        data = base.to_map(base.generate_data(seed=3, output_type='harmonic', rng='device'))
        tst.generate_sims(1)
        tst.Tl_numerator(data)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        num = tst.Tl_numerator(data)
        e1.record()
        torch.cuda.synchronize()
        print("tspec %s: Nside %d lmax %d, N_r %d: set-up (k integrals) %.1f s; Fisher contribution %.1f ms"
              " -> %.3f sims/s; numerator (1 sim pair) %.1f ms" % (prec, a.nside, a.lmax, a.nr, t_setup, best,
                                                                  1e3 / best, e0.elapsed_time(e1)), flush=True)
        print("tspec %s kernel ms: %s" % (prec, ", ".join("%s %.1f" % (k, v[1]) for k, v in st.items() if v[0])))
        print("tspec %s numerator %s" % (prec, num))
        del tst, wts, base
        torch.cuda.empty_cache()
    if "fp64" in res and "mixed" in res:
        F, G = res["fp64"], res["mixed"]
        d = np.sqrt(np.abs(np.outer(np.diag(F), np.diag(F))))
        print("tspec mixed vs fp64 Fisher: max |dF| / sqrt(F_ii F_jj) %.2e" % (np.abs(G - F) / d).max())


def tspecbin(a):
    """Binned-trispectrum numerator and Fisher contribution (T+E, log bins, ideal filter)."""
    import numpy as np
    from polyspec_b200 import PolySpec, Weightings, _lib
    from polyspec_b200 import workloads as W
    from polyspec_b200.tspec_bin import TSpecBin
    cltot, cl, beam, mask, l_bins, _ = W.bispec_setup(a.nside, a.lmax, a.nbins)
    fields = ['TTTT', 'TTTE', 'TTEE', 'TETE', 'TEEE', 'EEEE']
    res = {}
    for prec in a.precs.split(","):
        base = PolySpec(a.nside, dict(cltot), beam=list(beam), pol=True, lmax=a.lmax, prec=prec)
        wts = Weightings(base, np.stack([mask] * 3), dict(cl), noise_cov=W.white_noise_cov(a.nside))
        t = TSpecBin(base, mask, wts.make_applySinv('ideal'), l_bins, fields=fields, parity='both')
        t._compute_symmetry_factor()
        a_lms = [base.generate_data(seed=11 + i, deconvolve_beam=True, output_type='harmonic', rng='device')
                 for i in range(2)]
        t.compute_fisher_contribution(0, a_lms=a_lms)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        f = t.compute_fisher_contribution(0, a_lms=a_lms)
        e1.record()
        torch.cuda.synchronize()
        ms_f = e0.elapsed_time(e1)
        res[prec] = f
        _lib.call("ps_stats_reset")
        _lib.call("ps_stats_enable_timing", 1)
        t.compute_fisher_contribution(0, a_lms=a_lms)
        torch.cuda.synchronize()
        _lib.call("ps_stats_enable_timing", 0)
        st = {k: _lib.stats(k) for k in _lib.KERNEL_KINDS}
        print("tspecbin %s kernel ms: %s" % (prec, ", ".join("%s %.1f" % (k, v[1]) for k, v in st.items() if v[0])))
        data = base.to_map(base.generate_data(seed=3, output_type='harmonic', rng='device'))
        t.generate_sims(1)
        t.Tl_numerator(data)
        e0.record()
        t.Tl_numerator(data)
        e1.record()
        torch.cuda.synchronize()
        print("tspecbin %s: Nside %d lmax %d, %d bins, N_t %d, %d A pairs: Fisher contribution %.1f ms; numerator "
              "(1 sim pair, t0 cached) %.1f ms" % (prec, a.nside, a.lmax, len(l_bins) - 1, t.N_t,
                                                   t._tables['npair'], ms_f, e0.elapsed_time(e1)), flush=True)
        del t, wts, base
        torch.cuda.empty_cache()
    if "fp64" in res and "mixed" in res:
        F, G = res["fp64"], res["mixed"]
        d = np.sqrt(np.abs(np.outer(np.diag(F), np.diag(F))))
        print("tspecbin mixed vs fp64 Fisher: max |dF| / sqrt(F_ii F_jj) %.2e" % (np.abs(G - F) / d).max())


def tauconv(a):
    """The general F convolution alone (ps_convolve_F_general) on seeded random inputs."""
    import numpy as np
    from polyspec_b200 import pixel as P
    nmax_F, top = max(a.n, 2), a.Lmax + 2
    l = np.concatenate([np.arange(m, top + 1) for m in range(top + 1)]).astype(np.int32)
    m = np.concatenate([np.full(top + 1 - mm, mm) for mm in range(top + 1)]).astype(np.int32)
    ut = P.tauNL_utils(1, a.nr, l, m, 2, a.Lmax, l, m, l, m, nmax_F)
    rng = np.random.default_rng(1)
    dev = torch.device("cuda")
    F = torch.as_tensor(rng.normal(size=(2 * nmax_F + 1, top + 1, a.nr, a.nr)), device=dev)
    g = torch.Generator(device=dev).manual_seed(2)
    PQ = torch.randn((2 * a.n3 + 1, len(l), a.nr), dtype=torch.complex128, device=dev, generator=g)
    w = rng.uniform(0.5, 1.5, a.nr)
    inds = np.arange(a.nr, dtype=np.int32)
    o_re = torch.zeros((len(l), a.nr), dtype=torch.complex128, device=dev)
    o_im = torch.zeros_like(o_re)
    for _ in range(a.launches - 1):
        ut.convolve_F_general(PQ, F, w, o_re, o_im, a.n1, a.n3, a.n, 0, inds)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ut.convolve_F_general(PQ, F, w, o_re, o_im, a.n1, a.n3, a.n, 0, inds)
    e1.record()
    torch.cuda.synchronize()
    print("tauconv: %d rows, N_r %d, (n1, n3, n) = (%d, %d, %d): %.3f ms" % (len(l), a.nr, a.n1, a.n3, a.n,
                                                                          e0.elapsed_time(e1)))


def main(argv=None):
    p = argparse.ArgumentParser()
    sub = p.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("sht")
    s.add_argument("--nside", type=int, default=1024)
    s.add_argument("--lmax", type=int, default=2048)
    s.add_argument("--batch", type=int, default=1)
    s.add_argument("--prec", default="fp64")
    s.add_argument("--ops", default="s0,a0,s2,a2")
    s.add_argument("--tables", default="auto", choices=["auto", "on", "off"],
                   help="Legendre tables of a mixed plan (built before the first transform of each spin)")
    ip = sub.add_parser("inpaint")
    ip.add_argument("--nside", type=int, default=1024)
    ip.add_argument("--holes", type=int, default=2000)
    ip.add_argument("--layers", type=int, default=2)
    q = sub.add_parser("pix")
    q.add_argument("--nside", type=int, default=512)
    q.add_argument("--nr", type=int, default=24)
    q.add_argument("--reps", type=int, default=3)
    v = sub.add_parser("serve")
    v.add_argument("--n", type=int, default=64)
    v.add_argument("--reps", type=int, default=3)
    v.add_argument("--prec", default="mixed")
    b = sub.add_parser("bspec")
    b.add_argument("--nside", type=int, default=256)
    b.add_argument("--lmax", type=int, default=511)
    b.add_argument("--nbins", type=int, default=10)
    b.add_argument("--reps", type=int, default=2)
    b.add_argument("--precs", default="fp64,mixed")
    b.add_argument("--numerator-only", action="store_true", help="only Bl_numerator (for kernel captures)")
    c = sub.add_parser("tauconv")
    c.add_argument("--Lmax", type=int, default=600)
    c.add_argument("--nr", type=int, default=24)
    c.add_argument("--n1", type=int, default=1)
    c.add_argument("--n3", type=int, default=2)
    c.add_argument("--n", type=int, default=2)
    c.add_argument("--launches", type=int, default=4)
    t = sub.add_parser("tspec")
    t.add_argument("--nside", type=int, default=512)
    t.add_argument("--lmax", type=int, default=1000)
    t.add_argument("--nr", type=int, default=24)
    t.add_argument("--reps", type=int, default=2)
    t.add_argument("--precs", default="fp64,mixed")
    t.add_argument("--Lmax", type=int, default=None,
                   help="exchange-momentum L range top (default min(3 Nside - 1, 2 lmax); templates with n > 0 "
                        "need Lmax + n <= 3 Nside - 1)")
    t.add_argument("--templates", default="gNL-loc,lensing,point-source")
    t.add_argument("--K-coll", dest="K_coll", type=float, default=0.1,
                   help="collider cut-offs K_coll = k_coll (tauNL-light:s,nu_s / tauNL-heavy:s,mu_s templates)")
    tb = sub.add_parser("tspecbin")
    tb.add_argument("--nside", type=int, default=128)
    tb.add_argument("--lmax", type=int, default=255)
    tb.add_argument("--nbins", type=int, default=6)
    tb.add_argument("--precs", default="fp64,mixed")
    a = p.parse_args(argv)
    if a.cmd == "inpaint":
        inpaint(a)
    elif a.cmd == "tspecbin":
        tspecbin(a)
    elif a.cmd == "tspec":
        tspec(a)
    elif a.cmd == "bspec":
        bspec(a)
    elif a.cmd == "serve":
        serve(a)
    elif a.cmd == "sht":
        sht(a)
    elif a.cmd == "pix":
        pix(a)
    elif a.cmd == "tauconv":
        tauconv(a)


if __name__ == "__main__":
    sys.exit(main())
