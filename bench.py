#!/usr/bin/env python
"""Fisher simulations per second of PSpecBin with the masked CG S^-1 filter.

Workload (the reference's headline configuration, synthetic inputs): TEB at
Nside 1024, lmax 2048; PSpecBin fields TT, TE, EE, BB in 8 linear bins
linspace(2, 2048, 9) (N_p = 32); applySinv = Weightings.applySinv_optimal with
the harmonic preconditioner, stopping at rz/rz0 < 1e-6 (the reference's
test, polyspec/weighting.py:336-347), at most 500 steps; white noise of
30 uK arcmin; mask = |lat| < 5.74 deg plus 500 point-source holes of 10'.
One step = one PSpecBin.compute_fisher_contribution (polyspec/pspec_bin.py:94-164):
a GRF, 33 masked syntheses and 33 CG solves, and the N_p x N_p Fisher GEMM.
The CUDA arm solves the 33 systems as one batch (BatchedCGD: every A and M
application is one batched SHT pair of 33 maps per spin).  ``--prec mixed``
(default) runs the tensor-core / FP32 SHTs; the line also carries one step of
the plain FP64 GPU backend on the same workload (``plain_fp64_gpu``) and the
relative error of the mixed backend's binned spectra against FP64 at a fixed
CG step count (``accuracy``).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference] [--prec fp64|mixed]

N > 1 runs one independent replica per GPU (seeds partitioned across ranks,
no data-path collective); value = all ranks' simulations / max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Fisher sims/s at Nside 1024, mixed+learned vs plain FP64 GPU at ≤1e-6 rel err"
UNIT = "sims/s"
FIELDS = ("TT", "TE", "EE", "BB")
THRESH = 1e-6
NSTEP = 500
# CG steps per solve the plain harmonic-preconditioned CG takes on this workload
# (measured by the FP64 CUDA arm, one solve at a time: 17.45; the algorithm and its
# stopping rule are the reference's, so the reference takes the same count)
PLAIN_CG_ITERS = 17.5
# fixed CG step count of the accuracy comparison (mixed vs FP64 binned spectra)
ACC_CG_STEPS = 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    p.add_argument("--prec", default="mixed", choices=["fp64", "mixed"])
    p.add_argument("--unbatched", action="store_true", help="one CG solve at a time (reference structure)")
    p.add_argument("--precond", default="cut", choices=["harmonic", "cut", "learned"],
                   help="CG preconditioner of the CUDA arm (stopping test: the plain CG's r^T Sigma r / b^T Sigma b)")
    p.add_argument("--no-fp64-compare", action="store_true")
    p.add_argument("--nside", type=int, default=1024)
    p.add_argument("--lmax", type=int, default=2048)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-sample-pairs", type=int, default=1)
    return p.parse_args()


def workload_config(a):
    return {"workload": "PSpecBin TT/TE/EE/BB Fisher contribution, masked CG S^-1 to the reference's residual "
                        "test (r^T Sigma r / b^T Sigma b < 1e-6, Sigma the harmonic preconditioner), TEB Nside %d "
                        "lmax %d, 8 linear bins, 30uK' white noise, 10%% cut + 500 holes" % (a.nside, a.lmax),
            "nside": a.nside, "lmax": a.lmax, "fields": list(FIELDS), "n_bins": 8,
            "l2": "inputs larger than L2 (maps 3x%d MB, alm 3x%d MB per solve, batched working set several GB)"
                  % (12 * a.nside ** 2 * 8 // 2 ** 20, (a.lmax + 1) * (a.lmax + 2) // 2 * 16 // 2 ** 20)}


# ---------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu_id), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_smi_id(dev):
    import torch
    try:
        p = torch.cuda.get_device_properties(dev)
        return "%04x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
    except Exception:
        return str(dev)


# ---------------------------------------------------------------------- CPU (oracle) leg
def cpu_pair_time(a, setup, npairs=1):
    """Seconds of one TEB synthesis + one TEB adjoint of the oracle restatement
    (one A application of the reference's CG, polyspec/weighting.py:297-299) at
    the bench workload, on all host cores."""
    from oracle import polyspec_port as P
    from oracle import sht as osht
    cl, cltot, beam, mask, noise, l_bins = setup
    base = P.PortBase(a.nside, cltot, beam, pol=True, lmax=a.lmax)
    W = P.PortWeightings(base, mask, cl, noise)
    rng = np.random.default_rng(0)
    x = (rng.normal(size=(3, len(base.l_arr))) + 1j * rng.normal(size=(3, len(base.l_arr)))) * 1e-3
    cg = P.PortCGD.__new__(P.PortCGD)
    cg.W, cg.base, cg.preconditioner = W, base, "harmonic"
    t0 = time.time()
    for _ in range(npairs):
        cg._apply_A(x)
    return (time.time() - t0) / npairs, osht.default_threads()


def pairs_per_sim(iters):
    """TEB SHT pairs of one Fisher contribution with `iters` CG steps per solve:
    33 masked syntheses, 33 solves of (iters+1) syntheses and (iters+3) adjoints."""
    synth = 33 + 33 * (iters + 1)
    adj = 33 * (iters + 3)
    return 0.5 * (synth + adj)


def run_reference(a):
    import torch  # noqa: F401  (rank bookkeeping only)
    from polyspec_b200 import workloads as Wl
    setup = Wl.cg_fisher_setup(a.nside, a.lmax)
    for _ in range(a.warmup):
        cpu_pair_time(a, setup, 1)
    ts = []
    cores = 1
    for _ in range(a.steps):
        t, cores = cpu_pair_time(a, setup, 1)
        ts.append(t)
    t_pair = float(np.mean(ts))
    per_sim = pairs_per_sim(PLAIN_CG_ITERS) * t_pair
    v = 1.0 / per_sim
    sample = ("one A application (TEB synthesis + TEB adjoint, Nside %d lmax %d) of the FP64 oracle restatement "
              "of the reference path per step (%.1f s), scaled by the %.0f SHT pairs of one Fisher contribution "
              "with %d CG steps per solve" % (a.nside, a.lmax, t_pair, pairs_per_sim(PLAIN_CG_ITERS), PLAIN_CG_ITERS))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": per_sim * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(a),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def psb_rows_maps(base, mask, l_bins, a_lm):
    """The N_p + 1 masked maps whose S^-1 a Fisher contribution needs (training data)."""
    import torch
    from polyspec_b200 import PSpecBin
    psb = PSpecBin(base, mask, None, l_bins, fields=list(FIELDS))
    rows = psb._Q2_rows(base.applyAinv(a_lm, input_type='harmonic'))
    alms = torch.stack([psb.d_beam * a_lm] + [psb.d_beam * r for r in rows])
    return psb.d_mask[None] * base.to_map_batch(alms)


# ---------------------------------------------------------------------- plain FP64 GPU + accuracy
def fp64_compare(a, setup, seed):
    """One Fisher step (after a warm-up step) of the plain FP64 GPU backend
    (harmonic CG, same batched structure and stopping rule), and the relative
    error of the mixed backend's binned spectra (Cl_numerator of one masked GRF
    map, mixed-precision kernels throughout) against FP64 with both CG solves
    run for ACC_CG_STEPS steps, which isolates arithmetic error from the
    stopping test."""
    import torch
    from polyspec_b200 import PolySpec, Weightings, PSpecBin
    cl, cltot, beam, mask, noise, l_bins = setup
    out = {}

    def build(prec, nstep, thresh, autotune=True):
        b = PolySpec(a.nside, dict(cltot), beam=list(beam), pol=True, lmax=a.lmax, prec=prec, autotune=autotune)
        w = Weightings(b, mask, dict(cl), noise_cov=noise)
        ap = w.make_applySinv("optimal", preconditioner="harmonic", nstep=nstep, thresh=thresh)
        return b, PSpecBin(b, mask, ap, l_bins, fields=list(FIELDS))

    b64, p64 = build("fp64", NSTEP, THRESH)
    a_lm = b64.generate_data(seed=seed + int(2e7), output_type="harmonic", deconvolve_beam=True, rng="device")
    # warm-up step: plan set-up and tile autotuning outside the timed step
    p64.compute_fisher_contribution(seed + 1, a_lm=a_lm, batched=not a.unbatched)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    p64.compute_fisher_contribution(seed, a_lm=a_lm, batched=not a.unbatched)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    plain = {"value": 1e3 / ms, "unit": UNIT, "ms_per_step": ms, "steps": 1, "dtype": "f64",
             "note": "plain FP64 GPU backend (FP64 Legendre + FP64 ring FFTs), same batched CG and stopping rule"}
    del p64
    torch.cuda.empty_cache()

    mask_t = torch.as_tensor(np.asarray(mask), device="cuda")
    data = b64.generate_data(seed=seed + 7, output_type="map", rng="device") * mask_t
    nums = {}
    for prec in ("fp64", "mixed"):
        # autotuning off: every transform of the mixed solve runs the mixed-precision kernels
        b, p = build(prec, ACC_CG_STEPS, 0.0, autotune=False)
        num = p.Cl_numerator(data)
        nums[prec] = num.cpu().numpy() if isinstance(num, torch.Tensor) else np.asarray(num)
        del b, p
        torch.cuda.empty_cache()
    n64, nmx = nums["fp64"], nums["mixed"]
    # per field: max over bins of |d| / |C_fp64|; cross spectra (TE) also normalised by sqrt(TT EE)
    per_field = {f: float(np.max(np.abs(nmx[i] - n64[i]) / np.abs(n64[i]))) for i, f in enumerate(FIELDS)}
    per_field_l2 = {f: float(np.linalg.norm(nmx[i] - n64[i]) / np.linalg.norm(n64[i])) for i, f in enumerate(FIELDS)}
    iTT, iTE, iEE = FIELDS.index("TT"), FIELDS.index("TE"), FIELDS.index("EE")
    te_norm = float(np.max(np.abs(nmx[iTE] - n64[iTE]) / np.sqrt(np.abs(n64[iTT] * n64[iEE]))))
    acc = {"binned_cl_max_rel_err": float(np.max(np.abs(nmx - n64) / np.abs(n64))),
           "binned_cl_rel_l2_err": float(np.linalg.norm(nmx - n64) / np.linalg.norm(n64)),
           "max_rel_err_per_field": per_field, "rel_l2_err_per_field": per_field_l2,
           "TE_err_over_sqrt_TT_EE": te_norm,
           "tolerance": 1e-6, "cg_steps": ACC_CG_STEPS,
           "what": "PSpecBin.Cl_numerator (TT, TE, EE, BB x 8 bins) of one masked GRF map, mixed vs FP64 backend, "
                   "same fixed CG step count"}
    return plain, acc


# ---------------------------------------------------------------------- replicas
def replica_seeds(rank, nsteps):
    """Seeds of one rank's Fisher simulations: disjoint across ranks (replicas, no collective)."""
    return [rank * 100000 + i for i in range(nsteps)]


def max_over_ranks(ms, device):
    """The slowest rank's time (the job's time), from an all-reduce of one scalar."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


# ---------------------------------------------------------------------- CUDA arm
def run_cuda(a):
    import torch
    import torch.distributed as dist
    from polyspec_b200 import PolySpec, Weightings, PSpecBin, _lib
    from polyspec_b200 import workloads as Wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    setup = Wl.cg_fisher_setup(a.nside, a.lmax)
    cl, cltot, beam, mask, noise, l_bins = setup
    base = PolySpec(a.nside, dict(cltot), beam=list(beam), pol=True, lmax=a.lmax, prec=a.prec)
    wts = Weightings(base, mask, dict(cl), noise_cov=noise)
    # one-time set-up of the preconditioner (per Weightings, outside the timed region)
    torch.cuda.synchronize()
    t_setup = time.time()
    if a.precond == "cut":
        wts.cut_preconditioner()
    elif a.precond == "learned":
        from polyspec_b200.learned import LearnedBandPreconditioner
        lp = LearnedBandPreconditioner(wts)
        tr = [base.generate_data(seed=900 + i, output_type="harmonic", deconvolve_beam=True, rng="device")
              for i in range(2)]
        for i, t_alm in enumerate(tr):
            rows = psb_rows_maps(base, mask, l_bins, t_alm)
            lp.collect(rows, nstep=NSTEP)
        lp.train(epochs=400)
        wts.learned = lp
    torch.cuda.synchronize()
    setup_s = time.time() - t_setup
    applySinv = wts.make_applySinv("optimal", preconditioner=a.precond, nstep=NSTEP, thresh=THRESH)
    psb = PSpecBin(base, mask, applySinv, l_bins, fields=list(FIELDS))

    nsteps = a.warmup + 2 * a.steps
    seeds = replica_seeds(rank, nsteps)
    a_dev = [base.generate_data(seed=s + int(1e7), output_type="harmonic", deconvolve_beam=True, rng="device")
             for s in seeds]
    torch.cuda.synchronize()

    cg_iters = []
    solve_iters = []

    def one(i, a_lm):
        it0 = base.n_SHTs_forward
        f = psb.compute_fisher_contribution(seeds[i], a_lm=a_lm, batched=not a.unbatched)
        cg_iters.append(base.n_SHTs_forward - it0)
        if not a.unbatched and getattr(wts, "last_cgd", None) is not None:
            solve_iters.append([int(v) for v in wts.last_cgd.iters.cpu()])
        return f

    for i in range(a.warmup):
        one(i, a_dev[i])
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- device-resident timed region
    clk = ClockSampler(gpu_smi_id(local))
    _lib.call("ps_stats_reset")
    _lib.call("ps_stats_enable_timing", 1)
    f0, r0 = base.n_SHTs_forward, base.n_SHTs_reverse
    barrier()
    torch.cuda.synchronize()
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for k in range(a.steps):
        one(a.warmup + k, a_dev[a.warmup + k])
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    _lib.call("ps_stats_enable_timing", 0)
    t_ms = ev0.elapsed_time(ev1)
    stats = {k: _lib.stats(k) for k in _lib.KERNEL_KINDS}
    fwd = (base.n_SHTs_forward - f0) / a.steps
    rev = (base.n_SHTs_reverse - r0) / a.steps
    if world > 1:
        t_ms = max_over_ranks(t_ms, "cuda")
    value = world * a.steps / (t_ms / 1e3)

    # ---- end to end through the public API, host buffers
    host_a = [a_dev[a.warmup + a.steps + k].cpu().pin_memory() for k in range(a.steps)]
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    t0 = time.time()
    for k in range(a.steps):
        fish = psb.compute_fisher_contribution(seeds[a.warmup + a.steps + k], a_lm=host_a[k],
                                               batched=not a.unbatched)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.time() - t0) * 1e3)
    barrier()
    if world > 1:
        e2e_ms = max_over_ranks(e2e_ms, "cuda")
    e2e = {"value": world * a.steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int(host_a[0].numel() * host_a[0].element_size()),
           "d2h_bytes_per_step": int(fish.nbytes)}

    # ---- roofline of the dominant kernel (device time inside the timed region)
    dom = max(stats, key=lambda k: stats[k][1])
    n, ms, fl, by = stats[dom]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    if fl > 0:
        ach = fl / (ms / 1e3) / 1e12
        peak = peaks.get("bf16_tflops", 1590.0)
        sm_ghz = (clocks.get("sm_mhz") or 1965.0) / 1e3
        if a.prec == "fp64":
            pipe, pipe_peak = "FP64 FMA pipe (64 DFMA/clk/SM)", 64 * 2 * 148 * sm_ghz / 1e3
        elif dom == "leg_synth":
            # three TF32 MMAs per product (hi.hi + hi.lo + lo.hi): the algorithmic flops are a third of
            # the tensor-pipe flops; dense TF32 runs at half the bf16 rate
            pipe, pipe_peak = "tensor pipe, kind::tf32 (x3 split)", peak / 2 / 3
        else:
            pipe, pipe_peak = "FP32 FMA pipe (128 FFMA/clk/SM)", 128 * 2 * 148 * sm_ghz / 1e3
        roof = {"bound": "tensor", "kernel": dom, "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                "frac": ach / peak,
                "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst), of measured" if peaks else "fallback",
                "pipe": pipe, "pipe_peak_tflops": pipe_peak, "frac_of_pipe_peak": ach / pipe_peak,
                "launches": n, "avg_launch_ms": ms / max(n, 1), "traffic": None,
                "algorithmic_flops_per_launch": fl / max(n, 1),
                "note": "achieved = algorithmic Legendre flops (4 per ring pair, alm and map for spin 0, 16 for a "
                        "spin-s pair) / CUDA-event time of the kernel inside the timed region"}
    else:
        ach = by / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        peak = peaks.get("hbm_gbs", 6650.0)
        roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "launches": n, "avg_launch_ms": ms / max(n, 1), "traffic": None}
    launches = int(sum(v[0] for v in stats.values()))
    iters = [c for c in cg_iters[a.warmup:a.warmup + a.steps]]
    # forward SHTs per sim = 2 per TEB adjoint; solves = 33 with (iters + 3) adjoints each
    iters_per_solve = (np.mean(iters) / 2.0) / 33.0 - 3.0 if iters else float("nan")

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": t_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if a.prec == "fp64" else "f32+tf32", "data": "synthetic",
            "config": dict(workload_config(a), parallelism="replicas x%d" % world, prec=a.prec,
                           preconditioner=a.precond, batched=not a.unbatched),
            "preconditioner_setup_s": setup_s,
            "e2e": e2e, "gpu_launches": launches, "roofline": roof, "clocks": clocks,
            "sht_teb_per_step": {"synthesis": rev / 2.0, "adjoint": fwd / 2.0},
            "cg_iters_per_solve": iters_per_solve,
            "cg_iters_of_each_solve": solve_iters[-1] if solve_iters else None,
            "kernel_ms": {k: round(v[1], 3) for k, v in stats.items() if v[0]}}

    if a.prec != "fp64" and not a.no_fp64_compare and world == 1:
        del psb, applySinv, wts, a_dev, base
        torch.cuda.empty_cache()
        line["plain_fp64_gpu"], line["accuracy"] = fp64_compare(a, setup, seeds[0])
        torch.cuda.empty_cache()

    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        t_pair, cores = cpu_pair_time(a, setup, a.cpu_sample_pairs)
        # the reference's CPU path runs the plain harmonic CG: its step count, not this arm's
        ips = PLAIN_CG_ITERS
        per_sim = pairs_per_sim(ips) * t_pair
        line["cpu_baseline"] = {
            "value": 1.0 / per_sim, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d A application(s) (TEB synthesis + TEB adjoint) of the FP64 oracle restatement at the "
                      "same workload, %.1f s each, scaled by the %.0f SHT pairs of one Fisher contribution"
                      % (a.cpu_sample_pairs, t_pair, pairs_per_sim(ips))}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        run_reference(a)
        return
    run_cuda(a)


if __name__ == "__main__":
    main()
