#!/usr/bin/env python
"""Fisher simulations per second of PSpecBin with the masked CG S^-1 filter.

Workload (synthetic inputs of the reference's headline configuration): TEB at
Nside 1024, lmax 2048; PSpecBin fields TT, TE, EE, BB in 8 linear bins
linspace(2, 2048, 9) (N_p = 32); applySinv = Weightings.applySinv_optimal,
stopping when r^T Sigma r / b^T Sigma b < 1e-6 (the reference's statistic for
its harmonic preconditioner Sigma, polyspec/weighting.py:326-351), at most 500
steps; white noise of 30 uK arcmin; mask = |lat| < 5.74 deg plus 500
point-source holes of 10'.  One step = one PSpecBin.compute_fisher_contribution
(polyspec/pspec_bin.py:94-164): the GRF draw (on the device), 33 masked
syntheses, 33 CG solves and the N_p x N_p Fisher product.  The CUDA arm solves
the 33 systems as one batch (BatchedCGD; systems drop out as they converge).

The line (one JSON object) carries, besides the contract's keys:
  * config.preconditioner: the timed arm's CG preconditioner ('cut' = the
    masked-band Woodbury preconditioner by default, 'harmonic' = the
    reference's, 'learned');
  * fp64_same_preconditioner_gpu: the FP64 backend with the same preconditioner
    (separates the gain of mixed precision from the preconditioner's);
  * plain_fp64_gpu: the FP64 backend with the reference's harmonic CG;
  * accuracy: mixed against FP64 on the timed configuration (same
    preconditioner, both run to the 1e-6 stopping test): the alm of one S^-1
    solve, the binned spectra (Cl_numerator) and one Fisher contribution;
  * roofline of the dominant kernel, cpu_baseline (oracle port), clocks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference] [--prec fp64|mixed]

N > 1 runs one independent replica per GPU (seeds partitioned across ranks,
no data-path collective); value = all ranks' simulations / max-over-ranks time.

--impl reference times the reference's CPU algorithm (the oracle restatement of
polyspec/base.py, weighting.py, pspec_bin.py over the FP64 oracle SHT) on the
host cores: the simulation's S^-1 solve is run to convergence with the
reference's stopping test during warm-up (its CG steps counted), every timed
step is one CG step of that solve's system, and one Fisher contribution is
33 solves of that many steps.
"""
import argparse
import gc
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
# DRAM bytes (read + write) / algorithmic bytes of the table-driven Legendre kernels, from one ncu
# capture at Nside 512, lmax 1000, 32 maps (spin 0 and spin 2 launches together)
TABLE_TRAFFIC_RATIO = {"leg_adjoint": 1.015, "leg_synth": 0.991}
FIELDS = ("TT", "TE", "EE", "BB")
THRESH = 1e-6
NSTEP = 500


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    p.add_argument("--prec", default="mixed", choices=["fp64", "mixed"])
    p.add_argument("--unbatched", action="store_true", help="one CG solve at a time (reference structure)")
    p.add_argument("--precond", default="cut", choices=["harmonic", "cut", "learned"],
                   help="CG preconditioner of the timed arm (stopping test: the plain CG's r^T Sigma r / b^T Sigma b)")
    p.add_argument("--tables", default="auto", choices=["auto", "on", "off"],
                   help="Legendre tables of the mixed plans (streaming tensor-core Legendre stages)")
    p.add_argument("--fp64-steps", type=int, default=3, help="timed steps of each FP64 comparison arm")
    p.add_argument("--no-fp64-compare", action="store_true")
    p.add_argument("--nside", type=int, default=1024)
    p.add_argument("--lmax", type=int, default=2048)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--sims-per-step", type=int, default=1,
                   help="Fisher contributions per step, their K (N_p + 1) systems solved as one batch")
    p.add_argument("--workload", default="fisher-teb", choices=["fisher-teb", "pspec-t64"],
                   help="fisher-teb: the headline (default); pspec-t64: PSpecBin T at Nside 64, lmax 191, ideal "
                        "S^-1 of the latitude-masked map, Fisher from seeds 1-10, beside the CPU oracle port")
    return p.parse_args()


def workload_config(a):
    return {"workload": "PSpecBin TT/TE/EE/BB Fisher contribution, masked CG S^-1 to the reference's residual "
                        "test (r^T Sigma r / b^T Sigma b < 1e-6, Sigma the harmonic preconditioner), TEB Nside %d "
                        "lmax %d, 8 linear bins, 30uK' white noise, 10%% cut + 500 holes; GRF draw inside the step"
                        % (a.nside, a.lmax),
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
class CpuSolve:
    """The reference's S^-1 of one simulation's masked map (polyspec/pspec_bin.py:102-117 with
    polyspec/weighting.py:148-184, 217-367) on the FP64 oracle restatement, all host threads."""

    def __init__(self, a, setup, seed):
        from oracle import polyspec_port as P
        from oracle import sht as osht
        cl, cltot, beam, mask, noise, l_bins = setup
        self.cores = osht.default_threads()
        self.base = P.PortBase(a.nside, cltot, beam, pol=True, lmax=a.lmax)
        self.W = P.PortWeightings(self.base, mask, cl, noise)
        t0 = time.time()
        a_lm = self.base.generate_data(seed + int(1e7), deconvolve_beam=True)
        d = self.W.mask * self.base.to_map(self.base.beam_lm * a_lm)
        x0 = np.einsum('abi,bi->ai', self.W.x0op_lm, self.base.to_lm(d))
        self.cg = P.PortCGD(self.W, d, x0, "harmonic")
        self.t_setup = time.time() - t0  # masked synthesis, x0, b, A x0, M b0: the solve's fixed cost

    def step(self):
        t0 = time.time()
        self.cg.step()
        return time.time() - t0


def run_reference(a):
    """The reference's CPU algorithm on the bench workload: warm-up solves the simulation's system to
    convergence (counting its CG steps), then each timed step is one CG step of a fresh copy of it."""
    from polyspec_b200 import workloads as Wl
    setup = Wl.cg_fisher_setup(a.nside, a.lmax)
    s = CpuSolve(a, setup, 0)
    n_iter = 0
    while n_iter < NSTEP:
        s.step()
        n_iter += 1
        if s.cg.err < THRESH:
            break
    for _ in range(max(a.warmup - 1, 0)):
        s.step()
    s2 = CpuSolve(a, setup, 0)
    ts = [s2.step() for _ in range(a.steps)]
    t_step = float(np.mean(ts))
    n_solves = 1 + len(FIELDS) * 8
    per_sim = n_solves * (s2.t_setup + n_iter * t_step)
    v = 1.0 / per_sim
    sample = ("oracle restatement of the reference path, FP64, %d host threads: the simulation's S^-1 system solved "
              "to convergence with the reference's stopping test in warm-up (%d CG steps), then %d timed CG steps "
              "(%.2f s each, one TEB synthesis + adjoint and the harmonic preconditioner) plus the solve's fixed "
              "cost (%.1f s); one Fisher contribution = %d solves of that many steps (the BB-row solves take more "
              "steps than the simulation's, so this overstates the CPU rate)"
              % (s2.cores, n_iter, a.steps, t_step, s2.t_setup, n_solves))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(a),
            "cg_steps_counted": n_iter, "seconds_per_sim": per_sim,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": s2.cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------- CUDA helpers
def build_arm(a, setup, prec, precond, tables):
    """PolySpec + Weightings (+ preconditioner set-up) + PSpecBin of one precision and preconditioner."""
    import torch
    from polyspec_b200 import PolySpec, Weightings, PSpecBin
    cl, cltot, beam, mask, noise, l_bins = setup
    base = PolySpec(a.nside, dict(cltot), beam=list(beam), pol=True, lmax=a.lmax, prec=prec)
    if prec != "fp64":
        base.plan().tables = {"auto": "auto", "on": True, "off": False}[tables]
    wts = Weightings(base, mask, dict(cl), noise_cov=noise)
    torch.cuda.synchronize()
    t0 = time.time()
    if precond == "cut":
        wts.cut_preconditioner()
    elif precond == "learned":
        from polyspec_b200.learned import LearnedBandPreconditioner
        lp = LearnedBandPreconditioner(wts, base="cut")
        for i in range(2):
            t_alm = base.generate_data(seed=900 + i, output_type="harmonic", deconvolve_beam=True, rng="device")
            lp.collect(psb_rows_maps(base, mask, l_bins, t_alm), nstep=NSTEP)
        lp.train(epochs=400)
        wts.learned = lp
    torch.cuda.synchronize()
    setup_s = time.time() - t0
    ap = wts.make_applySinv("optimal", preconditioner=precond, nstep=NSTEP, thresh=THRESH)
    psb = PSpecBin(base, mask, ap, l_bins, fields=list(FIELDS))
    return base, wts, psb, setup_s


def psb_rows_maps(base, mask, l_bins, a_lm):
    """The N_p + 1 masked maps whose S^-1 a Fisher contribution needs (training data)."""
    import torch
    from polyspec_b200 import PSpecBin
    psb = PSpecBin(base, mask, None, l_bins, fields=list(FIELDS))
    rows = psb._Q2_rows(base.applyAinv(a_lm, input_type='harmonic'))
    alms = torch.stack([psb.d_beam * a_lm] + [psb.d_beam * r for r in rows])
    return psb.d_mask[None] * base.to_map_batch(alms)


def fisher_step(psb, seeds, batched, a_lms=None):
    """One step: the Fisher contributions of the simulations `seeds` (GRF drawn on the device, or host
    a_lms), several as one batched solve (PSpecBin.compute_fisher_contributions)."""
    if len(seeds) == 1:
        return psb.compute_fisher_contribution(seeds[0], batched=batched, rng="device",
                                               a_lm=None if a_lms is None else a_lms[0])
    return psb.compute_fisher_contributions(seeds, rng="device", a_lms=a_lms)


def groups(seeds, k):
    return [seeds[i:i + k] for i in range(0, len(seeds), k)]


def timed_steps(psb, seed_groups, batched, wts=None):
    """CUDA-event time (ms) of the Fisher steps over `seed_groups` (GRF drawn on the device inside each
    step) and the CG steps of each solve of the last one."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for g in seed_groups:
        fisher_step(psb, g, batched)
    e1.record()
    torch.cuda.synchronize()
    iters = None
    if wts is not None and getattr(wts, "last_cgd", None) is not None and hasattr(wts.last_cgd, "iters"):
        iters = [int(v) for v in wts.last_cgd.iters.cpu()]
    return e0.elapsed_time(e1), iters


def release():
    import torch
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def rel_errs(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    return {"max_rel": float(np.max(np.abs(x - ref)) / np.max(np.abs(ref))),
            "l2_rel": float(np.linalg.norm(x - ref) / np.linalg.norm(ref))}


def spectra_errs(x, ref):
    out = rel_errs(x, ref)
    out["max_rel_per_bin"] = float(np.max(np.abs(x - ref) / np.abs(ref)))
    return out


def fisher_errs(f, ref):
    out = rel_errs(f, ref)
    d = np.sqrt(np.abs(np.outer(np.diag(ref), np.diag(ref))))
    out["max_over_sqrt_FiiFjj"] = float(np.max(np.abs(f - ref) / d))
    return out


def accuracy_inputs(base, mask, seed):
    """Host inputs shared by both precisions: a masked GRF map (the S^-1 / Cl_numerator input)
    and a GRF a_lm (the Fisher contribution's simulation), drawn by numpy."""
    import torch
    a_f = base.generate_data(seed=seed + int(1e7), output_type="harmonic", deconvolve_beam=True, rng="numpy")
    a_d = base.generate_data(seed=seed + 7, output_type="harmonic", rng="numpy")
    a_d = torch.as_tensor(np.asarray(a_d), device="cuda")
    d = (torch.as_tensor(np.asarray(mask), device="cuda") * base.to_map_batch(a_d[None])[0]).cpu().numpy()
    return np.asarray(a_f), d


def accuracy_run(wts, psb, a_f, d):
    """S^-1 alm of the map d, its binned spectra and the Fisher contribution of a_f, with the
    per-system CG step counts."""
    import torch
    h = psb.applySinv(torch.as_tensor(d, device="cuda"), input_type="map")
    cg = wts.last_cgd
    it_h = int(cg.iters[0]) if hasattr(cg, "iters") else int(getattr(cg, "i", -1))
    spec = psb._binned_auto(h).cpu().numpy()
    fish = psb.compute_fisher_contribution(0, a_lm=a_f, batched=True)
    cg = wts.last_cgd
    it_f = [int(v) for v in cg.iters.cpu()] if hasattr(cg, "iters") else None
    return h.cpu().numpy(), spec, np.asarray(fish), it_h, it_f


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
def roofline(a, stats, clocks, tables_used):
    """Roofline of the kernel kind with the largest device time inside the timed region."""
    dom = max(stats, key=lambda k: stats[k][1])
    n, ms, fl, by = stats[dom]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    sm_ghz = (clocks.get("sm_mhz") or 1965.0) / 1e3
    tab_dom = dom.startswith("leg_") and a.prec != "fp64" and all(tables_used.values())
    if tab_dom and by > 0:
        # the table-driven Legendre stages stream their FP32 table from HBM: HBM bound.  DRAM traffic per
        # launch: the algorithmic bytes times the DRAM/algorithmic ratio of an ncu capture of the same
        # kernels at Nside 512, 32 maps (profiles/table_legendre_nside512_b32.md), scaled by the units
        # processed (traffic grows with the table and the maps)
        ratio = TABLE_TRAFFIC_RATIO[dom]
        ach = by / (ms / 1e3) / 1e9
        peak = peaks.get("hbm_gbs", 6650.0)
        return {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs, of measured" if peaks else "6650 GB/s, of fallback",
                "launches": n, "avg_launch_ms": ms / max(n, 1), "traffic": ratio * by / max(n, 1),
                "traffic_source": "ncu dram__bytes_read+write / algorithmic bytes = %.3f at Nside 512, 32 maps, "
                                  "scaled to the launch's algorithmic bytes" % ratio,
                "algorithmic_bytes_per_launch": by / max(n, 1),
                "tensor_tflops": fl / (ms / 1e3) / 1e12,
                "tensor_frac_of_bf16_sustained": fl / (ms / 1e3) / 1e12 / peaks.get("bf16_tflops_sustained", 1400.0),
                "note": "achieved = algorithmic bytes (the FP32 Legendre table of the launch's ring pairs, alm and "
                        "ring phases once) / CUDA-event time of the kernel inside the timed region; tensor_tflops = "
                        "algorithmic Legendre flops (4 per ring pair for spin 0, 16 for a spin-s pair) / same time"}
    if fl > 0:
        ach = fl / (ms / 1e3) / 1e12
        peak = peaks.get("bf16_tflops_sustained", 1400.0)
        if a.prec == "fp64":
            pipe, pipe_peak = "FP64 FMA pipe (64 DFMA/clk/SM)", 64 * 2 * 148 * sm_ghz / 1e3
        elif dom == "leg_synth":
            pipe, pipe_peak = "tensor pipe, kind::tf32 (x3 split)", peaks.get("bf16_tflops", 1590.0) / 2 / 3
        else:
            pipe, pipe_peak = "FP32 FMA pipe (128 FFMA/clk/SM)", 128 * 2 * 148 * sm_ghz / 1e3
        return {"bound": "tensor", "kernel": dom, "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                "frac": ach / peak,
                "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained, of measured" if peaks else "fallback",
                "pipe": pipe, "pipe_peak_tflops": pipe_peak, "frac_of_pipe_peak": ach / pipe_peak,
                "launches": n, "avg_launch_ms": ms / max(n, 1), "traffic": None,
                "algorithmic_flops_per_launch": fl / max(n, 1)}
    ach = by / (ms / 1e3) / 1e9 if ms > 0 else 0.0
    peak = peaks.get("hbm_gbs", 6650.0)
    return {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "launches": n, "avg_launch_ms": ms / max(n, 1), "traffic": None}


def run_cuda(a):
    import torch
    import torch.distributed as dist
    from polyspec_b200 import _lib
    from polyspec_b200 import workloads as Wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    setup = Wl.cg_fisher_setup(a.nside, a.lmax)
    mask = setup[3]
    base, wts, psb, setup_s = build_arm(a, setup, a.prec, a.precond, a.tables)
    batched = not a.unbatched
    K = max(1, a.sims_per_step)
    seeds = replica_seeds(rank, (a.warmup + 2 * a.steps) * K)
    steps_seeds = groups(seeds, K)  # warm-up, timed, end-to-end steps
    for g in steps_seeds[:a.warmup]:
        fisher_step(psb, g, batched)
    torch.cuda.synchronize()
    plan = base.plan()
    tables_used = {s: bool(plan.has_table(s)) for s in (0, 2)} if a.prec != "fp64" else {0: False, 2: False}

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- device-resident timed region (the GRF is drawn on the device inside each step)
    clk = ClockSampler(gpu_smi_id(local))
    _lib.call("ps_stats_reset")
    _lib.call("ps_stats_enable_timing", 1)
    f0, r0 = base.n_SHTs_forward, base.n_SHTs_reverse
    barrier()
    torch.cuda.synchronize()
    clk.start()
    # a profiler started with --profile-from-start off (ncu) captures the timed steps only
    torch.cuda.profiler.start()
    t_ms, solve_iters = timed_steps(psb, steps_seeds[a.warmup:a.warmup + a.steps], batched, wts)
    torch.cuda.profiler.stop()
    barrier()
    clocks = clk.stop()
    _lib.call("ps_stats_enable_timing", 0)
    stats = {k: _lib.stats(k) for k in _lib.KERNEL_KINDS}
    fwd = (base.n_SHTs_forward - f0) / a.steps
    rev = (base.n_SHTs_reverse - r0) / a.steps
    if world > 1:
        t_ms = max_over_ranks(t_ms, "cuda")
    value = world * a.steps * K / (t_ms / 1e3)

    # ---- end to end through the public API: host a_lm (pinned) in, the Fisher matrix out
    e2e_groups = steps_seeds[a.warmup + a.steps:]
    host_a = [[base.generate_data(seed=s + int(1e7), output_type="harmonic", deconvolve_beam=True, rng="device")
               .cpu().pin_memory() for s in g] for g in e2e_groups]
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    t0 = time.time()
    for k, g in enumerate(e2e_groups):
        fish = fisher_step(psb, g, batched, a_lms=host_a[k])
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.time() - t0) * 1e3)
    barrier()
    if world > 1:
        e2e_ms = max_over_ranks(e2e_ms, "cuda")
    e2e = {"value": world * a.steps * K / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int(sum(h.numel() * h.element_size() for h in host_a[0])),
           "d2h_bytes_per_step": int(fish.nbytes)}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": t_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if a.prec == "fp64" else "f32+tf32", "data": "synthetic",
            "config": dict(workload_config(a), parallelism="replicas x%d" % world, prec=a.prec,
                           preconditioner=a.precond, batched=batched, sims_per_step=K,
                           legendre_tables={"spin%d" % s: v for s, v in tables_used.items()}),
            "measured_arm": "%s precision, %s preconditioner%s" % (
                a.prec, {"cut": "masked-band (cut)", "harmonic": "harmonic", "learned": "learned on cut"}[a.precond],
                "" if a.precond == "learned" else "; the learned preconditioner is not in this arm"),
            "preconditioner_setup_s": setup_s,
            "e2e": e2e, "gpu_launches": int(sum(v[0] for v in stats.values())),
            "roofline": roofline(a, stats, clocks, tables_used), "clocks": clocks,
            "sht_teb_per_step": {"synthesis": rev / 2.0, "adjoint": fwd / 2.0},
            "cg_iters_of_each_solve": solve_iters,
            "kernel_ms": {k: round(v[1], 3) for k, v in stats.items() if v[0]},
            "peak_device_gb": round(torch.cuda.max_memory_allocated() / 1e9, 1)}

    if a.prec != "fp64" and not a.no_fp64_compare and world == 1:
        # ---- accuracy on the timed configuration, then the FP64 arms
        a_f, d = accuracy_inputs(base, mask, 4242)
        h_mx, spec_mx, fish_mx, ith_mx, itf_mx = accuracy_run(wts, psb, a_f, d)
        del psb, wts, base, plan, host_a
        release()
        base64, wts64, psb64, setup64 = build_arm(a, setup, "fp64", a.precond, "off")
        h_64, spec_64, fish_64, ith_64, itf_64 = accuracy_run(wts64, psb64, a_f, d)
        line["accuracy"] = {
            "what": "mixed vs FP64 backend on the timed configuration (%s preconditioner, both to the 1e-6 "
                    "stopping test): alm = applySinv_optimal of one masked GRF map; binned = Cl_numerator of that "
                    "map (TT, TE, EE, BB x 8 bins); fisher = compute_fisher_contribution of one GRF" % a.precond,
            "alm": rel_errs(h_mx, h_64), "binned": spectra_errs(spec_mx, spec_64),
            "fisher": fisher_errs(fish_mx, fish_64), "tolerance": 1e-6,
            "cg_steps_alm_solve": {"mixed": ith_mx, "fp64": ith_64},
            "cg_steps_fisher_solves_equal": itf_mx == itf_64}
        fisher_step(psb64, [99991 - j for j in range(K)], batched)  # warm-up
        ms64, it64 = timed_steps(psb64, groups([99992 + i for i in range(a.fp64_steps * K)], K), batched, wts64)
        line["fp64_same_preconditioner_gpu"] = {
            "value": a.fp64_steps * K / (ms64 / 1e3), "unit": UNIT, "ms_per_step": ms64 / a.fp64_steps,
            "steps": a.fp64_steps, "warmup": 1, "dtype": "f64", "preconditioner": a.precond,
            "preconditioner_setup_s": setup64, "cg_iters_of_each_solve": it64,
            "note": "FP64 backend (FP64 Legendre + FP64 ring FFTs), same preconditioner, batching and stopping rule"}
        del psb64, wts64, base64
        release()
        if a.precond != "harmonic":
            base_h, wts_h, psb_h, _ = build_arm(a, setup, "fp64", "harmonic", "off")
            fisher_step(psb_h, [99981 - j for j in range(K)], batched)
            msh, ith = timed_steps(psb_h, groups([99982 + i for i in range(a.fp64_steps * K)], K), batched, wts_h)
            line["plain_fp64_gpu"] = {
                "value": a.fp64_steps * K / (msh / 1e3), "unit": UNIT, "ms_per_step": msh / a.fp64_steps,
                "steps": a.fp64_steps, "warmup": 1, "dtype": "f64", "preconditioner": "harmonic",
                "cg_iters_of_each_solve": ith,
                "note": "FP64 backend with the reference's harmonic CG, same batching and stopping rule"}
            del psb_h, wts_h, base_h
            release()
        else:
            line["plain_fp64_gpu"] = line["fp64_same_preconditioner_gpu"]
        line["speedup"] = {
            "mixed_over_fp64_same_preconditioner": value / line["fp64_same_preconditioner_gpu"]["value"],
            "mixed_over_plain_fp64": value / line["plain_fp64_gpu"]["value"]}

    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        # bounded CPU sample: one CG step of the simulation's S^-1 system (+ the solve's fixed cost),
        # scaled by the CG steps of each of the 33 solves of the plain FP64 arm in this run
        s = CpuSolve(a, setup, 0)
        t_step = s.step()
        it_plain = (line.get("plain_fp64_gpu") or {}).get("cg_iters_of_each_solve")
        if it_plain:
            per_sim = (len(it_plain) * s.t_setup + sum(it_plain) * t_step) / K
            line["cpu_baseline"] = {
                "value": 1.0 / per_sim, "unit": UNIT, "cores": s.cores, "kind": "port",
                "sample": "one CG step (%.2f s: TEB synthesis + adjoint, harmonic preconditioner) and the fixed cost "
                          "of one solve (%.1f s) of the oracle restatement at the full workload, scaled by the %d CG "
                          "steps of the %d solves of %d simulation(s) of the reference algorithm (harmonic CG, FP64) "
                          "counted on the plain FP64 arm of this run" % (t_step, s.t_setup, sum(it_plain),
                                                                         len(it_plain), K)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------- PSpecBin T at Nside 64
def pspec_t64(a):
    """PSpecBin plain, T only: Nside 64, lmax 191 (the reference's default 3 Nside - 1), 8 bins of 16 from
    l = 2 (up to l = 130, within lmax as PSpecBin requires), C_l = 1000/(l+10)^2,
    30' beam, |lat| < 15 deg cut with a 5 deg cosine taper, applySinv = ideal S^-1 of the masked
    map; one step = the Fisher contributions of seeds 1-10 (polyspec/pspec_bin.py:94-164) and the
    numerator of the seed-0 GRF.  FP64 on the GPU and, on the host, the oracle restatement."""
    import torch
    from polyspec_b200 import PolySpec, Weightings, PSpecBin
    from polyspec_b200 import workloads as Wl
    nside, lmax = 64, 191
    cl = Wl.fiducial_cl(lmax, False)
    b = Wl.gaussian_beam(lmax, 30.0)
    cltot = {'TT': cl['TT'] * b ** 2}
    mask = Wl.latitude_mask(nside, 15.0, 5.0)
    l_bins = 2 + 16 * np.arange(9)
    seeds = list(range(1, 11))
    line = {"metric": "PSpecBin Fisher sims/s (T, Nside 64)", "unit": "sims/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "PSpecBin T, Nside 64, lmax 191, 8 bins of 16 from l=2, 30' beam, |lat|<15 deg "
                                   "cut + 5 deg taper, ideal S^-1, Fisher seeds 1-10 per step"}}
    base = PolySpec(nside, dict(cltot), beam=[b], pol=False, lmax=lmax, prec="fp64")
    wts = Weightings(base, mask[None], {'TT': cl['TT']})
    psb = PSpecBin(base, mask, wts.make_applySinv('ideal'), l_bins, fields=["TT"])
    data = base.generate_data(seed=0, output_type='map')
    for _ in range(a.warmup):
        for s in seeds:
            psb.compute_fisher_contribution(s)
    torch.cuda.synchronize()
    t0 = time.time()
    for _ in range(a.steps):
        fish = np.mean([psb.compute_fisher_contribution(s) for s in seeds], axis=0)
        num = psb.Cl_numerator(data)
    torch.cuda.synchronize()
    t_gpu = (time.time() - t0) / a.steps
    line["value"] = len(seeds) / t_gpu
    line["ms_per_step"] = 1e3 * t_gpu
    line["e2e"] = {"value": line["value"], "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                   "note": "numpy in, numpy out through the reference API (GRF drawn by numpy on the host)"}
    if not a.no_cpu_baseline:
        from oracle import polyspec_port as P
        from oracle import sht as osht
        pb = P.PortBase(nside, cltot, np.asarray([b]), pol=False, lmax=lmax)
        pw = P.PortWeightings(pb, mask[None], {'TT': cl['TT']}, np.ones((1, 12 * nside ** 2)))
        pp = P.PortPSpecBin(pb, mask, pw.applySinv_ideal, l_bins, ["TT"])
        t0 = time.time()
        fcpu = np.mean([pp.compute_fisher_contribution(a_lm=np.asarray(base.generate_data(
            seed=s + int(1e7), output_type='harmonic', deconvolve_beam=True))) for s in seeds], axis=0)
        t_cpu = time.time() - t0
        line["cpu_baseline"] = {"value": len(seeds) / t_cpu, "unit": "sims/s", "cores": osht.default_threads(),
                                "kind": "port", "sample": "the same 10 Fisher contributions on the oracle "
                                                          "restatement (FP64, all host threads)"}
        line["fisher_gpu_vs_cpu_max_rel"] = float(np.abs(fish - fcpu).max() / np.abs(fcpu).max())
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    if a.workload == "pspec-t64":
        pspec_t64(a)
        return
    if a.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        run_reference(a)
        return
    run_cuda(a)


if __name__ == "__main__":
    main()
