"""Learned band preconditioner: the GPU training kernels against the FP64 CPU
oracle (oracle/mlp.py), the moment / application kernels against their numpy
restatement, and what the trained network gains over the plain harmonic CG.

Tolerances: loss and gradients 1e-3 relative (FP32 activations and
accumulation on the GPU, bf16 weights in both); moments 1e-5, application
1e-6 relative (FP32 moments / correction)."""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import mlp as O  # noqa: E402


def _bf(t):
    return t.to("cpu").to(dtype=__import__("torch").float64).numpy()


@pytest.mark.gpu
def test_training_gradients_match_cpu_oracle():
    import torch
    from polyspec_b200 import learned as Lr
    band_l, D, K, OUT = Lr.lbp_dims()
    nb = 700
    g = np.random.default_rng(0)
    X = torch.as_tensor(g.normal(size=(nb, Lr.F_IN)).astype(np.float32), device="cuda")
    mlp = Lr.MLP(OUT, "cuda", seed=3, out_scale=0.5)
    for p, pb in zip(mlp.params, mlp.bf16):  # non-zero biases, exercised by the check
        if p.dim() == 1:
            p.copy_(torch.as_tensor(g.normal(size=p.shape[0]).astype(np.float32) * 0.1))
            pb.copy_(p.to(torch.bfloat16))
    U = g.normal(size=(nb, 6, D))
    Tt = g.normal(size=(nb, 6, D))
    C = np.einsum("nsd,nse->nde", U, U)
    Gr = np.einsum("nsd,nse->nde", U, Tt)
    G = 0.5 * (Gr + np.transpose(Gr, (0, 2, 1)))
    T = np.einsum("nsd,nsd->n", Tt, Tt)
    dC, dG, dT = (torch.as_tensor(a.astype(np.float32), device="cuda") for a in (C, G, T))
    # GPU: forward, loss/dL, backward
    h1, h2, out = mlp.forward(X)
    dL = torch.empty_like(out)
    lb = torch.empty(nb, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float64, device="cuda")
    scale = 1.0 / float(dT.sum())
    from polyspec_b200 import _lib
    _lib.call("ps_lbp_loss_grad", Lr._vp(out), Lr._vp(dC), Lr._vp(dG), Lr._vp(dT), nb, ctypes.c_float(scale),
              Lr._vp(dL), Lr._vp(lb), Lr._vp(loss), Lr._stream())
    grads = [x.cpu().numpy().astype(np.float64) for x in mlp.backward(X, (h1, h2, out), dL)]
    gpu_loss = float(loss) * scale
    # oracle on the same (bf16-rounded) weights and FP32-rounded moments
    params = [_bf(pb) for pb in mlp.bf16]
    Xo = X.cpu().numpy().astype(np.float64)
    want_loss, want = O.loss_and_grads(Xo, params, dC.cpu().numpy().astype(np.float64),
                                       dG.cpu().numpy().astype(np.float64), dT.cpu().numpy().astype(np.float64), D, K)
    assert abs(gpu_loss - want_loss) <= 1e-3 * abs(want_loss)
    for gg, ww in zip(grads, want):
        assert np.linalg.norm(gg - ww) <= 1e-3 * np.linalg.norm(ww)


def _spd_sigma(nalm, g):
    A = g.normal(size=(nalm, 3, 3))
    S = np.einsum("nab,ncb->nac", A, A) + 0.5 * np.eye(3)
    return np.ascontiguousarray(np.moveaxis(S, 0, 2))  # [3, 3, nalm]


@pytest.mark.gpu
@pytest.mark.parametrize("lmax", [20, 47])
def test_moments_and_apply_match_oracle(lmax):
    import torch
    from polyspec_b200 import learned as Lr, _lib
    band_l, D, K, OUT = Lr.lbp_dims()
    ms, l0s, nls, idx = Lr.band_blocks(lmax, band_l)
    nb = len(ms)
    nalm = (lmax + 1) * (lmax + 2) // 2
    g = np.random.default_rng(lmax)
    sigma = _spd_sigma(nalm, g)
    B = 3
    r = g.normal(size=(B, 3, nalm)) + 1j * g.normal(size=(B, 3, nalm))
    e = g.normal(size=(B, 3, nalm)) + 1j * g.normal(size=(B, 3, nalm))
    w = g.uniform(0.5, 2.0, size=B)
    d = {k: torch.as_tensor(v, device="cuda") for k, v in dict(sigma=sigma, r=r, e=e, w=w).items()}
    didx, dnl = torch.as_tensor(idx, device="cuda"), torch.as_tensor(nls, device="cuda")
    C = torch.zeros((nb, D, D), dtype=torch.float32, device="cuda")
    G = torch.zeros_like(C)
    T = torch.zeros(nb, dtype=torch.float32, device="cuda")
    for _ in range(2):  # accumulation across calls
        _lib.call("ps_lbp_moments", Lr._vp(didx), Lr._vp(dnl), nb, Lr._vp(d["r"]), Lr._vp(d["e"]), Lr._vp(d["w"]),
                  Lr._vp(d["sigma"]), B, nalm, Lr._vp(C), Lr._vp(G), Lr._vp(T), Lr._stream())
    blocks = list(zip(idx.tolist(), nls.tolist()))
    Co, Go, To = O.moments(blocks, r, e, w, sigma, band_l)
    for got, want in ((C, 2 * Co), (G, 2 * Go), (T, 2 * To)):
        got = got.cpu().numpy()
        assert np.max(np.abs(got - want)) <= 1e-5 * np.max(np.abs(want))
    Lm = g.normal(size=(nb, OUT)).astype(np.float32)  # L (row-major D x K), then q
    z = torch.einsum("abi,nbi->nai", d["sigma"].to(torch.complex128), d["r"]).contiguous()
    dLm = torch.as_tensor(Lm, device="cuda")
    _lib.call("ps_lbp_apply", Lr._vp(didx), Lr._vp(dnl), nb, Lr._vp(dLm), Lr._vp(d["sigma"]), Lr._vp(d["r"]),
              Lr._vp(z), B, nalm, Lr._stream())
    want = O.apply(blocks, Lm.astype(np.float64), sigma, r, band_l)
    got = z.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want))


@pytest.mark.gpu
def test_trained_network_against_plain_cg():
    """What the trained network gains over the plain harmonic CG, at the same
    residual tolerance, on a workload whose operator couples nearby l of an m
    (full sky, latitude-dependent noise): both solvers reach r^T Sigma r /
    b^T Sigma b < 1e-8 on the recomputed true residual, the training loss falls,
    and the learned CG takes at least 5 % fewer steps than the plain one over 8
    solves (measured: 98 plain, 80 learned).  On the masked benchmark workload
    the band network does not gain -- its band blocks cannot represent the per-m
    coupling of the masked equatorial band or the holes (Nside 256: 2815 learned
    vs 796 harmonic steps for 33 solves; on top of the masked-band
    preconditioner 117 vs 63) -- so the benchmark runs the masked-band
    preconditioner."""
    import torch
    from polyspec_b200 import PolySpec, Weightings
    from polyspec_b200 import workloads as W
    from polyspec_b200.learned import LearnedBandPreconditioner
    nside, lmax = 16, 32
    cl, cltot, beam, mask, noise = W.anisotropic_noise_setup(nside, lmax, amp=8.0, fwhm_arcmin=300.0, depth=300.0)
    base = PolySpec(nside, dict(cltot), beam=list(beam), pol=True, lmax=lmax, autotune=False)
    wts = Weightings(base, mask, dict(cl), noise_cov=noise)
    dnoise = torch.as_tensor(noise, device="cuda")

    def maps(seed, B=8):
        g = torch.Generator(device="cuda").manual_seed(seed)
        out = []
        for i in range(B):
            a = base.generate_data(seed=seed * 100 + i, output_type="harmonic", rng="device")
            out.append(base.to_map(a) + torch.sqrt(dnoise) * torch.randn(dnoise.shape, dtype=torch.float64,
                                                                        device="cuda", generator=g))
        return torch.stack(out)

    lp = LearnedBandPreconditioner(wts)
    for s in range(3):
        lp.collect(maps(10 + s), nstep=200)
    hist = lp.train(epochs=300, lr=2e-3)
    assert hist[-1] < 0.5 * hist[0]
    wts.learned = lp
    test = maps(99)
    its = {}
    for pre in ("harmonic", "learned"):
        wts.batched_applySinv_optimal(test, preconditioner=pre, nstep=200, thresh=1e-8)
        cg = wts.last_cgd
        b0 = cg._get_b(test)
        r = b0 - cg._apply_A(cg.x0 + cg.x)
        sig = lambda v: torch.einsum('abi,nbi->nai', wts.d_Sigma, v)
        assert bool((cg.dot(r, sig(r)) / cg.dot(b0, sig(b0)) < 1e-7).all()), pre
        its[pre] = int(cg.iters.sum())
    print("CG steps over 8 solves: plain %d, learned %d" % (its["harmonic"], its["learned"]))
    assert its["learned"] <= 0.95 * its["harmonic"], its
