"""Learned band preconditioner for the masked CG S^-1 filter (no counterpart in
the reference, whose CG offers 'harmonic' and 'pseudo_inverse' only,
polyspec/weighting.py:301-324).

    M r = Sigma r + S^1/2 L_b L_b^T S^1/2 r

on band blocks b = (m, 16 consecutive l, fields T/E/B), Sigma the harmonic
preconditioner, S = diag(Sigma).  ``L_b`` (48 x 4) is the output of a 3-layer
MLP (ReLU, bf16 weights, FP32 accumulation) evaluated on features of the block
(m, l, signal-to-noise of each field, Fourier features).  M is linear,
symmetric and M >= Sigma for any network output, so the reference's PCG
update applies unchanged.

Training (``train``): plain harmonic-preconditioned CG runs on a set of
right-hand sides twice -- once to its solution x*, once more to collect, at
every step k, the pair (r_k, e_k = x* - x_k) (A e_k = r_k).  The pairs are
reduced on the device into per-block moments; the loss
    J = Sum_k w_k || S^-1/2 (M r_k - e_k) ||^2 ,  w_k = 1 / ||S^-1/2 e_k||^2
is minimised by Adam through libpscuda's own forward/backward kernels.

Use: ``Weightings.applySinv_optimal(..., preconditioner='learned')`` (and the
batched form) with ``Weightings.learned`` set to a trained instance.  The CG
stops on the M-independent test  r^T Sigma r / b^T Sigma b < thresh  -- the
plain CG's own rz/rz0 -- so both solvers meet the same residual tolerance; a
system that the learned CG has not converged within its step limit is
finished by the plain CG from where it stopped (the fallback).
"""
import ctypes

import numpy as np
import torch

from . import _lib

F_IN = 32      # input features (padded)
HIDDEN = 64


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def lbp_dims():
    v = [ctypes.c_int() for _ in range(4)]
    _lib.call("ps_lbp_dims", *[ctypes.byref(x) for x in v])
    return tuple(int(x.value) for x in v)  # (band l, block dim, rank, outputs)


def band_blocks(lmax, band_l):
    """(m, l0, n_valid, alm index of (l0, m)) of every band block, m-major."""
    ms, l0s, nls, idx = [], [], [], []
    for m in range(lmax + 1):
        base = m * (2 * lmax + 1 - m) // 2
        for l0 in range(m, lmax + 1, band_l):
            ms.append(m)
            l0s.append(l0)
            nls.append(min(band_l, lmax + 1 - l0))
            idx.append(base + l0)
    return (np.asarray(ms), np.asarray(l0s), np.asarray(nls, dtype=np.int32), np.asarray(idx, dtype=np.int64))


def block_features(lmax, ms, l0s, nls, snr):
    """Network inputs of each block: position in (l, m), signal-to-noise of T, E, B
    at the block centre (log10, scaled), Fourier features; padded to F_IN."""
    lc = l0s + 0.5 * (nls - 1)
    f = [ms / lmax, lc / lmax, (lc - ms) / lmax, nls / 16.0, ms / (lc + 1.0), np.ones_like(lc)]
    li = np.clip(np.round(lc).astype(int), 0, lmax)
    for k in range(3):
        f.append(np.log10(1e-12 + snr[k][li]) / 6.0)
    for k in (1, 2, 4):
        f += [np.sin(np.pi * k * ms / lmax), np.cos(np.pi * k * ms / lmax),
              np.sin(np.pi * k * lc / lmax), np.cos(np.pi * k * lc / lmax)]
    X = np.stack(f, axis=1)
    out = np.zeros((len(ms), F_IN), dtype=np.float32)
    out[:, :X.shape[1]] = X
    return out


class MLP:
    """3-layer MLP F_IN -> HIDDEN -> HIDDEN -> OUT with FP32 master weights, bf16
    copies for the forward pass, Adam state; every step runs libpscuda kernels."""

    def __init__(self, out_dim, device, seed=0, out_scale=0.02):
        g = np.random.default_rng(seed)
        dims = [(HIDDEN, F_IN), (HIDDEN, HIDDEN), (out_dim, HIDDEN)]
        self.dims = dims
        self.params = []
        for li, (o, i) in enumerate(dims):
            std = np.sqrt(2.0 / i) if li < 2 else out_scale / np.sqrt(i)
            W = torch.as_tensor(g.normal(0.0, std, size=(o, i)).astype(np.float32), device=device)
            b = torch.zeros(o, dtype=torch.float32, device=device)
            self.params += [W, b]
        self.bf16 = [p.to(torch.bfloat16) for p in self.params]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.grads = [torch.zeros_like(p) for p in self.params]
        self.step_count = 0

    def forward(self, X):
        """Returns (h1, h2, out), all FP32 [n, *]."""
        n = X.shape[0]
        acts = []
        h = X
        for li, (o, i) in enumerate(self.dims):
            y = torch.empty((n, o), dtype=torch.float32, device=X.device)
            _lib.call("ps_mlp_dense_forward", _vp(h), _vp(self.bf16[2 * li]), _vp(self.bf16[2 * li + 1]), n, i, o,
                      int(li < 2), _vp(y), _stream())
            acts.append(y)
            h = y
        return acts

    def backward(self, X, acts, d_out):
        """Gradients of all parameters from dLoss/d_out (d_out is overwritten)."""
        n = X.shape[0]
        ins = [X, acts[0], acts[1]]
        dY = d_out
        for li in (2, 1, 0):
            o, i = self.dims[li]
            nb = ctypes.c_size_t()
            _lib.call("ps_mlp_dense_backward_workspace_bytes", n, i, o, ctypes.byref(nb))
            ws = torch.empty(max(int(nb.value), 8), dtype=torch.uint8, device=X.device)
            dX = torch.empty((n, i), dtype=torch.float32, device=X.device) if li > 0 else None
            _lib.call("ps_mlp_dense_backward", _vp(dY), _vp(acts[li]), _vp(ins[li]), _vp(self.bf16[2 * li]), n, i, o,
                      int(li < 2), _vp(dX), _vp(self.grads[2 * li]), _vp(self.grads[2 * li + 1]), _vp(ws),
                      int(nb.value), _stream())
            dY = dX
        return self.grads

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        for p, g, m, v, pb in zip(self.params, self.grads, self.m, self.v, self.bf16):
            _lib.call("ps_mlp_adam", _vp(p), _vp(g), _vp(m), _vp(v), _vp(pb), p.numel(), float(lr), float(beta1),
                      float(beta2), float(eps), self.step_count, _stream())


class LearnedBandPreconditioner:
    """``base='harmonic'``: M = Sigma + S^1/2 (L L^T + d I) S^1/2 on band blocks, trained on the
    plain CG's (r, e) pairs.  ``base='cut'``: the same correction on top of the masked-band
    preconditioner, M = M_cut + S^1/2 (L L^T + d I) S^1/2 (M_cut >= Sigma, so M stays SPD),
    trained on the pairs of the cut-preconditioned CG with targets e - M_cut r: the network
    only has to learn what M_cut leaves."""

    def __init__(self, weightings, seed=0, base='harmonic'):
        self.W = weightings
        self.base = weightings.base
        if base not in ('harmonic', 'cut'):
            raise ValueError("base must be 'harmonic' or 'cut'")
        self.base_prec = base
        self.cut = weightings.cut_preconditioner() if base == 'cut' else None
        if not self.base.pol:
            raise ValueError("the learned band preconditioner works on T, E, B (pol=True)")
        dev = self.base.device
        self.device = dev
        self.band_l, self.D, self.K, self.OUT = lbp_dims()
        lmax = self.base.lmax
        ms, l0s, nls, idx = band_blocks(lmax, self.band_l)
        self.nb = len(ms)
        self.d_idx0 = torch.as_tensor(idx, device=dev)
        self.d_nl = torch.as_tensor(nls, device=dev)
        # signal-to-noise per field and l: C_ff b^2 / N_f
        Cl = weightings.Cl_l_mat  # [L, 3, 3]
        beam = np.asarray(self.base.beam)
        snr = [Cl[:, k, k] * beam[k][:len(Cl)] ** 2 / weightings.Nl_iso[k] for k in range(3)]
        self.X = torch.as_tensor(block_features(lmax, ms, l0s, nls, snr), device=dev)
        self.mlp = MLP(self.OUT, dev, seed=seed)
        self.sigma_c = weightings.d_Sigma                     # [3, 3, nlm] complex128 (for einsum with alm)
        self.sigma = weightings.d_Sigma.real.contiguous()     # [3, 3, nlm] float64 (kernel argument)
        self.L = None
        self.history = []
        self._reset_moments()

    # ---------------------------------------------------------------- moments
    def _reset_moments(self):
        dev = self.device
        self.C = torch.zeros((self.nb, self.D, self.D), dtype=torch.float32, device=dev)
        self.G = torch.zeros_like(self.C)
        self.T = torch.zeros(self.nb, dtype=torch.float32, device=dev)
        self.n_pairs = 0

    def add_pairs(self, r, e):
        """Accumulate (residual, error) pairs r, e: complex128 [B, 3, nlm] with A e = r."""
        r = r.contiguous()
        e = e.contiguous()
        # w = 1 / ||S^-1/2 e||^2 per pair (real and imaginary parts, m-weighted as the CG's dot)
        S = torch.diagonal(self.sigma, dim1=0, dim2=1).T  # [3, nlm]
        inv = torch.where(S > 0, 1.0 / S, torch.zeros_like(S))
        wm = self.base.dev('m_weight')
        en = torch.sum((e.real ** 2 + e.imag ** 2) * inv[None] * wm, dim=(1, 2))
        w = torch.where(en > 0, 1.0 / en, torch.zeros_like(en)).contiguous()
        _lib.call("ps_lbp_moments", _vp(self.d_idx0), _vp(self.d_nl), self.nb, _vp(r), _vp(e), _vp(w),
                  _vp(self.sigma), r.shape[0], r.shape[-1], _vp(self.C), _vp(self.G), _vp(self.T), _stream())
        self.n_pairs += r.shape[0]

    def collect(self, maps, nstep=300, thresh_solve=1e-12, thresh_collect=1e-8):
        """Run the plain CG on maps [B, 3, Npix] twice: to x* (residual thresh_solve),
        then again collecting (r_k, x* - x_k) at every step until the residual falls
        below thresh_collect (well above thresh_solve, so that x* - x_k is accurate)."""
        from .weighting import BatchedCGD
        W = self.W
        x0 = torch.einsum('abi,nbi->nai', W.d_x0op, self.base.to_lm_batch(maps))
        cg = BatchedCGD(W, maps, x0, preconditioner=self.base_prec)
        cg.run(nstep=nstep, thresh=thresh_solve)
        xstar = cg.x.clone()
        cg = BatchedCGD(W, maps, x0, preconditioner=self.base_prec)

        def target(r, e):  # what the learned correction has to supply on top of the base operator
            return e if self.cut is None else e - self.cut.apply(r)
        self.add_pairs(cg.r, target(cg.r, xstar - cg.x))
        for _ in range(nstep):
            if not bool(cg.active.any()):
                break
            cg.step()
            cg.active &= ~(cg.err < thresh_collect)
            idx = cg.slots  # the rows of cg.r: the systems that took this step
            if idx.numel():
                self.add_pairs(cg.r, target(cg.r, xstar[idx] - cg.x[idx]))
        return cg

    # ---------------------------------------------------------------- training
    def loss_and_grad(self):
        """Normalised loss (1 at L = 0) and dLoss/dL for the current network."""
        h1, h2, out = self.mlp.forward(self.X)
        tot = float(self.T.sum())
        scale = 1.0 / max(tot, 1e-30)
        dL = torch.empty_like(out)
        lb = torch.empty(self.nb, dtype=torch.float32, device=self.device)
        loss = torch.empty(1, dtype=torch.float64, device=self.device)
        _lib.call("ps_lbp_loss_grad", _vp(out), _vp(self.C), _vp(self.G), _vp(self.T), self.nb,
                  ctypes.c_float(scale), _vp(dL), _vp(lb), _vp(loss), _stream())
        return float(loss) * scale, (h1, h2, out), dL

    def train(self, epochs=300, lr=2e-3, verbose=False):
        for ep in range(epochs):
            loss, acts, dL = self.loss_and_grad()
            self.mlp.backward(self.X, acts, dL)
            self.mlp.adam(lr)
            self.history.append(loss)
            if verbose and (ep % 50 == 0 or ep == epochs - 1):
                print("learned preconditioner epoch %d: loss %.4f" % (ep, loss))
        self.finalize()
        return self.history

    def finalize(self):
        """Evaluate the network once; the CG applies the stored L."""
        self.L = self.mlp.forward(self.X)[2].contiguous()

    # ---------------------------------------------------------------- application
    def apply(self, r):
        """M r for r complex128 [B, 3, nlm]."""
        if self.cut is not None:
            z = self.cut.apply(r).contiguous()
        else:
            z = torch.einsum('abi,nbi->nai', self.sigma_c, r).contiguous()
        if self.L is None:
            return z
        r = r.contiguous()
        _lib.call("ps_lbp_apply", _vp(self.d_idx0), _vp(self.d_nl), self.nb, _vp(self.L), _vp(self.sigma), _vp(r),
                  _vp(z), r.shape[0], r.shape[-1], _stream())
        return z
