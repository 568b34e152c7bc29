"""Mixed-size SHT serving: many map2alm / alm2map requests of different Nside,
lmax and spin run as a few batched transforms, captured once in a CUDA graph
and replayed (no counterpart in the reference, which calls ducc0 per map).

    srv = SHTServer([dict(nside=256, lmax=512, spin=2, direction="alm2map"), ...])
    for req, x in zip(srv.requests, srv.inputs):  # static input views
        x.copy_(...)
    outs = srv.run()                               # graph replay, output views

Requests are grouped by (Nside, lmax, spin, direction); each group is one
batched libpscuda transform (tile shapes and pipeline from the autotuner, tuned
in a warm-up pass before capture); all groups share one workspace, since the
graph runs them one after the other on one stream.  Inputs and outputs are
static buffers owned by the server: a replay overwrites the previous outputs.
Layouts as in `SHTPlan`: alm complex128 [ncomp, nalm], maps float64 [ncomp, npix]
(ncomp 1 for spin 0, 2 for spin s).
"""
import ctypes

import torch

from . import _lib
from .sht import SHTPlan, nalm as _nalm


class SHTServer:
    def __init__(self, requests, prec="mixed", use_graph=True, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("the CUDA backend needs a GPU (no CPU fallback)")
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.requests = [dict(r) for r in requests]
        self.prec = prec
        groups = {}
        for i, r in enumerate(self.requests):
            if r["direction"] not in ("alm2map", "map2alm"):
                raise ValueError("direction must be 'alm2map' or 'map2alm'")
            key = (int(r["nside"]), int(r["lmax"]), int(r["spin"]), r["direction"])
            groups.setdefault(key, []).append(i)
        # largest transforms first
        self.groups = sorted(groups.items(), key=lambda kv: -(kv[0][0] ** 2 * len(kv[1])))
        self.plans = {}
        for (nside, lmax, spin, d), idx in self.groups:
            if (nside, lmax) not in self.plans:
                self.plans[(nside, lmax)] = SHTPlan(nside, lmax, spins=(0, 2), prec=prec, device=self.device)
        # static inputs / outputs per group, and per-request views
        self.inputs = [None] * len(self.requests)
        self._gin, self._gout = [], []
        need = 0
        for (nside, lmax, spin, d), idx in self.groups:
            nc = 1 if spin == 0 else 2
            P = self.plans[(nside, lmax)]
            B = len(idx)
            if d == "alm2map":
                x = torch.zeros((B, nc, P.nalm), dtype=torch.complex128, device=self.device)
            else:
                x = torch.zeros((B, nc, P.npix), dtype=torch.float64, device=self.device)
            self._gin.append(x)
            for j, i in enumerate(idx):
                self.inputs[i] = x[j]
            for h in (P._h, P._h64 if B <= 8 else None):  # the autotuner tries FP64 for small batches only
                if h is None:
                    continue
                n = ctypes.c_size_t()
                _lib.call("ps_sht_workspace_bytes", h, B, spin, int(d == "map2alm"), ctypes.byref(n))
                need = max(need, int(n.value))
        # one workspace for every plan: the groups run one after the other
        self._ws = torch.empty(max(need, 256), dtype=torch.uint8, device=self.device)
        for P in self.plans.values():
            P._ws = self._ws
        self.graph = None
        self.outputs = None
        self._warm()
        if use_graph:
            self._capture()

    def _run_groups(self):
        outs = []
        for ((nside, lmax, spin, d), idx), x in zip(self.groups, self._gin):
            P = self.plans[(nside, lmax)]
            src = x if spin > 0 else x[:, 0]
            if d == "alm2map":
                y = P.synthesis(src, spin)
            else:
                y = P.adjoint(src, spin, 4.0 * torch.pi / P.npix)
            outs.append(y if spin > 0 else y[:, None])
        return outs

    def _warm(self):
        """One untimed pass: autotuning of every group's shape, lazy kernel set-up."""
        with torch.cuda.device(self.device):
            self._run_groups()
            torch.cuda.synchronize()

    def _capture(self):
        with torch.cuda.device(self.device):
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self._run_groups()  # allocations of the graph's outputs settle on this stream first
            torch.cuda.current_stream().wait_stream(s)
            torch.cuda.synchronize()
            with torch.cuda.graph(g):
                self._gout = self._run_groups()
            self.graph = g

    def run(self):
        """Run every request; returns the outputs in request order (views, valid until the next run)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._gout = self._run_groups()
        out = [None] * len(self.requests)
        for ((key, idx), y) in zip(self.groups, self._gout):
            for j, i in enumerate(idx):
                out[i] = y[j]
        return out

    def maps_per_call(self):
        return len(self.requests)
