"""Mixed-size submission (ps_batch_submit): single-map transforms of two plans, both
directions and spins 0 and 2, some back to back in memory (used in place) and some
scattered (staged through the workspace), must equal, bit for bit, one batched
ps_synthesis / ps_adjoint per group of (plan, direction, spin, scale) on the same
plan.  Also: the workspace query covers the submission, a short workspace and a bad
item are refused before anything runs, and a submission replays in a CUDA graph."""
import ctypes

import pytest


def _plan(nside, lmax, prec):
    from polyspec_b200 import _lib
    h = ctypes.c_void_p()
    _lib.call("ps_plan_create", nside, lmax, lmax, 0b101, prec, ctypes.byref(h))
    return h


def _batched(h, direction, spin, x, scale, npix, nalm):
    """One batched transform of the stacked inputs x [B, ...] on plan h."""
    import torch
    from polyspec_b200 import _lib
    B = x.shape[0]
    nc = 1 if spin == 0 else 2
    if direction == 0:
        out = torch.empty((B, nc, npix), dtype=torch.float64, device="cuda")
    else:
        out = torch.empty((B, nc, nalm), dtype=torch.complex128, device="cuda")
    n = ctypes.c_size_t()
    _lib.call("ps_sht_workspace_bytes", h, B, spin, direction, ctypes.byref(n))
    ws = torch.empty(max(int(n.value), 256), dtype=torch.uint8, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if direction == 0:
        _lib.call("ps_synthesis", h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), B, spin,
                  ctypes.c_void_p(ws.data_ptr()), int(n.value), st)
    else:
        _lib.call("ps_adjoint", h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), B, spin,
                  float(scale), ctypes.c_void_p(ws.data_ptr()), int(n.value), st)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_batch_submit_equals_grouped_transforms(prec):
    import torch
    from polyspec_b200 import _lib
    plans = {16: _plan(16, 31, prec), 32: _plan(32, 63, prec)}
    try:
        info = {}
        for ns, h in plans.items():
            npix, nalm = ctypes.c_int64(), ctypes.c_int64()
            _lib.call("ps_plan_info", h, None, None, ctypes.byref(npix), ctypes.byref(nalm))
            info[ns] = (int(npix.value), int(nalm.value))
        g = torch.Generator(device="cuda").manual_seed(5)

        def rin(ns, direction, spin, B, contiguous):
            npix, nalm = info[ns]
            nc = 1 if spin == 0 else 2
            if direction == 0:
                mk = lambda: torch.randn((nc, nalm), dtype=torch.complex128, device="cuda", generator=g)
            else:
                mk = lambda: torch.randn((nc, npix), dtype=torch.float64, device="cuda", generator=g)
            if contiguous:
                return list(torch.stack([mk() for _ in range(B)]).unbind(0))
            return [mk() for _ in range(B)]

        # (nside, direction, spin, scale, count, contiguous)
        spec = [(32, 0, 0, 1.0, 3, True), (16, 1, 2, 0.5, 2, False), (16, 0, 2, 1.0, 1, True),
                (32, 1, 0, 0.25, 2, False), (32, 1, 0, 2.0, 2, True), (16, 0, 0, 1.0, 2, False)]
        items, expect, outs, inputs = [], [], [], []
        for ns, d, spin, sc, B, contig in spec:
            xs = rin(ns, d, spin, B, contig)
            inputs.append(xs)  # the items hold raw pointers: keep every input alive
            npix, nalm = info[ns]
            ref = _batched(plans[ns], d, spin, torch.stack(xs), sc, npix, nalm)
            if contig:
                o = list(torch.empty_like(ref).unbind(0))
            else:
                o = [torch.empty_like(ref[0]) for _ in range(B)]
            for k in range(B):
                items.append(_lib.WorkItem(plans[ns], d, spin, xs[k].data_ptr(), o[k].data_ptr(), sc))
                expect.append(ref[k])
                outs.append(o[k])
        # interleave the groups' items: grouping must not depend on the order
        order = list(range(0, len(items), 2)) + list(range(1, len(items), 2))
        arr = (_lib.WorkItem * len(items))(*[items[i] for i in order])
        n = ctypes.c_size_t()
        _lib.call("ps_batch_workspace_bytes", arr, len(items), ctypes.byref(n))
        ws = torch.empty(int(n.value), dtype=torch.uint8, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert _lib.lib().ps_batch_submit(arr, len(items), ctypes.c_void_p(ws.data_ptr()), int(n.value) - 256,
                                          st) == -5  # PS_ERR_WORKSPACE
        bad = (_lib.WorkItem * 1)(_lib.WorkItem(plans[16], 2, 0, outs[0].data_ptr(), outs[1].data_ptr(), 1.0))
        assert _lib.lib().ps_batch_submit(bad, 1, ctypes.c_void_p(ws.data_ptr()), int(n.value), st) == -1
        for o in outs:
            o.zero_()
        _lib.call("ps_batch_submit", arr, len(items), ctypes.c_void_p(ws.data_ptr()), int(n.value), st)
        torch.cuda.synchronize()
        for k, (o, e) in enumerate(zip(outs, expect)):
            assert torch.equal(o, e), k
        # the same submission captured once and replayed
        for o in outs:
            o.zero_()
        graph = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            with torch.cuda.graph(graph, stream=s):
                _lib.call("ps_batch_submit", arr, len(items), ctypes.c_void_p(ws.data_ptr()), int(n.value),
                          ctypes.c_void_p(s.cuda_stream))
        graph.replay()
        torch.cuda.synchronize()
        for k, (o, e) in enumerate(zip(outs, expect)):
            assert torch.equal(o, e), k
        del graph
    finally:
        for h in plans.values():
            _lib.lib().ps_plan_destroy(h)
