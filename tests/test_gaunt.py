"""Small-momentum 3j symbols and Gaunt coefficients (ps_gaunt_table) against exact
rational evaluation (Racah's sum on Python integers, oracle/shims/pywigxjpf) for
l up to 3000 and n <= 5: 1e-12 relative where |3j| > 1e-10, 1e-14 of sqrt(1/(2l+1))
absolutely everywhere (including the zeros)."""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle", "shims"))


def _cases(seed, count=3000):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        n = int(rng.integers(0, 6))
        l1 = int(rng.integers(0, 3001))
        l2 = l1 + int(rng.integers(-n, n + 1))
        if l2 < 0:
            continue
        m3 = int(rng.integers(-n, n + 1))
        m1 = int(rng.integers(-l1, l1 + 1)) if l1 else 0
        m2 = -m1 - m3
        if abs(m2) > l2:
            continue
        out.append((l1, l2, n, m1, m2, m3))
    # edges: stretched and zero cases
    out += [(3000, 3005, 5, 3000, -3005, 5), (7, 7, 0, 3, -3, 0), (10, 13, 3, -10, 13, -3), (5, 5, 1, 0, 0, 0)]
    return np.asarray(out, dtype=np.int32)


def test_exact_reference_values():
    import pywigxjpf as W
    c = _cases(1, 50)
    for l1, l2, n, m1, m2, m3 in c:
        v = W.wig3jj(2 * int(l1), 2 * int(l2), 2 * int(n), 2 * int(m1), 2 * int(m2), 2 * int(m3))
        assert abs(v) <= 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("gaunt", [0, 1])
def test_gaunt_table(gaunt):
    import ctypes
    import torch
    import pywigxjpf as W
    from polyspec_b200 import _lib
    c = _cases(7 + gaunt)
    args = torch.as_tensor(c, device="cuda")
    out = torch.empty(len(c), dtype=torch.float64, device="cuda")
    _lib.call("ps_gaunt_table", ctypes.c_void_p(args.data_ptr()), len(c), gaunt, ctypes.c_void_p(out.data_ptr()),
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    got = out.cpu().numpy()
    for (l1, l2, n, m1, m2, m3), g in zip(c.tolist(), got):
        e = W.wig3jj(2 * l1, 2 * l2, 2 * n, 2 * m1, 2 * m2, 2 * m3)
        scale = 1. / math.sqrt(2 * l2 + 1)
        if gaunt:
            t0 = W.wig3jj(2 * l1, 2 * l2, 2 * n, 0, 0, 0)
            f = math.sqrt((2 * l1 + 1) * (2 * l2 + 1) * (2 * n + 1) / (4 * math.pi))
            e, scale = e * t0 * f, scale * scale * f
        assert abs(g - e) <= 1e-14 * scale + 1e-12 * abs(e), (l1, l2, n, m1, m2, m3, g, e)
