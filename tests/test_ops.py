"""torch.library operators (polyspec_b200.ops): registration and the fake (meta)
implementations, which give shapes and dtypes without a GPU and refuse mismatched
sizes before anything runs."""
import pytest


def test_ops_fake_shapes():
    import torch
    from torch._subclasses.fake_tensor import FakeTensorMode
    import polyspec_b200.ops  # noqa: F401  (registers torch.ops.polyspec.*)
    nside, lmax = 8, 20
    nalm = (lmax + 1) * (lmax + 2) // 2
    with FakeTensorMode():
        a = torch.empty((5, 2, nalm), dtype=torch.complex128)
        m = torch.ops.polyspec.synthesis(a, nside, lmax, 2, "mixed")
        assert tuple(m.shape) == (5, 2, 12 * nside ** 2) and m.dtype == torch.float64
        b = torch.ops.polyspec.adjoint(m, nside, lmax, 2, 0.5, "mixed")
        assert tuple(b.shape) == (5, 2, nalm) and b.dtype == torch.complex128
        x = torch.empty((4, 3, nalm), dtype=torch.complex128)
        w = torch.empty((3, 12 * nside ** 2), dtype=torch.float64)
        assert tuple(torch.ops.polyspec.weighted_roundtrip(x, w, None, nside, lmax, 1.0).shape) == (4, 3, nalm)
        S = torch.empty((3, 3, nalm), dtype=torch.float64)
        assert tuple(torch.ops.polyspec.lm_matvec3(S, x).shape) == (4, 3, nalm)
        d = torch.ops.polyspec.lm_dot(x, x, torch.empty(nalm, dtype=torch.float64))
        assert tuple(d.shape) == (4,) and d.dtype == torch.float64
        with pytest.raises(ValueError):
            torch.ops.polyspec.synthesis(torch.empty((1, nalm + 1), dtype=torch.complex128), nside, lmax, 0, "fp64")
        with pytest.raises(ValueError):
            torch.ops.polyspec.lm_matvec3(S, torch.empty((4, 2, nalm), dtype=torch.complex128))
