"""CG vector kernels (ps_lm_matvec3, ps_lm_dot) against torch FP64 references
of the same operations: 3x3 per-(l, m) products with optional per-field scales
to 1e-14, the m-weighted inner product to 1e-13 relative."""
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("B,nlm", [(1, 7), (5, 1000), (33, 20000)])
def test_matvec3_and_dot(B, nlm):
    import torch
    from polyspec_b200 import lmops
    g = torch.Generator(device="cuda").manual_seed(B)
    S = torch.randn((3, 3, nlm), dtype=torch.float64, device="cuda", generator=g)
    x = torch.randn((B, 3, nlm), dtype=torch.complex128, device="cuda", generator=g)
    y = torch.randn((B, 3, nlm), dtype=torch.complex128, device="cuda", generator=g)
    pre = torch.rand((3, nlm), dtype=torch.float64, device="cuda", generator=g)
    post = torch.rand((3, nlm), dtype=torch.float64, device="cuda", generator=g)
    want = torch.einsum("abi,nbi->nai", S.to(torch.complex128), x)
    got = lmops.matvec3(S, x)
    assert float((got - want).abs().max() / want.abs().max()) < 1e-14
    want = post[None] * torch.einsum("abi,nbi->nai", S.to(torch.complex128), pre[None] * x)
    got = lmops.matvec3(S, x, pre=pre, post=post)
    assert float((got - want).abs().max() / want.abs().max()) < 1e-14
    w = torch.rand(nlm, dtype=torch.float64, device="cuda", generator=g)
    want = torch.sum((x * y.conj()).real * w, dim=(-2, -1))
    got = lmops.dot(x, y, w)
    scale = torch.sum((x.abs() * y.abs()) * w, dim=(-2, -1))
    assert bool(((got - want).abs() <= 1e-13 * scale).all())
    assert torch.equal(lmops.dot(x, y, w), got)  # fixed-order sums
