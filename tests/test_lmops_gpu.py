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


@pytest.mark.gpu
@pytest.mark.parametrize("B,nlm", [(1, 7), (6, 5000)])
def test_fused_cg_updates(B, nlm):
    """ps_lm_matvec3_add, ps_lm_quad_dot, ps_cg_xr_update (with a slot map into a larger x)
    and ps_cg_direction against the torch FP64 expressions they replace in the CG step."""
    import torch
    from polyspec_b200 import lmops
    g = torch.Generator(device="cuda").manual_seed(10 + B)
    c = lambda *s: torch.randn(s, dtype=torch.complex128, device="cuda", generator=g)
    S = torch.randn((3, 3, nlm), dtype=torch.float64, device="cuda", generator=g)
    S = 0.5 * (S + S.transpose(0, 1))
    w = torch.rand(nlm, dtype=torch.float64, device="cuda", generator=g)
    x, y = c(B, 3, nlm), c(B, 3, nlm)
    want = y + torch.einsum("abi,nbi->nai", S.to(torch.complex128), x)
    lmops.matvec3_add(S, x, y)
    assert float((y - want).abs().max() / want.abs().max()) < 1e-14
    sx = torch.einsum("abi,nbi->nai", S.to(torch.complex128), x)
    want = torch.sum((x * sx.conj()).real * w, dim=(-2, -1))
    got = lmops.quad_dot(S, x, w)
    scale = torch.sum(x.abs() * sx.abs() * w, dim=(-2, -1))
    assert bool(((got - want).abs() <= 1e-13 * scale).all())
    X = c(B + 3, 3, nlm)
    slots = torch.randperm(B + 3, device="cuda", generator=g)[:B]
    alpha = torch.randn(B, dtype=torch.float64, device="cuda", generator=g)
    p, r, q = c(B, 3, nlm), c(B, 3, nlm), c(B, 3, nlm)
    Xw = X.clone()
    Xw[slots] = X[slots] + alpha[:, None, None] * p
    rw = r - alpha[:, None, None] * q
    lmops.xr_update(X, slots, alpha, p, r, q)
    assert torch.allclose(X, Xw, rtol=0, atol=1e-14) and torch.allclose(r, rw, rtol=0, atol=1e-14)
    z = c(B, 3, nlm)
    beta = torch.rand(B, dtype=torch.float64, device="cuda", generator=g)
    pw = z + beta[:, None, None] * p
    lmops.direction(p, z, beta)
    assert torch.allclose(p, pw, rtol=0, atol=1e-14)
