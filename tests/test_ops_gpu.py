"""torch.library operators on the GPU: the same results as the SHTPlan calls they wrap
(bit for bit: the same kernels), torch.library.opcheck's schema and fake-tensor checks,
and a capture of the operators in a CUDA graph that replays to the same values."""
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_ops_match_plan_and_graph_replay(prec):
    import torch
    import polyspec_b200.ops as ops
    from polyspec_b200.sht import SHTPlan
    nside, lmax = 16, 40
    g = torch.Generator(device="cuda").manual_seed(3)
    P = SHTPlan(nside, lmax, prec=prec, autotune=False)
    alm = torch.randn((3, 2, P.nalm), dtype=torch.complex128, device="cuda", generator=g)
    m = torch.ops.polyspec.synthesis(alm, nside, lmax, 2, prec)
    ref = P.synthesis(alm, 2)
    torch.cuda.synchronize()
    assert torch.equal(m, ref)
    a = torch.ops.polyspec.adjoint(m, nside, lmax, 2, 0.25, prec)
    assert torch.equal(a, P.adjoint(ref, 2, 0.25))
    for op, args in ((ops.synthesis, (alm, nside, lmax, 2, prec)), (ops.adjoint, (m, nside, lmax, 2, 0.25, prec))):
        torch.library.opcheck(op, args, test_utils=("test_schema", "test_faketensor"))
    # CUDA graph: capture synthesis + adjoint once, replay on new inputs in the same buffers
    x = alm.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        torch.ops.polyspec.adjoint(torch.ops.polyspec.synthesis(x, nside, lmax, 2, prec), nside, lmax, 2, 0.25, prec)
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        y = torch.ops.polyspec.adjoint(torch.ops.polyspec.synthesis(x, nside, lmax, 2, prec), nside, lmax, 2, 0.25, prec)
    x.copy_(torch.randn(x.shape, dtype=torch.complex128, device="cuda", generator=g))
    graph.replay()
    torch.cuda.synchronize()
    want = P.adjoint(P.synthesis(x, 2), 2, 0.25)
    assert torch.equal(y, want)
    del graph


@pytest.mark.gpu
def test_ops_cg_kernels():
    import torch
    import polyspec_b200.ops  # noqa: F401
    from polyspec_b200 import lmops
    g = torch.Generator(device="cuda").manual_seed(4)
    nlm = 500
    S = torch.randn((3, 3, nlm), dtype=torch.float64, device="cuda", generator=g)
    x = torch.randn((2, 3, nlm), dtype=torch.complex128, device="cuda", generator=g)
    w = torch.rand(nlm, dtype=torch.float64, device="cuda", generator=g)
    assert torch.equal(torch.ops.polyspec.lm_matvec3(S, x), lmops.matvec3(S, x))
    assert torch.equal(torch.ops.polyspec.lm_dot(x, x, w), lmops.dot(x, x, w))
