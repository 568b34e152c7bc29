"""Mixed-size SHT serving: the grouped, graph-captured transforms give the same
maps and alm as one SHTPlan call per request (FP64 to 1e-12, mixed to 1e-5 of
the largest value), and a second replay with new inputs gives the new results."""
import pytest


def _requests():
    reqs = []
    for nside in (16, 32):
        for spin in (0, 2):
            for d in ("alm2map", "map2alm"):
                for k in range(2 if nside == 16 else 3):
                    reqs.append(dict(nside=nside, lmax=2 * nside, spin=spin, direction=d))
    return reqs


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_serving_matches_single_calls(prec, tol):
    import torch
    from polyspec_b200.serve import SHTServer
    from polyspec_b200.sht import SHTPlan
    reqs = _requests()
    srv = SHTServer(reqs, prec=prec)
    g = torch.Generator(device="cuda").manual_seed(1)
    for rnd in range(2):
        for x in srv.inputs:
            if x.is_complex():
                x.copy_(torch.randn(x.shape, dtype=torch.complex128, device="cuda", generator=g))
            else:
                x.copy_(torch.randn(x.shape, dtype=torch.float64, device="cuda", generator=g))
        outs = srv.run()
        torch.cuda.synchronize()
        for r, x, y in zip(reqs, srv.inputs, outs):
            P = SHTPlan(r["nside"], r["lmax"], prec=prec, autotune=False)
            src = x[None] if r["spin"] > 0 else x[0][None]
            if r["direction"] == "alm2map":
                want = P.synthesis(src, r["spin"])[0]
            else:
                want = P.adjoint(src, r["spin"], 4.0 * torch.pi / P.npix)[0]
            want = want if r["spin"] > 0 else want[None]
            assert float((y - want).abs().max() / want.abs().max()) < tol, (r, rnd)
