"""The tile/pipeline autotuner: every candidate tile gives the same transform
(FP64 tiles to 1e-12, mixed tiles to the mixed tolerance 1e-5 of the map), the
choice is the measured fastest, and it is written to and read back from the
JSON cache."""
import json

import pytest


@pytest.mark.gpu
def test_tiles_agree_and_choice_is_cached(tmp_path, monkeypatch):
    import torch
    from polyspec_b200 import _lib
    from polyspec_b200.autotune import TILES
    from polyspec_b200.sht import SHTPlan
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("PS_TUNE_CACHE", str(cache))
    nside, lmax = 32, 64
    ref = SHTPlan(nside, lmax, autotune=False)
    g = torch.Generator(device="cuda").manual_seed(0)
    alm = torch.randn((5, 2, ref.nalm), dtype=torch.complex128, device="cuda", generator=g)
    want = ref.synthesis(alm, 2)
    mx = SHTPlan(nside, lmax, prec="mixed", autotune=False)
    for pipeline, plan, tol in (("fp64", ref, 1e-12), ("mixed", mx, 1e-5)):
        for tile in TILES[(pipeline, 0, True)]:
            _lib.call("ps_plan_set_tile", plan._h, 0, 2, tile)
            got = plan.synthesis(alm, 2)
            assert float((got - want).abs().max() / want.abs().max()) < tol, (pipeline, tile)
        _lib.call("ps_plan_set_tile", plan._h, 0, 2, 0)
    with pytest.raises(_lib.PSError):
        _lib.call("ps_plan_set_tile", ref._h, 0, 2, 3)  # not an allowed tile
    P = SHTPlan(nside, lmax, prec="mixed")
    out = P.synthesis(alm, 2)
    assert float((out - want).abs().max() / want.abs().max()) < 1e-5
    d = json.loads(cache.read_text())
    (key, choice), = [(k, v) for k, v in d.items() if "fp64+mixed|synthesis|spin2|b5" in k]
    assert choice["ms"]["%s/%d" % (choice["pipeline"], choice["tile"])] == min(choice["ms"].values())
    # a new plan reads the choice back without timing again
    P2 = SHTPlan(nside, lmax, prec="mixed")
    P2.synthesis(alm, 2)
    assert P2._tuner.choices[key]["tile"] == choice["tile"]
