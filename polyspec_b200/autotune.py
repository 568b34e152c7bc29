"""Autotuner of the SHT's Legendre tile shapes and pipeline (no reference
counterpart; the reference's ducc0 picks its own blocking internally).

For each (direction, spin, batch bucket) of a plan the first call times every
candidate -- the mixed-precision pipeline with each allowed number of maps per
CTA of its Legendre kernels, and (for batches of up to 8 maps) the FP64
pipeline with each of its allowed tiles (ps_plan_set_tile) -- with CUDA
events, after one untimed run, and keeps the fastest.  Results are kept per process and in a JSON cache keyed by GPU
model, Nside, lmax and the call's shape, so later processes reuse them; the
cache file is $PS_TUNE_CACHE, default ~/.cache/polyspec_b200/tune.json.
"""
import ctypes
import json
import os

import torch

from . import _lib

# allowed maps per CTA (as ps_plan_set_tile accepts them): [pipeline][direction][spin > 0]
TILES = {
    ("mixed", 0, False): (8, 16, 32), ("mixed", 0, True): (4, 8),
    ("mixed", 1, False): (1, 8), ("mixed", 1, True): (1, 4),
    ("fp64", 0, False): (1, 4), ("fp64", 0, True): (1, 2),
    ("fp64", 1, False): (1, 4), ("fp64", 1, True): (1,),
}


def cache_path():
    return os.environ.get("PS_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "polyspec_b200",
                                                        "tune.json"))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _save(d):
    try:
        p = cache_path()
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + ".tmp%d" % os.getpid()
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except Exception:
        pass


class Tuner:
    """Per-plan tile and pipeline choices; `handles` maps pipeline name -> plan handle."""

    def __init__(self, nside, lmax, handles, device):
        self.handles = dict(handles)
        try:
            gpu = torch.cuda.get_device_name(device)
        except Exception:
            gpu = "gpu"
        # the candidate set is part of the key: an FP64-only plan and a mixed plan (which
        # may also run the FP64 pipeline) tune separately
        self.prefix = "%s|nside%d|lmax%d|%s" % (gpu, nside, lmax, "+".join(sorted(self.handles)))
        self.choices = {}
        self.disk = _load()

    @staticmethod
    def bucket(B):
        if B <= 8:
            return B
        b = 16
        while b < B:
            b *= 2
        return b

    def _set(self, pipeline, direction, spin, tile):
        _lib.call("ps_plan_set_tile", self.handles[pipeline], direction, spin, tile)

    def select(self, direction, spin, B, run, table=False):
        """Handle to run the transform with (its tile already set); `run(handle)` issues it.
        With `table` the mixed plan streams its Legendre table (ps_plan_build_table): its
        on-the-fly tile shapes do not apply, and the choice is cached under its own key."""
        key = "%s|%s|spin%d|b%d%s" % (self.prefix, ("synthesis", "adjoint")[direction], spin, self.bucket(B),
                                      "|tab" if table else "")
        choice = self.choices.get(key) or self.disk.get(key)
        if choice is None or choice.get("pipeline") not in self.handles:
            times = {}
            # the FP64 pipeline only competes for small batches (its workspace is twice the mixed one's)
            cands = [pl for pl in self.handles if not (pl == "fp64" and len(self.handles) > 1 and B > 8)]
            for pipeline in cands:
                tiles = (0,) if (table and pipeline == "mixed") else TILES[(pipeline, direction, spin > 0)]
                for tile in tiles:
                    self._set(pipeline, direction, spin, tile)
                    h = self.handles[pipeline]
                    run(h)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    run(h)
                    e1.record()
                    torch.cuda.synchronize()
                    times["%s/%d" % (pipeline, tile)] = e0.elapsed_time(e1)
            best = min(times, key=times.get)
            pipeline, tile = best.split("/")
            choice = {"pipeline": pipeline, "tile": int(tile), "ms": times}
            self.disk[key] = choice
            _save(self.disk)
        self.choices[key] = choice
        self._set(choice["pipeline"], direction, spin, choice["tile"])
        return self.handles[choice["pipeline"]]
