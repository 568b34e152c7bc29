"""PyTorch custom operators over libpscuda (``torch.ops.polyspec.*``).

The C ABI (include/pscuda.h) behind ``torch.library`` ops, so that the transforms and
the CG kernels compose with other torch code: they run on the current CUDA stream,
can be captured in CUDA graphs, and have fake (meta) implementations, so shapes and
dtypes propagate through tracing without a GPU.  Plans are cached per (device,
Nside, lmax, precision); a mixed-precision plan builds its Legendre tables on first
use (``SHTPlan(tables='auto')``).

    torch.ops.polyspec.synthesis(alm, nside, lmax, spin, prec)        # [B, (2,) nalm] -> [B, (2,) npix]
    torch.ops.polyspec.adjoint(map, nside, lmax, spin, scale, prec)   # [B, (2,) npix] -> [B, (2,) nalm]
    torch.ops.polyspec.weighted_roundtrip(alm, weight, lscale, nside, lmax, scale)
    torch.ops.polyspec.lm_matvec3(S, x)                                # [3, 3, nalm] x [B, 3, nalm]
    torch.ops.polyspec.lm_dot(x, y, w)                                 # -> [B]

The reference's map <-> alm calls they replace: ducc0.sht.synthesis and
adjoint_synthesis in polyspec/base.py:145-288; the CG operator and inner product of
polyspec/weighting.py:255, 297-299."""
import torch

from .sht import nalm as _nalm

_PLANS = {}


def _plan(device, nside, lmax, prec):
    from .sht import SHTPlan
    key = (str(device), int(nside), int(lmax), prec)
    p = _PLANS.get(key)
    if p is None:
        p = SHTPlan(int(nside), int(lmax), prec=prec, device=device, autotune=False)
        _PLANS[key] = p
    return p


def _map_shape(alm, nside, spin):
    npix = 12 * nside * nside
    return tuple(alm.shape[:-1]) + (npix,)


@torch.library.custom_op("polyspec::synthesis", mutates_args=())
def synthesis(alm: torch.Tensor, nside: int, lmax: int, spin: int, prec: str) -> torch.Tensor:
    p = _plan(alm.device, nside, lmax, prec)
    return p.synthesis(alm.contiguous(), int(spin))


@synthesis.register_fake
def _(alm, nside, lmax, spin, prec):
    if alm.shape[-1] != _nalm(lmax):
        raise ValueError("alm has %d coefficients, expected %d" % (alm.shape[-1], _nalm(lmax)))
    return alm.new_empty(_map_shape(alm, nside, spin), dtype=torch.float64)


@torch.library.custom_op("polyspec::adjoint", mutates_args=())
def adjoint(map: torch.Tensor, nside: int, lmax: int, spin: int, scale: float, prec: str) -> torch.Tensor:
    p = _plan(map.device, nside, lmax, prec)
    return p.adjoint(map.contiguous(), int(spin), float(scale))


@adjoint.register_fake
def _(map, nside, lmax, spin, scale, prec):
    if map.shape[-1] != 12 * nside * nside:
        raise ValueError("map has %d pixels, expected %d" % (map.shape[-1], 12 * nside * nside))
    return map.new_empty(tuple(map.shape[:-1]) + (_nalm(lmax),), dtype=torch.complex128)


@torch.library.custom_op("polyspec::weighted_roundtrip", mutates_args=())
def weighted_roundtrip(alm: torch.Tensor, weight: torch.Tensor, lscale: torch.Tensor | None, nside: int, lmax: int,
                       scale: float) -> torch.Tensor:
    p = _plan(alm.device, nside, lmax, "mixed")
    out = p.weighted_roundtrip(alm.contiguous(), weight, lscale, float(scale))
    if out is None:
        raise RuntimeError("weighted_roundtrip needs the plan's Legendre tables (ps_sht_weighted_roundtrip)")
    return out


@weighted_roundtrip.register_fake
def _(alm, weight, lscale, nside, lmax, scale):
    if alm.dim() != 3 or alm.shape[1] not in (1, 3):
        raise ValueError("alm must be [B, 1 or 3, nalm]")
    return torch.empty_like(alm)


@torch.library.custom_op("polyspec::lm_matvec3", mutates_args=())
def lm_matvec3(S: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    from . import lmops
    return lmops.matvec3(S.contiguous(), x)


@lm_matvec3.register_fake
def _(S, x):
    if x.dim() != 3 or x.shape[1] != 3 or tuple(S.shape) != (3, 3, x.shape[2]):
        raise ValueError("lm_matvec3 takes S [3, 3, nalm] and x [B, 3, nalm]")
    return torch.empty_like(x)


@torch.library.custom_op("polyspec::lm_dot", mutates_args=())
def lm_dot(x: torch.Tensor, y: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
    from . import lmops
    return lmops.dot(x, y, w.contiguous())


@lm_dot.register_fake
def _(x, y, w):
    if x.shape != y.shape or x.dim() != 3 or x.shape[1] != 3:
        raise ValueError("lm_dot takes x, y [B, 3, nalm]")
    return x.new_empty((x.shape[0],), dtype=torch.float64)
