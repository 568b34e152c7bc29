"""Small fixed workloads for profiling the kernels under ncu.

    python -m polyspec_b200.profile_cli sht --nside 1024 --lmax 2048 --ops s0,a0,s2,a2 [--batch 1]

Each op runs once (no warm-up) so that a launch list or an ncu capture of
``-k <kernel> -c 1`` sees exactly one launch per transform stage.
ops: s0/a0 = spin-0 synthesis/adjoint, s2/a2 = spin-2 synthesis/adjoint.
"""
import argparse
import sys

import torch


def sht(a):
    from polyspec_b200.sht import SHTPlan
    P = SHTPlan(a.nside, a.lmax, prec=a.prec)
    B = a.batch
    alm0 = torch.randn(B, P.nalm, dtype=torch.complex128, device="cuda")
    map0 = torch.randn(B, P.npix, dtype=torch.float64, device="cuda")
    alm2 = torch.randn(B, 2, P.nalm, dtype=torch.complex128, device="cuda")
    map2 = torch.randn(B, 2, P.npix, dtype=torch.float64, device="cuda")
    for op in a.ops.split(","):
        if op == "s0":
            P.synthesis(alm0, 0)
        elif op == "a0":
            P.adjoint(map0, 0)
        elif op == "s2":
            P.synthesis(alm2, 2)
        elif op == "a2":
            P.adjoint(map2, 2)
        else:
            raise SystemExit("unknown op " + op)
    torch.cuda.synchronize()
    print("done", a.ops)


def main(argv=None):
    p = argparse.ArgumentParser()
    sub = p.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("sht")
    s.add_argument("--nside", type=int, default=1024)
    s.add_argument("--lmax", type=int, default=2048)
    s.add_argument("--batch", type=int, default=1)
    s.add_argument("--prec", default="fp64")
    s.add_argument("--ops", default="s0,a0,s2,a2")
    a = p.parse_args(argv)
    if a.cmd == "sht":
        sht(a)


if __name__ == "__main__":
    sys.exit(main())
