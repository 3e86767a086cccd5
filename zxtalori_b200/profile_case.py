"""Small fixed workloads for profiling the engine's kernels (for example under Nsight
Compute), each a few relaxation steps of one sample through the public API:

    python -m zxtalori_b200.profile_case near      # O, N=100,000 Haar (seed 193), delta 20
    python -m zxtalori_b200.profile_case pairs     # O, N=16,384 Haar (seed 193), all pairs
    python -m zxtalori_b200.profile_case spacing   # I, N=1,000,000 Haar (seed 7), spacing pass

`--steps` sets the number of relaxation steps (default 2) or, for spacing, of spacing
passes; `--count` the spacing sample's size. Prints the resulting energy or separation, so a
run can be checked against a plain one.
"""
from __future__ import annotations

import argparse

import zxtalori_b200 as zo


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["near", "pairs", "spacing"])
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--count", type=int, default=1_000_000)
    args = p.parse_args(argv)
    if args.case == "near":
        with zo.haar("O", 100_000, 193) as g:
            g.relax(args.steps, neighbourhood=20)
            print(g.stats["energy"])
    elif args.case == "pairs":
        with zo.haar("O", 16_384, 193) as g:
            g.relax(args.steps)
            print(g.stats["energy"])
    else:
        with zo.haar("I", args.count, 7) as g:
            for _ in range(max(1, args.steps)):
                separation = g.spacing()["separation_deg"]
            print(separation)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
