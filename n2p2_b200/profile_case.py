"""A small, fixed evaluation for profilers (ncu) and quick timings.

    python -m n2p2_b200.profile_case [--molecules 4096] [--potential h2o_52]
                                     [--precision fp64|mixed|bf16]
                                     [--evaluations 5] [--autotune]

Builds a seeded water box (seed 77), sets it on a Prediction of one of the
test potentials, evaluates `--evaluations` times (energy + forces) and
prints the per-stage device times of the last three evaluations.  The
symmetry-function kernel of evaluation k is launch k of that kernel (after
the first evaluation's sizing pass, which launches the neighbor list only).

`--autotune` runs the library's tuner (Prediction.autotune) first and
prints its choice; the tuner launches every configuration, so a capture
that should see launch k takes the printed choice through the
N2P2B_SF_VARIANT / N2P2B_SF_SORT environment variables instead.
"""
from __future__ import annotations

import argparse
import os

from . import synth
from .mode import Prediction

POTENTIALS = os.path.join(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))), "tests", "golden", "potentials")


def main():
    a = argparse.ArgumentParser()
    a.add_argument("--molecules", type=int, default=4096)
    a.add_argument("--potential", default="h2o_52")
    a.add_argument("--precision", default="fp64",
                   choices=["fp64", "mixed", "bf16"])
    a.add_argument("--evaluations", type=int, default=5)
    a.add_argument("--autotune", action="store_true")
    args = a.parse_args()
    box, pos, elem = synth.water_box(args.molecules, 77)
    p = Prediction(os.path.join(POTENTIALS, args.potential))
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_precision(args.precision)
    p.set_structure(pos, elem, box)
    if args.autotune:
        p.evaluate_nnp(True)
        print("autotune", p.autotune(True, 3))
    for _ in range(max(args.evaluations - 3, 1)):
        p.evaluate_nnp(True)
    p.set_profiling(True)
    p.stage_times(True)
    for _ in range(3):
        p.evaluate_nnp(True)
    ms, runs = p.stage_times(True)
    print(args.potential, args.precision, len(elem), "atoms; stage ms "
          "(NL, SF, NN, E, F):", [round(x / runs, 3) for x in ms],
          "energy", p.energy)


if __name__ == "__main__":
    main()
