"""Writes stochasticphysics_b200/flops_table.json: algorithmic work per particle-step.

Counts come from running the oracle's restated formulas with an operation-
counting scalar (adds, subtracts and multiplies; a fused multiply-add counts 2;
divisions, transcendental calls and square roots separately; noise generation
excluded).  bench.py reads the table to express throughput as FLOP/s.

    python oracle/make_flops_table.py
"""
import dataclasses
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from stochasticphysics_b200 import provider  # noqa: E402
from stochasticphysics_b200._abi import Anisotropy, Problem, Solver  # noqa: E402


def main():
    table = {}
    for problem in Problem:
        for aniso in Anisotropy:
            for solver in Solver:
                if solver == Solver.Implicit_Midpoint and problem == Problem.BrownAndNeelEulerSpherical:
                    continue
                if problem in (Problem.BrownAndNeelEulerSpherical, Problem.BrownAndNeel):
                    spec = provider.brown_neel_relaxation(n=8, steps=4000, oversampling=100)
                else:
                    spec = provider.neel_relaxation(n=8, steps=4000, oversampling=100)
                spec = dataclasses.replace(spec, problem=problem, anisotropy=aniso, solver=solver,
                                           use_coordinate_transformation=problem == Problem.NeelSpherical)
                if aniso == Anisotropy.Cubic:
                    spec = dataclasses.replace(spec, anisotropy_constant=spec.anisotropy_constant * 0 - 1.1e4,
                                               magnetisation=provider.cubic_easy_direction(
                                                   problem if problem != Problem.BrownAndNeel else Problem.Neel,
                                                   spec.orientation))
                ops = oracle.count_ops(spec)
                table[f"{problem.name}/{aniso.name}/{solver.name}"] = {k: round(v, 3) for k, v in ops.items()}
    out = ROOT / "stochasticphysics_b200" / "flops_table.json"
    out.write_text(json.dumps({"definition": "per particle-step: flops = adds+subs+muls (FMA = 2) of the "
                               "restated reference formulas incl. the Kahan window sum; divs, transcendentals, "
                               "sqrts counted separately; Philox/Box-Muller excluded",
                               "table": table}, indent=1))
    print(f"wrote {out} ({len(table)} entries)")


if __name__ == "__main__":
    main()
