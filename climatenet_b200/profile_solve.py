"""Runs the global solve of the 500 x 500 cloth workload in isolation, for
profiling: one full step (so that the right-hand side is realistic), then
`reps` back-to-back forward + backward supernodal sweeps.

  python -m climatenet_b200.profile_solve [--n 500] [--reps 3] [--precision fp64|fp32]
"""
import argparse

from . import abi, native, scenes


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=500)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--phase", type=int, default=0)
    args = ap.parse_args()
    s, pk, _ = scenes.workload(3, n_override=args.n)
    if args.precision == "fp32":
        pk["precision"] = abi.PDF_FP32_REFINE
    sim = native.Simulation(s, abi.params(**pk))
    sim.step(1)
    ms, by = sim.time_phase(args.phase, args.reps)
    print("phase %d: %.4f ms per repetition, %.1f MB algorithmic, %.1f GB/s"
          % (args.phase, ms, by / 1e6, by / (ms * 1e-3) / 1e9 if ms > 0 else 0.0))


if __name__ == "__main__":
    main()
