"""Runs parts of the 500 x 500 cloth workload for profiling.

Default: one full step (so that the right-hand side is realistic), then
`reps` back-to-back repetitions of one phase in isolation (0 = global solve:
forward + backward supernodal sweeps and the write-back, 1 = local step,
2 = contact projection, 3 = detection).  With --steps K: K full steps of the
step loop instead (for a launch list of whole steps).  With --mlp-samples M:
one forward and one gradient launch of the warm-start MLP on M seeded random
samples instead (for the tensor-pipe counters of k_mlp_forward / k_mlp_grad).
With --window: the measured repetitions (or steps) are bracketed by
cudaProfilerStart / cudaProfilerStop, so that a profiler started with
`--profile-from-start off` sees only them (not the schedule autotuner's
solves at create).  --schedule CHUNK,CUT,MODE,SHAPE pins the solve schedule
after create.

  python -m climatenet_b200.profile_solve [--n 500] [--reps 3] [--precision fp64|fp32]
                                          [--phase 0] [--steps 0] [--iterations 20]
                                          [--mlp-samples 0] [--window]
                                          [--schedule 64,4,1,1]
"""
import argparse
import time

import numpy as np

from . import abi, native, scenes


class _null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class _profiler_window:
    """cudaProfilerStart / cudaProfilerStop around a block (CUDA runtime)."""

    def __init__(self):
        from cuda.bindings import runtime as rt
        self.rt = rt

    def __enter__(self):
        err, = self.rt.cudaProfilerStart()
        if int(err) != 0:
            raise RuntimeError("cudaProfilerStart failed: %s" % err)
        return self

    def __exit__(self, *exc):
        self.rt.cudaProfilerStop()
        return False


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=500)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--phase", type=int, default=0)
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--mlp-samples", type=int, default=0)
    ap.add_argument("--window", action="store_true")
    ap.add_argument("--schedule", default="")
    args = ap.parse_args()
    if args.mlp_samples > 0:
        rng = np.random.default_rng(0)
        X = rng.standard_normal((args.mlp_samples, 10)).astype(np.float32)
        T = rng.standard_normal((args.mlp_samples, 3)).astype(np.float32)
        w = native.mlp_init(1)
        t0 = time.time()
        native.mlp_forward(w, X)
        native.mlp_gradient(w, X, T)
        print("MLP forward + gradient on %d samples: %.3f s wall (host copies included)"
              % (args.mlp_samples, time.time() - t0))
        return
    s, pk, _ = scenes.workload(3, n_override=args.n)
    pk["iterations"] = args.iterations
    if args.precision == "fp32":
        pk["precision"] = abi.PDF_FP32_REFINE
    sim = native.Simulation(s, abi.params(**pk))
    if args.schedule:
        sim.set_sweep_schedule(*[int(t) for t in args.schedule.split(",")])
    st = sim.stats()
    print("schedule: cut level %d, %d blocks, chunk %d, upper mode %d, block shape %d; solve ms per cut level %s"
          % (st.sweep_cut_level, st.sweep_blocks, st.sweep_chunk, st.sweep_upper_mode, st.sweep_block_shape,
             [round(x, 4) for x in st.sweep_cut_ms]))
    sim.step(1)
    window = _profiler_window() if args.window else None
    if args.steps > 0:
        with window or _null():
            r = sim.step(args.steps)
        print("%d steps: %.3f ms per step on the device, %d PD iterations in the last step"
              % (args.steps, r.device_ms / args.steps, r.iterations))
        return
    with window or _null():
        ms, by = sim.time_phase(args.phase, args.reps)
    print("phase %d: %.4f ms per repetition, %.1f MB algorithmic, %.1f GB/s"
          % (args.phase, ms, by / 1e6, by / (ms * 1e-3) / 1e9 if ms > 0 else 0.0))


if __name__ == "__main__":
    main()
