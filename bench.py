"""Benchmark of the projective-dynamics frictional-contact step loop on B200.

One "step" is SimulationBase::step(): detection, LocalGlobal PD iterations
(local step, friction, global solve), write-back.  Workload (N=1): the
500 x 500 cloth (250k vertices) draped over a sphere of radius 0.5 m rotating
about z at 1 rad/s, mu 0.5, self-collision on (tol 2 mm), dt 2e-3; synthetic,
seeded.  Arms, all on the same workload:

  fp64_plain_fixed20 : the reference's method, FP64, 20 PD iterations per step;
                       its mean Alart-Curnier residual after the 20 iterations
                       defines the tolerance tau ("same residual");
  fp64_plain         : FP64, cold start, iterate to tau (cap 60);
  fp32_refine        : FP32 solves of the FP64-residual correction (the PD loop
                       is the refinement), iterate to tau;
  learned            : fp32_refine + learned warm start of the contact forces,
                       iterate to tau (the headline); the cold-start solver
                       judges the warm start on a short stretch of the
                       workload first and replaces it when it does not save
                       iterations.

Iterate-to-tolerance runs as a conditional CUDA-graph loop on the device.
value = the learned arm's whole-job steps/s, timed on the device (CUDA events
on the simulation's stream, max over ranks); every arm's steps/s, iterations
and residual are in the same line.  The warm-start network is trained before
the timed region (untimed) on contacts of a cold run of a sibling scene
(different friction, rotation and initial gap).  e2e = the learned arm through
the public C ABI with host buffers: the state uploaded from pinned memory and
read back every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--n 500] [--workload cloth|batch] [--arm same-residual|fp64|fp32]

Multi-GPU: the single-cloth step loop does not shard (triangular solve and
level-ordered Gauss-Seidel are sequential over the elimination tree), so N
ranks run N independent replicas ("replicas only"); no collective is on the
data path.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s at 250k-vertex cloth: plain FP64 vs FP32+refine+learned, same residual"
PLAIN_ITERATIONS = 20


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                f = [x.strip() for x in out.split(",")]
                if len(f) >= 7:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.1)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if "Active" in s[3 + k]
                          and "Not" not in s[3 + k]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def workload(args):
    from climatenet_b200 import scenes
    if args.workload == "batch":
        s, _, pk = scenes.batch_scene(n_instances=64, seed=4)
    else:
        s, pk, _ = scenes.workload(3, n_override=args.n)
    return s, dict(pk)


def workload_name(args):
    if args.workload == "batch":
        return ("64 independent cloths, n ~ U{20..150} (seed 4), each over its own sphere R ~ U[0.2, 0.5], "
                "mu ~ U[0.1, 0.8], dt=2.5e-3, stepped as one block-diagonal scene")
    return ("%dx%d cloth (%d vertices) on a sphere R=0.5 m rotating about z at 1 rad/s, mu=0.5, "
            "self-collision tol 2 mm, dt=2e-3" % (args.n, args.n, args.n * args.n))


def cpu_baseline(args, steps):
    """The FP64 CPU oracle (restatement of the reference loop, OpenMP) on the host cores."""
    from climatenet_b200 import abi
    from oracle.oracle import Oracle
    s, pk = workload(args)
    pk["iterations"] = PLAIN_ITERATIONS
    t0 = time.time()
    o = Oracle(s, abi.params(**pk))
    setup = time.time() - t0
    o.step(1)  # warm-up
    t0 = time.time()
    for _ in range(steps):
        o.step(1)
    dt = time.time() - t0
    cores = os.cpu_count()
    return {"value": steps / dt, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": "%d steps of the same workload (%d PD iterations, FP64) after 1 warm-up step "
                      "(set-up %.1f s untimed), OMP_NUM_THREADS=%s"
                      % (steps, PLAIN_ITERATIONS, setup, os.environ.get("OMP_NUM_THREADS", cores))}


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = max(1, min(args.steps, 3))
    cb = cpu_baseline(args, steps)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "steps/s", "n_gpus": world,
            "steps": steps, "warmup": 1, "ms_per_step": 1e3 / cb["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args), "pd_iterations": PLAIN_ITERATIONS,
                       "parallelism": "replicas"},
            "cpu_baseline": {k: cb[k] for k in ("kind", "cores", "sample")} | {"value": cb["value"],
                                                                                "unit": "steps/s"},
            "e2e": {"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def train_warm_start(args, tolerance, candidates=4):
    """Untimed: contacts logged from a cold run with 60 PD iterations (forces
    close to converged) of a sibling of the measured scene (same cloth and
    sphere; friction 0.4 instead of 0.5, rotation reversed, 8 mm instead of
    5 mm above the sphere); `candidates` networks trained on the GPU (seeds
    1..candidates); the one needing the fewest PD iterations to reach
    `tolerance` on 10 steps of a second sibling (friction 0.45, rotation
    0.5 rad/s, 6 mm above the sphere: in neither the training data nor the
    measured workload) is kept.  For the batch workload: the batch scene
    itself, validated on the 10 steps after its logged run."""
    from climatenet_b200 import abi, native, scenes, warmstart
    if args.workload == "batch":
        s, _, pk = scenes.batch_scene(n_instances=64, seed=4)
        what, steps = "64-instance batch scene", 200
        sval = None
    else:
        _, pk, _ = scenes.workload(3, n_override=args.n)
        s = scenes.cloth_on_sphere(n=args.n, side=2.0, z=0.008, mu=0.4, sphere_center=(0, 0, -0.5),
                                   sphere_radius=0.5, rotating=-1.0)
        sval = scenes.cloth_on_sphere(n=args.n, side=2.0, z=0.006, mu=0.45, sphere_center=(0, 0, -0.5),
                                      sphere_radius=0.5, rotating=0.5)
        what, steps = "sibling scene (mu 0.4, rotation -1 rad/s, 8 mm gap)", 120
    pk = dict(pk)
    pk["iterations"] = 60
    t0 = time.time()
    X, T, end_state = warmstart.collect(s, abi.params(**pk), steps=steps, capacity=8_000_000, return_state=True)
    t1 = time.time()
    trained = [warmstart.train(X, T, epochs=40, batch=4096, lr=2e-3, seed=seed)
               for seed in range(1, candidates + 1)]
    t2 = time.time()
    pv = dict(pk)
    pv["precision"] = abi.PDF_FP32_REFINE
    if sval is None:
        val_scene, start = s, end_state
    else:
        # the validation sibling from its state after the warm-up steps
        val_scene = sval
        vsim = native.Simulation(sval, abi.params(**pv))
        vsim.step(args.warmup)
        start = vsim.state()
        vsim.close()
    best, stats = warmstart.select(val_scene, pv, [w for w, _ in trained], tolerance, start, steps=10,
                                   cap=3 * PLAIN_ITERATIONS)
    cold = warmstart.cold_stretch(val_scene, pv, tolerance, start, steps=10, cap=3 * PLAIN_ITERATIONS)
    w, info = trained[best]
    # a network that does not beat the cold start on the validation stretch
    # is not offered to the judge
    info["validation_cold"] = cold
    info["beats_cold_on_validation"] = stats[best]["mean_pd_iterations"] < cold["mean_pd_iterations"]
    info.update(collect_s=t1 - t0, train_s=t2 - t1, select_s=time.time() - t2, chosen_seed=best + 1,
                candidates=[dict(seed=k + 1, val_loss=trained[k][1]["val_loss"], **stats[k])
                            for k in range(candidates)],
                data="%s, %d steps, 60 PD iterations, cold start; selection on %s"
                     % (what, steps, "the next 10 steps" if sval is None else
                        "a second sibling (mu 0.45, rotation 0.5 rad/s, 6 mm gap), 10 steps"))
    return w, info


def make_sim(s, pk, iterations, precision, weights=None, device=0, tolerance=0.0):
    from climatenet_b200 import abi, native
    p = dict(pk)
    p["iterations"] = iterations
    p["residual_tolerance"] = tolerance
    p["precision"] = abi.PDF_FP32_REFINE if precision == "fp32" else abi.PDF_FP64
    if weights is not None:
        p["warm_start"] = abi.PDF_WARM_MLP
    prm = abi.params(**p)
    prm.device = device
    sim = native.Simulation(s, prm)
    if weights is not None:
        sim.mlp_set_weights(weights)
    return sim


def residual_pass(sim, steps):
    """Over `steps` steps (a replay of the timed stretch from its start
    state): mean Alart-Curnier residual after the last iteration (steps with
    contacts), mean per-iteration curve (fixed iteration counts only) and mean
    iterations per step."""
    res, curves, its = [], [], []
    for _ in range(steps):
        r = sim.step(1)
        its.append(r.iterations)
        if r.n_contacts + r.n_self_contacts > 0:
            res.append(r.residual)
            curves.append(sim.residual_history())
    curve = []
    if curves and len({len(c) for c in curves}) == 1:
        curve = [float(x) for x in np.mean(np.array(curves), axis=0)]
    return (float(np.mean(res)) if res else 0.0), curve, float(np.mean(its))


def max_over_ranks(value, dist):
    """The largest `value` over all ranks (every rank gets it); the value
    itself without a process group.  Runs on the GPU under NCCL, on the CPU
    under gloo."""
    if dist is None:
        return float(value)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, ms_max):
    """Steps per second of the whole job: every replica runs `steps` steps,
    the job takes as long as its slowest rank."""
    return world * steps / (ms_max / 1e3)


def timed_steps(sim, steps, barrier, dist, device):
    import torch
    s0 = sim.stats()
    barrier()
    with ClockSampler(device) as clk:
        rep = sim.step(steps)
    barrier()
    s1 = sim.stats()
    return (max_over_ranks(rep.device_ms, dist), int(s1.kernel_launches - s0.kernel_launches), clk.summary(),
            (s1.iterations - s0.iterations) / steps)


def e2e_steps(sim, steps, barrier, dist, world, start):
    """Through the C ABI with host buffers: upload (q, v) from pinned memory,
    step, read (q, v) back, every step, starting from the state `start`."""
    import torch
    from climatenet_b200 import native
    q0, v0 = start
    # two pinned (q, v) pairs: each step reads back into the pair the next
    # step uploads from
    bufs = [(torch.from_numpy(q0).pin_memory(), torch.from_numpy(v0).pin_memory())]
    bufs.append((torch.empty_like(bufs[0][0]).pin_memory(), torch.empty_like(bufs[0][1]).pin_memory()))
    L = native.lib()
    barrier()
    t0 = time.perf_counter()
    for k in range(steps):
        qh, vh = bufs[k % 2]
        qo, vo = bufs[(k + 1) % 2]
        native._check(L.pdf_set_state(sim.h, C.c_void_p(qh.data_ptr()), C.c_void_p(vh.data_ptr())), sim.h)
        native._check(L.pdf_step(sim.h, 1, None), sim.h)
        native._check(L.pdf_get_state(sim.h, C.c_void_p(qo.data_ptr()), C.c_void_p(vo.data_ptr())), sim.h)
    barrier()
    return whole_job_rate(world, steps, 1e3 * max_over_ranks(time.perf_counter() - t0, dist))


# DRAM bytes (read + write) of one global solve of the 500 x 500 cloth,
# forward + backward sweep, from ncu's dram__bytes_read.sum +
# dram__bytes_write.sum (a profiler is needed to count them, so they cannot be
# measured inside this run); None for other workloads.
SOLVE_TRAFFIC_500 = {True: 419.2e6, False: 831.8e6}


def roofline(sim, fp32, n=None):
    ms, by = sim.time_phase(0, reps=20)
    pk_ = peaks()
    peak = pk_["hbm_gbs"] if pk_ else 6650.0
    st = sim.stats()
    achieved = by / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "supernodal forward+backward sweeps (one global solve, %s)"
            % ("FP32" if fp32 else "FP64"), "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": SOLVE_TRAFFIC_500[fp32] if n == 500 else None,
            "traffic_unit": "bytes per solve (ncu)", "ms": ms, "algorithmic_bytes": by,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if pk_ else "fallback",
            "factor_elements_stored": st.factor_nnz, "nnz_L": st.factor_nnz_true}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=500)
    ap.add_argument("--workload", default="cloth", choices=["cloth", "batch"])
    ap.add_argument("--arm", default="same-residual", choices=["same-residual", "fp64", "fp32"])
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    s, pk = workload(args)
    N = s.n_vertices
    K = args.steps
    line_extra = {}
    weights = None

    # ---- the reference's method: FP64, 20 PD iterations per step ---------
    sim_r = make_sim(s, pk, PLAIN_ITERATIONS, "fp64", device=local)
    sim_r.step(args.warmup)
    start_state = sim_r.state()
    ms_r, launches_r, clk_r, _ = timed_steps(sim_r, K, barrier, dist, local)
    # residuals over the same stretch of the run, replayed from its start
    sim_r.set_state(*start_state)
    res_r, curve_r, _ = residual_pass(sim_r, K)
    line_extra["fp64_plain_fixed20"] = {"steps_per_s": whole_job_rate(world, K, ms_r), "ms_per_step": ms_r / K,
                                        "pd_iterations": PLAIN_ITERATIONS, "mean_residual": res_r,
                                        "residual_curve": curve_r, "gpu_launches": launches_r}
    line_extra["roofline_fp64"] = roofline(sim_r, False, args.n if args.workload == "cloth" else None)
    if args.arm == "fp64":
        sim, ms, launches, clk, iters, res, prec, tol = (sim_r, ms_r, launches_r, clk_r, PLAIN_ITERATIONS, res_r,
                                                        "fp64", 0.0)
    else:
        sim_r.close()
        # ---- same residual: every arm iterates to tau (the mean residual the
        # reference's method reaches after 20 iterations), cap 60 -----------
        tol = res_r
        # no contact in the stretch (tau = 0): no residual to reach, so the
        # arms run the reference's 20 iterations
        cap = 3 * PLAIN_ITERATIONS if tol > 0 else PLAIN_ITERATIONS
        arms = [("fp64_plain", "fp64", None), ("fp32_refine", "fp32", None)]
        if args.arm == "same-residual":
            from climatenet_b200 import abi, warmstart
            weights, tinfo = train_warm_start(args, tol)
            line_extra["warm_start_training"] = tinfo
            # the cold-start solver judges the learned warm start on a short
            # stretch of the workload and is the fallback when it does not help
            pj = dict(pk)
            pj["precision"] = abi.PDF_FP32_REFINE
            verdict = warmstart.judge(s, pj, weights, tol, steps=10, warmup=args.warmup, cap=cap)
            verdict["use"] = bool(verdict["use"] and tinfo["beats_cold_on_validation"])
            line_extra["warm_start_judge"] = verdict
            if not verdict["use"]:
                weights = None
            arms.append(("learned", "fp32", weights))
        for name, precision, w in arms:
            sim = make_sim(s, pk, cap, precision, w, device=local, tolerance=tol)
            sim.step(args.warmup)
            start_state = sim.state()
            ms, launches, clk, timed_it = timed_steps(sim, K, barrier, dist, local)
            sim.set_state(*start_state)
            res, _, mean_it = residual_pass(sim, K)
            line_extra[name] = {"steps_per_s": whole_job_rate(world, K, ms), "ms_per_step": ms / K,
                                "mean_pd_iterations": timed_it, "mean_pd_iterations_replay": mean_it,
                                "mean_residual": res, "tolerance": tol,
                                "iteration_cap": cap, "gpu_launches": launches}
            if name != arms[-1][0]:
                sim.close()
        prec, iters = "fp32", cap
        head = arms[-1][0]
        line_extra["speedup_same_residual_vs_fp64_plain"] = (line_extra[head]["steps_per_s"] /
                                                            line_extra["fp64_plain"]["steps_per_s"])
        line_extra["speedup_vs_fixed20"] = (line_extra[head]["steps_per_s"] /
                                            line_extra["fp64_plain_fixed20"]["steps_per_s"])

    value = whole_job_rate(world, K, ms)
    # end to end over the same stretch of the run as `value`: from the state
    # the timed steps started from
    e2e_value = e2e_steps(sim, K, barrier, dist, world, start_state)
    roof = roofline(sim, prec == "fp32", args.n if args.workload == "cloth" else None)
    ms_local, bytes_local = sim.time_phase(1, reps=20)
    st = sim.stats()
    if dist is not None:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == "fp64" else "f32 solves + f64 residual / state",
            "data": "synthetic",
            "config": {"workload": workload_name(args), "vertices": N, "arm": args.arm,
                       "pd_iterations": iters, "precision": prec, "residual_tolerance": tol,
                       "warm_start": ("mlp" if weights is not None else
                                      ("none (the cold-start judge rejected the learned warm start)"
                                       if "warm_start_judge" in line_extra else "none")),
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2: factor panels %.0f MB per sweep copy"
                             % (st.factor_nnz * (4 if prec == "fp32" else 8) / 1e6),
                       "nnz_L": st.factor_nnz_true, "supernodes": st.n_supernodes, "etree_levels": st.n_levels,
                       "mean_residual": res},
            "roofline": roof,
            "local_step": {"ms": ms_local, "algorithmic_bytes": bytes_local,
                           "achieved_gbs": bytes_local / (ms_local * 1e-3) / 1e9},
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 2 * 24 * N,
                    "d2h_bytes_per_step": 2 * 24 * N},
            "gpu_launches": launches,
            "clocks": clk,
        }
        line.update(line_extra)
        if not args.no_cpu and world == 1:
            line["cpu_baseline"] = cpu_baseline(args, args.cpu_steps)
        print(json.dumps(line), flush=True)
    sim.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
