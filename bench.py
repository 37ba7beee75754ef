"""Benchmark of the projective-dynamics frictional-contact step loop on B200.

One "step" is SimulationBase::step(): detection, LocalGlobal PD iterations
(local step, friction, global solve), write-back.  Workload (N=1): the
500 x 500 cloth (250k vertices) draped over a sphere of radius 0.5 m rotating
about z at 1 rad/s, mu 0.5, self-collision on (tol 2 mm), dt 2e-3, 20 PD
iterations per step; synthetic, seeded.  value = whole-job steps/s timed on the
device (CUDA events on the simulation's stream, max over ranks); e2e = the
same metric through the public C-ABI with host buffers (state uploaded from
pinned memory and the new positions read back every step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--precision fp64|fp32] [--n 500]

Multi-GPU: the single-cloth step loop does not shard (triangular solve and
level-ordered Gauss-Seidel are sequential over the elimination tree), so N
ranks run N independent replicas ("replicas only"); no collective is on the
data path.
"""
import argparse
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
            self._stop.wait(0.2)

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


def build_workload(args):
    from climatenet_b200 import abi, scenes
    if args.workload == "batch":
        s, _, pk = scenes.batch_scene(n_instances=64, seed=4)
    else:
        s, pk, _ = scenes.workload(3, n_override=args.n)
    pk = dict(pk)
    if args.precision == "fp32":
        pk["precision"] = abi.PDF_FP32_REFINE
    return s, abi.params(**pk), pk


def workload_name(args):
    if args.workload == "batch":
        return ("64 independent cloths, n ~ U{20..150} (seed 4), each over its own sphere R ~ U[0.2, 0.5], "
                "mu ~ U[0.1, 0.8], dt=2.5e-3, 20 PD iterations/step, stepped as one block-diagonal scene")
    return ("%dx%d cloth (%d vertices) on a sphere R=0.5 m rotating about z at 1 rad/s, mu=0.5, "
            "self-collision tol 2 mm, dt=2e-3, 20 PD iterations/step" % (args.n, args.n, args.n * args.n))


def cpu_baseline(args, steps):
    """The FP64 CPU oracle (restatement of the reference loop, OpenMP) on the host cores."""
    from oracle.oracle import Oracle
    s, p, _ = build_workload(argparse.Namespace(**{**vars(args), "precision": "fp64"}))
    t0 = time.time()
    o = Oracle(s, p)
    setup = time.time() - t0
    o.step(1)  # warm-up
    t0 = time.time()
    for _ in range(steps):
        o.step(1)
    dt = time.time() - t0
    cores = os.cpu_count()
    return {"value": steps / dt, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": "%d steps of the same %dx%d workload after 1 warm-up step (setup %.1f s untimed), "
                      "OMP_NUM_THREADS=%s" % (steps, args.n, args.n, setup, os.environ.get("OMP_NUM_THREADS", cores))}


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = max(1, min(args.steps, 3))
    cb = cpu_baseline(args, steps)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "steps/s", "n_gpus": world,
            "steps": steps, "warmup": 1, "ms_per_step": 1e3 / cb["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args), "parallelism": "replicas"},
            "cpu_baseline": {k: cb[k] for k in ("kind", "cores", "sample")} | {"value": cb["value"],
                                                                                "unit": "steps/s"},
            "e2e": {"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--n", type=int, default=500)
    ap.add_argument("--workload", default="cloth", choices=["cloth", "batch"])
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

    from climatenet_b200 import abi, native
    s, p, pk = build_workload(args)
    p.device = local
    sim = native.Simulation(s, p)
    for _ in range(args.warmup):
        sim.step(1)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    stats0 = sim.stats()
    barrier()
    with ClockSampler(local) as clk:
        rep = sim.step(args.steps)
    barrier()
    stats1 = sim.stats()
    dev_ms = rep.device_ms
    t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dev_ms = float(t.item())
    value = world * args.steps / (dev_ms / 1e3)

    # end to end through the C ABI with host buffers (pinned)
    q0, v0 = sim.state()
    qh = torch.from_numpy(q0).pin_memory()
    vh = torch.from_numpy(v0).pin_memory()
    qout = torch.empty_like(qh).pin_memory()
    import ctypes as C
    L = native.lib()
    e2e_steps = max(3, args.steps // 2)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        native._check(L.pdf_set_state(sim.h, C.c_void_p(qh.data_ptr()), C.c_void_p(vh.data_ptr())), sim.h)
        native._check(L.pdf_step(sim.h, 1, None), sim.h)
        native._check(L.pdf_get_state(sim.h, C.c_void_p(qout.data_ptr()), None), sim.h)
        qh.copy_(qout)
    barrier()
    e2e_t = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * e2e_steps / float(e2e_t.item())

    # roofline of the dominant kernel: the supernodal solve sweeps
    ms_solve, bytes_solve = sim.time_phase(0, reps=20)
    ms_local, bytes_local = sim.time_phase(1, reps=20)
    pk_ = peaks()
    peak = pk_["hbm_gbs"] if pk_ else 6650.0
    st = sim.stats()
    achieved = bytes_solve / (ms_solve * 1e-3) / 1e9
    if dist is not None:
        dist.barrier()
    if rank == 0:
        N = s.n_vertices
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 solves + f64 residual",
            "data": "synthetic",
            "config": {"workload": workload_name(args), "vertices": N, "pd_iterations": pk["iterations"],
                       "precision": args.precision, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2: factor panels %.0f MB per sweep copy"
                             % (st.factor_nnz * (4 if args.precision == "fp32" else 8) / 1e6),
                       "nnz_L": st.factor_nnz_true, "nnz_L_stored": st.factor_nnz,
                       "supernodes": st.n_supernodes, "etree_levels": st.n_levels,
                       "contacts_last_step": rep.n_contacts, "self_contacts_last_step": rep.n_self_contacts,
                       "residual_last_step": rep.residual},
            "roofline": {"bound": "hbm", "kernel": "supernodal forward+backward sweeps (one global solve)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "ms": ms_solve, "algorithmic_bytes": bytes_solve,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if pk_ else "fallback"},
            "local_step": {"ms": ms_local, "algorithmic_bytes": bytes_local,
                           "achieved_gbs": bytes_local / (ms_local * 1e-3) / 1e9},
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 2 * 24 * N,
                    "d2h_bytes_per_step": 24 * N},
            "gpu_launches": int(stats1.kernel_launches - stats0.kernel_launches),
            "clocks": clk.summary(),
        }
        if not args.no_cpu and world == 1:
            line["cpu_baseline"] = cpu_baseline(args, args.cpu_steps)
        print(json.dumps(line), flush=True)
    sim.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
