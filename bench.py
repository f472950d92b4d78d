"""Benchmark: 2D vector Hodge Laplacian (delta d + d delta) on a 1-form,
4096 x 4096 nodes, FP64, single fused pass (the DEC operator throughput
workload), on N GPUs of one node.

A step is one Laplacian of the whole 4096^2 field.  The field (268 MB in,
268 MB out) is larger than the 126 MB L2, so consecutive steps stream from
HBM without an explicit flush.  Multi-GPU: every rank runs its own field
(independent problems, no collective on the data path; weak scaling); the
timed region is bracketed by a barrier and a device synchronisation and the
reported time is the maximum over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload laplacian|solve|mag3d]

--impl reference times the reference algorithm's CPU path (the oracle's
C++/OpenMP restatement, reference-structured staged chain) on the host cores,
on the same 4096^2 field.

On one GPU the default line also carries two records beside the headline
(--no-solve leaves them out): "config1", the 512^2 scalar Laplacian timed warm
and L2-flushed cold with its oracle parity, and "solve", the 64-problem
batched 2D magnetostatics time-to-1e-10 of the plain FP64, FP32-inner and
learned solvers with every solution checked by the oracle's FP64 operator.

Secondary workloads (one JSON line each, not the headline):
  --workload solve   batched 2D magnetostatics: 64 problems of {128..1024}^2
                     nodes, time to a 1e-10 FP64 relative residual with the
                     plain FP64 solver, FP32-inner / FP64-refinement, and the
                     learned preconditioner (weights similie_b200/data/precond_2d.npy);
                     under torchrun the problems shard across ranks by work
  --workload mag3d   batched 3D curl-curl + gauge penalty on stretched grids
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_NODES = 4096
WORKLOAD = "2D vector Hodge Laplacian (delta d + d delta) of a 1-form, 4096x4096 nodes, spacing 1/4096, FP64, fused single pass"
METRIC = "DEC op GB/s: 2D vector Hodge Laplacian, 1-form, 4096^2, FP64"


def algorithmic_bytes(n, es=8):
    """Read the 1-form once (n^2 nodes x 2 comps), write the (n-1)^2 x 2 result once."""
    return (n * n * 2 + (n - 1) * (n - 1) * 2) * es


def cell_updates(n):
    return (n - 1) * (n - 1)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def ncu_traffic(name):
    """DRAM bytes per launch from a committed ncu summary (profiles/<name>), if present."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device_index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread is not None:
                self.thread.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(names, parts[2:6]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_baseline(steps=1, warmup=1, sample_n=N_NODES, seed=2):
    """Oracle staged chain (stored Hodge tensors, separate passes, FP64) on the
    workload's own sample_n^2 field (the full 4096^2 field by default, the same
    input the GPU arm reads); the staged set-up (Hodge fill) is excluded, as
    the reference's staged constructor is, and `warmup` untimed runs come
    first."""
    import oracle as O
    from tests.helpers import gaussian_random_field
    w = gaussian_random_field(sample_n, seed=seed)
    coords = [np.arange(sample_n) / N_NODES, np.arange(sample_n) / N_NODES]
    pos = O.position_from_coords(coords)
    t0 = time.perf_counter()
    st = O.StagedLaplacian(2, 1, pos)
    setup_s = time.perf_counter() - t0
    out = np.zeros((sample_n - 1, sample_n - 1, 2))
    for _ in range(max(warmup, 0)):
        st.run(w, out)
    times = []
    for _ in range(max(steps, 1)):
        t0 = time.perf_counter()
        st.run(w, out)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    gbs = algorithmic_bytes(sample_n) / t / 1e9
    what = "the full 4096^2 1-form" if sample_n == N_NODES else f"a {sample_n}x{sample_n} sample of the 4096^2 1-form"
    return {"value": gbs, "unit": "GB/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"{what}, reference-structured staged chain (d+star, transposed d+star, star, "
                      f"transposed d+star, d, add), Hodge fill excluded ({setup_s:.1f} s), "
                      f"median of {len(times)} runs after {max(warmup, 0)} warm-up",
            "cell_updates_per_s": cell_updates(sample_n) / t, "seconds_per_sample": t,
            "seconds_per_step": times, "same_config": sample_n == N_NODES}


def run_reference(args):
    """The reference algorithm's CPU path (the oracle's staged chain on all
    host threads) on the same 4096^2 FP64 field as the GPU arm: W untimed
    warm-up applies, then K timed applies; rank 0 only."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    os.environ.setdefault("OMP_PROC_BIND", "close")
    cb = cpu_baseline(steps=max(args.steps, 1), warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["seconds_per_sample"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded k^-2 Gaussian random field)",
        "config": {"workload": WORKLOAD, "sample": cb["sample"], "l2": "inputs larger than L2"},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solve", action="store_true",
                    help="leave the configuration-1 and configuration-3 records out of the default line")
    ap.add_argument("--extras", action="store_true", help="also time the unfused chain, FP32 and the 512^2 0-form")
    ap.add_argument("--workload", default="laplacian",
                    choices=["laplacian", "solve", "mag3d", "precond", "hodge3d", "apply3d", "nonlinear",
                             "nonlinear3d", "assembled"])
    ap.add_argument("--n2d", type=int, default=257, help="nonlinear: nodes per axis")
    ap.add_argument("--chunk", type=int, default=64, help="solve: problems per solver call (at most 64 for learned)")
    ap.add_argument("--concurrent", type=int, default=1,
                    help="solve: solver calls in flight at once (host threads, one stream and one network each)")
    ap.add_argument("--solvers", default="cg,mixed,learned", help="solve / mag3d: solver kinds to time")
    ap.add_argument("--max-iterations", type=int, default=200000, help="solve / mag3d: iteration budget")
    ap.add_argument("--shapes", default=None, help="precond: NxC (C grids of N^2 nodes); default the 64-problem batch")
    ap.add_argument("--sizes", default=None, help="solve: comma-separated grid sizes drawn from (default 128..1024)")
    ap.add_argument("--seed", type=int, default=7, help="solve: problem seed")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="solve / mag3d: also time the oracle's FP64 CPU CG on this many problems of the batch")
    ap.add_argument("--count", type=int, default=None, help="solve / mag3d: problems per batch (64 / 8)")
    ap.add_argument("--n3d", type=int, default=256, help="mag3d: nodes per axis")
    ap.add_argument("--nl3d", type=int, default=25, help="nonlinear3d: nodes per axis")
    ap.add_argument("--asm-n", type=int, default=512, help="assembled: nodes per axis of the 2D problem")
    ap.add_argument("--nodes", type=int, default=N_NODES,
                    help="headline field size (nodes per axis) for profiling runs; the benchmark is 4096")
    ap.add_argument("--kernel-only", action="store_true",
                    help="warm-up + timed launches of the fused kernel only (profiling runs): no e2e, extras or CPU leg")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "solve":
        run_solve_workload(args)
        return
    if args.workload == "mag3d":
        run_mag3d_workload(args)
        return
    if args.workload == "nonlinear":
        run_nonlinear_workload(args)
        return
    if args.workload == "nonlinear3d":
        run_nonlinear3d_workload(args)
        return
    if args.workload == "assembled":
        run_assembled_workload(args)
        return
    if args.workload == "precond":
        run_precond_workload(args)
        return
    if args.workload == "hodge3d":
        import torch
        import similie_b200.magnetostatics3d as m3
        torch.cuda.set_device(0)
        x = m3.stretched_coords(args.n3d, 1.01)
        print(json.dumps({"metric": f"3D Hodge star 1-form -> 2-form, {args.n3d}^3, FP64",
                          "hodge": hodge3d_gbs(torch, x, x.copy(), x.copy(), steps=args.steps)}))
        return
    if args.workload == "apply3d":
        import torch
        import similie_b200.magnetostatics3d as m3
        torch.cuda.set_device(0)
        prob = m3.synthetic_problem(np.random.default_rng(5), args.n3d)
        mu = torch.from_numpy(prob.node_mu()).cuda()
        print(json.dumps({"metric": f"3D curl-curl + gauge-penalty apply, {args.n3d}^3, FP64",
                          "apply": apply3d_gbs(torch, prob, mu, steps=args.steps)}))
        return

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    import similie_b200 as sil
    from tests.helpers import gaussian_random_field

    n = args.nodes
    w_host = gaussian_random_field(n, seed=2 + rank)
    coords = [np.arange(n) / n, np.arange(n) / n]
    geo = sil.Geometry(coords)
    inp = torch.from_numpy(w_host).cuda()
    out = torch.empty((n - 1, n - 1, 2), device="cuda", dtype=torch.float64)
    plan = sil.make_staged_laplacian(geo, out, inp, 1)
    assert plan.kernel == 2, "the 4096^2 FP64 1-form must take the TMA kernel"
    stream = torch.cuda.current_stream()

    def barrier():
        if pg is not None:
            pg.barrier()

    # nvidia-smi samples every 200 ms, longer than the timed region itself, so
    # the sampler starts one second earlier with the GPU busy on the same
    # kernel (untimed preheat), then the W warm-up steps, then the timed steps.
    clocks = ClockSampler(local).__enter__()
    t_pre = time.perf_counter()
    while time.perf_counter() - t_pre < 1.0:
        for _ in range(50):
            plan.run(out, inp)
        torch.cuda.synchronize()
    for _ in range(args.warmup):
        plan.run(out, inp)
    torch.cuda.synchronize()
    plan.status()

    # Device-timed region: the K launches run back to back from one CUDA
    # graph (captured after the warm-up, replayed once untimed), bracketed by
    # CUDA events on the launching stream, so neither the host's launch rate
    # nor per-launch events pace the kernels.
    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        plan.run(out, inp)
    stream.wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(args.steps):
            plan.run(out, inp)
    graph.replay()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with clocks:
        t_start.record(stream)
        graph.replay()
        t_end.record(stream)
        torch.cuda.synchronize()
    barrier()
    total_ms = t_start.elapsed_time(t_end)
    plan.status()
    if pg is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    bytes_per_step = algorithmic_bytes(n)
    value = world * bytes_per_step * args.steps / (total_ms * 1e-3) / 1e9
    avg_launch_ms = total_ms / args.steps  # launches back to back: the kernel's steady-state duration
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_step / (avg_launch_ms * 1e-3) / 1e9
    traffic = ncu_traffic("lap2d_1form_tma_4096_fp64.md")

    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": world * bytes_per_step * args.steps / (total_ms * 1e-3) / 1e9,
                              "unit": "GB/s", "ms_per_step": ms_per_step, "kernel_only": True, "nodes": n}))
        if pg is not None:
            pg.destroy_process_group()
        return

    # End to end through the public API with host buffers: every step copies
    # its input from pinned host memory, runs the Laplacian and copies the
    # result back.  Steps are pipelined over three streams (H2D, compute,
    # D2H) with two device buffers each, so step s+1's upload and step s-1's
    # download overlap step s's kernel; events order each buffer's reuse.
    h_in = torch.from_numpy(w_host).pin_memory()
    h_out = [torch.empty((n - 1, n - 1, 2), dtype=torch.float64).pin_memory() for _ in range(2)]
    d_in = [torch.empty_like(inp) for _ in range(2)]
    d_out = [torch.empty_like(out) for _ in range(2)]
    s_up, s_run, s_down = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev_up = [torch.cuda.Event() for _ in range(2)]
    ev_run = [torch.cuda.Event() for _ in range(2)]
    ev_down = [torch.cuda.Event() for _ in range(2)]
    ev_in_free = [torch.cuda.Event() for _ in range(2)]

    def e2e_steps_run(count):
        for st in range(count):
            b = st % 2
            with torch.cuda.stream(s_up):
                if st >= 2:
                    s_up.wait_event(ev_in_free[b])
                d_in[b].copy_(h_in, non_blocking=True)
                ev_up[b].record(s_up)
            s_run.wait_event(ev_up[b])
            if st >= 2:
                s_run.wait_event(ev_down[b])
            plan.run(d_out[b], d_in[b], stream=s_run)
            ev_run[b].record(s_run)
            ev_in_free[b].record(s_run)
            with torch.cuda.stream(s_down):
                s_down.wait_event(ev_run[b])
                h_out[b].copy_(d_out[b], non_blocking=True)
                ev_down[b].record(s_down)

    e2e_steps = max(4, min(args.steps, 20))
    e2e_steps_run(4)
    torch.cuda.synchronize()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for sx in (s_up, s_run, s_down):
        sx.wait_event(e0)
    e2e_steps_run(e2e_steps)
    for sx in (s_up, s_run, s_down):
        stream.wait_stream(sx)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    if pg is not None:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * bytes_per_step * e2e_steps / (e2e_ms * 1e-3) / 1e9

    extras = {}
    if args.extras and rank == 0:
        extras = run_extras(torch, sil, geo, inp, out, args)
    # configurations 1 and 3 beside the headline (one GPU: the batch would
    # otherwise shard across ranks, as --workload solve does)
    secondary = {}
    if rank == 0 and world == 1 and not args.no_solve:
        secondary["config1"] = config1_record(torch, sil)
        secondary["solve"] = solve_record(torch)

    if rank == 0:
        cb = None
        if not args.no_cpu_baseline and world == 1:
            cb = cpu_baseline(steps=2, warmup=1)
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded k^-2 Gaussian random field per component)",
            "config": {"workload": WORKLOAD, "global_batch": world, "nodes_per_rank": [n, n],
                       "parallelism": f"independent fields x{world}", "l2": "inputs larger than L2 (268 MB in + 268 MB out per step)",
                       "kernel": "lap2d_1form_tma_kernel<double>", "pipeline_variant": plan.variant,
                       "cell_updates_per_s": world * cell_updates(n) * args.steps / (total_ms * 1e-3)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6650 GB/s",
                         "traffic": traffic, "algorithmic_bytes_per_launch": bytes_per_step,
                         "avg_launch_ms": avg_launch_ms,
                         "timing": f"{args.steps} launches back to back from one CUDA graph, CUDA events around the replay",
                         "traffic_source": "profiles/lap2d_1form_tma_4096_fp64.md (steady state: mean over 4 "
                                           "back-to-back launches without cache flushes)"},
            "cpu_baseline": cb,
            "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": int(n * n * 2 * 8),
                    "d2h_bytes_per_step": int((n - 1) * (n - 1) * 2 * 8), "steps": e2e_steps,
                    "ms_per_step": e2e_ms / e2e_steps,
                    "pipelining": "H2D, kernel and D2H of consecutive steps on three streams, two buffers each"},
            "gpu_launches": args.steps,
            "clocks": dict(clocks.summary() or {}, window="1 s preheat on the same kernel + warm-up + timed region"),
        }
        line.update(secondary)
        if extras:
            line["extras"] = extras
        print(json.dumps(line))
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def run_extras(torch, sil, geo, inp, out, args):
    """Secondary measurements (not the headline): unfused chain, FP32, 512^2 0-form."""
    from tests.helpers import sinusoid_field
    res = {}
    n = N_NODES

    def timed(fn, steps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    unf = sil.make_staged_laplacian(geo, out, inp, 1, mode="unfused")
    ms = timed(lambda: unf.run(out, inp), 10)
    res["unfused_fp64"] = {"ms": ms, "GB/s_algorithmic": algorithmic_bytes(n) / ms / 1e6,
                           "scratch_bytes": unf.scratch_bytes}
    gen_ms = timed(lambda: sil.laplacian(geo, out, inp, 1), 10)
    res["table_driven_fused_fp64"] = {"ms": gen_ms, "GB/s_algorithmic": algorithmic_bytes(n) / gen_ms / 1e6}
    i32 = inp.float()
    o32 = torch.empty((n - 1, n - 1, 2), device="cuda", dtype=torch.float32)
    p32 = sil.make_staged_laplacian(geo, o32, i32, 1)
    ms32 = timed(lambda: p32.run(o32, i32), 20)
    res["fused_fp32"] = {"ms": ms32, "GB/s_algorithmic": algorithmic_bytes(n, 4) / ms32 / 1e6, "kernel": p32.kernel}
    m = 512
    phi = torch.from_numpy(sinusoid_field(m, seed=1)[..., None].copy()).cuda()
    g2 = sil.Geometry([np.arange(m) / m, np.arange(m) / m])
    o2 = torch.empty((m - 1, m - 1, 1), device="cuda", dtype=torch.float64)
    p2 = sil.make_staged_laplacian(g2, o2, phi, 0)
    ms2 = timed(lambda: p2.run(o2, phi), 50)
    res["scalar_512_fp64"] = {"ms": ms2, "cell_updates_per_s": (m - 1) ** 2 / (ms2 * 1e-3),
                              "GB/s_algorithmic": (m * m + (m - 1) ** 2) * 8 / ms2 / 1e6, "note": "L2 resident"}
    return res


def weights_path():
    """The learned preconditioner's weights: $SIMILIE_B200_WEIGHTS, else the shipped file."""
    return os.environ.get("SIMILIE_B200_WEIGHTS") or os.path.join(ROOT, "similie_b200", "data", "precond_2d.npy")


def load_network():
    """The trained network (weights_path()), or None when the file is absent."""
    from similie_b200.precond import LearnedPreconditioner
    weights = weights_path()
    if not os.path.exists(weights):
        return None, weights
    net = LearnedPreconditioner(seed=0)
    net.load(weights)
    return net, weights


def oracle_residuals(probs, sols):
    """FP64 true relative residual ||b - A x|| / ||b|| of every solution, by the oracle's operator."""
    import oracle as O
    out = []
    for p, x in zip(probs, sols):
        b = p.rhs()
        r = b - O.mag2d_apply(p.nx, p.ny, p.node_mu(), x.cpu().numpy())
        out.append(float(np.linalg.norm(r) / np.linalg.norm(b)))
    return out


def time_solver_kinds(torch, probs, kinds, net, weights=None, chunk=64, concurrent=1, max_iterations=200000):
    """Time each solver kind on the batch (device-resident inputs, a fresh
    zero initial guess per kind) and check every problem's solution with the
    oracle's FP64 operator."""
    import similie_b200.magnetostatics as mag
    from similie_b200 import dist as sd
    from similie_b200.precond import LearnedPreconditioner
    shapes = [(p.nx, p.ny) for p in probs]
    mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    results = {}
    for kind in kinds:
        sols = [torch.zeros_like(r) for r in rhss]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        chunk = min(chunk, 64)  # the learned solver takes 64 problems per call
        slices = [slice(c0, c0 + chunk) for c0 in range(0, len(probs), chunk)]
        per_chunk = [None] * len(slices)

        def run(mine, stream, pnet):
            for ci in mine:
                sl = slices[ci]
                per_chunk[ci] = mag.solve_batch(
                    mus[sl], rhss[sl], sols[sl], shapes[sl], solver=kind, tol=1e-10,
                    max_iterations=max_iterations, inner_iterations=min(4000, max_iterations),
                    preconditioner=pnet if kind == "learned" else None,
                    stream=None if stream is None else stream.cuda_stream)

        workers = max(1, min(concurrent, len(slices)))
        if workers == 1:
            run(range(len(slices)), None, net)
        else:
            # solver calls in flight together on their own streams, so one
            # call's straggling problems overlap the others' work
            nets = [net] + [LearnedPreconditioner(seed=0) for _ in range(workers - 1)]
            if kind == "learned":
                for extra in nets[1:]:
                    extra.load(weights)
            streams = [torch.cuda.Stream() for _ in range(workers)]
            torch.cuda.synchronize()
            threads = [threading.Thread(target=run, args=(range(w, len(slices), workers), streams[w], nets[w]))
                       for w in range(workers)]
            for th in threads:
                th.start()
            for th in threads:
                th.join()
        d = [x for part in per_chunk for x in part]
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        rels = oracle_residuals(probs, sols)
        # concurrent calls run on their own streams: time them by the host
        # clock between device-wide synchronisations
        sec = sd.max_over_ranks(e0.elapsed_time(e1) / 1e3 if workers == 1 else wall, device="cuda")
        results[kind] = {"seconds": sec, "wall_seconds": wall, "solves_per_s": len(probs) / sec,
                         "converged": sum(x.converged for x in d),
                         "converged_by_oracle": sum(r <= 1e-10 for r in rels),
                         "max_iterations": max(x.iterations for x in d),
                         "median_iterations": float(np.median([x.iterations for x in d])),
                         "total_iterations": int(sum(x.iterations for x in d)),
                         "fallbacks": sum(x.fallback for x in d),
                         "median_learned_iterations": float(np.median([x.learned_iterations for x in d])),
                         "max_rel_residual_gpu": max(x.final_relative_residual for x in d),
                         "max_rel_residual_oracle": max(rels), "problems_checked_by_oracle": len(rels)}
    return results


def solve_record(torch, kinds=("cg", "mixed", "learned"), seed=7, count=64):
    """Configuration 3 inside the default line: the 64-problem batch of
    {128..1024}^2 grids (seed 7) solved to a 1e-10 relative residual by the
    plain FP64 solver, FP32-inner / FP64-refinement and the learned
    preconditioner, every solution checked by the oracle's FP64 operator."""
    import similie_b200.magnetostatics as mag
    t0 = time.perf_counter()
    probs = mag.synthetic_batch(seed=seed, count=count)
    net, weights = load_network()
    kinds = [k for k in kinds if k != "learned" or net is not None]
    setup = time.perf_counter() - t0
    # untimed one-iteration solves first: the solver's one-time work-item
    # tuning (first large batch per precision) and the network's workspace
    # happen there, as in any long-running caller
    import similie_b200.magnetostatics as mag_w
    wmus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    wrhs = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    for kind in kinds:
        mag_w.solve_batch(wmus, wrhs, [torch.zeros_like(r) for r in wrhs], [(p.nx, p.ny) for p in probs],
                          solver=kind, max_iterations=1, preconditioner=net if kind == "learned" else None)
    del wmus, wrhs
    torch.cuda.synchronize()
    res = time_solver_kinds(torch, probs, kinds, net, weights)
    base = res["cg"]["seconds"] if "cg" in res else None
    return {"metric": "time-to-1e-10 relative residual (FP64, checked by the oracle's operator), batch of "
                      f"{count} 2D magnetostatics problems",
            "workload": f"{count} problems, sizes uniform over {{128,256,384,512,768,1024}}^2 (seed {seed}), "
                        "1-8 coils, 0-3 permeability-1000 rectangles, tol 1e-10, one solver call for the batch",
            "nodes": int(sum(p.nx * p.ny for p in probs)), "host_setup_s": setup, "solvers": res,
            "speedup_vs_plain_fp64": {k: base / v["seconds"] for k, v in res.items()} if base else None}


def config1_record(torch, sil):
    """Configuration 1: the 2D scalar Hodge Laplacian (delta d of a 0-form) on
    a uniform 512^2 grid, FP64, 16 algorithmic bytes per cell update; timed
    warm (back-to-back launches, the 4 MB of fields stay in L2) and cold (a
    256 MB buffer written between launches flushes the 126 MB L2, each launch
    timed alone), with its parity against the oracle."""
    import oracle as O
    from tests.helpers import sinusoid_field
    m = 512
    host = sinusoid_field(m, seed=1)[..., None].copy()
    phi = torch.from_numpy(host).cuda()
    coords = [np.arange(m) / m, np.arange(m) / m]
    g2 = sil.Geometry(coords)
    o2 = torch.empty((m - 1, m - 1, 1), device="cuda", dtype=torch.float64)
    p2 = sil.make_staged_laplacian(g2, o2, phi, 0)
    nbytes = (m * m + (m - 1) ** 2) * 8
    for _ in range(5):
        p2.run(o2, phi)
    torch.cuda.synchronize()
    # warm: 200 launches replayed from one CUDA graph, so the host's launch
    # rate does not pace the 5-us kernels
    reps = 200
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        p2.run(o2, phi)
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(reps):
            p2.run(o2, phi)
    graph.replay()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    graph.replay()
    b.record()
    torch.cuda.synchronize()
    warm_ms = a.elapsed_time(b) / reps
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    cold = []
    for _ in range(30):
        flush.fill_(1)
        a.record()
        p2.run(o2, phi)
        b.record()
        torch.cuda.synchronize()
        cold.append(a.elapsed_time(b))
    cold_ms = statistics.median(cold)
    ref = O.laplacian(2, 0, O.position_from_coords(coords), host)
    got = o2.cpu().numpy()
    rel = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
    d = torch.zeros((m - 1, m - 1, 2), device="cuda", dtype=torch.float64)
    sil.deriv(d, phi, 0)
    dref = np.zeros((m - 1, m - 1, 2))
    O.coboundary(host, dref, 0)
    cu = (m - 1) ** 2
    return {"workload": "2D scalar Hodge Laplacian delta d of a 0-form, 512x512 uniform grid, spacing 1/512, FP64 "
                        "(8 sinusoidal modes + 1e-3 noise, seed 1)",
            "bytes_per_cell_update": 16, "algorithmic_bytes_per_launch": nbytes,
            "warm": {"us": warm_ms * 1e3, "GB/s": nbytes / (warm_ms * 1e-3) / 1e9,
                     "cell_updates_per_s": cu / (warm_ms * 1e-3),
                     "how": f"{reps} back-to-back launches from one CUDA graph, L2 resident"},
            "cold": {"us": cold_ms * 1e3, "GB/s": nbytes / (cold_ms * 1e-3) / 1e9,
                     "cell_updates_per_s": cu / (cold_ms * 1e-3),
                     "how": "median of 30 launches, each after a 256 MB write that flushes L2"},
            "laplacian_rel_err_vs_oracle": rel, "coboundary_bit_exact": bool(np.array_equal(d.cpu().numpy(), dref)),
            "kernel": p2.kernel}


SOLVE_SUM_KEYS = ("converged", "converged_by_oracle", "fallbacks", "total_iterations", "problems_checked_by_oracle")
SOLVE_MAX_KEYS = ("max_iterations", "max_rel_residual_gpu", "max_rel_residual_oracle")


def run_solve_workload(args):
    """Batched 2D magnetostatics time-to-1e-10 (device-resident inputs, whole batch per solve call)."""
    import torch
    import oracle as O
    import similie_b200.magnetostatics as mag
    from similie_b200 import dist as sd
    rank, world, local = sd.env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    count = args.count or 64
    if args.sizes:
        allp = mag.synthetic_batch(seed=args.seed, count=count, sizes=tuple(int(v) for v in args.sizes.split(",")))
    else:
        allp = mag.synthetic_batch(seed=args.seed, count=count)
    # problems shard across ranks by work (nodes), no collective on the data path
    mine = sd.shard_by_work([p.nx * p.ny for p in allp], world)[rank]
    probs = [allp[i] for i in mine]
    net, weights = load_network()
    kinds = [k for k in args.solvers.split(",") if k in ("cg", "mixed") or (k == "learned" and net is not None)]
    with ClockSampler(local) as clocks:
        results = time_solver_kinds(torch, probs, kinds, net, weights, chunk=args.chunk, concurrent=args.concurrent,
                                    max_iterations=args.max_iterations)
    gathered = sd.gather_to_rank0(results)
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()
    if rank != 0:
        return
    # per-problem figures over all ranks (the seconds are already the maximum over ranks)
    results = sd.merge_records(gathered, SOLVE_SUM_KEYS, SOLVE_MAX_KEYS)
    cpu = None
    if args.cpu_sample > 0:
        sample = allp[:args.cpu_sample]
        t0 = time.perf_counter()
        for p in sample:
            O.mag2d_cg(p.nx, p.ny, p.node_mu(), p.rhs(), tol=1e-10, max_iter=200000)
        sec = time.perf_counter() - t0
        nodes = sum(p.nx * p.ny for p in sample)
        cpu = {"value": len(sample) / sec, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"first {len(sample)} problems of the batch ({nodes} nodes), FP64 Jacobi-CG to 1e-10",
               "seconds": sec}
    base = results[kinds[0]]["seconds"]
    best = min(results, key=lambda k: results[k]["seconds"])
    line = {"metric": "time-to-1e-10 residual, batch of 2D magnetostatics problems (plain FP64 solve vs mixed vs learned)",
            "value": results[best]["solves_per_s"], "unit": "solves/s", "n_gpus": world, "steps": 1, "warmup": 0,
            "ms_per_step": results[best]["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 outer / f32 inner",
            "data": "synthetic (seeded coils and permeability-1000 rectangles)",
            "config": {"chunk": min(args.chunk, 64), "concurrent": args.concurrent,
                       "workload": f"{count} problems, sizes {args.sizes or '128..1024'} squared (seed {args.seed}), "
                                   f"tol 1e-10, solved {min(args.chunk, 64)} per call", "best": best},
            "solvers": results, "speedup_vs_plain_fp64": {k: base / v["seconds"] for k, v in results.items()},
            "cpu_baseline": cpu, "clocks": clocks.summary()}
    print(json.dumps(line))


def run_mag3d_workload(args):
    """Batched 3D magnetostatics (curl-curl + gauge penalty) time-to-1e-10."""
    import torch
    import similie_b200.magnetostatics3d as m3
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    probs = m3.synthetic_batch(seed=5, count=args.count or 8, n=args.n3d)
    coords = [(p.x, p.y, p.z) for p in probs]
    mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    setup = time.perf_counter() - t0
    results = {}
    with ClockSampler(0) as clocks:
        for kind in [k for k in args.solvers.split(",") if k in ("cg", "mixed")]:
            sols = [torch.zeros_like(r) for r in rhss]
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            d = m3.solve_batch(coords, mus, rhss, sols, solver=kind, tol=1e-10, max_iterations=args.max_iterations)
            e1.record()
            torch.cuda.synchronize()
            sec = e0.elapsed_time(e1) / 1e3
            results[kind] = {"seconds": sec, "solves_per_s": len(probs) / sec, "converged": sum(x.converged for x in d),
                             "max_iterations": max(x.iterations for x in d),
                             "ms_per_batch_iteration": sec * 1e3 / max(1, max(x.iterations for x in d)),
                             "max_rel_residual_gpu": max(x.final_relative_residual for x in d)}
    best = min(results, key=lambda k: results[k]["seconds"])
    n = args.n3d
    hodge = hodge3d_gbs(torch, probs[0].x, probs[0].y, probs[0].z)
    apply3d = apply3d_gbs(torch, probs[0], mus[0])
    line = {"metric": f"time-to-1e-10 residual, batch of {len(probs)} 3D curl-curl problems {n}^3",
            "value": results[best]["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "ms_per_step": results[best]["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 / f32 inner",
            "data": "synthetic (seeded toroidal loops, ratio-1.01 stretched grid)",
            "config": {"workload": f"{len(probs)} x {n}^3 nodes x 3 components, gamma 20", "host_setup_s": setup,
                       "best": best},
            "solvers": results, "hodge_star_1_to_2_form": hodge, "curl_curl_apply": apply3d,
            "clocks": clocks.summary()}
    print(json.dumps(line))


def run_nonlinear_workload(args):
    """Batch of seeded 2D problems whose permeability-1000 rectangles are a
    saturating material: Newton (at most 30 steps) + line search, each step a
    Jacobi-CG solve of the Jacobian to 1e-10.  Beside it, the oracle's solve
    of the batch's first problem on all host cores (same algorithm)."""
    import torch
    import similie_b200.magnetostatics as mag
    torch.cuda.set_device(0)
    n = args.n2d
    count = args.count or 8
    cases = [mag.nonlinear_problem(n, s) for s in range(count)]
    mus = [torch.from_numpy(c[1]).cuda() for c in cases]
    fes = [torch.from_numpy(c[2]).cuda() for c in cases]
    rhss = [torch.from_numpy(c[0].rhs()).cuda() for c in cases]
    curves = [(c[3], c[4]) for c in cases]
    with ClockSampler(0) as clocks:
        sols = [torch.zeros_like(r) for r in rhss]
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        d = mag.nl_solve_batch(mus, fes, curves, rhss, sols, [(n, n)] * count, tol=1e-10,
                               max_iterations=args.max_iterations)
        e1.record()
        torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    steps = sum(x.refinements for x in d)
    cpu = None
    if not args.no_cpu_baseline:
        import oracle as O
        p, mu, fe, b, h = cases[0]
        t0 = time.perf_counter()
        xo, it, st, rel = O.mag2d_nl_solve(n, n, mu, fe, b, h, p.rhs(), tol=1e-10, max_iter=args.max_iterations)
        tc = time.perf_counter() - t0
        cpu = {"value": 1.0 / tc, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"the batch's first problem ({n}^2, {st} Newton steps, {it} CG iterations) in {tc:.2f} s",
               "gpu_solution_rel_diff": float(np.linalg.norm(sols[0].cpu().numpy() - xo) / np.linalg.norm(xo))}
    line = {"metric": f"nonlinear 2D magnetostatics (Newton + line search), batch of {count} problems {n}^2",
            "value": count / sec, "unit": "solves/s", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded coils; saturating permeability-1000 rectangles, 64-sample B-H curve)",
            "config": {"workload": f"{count} x {n}^2 nodes, tol 1e-10, at most 30 Newton steps"},
            "newton_steps": steps, "ms_per_newton_step": sec * 1e3 / max(steps, 1),
            "cg_iterations": sum(x.iterations for x in d), "converged": sum(x.converged for x in d),
            "final_relative_residuals": [x.final_relative_residual for x in d],
            "cpu_baseline": cpu, "clocks": clocks.summary()}
    print(json.dumps(line))


def run_nonlinear3d_workload(args):
    """Batch of seeded 3D loop-current problems with a box core of the
    saturating material: Newton (at most 30 steps) + line search, each step a
    Jacobi-CG solve of the Jacobian to 1e-10.  Beside it, the oracle's solve
    of the batch's first problem on all host cores (same algorithm)."""
    import torch
    import similie_b200.magnetostatics3d as m3
    torch.cuda.set_device(0)
    n = args.nl3d
    count = args.count or 8
    cases = [m3.nonlinear_problem(n, s) for s in range(count)]
    coords = [(c[0].x, c[0].y, c[0].z) for c in cases]
    mus = [torch.from_numpy(c[1]).cuda() for c in cases]
    fes = [torch.from_numpy(c[2]).cuda() for c in cases]
    rhss = [torch.from_numpy(c[0].rhs()).cuda() for c in cases]
    curves = [(c[3], c[4]) for c in cases]
    with ClockSampler(0) as clocks:
        sols = [torch.zeros_like(r) for r in rhss]
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        d = m3.nl_solve_batch(coords, mus, fes, curves, rhss, sols, tol=1e-10, max_iterations=args.max_iterations)
        e1.record()
        torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    steps = sum(x.refinements for x in d)
    cpu = None
    if not args.no_cpu_baseline:
        import oracle as O
        p, mu, fe, b, h = cases[0]
        t0 = time.perf_counter()
        xo, it, st, rel = O.mag3d_nl_solve(p.x, p.y, p.z, mu, fe, p.gamma, b, h, p.rhs(), tol=1e-10,
                                           max_iter=args.max_iterations)
        tc = time.perf_counter() - t0
        cpu = {"value": 1.0 / tc, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"the batch's first problem ({n}^3, {st} Newton steps, {it} CG iterations) in {tc:.2f} s",
               "gpu_solution_rel_diff": float(np.linalg.norm(sols[0].cpu().numpy() - xo) / np.linalg.norm(xo))}
    line = {"metric": f"nonlinear 3D magnetostatics (Newton + line search), batch of {count} problems {n}^3",
            "value": count / sec, "unit": "solves/s", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded current loops; saturating permeability-1000 box core, 64-sample B-H curve)",
            "config": {"workload": f"{count} x {n}^3 nodes x 3 components, gamma 20, tol 1e-10, "
                                   "at most 30 Newton steps"},
            "newton_steps": steps, "ms_per_newton_step": sec * 1e3 / max(steps, 1),
            "cg_iterations": sum(x.iterations for x in d), "converged": sum(x.converged for x in d),
            "final_relative_residuals": [x.final_relative_residual for x in d],
            "cpu_baseline": cpu, "clocks": clocks.summary()}
    print(json.dumps(line))


def run_assembled_workload(args):
    """The assembled-matrix path on one seeded 2D problem of the batched
    distribution: CSR assembly, then every entry of the reference's
    preconditioner menu built on it and a preconditioned CG to 1e-10 (at most
    20,000 iterations).  Beside it, the oracle's Jacobi-preconditioned CG on
    the same matrix on all host cores."""
    import torch
    import similie_b200.assembled as asm
    import similie_b200.magnetostatics as mag
    torch.cuda.set_device(0)
    n = args.asm_n
    rng = np.random.default_rng(args.seed)
    p = mag.synthetic_problem(rng, n, cores=2)
    mu = torch.from_numpy(p.node_mu()).cuda()
    b = torch.from_numpy(p.rhs()).cuda()
    max_it = 20000

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    results = {}
    with ClockSampler(0) as clocks:
        A, t_asm = timed(lambda: asm.CsrMatrix.mag2d(n, n, mu))
        for kind in asm.KINDS:
            P, t_setup = timed(lambda: asm.Preconditioner(A, kind))
            x = torch.zeros_like(b)
            asm.solve(A, P, b, x, tol=1e-10, max_iterations=20)      # warm-up
            d, t_solve = timed(lambda: asm.solve(A, P, b, x, tol=1e-10, max_iterations=max_it))
            results[kind] = {"setup_s": t_setup, "solve_s": t_solve, "iterations": d.iterations,
                             "converged": d.converged, "final_relative_residual": d.final_relative_residual,
                             "ms_per_iteration": 1e3 * t_solve / max(d.iterations, 1)}
            P.close()
    best = min((k for k in results if results[k]["converged"]), key=lambda k: results[k]["solve_s"])
    # the SpMV alone: 12 algorithmic bytes per nonzero (value + column) and 16
    # per row (x and y once each, row pointer), against the HBM peak
    xs = torch.randn(n * n, dtype=torch.float64, device="cuda")
    ys = torch.empty_like(xs)
    for _ in range(5):
        A.spmv(xs, ys)
    torch.cuda.synchronize()
    reps = 50
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(reps):
        A.spmv(xs, ys)
    s1.record()
    torch.cuda.synchronize()
    spmv_s = s0.elapsed_time(s1) / 1e3 / reps
    peak, kind = measured_peaks()
    spmv_bytes = 12 * A.nnz + 16 * n * n
    roofline = {"kernel": "spmv_kernel", "bound": "hbm", "achieved": spmv_bytes / spmv_s / 1e9, "peak": peak,
                "unit": "GB/s", "frac": spmv_bytes / spmv_s / 1e9 / peak, "traffic": None,
                "bytes_per_launch": spmv_bytes, "us_per_launch": spmv_s * 1e6, "peak_source": kind,
                "note": "the matrix (15.6 MB at 512^2) is L2 resident between launches"}
    cpu = None
    if not args.no_cpu_baseline:
        import oracle as O
        G = A.to_scipy()
        t0 = time.perf_counter()
        xo, it, rel = O.csr_pcg(G, p.rhs(), "jacobi", tol=1e-10, max_iter=max_it)
        tc = time.perf_counter() - t0
        cpu = {"value": 1.0 / tc, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"Jacobi-preconditioned CG on the same {n}^2 CSR matrix ({it} iterations) in {tc:.2f} s"}
    jac = results["jacobi"]
    line = {"metric": f"assembled-matrix magnetostatics solve, {n}^2, reference preconditioner menu",
            "value": 1.0 / jac["solve_s"], "unit": "solves/s (Jacobi)", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": jac["solve_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded coils, permeability-1000 rectangles)",
            "config": {"workload": f"one {n}^2 problem, CSR {A.nnz} nonzeros, tol 1e-10", "assembly_s": t_asm,
                       "fastest_converged": best},
            "menu": results, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary()}
    print(json.dumps(line))


def apply3d_gbs(torch, prob, mu, steps=20):
    """The FP64 3D curl-curl + gauge-penalty operator applied to one problem's
    node field by the operator object (set-up once, one kernel per apply),
    timed with CUDA events over back-to-back applies replayed from a CUDA
    graph (inputs far larger than L2): 56 algorithmic bytes per node (3
    components in, 3 out, the node reluctivity)."""
    import similie_b200.magnetostatics3d as m3
    g = torch.Generator(device="cuda").manual_seed(4)
    a = torch.randn(3 * mu.numel(), dtype=torch.float64, device="cuda", generator=g)
    out = torch.empty_like(a)
    op = m3.Operator(prob.x, prob.y, prob.z, mu, gamma=prob.gamma)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            op.apply(a, out)
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(steps):
            op.apply(a, out)
    graph.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    graph.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    nodes = mu.numel()
    peak, kind = measured_peaks()
    gbs = nodes * 56 / (ms * 1e-3) / 1e9
    return {"ms": ms, "GB/s_algorithmic": gbs, "frac_of_peak": gbs / peak, "peak_source": kind,
            "bytes_per_node": 56, "nodes": nodes, "call": "sil_mag3d_operator_apply (one kernel, CUDA graph)"}


def hodge3d_gbs(torch, x, y, z, steps=20):
    """Hodge star of a 3D 1-form into a 2-form on the stretched grid (FP64, DDC layout
    [x][y][z][component]): 48 algorithmic bytes per node (3 components in, 3 out)."""
    import similie_b200 as sil
    geo = sil.Geometry([x, y, z])
    n = (len(x), len(y), len(z))
    g = torch.Generator(device="cuda").manual_seed(3)
    w = torch.randn(*n, 3, dtype=torch.float64, device="cuda", generator=g)
    out = torch.empty_like(w)
    for _ in range(3):
        sil.hodge_star(geo, out, w, 1)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sil.hodge_star(geo, out, w, 1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    nodes = n[0] * n[1] * n[2]
    peak, kind = measured_peaks()
    gbs = nodes * 48 / (ms * 1e-3) / 1e9
    return {"ms": ms, "GB/s_algorithmic": gbs, "frac_of_peak": gbs / peak, "peak_source": kind,
            "bytes_per_node": 48, "nodes": nodes}


def run_precond_workload(args):
    """Learned-preconditioner applies M(r) on a batch of node grids (device-resident FP32)."""
    import torch
    from similie_b200.precond import LearnedPreconditioner
    torch.cuda.set_device(0)
    rng = np.random.default_rng(7)
    if args.shapes:
        n, c = (int(v) for v in args.shapes.split("x"))
        sizes = [n] * c
    else:
        sizes = [int(rng.choice([128, 256, 384, 512, 768, 1024])) for _ in range(64)]
    shapes = [(n, n) for n in sizes]
    tot = sum(n * n for n in sizes)
    g = torch.Generator(device="cuda").manual_seed(7)
    nu = torch.rand(tot, device="cuda", generator=g) * 0.9 + 0.1
    r = torch.randn(tot, device="cuda", generator=g)
    out = torch.zeros_like(r)
    net = LearnedPreconditioner(seed=1)
    weights = weights_path()
    if os.path.exists(weights):
        net.load(weights)
    for _ in range(args.warmup):
        net.apply(shapes, nu, r, out)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        net.apply(shapes, nu, r, out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    top = sum(((n + 1) // 2) ** 2 for n in sizes)
    print(json.dumps({"metric": "learned preconditioner apply", "value": ms, "unit": "ms", "higher_is_better": False,
                      "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "config": {"workload": f"{len(sizes)} grids, {tot} nodes, {top} top-level pixels"}}))


if __name__ == "__main__":
    main()
