"""Benchmark: Mnodes/s to the exact min-cut on the plain-GPU workload
(2D 4-connected 15000 x 10000 RGB image, 150M nodes: 20 random overlapping
ellipses, N(0,15) noise, random strokes over 0.5% of pixels, 5-means colour
models, int32 capacities; synthetic, seeded).

One step = capacity build from the device-resident image + seeds (n-links,
k-means t-links) -> push-relabel to convergence -> canonical cut labels.
`value` times steps with inputs already in HBM; `e2e` times the same call
through the C ABI from pinned host buffers, with the H2D upload of image +
seeds and the D2H read of the labels inside the timed region.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Multi-GPU: one process per GPU (torchrun); every rank solves its own replica
of the workload (replicas only: one grid does not shard without a per-sweep
halo exchange), value = all ranks' nodes / max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "jf-cut_b200"))

W_FULL, H_FULL = 15000, 10000
SEED = 20240601
MODEL = dict(lambda_n=100, z_weight_pct=100, lambda_t=10, k_fg=5, k_bg=5, seed_cap=1000000, kmeans_iters=32)
METRIC = "Mnodes/s to exact min-cut (plain, 2D 4-conn 15000x10000 RGB)"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def make_workload(w, h, seed):
    import jfcut
    return jfcut.synth_rgb_ellipses(w, h, seed=seed, n_ellipses=20, noise_sigma=15, stroke_permille_x10=50)


def reference_sample(budget_s=20.0, side=(2048, 1536)):
    """Bounded sample of the same workload for the CPU solvers: one image of
    `side` generated like the full one."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    w, h = side
    img, seeds = make_workload(w, h, SEED)
    e, caps, sink = oracle.build_graph(img, seeds, 1, MODEL)
    return oracle, (h, w), e, caps


def run_reference(args):
    """Reference arm: the reference's own CPU solver (GridCut 1.1 multi-threaded,
    built from the reference sources) on the host cores, bounded sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    cores = os.cpu_count() or 1
    orc, shape, e, caps = reference_sample()
    n = e.size
    for _ in range(args.warmup):
        orc.gridcut_maxflow(shape, e, caps, cores)
    times = []
    for _ in range(args.steps):
        f, t = orc.gridcut_maxflow(shape, e, caps, cores)
        times.append(sum(t))
    ms = 1000.0 * sum(times) / len(times)
    v = n / (ms / 1000.0) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mnodes/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "plain 2D 4-conn RGB ellipses, bounded CPU sample %dx%d" % (shape[1], shape[0]),
                       "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": "Mnodes/s", "cores": cores, "kind": "reference",
                             "sample": "GridCut 1.1 MT (reference benchmark/GridCut) on a %dx%d instance of the "
                                       "workload, init+maxflow+labels per step" % (shape[1], shape[0])},
            "e2e": {"value": v, "unit": "Mnodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def cpu_baseline_bk():
    """BK 3.03 (reference CPU path, 1 core) on a bounded sample, ~10-30 s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available():
        return None
    orc, shape, e, caps = reference_sample()
    total, reps = 0.0, 0
    while total < 10.0 and reps < 8:
        f, _, t = orc.bk_maxflow(shape, e, caps, want_labels=True)
        total += sum(t)
        reps += 1
    v = e.size * reps / total / 1e6
    return {"value": v, "unit": "Mnodes/s", "cores": 1, "kind": "reference",
            "sample": "BK 3.03 (reference benchmark/GridCut/code/BK303, int64 flow) on a %dx%d instance of the "
                      "workload x%d, init+maxflow+labels" % (shape[1], shape[0], reps)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--width", type=int, default=W_FULL)
    ap.add_argument("--height", type=int, default=H_FULL)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import jfcut

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    w, h = args.width, args.height
    n = w * h
    img, seeds = make_workload(w, h, SEED + rank)
    stream = torch.cuda.Stream()
    ctx = jfcut.Context(local)
    ctx.set_stream(stream.cuda_stream)
    g = jfcut.Graph(ctx, (h, w))
    d_img = torch.from_numpy(img).to("cuda")
    d_seeds = torch.from_numpy(seeds).to("cuda")
    d_lab = torch.empty(n, dtype=torch.uint8, device="cuda")
    h_img = torch.from_numpy(img).pin_memory()
    h_seeds = torch.from_numpy(seeds).pin_memory()
    h_lab = torch.empty(n, dtype=torch.uint8).pin_memory()
    torch.cuda.synchronize()

    def step_device():
        g.build_from_device(d_img.data_ptr(), d_seeds.data_ptr(), jfcut.PIX_RGB8, MODEL)
        st = g.solve()
        g.read_labels_device(d_lab.data_ptr())
        return st

    def step_e2e():
        g.build_from_image(h_img.numpy(), h_seeds.numpy(), jfcut.PIX_RGB8, MODEL)
        st = g.solve()
        out = h_lab.numpy()
        jfcut.lib().jfc_read_labels(g.handle, out.ctypes.data_as(jfcut.U8P))
        return st

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step_device()
        flow_ref = g.flow()
        # ---- value: device-resident inputs
        clocks = ClockSampler(local)
        clocks.start()
        barrier()
        l0 = jfcut.kernel_launches()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        visits, ms_pr, sweeps = 0, 0.0, 0
        agg = {"ms_total": 0.0, "ms_push_relabel": 0.0, "ms_global_relabel": 0.0, "ms_cut": 0.0,
               "global_relabels": 0, "bfs_passes": 0}
        for _ in range(args.steps):
            st = step_device()
            visits += st.tile_visits
            ms_pr += st.ms_push_relabel
            sweeps += st.sweeps
            for k in agg:
                agg[k] += getattr(st, k)
            assert g.flow() == flow_ref
        ev1.record(stream)
        barrier()
        ms = ev0.elapsed_time(ev1)
        launches = jfcut.kernel_launches() - l0
        clk = clocks.stop()
        ms = max_over_ranks(ms)
        # ---- e2e: host buffers through the C ABI
        for _ in range(1):
            step_e2e()
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            step_e2e()
            assert g.flow() == flow_ref
        ev1.record(stream)
        barrier()
        ms_e2e = max_over_ranks(ev0.elapsed_time(ev1))

    ms_step = ms / args.steps
    value = world * n * args.steps / (ms / 1000.0) / 1e6
    e2e = world * n * args.steps / (ms_e2e / 1000.0) / 1e6
    tr = ctx.params().tile_rows
    bytes_per_visit = 32 * tr * 48 + (2 * 32 + 2 * tr) * 12
    achieved = visits * bytes_per_visit / (ms_pr / 1000.0) / 1e9 if ms_pr > 0 else 0.0
    peak, peak_kind = peaks()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mnodes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "plain: 2D 4-conn %dx%d RGB, 20 ellipses, N(0,15), 0.5%% strokes, 5-means "
                                   "(build + solve + labels per step)" % (w, h),
                       "nodes": n, "global_batch": world, "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (state %.1f GB)" % (jfcut.lib().jfc_graph_bytes(2, w, h, 1) / 1e9),
                       "params": {k: getattr(ctx.params(), k) for k in ("tile_rows", "local_iters", "relabel_interval")},
                       "flow": flow_ref, "sweeps_per_step": sweeps / args.steps,
                       "solve_breakdown_per_step": {k: v / args.steps for k, v in agg.items()},
                       "pr_tile_visits_per_step": visits / args.steps},
            "e2e": {"value": e2e, "unit": "Mnodes/s", "h2d_bytes_per_step": int(img.nbytes + seeds.nbytes),
                    "d2h_bytes_per_step": int(n)},
            "gpu_launches": int(launches),
            "clocks": clk,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "k_pr_sweep (push-relabel tile visits; %d B/visit algorithmic, %s peak)"
                                   % (bytes_per_visit, peak_kind)},
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_bk()
        print(json.dumps(line), flush=True)
    g.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
