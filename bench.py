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
import faulthandler
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
# seeded input generators (oracle/synthetic.cpp): both arms build their graph
# from the same bytes; they run before any timed region
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import synthetic  # noqa: E402

W_FULL, H_FULL = 15000, 10000
SEED = 20240601
MODEL = dict(lambda_n=100, z_weight_pct=100, lambda_t=10, k_fg=5, k_bg=5, seed_cap=1000000, kmeans_iters=32)
METRIC = "Mnodes/s to exact min-cut (plain, 2D 4-conn 15000x10000 RGB)"


def pr_traffic_per_visit():
    """DRAM bytes per push-relabel tile visit, from the committed summary of the
    one-pass ncu capture of every push-relabel launch of this workload's run
    (profiles/k_pr_phase_traffic_15000x10000.md), else of a 4096x3072 run, or
    None.  A launch's traffic is this times its visits (each visit reads and
    writes one tile)."""
    for name in ("k_pr_phase_traffic_15000x10000.md", "k_pr_phase_traffic_4096x3072.md"):
        try:
            with open(os.path.join(ROOT, "profiles", name)) as f:
                for line in f:
                    if line.startswith("traffic_bytes_per_visit:"):
                        return float(line.split(":")[1])
        except OSError:
            pass
    return None


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
    return synthetic.rgb_ellipses(w, h, seed=seed, n_ellipses=20, noise_sigma=15, stroke_permille_x10=50)


def workload_name(w, h):
    return ("plain: 2D 4-conn %dx%d RGB, 20 ellipses, N(0,15), 0.5%% strokes, 5-means "
            "(build + solve + labels per step)" % (w, h))


def cpu_graph(w, h, seed):
    """The workload's graph built on the host by the CPU restatement of the
    capacity build (the GPU build equals it bit for bit: the parity tests):
    (oracle module, shape, e, caps, sum ct)."""
    import oracle
    img, seeds = make_workload(w, h, seed)
    e, caps, sink = oracle.build_graph(img, seeds, 1, MODEL)
    return oracle, (h, w), e, caps, sink


def full_flow(e0, folded, sink):
    """Max-flow of the image graph from a solver's folded flow on the
    net-excess graph (terminal arcs cs = max(e,0), ct = max(-e,0)):
    sum ct + folded - sum max(-e, 0)."""
    return int(sink) + int(folded) - int(np.maximum(-e0.astype(np.int64), 0).sum())


def run_reference(args):
    """Reference arm: the reference's own CPU solver, GridCut 1.1
    multi-threaded (benchmark/GridCut/bench-GridCut.cpp:76-100, built from the
    reference sources under oracle/_ref), with every host thread, on the same
    full workload as our arm: one step = graph init from the capacity arrays
    + maxflow + labels into host memory.  Loads no part of the product."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    cores = os.cpu_count() or 1
    w, h = args.width, args.height
    orc, shape, e, caps, sink = cpu_graph(w, h, replica_seed(0))
    n = e.size
    labels = np.empty(n, np.uint8)
    for _ in range(args.warmup):
        orc.gridcut_maxflow(shape, e, caps, cores, labels)
    times, parts, flows = [], np.zeros(3), set()
    for _ in range(args.steps):
        f, t = orc.gridcut_maxflow(shape, e, caps, cores, labels)
        times.append(sum(t))
        parts += np.asarray(t)
        flows.add(full_flow(e, f, sink))
    ms = 1000.0 * sum(times) / len(times)
    v = n / (ms / 1000.0) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mnodes/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": workload_name(w, h), "nodes": n, "global_batch": 1,
                       "parallelism": "host threads x%d" % cores,
                       "flow": flows.pop() if len(flows) == 1 else None,
                       "ms_split_per_step": {k: 1000.0 * float(x) / args.steps
                                             for k, x in zip(("init", "maxflow", "labels"), parts)}},
            "cpu_baseline": {"value": v, "unit": "Mnodes/s", "cores": cores, "kind": "reference",
                             "sample": "GridCut 1.1 MT (reference benchmark/GridCut) on the full %dx%d workload "
                                       "graph, init + maxflow + labels per step" % (w, h)},
            "e2e": {"value": v, "unit": "Mnodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_bk(w, h, seed, flow_gpu):
    """BK 3.03 (the reference's CPU path, benchmark/GridCut/bench-BK303.cpp,
    1 core, int64 flow) on the full workload graph: one init + maxflow +
    labels (~30 s and ~30 GB on the host)."""
    import oracle
    if not oracle.ref_available():
        return None
    orc, shape, e, caps, sink = cpu_graph(w, h, seed)
    f, lab, t = orc.bk_maxflow(shape, e, caps, want_labels=True)
    v = e.size / sum(t) / 1e6
    return {"value": v, "unit": "Mnodes/s", "cores": 1, "kind": "reference",
            "sample": "BK 3.03 (reference benchmark/GridCut/code/BK303, int64 flow) on the full %dx%d workload "
                      "graph, one init + maxflow + labels" % (w, h),
            "s_split": {"init": t[0], "maxflow": t[1], "labels": t[2]},
            "flow_equals_gpu": full_flow(e, f, sink) == flow_gpu}


def max_over_ranks(x, dist=None, device="cuda"):
    """The slowest rank's value (timings are taken per rank on the device)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(nodes_per_rank, world, steps, ms_max):
    """Whole-job Mnodes/s of N independent replicas: every rank solved
    nodes_per_rank per step; the job takes the slowest rank's time."""
    return world * nodes_per_rank * steps / (ms_max / 1000.0) / 1e6


def replica_seed(rank):
    """Each rank solves its own replica (same shape, its own seed)."""
    return SEED + rank


def pct(v, q):
    return float(np.percentile(np.asarray(v, dtype=np.float64), q)) if len(v) else None


def bench_batched(jfcut, torch, ctx, stream, steps, warmup, n_inst=256):
    """Batched workload: n_inst independent 2D 4-conn RGB instances with sides
    drawn uniformly in [128, 2048] (seeded), generated like the plain workload.
    Batched = every instance in one persistent launch per phase (device work
    queue, CUDA-graph cycles, the schedule the autotuner chose for the batch);
    plain = the same graphs solved one after another by the plain solver with
    its default schedule.  Both time the solve only
    (capacity build untimed between steps: it is the same per-instance work in
    both); every flow and cut of the batch must equal the plain ones."""
    rng = np.random.default_rng(SEED + 256)
    sides = rng.integers(128, 2049, size=(n_inst, 2))
    graphs, dev, total = [], [], 0
    for i, (w, h) in enumerate(sides):
        w, h = int(w), int(h)
        img, seeds = make_workload(w, h, SEED + 5000 + i)
        dev.append((torch.from_numpy(img).cuda(), torch.from_numpy(seeds).cuda()))
        graphs.append(jfcut.Graph(ctx, (h, w)))
        total += w * h
    offs = np.concatenate([[0], np.cumsum([g.shape[0] * g.shape[1] for g in graphs])])
    lab_plain = torch.empty(total, dtype=torch.uint8, device="cuda")
    lab_batch = torch.empty(total, dtype=torch.uint8, device="cuda")

    def build_all():
        for g, (di, ds) in zip(graphs, dev):
            g.build_from_device(di.data_ptr(), ds.data_ptr(), jfcut.PIX_RGB8, MODEL)
        torch.cuda.synchronize()

    def read_all(buf):
        for i, g in enumerate(graphs):
            g.read_labels_device(buf[int(offs[i]):].data_ptr())

    build_all()
    b = jfcut.Batch(ctx)
    for g in graphs:
        b.add(g)
    t0 = time.perf_counter()
    tuned = b.autotune()
    t_tune = time.perf_counter() - t0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = jfcut.kernel_launches()
    ms_plain = []
    for it in range(warmup + steps):
        build_all()
        ev0.record(stream)
        for g in graphs:
            g.solve()
        ev1.record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            ms_plain.append(ev0.elapsed_time(ev1))
    launches_plain = (jfcut.kernel_launches() - l0) / (warmup + steps)
    flows_plain = [g.flow() for g in graphs]
    read_all(lab_plain)
    ms_batch = []
    l0 = jfcut.kernel_launches()
    for it in range(warmup + steps):
        build_all()
        ev0.record(stream)
        st = b.solve()
        ev1.record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            ms_batch.append(ev0.elapsed_time(ev1))
    launches_batch = (jfcut.kernel_launches() - l0) / (warmup + steps)
    read_all(lab_batch)
    torch.cuda.synchronize()
    exact = all(g.flow() == f for g, f in zip(graphs, flows_plain)) and bool(torch.equal(lab_plain, lab_batch))
    mp, mb = float(np.mean(ms_plain)), float(np.mean(ms_batch))
    out = {"workload": "%d x 2D 4-conn RGB, sides U[128,2048], seeded; solve only" % n_inst,
           "instances": n_inst, "nodes": int(total),
           "plain_ms": mp, "batched_ms": mb,
           "plain_mnodes_s": total / (mp / 1e3) / 1e6, "batched_mnodes_s": total / (mb / 1e3) / 1e6,
           "speedup": mp / mb, "bit_exact_vs_plain": exact,
           "launches_per_step": {"plain": launches_plain, "batched": launches_batch},
           "used_graph": int(st[0].used_graph), "autotune_s": t_tune,
           "schedule": {k: getattr(tuned, k) for k in ("tile_rows", "local_iters", "relabel_interval")}}
    b.close()
    for g in graphs:
        g.close()
    return out


def bench_video(jfcut, torch, ctx, stream, steps=2, warmup=1, size=(2560, 1440, 50)):
    """3D plain workload: 6-connected 2560x1440x50 RGB video (184M nodes), an
    ellipse moving 4 px/frame over seeded value-noise texture, temporal n-link
    weight 0.5x the spatial one, 5-means colour models, strokes on frames 0
    and 49.  One step = capacity build from device-resident frames + solve +
    labels into a device buffer; flows must repeat exactly."""
    w, h, d = size
    img, seeds = synthetic.rgb_video(w, h, d, seed=SEED + 50)
    model = dict(MODEL, z_weight_pct=50)
    d_img = torch.from_numpy(img).cuda()
    d_seeds = torch.from_numpy(seeds).cuda()
    d_lab = torch.empty(w * h * d, dtype=torch.uint8, device="cuda")
    g = jfcut.Graph(ctx, (d, h, w))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms, flows, agg = [], set(), None
    for it in range(warmup + steps):
        torch.cuda.synchronize()
        ev0.record(stream)
        g.build_from_device(d_img.data_ptr(), d_seeds.data_ptr(), jfcut.PIX_RGB8, model)
        st = g.solve()
        g.read_labels_device(d_lab.data_ptr())
        ev1.record(stream)
        torch.cuda.synchronize()
        flows.add(g.flow())
        if it >= warmup:
            ms.append(ev0.elapsed_time(ev1))
            agg = st
    g.close()
    n = w * h * d
    m = float(np.mean(ms))
    return {"workload": "3D 6-conn %dx%dx%d RGB video (build + solve + labels per step)" % (w, h, d), "nodes": n,
            "ms_per_step": m, "mnodes_s": n / (m / 1e3) / 1e6, "flow": flows.pop() if len(flows) == 1 else None,
            "flow_repeatable": len(flows) <= 1,
            "solve_breakdown": {k: round(getattr(agg, k), 2) for k in
                                ("ms_total", "ms_push_relabel", "ms_global_relabel", "ms_cut", "sweeps",
                                 "global_relabels")}}


def bench_fastcut(jfcut, torch, w=4096, h=3072, reps=2):
    """The reference's Fast-Cut line sweeps (pr_mode 1) against the block-wise
    push-relabel on a 4096x3072 instance of the plain workload: solve time,
    sweeps and relabels of each (flows must agree)."""
    img, seeds = make_workload(w, h, SEED)
    d_img, d_seeds = torch.from_numpy(img).cuda(), torch.from_numpy(seeds).cuda()
    out = {"workload": "plain 2D 4-conn %dx%d RGB (solve only)" % (w, h)}
    flows = set()
    for name, params in (("block", dict(pr_mode=0)), ("fastcut", dict(pr_mode=1, relabel_interval=2))):
        ctx = jfcut.Context(0, **params)
        g = jfcut.Graph(ctx, (h, w))
        best = None
        for _ in range(reps):
            g.build_from_device(d_img.data_ptr(), d_seeds.data_ptr(), jfcut.PIX_RGB8, MODEL)
            st = g.solve()
            if best is None or st.ms_total < best.ms_total:
                best = st
            flows.add(g.flow())
        out[name] = {"ms": best.ms_total, "sweeps": best.sweeps, "global_relabels": best.global_relabels}
        g.close()
        ctx.close()
    out["speedup_block_vs_fastcut"] = out["fastcut"]["ms"] / out["block"]["ms"]
    out["flows_agree"] = len(flows) == 1
    return out


def bench_serve(jfcut, torch, ctx, seconds=20.0, rate=200.0, budget_gb=96, max_cold_outstanding=64,
                pool_2d=16, pool_3d=8, baseline_samples=8):
    """Serving workload: `seconds` of Poisson arrivals (mean `rate`/s), each a
    new session: 70% 2D RGB images (sides U[256,4096], 4-conn), 30% int16
    sphere-and-tube phantom volumes (sides U[128,512], 6-conn, N(0,10)
    noise); after its cold result a session sends 1-5 stroke edits (0.1-2%
    of its nodes) one after another, each re-solved warm on the
    device-resident residual graph, then closes.  Inputs come from a seeded
    pool (pool_2d images, pool_3d volumes, 5 strokes each).

    The offered load is several times what one GPU solves, so the client
    sheds: an arrival that finds max_cold_outstanding cold requests
    unfinished is rejected (counted, never submitted), which bounds the
    admission queue the way a front end returning "busy" would.  Reported:
    offered vs served load, shed fraction, p50/p99 latency (client side of the
    C ABI, submit -> result) per class (cold / warm x 2D / volume), and a
    baseline of cold plain re-solves (build + the session's edits + solve on
    the idle GPU) of sampled sessions, whose flows must equal the served
    ones."""
    rng = np.random.default_rng(SEED + 200)
    pool = []
    for i in range(pool_2d + pool_3d):
        if i < pool_2d:
            w, h = (int(v) for v in rng.integers(256, 4097, 2))
            img, seeds = make_workload(w, h, SEED + 9000 + i)
            pf = jfcut.PIX_RGB8
        else:
            w, h, d = (int(v) for v in rng.integers(128, 513, 3))
            img, seeds = synthetic.i16_phantom(w, h, d, seed=SEED + 9000 + i, noise_sigma=10)
            pf = jfcut.PIX_I16
        n = seeds.size
        strokes = []
        for k in range(5):
            m = max(1, int(n * rng.uniform(0.001, 0.02)))
            strokes.append(synthetic.stroke(seeds.shape, seed=SEED + 100 * i + k, n=m, label=1 + (k % 2)))
        pool.append(dict(img=img, seeds=seeds, pf=pf, strokes=strokes, n=n, dims=seeds.ndim))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, int(rate * seconds * 1.5) + 16))
    arrivals = arrivals[arrivals < seconds]
    picks = [(int(rng.integers(0, pool_2d)) if rng.random() < 0.7 else pool_2d + int(rng.integers(0, pool_3d)),
              int(rng.integers(1, 6))) for _ in arrivals]
    srv = jfcut.Server(ctx, int(budget_gb * (1 << 30)), max_slots=64)
    lock = threading.Lock()
    records, served, failures = [], [], []
    state = {"cold_out": 0, "shed": 0, "offered_nodes": 0}

    def session(j, p, k):
        s = pool[p]
        try:
            sid = srv.submit(s["img"], s["seeds"], s["pf"], MODEL)
            info = srv.wait(sid, 300000)
            with lock:
                state["cold_out"] -= 1
            rec = [("cold", s["dims"], s["n"], info.ms_total, info.status, info.ms_queue, info.ms_solve)]
            flow = info.flow
            for idx, ns in s["strokes"][:k]:
                if info.status:
                    break
                srv.edit(sid, idx, ns)
                info = srv.wait(sid, 300000)
                rec.append(("warm", s["dims"], s["n"], info.ms_total, info.status, info.ms_queue, info.ms_solve))
                flow = info.flow
            srv.close_session(sid)
            with lock:
                records.extend(rec)
                if info.status == 0:
                    served.append((p, k, flow, rec[-1][3]))
        except Exception as ex:   # reported, the run goes on
            with lock:
                failures.append("%s: %s" % (type(ex).__name__, ex))

    threads = []
    t_start = time.perf_counter()
    for j, (t_arr, (p, k)) in enumerate(zip(arrivals, picks)):
        delay = t_arr - (time.perf_counter() - t_start)
        if delay > 0:
            time.sleep(delay)
        with lock:
            state["offered_nodes"] += pool[p]["n"]
            if state["cold_out"] >= max_cold_outstanding:
                state["shed"] += 1
                continue
            state["cold_out"] += 1
        th = threading.Thread(target=session, args=(j, p, k))
        th.start()
        threads.append(th)
    t_arrivals = time.perf_counter() - t_start
    for th in threads:
        th.join()
    wall = time.perf_counter() - t_start
    sstats = srv.stats()
    srv.close()
    # baseline: cold plain re-solves of sampled served sessions on the idle
    # GPU (build + the same edits + solve), flows equal to the served ones
    base_ms, exact = [], True
    picked = served[:: max(1, len(served) // baseline_samples)][:baseline_samples]
    for p, k, flow, warm_ms in picked:
        s = pool[p]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = jfcut.Graph(ctx, s["seeds"].shape)
        g.build_from_image(s["img"], s["seeds"], s["pf"], MODEL)
        for idx, ns in s["strokes"][:k]:
            g.edit_seeds(idx, ns)
        g.solve()
        base_ms.append((time.perf_counter() - t0) * 1e3)
        exact &= g.flow() == flow
        g.close()

    def lat(kind, dims):
        rs = [r for r in records if r[0] == kind and r[1] == dims and r[4] == 0]
        v = [r[3] for r in rs]
        # the server's split of a request's latency: waiting for admission
        # (queue) and admitted until its result (solve, sharing the GPU)
        return {"n": len(v), "p50_ms": pct(v, 50), "p99_ms": pct(v, 99),
                "queue_p50_ms": pct([r[5] for r in rs], 50), "queue_p99_ms": pct([r[5] for r in rs], 99),
                "solve_p50_ms": pct([r[6] for r in rs], 50), "solve_p99_ms": pct([r[6] for r in rs], 99)}

    ok = [r for r in records if r[4] == 0]
    served_nodes = sum(r[2] for r in ok)
    cold_nodes = sum(r[2] for r in ok if r[0] == "cold")
    return {"workload": "Poisson %.0f req/s for %.0f s: new sessions of 70%% 2D RGB (sides 256-4096) and 30%% int16 "
                        "phantom volumes (sides 128-512), 1-5 warm stroke edits each (0.1-2%% of nodes); arrivals "
                        "finding %d cold requests unfinished are shed" % (rate, seconds, max_cold_outstanding),
            "arrivals": int(len(arrivals)), "shed": state["shed"], "sessions_served": len(served),
            "requests_ok": len(ok), "requests_failed": len(records) - len(ok) + len(failures),
            "failures": failures[:3],
            "offered_gnodes_s": state["offered_nodes"] / seconds / 1e9,
            "served_cold_gnodes_s": cold_nodes / wall / 1e9,
            "served_all_gnodes_s": served_nodes / wall / 1e9,
            "latency": {"cold_2d": lat("cold", 2), "cold_3d": lat("cold", 3),
                        "warm_2d": lat("warm", 2), "warm_3d": lat("warm", 3)},
            "cold_resolve_baseline": {"samples": len(base_ms), "p50_ms": pct(base_ms, 50),
                                      "bit_exact_vs_served": bool(exact)},
            "wall_s": wall, "arrival_window_s": t_arrivals,
            "budget_gb": budget_gb, "peak_used_gb": sstats["peak_used"] / 2**30,
            "peak_solving": sstats["peak_solving"], "loops": sstats["loops"]}


def bench_edit4096(jfcut, torch, ctx, n_edits=100):
    """Interactive edits at 4096^2: one 2D RGB session, n_edits sequential
    stroke edits (0.1-2% of nodes each) re-solved warm in the server, against
    a cold plain re-solve (build + the same edits + solve) of the same graph;
    flows must agree.  100 edits, so that p99 is a percentile rather than the
    single slowest edit."""
    w = h = 4096
    img, seeds = make_workload(w, h, SEED + 4096)
    rng = np.random.default_rng(SEED + 4097)
    edits = []
    for k in range(n_edits):
        m = max(1, int(w * h * rng.uniform(0.001, 0.02)))
        edits.append(synthetic.stroke(seeds.shape, seed=SEED + 7000 + k, n=m, label=1 + (k % 2)))
    srv = jfcut.Server(ctx, 0, max_slots=8)
    sid = srv.submit(img, seeds, jfcut.PIX_RGB8, MODEL)
    cold_first = srv.wait(sid).ms_total
    warm, flows = [], []
    for idx, ns in edits:
        srv.edit(sid, idx, ns)
        info = srv.wait(sid)
        warm.append(info.ms_total)
        flows.append(info.flow)
    srv.close()
    cold, exact = [], True
    for k in range(4, n_edits, max(1, n_edits // 5)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = jfcut.Graph(ctx, (h, w))
        g.build_from_image(img, seeds, jfcut.PIX_RGB8, MODEL)
        for idx, ns in edits[:k + 1]:
            g.edit_seeds(idx, ns)
        g.solve()
        cold.append((time.perf_counter() - t0) * 1e3)
        exact &= g.flow() == flows[k]
        g.close()
    return {"workload": "2D 4-conn RGB 4096x4096, %d sequential stroke edits (0.1-2%% of nodes)" % n_edits,
            "first_solve_ms": cold_first, "warm_p50_ms": pct(warm, 50), "warm_p99_ms": pct(warm, 99),
            "cold_resolve_p50_ms": pct(cold, 50), "cold_resolve_p99_ms": pct(cold, 99),
            "cold_samples": len(cold), "bit_exact_vs_cold": bool(exact),
            "warm_ms_first10": [round(v, 2) for v in warm[:10]], "warm_ms_max": round(max(warm), 2)}


def main():
    faulthandler.enable()   # a crash reports every thread's Python stack on stderr
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--width", type=int, default=W_FULL)
    ap.add_argument("--height", type=int, default=H_FULL)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--extras", default="video,batched,edit4096,serve,fastcut",
                    help="comma list of extra sections at N=1 (video, batched, edit4096, serve, fastcut) "
                         "or 'none'")
    ap.add_argument("--serve-seconds", type=float, default=20.0, help="arrival window of the serve section")
    ap.add_argument("--video-size", default="2560x1440x50", help="WxHxD of the video section")
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
    img, seeds = make_workload(w, h, replica_seed(rank))
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
        visits, ms_pr, sweeps, pr_phases = 0, 0.0, 0, 0
        agg = {"ms_total": 0.0, "ms_push_relabel": 0.0, "ms_global_relabel": 0.0, "ms_cut": 0.0,
               "global_relabels": 0, "bfs_passes": 0}
        for _ in range(args.steps):
            st = step_device()
            visits += st.tile_visits
            pr_phases += st.pr_phases
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
        ms = max_over_ranks(ms, dist)
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
        ms_e2e = max_over_ranks(ev0.elapsed_time(ev1), dist)

    ms_step = ms / args.steps
    value = replica_throughput(n, world, args.steps, ms)
    e2e = replica_throughput(n, world, args.steps, ms_e2e)
    # one push-relabel visit: a 32 x rows tile (32 x 8 halves of the 32 x 16
    # relabel tiles unless pr_mode 2), 48 B per node + 12 B per halo cell
    tr = ctx.params().tile_rows
    rows = 8 if tr == 16 and ctx.params().pr_mode != 2 else tr
    bytes_per_visit = 32 * rows * 48 + (2 * 32 + 2 * rows) * 12
    achieved = visits * bytes_per_visit / (ms_pr / 1000.0) / 1e9 if ms_pr > 0 else 0.0
    peak, peak_kind = peaks()
    pr_launches = pr_phases   # push-relabel phase launches in the timed steps
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mnodes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": workload_name(w, h),
                       "nodes": n, "global_batch": world, "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (state %.1f GB)" % (jfcut.lib().jfc_graph_bytes(2, w, h, 1) / 1e9),
                       "params": {"tile_rows": ctx.params().tile_rows, "local_iters": ctx.params().local_iters,
                                  "relabel_interval": ctx.params().relabel_interval or "auto (2 for 2D grids)"},
                       "flow": flow_ref, "sweeps_per_step": sweeps / args.steps,
                       "solve_breakdown_per_step": {k: v / args.steps for k, v in agg.items()},
                       "pr_tile_visits_per_step": visits / args.steps},
            "e2e": {"value": e2e, "unit": "Mnodes/s", "h2d_bytes_per_step": int(img.nbytes + seeds.nbytes),
                    "d2h_bytes_per_step": int(n)},
            "gpu_launches": int(launches),
            "clocks": clk,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": (pr_traffic_per_visit() * visits / max(1, pr_launches)
                                     if pr_traffic_per_visit() else None),
                         "algorithmic_bytes_per_launch": visits * bytes_per_visit / max(1, pr_launches),
                         "launches": pr_launches,
                         "kernel": "k_pr_phase / k_pr_async (push-relabel phases: parity sweeps, and the "
                                   "worklist after the exact relabel; %d B per tile visit algorithmic, %s peak; "
                                   "traffic: DRAM bytes per visit of the committed one-pass ncu capture of "
                                   "this workload's push-relabel launches times the visits per launch)"
                                   % (bytes_per_visit, peak_kind)},
        }
        if world == 1 and not args.no_cpu_baseline:
            print("bench: cpu baseline", file=sys.stderr, flush=True)
            line["cpu_baseline"] = cpu_baseline_bk(w, h, replica_seed(rank), flow_ref)
        extras = [] if world > 1 or args.extras == "none" else args.extras.split(",")
        vsize = tuple(int(v) for v in args.video_size.split("x"))
        sections = {"video": lambda: bench_video(jfcut, torch, ctx, stream, size=vsize),
                    "batched": lambda: bench_batched(jfcut, torch, ctx, stream, 2, 1),
                    "edit4096": lambda: bench_edit4096(jfcut, torch, ctx),
                    "fastcut": lambda: bench_fastcut(jfcut, torch),
                    "serve": lambda: bench_serve(jfcut, torch, ctx, seconds=args.serve_seconds)}
        with torch.cuda.stream(stream):
            for name in ("video", "batched", "edit4096", "serve", "fastcut"):
                if name in extras:
                    print("bench: section %s" % name, file=sys.stderr, flush=True)
                    t0 = time.perf_counter()
                    try:
                        line[name] = sections[name]()
                    except Exception as ex:   # a failed section is reported, the headline stands
                        line[name] = {"error": "%s: %s" % (type(ex).__name__, ex)}
                    line[name]["section_s"] = time.perf_counter() - t0
        print(json.dumps(line), flush=True)
    g.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
