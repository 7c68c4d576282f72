#!/usr/bin/env python
"""Benchmark: PKT truss edges/s on R-MAT-22 (bit-exact k-truss decomposition).

One step = one full PKT decomposition (orientation, triangle support, peel,
truss per CSR slot) of the workload graph.  Prints ONE JSON line on rank 0.

  value  device-resident inputs (CSR already in HBM), CUDA-event timed on the
         launching stream; edges/s = CSR width (directed slots, the
         reference's throughput factor g.width()) / time, summed over ranks.
  e2e    the same through the reference-layout C ABI call (sparx_pkt_run) with
         host u64 arrays: host->device upload and the download of the 32-bit
         truss numbers (one u32 per slot) are inside the timed region.
  --impl reference   the reference's CPU PKT (the oracle's restatement of
         pkt.rs, hash maps, all host threads) on a bounded sample of the same
         workload family.

Multi-GPU: a single graph does not shard (PKT's sub-level barrier would need a
cross-GPU exchange per sub-level), so for the R-MAT-22 workload N ranks run N
replicas (weak scaling).  Independent graphs do shard: --workload mix places
the batched mix's members on the ranks (LPT) and each rank decomposes its own
through shard.run_sharded_batch.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "PKT truss edges/s on R-MAT-22 (bit-exact)"
WORKLOADS = {
    "rmat22": dict(kind="rmat", scale=22, ef=16, seed=2,
                   desc="R-MAT scale 22, edge factor 16 (67,108,864 generated pairs), a=.57 b=.19 c=.19 "
                        "d=.05, seed 2, permuted ids, self-loops/duplicates removed, symmetrised"),
    "rmat20": dict(kind="rmat", scale=20, ef=16, seed=2, desc="R-MAT scale 20, edge factor 16, seed 2"),
    "rmat21": dict(kind="rmat", scale=21, ef=16, seed=2, desc="R-MAT scale 21, edge factor 16, seed 2"),
    "er1": dict(kind="er", n=100_000, m=1_000_000, seed=1,
                desc="Erdos-Renyi n=100,000, m=1,000,000 distinct pairs, seed 1 (config 1)"),
    "dbg": dict(kind="dbg", seq_len=20_000_000, k=21, copies=1000, seg_len=10_000, mut_rate=0.05, seed=3,
                desc="de Bruijn 21-mer graph of a 20,000,000-base seeded sequence plus 1,000 mutated 10 kb "
                     "segment copies, seed 3 (config 3)"),
}
CPU_SAMPLE_SCALE = 16


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_graph(spec):
    from sparkx_b200 import gen
    if spec["kind"] == "rmat":
        return gen.rmat(spec["scale"], spec["ef"], seed=spec["seed"])
    if spec["kind"] == "er":
        return gen.erdos_renyi(spec["n"], spec["m"], spec["seed"])
    if spec["kind"] == "dbg":
        return gen.debruijn(spec["seq_len"], spec["k"], spec["copies"], spec["seg_len"], spec["mut_rate"],
                            spec["seed"])
    raise ValueError(spec)


def oriented_sums(g):
    """S+ = sum over oriented edges of d+(a) + d+(b), and m (degree order, ties by id)."""
    off = g.offsets.astype(np.int64)
    nbr = g.neighbours.astype(np.int64)
    deg = np.diff(off)
    src = np.repeat(np.arange(g.n, dtype=np.int64), deg)
    up = (deg[src] < deg[nbr]) | ((deg[src] == deg[nbr]) & (src < nbr))
    a, b = src[up], nbr[up]
    dplus = np.bincount(a, minlength=g.n)
    return int((dplus[a] + dplus[b]).sum()), int(a.shape[0])


class ClockSampler:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, bus_id: str | None):
        self.rows = []
        self.proc = None
        self.sel = bus_id if bus_id else str(device_index)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", self.sel],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_pkt_sample(threads: int):
    """The reference's CPU PKT (restated, hash maps) on a bounded sample."""
    from oracle import oracle as O
    from sparkx_b200 import gen
    g = gen.rmat(CPU_SAMPLE_SCALE, 16, seed=2)
    t0 = time.perf_counter()
    O.pkt(g.offsets, g.neighbours, threads=threads, hash_map=True)
    dt = time.perf_counter() - t0
    sample = (f"full PKT (oracle restatement of pkt.rs/triangles.rs/impl_csc.rs, std::unordered_map, "
              f"{threads} threads) on R-MAT scale {CPU_SAMPLE_SCALE} ef 16 seed 2, "
              f"width {g.width} slots, same generator and parameters as the workload")
    return g.width / dt, dt, sample


def gpu_on_cpu_sample(opts, stream, dev):
    """The GPU on the CPU baseline's own sample graph (R-MAT-16), so one GPU/CPU pair exists on
    one graph: device-resident (CUDA events) and end to end (host u64 CSR in, u32 truss out)."""
    import torch
    from sparkx_b200 import gen, pkt
    g = gen.rmat(CPU_SAMPLE_SCALE, 16, seed=2)
    d_off = torch.from_numpy(g.offsets.view(np.int64)).to(dev)
    d_nbr = torch.from_numpy(g.neighbours.view(np.int32)).to(dev)
    d_out = torch.empty(g.width, dtype=torch.int32, device=dev)

    def step():
        pkt.run_pkt_device(d_off.data_ptr(), g.n + 1, d_nbr.data_ptr(), g.width, d_out.data_ptr(), opts,
                           stream.cuda_stream)
    for _ in range(3):
        step()
    steps = 10
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1) / steps
    nbr64 = g.neighbours.astype(np.uint64)
    pkt.run_pkt(g.offsets, nbr64, opts)
    times = []
    for _ in range(5):
        t1 = time.perf_counter()
        pkt.run_pkt(g.offsets, nbr64, opts)
        times.append(time.perf_counter() - t1)
    return {"graph": f"R-MAT scale {CPU_SAMPLE_SCALE} ef 16 seed 2 (the CPU baseline's sample), width {g.width}",
            "gpu_edges_per_s": g.width / (ms / 1000), "gpu_e2e_edges_per_s": g.width / statistics.median(times)}


def run_mix(args, rank=0, world=1, local=0):
    """Config 4: the batched mix, batched (one union per HBM budget, one launch per wave) vs one
    decomposition per call, in chunks of --mix-chunk members (bounded host memory).  Both arms
    decompose the same graphs and every member's truss numbers must agree.  With --autotune the
    knobs are first tuned on a sample of the mix (both arms then use the cache).  Under torchrun
    (N ranks) the members are placed with LPT and each rank generates and decomposes its own
    (shard.run_sharded_batch); times are the slowest rank's."""
    import torch
    from sparkx_b200 import gen, shard
    from sparkx_b200.pkt import PktOptions, autotune_batch, run_batch, run_pkt
    torch.cuda.set_device(local)
    opts = PktOptions(out_bits=32, device=local)
    members = [gen.mix_member(i) for i in range(args.mix_count)]
    works = [shard.work_estimate(m.n, 2 * m.pairs) for m in members]
    mine = shard.assign_lpt(works, world)[rank]
    tuned = None
    if args.autotune:
        sample = [gen.mix_graph(members[i]) for i in mine[: min(24, len(mine))]]
        tuned = autotune_batch([(g.offsets, g.neighbours) for g in sample], opts, repeats=2)
        log(f"rank {rank}: autotuned {tuned}")
    from concurrent.futures import ThreadPoolExecutor

    def make_member(m):
        gen.set_threads(1)
        return gen.mix_graph(m)
    gen_pool = ThreadPoolExecutor(max_workers=host_threads())
    warm = gen.mix_graph(members[mine[0]])
    run_batch([(warm.offsets, warm.neighbours)], opts)
    run_pkt(warm.offsets, warm.neighbours, opts)
    t_gen = t_batch = t_plain = dev_plain = dev_batch_union = 0.0
    slots = n_done = 0
    same = True
    small = {"batch": 0.0, "plain": 0.0, "count": 0}
    step = args.mix_chunk * world
    for c0 in range(0, len(members), step):
        chunk = list(range(c0, min(c0 + step, len(members))))
        # this rank's graphs of the chunk (the placement run_sharded_batch makes), generated in
        # parallel, one generator thread per graph: small graphs are dominated by per-graph setup
        mine_j = shard.assign_lpt([works[i] for i in chunk], world)[rank]
        t1 = time.perf_counter()
        loaded = dict(zip(mine_j, gen_pool.map(make_member, [members[chunk[j]] for j in mine_j])))
        t_gen += time.perf_counter() - t1

        def load(j):  # j indexes the chunk; each rank builds only the graphs placed on it
            g = loaded[j]
            return g.offsets, g.neighbours

        out = shard.run_sharded_batch([works[i] for i in chunk], load, opts=opts, gather=False)
        t_batch += out.seconds  # slowest rank's time for this chunk
        res = out.local
        assert all(r[2] == 0 for r in res.values()), [r[2] for r in res.values() if r[2]]
        seen = set()
        for r in res.values():  # members of a union share its phases: count each union once
            key = (r[1].ms_orient, r[1].ms_support, r[1].ms_peel)
            if key not in seen:
                seen.add(key)
                dev_batch_union += (r[1].ms_orient + r[1].ms_support + r[1].ms_peel + r[1].ms_finalize) / 1e3
        t_plain_chunk = 0.0
        for j, r in sorted(res.items()):
            g = loaded[j]
            t1 = time.perf_counter()
            t, st = run_pkt(g.offsets, g.neighbours, opts)
            dt = time.perf_counter() - t1
            t_plain_chunk += dt
            dev_plain += (st.ms_orient + st.ms_support + st.ms_peel + st.ms_finalize) / 1e3
            same &= bool(np.array_equal(t, r[0]))
            if g.n < 10_000:
                small["plain"] += dt
                small["count"] += 1
        t_plain += shard.max_over_ranks(t_plain_chunk, torch.device("cuda", local))
        sp = [(loaded[j].offsets, loaded[j].neighbours) for j in sorted(loaded) if loaded[j].n < 10_000]
        if sp:
            t1 = time.perf_counter()
            run_batch(sp, opts)
            small["batch"] += time.perf_counter() - t1
        slots += sum(g.width for g in loaded.values())
        n_done += len(loaded)
        log(f"rank {rank}: {n_done} members, batch {t_batch:.1f}s plain {t_plain:.1f}s gen {t_gen:.1f}s")
        del loaded, res, out
    same = shard.max_over_ranks(0.0 if same else 1.0, torch.device("cuda", local)) == 0.0
    if rank == 0:
        out = {"metric": "PKT batched mix graphs/s", "value": args.mix_count / t_batch, "unit": "graphs/s",
               "n_gpus": world, "per_graph_value": args.mix_count / t_plain, "batched_speedup": t_plain / t_batch,
               "n_graphs": args.mix_count, "slots_rank0": slots, "same_results_as_per_graph": same,
               "edges_per_s_batched_rank0": slots / t_batch,
               "device_seconds_rank0": {"per_graph_sum": dev_plain, "batched_unions_sum": dev_batch_union},
               "wall_seconds": {"batched": t_batch, "per_graph": t_plain, "generation_rank0": t_gen},
               "small_graphs_rank0": {"count": small["count"],
                                      "speedup": small["plain"] / small["batch"] if small["batch"] else None},
               "autotuned": None if tuned is None else {"tuning": tuned[0].__dict__, "key": list(tuned[1])},
               "config": {"workload": f"batched mix, members 0..{args.mix_count - 1} (config 4 distribution: "
                                      "ER or R-MAT 50/50, n log-uniform in [1e3,1e6], avg degree uniform [4,64], "
                                      "seeds 1000+i)", "chunk": args.mix_chunk,
                          "parallelism": f"LPT shards x{world}", "timing": "host wall clock per call "
                          "(the batch API is host-synchronous: uploads, decompositions and downloads), "
                          "max over ranks"}}
        print(json.dumps(out), flush=True)
    return 0


def run_serve(args):
    """Config 5: Poisson arrivals served with continuous batching vs plain per-graph calls."""
    import threading as th
    import torch  # noqa: F401
    from sparkx_b200 import gen
    from sparkx_b200.pkt import PktOptions, run_pkt
    from sparkx_b200.serve import PktServer
    rng = np.random.default_rng(5)
    graphs = [gen.mix_graph(gen.mix_member(i)) for i in range(args.mix_count)]
    if args.tail:
        ntail = max(1, len(graphs) // 100)
        for j in range(ntail):
            graphs.insert(int(rng.integers(0, len(graphs))), gen.rmat(24, 16, seed=100 + j))
    n = len(graphs)
    opts = PktOptions(out_bits=32)
    run_pkt(graphs[0].offsets, graphs[0].neighbours, opts)
    rows = []
    for rate in args.rates:
        gaps = rng.exponential(1.0 / rate, size=n)
        # served
        lat = [0.0] * n
        with PktServer(0, opts) as srv:
            t0 = time.perf_counter()
            tickets = []
            sched = np.cumsum(gaps)
            for i, g in enumerate(graphs):
                d = t0 + sched[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets.append((srv.submit(g.offsets, g.neighbours), time.perf_counter()))
            for i, (t, ts) in enumerate(tickets):
                r = srv.wait(t, timeout_ms=600_000)
                assert r.status == 0
                lat[i] = r.latency_ms
            span = time.perf_counter() - t0
            info = srv.info()
        # plain: one call at a time in arrival order (FIFO, single stream)
        plain_lat = []
        t0 = time.perf_counter()
        sched = np.cumsum(gaps)
        for i, g in enumerate(graphs):
            arrive = t0 + sched[i]
            d = arrive - time.perf_counter()
            if d > 0:
                time.sleep(d)
            run_pkt(g.offsets, g.neighbours, opts)
            plain_lat.append((time.perf_counter() - arrive) * 1000)
        span_plain = time.perf_counter() - t0
        rows.append({"rate_per_s": rate, "served_graphs_per_s": n / span, "plain_graphs_per_s": n / span_plain,
                     "served_p50_ms": float(np.percentile(lat, 50)), "served_p99_ms": float(np.percentile(lat, 99)),
                     "plain_p50_ms": float(np.percentile(plain_lat, 50)),
                     "plain_p99_ms": float(np.percentile(plain_lat, 99)),
                     "served_unions": info["unions"], "joined_running_union": info["joined"]})
        log(json.dumps(rows[-1]))
    out = {"metric": "PKT served stream latency/throughput", "n_requests": n, "tail_rmat24": bool(args.tail),
           "rows": rows,
           "config": {"workload": f"{n} requests: first {args.mix_count} members of the config-4 mix"
                                  + (" + 1% R-MAT-24 tail" if args.tail else "") + ", Poisson arrivals",
                      "budget": "150 GB (4 lanes: one of 75 GB, three of 25 GB; requests join running "
                                "unions at wave boundaries and leave when their own peel ends)"}}
    print(json.dumps(out), flush=True)
    return 0


def host_threads() -> int:
    return max(1, min(os.cpu_count() or 1, 255))


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle import oracle as O
    threads = host_threads()
    O.build()
    vals = []
    for i in range(args.warmup + args.steps):
        v, dt, sample = cpu_pkt_sample(threads)
        log(f"reference step {i}: {dt:.2f}s")
        if i >= args.warmup:
            vals.append((v, dt))
    value = statistics.median(v for v, _ in vals)
    ms = statistics.median(dt for _, dt in vals) * 1000
    spec = WORKLOADS[args.workload]
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        # the line names the graph it timed: the restatement's hash maps cost sum(d^2) ~ 5e11 on
        # R-MAT-22 (about 25 minutes per step on 16 threads), far past the bounded sample a
        # reference step may take; the GPU arm reports its own time on this same graph
        # ("same_graph") so one GPU/CPU pair exists on one graph
        "config": {"workload": f"R-MAT scale {CPU_SAMPLE_SCALE}, edge factor 16, seed 2 (same generator and "
                               f"parameters as the GPU arm's graph, 64x fewer vertices)",
                   "stands_for": spec["desc"]},
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["mix", "serve"], default="rmat22")
    ap.add_argument("--mix-count", type=int, default=256)
    ap.add_argument("--mix-chunk", type=int, default=256, help="mix: members generated and run per chunk")
    ap.add_argument("--autotune", action="store_true", help="mix: tune the knobs on a sample first")
    ap.add_argument("--rates", type=float, nargs="*", default=[50.0, 200.0, 1000.0])
    ap.add_argument("--tail", action="store_true", help="serve: add the 1% R-MAT-24 tail")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="device steps only (warm-up and steps as given), for profiler captures")
    ap.add_argument("--loop", choices=["graph", "host"], default="graph",
                    help="peel loop: CUDA-graph WHILE node (default) or host-launched waves")
    ap.add_argument("--support-kernel", type=int, default=0, choices=[0, 1, 2],
                    help="0 auto, 1 balanced edge form, 2 vertex form")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "mix":
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
            try:
                return run_mix(args, rank, world, local)
            finally:
                dist.barrier()
                dist.destroy_process_group()
        return run_mix(args)
    if args.workload == "serve":
        return run_serve(args)

    import torch
    from sparkx_b200 import pkt
    from sparkx_b200.pkt import PktOptions

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    spec = WORKLOADS[args.workload]
    t0 = time.perf_counter()
    g = make_graph(spec)
    log(f"rank {rank}: generated {args.workload}: n={g.n} width={g.width} in {time.perf_counter() - t0:.1f}s")
    n1 = g.n + 1
    dev = torch.device("cuda", local)
    d_off = torch.from_numpy(g.offsets.view(np.int64)).to(dev)
    d_nbr = torch.from_numpy(g.neighbours.view(np.int32)).to(dev)
    # 32-bit truss output: R-MAT-22's truss numbers exceed the reference's u8 layout (k_max 543)
    d_out = torch.empty(g.width, dtype=torch.int32, device=dev)
    opts = PktOptions(out_bits=32, device=local, loop=0 if args.loop == "graph" else 1,
                      support_kernel=args.support_kernel)
    stream = torch.cuda.current_stream(dev)

    def step():
        return pkt.run_pkt_device(d_off.data_ptr(), n1, d_nbr.data_ptr(), g.width, d_out.data_ptr(), opts,
                                  stream.cuda_stream)

    if args.profile:
        for _ in range(args.warmup + args.steps):
            st = step()
        torch.cuda.synchronize(dev)
        print(json.dumps({"profile": args.workload, "waves": st.waves, "ms_total": st.ms_total,
                          "ms_orient": st.ms_orient, "ms_support": st.ms_support,
                          "ms_peel": st.ms_peel, "launches": st.launches, "peel_elements": st.peel_elements,
                          "peel_hits": st.peel_hits, "peel_scanned": st.peel_scanned,
                          "compactions": st.compactions, "hub_maps": st.hub_maps,
                          "merge_iters": st.merge_iters,
                          "lane_iters": st.lane_iters, "merge_chunks": st.merge_chunks}), flush=True)
        return 0
    for _ in range(max(3, args.warmup)):
        st = step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    try:
        bus = torch.cuda.get_device_properties(dev).pci_bus_id
    except AttributeError:
        bus = None
    sampler = ClockSampler(local, None)
    sampler.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    ev0.record(stream)
    stats = []
    for _ in range(args.steps):
        stats.append(step())
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * g.width / (ms / 1000.0)

    # end to end: host u64 arrays (the reference's layout) through the C ABI
    g64_nbr = g.neighbours.astype(np.uint64)
    pkt.run_pkt(g.offsets, g64_nbr, opts)  # warm the staging path
    if dist:
        dist.barrier()
    e2e_times = []
    for _ in range(args.e2e_steps):
        t1 = time.perf_counter()
        out, st_e = pkt.run_pkt(g.offsets, g64_nbr, opts)
        e2e_times.append(time.perf_counter() - t1)
    e2e_s = statistics.median(e2e_times)
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    same = bool(np.array_equal(out, d_out.cpu().numpy().view(np.uint32)))

    last = stats[-1]
    peaks = {}
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    # algorithmic bytes of the two dominant kernels (units from the engine's counters)
    #   peel:    44 B per frontier edge, 8 B per shorter-row element, 24 B per triangle hit,
    #            16 B per active-list entry scanned
    #   support: 8 B per shorter-out-list element, 24 B per oriented edge, 24 B per triangle
    b_peel = 44 * last.peel_edges + 8 * last.peel_elements + 24 * last.peel_hits + 16 * last.peel_scanned
    b_sup = 8 * last.support_elements + 24 * last.m + 24 * last.triangles
    splus, _ = oriented_sums(g)
    b_sup_survey = 4 * splus + 24 * last.m + 16 * last.n + 16 * last.triangles
    ms_peel = statistics.median(s.ms_peel for s in stats)
    ms_sup = statistics.median(s.ms_support for s in stats)
    # DRAM traffic per unit from cold-cache ncu captures on R-MAT-21 (profiles/traffic.json),
    # scaled by the units this run processed: the peel's frontier elements (its scan waves are
    # not in the figure) and the support pass's elements
    traffic = traffic_sup = None
    prof = os.path.join(HERE, "profiles", "traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            tj = json.load(f)
        per_el = tj.get("k_wave", {}).get("dram_bytes_per_frontier_element")
        per_sup = tj.get("k_support_balanced", {}).get("dram_bytes_per_element")
        traffic = per_el * last.peel_elements if per_el else None
        traffic_sup = per_sup * last.support_elements if per_sup else None
    dominant = ("peel (k_wave in a CUDA-graph WHILE loop; each wave's last block plans the next)"
                if ms_peel >= ms_sup else "support (k_support_balanced)")
    roof_peel = {"kernel": "peel (k_wave, %d waves per run)" % last.waves, "bound": "hbm",
                 "achieved": b_peel / (ms_peel / 1000) / 1e9, "peak": hbm, "unit": "GB/s",
                 "frac": b_peel / (ms_peel / 1000) / 1e9 / hbm, "traffic": traffic,
                 "traffic_scope": "frontier waves; cold-cache capture of R-MAT-21's first sub-level, "
                                  "scaled by frontier elements",
                 "algorithmic_bytes_per_run": b_peel, "ms_per_run": ms_peel, "peak_source": peak_src}
    roof_sup = {"kernel": "k_support_balanced", "bound": "hbm",
                "achieved": b_sup / (ms_sup / 1000) / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": b_sup / (ms_sup / 1000) / 1e9 / hbm,
                "frac_survey_bytes": b_sup_survey / (ms_sup / 1000) / 1e9 / hbm, "traffic": traffic_sup,
                "traffic_scope": "cold-cache capture of R-MAT-21's support pass, scaled by elements",
                "algorithmic_bytes_per_run": b_sup, "survey_bytes_per_run": b_sup_survey,
                "ms_per_run": ms_sup, "peak_source": peak_src}
    roofline = roof_peel if ms_peel >= ms_sup else roof_sup

    cpu = None
    same_graph = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, dt, sample = cpu_pkt_sample(host_threads())
        cpu = {"value": v, "unit": "edges/s", "cores": host_threads(), "kind": "port", "sample": sample,
               "seconds": dt}
        same_graph = gpu_on_cpu_sample(opts, stream, dev)
        same_graph["cpu_edges_per_s"] = v

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": spec["desc"], "n": g.n, "width": g.width, "m": last.m,
                       "triangles": last.triangles, "k_max": last.k_max, "levels": last.levels,
                       "waves": last.waves, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (u32 ids %.0f MB)" % (4 * g.width / 1e6),
                       "dominant": dominant},
            "phases_ms": {"orient": last.ms_orient, "support": ms_sup, "peel": ms_peel,
                          "finalize": last.ms_finalize, "upload": last.ms_upload},
            "work": {"support_elements": last.support_elements, "peel_elements": last.peel_elements,
                     "peel_hits": last.peel_hits, "peel_scanned": last.peel_scanned,
                     "peel_edges": last.peel_edges, "compactions": last.compactions,
                     "merge_iters": last.merge_iters, "lane_iters": last.lane_iters,
                     "merge_chunks": last.merge_chunks},
            "e2e": {"value": world * g.width / e2e_s, "unit": "edges/s",
                    "h2d_bytes_per_step": 8 * n1 + 8 * g.width, "d2h_bytes_per_step": 4 * g.width,
                    "ms_per_step": e2e_s * 1000, "same_result_as_device_run": same},
            "gpu_launches": int(sum(s.launches for s in stats)),
            "roofline": roofline,
            "roofline_support": roof_sup,
            "roofline_peel": roof_peel,
            "cpu_baseline": cpu,
            "same_graph": same_graph,
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
