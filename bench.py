#!/usr/bin/env python
"""GCMC trial-move throughput on B200 (moves/s), plus the reference CPU arm.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload plain|batched]
    python bench.py --impl reference ...      # the reference algorithm on the host cores

Workloads (synthetic inputs written in FastMC's own CONTROL/FIELD/CONFIG formats):
  plain   -- one FP64 chain, 3392-atom cubic framework (a = 51.664 A), CO2 at 1 bar,
             kmax 12 (K = 4192), host move loop with every energy on the GPU.
A step is `--moves` trial moves of every chain on the rank.  Multi-GPU runs are independent
replicas per rank ("weak" scaling); the only collective is the timing barrier/max.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fastmc-1.4.0_b200"))
# before any CUDA context: separate hardware queues for the serving worker streams (the package
# sets the same default on import)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

PASS_SITES_MEAN_KEY = "pass_sites"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["plain", "batched", "serve", "mixture"])
    ap.add_argument("--serve-requests", type=int, default=1500)
    ap.add_argument("--serve-slots", type=int, default=296)
    ap.add_argument("--serve-moves", type=int, default=1000, help="moves per slot per serving step")
    ap.add_argument("--serve-voxel-edge", type=float, default=2.0, help="neighbour-list voxel edge of serving slots (A)")
    ap.add_argument("--serve-kcap", type=int, default=0, help="0: the largest request's K")
    ap.add_argument("--serve-cycle-scale", type=float, default=0.1,
                    help="scale of the U(2k,20k) cycle budgets so that requests finish within the run")
    ap.add_argument("--serve-sub-requests", type=int, default=1200,
                    help="batched workload: requests of the serving sub-record on the same line (0: none)")
    ap.add_argument("--serve-sub-scale", type=float, default=0.05,
                    help="cycle-budget scale of the serving sub-record's U(2k,20k) budgets")
    ap.add_argument("--moves", type=int, default=2000, help="trial moves per chain per step")
    ap.add_argument("--chains", type=int, default=256,
                    help="batched: the first N of the 256 chains (framework-major), for reduced profiling cases")
    ap.add_argument("--voxel-edge", type=float, default=0.0,
                    help="batched: neighbour-list voxel edge in A (0: picked by the autotuner)")
    ap.add_argument("--resident", action="store_true",
                    help="plain: passes through the resident pass kernel instead of a launch each")
    ap.add_argument("--tile", type=int, default=-1,
                    help="batched: index into the kernel's tile shapes (-1: picked by the autotuner)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bounded CPU baseline sample")
    ap.add_argument("--skip-baselines", action="store_true",
                    help="omit the plain-path and CPU samples (profiling runs of the batched kernel)")
    return ap.parse_args()


# ------------------------------------------------------------------ distributed plumbing
class Dist:
    """One process per GPU (NCCL); on a host without GPUs the same steps run over gloo, which is
    how the multi-rank logic is tested on CPU."""

    def __init__(self, n):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist

            backend = "gloo"
            if torch.cuda.is_available():
                torch.cuda.set_device(self.local)
                backend, self.device = "nccl", f"cuda:{self.local}"
            dist.init_process_group(backend, timeout=__import__("datetime").timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch

        t = torch.tensor([float(x)], device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.pg:
            return x
        import torch

        t = torch.tensor([float(x)], device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def ready(self, timeout=5.0):
        """Waits for the first sample, so that nvidia-smi's start-up stays outside a timed region."""
        t0 = time.perf_counter()
        while self.proc and time.perf_counter() - t0 < timeout:
            self.f.flush()
            if os.path.getsize(self.path) > 0 or self.proc.poll() is not None:
                return
            time.sleep(0.02)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel, key="traffic_bytes_per_launch"):
    """A DRAM-bytes figure of `kernel` from its committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", f"{kernel}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------------ workloads
def make_plain_deck(tmp):
    from fastmc_b200 import synth

    return synth.write_plain_large(os.path.join(tmp, "plain_large"))


def n_rc(deck_dir, info, nguest_sites):
    """Atoms within rcut of a site: framework density and current guest density."""
    import math

    vol = info["volm"]
    sphere = 4.0 / 3.0 * math.pi * info["rcut"] ** 3
    return (info["nframework"] + nguest_sites) / vol * sphere


def cpu_sample(deck, seed, guest_xyz, seconds, threads=1):
    """The oracle (the reference's algorithm restated) on host cores, starting from the GPU
    chain's state; returns aggregate moves/s over `threads` independent chains."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    chains = []
    for t in range(threads):
        c = oracle.Chain(deck, seed=(seed[0], seed[1], seed[2], (seed[3] + t) % 169))
        if guest_xyz is not None and len(guest_xyz):
            c.load_guests(0, guest_xyz.reshape(-1, 3))
        chains.append(c)
    # calibrate moves for ~seconds
    t0 = time.perf_counter()
    chains[0].run(200, trace=False)
    per = (time.perf_counter() - t0) / 200
    n = max(200, int(seconds / max(per, 1e-7)))
    done = [0] * threads

    def work(i):
        chains[i].run(n, trace=False)
        done[i] = n

    ths = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
    t0 = time.perf_counter()
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    dt = time.perf_counter() - t0
    return sum(done) / dt, n, dt


PLAIN_METRIC = "MC trial moves/s (plain FP64 single-chain GPU path)"
PLAIN_WORKLOAD = ("plain FP64 GPU drop-in: 3392-atom cubic framework a=51.664 A, CO2 1 bar, kmax 12 (K=4192), "
                  "host move loop")
BATCHED_METRIC = "MC trial moves/s on 1 B200 (batched vs plain)"


def run_plain(args, dist):
    import numpy as np

    import fastmc_b200 as fm

    tmp = tempfile.mkdtemp(prefix="fmcbench")
    deck = make_plain_deck(tmp)
    seed = (12, 34, 56, (78 + dist.rank) % 169)
    chain = fm.Chain(deck, seed=seed, device=dist.local)
    chain.resident(args.resident)
    info = chain.info()
    for _ in range(args.warmup):
        chain.run(args.moves, trace=False)
    chain.profile(-1)  # clear the launch counters ...
    chain.profile(0)  # ... and time no pass on its own inside the timed loop
    guests_at_start = chain.guest_coords(0)
    _, rl0, rp0 = chain.resident()
    dist.barrier()
    ms_total = 0.0
    traces = []
    with ClockSampler(dist.local) as clk:
        clk.ready()
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            tr, ms = chain.run_timed(args.moves, trace=True)
            traces.append(tr)
            ms_total += ms
        wall = time.perf_counter() - wall0
    dist.barrier()
    counts = chain.profile(0)  # passes and commits of the timed loop
    _, rl1, rp1 = chain.resident()
    # the pass kernel's own time for the roofline, from CUDA events around every pass of a further
    # run after the timed loop (per-pass events would slow the loop they time)
    chain.profile(-1)
    chain.run(args.moves, trace=False)
    prof = chain.profile(0)
    t_dev = dist.max(ms_total / 1000.0)
    t_wall = dist.max(wall)
    moves = args.steps * args.moves
    total_moves = dist.sum(moves)
    tr = np.concatenate(traces)
    sites = {1: 3, 2: 3, 3: 6, 4: 6, 5: 6}
    mean_sites = float(np.mean([sites[int(m)] for m in tr["mtype"]]))
    nsites_guest = float(np.mean(tr["nmols_after"])) * 3
    nrc = n_rc(deck, info, nsites_guest)
    bytes_per_launch = info["K"] * 40 + mean_sites * nrc * 36
    avg_kernel_s = prof["pass_ms"] / max(prof["timed_passes"], 1) / 1000.0
    achieved = bytes_per_launch / avg_kernel_s / 1e9
    peak, peak_kind = peaks()
    # launches in the timed loop: one per pass, or with the resident kernel its own launches plus
    # any pass it did not serve; commit kernels only where an update could not wait for the next pass
    launches = int(counts["passes"] - (rp1 - rp0) + (rl1 - rl0) + counts["commits"])
    # bytes crossing PCIe per step: trial sites (xyz, q, type) of every pass and of every commit
    # go host->device as kernel arguments; each pass returns {ewld1, ewld2, vdw} device->host
    acc = tr["accepted"] == 1
    h2d_total = sum(sites[int(m)] * 36 for m in tr["mtype"]) + int(np.sum(acc & (tr["mtype"] != 2))) * 3 * 36
    h2d = int(h2d_total / args.steps)
    d2h = int(counts["passes"] * 24 / args.steps)
    result = {
        "metric": PLAIN_METRIC,
        "value": total_moves / t_dev,
        "unit": "moves/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_dev * 1000.0 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded framework generator, FastMC input formats)",
        "config": {"workload": PLAIN_WORKLOAD, "moves_per_step": args.moves,
                   "resident_kernel": {"on": bool(args.resident), "launches": int(rl1 - rl0),
                                       "passes_served": int(rp1 - rp0)},
                   "chains_per_gpu": 1, "guests_mean": float(np.mean(tr["nmols_after"])),
                   "l2": "working set (S(k) 67 KB + framework 130 KB) is L2-resident; no flush between moves",
                   "parallelism": f"replicas{dist.world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": profiled_traffic("pass_kernel_plain_large"),
                     "kernel": "fmc_pass_kernel", "bytes_per_launch": bytes_per_launch,
                     "avg_launch_us": avg_kernel_s * 1e6, "peak_kind": f"{peak_kind} (hbm_gbs)"},
        "gpu_launches": launches,
        "e2e": {"value": total_moves / t_wall, "unit": "moves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "clocks": clk.summary(),
    }
    if dist.rank == 0 and dist.world == 1:
        cps, n, dt = cpu_sample(deck, seed, guests_at_start, args.cpu_seconds, threads=1)
        result["cpu_baseline"] = {"value": cps, "unit": "moves/s", "cores": 1, "kind": "port",
                                  "sample": f"{n} moves of the same chain from the GPU chain's state at "
                                            f"timing start, oracle FP64 restatement, 1 thread, {dt:.1f} s"}
    chain.close()
    return result


BATCHED_WORKLOAD = ("batched FP64: 256 chains = 16 orthorhombic frameworks (edges U(18,52) A, rho 0.025 A^-3, "
                    "edges < 25 A replicated) x 16 CO2 pressures log-spaced 0.01-10 bar, 298 K, kmax from a "
                    "0.9 A^-1 reciprocal cutoff, one persistent launch per step")


def make_batched_decks(tmp, nfw=16, npress=16):
    from fastmc_b200 import synth

    return synth.write_batched(os.path.join(tmp, "batched"), n_frameworks=nfw, n_pressures=npress)


def run_batched(args, dist):
    import math

    import numpy as np

    import fastmc_b200 as fm

    tmp = tempfile.mkdtemp(prefix="fmcbatch")
    t0 = time.perf_counter()
    from fastmc_b200 import synth

    n = max(1, min(args.chains, 256))
    dirs = synth.write_batched(os.path.join(tmp, "batched"), select=list(range(n)))
    seeds = [synth.batched_seed(i, dist.rank) for i in range(n)]
    # neighbour-list voxel edge: the autotuner times throwaway batches of the same chains
    tune = None
    edge = args.voxel_edge
    if edge <= 0:
        edge, tune = fm.autotune_voxel_edge(dirs, seeds, device=dist.local)
    # tile shape (threads per chain, k-vectors and candidates per loop trip): timed on one more
    # throwaway batch at that edge, each tile twice in palindromic order
    tiles = fm.batch_tiles()
    tile, tile_tune = args.tile, None
    if tile < 0:
        tile, tile_tune = fm.autotune_tiles(dirs, seeds, device=dist.local, voxel_edge=edge, warm_moves=args.moves,
                                            moves=args.moves // 2)
    b = fm.Batch(dirs, seeds, device=dist.local, voxel_edge=edge)
    b.tile = tile
    setup_s = time.perf_counter() - t0
    infos = {}
    for d in dirs:
        key = d.rsplit("_", 1)[0]
        if key not in infos:
            infos[key] = fm.deck_inspect(d)
    for _ in range(args.warmup):
        b.run(args.moves)
    dist.barrier()
    kernel_ms = 0.0
    with ClockSampler(dist.local) as clk:
        clk.ready()
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            _, ms = b.run(args.moves)
            kernel_ms += ms
        wall = time.perf_counter() - wall0
    dist.barrier()
    t_dev = dist.max(kernel_ms / 1000.0)
    t_wall = dist.max(wall)
    moves = n * args.moves * args.steps
    total_moves = dist.sum(moves)
    # load balance of the last timed launch: every CTA's own time on the device clock
    tm = b.timing()
    cta_ms = (tm[:, 1] - tm[:, 0]) / 1e6
    balance = {"cta_ms_max": float(cta_ms.max()), "cta_ms_mean": float(cta_ms.mean()),
               "cta_ms_min": float(cta_ms.min()), "max_over_mean": float(cta_ms.max() / cta_ms.mean()),
               "launch_span_ms": float((tm[:, 1].max() - tm[:, 0].min()) / 1e6),
               "sms_used": int(len(set(tm[:, 2].tolist())))}
    # algorithmic bytes of one launch: every move of every chain reads S(k), akk and writes
    # S_new (40 B per k-vector) and reads its sites' neighbours within rcut (36 B each)
    per_launch = 0.0
    states = [b.state(i) for i in range(n)]
    for d, st in zip(dirs, states):
        inf = infos[d.rsplit("_", 1)[0]]
        sphere = 4.0 / 3.0 * math.pi * inf["rcut"] ** 3
        nrc = (inf["nframework"] + 3 * st["nmol0"]) / inf["volm"] * sphere
        per_launch += args.moves * (inf["K"] * 40 + 4.5 * nrc * 36)
    avg_launch_s = t_dev / args.steps
    achieved = per_launch / avg_launch_s / 1e9
    # ncu DRAM bytes per chain-move (captured on a 200-move launch), scaled to this launch
    tpm = profiled_traffic("batch_kernel_batched", "traffic_bytes_per_chain_move")
    traffic = tpm * n * args.moves if tpm else None
    peak, peak_kind = peaks()
    from fastmc_b200._lib import lib as _l
    cb = int(_l().fmc_batch_control_block_bytes())  # one chain's control block, moved each way per step
    result = {
        "metric": BATCHED_METRIC,
        "value": total_moves / t_dev,
        "unit": "moves/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_dev * 1000.0 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded framework generator, FastMC input formats)",
        "config": {"workload": BATCHED_WORKLOAD, "chains": n, "moves_per_chain_per_step": args.moves,
                   "guests_mean": float(np.mean([s["nmol0"] for s in states])),
                   "K_range": [int(min(i["K"] for i in infos.values())), int(max(i["K"] for i in infos.values()))],
                   "setup_s": setup_s, "voxel_edge_A": edge, "load_balance": balance,
                   "voxel_autotune_ms": tune,
                   "tile": {"index": tile, "threads_per_chain": tiles[tile][0], "kvec_per_trip": tiles[tile][1],
                            "cand_per_trip": tiles[tile][2], "chains_per_cta": 1},
                   "tile_autotune_ms": ({f"{tiles[k][0]}/{tiles[k][1]}/{tiles[k][2]}": v for k, v in tile_tune.items()}
                                        if tile_tune else None),
                   "l2": "per-chain S(k) is shared-memory resident; frameworks + voxel lists exceed L2 (no flush)",
                   "parallelism": f"replicas{dist.world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "fmc_batch_kernel",
                     "bytes_per_launch": per_launch, "avg_launch_us": avg_launch_s * 1e6,
                     "peak_kind": f"{peak_kind} (hbm_gbs)"},
        "gpu_launches": args.steps,
        "e2e": {"value": total_moves / t_wall, "unit": "moves/s", "h2d_bytes_per_step": n * cb,
                "d2h_bytes_per_step": n * (cb + 24)},
        "clocks": clk.summary(),
    }
    if dist.rank == 0 and dist.world == 1 and not args.skip_baselines:
        # the plain single-chain GPU path on a sample of the same chains
        sample = list(range(0, n, max(1, n // 8)))[:8]
        pm, pt = 0, 0.0
        for i in sample:
            c = fm.Chain(dirs[i], seed=seeds[i], device=dist.local)
            g = b.guest_coords(i, 0)
            if len(g):
                c.set_guests(0, g)
            c.run(200, trace=False)
            _, ms = c.run_timed(1000)
            pm += 1000
            pt += ms / 1000.0
            c.close()
        result["plain_moves_per_s"] = pm / pt
        result["batched_vs_plain"] = result["value"] / result["plain_moves_per_s"]
        # CPU baseline: the oracle on the same sampled chains, from the GPU chains' states
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        oracle.build()
        cm, ct = 0, 0.0
        budget = args.cpu_seconds / len(sample)
        for i in sample:
            oc = oracle.Chain(dirs[i], seed=seeds[i])
            g = b.guest_coords(i, 0)
            if len(g):
                oc.load_guests(0, g.reshape(-1, 3))
            t1 = time.perf_counter()
            oc.run(100, trace=False)
            per = (time.perf_counter() - t1) / 100
            k = max(100, int(budget / max(per, 1e-7)))
            t1 = time.perf_counter()
            oc.run(k, trace=False)
            ct += time.perf_counter() - t1
            cm += k
        result["cpu_baseline"] = {"value": cm / ct, "unit": "moves/s", "cores": 1, "kind": "port",
                                  "sample": f"{cm} moves over {len(sample)} of the 256 chains (every "
                                            f"{max(1, n // 8)}th), each from its GPU chain's state, oracle "
                                            f"FP64 restatement, 1 thread, {ct:.1f} s"}
    b.close()
    if args.serve_sub_requests > 0:
        # the serving half of the metric on the same line: p50/p99 time-to-completion beside the
        # aggregate moves/s of continuous batching (bounded run; its own timing and clocks)
        srv, log, done_t, arrivals, wall, clk, meta = serve_record(args, dist, args.serve_sub_requests,
                                                                  args.serve_sub_scale, "serve_sub")
        rec = summarize_serve(args, dist, srv, log, done_t, arrivals, wall, meta, args.serve_sub_scale,
                              args.serve_sub_requests)
        srv.close()
        rec["clocks"] = clk.summary()
        result["serve"] = rec
    return result


MIXTURE_WORKLOAD = ("batched binary mixture: 256 chains = the 16 batched frameworks x 16 seeds, CO2/N2 at 15:85 "
                    "mole fraction and 1 bar total, 298 K, one persistent launch per step")


def run_mixture(args, dist):
    """The binary-mixture batched workload (FP64): 256 chains of CO2/N2 at 15:85 and 1 bar."""
    import numpy as np

    import fastmc_b200 as fm
    from fastmc_b200 import synth

    tmp = tempfile.mkdtemp(prefix="fmcmix")
    dirs = synth.write_batched(os.path.join(tmp, "mix"), gases=("CO2", "N2"), fractions=(0.15, 0.85), total_bar=1.0)
    n = len(dirs)
    seeds = [synth.batched_seed(i, dist.rank) for i in range(n)]
    edge = args.voxel_edge if args.voxel_edge > 0 else 1.0
    b = fm.Batch(dirs, seeds, device=dist.local, voxel_edge=edge)
    for _ in range(args.warmup):
        b.run(args.moves)
    dist.barrier()
    ms_tot = 0.0
    with ClockSampler(dist.local) as clk:
        clk.ready()
        for _ in range(args.steps):
            ms_tot += b.run(args.moves)[1]
    t_dev = dist.max(ms_tot / 1000.0)
    moves = dist.sum(n * args.moves * args.steps)
    states = [b.state(i) for i in range(n)]
    b.close()
    return {
        "metric": "MC trial moves/s on 1 B200 (batched binary mixture)", "value": moves / t_dev,
        "unit": "moves/s", "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev * 1000.0 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded framework generator, FastMC input formats)",
        "config": {"workload": MIXTURE_WORKLOAD, "chains": n, "moves_per_chain_per_step": args.moves,
                   "voxel_edge_A": edge, "guests_mean": {"CO2": float(np.mean([s["nmol0"] for s in states])),
                                                         "N2": float(np.mean([s["nmol1"] for s in states]))},
                   "precision": "FP64 (the FP32 build, measured slower and outside 1e-6, was removed)",
                   "parallelism": f"replicas{dist.world}"},
        "gpu_launches": args.steps, "clocks": clk.summary(),
    }


def _write_request(job):
    from fastmc_b200 import synth

    path, req = job
    return synth.write_request(path, req)


def write_requests(root, reqs):
    """Request decks are client-side inputs: written before any GPU work, in a spawn pool."""
    import multiprocessing as mp

    jobs = [(os.path.join(root, f"req_{r['id']:05d}"), r) for r in reqs]
    with mp.get_context("spawn").Pool(max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        return pool.map(_write_request, jobs, chunksize=4)


SERVE_WORKLOAD = ("serving: Poisson stream of isotherm-point requests, each a fresh cubic framework of 400-6000 "
                  "atoms (rho 0.025 A^-3), gas CO2 / N2 / CH4, T U(273,348) K, P log-U(0.01,10) bar, cycle budget "
                  "U(2k,20k) x {scale} per phase (a cycle = N_guests+1 moves), continuous batching over {slots} slots")


def serve_record(args, dist, n_req, cycle_scale, tag):
    """Continuous-batching server on a Poisson request stream: time-to-completion p50/p99, device
    and end-to-end moves/s over the loaded window (the steps started while requests still
    arrived), slot occupancy.  A saturating pilot first measures the server's capacity; arrivals
    are then offered at 90% of it."""
    import numpy as np

    from fastmc_b200 import synth

    tmp = tempfile.mkdtemp(prefix="fmcserve")
    n_pilot = args.serve_slots + 64
    reqs = synth.serving_requests(n_pilot + n_req, seed=7 + 1000 * dist.rank)
    for r in reqs:
        r["cycles"] = max(1, int(round(r["cycles"] * cycle_scale)))
    t0 = time.perf_counter()
    dirs = write_requests(os.path.join(tmp, tag), reqs)  # spawned pool
    gen_s = time.perf_counter() - t0
    import fastmc_b200 as fm

    # k capacity: the largest request's K (cubic cells: K grows with the edge)
    kcap = args.serve_kcap or int(fm.deck_inspect(dirs[int(np.argmax([r["edge"] for r in reqs]))])["K"])
    srv = fm.Server(slots=args.serve_slots, device=dist.local, k_capacity=kcap, voxel_edge=args.serve_voxel_edge)
    # pilot (warm-up): more requests than slots at once; the launches that ran with every slot busy
    # give the server's capacity in moves/s
    ids = [srv.submit(d, (12, 34, 56, 1 + r["id"] % 168)) for d, r in zip(dirs[:n_pilot], reqs[:n_pilot])]
    full_ms, full_wall, full_moves = [], 0.0, 0
    while srv.busy():
        t_step = time.perf_counter()
        a, q, ms = srv.step(args.serve_moves)
        if a == args.serve_slots:
            full_ms.append(ms)
            full_wall += time.perf_counter() - t_step
            full_moves += int(srv.stats()["last_moves"])
    srv.poll_done()
    pil = [srv.poll(i) for i in ids]
    moves_per_req = float(np.mean([r["moves"] for r in pil]))
    capacity = args.serve_slots * args.serve_moves / (float(np.median(full_ms)) / 1000.0) if full_ms else None
    rate = 0.9 * capacity / moves_per_req if capacity else 50.0
    rng = np.random.default_rng(99 + dist.rank)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    dist.barrier()
    live, done_t = {}, {}
    nxt = 0
    log = []  # per step: wall start, wall end, device ms and moves of the launch it completed, slots in it
    with ClockSampler(dist.local) as clk:
        clk.ready()
        wall0 = time.perf_counter()
        while len(done_t) < n_req:
            now = time.perf_counter() - wall0
            while nxt < n_req and arrivals[nxt] <= now:
                rid = srv.submit(dirs[n_pilot + nxt], (12, 34, 56, 1 + reqs[n_pilot + nxt]["id"] % 168))
                live[rid] = nxt
                nxt += 1
            if not srv.busy():
                time.sleep(max(0.0, min(arrivals[nxt] - now, 0.05)) if nxt < n_req else 0.0)
                continue
            a, q, ms = srv.step(args.serve_moves)
            end = time.perf_counter() - wall0
            log.append((now, end, ms, int(srv.stats()["last_moves"]) if ms > 0 else 0, a))
            for rid, state, _ in srv.poll_done():
                if rid in live:
                    k = live.pop(rid)
                    done_t[k] = (end - arrivals[k], state)
        wall = time.perf_counter() - wall0
    dist.barrier()
    saturated = {"what": "the pilot's launches with every slot busy", "steps": len(full_ms),
                 "moves": full_moves, "device_s": sum(full_ms) / 1000.0, "wall_s": full_wall,
                 "moves_per_device_s": full_moves / max(sum(full_ms) / 1000.0, 1e-9),
                 "moves_per_wall_s": full_moves / max(full_wall, 1e-9), "slot_occupancy": 1.0}
    return srv, log, done_t, arrivals, wall, clk, {"capacity": capacity, "rate": rate, "n_pilot": n_pilot,
                                                   "moves_per_req": moves_per_req, "gen_s": gen_s, "kcap": kcap,
                                                   "saturated": saturated}


def summarize_serve(args, dist, srv, log, done_t, arrivals, wall, meta, cycle_scale, n_req):
    import numpy as np

    lat = np.array([v[0] for v in done_t.values()])
    rejected = sum(1 for v in done_t.values() if v[1] != srv.DONE)
    t_last = float(arrivals[-1])
    win = [x for x in log if x[0] <= t_last]
    w_moves = sum(x[3] for x in win)
    w_dev = sum(x[2] for x in win) / 1000.0
    w_wall = win[-1][1] if win else 0.0
    w_occ = sum(x[4] * x[2] for x in win) / max(sum(x[2] for x in win), 1e-9) / args.serve_slots
    all_moves = sum(x[3] for x in log)
    dev_ms = sum(x[2] for x in log)
    occ = sum(x[4] * x[2] for x in log)
    t_dev = dist.max(w_dev)
    t_wall = dist.max(w_wall)
    total = dist.sum(w_moves)
    used, budget = srv.memory()
    sstats = srv.stats()
    from fastmc_b200._lib import lib as _l
    cb, sb = int(_l().fmc_batch_control_block_bytes()), int(_l().fmc_system_block_bytes())
    return {
        "value": total / t_dev, "e2e_value": total / t_wall, "unit": "moves/s",
        "e2e_over_device": (total / t_wall) / (total / t_dev),
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "mean": float(lat.mean()), "max": float(lat.max())},
        "requests": n_req, "rejected": rejected, "cycle_scale": cycle_scale,
        "workload": SERVE_WORKLOAD.format(scale=cycle_scale, slots=args.serve_slots),
        "pilot_requests": meta["n_pilot"], "arrival_rate_hz": meta["rate"],
        "capacity_moves_per_s": meta["capacity"], "offered_load": 0.9, "moves_per_request_mean": meta["moves_per_req"],
        "moves_per_step": args.serve_moves, "k_capacity": meta["kcap"], "deck_generation_s": meta["gen_s"],
        "voxel_edge_A": args.serve_voxel_edge,
        "saturated": meta["saturated"],
        "window": {"what": "device and end-to-end figures cover the steps started before the last arrival",
                   "steps": len(win), "moves": w_moves, "device_s": w_dev, "wall_s": w_wall,
                   "slot_occupancy": w_occ},
        "whole_run": {"steps": len(log), "moves": all_moves, "device_s": dev_ms / 1000.0, "wall_s": wall,
                      "moves_per_device_s": all_moves / max(dev_ms / 1000.0, 1e-9),
                      "moves_per_wall_s": all_moves / max(wall, 1e-9),
                      "slot_occupancy": occ / max(dev_ms, 1e-9) / args.serve_slots},
        "h2d_bytes_per_step": args.serve_slots * (sb + cb), "d2h_bytes_per_step": args.serve_slots * cb,
        "memory": {"slots_bytes_at_end": used, "budget_bytes": budget}, "server": sstats,
    }


def run_serve(args, dist):
    """The serving workload on its own line (metric: moves/s with p50/p99 time-to-completion)."""
    srv, log, done_t, arrivals, wall, clk, meta = serve_record(args, dist, args.serve_requests,
                                                              args.serve_cycle_scale, "serve")
    rec = summarize_serve(args, dist, srv, log, done_t, arrivals, wall, meta, args.serve_cycle_scale,
                          args.serve_requests)
    srv.close()
    w = rec["window"]
    return {
        "metric": "MC trial moves/s on 1 B200 (continuous-batching serving); p50/p99 time-to-completion",
        "value": rec["value"], "unit": "moves/s", "n_gpus": dist.world, "steps": w["steps"], "warmup": 1,
        "ms_per_step": w["device_s"] * 1000.0 / max(w["steps"], 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded request generator, FastMC input formats)",
        "config": {"workload": rec["workload"], "requests": rec["requests"], "pilot_requests": rec["pilot_requests"],
                   "arrival_rate_hz": rec["arrival_rate_hz"], "capacity_moves_per_s": rec["capacity_moves_per_s"],
                   "offered_load": 0.9, "moves_per_request_mean": rec["moves_per_request_mean"],
                   "moves_per_step": args.serve_moves, "k_capacity": rec["k_capacity"],
                   "voxel_edge_A": args.serve_voxel_edge,
                   "l2": "per-chain S(k) shared-memory resident; frameworks + voxel lists exceed L2 (no flush)",
                   "parallelism": f"replicas{dist.world}"},
        "latency_s": rec["latency_s"], "rejected": rec["rejected"], "saturated": rec["saturated"],
        "window": rec["window"],
        "whole_run": rec["whole_run"], "gpu_launches": w["steps"],
        "e2e": {"value": rec["e2e_value"], "unit": "moves/s", "h2d_bytes_per_step": rec["h2d_bytes_per_step"],
                "d2h_bytes_per_step": rec["d2h_bytes_per_step"]},
        "clocks": clk.summary(), "memory": rec["memory"], "server": rec["server"],
    }


def run_reference(args, dist):
    """The reference algorithm (oracle restatement; the Fortran reference cannot be built here)
    on all host cores, on the default arm's workload: one chain per thread at a time, like the
    reference's independent MPI replicas."""
    if dist.rank != 0:
        return None
    tmp = tempfile.mkdtemp(prefix="fmcref")
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    if args.workload == "plain":
        dirs = [make_plain_deck(tmp)] * threads
        metric = PLAIN_METRIC
        workload = PLAIN_WORKLOAD
    else:
        dirs = make_batched_decks(tmp)
        metric = BATCHED_METRIC
        workload = BATCHED_WORKLOAD
    n = len(dirs)
    seeds = [(12, 34, 56, (78 + 7 * i) % 169) for i in range(n)]
    chains = [oracle.Chain(d, seed=s) for d, s in zip(dirs, seeds)]
    # bounded sample per step: ~4 s of moves per thread, on chains taken round-robin
    t0 = time.perf_counter()
    chains[0].run(100, trace=False)
    per = (time.perf_counter() - t0) / 100
    m = max(50, int(4.0 / max(per, 1e-7)))
    state = {"next": 0}

    def step():
        pick = [(state["next"] + t) % n for t in range(threads)]
        state["next"] = (state["next"] + threads) % n
        ths = [threading.Thread(target=lambda c=chains[i]: c.run(m, trace=False)) for i in pick]
        for th in ths:
            th.start()
        for th in ths:
            th.join()

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    v = args.steps * m * threads / dt
    return {
        "metric": metric, "value": v, "unit": "moves/s",
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1000 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded framework generator, FastMC input formats)",
        "config": {"workload": workload, "chains": n, "moves_per_thread_per_step": m, "threads": threads},
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "moves/s", "cores": threads, "kind": "port",
                         "sample": f"{m} moves per thread per step, {threads} threads each on one of the {n} "
                                   f"chains (round-robin over steps), oracle FP64 restatement of the reference"},
        "e2e": {"value": v, "unit": "moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    dist = Dist(args.gpus)
    try:
        if args.impl == "reference":
            res = run_reference(args, dist)
        elif args.workload == "plain":
            res = run_plain(args, dist)
        elif args.workload == "serve":
            res = run_serve(args, dist)
        elif args.workload == "mixture":
            res = run_mixture(args, dist)
        else:
            res = run_batched(args, dist)
        if dist.rank == 0 and res is not None:
            print(json.dumps(res))
    finally:
        dist.close()


if __name__ == "__main__":
    main()
