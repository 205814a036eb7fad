#!/usr/bin/env python
"""AWSEM-MD step benchmark: residue-steps/s on one B200.

Workload (default, `--workload c3`): benchmark configuration 3, 1,024
independent single-chain replicas with lengths uniform in [40, 500] residues
(278,062 residues), each built as in configuration 0 from its own seed with
its own fragment-memory tables (20 memories per 9-residue window), all AWSEM
terms on, pair vexcluded, harmonic bonds, Langevin 300 K, dt 2 fs, damping
500 fs.  The batched form advances all replicas with one launch sequence per
MD step (captured in CUDA graphs), in the mixed arithmetic form.  One bench
step = `--md-steps` MD steps of every replica.

`--workload c1`: configuration 1, one system of 8 chains x 250 residues.

Timing: W untimed warm-up bench steps, then K timed ones; L2 is flushed (a
512 MiB write) before each; device time from CUDA events on the engine's
stream; with N GPUs every rank runs its own copy of the workload (replicas
only) and the slowest rank's time sets the aggregate.

Reported beside the headline: the plain single-instance FP64 form on the
same replicas (one replica at a time, a sample), the end-to-end rate through
the C ABI with host buffers, the roofline of the dominant kernel, and the
reference CPU implementation on a bounded sample (`cpu_baseline`).
`--impl reference` times the reference implementation (FixBackbone +
PairExcludedVolume compiled unmodified against the LAMMPS-API shim) on the
box's host cores on the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0
RUN = dict(dt=2.0, t_start=300.0, t_stop=300.0, damp=500.0)
CACHE = os.path.join(tempfile.gettempdir(), "awsem_chain_cache")

C2_CPU_NOTE = ("the reference keeps n x n pair caches (cR, cWell, cP_AP in smart_matrix_lib.h; about 128 bytes "
               "per residue pair): about 205 GB at 40,000 residues")


WORKLOADS = {
    "c3": "config3: 1,024 independent chains, lengths uniform in [40, 500] (278,062 residues), each with its own "
          "fragment-memory tables (20 memories per 9-residue window), all AWSEM terms, pair vexcluded, harmonic "
          "bonds, Langevin 300 K, dt 2 fs, damping 500 fs",
    "c1": "config1: 8 chains x 250 residues (2,000 residues, 6,000 beads), 150 A cube, all AWSEM terms + fragment "
          "memory (20 memories per 9-residue window), pair vexcluded, harmonic bonds, Langevin 300 K, dt 2 fs, "
          "damping 500 fs",
    "c2": "config2: one system of 160 chains x 250 residues (40,000 residues) randomly packed in a 320 A cube "
          "(0.0012 residues/A^3), all AWSEM terms + fragment memory (20 memories per 9-residue window), pair "
          "vexcluded, harmonic bonds, Langevin 300 K, dt 2 fs, damping 500 fs, skin 2 A, list rebuilt every 10 "
          "steps (cell grid)",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=list(WORKLOADS))
    ap.add_argument("--md-steps", type=int, default=None, help="MD steps per bench step")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--replicas", type=int, default=1024, help="c3: number of replicas")
    ap.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--shapes", default=None,
                    help="launch shapes d,p,h,f (as autotune reports them) instead of autotuning, e.g. for profiling")
    ap.add_argument("--serve-requests", type=int, default=750,
                    help="configuration-4 stream: requests served after the batched measurement (0: skip)")
    ap.add_argument("--serve-plain", type=int, default=8,
                    help="configuration-4 stream: its first requests also served one at a time in plain FP64")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the error-against-oracle, configuration-1 and configuration-2 measurements")
    ap.add_argument("--serve-steps", type=int, default=20000, help="MD steps of each served request")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0, help="HBM budget of the serving handle")
    a = ap.parse_args()
    if a.md_steps is None:
        a.md_steps = {"c3": 20, "c2": 50}.get(a.workload, 100)
    return a


# --------------------------------------------------------------------------

class Dist:
    """One process per GPU; replicas only (no data-path collective).  NCCL
    on GPUs; gloo when there is no GPU (the CPU tests of the rank logic)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            timeout = datetime.timedelta(seconds=600)
            if torch.cuda.is_available():
                torch.cuda.set_device(self.local)
                self.device = f"cuda:{self.local}"
                dist.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group("gloo", timeout=timeout)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        """The largest value over the ranks (timings: the slowest rank)."""
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.rows, self.proc, self.thread = gpu, [], None, None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [num(r[1]) for r in self.rows if num(r[1])]
        mx = [num(r[2]) for r in self.rows if num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def flush_l2(buf):
    import torch

    buf.fill_(1.0)
    torch.cuda.synchronize()


def peaks():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM, "fallback"


# --------------------------------------------------------------------------
# workloads

def c3_chain(L: int, seed: int) -> dict:
    """Configuration-3 chain in array form, cached on disk by (L, seed)."""
    from awsemmd_b200 import synth

    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"chain_{L}_{seed}.npz")
    if os.path.exists(path):
        try:
            z = np.load(path)
            c = {k: z[k] for k in z.files}
            for k in ("seq", "mem_seq"):
                c[k] = bytes(c[k])
            for k in ("n_res", "n_mem"):
                c[k] = int(c[k])
            return c
        except Exception:
            pass
    c = synth.chain_arrays(L, seed)
    tmp = path + f".{os.getpid()}.npz"
    np.savez(tmp, **{k: (np.frombuffer(v, dtype=np.uint8) if isinstance(v, bytes) else v) for k, v in c.items()})
    os.replace(tmp, path)
    return c


def _gen_chain(args):
    L, seed = args
    sys.path.insert(0, ROOT)
    c3_chain(L, seed)
    return 0


def prefetch_chains(pairs):
    """Generate the (length, seed) chains missing from the on-disk cache,
    in parallel over the host cores (spawned processes)."""
    todo = sorted({(int(L), int(s)) for L, s in pairs
                   if not os.path.exists(os.path.join(CACHE, f"chain_{int(L)}_{int(s)}.npz"))})
    if not todo:
        return
    os.makedirs(CACHE, exist_ok=True)
    # spawned workers re-import the main module: only bench.py itself (whose
    # work sits behind its __main__ guard) may start them; other callers
    # generate in this process
    main = getattr(sys.modules.get("__main__"), "__file__", None)
    if len(todo) < 8 or not main or os.path.abspath(main) != os.path.abspath(__file__):
        for L, seed in todo:
            c3_chain(L, seed)
        return
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, 32)) as pool:
        pool.map(_gen_chain, todo, chunksize=4)


def c3_lengths(n: int):
    from awsemmd_b200 import synth

    return synth.replica_lengths(n=1024)[:n]


def c3_seed(k: int, rank: int = 0) -> int:
    return 3000 + k + 100000 * rank


# DRAM bytes (read + write) per algorithmic byte of a launch, from one ncu
# capture of the kernel on the first 256 replicas of configuration 3, whose
# fragment-memory table (458 MB) is larger than L2
# (profiles/sections_c3_256replicas.txt: 483.8 MB for 458.1 MB)
TRAFFIC_PER_ALGORITHMIC_BYTE = {"fragmem": 483.8 / 458.053744}
TRAFFIC_SOURCE = "ncu dram read+write of a 256-replica launch per algorithmic byte, times this launch's algorithmic " \
                 "bytes (profiles/sections_c3_256replicas.txt)"


def workload_text(args) -> str:
    if args.workload == "c3" and args.replicas != 1024:
        return (f"first {args.replicas} replicas of " + WORKLOADS["c3"]).replace(" (278,062 residues)", "")
    return WORKLOADS[args.workload]


def algorithmic_bytes(kernel: str, info) -> float:
    """Bytes one launch must move at least (data layout of the engine):
    fragmem -- every stored memory distance once, the block table, the two
    target beads per residue and the force accumulators it updates;
    radial / pair / density / water_xi -- the residue pair array (8 bytes a pair)
    once, every residue's working coordinates and per-residue scalars once,
    the force accumulators once."""
    n_res, n_atoms, records, rbytes, nd, pcap, npairs, nonuni = [int(v) for v in info]
    bead = 32
    if kernel == "fragmem":
        return (records * 4 * rbytes + records * rbytes * nonuni + ((n_res + 31) // 32) * nd * 8 + n_res * 2 * bead
                + n_res * 2 * 3 * 8 * 2)
    if kernel in ("radial", "pair", "density", "water_xi"):
        return npairs * 8 + n_res * 6 * bead + n_res * 10 * 8 + n_res * 4 * 4 + n_atoms * 3 * 8
    if kernel == "prepare":
        return n_atoms * 3 * 8 + n_res * 6 * bead + n_atoms * 3 * 8 + n_res * 32
    if kernel == "finish":
        return n_atoms * 3 * 8 * 5 + n_res * 8
    return n_res * 6 * bead


# --------------------------------------------------------------------------
# CPU reference (the shim-hosted reference FixBackbone + PairExcludedVolume)

# categories of the reference's timer.log (final_log_output, fix_backbone.cpp:1186-1206)
TIMER_NAMES = ["Chain", "Shake", "Chi", "Rama", "Vexcluded", "DSSP", "PAP", "Water", "Burial", "Helix", "AHM-Go",
               "Frag_Mem", "Vec_FM", "Membrane", "SSB", "DH", "Frust_Analysis", "Pair", "Pair_Double_Loop1",
               "Pair_Single_Loop", "Pair_Double_Loop2", "Pair_Double_Loop3", "Total"]
# the GPU kernels that do the work of each timed reference section
TIMER_TO_KERNELS = {"Chain": "backbone", "Chi": "backbone", "Rama": "backbone", "DSSP": "pair (detection) + hbond",
                    "PAP": "pair (detection) + hbond", "Frag_Mem": "fragmem", "Pair_Double_Loop1": "density",
                    "Pair_Single_Loop": "residue (switching, burial, helical pairs)", "Pair_Double_Loop2": "water_xi",
                    "Pair_Double_Loop3": "radial + pair (detection)", "Vexcluded": "pair + residue"}


def read_timer_log(path: str) -> dict:
    out = {}
    try:
        for line in open(path):
            name, _, val = line.partition(" time = ")
            if val:
                out[name.strip()] = float(val)
    except OSError:
        pass
    return out


def _ref_worker(args):
    """Runs in a spawned process: reference MD on a list of c3 replicas.
    Returns residue-steps, the seconds of its timed MD steps, and the sum of
    the replicas' timer.log sections (the reference's own per-term clocks,
    written when the fix is destroyed)."""
    lens_seeds, md, tmp = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    from awsemmd_b200 import synth

    done_res_steps, t_total, timers = 0, 0.0, {}
    for L, seed in lens_seeds:
        c = c3_chain(L, seed)
        files = synth.write_chain_arrays(c, os.path.join(tmp, f"r{seed}"))
        r = ref.RefSystem(files)
        r.run(1, langevin=True, seed=seed)  # warm-up (setup caches)
        t0 = time.perf_counter()
        r.run(md, langevin=True, seed=seed)
        t_total += time.perf_counter() - t0
        done_res_steps += L * md
        r.close()
        for k, v in read_timer_log(os.path.join(files["workdir"], "timer.log")).items():
            timers[k] = timers.get(k, 0.0) + v
    return done_res_steps, t_total, timers


def reference_c3(n_procs: int, md: int, n_replicas: int = 1024, sample: int | None = None):
    """Aggregate residue-steps/s of the reference over `n_procs` host
    processes (one per core).  Every replica of the workload (or a random
    `sample` of them) runs `md` MD steps; replicas are dealt to the processes
    longest first to the least-loaded one, each process times only its MD
    steps, and the slowest process sets the aggregate."""
    lens = c3_lengths(n_replicas)
    ks = list(range(n_replicas))
    if sample is not None:
        ks = [int(k) for k in np.random.default_rng(1).choice(n_replicas, size=sample, replace=False)]
    jobs, load = [[] for _ in range(n_procs)], [0] * n_procs
    for k in sorted(ks, key=lambda k: -lens[k]):
        p = int(np.argmin(load))
        jobs[p].append((lens[k], c3_seed(k)))
        load[p] += lens[k]
    jobs = [j for j in jobs if j]
    with tempfile.TemporaryDirectory() as tmp:
        ctx = mp.get_context("spawn")
        t0 = time.perf_counter()
        with ctx.Pool(len(jobs)) as pool:
            out = pool.map(_ref_worker, [(j, md, tmp) for j in jobs])
        wall = time.perf_counter() - t0
    res_steps = sum(o[0] for o in out)
    busy = max(o[1] for o in out)
    timers = {}
    for o in out:
        for k, v in o[2].items():
            timers[k] = timers.get(k, 0.0) + v
    return res_steps / busy, res_steps, busy, wall, timers, len(ks)


def timer_breakdown(timers: dict) -> dict:
    """The reference's timer.log sections as shares of its timed total, each
    with the GPU kernels that do that work here."""
    total = timers.get("Total", 0.0)
    if total <= 0:
        return {}
    return {k: {"share": round(timers[k] / total, 4), "gpu": TIMER_TO_KERNELS.get(k, "")}
            for k in TIMER_NAMES[:-1] if timers.get(k, 0.0) > 0}


def reference_c1(md: int, warmup: int, steps: int):
    import ref
    from awsemmd_b200 import synth

    with tempfile.TemporaryDirectory() as tmp:
        files = synth.write_system(synth.config_system(1), os.path.join(tmp, "c1"))
        r = ref.RefSystem(files)
        for _ in range(warmup):
            r.run(md, langevin=True, seed=11)
        t = []
        for _ in range(steps):
            t0 = time.perf_counter()
            r.run(md, langevin=True, seed=11)
            t.append(time.perf_counter() - t0)
        r.close()
    return 2000 * md * steps / sum(t), sum(t)


def serving_bench(args, dist: Dist, tmp: str) -> dict:
    """Configuration 4 on one GPU: requests arrive as a Poisson process at
    50/s with chain lengths log-uniform in [30, 1000], each an annealing run
    of --serve-steps steps from 600 K to 300 K, served with continuous
    batching by a handle whose device memory is the --serve-budget-gb budget.
    Latencies are reported over the whole stream and over the requests that
    arrive after its first 10 s (the stream once it is full).  Beside it, the
    plain FP64 form serving the first --serve-plain requests of the same
    stream for real, one at a time in arrival order on their arrival times
    (each request its own handle, created when its turn comes)."""
    from awsemmd_b200 import serve, synth
    from awsemmd_b200.engine import AwsemBatch, AwsemServer

    rng = np.random.default_rng(4000 + dist.rank)
    n = args.serve_requests
    lens = serve.log_uniform_lengths(n, 30, 1000, rng)
    arrivals = serve.poisson_arrivals(n, 50.0, rng)
    seeds = [400000 + 1000 * dist.rank + k for k in range(n)]
    prefetch_chains(zip(lens, seeds))
    chains = [c3_chain(int(L), seeds[k]) for k, L in enumerate(lens)]
    ff = synth.forcefield_dir(os.path.join(tmp, "ff4"))
    plan = serve.plan_capacities(ff, args.serve_budget_gb * 1e9, args.precision, device=dist.local)
    t0 = time.perf_counter()
    with AwsemServer(ff, plan["max_residues"], plan["max_requests"], plan["max_memory_records"],
                     precision=args.precision, device=dist.local) as srv:
        t_create = time.perf_counter() - t0
        # warm-up request (graph capture, first list build), not part of the stream
        w = srv.admit(chains[0], 30, 600.0, 300.0, seed=7)
        while srv.progress(w)[0] < 30:
            srv.advance(31)
        srv.collect(w)
        reqs = [serve.Request(k, float(arrivals[k]), chains[k], args.serve_steps, 600.0, 300.0,
                              seed=4000 + 1000 * dist.rank + k) for k in range(n)]
        done = serve.run_stream(srv, reqs, chunk=100, keep_state=False)
        usage = srv.usage()
    st = serve.stream_stats(done)
    late = [d for d in done if d.arrival >= 10.0]
    steady = serve.stream_stats(late) if len(late) >= 20 else None
    # plain FP64, one request at a time, for real, on the first requests' arrival times
    plain = None
    m = min(args.serve_plain, n)
    if m > 0:
        first = sorted(range(n), key=lambda k: arrivals[k])[:m]
        lat, free, work = [], 0.0, 0.0
        clock0 = time.perf_counter()
        for k in first:
            wait = arrivals[k] - arrivals[first[0]] - (time.perf_counter() - clock0)
            if wait > 0:
                time.sleep(wait)
            with AwsemBatch.from_arrays(ff, [chains[k]], precision="fp64", device=dist.local,
                                        seeds=[4000 + 1000 * dist.rank + k]) as one:
                one.run(args.serve_steps, t_start=600.0, t_stop=300.0)
            lat.append(time.perf_counter() - clock0 - (arrivals[k] - arrivals[first[0]]))
            work += float(lens[k]) * args.serve_steps
        span = time.perf_counter() - clock0
        mine = {d.rid: d.latency for d in done}
        served_same = [mine[k] for k in first]
        plain = {"requests": m, "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                 "residue_steps_per_s": work / span,
                 "served_p50_s_same_requests": float(np.percentile(served_same, 50)),
                 "served_p99_s_same_requests": float(np.percentile(served_same, 99)),
                 "method": f"the stream's first {m} requests run for real, one at a time in arrival order on their "
                           f"arrival times: each a plain FP64 single-system handle created when its turn comes, "
                           f"{args.serve_steps} steps, wall clock"}
    return {"workload": f"config4: {n} requests, Poisson 50/s, lengths log-uniform [30, 1000], "
                        f"{args.serve_steps} Langevin steps each, 600 -> 300 K ramp, dt 2 fs, damping 500 fs, "
                        f"{args.precision} form",
            "p50_s": st["p50_s"], "p99_s": st["p99_s"], "mean_s": st["mean_s"], "makespan_s": st["makespan_s"],
            "residue_steps_per_s": st["residue_steps_per_s"], "residue_steps": st["residue_steps"],
            "after_first_10s": None if steady is None else {
                "requests": steady["requests"], "p50_s": steady["p50_s"], "p99_s": steady["p99_s"],
                "mean_s": steady["mean_s"]},
            "arrivals_span_s": float(arrivals[-1] - arrivals[0]),
            "budget_gb": args.serve_budget_gb, "device_bytes": usage["device_bytes"],
            "residue_capacity": usage["residue_capacity"], "record_capacity": usage["record_capacity"],
            "create_s": t_create, "plain_fp64_one_at_a_time": plain}


TERM_NAMES = ["total", "chain", "shake", "chi", "rama", "excluded", "dssp", "p_ap", "water", "burial", "helix",
              "amh_go", "frag_mem", "vec_fm", "contact_restraints", "membrane", "ssb", "dh", "vexcluded", "bonds"]


def error_vs_oracle(dev: int, tmp: str) -> dict:
    """Both arithmetic forms against the FP64 oracle on eight of the
    workload's replicas (its longest, 500 residues, and seven drawn with a
    fixed seed), run as one batch: per energy term the largest relative error
    over the replicas (relative to max(|term|, 0.01 kcal/mol)), the largest
    force error relative to the replica's largest force, and the selections
    (awsem_debug_selections) of the longest replica against the oracle's."""
    import ref
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch, AwsemSystem

    lens = c3_lengths(1024)
    pick = [int(np.argmax(lens))] + [int(k) for k in np.random.default_rng(31).choice(1024, 7, replace=False)]
    chains = [c3_chain(lens[k], c3_seed(k)) for k in pick]
    ff = synth.forcefield_dir(os.path.join(tmp, "ffe"))
    files = [synth.write_chain_arrays(c, os.path.join(tmp, f"err{r}")) for r, c in enumerate(chains)]
    oracle = []
    for r, c in enumerate(chains):
        o = ref.OracleSystem(files[r])
        x = c["x"].reshape(-1, 3)
        oracle.append((x,) + o.compute(x))
        o.close()
    out = {"sample": f"replicas {pick} of the workload ({sum(lens[k] for k in pick)} residues), step 0"}
    for prec in ("fp64", "mixed"):
        with AwsemBatch.from_arrays(ff, chains, precision=prec, device=dev, seeds=[c3_seed(k) for k in pick]) as b:
            b.run(0, langevin=False)
            terms = np.zeros(20)
            ferr = 0.0
            for r in range(len(chains)):
                x, fo, eo = oracle[r]
                f, e = b.forces(r), b.energies(r)
                terms = np.maximum(terms, np.abs(e[:20] - eo[:20]) / np.maximum(np.abs(eo[:20]), 1e-2))
                ferr = max(ferr, float(np.abs(f - fo).max() / np.abs(fo).max()))
        out[prec] = {"energy_rel": {TERM_NAMES[k]: float(terms[k]) for k in range(20)}, "force_rel": ferr}
    o = ref.OracleSystem(files[0])
    x = oracle[0][0]
    want, near = o.selections(x), o.selections(x, "near")
    o.close()
    sel = {}
    for prec in ("fp64", "mixed"):
        with AwsemSystem(files[0], precision=prec, device=dev) as s:
            cmp = ref.compare_selections(s.selections(x), want, near)
        sel[prec] = {k: v for k, v in cmp.items() if v["want"] or v["got"]}
    out["selections_longest_replica"] = {
        "fp64_identical": all(v["cand"] == 0 and v["gate"] == 0 for v in sel["fp64"].values()),
        "mixed": sel["mixed"], "near_threshold_in_oracle": int(len(near)),
        "note": "cand: items one side selects and the other does not (gated kinds without their gate bits); "
                "cand_far: of those, not within 2e-6 of a threshold; gate: items both select with other gate bits"}
    return out


def config1_extra(dev: int, tmp: str, run_kw: dict, l2buf) -> dict:
    """Configuration 1 (8 x 250 residues): the plain FP64 form (and the mixed
    form) on the GPU against the reference on one host core."""
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemSystem

    files = synth.write_system(synth.config_system(1), os.path.join(tmp, "c1x"))
    out = {"workload": WORKLOADS["c1"]}
    for prec in ("fp64", "mixed"):
        with AwsemSystem(files, precision=prec, device=dev) as s:
            s.run(100, **run_kw)
            ms = []
            for _ in range(3):
                flush_l2(l2buf)
                s.run(100, **run_kw)
                ms.append(s.last_run_ms())
        t = sum(ms) / 1e3
        out[prec] = {"steps_per_s": 300 / t, "residue_steps_per_s": 2000 * 300 / t}
    v, busy = reference_c1(5, 1, 2)
    out["reference_1_core"] = {"residue_steps_per_s": v, "sample": f"2 x 5 MD steps ({busy:.1f} s), 1 rank"}
    out["fp64_over_reference"] = out["fp64"]["residue_steps_per_s"] / v
    return out


def config2_extra(dev: int, tmp: str, run_kw: dict, l2buf, peak: float) -> dict:
    """Configuration 2 (40,000 residues, one system, mixed form): steps/s,
    residue-steps/s and per-kernel achieved HBM GB/s against the peak."""
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch

    ff = synth.forcefield_dir(os.path.join(tmp, "ff2x"))
    c2 = synth.packed_arrays([250] * 160, 320.0, 2000)
    kw = dict(run_kw, skin=2.0, neigh_every=10)
    with AwsemBatch.from_arrays(ff, [c2], precision="mixed", device=dev, seeds=[2000]) as s:
        shapes = s.autotune(2)
        s.run(50, **kw)
        ms = []
        for _ in range(3):
            flush_l2(l2buf)
            s.run(50, **kw)
            ms.append(s.last_run_ms())
        prof = s.profile_step(10)
        info = s.model_info()
    t = sum(ms) / 1e3
    per_kernel = {}
    for k in ("fragmem", "radial", "pair", "density", "water_xi", "prepare", "finish"):
        if prof.get(k, 0) > 0:
            b = algorithmic_bytes(k, info)
            per_kernel[k] = {"ms": round(prof[k], 5), "achieved_gbs": round(b / (prof[k] * 1e-3) / 1e9, 1),
                             "frac": round(b / (prof[k] * 1e-3) / 1e9 / peak, 4)}
    return {"workload": WORKLOADS["c2"], "steps_per_s": 150 / t, "residue_steps_per_s": 40000 * 150 / t,
            "kernel_ms": {k: round(v, 5) for k, v in prof.items()}, "per_kernel": per_kernel,
            "launch_shapes": shapes, "peak_gbs": peak}


def reference_arm(args, dist: Dist):
    if dist.rank != 0:
        return
    import ref

    if not ref.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library not built (make -C oracle ref)"}))
        return
    cores = os.cpu_count() or 1
    if args.workload == "c2":
        print(json.dumps({"impl": "reference", "unavailable": "configuration 2 does not fit a host: " + C2_CPU_NOTE}))
        return
    timers = None
    if args.workload == "c3":
        md = args.md_steps
        # the whole workload: every replica for the repo arm's MD steps per bench step
        value, res_steps, busy, wall, tm, nrep = reference_c3(cores, md, args.replicas)
        timers = timer_breakdown(tm)
        ms = 1e3 * busy
        steps = 1
        sample = (f"the whole workload once: all {nrep} replicas x {md} MD steps ({res_steps} residue-steps, one "
                  f"bench step of the repo arm; +1 untimed warm-up step each), dealt longest first over {cores} "
                  f"processes (one per host core); reference FixBackbone + PairExcludedVolume compiled -O2 "
                  f"against the LAMMPS-API shim, 1 rank per process; slowest process's MD time {busy:.1f} s, "
                  f"wall {wall:.1f} s")
    else:
        md = 5
        value, busy = reference_c1(md, args.warmup, args.steps)
        cores = 1
        ms = 1e3 * busy / args.steps
        steps = args.steps
        sample = f"{md} MD steps per bench step of the 2,000-residue system, 1 core, 1 rank"
    line = {"metric": "residue-steps/s", "value": value, "unit": "residue-steps/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_text(args), "md_steps_per_step": md,
                       "parallelism": f"{cores} host processes x 1 MPI rank (serial reference; no MPI in the image)"},
            "cpu_baseline": {"value": value, "unit": "residue-steps/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "residue-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if timers:
        line["reference_timer_log"] = timers
    print(json.dumps(line))


# --------------------------------------------------------------------------

def build_c3(n: int, rank: int, precision: str, dev: int, tmp: str):
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch

    lens = c3_lengths(n)
    prefetch_chains((L, c3_seed(k, rank)) for k, L in enumerate(lens))
    chains = (c3_chain(L, c3_seed(k, rank)) for k, L in enumerate(lens))
    ff = synth.forcefield_dir(os.path.join(tmp, "ff"))
    seeds = [c3_seed(k, rank) for k in range(n)]
    return AwsemBatch.from_arrays(ff, chains, precision=precision, device=dev, seeds=seeds), sum(lens), ff, lens


def free_port() -> int:
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def launch_command(argv, n: int, port: int):
    """The command that runs this benchmark as n ranks, one process per GPU,
    when it was started plainly with --gpus n (no torchrun around it)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
            "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)


def main():
    args = parse()
    if args.impl == "ours" and args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(subprocess.call(launch_command(sys.argv[1:], args.gpus, free_port())))
    dist = Dist()
    if args.impl == "reference":
        reference_arm(args, dist)
        dist.close()
        return
    if dist.world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but {dist.world} ranks are running")
    import torch

    from awsemmd_b200 import build
    from awsemmd_b200.engine import AwsemBatch, AwsemSystem

    if dist.rank == 0:
        build.build()
    dist.barrier()
    dev = dist.local
    torch.cuda.set_device(dev)
    l2buf = torch.empty(128 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")  # 512 MiB > 126 MB L2
    tmp = tempfile.mkdtemp()
    md = args.md_steps
    run_kw = dict(dt=RUN["dt"], langevin=True, t_start=RUN["t_start"], t_stop=RUN["t_stop"], damp=RUN["damp"],
                  seed=1000 + dist.rank)
    t_setup = time.perf_counter()
    if args.workload == "c3":
        eng, n_res, ff, lens = build_c3(args.replicas, dist.rank, args.precision, dev, tmp)
    elif args.workload == "c2":
        from awsemmd_b200 import synth

        ff = synth.forcefield_dir(os.path.join(tmp, "ff2"))
        c2 = synth.packed_arrays([250] * 160, 320.0, 2000 + dist.rank)
        eng = AwsemBatch.from_arrays(ff, [c2], precision=args.precision, device=dev, seeds=[2000 + dist.rank])
        n_res = eng.nres
        run_kw.update(skin=2.0, neigh_every=10)
    else:
        from awsemmd_b200 import synth

        files = synth.write_system(synth.config_system(1, replica=dist.rank), os.path.join(tmp, "c1"))
        eng = AwsemSystem(files, precision=args.precision, device=dev)
        n_res = eng.nres
    t_setup = time.perf_counter() - t_setup
    if args.shapes:
        eng.set_launch_shapes([int(t) for t in args.shapes.split(",")])
        shapes = {**dict(zip(eng.SHAPE_KEYS, [int(t) for t in args.shapes.split(",")])), **eng.step_form(),
                  "source": "--shapes"}
    else:
        shapes = eng.autotune(3)  # launch shapes measured on this workload (results do not depend on them)
    for _ in range(args.warmup):
        eng.run(md, **run_kw)
    clocks = ClockSampler(dev)
    clocks.start()
    dev_ms = []
    for _ in range(args.steps):
        flush_l2(l2buf)
        dist.barrier()
        torch.cuda.synchronize()
        eng.run(md, **run_kw)
        torch.cuda.synchronize()
        dev_ms.append(eng.last_run_ms())
        dist.barrier()
    clk = clocks.stop()
    total_ms = dist.max(sum(dev_ms))
    value = dist.world * n_res * md * args.steps / (total_ms / 1e3)

    # end to end through the C ABI with host buffers: every replica's state
    # in from pinned host memory (awsem_batch_set_state), `run`, every
    # replica's state out (awsem_batch_get_state)
    nrep = getattr(eng, "nreplicas", 1)
    pinned = [torch.empty((eng.natoms, 3), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    hx, hv = pinned[0].numpy(), pinned[1].numpy()
    if nrep > 1:
        eng.get_state_all(hx, hv)
    else:
        hx[:], hv[:] = eng.get_state()
    e2e_t = []
    for _ in range(max(2, args.steps // 2)):
        dist.barrier()
        t0 = time.perf_counter()
        if nrep > 1:
            eng.set_state_all(hx, hv)
            eng.run(md, **run_kw)
            eng.get_state_all(hx, hv)
        else:
            eng.set_state(hx, hv)
            eng.run(md, **run_kw)
            x1, v1 = eng.get_state()
            hx[:], hv[:] = x1, v1
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = dist.max(sum(e2e_t))
    e2e_value = dist.world * n_res * md * len(e2e_t) / e2e_total
    natoms = eng.natoms

    # roofline of the dominant kernel from per-kernel CUDA-event times
    eng.run(2, **run_kw)
    prof = eng.profile_step(20)
    info = eng.model_info()
    names = list(prof)
    top = max(names, key=lambda k: prof[k])
    peak, peak_kind = peaks()
    abytes = algorithmic_bytes(top, info)
    achieved = abytes / (prof[top] * 1e-3) / 1e9
    fm_gbs = algorithmic_bytes("fragmem", info) / (prof["fragmem"] * 1e-3) / 1e9 if prof["fragmem"] > 0 else None
    traffic = TRAFFIC_PER_ALGORITHMIC_BYTE[top] * abytes if top in TRAFFIC_PER_ALGORITHMIC_BYTE else None
    # per kernel: algorithmic bytes / CUDA-event time against the same peak
    per_kernel = {}
    for k in ("fragmem", "radial", "pair", "density", "water_xi", "prepare", "finish"):
        if prof.get(k, 0) > 0:
            b = algorithmic_bytes(k, info)
            per_kernel[k] = {"ms": round(prof[k], 5), "algorithmic_bytes": b,
                             "achieved_gbs": round(b / (prof[k] * 1e-3) / 1e9, 1),
                             "frac": round(b / (prof[k] * 1e-3) / 1e9 / peak, 4)}
    roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "traffic_source": TRAFFIC_SOURCE if traffic else None,
                "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                "algorithmic_bytes_per_launch": abytes, "launch_ms": prof[top],
                "kernel_ms": {k: round(v, 5) for k, v in prof.items()}, "fragmem_gbs": fm_gbs,
                "per_kernel": per_kernel,
                "model_info": {"residues": int(info[0]), "records": int(info[2]), "pairs": int(info[6])}}

    # the plain single-instance FP64 form (one replica at a time)
    plain = None
    if args.workload == "c3":
        sample = np.random.default_rng(7).choice(args.replicas, size=min(24, args.replicas), replace=False)
        res_steps, ms_sum = 0, 0.0
        for k in sample:
            c = c3_chain(lens[k], c3_seed(k, dist.rank))
            with AwsemBatch.from_arrays(ff, [c], precision="fp64", device=dev, seeds=[c3_seed(k, dist.rank)]) as one:
                one.run(md, **run_kw)
                flush_l2(l2buf)
                one.run(md, **run_kw)
                ms_sum += one.last_run_ms()
                res_steps += lens[k] * md
        pv = res_steps / (ms_sum / 1e3)
        plain = {"value": pv, "unit": "residue-steps/s", "speedup_of_headline": value / pv / dist.world,
                 "sample": f"{len(sample)} of the replicas run one at a time, plain FP64 single-system form, "
                           f"{md} MD steps each after a warm-up run, device time"}
    elif args.precision != "fp64":
        with (AwsemBatch.from_arrays(ff, [c2], precision="fp64", device=dev, seeds=[2000 + dist.rank])
              if args.workload == "c2" else AwsemSystem(files, precision="fp64", device=dev)) as sp:
            sp.run(md, **run_kw)
            pm = []
            for _ in range(max(2, args.steps // 2)):
                flush_l2(l2buf)
                sp.run(md, **run_kw)
                pm.append(sp.last_run_ms())
            plain = {"value": n_res * md * len(pm) / (sum(pm) / 1e3), "unit": "residue-steps/s"}

    base = None
    if dist.rank == 0 and dist.world == 1 and not args.no_baseline:
        try:
            if args.workload == "c3":
                v, rs, busy, wall, tm, nsamp = reference_c3(1, md, args.replicas, sample=16)
                base = {"value": v, "unit": "residue-steps/s", "cores": 1, "kind": "reference",
                        "sample": f"{nsamp} random replicas x {md} MD steps ({rs} residue-steps, {busy:.1f} s) on 1 "
                                  f"host core; reference FixBackbone + PairExcludedVolume compiled -O2 against the "
                                  f"LAMMPS-API shim, 1 MPI rank",
                        "reference_timer_log": timer_breakdown(tm)}
            elif args.workload == "c2":
                base = {"value": None, "unit": "residue-steps/s", "cores": 1, "kind": "reference",
                        "sample": "not runnable: " + C2_CPU_NOTE}
            else:
                v, busy = reference_c1(5, 1, 2)
                base = {"value": v, "unit": "residue-steps/s", "cores": 1, "kind": "reference",
                        "sample": f"2 x 5 MD steps of the 2,000-residue system ({busy:.1f} s), 1 core, 1 rank"}
        except Exception as e:  # reported, never replaced by something else
            base = {"value": None, "unit": "residue-steps/s", "cores": 1, "kind": "reference",
                    "sample": f"not measured: {e}"}
    eng.close()
    extras = {}
    if args.workload == "c3" and dist.world == 1 and not args.no_extras:
        for key, fn in (("error_vs_oracle", lambda: error_vs_oracle(dev, tmp)),
                        ("config1", lambda: config1_extra(dev, tmp, run_kw, l2buf)),
                        ("config2", lambda: config2_extra(dev, tmp, run_kw, l2buf, peak))):
            try:
                extras[key] = fn()
            except Exception as e:  # reported, never replaced by something else
                extras[key] = {"not_measured": f"{type(e).__name__}: {e}"}
    served = None
    if args.workload == "c3" and args.serve_requests > 0 and dist.world == 1:
        del l2buf
        torch.cuda.empty_cache()  # the serving handle takes the memory budget
        served = serving_bench(args, dist, tmp)
    from awsemmd_b200.engine import NKERNELS
    launches = NKERNELS * (md + 1) * args.steps  # every kernel of every MD step (setup evaluation included)
    if dist.rank == 0:
        line = {"metric": "residue-steps/s", "value": value, "unit": "residue-steps/s", "n_gpus": dist.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32/f64" if args.precision == "mixed" else "f64", "data": "synthetic",
                "config": {"workload": workload_text(args), "form": args.precision, "md_steps_per_step": md,
                           "residues": n_res, "replicas": nrep, "global_batch": dist.world * nrep,
                           "parallelism": f"replicas x{dist.world} GPUs (independent copies per GPU)",
                           "l2": "flushed (512 MiB write) before every timed bench step",
                           "setup_s": round(t_setup, 1), "launch_shapes": shapes},
                "roofline": roofline, "cpu_baseline": base,
                "e2e": {"value": e2e_value, "unit": "residue-steps/s",
                        "h2d_bytes_per_step": 2 * natoms * 3 * 8, "d2h_bytes_per_step": 2 * natoms * 3 * 8,
                        "path": "awsem_batch_set_state (pinned host x, v of every replica) + awsem_run + "
                                "awsem_batch_get_state, per bench step; wall clock"},
                "plain_fp64": plain, "clocks": clk, "gpu_launches": launches, "served": served, **extras}
        print(json.dumps(line))
    dist.close()


if __name__ == "__main__":
    main()
