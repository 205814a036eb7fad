#!/usr/bin/env python
"""AWSEM-MD step benchmark: residue-steps/s on B200.

One bench step = `--md-steps` velocity-Verlet + Langevin MD steps (300 K,
dt 2 fs, damping 500 fs) of the workload with every force term on the GPU.
Workload (default): benchmark configuration 1, a single system of 8 chains
x 250 residues (2,000 residues, 6,000 beads) in a 150 A cube with all
AWSEM terms and fragment memory on, run in the mixed form.

Timing: W untimed warm-up bench steps, then K timed ones, each bracketed by
a barrier and a device synchronize, device time from CUDA events on the
engine's stream; L2 is flushed (a 512 MiB write) before every timed bench
step.  With N GPUs (torchrun) every rank runs its own replica (replicas
only: the path has no cross-GPU exchange) and the slowest rank's time sets
the aggregate.

`--impl reference` times the reference implementation (FixBackbone +
PairExcludedVolume compiled unmodified against the LAMMPS-API shim, serial,
one core) on the same workload and metric.
"""
from __future__ import annotations

import argparse
import ctypes as C
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
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0

RUN = dict(dt=2.0, t_start=300.0, t_stop=300.0, damp=500.0)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--md-steps", type=int, default=100)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline sample")
    return ap.parse_args()


# --------------------------------------------------------------------------
# distributed plumbing (one process per GPU, replicas only)

class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", self.local))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# --------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
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
    buf.fill_(1.0)
    import torch

    torch.cuda.synchronize()


def peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM, "fallback"


def make_workload(tmp: str, replica: int):
    from awsemmd_b200 import synth

    s = synth.config_system(1, replica=replica)
    files = synth.write_system(s, os.path.join(tmp, f"c1_r{replica}"))
    return files, s.n_res


# algorithmic bytes per launch of each kernel (see the engine's data layout):
#   fragmem: every stored memory distance once, the row table, the two target
#            beads per row and the force accumulators of i and j
#   pair / density / water_xi: the residue pair list once, every residue's
#            working coordinates and per-residue scalars once
def algorithmic_bytes(kernel: str, info) -> float:
    n_res, n_atoms, records, rbytes, nd, cap, entries, nonuni = [int(v) for v in info]
    bead = 32  # double4 working coordinates
    if kernel == "fragmem":
        return records * 4 * rbytes + records * rbytes * nonuni + (n_res * nd + 1) * 4 + n_res * 2 * bead \
            + n_res * 2 * 3 * 8 * 2
    if kernel in ("pair", "density", "water_xi"):
        return entries * 4 + n_res * 6 * bead + n_res * 10 * 8 + n_res * 4 * 4 + n_atoms * 3 * 8
    if kernel == "prepare":
        return n_atoms * 3 * 8 + n_res * 6 * bead + n_atoms * 3 * 8 + n_res * 32
    if kernel == "finish":
        return n_atoms * 3 * 8 * 5 + n_res * 8
    return n_res * 6 * bead


def cpu_baseline(files, n_res, seconds_target=12.0):
    """The reference (shim-hosted, one core) on a bounded sample of the
    workload; falls back to the FP64 restatement when the reference library
    was not built."""
    import ref

    if ref.ref_available():
        r = ref.RefSystem(files)
        r.run(2, langevin=True, seed=7)  # warm-up (includes the O(n^2) cache reset at setup)
        steps, t = 5, 0.0
        while True:
            t0 = time.perf_counter()
            r.run(steps, langevin=True, seed=7)
            t = time.perf_counter() - t0
            if t * 4 > seconds_target or steps >= 400:
                break
            steps *= 2
        r.close()
        return {"value": n_res * steps / t, "unit": "residue-steps/s", "cores": 1, "kind": "reference",
                "sample": f"{steps} MD steps (one `run`, incl. its setup evaluation) of the same 2,000-residue "
                          f"system, reference FixBackbone+PairExcludedVolume compiled -O2 against the LAMMPS-API "
                          f"shim, 1 MPI rank, {t:.1f} s"}
    # the FP64 restatement (all-pairs loops) as the port baseline
    o = ref.OracleSystem(files)
    from awsemmd_b200.engine import AwsemSystem  # noqa: F401  (state comes from the data file)
    x0 = np.zeros((o.natoms, 3))
    v0 = np.zeros((o.natoms, 3))
    with open(os.path.join(files["workdir"], files["data"])) as fh:
        lines = fh.read().split("\n")
    at = lines.index("Atoms") + 2
    for k in range(o.natoms):
        w = lines[at + k].split()
        x0[int(w[0]) - 1] = [float(w[5]), float(w[6]), float(w[7])]
    steps = 2
    t0 = time.perf_counter()
    o.run(x0, v0, steps, langevin=True, seed=7)
    t = time.perf_counter() - t0
    return {"value": n_res * steps / t, "unit": "residue-steps/s", "cores": 1, "kind": "port",
            "sample": f"{steps} MD steps of the FP64 restatement (all-pairs loops), {t:.1f} s"}


def reference_arm(args, dist: Dist):
    """--impl reference: the reference CPU implementation, same workload/metric."""
    if dist.rank != 0:
        return
    import ref

    with tempfile.TemporaryDirectory() as tmp:
        files, n_res = make_workload(tmp, 0)
        if not ref.ref_available():
            print(json.dumps({"impl": "reference", "unavailable": "reference library not built (make -C oracle ref)"}))
            return
        r = ref.RefSystem(files)
        md = 5  # MD steps per bench step (a bounded sample of the workload)
        for _ in range(args.warmup):
            r.run(md, langevin=True, seed=11)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            r.run(md, langevin=True, seed=11)
            times.append(time.perf_counter() - t0)
        r.close()
    total = sum(times)
    value = n_res * md * args.steps / total
    line = {"metric": "residue-steps/s", "value": value, "unit": "residue-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": "config1: 8 chains x 250 residues, 2,000 residues, 150 A cube, all terms + "
                                   "fragment memory, Langevin 300 K dt 2 fs", "md_steps_per_step": md,
                       "parallelism": "1 MPI rank (serial reference; no MPI in the image)"},
            "cpu_baseline": {"value": value, "unit": "residue-steps/s", "cores": 1, "kind": "reference",
                             "sample": f"{md} MD steps per bench step, reference FixBackbone+PairExcludedVolume "
                                       f"compiled -O2 against the LAMMPS-API shim"},
            "e2e": {"value": value, "unit": "residue-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    dist = Dist()
    if args.impl == "reference":
        reference_arm(args, dist)
        dist.close()
        return
    import torch

    from awsemmd_b200 import build
    from awsemmd_b200.engine import AwsemSystem, load_library

    if dist.rank == 0 or not os.path.exists(os.path.join(ROOT, "awsemmd_b200", "libawsem_gpu.so")):
        build.build()
    dist.barrier()
    lib = load_library()
    dev = dist.local
    torch.cuda.set_device(dev)
    l2buf = torch.empty(128 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")  # 512 MiB > 126 MB L2
    tmp = tempfile.mkdtemp()
    files, n_res = make_workload(tmp, dist.rank)
    sysm = AwsemSystem(files, precision=args.precision, device=dev)
    x0, v0 = sysm.get_state()
    md = args.md_steps
    run_kw = dict(dt=RUN["dt"], langevin=True, t_start=RUN["t_start"], t_stop=RUN["t_stop"], damp=RUN["damp"],
                  seed=1000 + dist.rank)
    for _ in range(args.warmup):
        sysm.run(md, **run_kw)
    clocks = ClockSampler(dev)
    clocks.start()
    dev_ms = []
    for _ in range(args.steps):
        flush_l2(l2buf)
        dist.barrier()
        torch.cuda.synchronize()
        sysm.run(md, **run_kw)
        torch.cuda.synchronize()
        dev_ms.append(lib.awsem_last_run_ms(sysm.h))
        dist.barrier()
    clk = clocks.stop()
    total_ms = dist.max(sum(dev_ms))
    value = dist.world * n_res * md * args.steps / (total_ms / 1e3)

    # end to end through the public API with host buffers: host state in,
    # `run`, host state out
    sysm.set_state(x0, v0)
    e2e_t = []
    for _ in range(max(2, args.steps // 2)):
        dist.barrier()
        t0 = time.perf_counter()
        sysm.set_state(x0, v0)
        sysm.run(md, **run_kw)
        xh, vh = sysm.get_state()
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = dist.max(sum(e2e_t))
    e2e_value = dist.world * n_res * md * len(e2e_t) / e2e_total
    natoms = sysm.natoms

    # roofline of the dominant kernel: per-kernel CUDA-event times of the step
    lib.awsem_kernel_name.restype = C.c_char_p
    names = [lib.awsem_kernel_name(k).decode() for k in range(10)]
    ms = np.zeros(10)
    sysm.run(5, **run_kw)
    rc = lib.awsem_profile_step(sysm.h, 50, ms.ctypes.data_as(C.c_void_p))
    info = np.zeros(8, dtype=np.int64)
    lib.awsem_model_info(sysm.h, info.ctypes.data_as(C.c_void_p))
    top = int(np.argmax(ms))
    peak, peak_kind = peaks()
    abytes = algorithmic_bytes(names[top], info)
    achieved = abytes / (ms[top] * 1e-3) / 1e9
    fm_k = names.index("fragmem")
    fm_bytes = algorithmic_bytes("fragmem", info)
    roofline = {"bound": "hbm", "kernel": names[top], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "peak_source": f"{peak_kind} hbm_gbs",
                "algorithmic_bytes": abytes, "launch_ms": float(ms[top]),
                "kernel_ms": {names[k]: round(float(ms[k]), 5) for k in range(10)},
                "fragmem_gbs": fm_bytes / (ms[fm_k] * 1e-3) / 1e9 if ms[fm_k] > 0 else None}

    # the plain FP64 form on the same workload (the comparison point)
    plain = None
    if args.precision != "fp64":
        with AwsemSystem(files, precision="fp64", device=dev) as sp:
            sp.run(md, **run_kw)
            pm = []
            for _ in range(max(2, args.steps // 2)):
                flush_l2(l2buf)
                sp.run(md, **run_kw)
                pm.append(lib.awsem_last_run_ms(sp.h))
            pms = dist.max(sum(pm))
            plain = {"value": dist.world * n_res * md * len(pm) / (pms / 1e3), "unit": "residue-steps/s"}

    base = None
    if dist.rank == 0 and dist.world == 1 and not args.no_baseline:
        try:
            base = cpu_baseline(files, n_res)
        except Exception as e:  # reported, never silently replaced
            base = {"value": None, "unit": "residue-steps/s", "cores": 1, "kind": "reference",
                    "sample": f"not measured: {e}"}
    sysm.close()
    launches = 10 * (md + 1) * args.steps
    if dist.rank == 0:
        line = {"metric": "residue-steps/s", "value": value, "unit": "residue-steps/s", "n_gpus": dist.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32/f64" if args.precision == "mixed" else "f64", "data": "synthetic",
                "config": {"workload": "config1: 8 chains x 250 residues (2,000 residues, 6,000 beads), 150 A cube, "
                                       "all AWSEM terms + fragment memory (20 memories per 9-residue window), "
                                       "pair vexcluded, harmonic bonds, Langevin 300 K, dt 2 fs, damping 500 fs",
                           "form": args.precision, "md_steps_per_step": md, "global_batch": dist.world,
                           "parallelism": f"replicas x{dist.world} (one independent system per GPU)",
                           "l2": "flushed (512 MiB write) before every timed bench step; fragment-memory tables "
                                 "stay L2-resident across the MD steps inside one bench step"},
                "roofline": roofline, "cpu_baseline": base,
                "e2e": {"value": e2e_value, "unit": "residue-steps/s",
                        "h2d_bytes_per_step": 2 * natoms * 3 * 8, "d2h_bytes_per_step": 2 * natoms * 3 * 8,
                        "path": "awsem_set_state(host x, v) + awsem_run + awsem_get_state per bench step"},
                "plain_fp64": plain, "clocks": clk, "gpu_launches": launches}
        print(json.dumps(line))
    dist.close()


if __name__ == "__main__":
    main()
