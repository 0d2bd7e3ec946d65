#!/usr/bin/env python
"""Benchmark of the Heisenberg Metropolis / parallel-tempering hot path on B200.

One step = one parallel-tempering round of the workload: `sweeps_per_swap` colour-class
sweeps of every replica followed by one replica exchange, replayed from a CUDA graph.
metric: spin-updates/s = attempted single-site updates (N per replica per sweep) / s.

Default workload (N=1): simple cubic L=128, 16 replicas, T geometric 0.1-1.5, J=1
(ferromagnetic, passed as J=-1 in the reference sign convention), bulk DMI D=0.7,
B=0.3 along z, K=0.05 along z, ball move r=0.2, swaps every 10 sweeps.  Spin state is
384 MiB (> 126 MB L2), so no L2 flush is needed between steps.

Under torchrun each rank runs its own copy of the workload on its GPU (independent
ensembles, weak scaling, no collective on the data path); the timed region is bracketed
by barriers and the max over ranks is reported.

--impl reference times the reference algorithm on the host cores instead: the CPU
restatement of Metropolis_mcs (src/energyMin.f90:234-374) with all host threads.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: lattice L, replicas, T range, J, D, B, K, move, r, sweeps per swap
    "c3": dict(L=128, R=16, tmin=0.1, tmax=1.5, J=-1.0, D=0.7, B=0.3, K=0.05, move="ball", r=0.2, k=10,
               desc="SC L=128 x 16 PT replicas, T 0.1-1.5, J=1, bulk D=0.7, B=0.3 z, K=0.05 z"),
    "c2": dict(L=32, R=32, tmin=0.2, tmax=2.0, J=-1.0, D=0.5, B=0.2, K=0.0, move="ball", r=0.2, k=10,
               desc="SC L=32 x 32 PT replicas, T 0.2-2.0, J=1, bulk D=0.5, B=0.2 z"),
    "c5": dict(L=96, R=48, tmin=0.1, tmax=1.5, J=-1.0, D=0.5, B=0.25, K=0.0, move="ball", r=0.2, k=10,
               desc="SC L=96 x 48 PT replicas, T 0.1-1.5, J=1, bulk D=0.5, B=0.25 z"),
}
BYTES_PER_UPDATE = 24  # algorithmic: one FP32 x,y,z read and write per site per sweep


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus=None):
        self.bus = bus if isinstance(bus, int) else None  # PCI bus number of the timed GPU
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                bus = int(parts[0].split(":")[1], 16)
            except (IndexError, ValueError):
                bus = None
            if self.bus is not None and bus is not None and bus != self.bus:
                continue
            rows.append(parts)
        if not rows:
            return out
        try:
            sm = [float(r[1]) for r in rows]
            mx = max(float(r[2]) for r in rows)
        except ValueError:
            return out
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() in ("active", "1")})
        out.update(sm_mhz=statistics.median(sm), sm_max_mhz=mx, reasons=reasons, samples=len(rows))
        return out


# ---------------------------------------------------------------- reference (CPU) arm
def cpu_reference_rate(w, steps, warmup, threads, L_sample=None):
    """Throughput of the CPU restatement of Metropolis_mcs on the host cores: one sweep of
    one replica per step (numAtoms trials), the reference's parallel structure (OpenMP over
    trials, snapshot semantics), same Hamiltonian.  Returns (updates/s, sample text)."""
    from oracle import oracle as O
    O.build()
    L = L_sample or w["L"]
    m = O.Mesh.sc(L)
    m.init_uniform(0x15196)
    p = O.Params(J=w["J"], Dz=w["D"], B=w["B"], K=w["K"], dmi_bulk=True)
    beta = 1.0 / w["tmin"]
    for _ in range(warmup):
        m.metropolis_mcs_omp(beta, 1, p, w["r"], n_threads=threads, time_seed=1)
    t0 = time.perf_counter()
    for _ in range(steps):
        m.metropolis_mcs_omp(beta, 1, p, w["r"], n_threads=threads, time_seed=1)
    dt = time.perf_counter() - t0
    rate = steps * m.natoms / dt
    return rate, f"{steps} sweep(s) of one SC L={L} replica ({m.natoms} trials each), {threads} threads"


def run_reference(args, w):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = host_cores()
    rate, sample = cpu_reference_rate(w, max(args.steps, 1), max(args.warmup, 0), threads)
    line = {
        "metric": "spin-updates/s", "value": rate, "unit": "spin-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * (w["L"] ** 3) / rate, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "sample": "one replica per step"},
        "cpu_baseline": {"value": rate, "unit": "spin-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": "spin-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def run_gpu(args, w):
    import numpy as np
    import torch
    import torch.distributed as dist

    import ising_b200 as ib
    from ising_b200 import _lib

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    L, R = args.L or w["L"], args.replicas or w["R"]
    k = w["k"]
    N = L ** 3
    mesh = ib.ChainMesh.simple_cubic(L, n_replicas=R, device=dev)
    mesh.set_stream(stream.cuda_stream)
    mesh.init_uniform(0x15196, ensemble=rank)
    p = ib.params(J=w["J"], Dz=w["D"], B=w["B"], K=w["K"], dmi="bulk")
    T = ib.temperature_ladder(w["tmin"], w["tmax"], R)
    betas = 1.0 / T
    move = _lib.MOVE_BALL if w["move"] == "ball" else _lib.MOVE_UNIFORM
    pt = ib.ParallelTempering(mesh, betas, p, seed=0x15196, ensemble=rank, move=move, r=w["r"])

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # warm-up (also builds the CUDA graph)
    pt.run(k, max(args.warmup, 1) if args.warmup > 0 else 1)
    barrier()

    clocks = ClockSampler(getattr(torch.cuda.get_device_properties(dev), "pci_bus_id", None))
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    pt.run(k, args.steps)
    ev1.record(stream)
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    clk = clocks.stop()
    updates_per_step = R * N * k
    value = world * updates_per_step * args.steps / (ms / 1e3)

    # dominant kernel: the colour-pass kernel, timed alone on the same stream over n_relax
    # sweeps (the relax call issues only colour-pass launches plus one fold and one advance)
    group, per_round, kern_id = pt.schedule(k)
    n_relax = max(4, min(40, args.steps * k // 2))
    launches = pt.schedule(n_relax)[1]
    pt.relax(2)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pt.relax(n_relax)
    e1.record(stream)
    barrier()
    sweep_ms = e0.elapsed_time(e1) / n_relax
    launch_ms = e0.elapsed_time(e1) / launches
    bytes_per_launch = BYTES_PER_UPDATE * R * N * n_relax / launches
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    achieved = bytes_per_launch / (launch_ms / 1e3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    if os.path.exists(tfile):
        try:
            t = json.load(open(tfile))
            if t.get("workload") == args.workload and t.get("bytes_per_update"):
                traffic = t["bytes_per_update"] * R * N / 2
        except Exception:
            traffic = None

    # end to end through the C-ABI with host-owned FP64 spins (the reference's atomSpins):
    # every step uploads all replicas from pinned host memory, runs the round, downloads
    # all replicas and the per-replica energies.
    e2e = None
    if not args.no_e2e:
        L_ = _lib.load()
        host = [torch.empty(3 * N, dtype=torch.float64, pin_memory=True) for _ in range(R)]
        for r in range(R):
            _lib.check(L_.ising_spins_get(mesh.handle, r, C.cast(host[r].data_ptr(), C.POINTER(C.c_double))), "get")
        e_host = np.empty(R)
        m_host = np.empty((R, 3))
        e2e_steps = max(1, min(args.steps, 5))

        def e2e_step():
            for r in range(R):
                _lib.check(L_.ising_spins_set(mesh.handle, r, C.cast(host[r].data_ptr(), C.POINTER(C.c_double))), "set")
            pt.run(k, 1)
            for r in range(R):
                _lib.check(L_.ising_spins_get(mesh.handle, r, C.cast(host[r].data_ptr(), C.POINTER(C.c_double))), "get")
            e_, m_ = pt.energies()
            e_host[:] = e_
            m_host[:] = m_

        e2e_step()
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        a1.record(stream)
        barrier()
        wall = time.perf_counter() - t0
        e_ms = max_over_ranks(max(a0.elapsed_time(a1), wall * 1e3))
        e2e = {"value": world * updates_per_step * e2e_steps / (e_ms / 1e3), "unit": "spin-updates/s",
               "h2d_bytes_per_step": R * 3 * N * 8, "d2h_bytes_per_step": R * 3 * N * 8 + R * 32,
               "steps": e2e_steps, "path": "ising_spins_set x R -> ising_pt_run -> ising_spins_get x R + energies"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_cores()
        rate, sample = cpu_reference_rate(w, 2, 1, threads, L_sample=min(L, 64))
        cpu = {"value": rate, "unit": "spin-updates/s", "cores": threads, "kind": "port", "sample": sample}

    # launches of this library inside the timed region: the paired colour passes of a round
    # (G*k + 1, or 2k with one group) plus fold + exchange + counter advance
    launches = args.steps * (per_round + 3)
    if rank == 0:
        line = {
            "metric": "spin-updates/s", "value": value, "unit": "spin-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (uniform random initial spins from Philox, seed 0x15196)",
            "config": {"workload": args.workload, "desc": w["desc"], "L": L, "replicas": R,
                       "sweeps_per_step": k, "sites": R * N, "parallelism": f"replicas x{world} (independent ensembles)",
                       "l2": "state larger than L2 (no flush)" if R * N * 12 > 126e6 else "state fits L2; no flush"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_src,
                         "kernel": "k_cb_sweep", "launch_ms": launch_ms,
                         "bytes_per_launch": bytes_per_launch, "sweep_ms": sweep_ms,
                         "basis": "24 B per attempted update (one FP32 x,y,z read + write per site per sweep)"},
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "schedule": {"l2_group_replicas": group, "colour_pass_launches_per_round": per_round,
                         "kernel": {0: "stencil", 1: "k_cb_sweep", 2: "k_cb_tma"}[kern_id]},
        }
        print(json.dumps(line), flush=True)
    pt.close()
    mesh.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--L", type=int, default=0, help="override lattice size (profiling)")
    ap.add_argument("--replicas", type=int, default=0, help="override replica count (profiling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w)
    else:
        run_gpu(args, w)


if __name__ == "__main__":
    main()
