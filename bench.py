#!/usr/bin/env python
"""Benchmark of the Heisenberg Metropolis / parallel-tempering hot path on B200.

One step = one parallel-tempering round of the workload: `sweeps_per_swap` colour-class
sweeps of every replica of every ensemble, then each ensemble's replica exchange, run by the
persistent multi-ensemble kernel (ising_ensembles_*, replayed from a CUDA graph) with its
schedule picked by the library's autotuner during warm-up; the FP64 recomputation of the
energy / magnetisation accumulators runs inside the timed region every `--resync-every`
rounds (default 10 rounds = 100 sweeps).  `--engine pt` times the per-colour-pass launch path
(ising_pt_*) instead.  metric: spin-updates/s = attempted single-site updates (N per replica
per sweep) / s.

Default workload (N=1), the configuration the metric "spin-updates/s and Q-ESS/s, learned vs
plain" is quoted on: simple cubic L=96, 48 replicas, T geometric 0.1-1.5, J=1 (ferromagnetic,
passed as J=-1 in the reference sign convention), bulk DMI D=0.5, B=0.25 along z, K=0, ball
move r=0.2, swaps every 10 sweeps.  Spin state 486 MiB (> 126 MB L2), so no L2 flush is needed
between steps.  The line also carries `fp64_error` (accumulator drift and snapshot errors of E,
|M| and Q against the FP64 oracle) and `q_ess` (learned patch proposal against plain
Metropolis: tau_int and effective samples per second of Q and E, observables per slot).
Workloads c3 (L=128 x 16) and c4 (12 ensembles L in {16,24,32,48,64,96}, 16-64 replicas each,
148,160,512 sites) are --workload options.

Under torchrun a single-ensemble workload runs one copy per rank (independent ensembles, weak
scaling); c4's ensembles are split across ranks by whole ensembles (strong scaling).  No
collective on the data path; the timed region is bracketed by barriers and the max over ranks
is reported.

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
    "c1": dict(L=16, R=1, tmin=0.5, tmax=0.5, J=-1.0, D=0.3, B=0.1, K=0.0, move="uniform", r=0.0, k=1,
               desc="SC L=16, T=0.5, J=1, bulk D=0.3, B=0.1, uniform unit-vector moves"),
    "c4": dict(L=96, R=64, tmin=0.1, tmax=2.0, J=-1.0, D=0.5, B=0.1, K=0.0, move="ball", r=0.2, k=10,
               desc="12 SC PT ensembles, L in {16,24,32,48,64,96} x2, (D,B) in {0.3,0.5,0.7}x{0.1,0.3}, "
                    "16-64 replicas, T 0.1-2.0, J=1, bulk DMI, B z",
               ensembles=[(L, {16: 16, 24: 16, 32: 32, 48: 32, 64: 48, 96: 64}[L],
                           [(0.3, 0.1), (0.3, 0.3), (0.5, 0.1), (0.5, 0.3), (0.7, 0.1), (0.7, 0.3)][i % 6])
                          for i, L in enumerate([16, 16, 24, 24, 32, 32, 48, 48, 64, 64, 96, 96])]),
}
# the reference's own crystals (src/unit_cells.f90): BCC as bin/PT runs it (shell 1 only, J' = 0,
# src/PT.f90:145,229-230) and hyper-kagome as bin/ISING does (src/ISING.f90:105), both with the
# default interfacial DMI of calculateHeisenbergEnergy; run by the per-pass PT path on the
# sublattice planes (BCC) and octant order (hyper-kagome) (the persistent engine covers simple cubic)
WORKLOADS["bcc"] = dict(cell="bcc", L=96, R=16, tmin=0.1, tmax=2.0, J=-1.0, D=0.5, B=0.2, K=0.0, move="ball", r=0.2,
                        k=10, dmi="interfacial",
                        desc="BCC 96^3 cells (2 atoms) x 16 PT replicas, T 0.1-2.0, J=1, interfacial D=0.5, B=0.2 z, "
                             "shell 1")
WORKLOADS["hk"] = dict(cell="hk", L=48, R=16, tmin=0.1, tmax=2.0, J=-1.0, D=0.3, B=0.1, K=0.0, move="ball", r=0.2,
                       k=10, dmi="interfacial",
                       desc="hyper-kagome 48^3 cells (12 atoms) x 16 PT replicas, T 0.1-2.0, J=1, interfacial D=0.3, "
                            "B=0.1 z, shell 1")
# bin/ISING takes J' from its command line (src/ISING.f90:50-58): hyper-kagome with shell 2 on
WORKLOADS["hkjp"] = dict(cell="hk", L=48, R=16, tmin=0.1, tmax=2.0, J=-1.0, Jp=0.1, D=0.3, B=0.1, K=0.0,
                         move="ball", r=0.2, k=10, dmi="interfacial",
                         desc="hyper-kagome 48^3 cells (12 atoms) x 16 PT replicas, T 0.1-2.0, J=1, J'=0.1 "
                              "(shells 1-2), interfacial D=0.3, B=0.1 z")
WORKLOADS["stats"] = dict(L=96, nz=96, scale=10, J=-1.0, D=0.5, B=0.25, K=0.0, move="ball", r=0.2, tmin=0.1,
                          desc="chainMesh_statistics on SC L=96 (96 slices): winding per slice, magnetisation and "
                               "the 60 x 20 skyrmion search on the middle slice's 960 x 960 interpolated density")
WORKLOADS["setup"] = dict(cell="bcc", L=128, sample_L=48,
                          desc="mesh set-up (makeChainMesh: positions, shells, neighbour and derivative lists, "
                               "colouring, device state) of the reference's BCC cell at 128^3 cells (4,194,304 atoms)")
WORKLOADS["demag"] = dict(cell="sc", L=64,
                          desc="calculate_demagnetisation_field on SC 64^3 (262,144 atoms): CIC deposit, 3-D "
                               "transforms, k-space projection, gather; FP64 field returned to the host")
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
_NVML_POLLER = r"""
import sys, time
import pynvml as nv
nv.nvmlInit()
bus = int(sys.argv[1])
h = None
for i in range(nv.nvmlDeviceGetCount()):
    d = nv.nvmlDeviceGetHandleByIndex(i)
    if bus < 0 or nv.nvmlDeviceGetPciInfo(d).bus == bus:
        h = d
        break
mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
print("max", mx, flush=True)
while True:
    print(time.time_ns(), nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), nv.nvmlDeviceGetCurrentClocksEventReasons(h),
          flush=True)
    time.sleep(0.002)
"""


class ClockSampler:
    """SM clock and clock-event reasons of the timed GPU while the timed region runs.

    A separate process polls NVML (read-only queries) every ~2 ms and timestamps each sample;
    mark() / stop() bracket the timed region and only samples inside it are kept.  (An
    in-process NVML poller waits behind the CUDA driver call that blocks on the stream.)
    Without NVML an `nvidia-smi -lms 200` subprocess is the fallback."""
    FIELDS = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvmlClocksEventReason*)
    REASONS = (("sw_power_cap", 0x4), ("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20),
               ("hw_thermal_slowdown", 0x40))

    def __init__(self, bus=None):
        self.bus = bus if isinstance(bus, int) else None  # PCI bus number of the timed GPU
        self.proc = None
        self.kind = None
        self.t0 = None
        # the raw samples (the line carries their summary): $BENCH_CLOCKS_DIR or the temp dir
        import tempfile
        self.path = os.path.join(os.environ.get("BENCH_CLOCKS_DIR") or tempfile.gettempdir(),
                                 f"ising_bench_clocks_{os.getpid()}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        self.f = open(self.path, "w")
        try:
            import pynvml  # noqa: F401
            self.proc = subprocess.Popen([sys.executable, "-c", _NVML_POLLER, str(-1 if self.bus is None else self.bus)],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            self.kind = "nvml"
            deadline = time.time() + 10.0
            while time.time() < deadline and self.proc.poll() is None:   # wait for the first sample
                if sum(1 for _ in open(self.path)) >= 2:
                    break
                time.sleep(0.01)
            if self.proc.poll() is None:
                self.t0 = time.time_ns()
                return
            self.proc = None
        except Exception:
            self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
            self.kind = "nvidia-smi"
        except Exception:
            self.proc = None
        self.t0 = time.time_ns()

    def mark(self):
        """Start of the timed region (after warm-up work queued since start())."""
        self.t0 = time.time_ns()

    def stop(self):
        t1 = time.time_ns()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        if self.kind == "nvml":
            time.sleep(0.01)   # one more sample after the region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        lines = open(self.path).read().split("\n")
        if self.kind == "nvml":
            mx, rows = None, []
            for line in lines:
                parts = line.split()
                if len(parts) == 2 and parts[0] == "max":
                    mx = int(parts[1])
                elif len(parts) == 3:
                    try:
                        rows.append((int(parts[0]), int(parts[1]), int(parts[2])))
                    except ValueError:
                        pass
            inside = [r for r in rows if self.t0 <= r[0] <= t1]
            if not inside and rows:   # region shorter than the poll period: the nearest samples
                inside = sorted(rows, key=lambda r: min(abs(r[0] - self.t0), abs(r[0] - t1)))[:2]
            if inside:
                out.update(sm_mhz=statistics.median(r[1] for r in inside), sm_max_mhz=mx,
                           reasons=sorted({n for r in inside for n, bit in self.REASONS if r[2] & bit}),
                           samples=len(inside), source="nvml")
            return out
        rows = []
        for line in lines:
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
        out.update(sm_mhz=statistics.median(sm), sm_max_mhz=mx, reasons=reasons, samples=len(rows),
                   source="nvidia-smi")
        return out


# ---------------------------------------------------------------- reference (CPU) arm
def oracle_cell(O, w):
    return {"bcc": O.BCC_CELL, "hk": O.HYPER_KAGOME_CELL}.get(w.get("cell"), O.SC_CELL)


def cpu_reference_rate(w, steps, warmup, threads, L_sample=None):
    """Throughput of the CPU restatement of Metropolis_mcs on the host cores: one sweep of
    one replica per step (numAtoms trials), the reference's parallel structure (OpenMP over
    trials, snapshot semantics), same Hamiltonian.  Returns (updates/s, sample text)."""
    from oracle import oracle as O
    O.build()
    L = L_sample or w["L"]
    frac, (a, b, c, ab, bc, ca) = oracle_cell(O, w)
    m = O.Mesh(frac, L, L, L, a, b, c, ab, bc, ca)
    m.init_uniform(0x15196)
    p = O.Params(J=w["J"], J_prime=w.get("Jp", 0.0), Dz=w["D"], B=w["B"], K=w["K"],
                 dmi_bulk=w.get("dmi", "bulk") == "bulk")
    beta = 1.0 / w["tmin"]
    for _ in range(warmup):
        m.metropolis_mcs_omp(beta, 1, p, w["r"], n_threads=threads, time_seed=1)
    t0 = time.perf_counter()
    for _ in range(steps):
        m.metropolis_mcs_omp(beta, 1, p, w["r"], n_threads=threads, time_seed=1)
    dt = time.perf_counter() - t0
    rate = steps * m.natoms / dt
    return rate, (f"{steps} sweep(s) of one {w.get('cell', 'sc').upper()} L={L} replica ({m.natoms} trials each), "
                  f"{threads} threads")


def cpu_fast_rate(w, threads, L=64, sweeps=4):
    """The fastest CPU form of the sweep: the oracle library's FP32 OpenMP checkerboard on SC
    L^3 (same Hamiltonian, moves and Philox keys as the device path; it replays the FP64
    colour-class sweep decision for decision).  Returns (updates/s, sample text)."""
    import numpy as np
    from oracle import oracle as O
    O.build()
    m = O.Mesh.sc(L)
    m.init_uniform(0x15196)
    planes = np.ascontiguousarray(m.spins.T.astype(np.float32))
    p = O.Params(J=w["J"], Dz=w["D"], B=w["B"], K=w["K"], dmi_bulk=True)
    key = O.SweepKey(seed=0x15196, ensemble=0, replica=0, move=1 if w["move"] == "ball" else 0, r=w["r"],
                     philox_rounds=10)
    beta = 1.0 / w["tmin"]
    O.cb_sweeps_f32(planes, L, 1, 0, beta, p, key, threads)
    t0 = time.perf_counter()
    O.cb_sweeps_f32(planes, L, sweeps, 1, beta, p, key, threads)
    dt = time.perf_counter() - t0
    return sweeps * L ** 3 / dt, f"{sweeps} sweeps of one SC L={L} replica, FP32 checkerboard, {threads} threads"


def run_reference(args, w):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    if args.workload in ("setup", "demag"):
        if args.workload == "setup":
            cpu = setup_cpu_baseline(w)
        else:
            import numpy as np
            rng = np.random.default_rng(0x15196)
            sp = rng.normal(size=(w["L"] ** 3, 3))
            sp /= np.linalg.norm(sp, axis=1, keepdims=True)
            cpu, _ = demag_cpu_baseline(w, sp.astype(np.float32).astype(np.float64))
        line = {"metric": cpu["unit"], "value": cpu["value"], "unit": cpu["unit"], "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / cpu["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": args.workload, "desc": w["desc"]},
                "cpu_baseline": cpu,
                "e2e": {"value": cpu["value"], "unit": cpu["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    if args.workload == "stats":
        L, nz = args.L or w["L"], w["nz"]
        cpu = stats_cpu_baseline(w, L, nz, skyrmion_texture(L, nz, L / 6, [(L / 4, L / 4), (3 * L / 4, L / 3),
                                                                           (L / 2, 3 * L / 4)], 0x15196))
        line = {"metric": "statistics calls/s", "value": cpu["value"], "unit": cpu["unit"], "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / cpu["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": "stats", "desc": w["desc"]},
                "cpu_baseline": cpu,
                "e2e": {"value": cpu["value"], "unit": cpu["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    threads = host_cores()
    rate, sample = cpu_reference_rate(w, max(args.steps, 1), max(args.warmup, 0), threads)
    line = {
        "metric": "spin-updates/s", "value": rate, "unit": "spin-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * (w["L"] ** 3) * cell_atoms(w) / rate, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "sample": "one replica per step"},
        "cpu_baseline": {"value": rate, "unit": "spin-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": "spin-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def link_rates(torch, host, stream):
    """Host<->device copy rates over the given pinned host arrays (lists of 1-D FP64 tensors):
    all of them to the device, all back, and both directions at once on two streams."""
    flat = [t for hs in host for t in hs]
    dev = [torch.empty_like(t, device="cuda") for t in flat]
    nbytes = sum(t.numel() * 8 for t in flat)
    up, down = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(fn):
        best = float("inf")
        for _ in range(3):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            for st in (up, down):
                stream.wait_stream(st)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    def h2d():
        with torch.cuda.stream(up):
            for d, h in zip(dev, flat):
                d.copy_(h, non_blocking=True)

    def d2h():
        with torch.cuda.stream(down):
            for d, h in zip(dev, flat):
                h.copy_(d, non_blocking=True)

    t_up, t_down = timed(h2d), timed(d2h)
    t_both = timed(lambda: (h2d(), d2h()))
    del dev
    return {"h2d_gbs": nbytes / t_up / 1e6, "d2h_gbs": nbytes / t_down / 1e6,
            "bidir_gbs_each": nbytes / t_both / 1e6, "bidir_ms": t_both}


def cell_atoms(w):
    return {"bcc": 2, "hk": 12}.get(w.get("cell"), 1)


def make_mesh(ib, w, L, R, dev):
    """The workload's mesh: simple cubic, or the reference's BCC / hyper-kagome cell."""
    if w.get("cell") == "bcc":
        a, b, c, ab, bc, ca, f = ib.bcc_unit_cell()
    elif w.get("cell") == "hk":
        a, b, c, ab, bc, ca, f = ib.hyper_kagome_unit_cell()
    else:
        return ib.ChainMesh.simple_cubic(L, n_replicas=R, device=dev)
    return ib.ChainMesh(L, L, L, f, a, b, c, ab, bc, ca, n_replicas=R, device=dev)


def ensembles_of(args, w):
    """[(L, replicas, D, B)] of the workload."""
    if "ensembles" in w:
        return [(L, R, D, B) for L, R, (D, B) in w["ensembles"]]
    return [(args.L or w["L"], args.replicas or w["R"], w["D"], w["B"])]


def fp64_errors(ib, O, eng, members, w, k):
    """Error of the reported observables against FP64: (1) the drift of the running FP64
    accumulators (sums of FP32 dE, dM) over 9 rounds since the last resync, against the device
    recomputation; (2) on the downloaded spins of the coldest and the hottest slot of the
    first ensemble, the device E, |M| and winding numbers against the FP64 oracle."""
    import numpy as np
    eng.run(k, 9)
    acc = [eng.energies(i) for i in range(len(members))]
    eng.resync()
    fresh = [eng.energies(i) for i in range(len(members))]
    drift_e = max(float(np.max(np.abs(a[0] - f[0]))) / m.numAtoms for a, f, (m, *_) in zip(acc, fresh, members))
    drift_m = max(float(np.max(np.abs(a[1] - f[1]))) / m.numAtoms for a, f, (m, *_) in zip(acc, fresh, members))
    m, betas, _, _ = members[0]
    L = m.numCellsX
    N = m.numAtoms
    perm = eng.permutation(0)
    if "ensembles" in w:
        D0, B0 = w["ensembles"][0][2]
    else:
        D0, B0 = w["D"], w["B"]
    op = O.Params(J=w["J"], Dz=D0, B=B0, K=w["K"], dmi_bulk=True)
    E_dev, M_dev = fresh[0]
    snaps = []
    for t in (0, len(betas) - 1):
        r = int(perm[t])
        s = m.get_spins(r)
        om = O.Mesh.sc(L)
        om.set_spins(s)
        e_o = om.canonical_energy(op)
        mo = float(np.linalg.norm(s.sum(axis=0))) / N
        md = float(np.linalg.norm(M_dev[r])) / N
        q_dev = ib.winding_all_slices(m, r)
        q_o = np.array([om.winding_number(z) for z in range(1, L + 1)])
        snaps.append({"slot": t, "T": float(1.0 / betas[t]),
                      "E_per_site": {"device": float(E_dev[r]) / N, "oracle": e_o / N,
                                     "abs_err": abs(float(E_dev[r]) - e_o) / N},
                      "absM": {"device": md, "oracle": mo, "abs_err": abs(md - mo)},
                      "Q_sum": {"device": float(q_dev.sum()), "oracle": float(q_o.sum()),
                                "max_abs_err_per_slice": float(np.max(np.abs(q_dev - q_o))),
                                "rounded_equal": bool(round(q_dev.sum()) == round(q_o.sum()))}})
    return {"accumulator_drift_per_site_after_90_sweeps": {"E": drift_e, "M": drift_m},
            "snapshots_vs_fp64_oracle": snaps,
            "note": "device E: FP64 sums of FP32 terms; Q: FP64 Berg-Luscher per slice; C_v and chi derive from "
                    "the recorded E and |M|, whose errors are those above"}


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
    k = w["k"]
    move = _lib.MOVE_BALL if w["move"] == "ball" else _lib.MOVE_UNIFORM
    spec = ensembles_of(args, w)
    # multi-ensemble workloads are split across ranks by whole ensembles (the parameter slots
    # of src/PT.f90:147-176 never exchange data): strong scaling; a single ensemble runs as
    # one independent copy per rank (distinct Philox ensemble ids): weak scaling
    split = world > 1 and len(spec) > 1
    if split:
        from ising_b200.sharding import partition_ensembles
        mine = partition_ensembles([float(L ** 3 * R) for L, R, _, _ in spec], world)[rank]
    else:
        mine = list(range(len(spec)))
    members = []
    for i in mine:
        L, R, D, B = spec[i]
        ens_id = i if split else rank * len(spec) + i
        m = make_mesh(ib, w, L, R, dev)
        m.set_stream(stream.cuda_stream)
        m.init_uniform(0x15196, ensemble=ens_id)
        p = ib.params(J=w["J"], J_prime=w.get("Jp", 0.0), Dz=D, B=B, K=w["K"], dmi=w.get("dmi", "bulk"))
        members.append((m, 1.0 / ib.temperature_ladder(w["tmin"], w["tmax"], R), p, ens_id))
    sites = sum(spec[i][0] ** 3 * spec[i][1] for i in mine) * cell_atoms(w)
    sites_job = sum(L ** 3 * R for L, R, _, _ in spec) if split else world * sites
    updates_per_step = sites * k

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

    sched_info = {}
    eng = None
    n_chunks = 1
    engine = "pt" if w.get("cell") else args.engine      # the engine runs simple cubic only
    if engine == "ensembles":
        eng = ib.Ensembles(members, seed=0x15196, move=move, r=w["r"]) if members else None
        if eng:
            eng.set_stream(stream.cuda_stream)
            if args.schedule:   # threads,chunk_pairs,loader: a fixed schedule instead of the autotuner
                bt, cp, ld = (int(v) for v in args.schedule.split(","))
                eng.set_schedule(block_threads=bt, chunk_pairs=cp, loader=ld)
            # 4 rounds per candidate: near-tied schedules are told apart by more than timer noise
            trials = eng.autotune(k, 4) if not (args.no_autotune or args.schedule) else []
            eng.run(k, max(args.warmup, 1))
            # the periodic FP64 resync that bounds the accumulators' drift runs inside the
            # timed region, every resync_every rounds counted from here
            eng.set_resync(args.resync_every)
            sched_info = eng.schedule()
            sched_info["autotune_trials"] = len(trials)
            if trials:
                best = min(trials, key=lambda t: t["ms_per_round"])
                worst = max(trials, key=lambda t: t["ms_per_round"])
                sched_info["autotune_spread_ms"] = [best["ms_per_round"], worst["ms_per_round"]]
        run = (lambda n: eng.run(k, n)) if eng else (lambda n: None)
        energies = lambda: [eng.energies(i) for i in range(len(members))]
        kernel_name = "k_ensembles_fused" if sched_info.get("loader") == "fused" else "k_ensembles"
        # one persistent launch per resync interval (plus a memset node), then the resync's
        # energy reduction (energy pass + block fold) and its copy into the accumulators
        n_chunks = -(-args.steps // args.resync_every) if args.resync_every else 1
        launches_timed = n_chunks + (args.steps // args.resync_every) * 2 if args.resync_every else 1
        closers = [eng] if eng else []
    else:
        if len(members) != 1:
            raise SystemExit("--engine pt runs single-ensemble workloads only")
        m, betas, p, ens_id = members[0]
        pt = ib.ParallelTempering(m, betas, p, seed=0x15196, ensemble=ens_id, move=move, r=w["r"],
                                  l2_group=args.l2_group, sweep_kernel=args.sweep_kernel)
        pt.run(k, max(args.warmup, 1))
        run = lambda n: pt.run(k, n)
        energies = lambda: [pt.energies()]
        group, per_round, kern_id = pt.schedule(k)
        sched_info = {"l2_group_replicas": group, "colour_pass_launches_per_round": per_round,
                      "kernel": {0: "k_octant_colour" if m.layout == "octant" else "k_general_colour",
                                 1: "k_cb_sweep", 2: "k_cb_tma", 3: "k_octant_fast",
                                 4: "k_octant_engine", 5: "k_bip_sweep", 6: "k_octant_pair"}[kern_id],
                      "layout": m.layout}
        kernel_name = sched_info["kernel"]
        launches_timed = args.steps * (per_round + 3)   # colour passes + fold + exchange + advance
        closers = [pt]
    barrier()

    clocks = ClockSampler(getattr(torch.cuda.get_device_properties(dev), "pci_bus_id", None))
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    clocks.mark()
    ev0.record(stream)
    run(args.steps)
    ev1.record(stream)
    barrier()
    ms_local = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms_local)
    clk = clocks.stop()
    value = sites_job * k * args.steps / (ms / 1e3)

    # dominant kernel: with the engine the timed region is the persistent launches (one per
    # resync interval) and the resyncs (one FP64 energy pass each, about 1-1.4 ms per 10
    # rounds of C5: 2-3 % of the region), so the region's duration stands for the launches'
    # duration (the roofline fraction is a little low by that); with --engine pt the
    # colour-pass kernel is timed alone over relax sweeps
    if engine == "ensembles":
        launch_ms = ms_local / max(n_chunks, 1)
        bytes_per_launch = BYTES_PER_UPDATE * updates_per_step * args.steps / max(n_chunks, 1)
    else:
        n_relax = max(4, min(40, args.steps * k // 2))
        launches = pt.schedule(n_relax)[1]
        pt.relax(2)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pt.relax(n_relax)
        e1.record(stream)
        barrier()
        launch_ms = e0.elapsed_time(e1) / launches
        bytes_per_launch = BYTES_PER_UPDATE * sites * n_relax / launches
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    achieved = bytes_per_launch / (launch_ms / 1e3) / 1e9 if launch_ms > 0 else 0.0
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    if os.path.exists(tfile):
        try:
            for t in json.load(open(tfile)).get("kernels", []):
                # an entry with "only" holds for those workloads alone (the traffic of a class
                # pass depends on the stencil)
                if t.get("only") and args.workload not in t["only"]:
                    continue
                if t.get("kernel") == kernel_name and t.get("bytes_per_update"):
                    traffic = t["bytes_per_update"] * bytes_per_launch / BYTES_PER_UPDATE
        except Exception:
            traffic = None

    # end to end through the C-ABI with host-owned FP64 spins (the reference's atomSpins):
    # every step uploads all replicas from pinned host memory, runs the round, downloads
    # all replicas and the per-replica energies.  The transfers are queued per replica
    # (ising_spins_*_async): the upload of replica r starts once the previous step's download
    # of r has landed in the host array, while other replicas still download, so the two
    # directions of the link overlap; the run waits for every upload, and the timed region
    # ends after the last downloads have landed.
    e2e = None
    if not args.no_e2e and members:
        L_ = _lib.load()
        host = [[torch.empty(3 * mm.numAtoms, dtype=torch.float64, pin_memory=True) for _ in range(len(b))]
                for mm, b, _, _ in members]
        dp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_double))
        for (mm, b, _, _), hs in zip(members, host):
            for r in range(len(b)):
                _lib.check(L_.ising_spins_get(mm.handle, r, dp(hs[r])), "get")
        e2e_steps = max(1, min(args.steps, 5))

        def e2e_step():
            for (mm, b, _, _), hs in zip(members, host):
                for r in range(len(b)):
                    _lib.check(L_.ising_spins_set_async(mm.handle, r, dp(hs[r])), "set")
            run(1)          # waits for the uploads
            for (mm, b, _, _), hs in zip(members, host):
                for r in range(len(b)):
                    _lib.check(L_.ising_spins_get_async(mm.handle, r, dp(hs[r])), "get")
            return energies()

        def e2e_wait():
            for mm, _, _, _ in members:
                _lib.check(L_.ising_spins_wait(mm.handle), "wait")

        e2e_step()
        e2e_wait()
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        e2e_wait()
        a1.record(stream)
        barrier()
        wall = time.perf_counter() - t0
        e_ms = max_over_ranks(max(a0.elapsed_time(a1), wall * 1e3))
        n_rep = sum(len(b) for _, b, _, _ in members)
        e2e = {"value": sites_job * k * e2e_steps / (e_ms / 1e3), "unit": "spin-updates/s",
               "h2d_bytes_per_step": sites * 3 * 8, "d2h_bytes_per_step": sites * 3 * 8 + n_rep * 32,
               "steps": e2e_steps,
               "path": "ising_spins_set_async per replica -> one round -> ising_spins_get_async per replica "
                       "+ energies; ising_spins_wait at the end"}
        # the link's own rates on the same pinned arrays (one bulk copy per direction, device
        # buffers of the same size): the floor of a step that does not overlap the round with
        # the copies is (both directions at once) + (the round)
        link = link_rates(torch, host, stream)
        floor_ms = link["bidir_ms"] + ms / args.steps
        e2e["link"] = {k_: v for k_, v in link.items() if k_ != "bidir_ms"}
        e2e["floor_ms_per_step"] = floor_ms
        e2e["frac_of_floor"] = floor_ms / (e_ms / e2e_steps)
        del host

    errors = None
    if rank == 0 and world == 1 and eng is not None and not args.no_cpu:
        from oracle import oracle as O
        O.build()
        errors = fp64_errors(ib, O, eng, members, w, k)

    cpu = cpu_fast = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_cores()
        # one replica of the workload's largest lattice (about a second of CPU work)
        L_cpu = max(L for L, _, _, _ in spec)
        rate, sample = cpu_reference_rate(w, 2, 1, threads, L_sample=L_cpu)
        cpu = {"value": rate, "unit": "spin-updates/s", "cores": threads, "kind": "port", "sample": sample}
        if not w.get("cell"):     # the fast CPU form is the simple-cubic checkerboard
            rate, sample = cpu_fast_rate(w, threads, L=L_cpu)
            cpu_fast = {"value": rate, "unit": "spin-updates/s", "cores": threads, "kind": "optimised port",
                        "sample": sample}

    for c in closers:
        c.close()
    for mm, *_ in members:
        mm.close()
    q_ess = training = None
    if rank == 0 and world == 1 and args.workload == "c5" and not args.no_learned:
        q_ess, training = learned_vs_plain(args, w)

    if rank == 0:
        line = {
            "metric": "spin-updates/s", "value": value, "unit": "spin-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong" if split else "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (uniform random initial spins from Philox, seed 0x15196)",
            "config": {"workload": args.workload, "desc": w["desc"], "ensembles": len(spec),
                       "lattices": sorted({L for L, _, _, _ in spec}), "replicas": sum(R for _, R, _, _ in spec),
                       "sweeps_per_step": k, "sites": sites_job, "engine": engine,
                       "resync_every_rounds": args.resync_every if engine == "ensembles" else None,
                       "parallelism": (f"whole ensembles over {world} ranks" if split
                                       else f"replicas x{world} (independent ensembles)"),
                       "l2": "state larger than L2 (no flush)" if sites * 12 > 126e6 else "state fits L2; no flush"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_src,
                         "kernel": kernel_name, "launch_ms": launch_ms, "bytes_per_launch": bytes_per_launch,
                         "basis": "24 B per attempted update (one FP32 x,y,z read + write per site per sweep)"},
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                       "samples": clk["samples"]},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "cpu_fastest": cpu_fast,
            "gpu_launches": launches_timed,
            "schedule": sched_info,
            "fp64_error": errors,
        }
        if q_ess is not None:
            line["q_ess"] = q_ess
            line["training"] = training
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------- post-processing: chainMesh_statistics
def skyrmion_texture(L, nz, R, centres, seed):
    """A z-uniform texture of Bloch skyrmions of radius R at the given (x, y) centres on a
    core-down background, plus small seeded noise: (L*L*nz, 3) unit vectors in atom order."""
    import numpy as np
    rng = np.random.default_rng(seed)
    x, y = np.meshgrid(np.arange(L, dtype=np.float64), np.arange(L, dtype=np.float64), indexing="ij")
    theta = np.zeros((L, L))
    phi = np.zeros((L, L))
    for cx, cy in centres:
        dx = (x - cx + L / 2) % L - L / 2
        dy = (y - cy + L / 2) % L - L / 2
        r = np.hypot(dx, dy)
        inside = r < R
        theta = np.where(inside, np.pi * (1.0 - r / R), theta)
        phi = np.where(inside, np.arctan2(dy, dx) + np.pi / 2, phi)
    s = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), -np.cos(theta)], axis=-1)
    s = np.repeat(s[:, :, None, :], nz, axis=2).reshape(-1, 3) + 0.05 * rng.normal(size=(L * L * nz, 3))
    return s / np.linalg.norm(s, axis=1, keepdims=True)


def stats_cpu_baseline(w, L, nz, spins, n_sample=4):
    """chainMesh_statistics on the oracle (one host thread): the nz slice winding numbers and
    magnetisation, the FFT interpolation of the middle slice, and n_sample pairs of the
    60 x 20 threshold/sigma search through the literal calculate_skyrmion_number restatement,
    scaled to the 1200 pairs a search without an early exit evaluates."""
    from oracle import oracle as O
    O.build()
    om = O.Mesh.sc(L, L, nz)
    om.set_spins(spins)
    t0 = time.perf_counter()
    for z in range(1, nz + 1):
        om.winding_number(z)
    om.statistics()
    dens = O.winding_density_interpolated(om, nz // 2, w["scale"], w["scale"])
    t_fixed = time.perf_counter() - t0
    t0 = time.perf_counter()
    for k in range(n_sample):      # the first pairs of the search: threshold index 1, sigma index 1..n
        thr = 0.95 - (1 / 60) * (0.95 - 1e-5)
        O.skyrmion_number(dens, L, L, thr, 1, 1.0 - ((k + 1) / 20.0) * (1.0 - 0.00001))
    t_pair = (time.perf_counter() - t0) / n_sample
    pairs = 1200
    t_call = t_fixed + pairs * t_pair
    fx = L * w["scale"]
    return {"value": 1.0 / t_call, "unit": "statistics calls/s", "cores": 1, "kind": "port",
            "sample": f"{n_sample} of the {pairs} (threshold, sigma) pairs through the literal "
                      f"calculate_skyrmion_number restatement on the {fx}x{fx} density ({t_pair*1e3:.1f} ms each, "
                      f"scaled to {pairs}) plus the {nz} slice winding numbers, magnetisation and one FFT "
                      f"interpolation ({t_fixed*1e3:.1f} ms); the reference redoes the interpolation per pair"}


def _secondary_line(args, w, metric, unit, value, world, per_step_s, clocks, cpu, e2e, extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * per_step_s, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "desc": w["desc"],
                       "timer": "host wall clock around synchronous C-ABI calls"},
            "roofline": None,
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "e2e": e2e, "cpu_baseline": cpu}
    line.update(extra)
    print(json.dumps(line), flush=True)


def setup_cpu_baseline(w):
    """The oracle's restatement of makeChainMesh (src/chainMesh.f90:729-911: shells by a scan of
    the 125 surrounding cells per atom, neighbour and derivative lists) on one host thread, on a
    smaller mesh of the same cell, scaled by atom count (its cost is linear in the atoms)."""
    from oracle import oracle as O
    O.build()
    frac, (a, b, c, ab, bc, ca) = O.BCC_CELL if w["cell"] == "bcc" else O.SC_CELL
    Ls = w["sample_L"]
    t0 = time.perf_counter()
    m = O.Mesh(frac, Ls, Ls, Ls, a, b, c, ab, bc, ca)
    dt = time.perf_counter() - t0
    n_sample = m.natoms
    del m
    n_full = w["L"] ** 3 * len(frac)
    t_full = dt * n_full / n_sample
    return {"value": 1.0 / t_full, "unit": "mesh set-ups/s", "cores": 1, "kind": "port",
            "sample": f"BCC {Ls}^3 ({n_sample} atoms) in {dt:.2f} s, scaled by atoms to {n_full}"}


def run_setup(args, w):
    """One step = ising_mesh_create + ising_mesh_destroy of the workload's mesh (one replica):
    the lattice compiler (per-sublattice stencils from one scan at cell 0, octant colouring) and
    the device state, against the oracle's per-atom restatement of makeChainMesh."""
    import torch
    import ising_b200 as ib
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    L = args.L or w["L"]
    a, b, c, ab, bc, ca, f = ib.bcc_unit_cell()
    for _ in range(max(args.warmup, 1)):
        ib.ChainMesh(L, L, L, f, a, b, c, ab, bc, ca, n_replicas=1, device=local).close()
    clk = ClockSampler(getattr(torch.cuda.get_device_properties(local), "pci_bus_id", None))
    clk.start()
    torch.cuda.synchronize()
    clk.mark()
    t0 = time.perf_counter()
    natoms = 0
    for _ in range(args.steps):
        m = ib.ChainMesh(L, L, L, f, a, b, c, ab, bc, ca, n_replicas=1, device=local)
        natoms = m.numAtoms
        m.close()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / args.steps
    clocks = clk.stop()
    cpu = setup_cpu_baseline(w) if rank == 0 and world == 1 and not args.no_cpu else None
    if rank == 0:
        _secondary_line(args, w, "mesh set-ups/s", "mesh set-ups/s", 1.0 / dt, world, dt, clocks, cpu,
                        {"value": 1.0 / dt, "unit": "mesh set-ups/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0, "path": "ising_mesh_create from the unit cell (host arrays in, "
                                                           "device state out) + ising_mesh_destroy"},
                        {"gpu_launches": args.steps * 2, "result": {"atoms": natoms}})


def demag_cpu_baseline(w, spins):
    """oracle/demag_ref.demag_field (numpy FP64, numpy's FFTs standing in for FFTW) on the same
    mesh and spins, one host process."""
    from oracle import oracle as O
    from oracle import demag_ref as D
    O.build()
    L = w["L"]
    om = O.Mesh.sc(L)
    t0 = time.perf_counter()
    H = D.demag_field(om, spins)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": "demag fields/s", "cores": 1, "kind": "port",
            "sample": f"one field of SC {L}^3 ({om.natoms} atoms) in {dt:.2f} s"}, H


def run_demag(args, w):
    """One step = one ising_demag_field call on a resident replica (the field returned to the host
    in FP64); e2e adds the upload of the spins.  The result is checked against the oracle."""
    import numpy as np
    import torch
    import ising_b200 as ib
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    L = args.L or w["L"]
    mesh = ib.ChainMesh.simple_cubic(L, device=local)
    rng = np.random.default_rng(0x15196)
    spins = rng.normal(size=(mesh.numAtoms, 3))
    spins /= np.linalg.norm(spins, axis=1, keepdims=True)
    spins = spins.astype(np.float32).astype(np.float64)
    mesh.set_spins(spins)
    for _ in range(max(args.warmup, 1)):
        H = ib.demag_field(mesh, 0)
    clk = ClockSampler(getattr(torch.cuda.get_device_properties(local), "pci_bus_id", None))
    clk.start()
    torch.cuda.synchronize()
    clk.mark()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        H = ib.demag_field(mesh, 0)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / args.steps
    clocks = clk.stop()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        mesh.set_spins(spins)
        H = ib.demag_field(mesh, 0)
    e2e_dt = (time.perf_counter() - t0) / max(1, args.steps // 2)
    cpu, err = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, Href = demag_cpu_baseline(w, spins)
        err = float(np.max(np.abs(H - Href)))
    mesh.close()
    if rank == 0:
        n = spins.shape[0]
        _secondary_line(args, w, "demag fields/s", "demag fields/s", 1.0 / dt, world, dt, clocks, cpu,
                        {"value": 1.0 / e2e_dt, "unit": "demag fields/s", "h2d_bytes_per_step": int(n * 24),
                         "d2h_bytes_per_step": int(n * 24), "path": "ising_spins_set (host doubles) -> "
                                                                   "ising_demag_field (host doubles)"},
                        {"gpu_launches": args.steps * 9, "result": {"max_abs_err_vs_oracle": err,
                                                                    "max_abs_field": float(np.abs(H).max())}})


def run_stats(args, w):
    """One step = one chainMesh_statistics call (src/PT-Utils.f90:33-66) through the C-ABI on a
    resident replica; e2e adds the upload of the spins from pinned host memory."""
    import numpy as np
    import torch
    import ising_b200 as ib
    rank, world, local = dist_env()
    L, nz = args.L or w["L"], w["nz"]
    torch.cuda.set_device(local)
    mesh = ib.ChainMesh.simple_cubic(L, L, nz, device=local)
    ib.set_interpolation_scale(mesh, w["scale"], w["scale"])
    spins = skyrmion_texture(L, nz, L / 6, [(L / 4, L / 4), (3 * L / 4, L / 3), (L / 2, 3 * L / 4)], 0x15196)
    host = torch.from_numpy(np.ascontiguousarray(spins)).pin_memory()
    mesh.set_spins(host.numpy())
    for _ in range(args.warmup):
        res = ib.chain_mesh_statistics_full(mesh)
    clk = ClockSampler(getattr(torch.cuda.get_device_properties(local), "pci_bus_id", None))
    clk.start()
    torch.cuda.synchronize()
    clk.mark()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res = ib.chain_mesh_statistics_full(mesh)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    clocks = clk.stop()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        mesh.set_spins(host.numpy())
        res = ib.chain_mesh_statistics_full(mesh)
    torch.cuda.synchronize()
    e2e_dt = (time.perf_counter() - t0) / max(1, args.steps // 2)
    sk, wmid, wspread, mag = res
    zmid = nz // 2
    total = ib.calculate_winding_number2(mesh, zmid)
    early = abs(sk - total) < 0.1      # the search stops at the first pair that matches Q
    fx, fy = L * w["scale"], L * w["scale"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = stats_cpu_baseline(w, L, nz, mesh.get_spins(0))
    if rank == 0:
        line = {
            "metric": "statistics calls/s", "value": args.steps / dt, "unit": "statistics calls/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (three Bloch skyrmions of radius L/6, z-uniform, 5% seeded noise)",
            "config": {"workload": "stats", "desc": w["desc"], "L": L, "nz": nz, "fine_grid": [fx, fy],
                       "pairs_searched": 1200 if not early else "early exit",
                       "timer": "host wall clock around synchronous C-ABI calls (device and host stages)"},
            "result": {"skyrmion_number_middle": sk, "winding_number_middle": wmid,
                       "winding_number_spread": wspread, "magnetisation": list(map(float, mag))},
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "e2e": {"value": 1.0 / e2e_dt, "unit": "statistics calls/s", "h2d_bytes_per_step": int(spins.size * 8),
                    "d2h_bytes_per_step": int(20 * L * L * 8 + 2 * nz * 8 + 20 * 12),
                    "path": "ising_spins_set (host doubles) -> ising_chain_mesh_statistics; d2h excludes the "
                            "local-maximum lists (12 B per listed cell)"},
            "cpu_baseline": cpu,
            "gpu_launches": args.steps * 10,
        }
        print(json.dumps(line), flush=True)
    mesh.close()


# ---------------------------------------------------------------- C1: GPU vs the CPU reference chain
def run_c1(args):
    """The reference's CPU-runnable configuration: SC L=16, T=0.5, J=1, bulk D=0.3, B=0.1,
    K=0, fresh uniform unit-vector proposals, 1000 thermalisation + 5000 measurement sweeps
    with E, |M| and Q (middle slice) sampled every `c1_every` sweeps.  At T=0.5 single chains
    freeze into different metastable skyrmion states, so the comparison is between ensembles
    of independent chains from uniform random spins: GPU (c1_gpu_chains replicas of one mesh,
    FP32 sweeps) and the FP64 CPU restatement of the reference's sweep (oracle, c1_cpu_chains
    chains).  Per chain: time averages of E/N, |M|, Q, C_v and chi; the ensemble means are
    compared within 2 standard errors of the mean over chains."""
    import numpy as np
    import torch

    import ising_b200 as ib
    from ising_b200 import _lib
    from oracle import oracle as O

    L, beta, n_th, n_me, every = 16, 2.0, args.c1_therm, args.c1_meas, args.c1_every
    N = L ** 3
    R, RC = args.c1_gpu_chains, args.c1_cpu_chains
    mesh = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    stream = torch.cuda.current_stream()
    mesh.set_stream(stream.cuda_stream)
    mesh.init_uniform(0x15196)
    p = ib.params(J=-1.0, Dz=0.3, B=0.1, dmi="bulk", include_Jp=False)
    pt = ib.ParallelTempering(mesh, np.full(R, beta), p, seed=0x15196, move=_lib.MOVE_UNIFORM)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pt.relax(n_th)
    e1.record(stream)
    torch.cuda.synchronize()
    t_gpu = e0.elapsed_time(e1) / 1e3
    gs = {"E": [], "M": [], "Q": []}
    q = C.c_double()
    for it in range(n_me // every):
        pt.relax(every)
        e, m = pt.energies()
        gs["E"].append(e / N)
        gs["M"].append(np.linalg.norm(m, axis=1) / N)
        qq = []
        for r in range(R):
            _lib.call("ising_winding_number", mesh.handle, r, L // 2, C.byref(q))
            qq.append(q.value)
        gs["Q"].append(np.array(qq))
    g = {k: np.array(v).T for k, v in gs.items()}             # [chain][sample]

    O.build()
    op = O.Params(J=-1.0, Dz=0.3, B=0.1, dmi_bulk=True)
    col = O.checkerboard(L, L, L)
    cs = {"E": [], "M": [], "Q": []}
    t_cpu = 0.0
    for ch in range(RC):
        om = O.Mesh.sc(L)
        om.init_uniform(0x15196 + 1 + ch)
        key = O.SweepKey(seed=0x5EED + ch, ensemble=0, replica=0, move=0, r=0.0, philox_rounds=10)
        E, M, Q = [], [], []
        for sw in range(n_th + n_me):
            ts = time.perf_counter()
            om.colour_pass(col, 0, sw, beta, op, key)
            om.colour_pass(col, 1, sw, beta, op, key)
            t_cpu += time.perf_counter() - ts
            if sw >= n_th and (sw - n_th + 1) % every == 0:
                E.append(om.canonical_energy(op) / N)
                M.append(float(np.linalg.norm(om.spins.sum(axis=0))) / N)
                Q.append(om.winding_number(L // 2))
        cs["E"].append(E); cs["M"].append(M); cs["Q"].append(Q)
    c = {k: np.array(v) for k, v in cs.items()}

    def per_chain(x):
        return {"E": x["E"].mean(1), "M": x["M"].mean(1), "Q": x["Q"].mean(1),
                "C_v": beta * beta * N * x["E"].var(1), "chi": beta * N * x["M"].var(1)}

    pg, pc = per_chain(g), per_chain(c)
    obs = {}
    for name in ("E", "M", "Q", "C_v", "chi"):
        a, b = pg[name], pc[name]
        err = float(np.hypot(a.std(ddof=1) / np.sqrt(len(a)), b.std(ddof=1) / np.sqrt(len(b))))
        obs[name] = {"gpu": float(a.mean()), "cpu": float(b.mean()), "err": err,
                     "within_2sigma": bool(abs(a.mean() - b.mean()) <= 2 * err + 1e-12)}
    value = n_th * N * R / t_gpu
    cpu_rate = (n_th + n_me) * N * RC / t_cpu
    line = {
        "metric": "spin-updates/s", "value": value, "unit": "spin-updates/s", "n_gpus": 1, "steps": n_th,
        "warmup": 0, "ms_per_step": 1e3 * t_gpu / n_th, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (uniform random initial spins)",
        "config": {"workload": "c1", "desc": "SC L=16, T=0.5, J=1, bulk D=0.3, B=0.1, uniform unit-vector moves, "
                   "1000 + 5000 sweeps", "gpu_chains": R, "cpu_chains": RC, "sample_every": every,
                   "note": "value = GPU sweeps of all chains during thermalisation (launch-bound size)"},
        "observables_vs_cpu_reference": obs,
        "all_within_2sigma": all(v["within_2sigma"] for v in obs.values()),
        "cpu_baseline": {"value": cpu_rate, "unit": "spin-updates/s", "cores": 1, "kind": "port",
                         "sample": f"{RC} chains x {n_th + n_me} colour-class sweeps of SC L=16 in FP64 (oracle)"},
        "roofline": None, "e2e": None, "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)
    pt.close()
    mesh.close()


# ---------------------------------------------------------------- patch-step timing
def run_patch_probe(args, w):
    """Times learned patch steps (one colour class on every replica) on an SC PT object of
    the C5 Hamiltonian; --L / --replicas shrink it for profiling."""
    import numpy as np
    import torch

    import ising_b200 as ib

    L, R = args.L or w["L"], args.replicas or w["R"]
    mesh = ib.ChainMesh.simple_cubic(L, n_replicas=R)
    mesh.init_uniform(0x15196, 0)
    p = ib.params(J=w["J"], Dz=w["D"], B=w["B"], dmi="bulk", include_Jp=False)
    pt = ib.ParallelTempering(mesh, 1.0 / ib.temperature_ladder(w["tmin"], w["tmax"], R), p, seed=1)
    net = ib.ProposalNet(max_batch=min(args.c5_batch, pt.patch_count()), seed=1)
    pt.patch_set_scale(np.full(R, 0.3, np.float32), 0.25)
    pt.patch_step(net, 0, (0, 0, 0))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    n = max(1, args.steps)
    for i in range(n):
        pt.patch_step(net, i % 8, (i % 4, 0, 0))
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / n
    print(json.dumps({"metric": "patch-step time", "value": dt * 1e3, "unit": "ms", "windows": pt.patch_count(),
                      "L": L, "replicas": R, "steps": n}), flush=True)
    net.close()
    pt.close()
    mesh.close()


# ---------------------------------------------------------------- C5: learned vs plain
def _jackknife_var_obs(x, beta, N, kind, n_blocks=20):
    """Blocked jackknife error of C_v = beta^2 N var(e) (kind 'cv', x = E/N) or
    chi = beta N var(|m|) (kind 'chi', x = |M|/N) over one time series."""
    import numpy as np
    x = np.asarray(x, dtype=np.float64)
    f = (beta * beta * N) if kind == "cv" else (beta * N)
    nb = min(n_blocks, len(x) // 2)
    if nb < 2:
        return f * x.var(), 0.0
    b = len(x) // nb
    x = x[: nb * b]
    full = f * x.var()
    reps = np.array([f * np.delete(x.reshape(nb, b), i, axis=0).ravel().var() for i in range(nb)])
    return full, float(np.sqrt((nb - 1) / nb * ((reps - reps.mean()) ** 2).sum()))


def compare_arms(a, b, betas, N):
    """Per temperature slot: E/N, |M|/N, Q, C_v, chi of two recorded series [slot][sample][E,|M|,Qmid,Qmean]
    (E total) with binning (mean) and blocked jackknife (C_v, chi) errors; counts of slots
    within 2 combined standard errors.  A slot whose Q is frozen in both series agrees only
    when the two frozen values are equal.  A slot counts as resolved for an observable when both
    series are at least 50 tau_int long (tau of E for C_v, of |M| for chi)."""
    import numpy as np
    from ising_b200 import analysis as A
    R = a.shape[0]
    per = {k: [] for k in ("E", "absM", "Q", "C_v", "chi")}
    resolved = {k: [] for k in per}
    detail = {k: [] for k in ("E", "absM", "Q")}   # [slot, mean a, mean b, 2-sigma bar, tau a, tau b]
    for t in range(R):
        taus = {}
        for name, col in (("E", 0), ("absM", 1), ("Q", 3)):
            xa, xb = a[t, :, col], b[t, :, col]
            if col == 0:
                xa, xb = xa / N, xb / N
            err = float(np.hypot(A.binning_error(xa), A.binning_error(xb)))
            d = float(abs(xa.mean() - xb.mean()))
            # Q of a texture-free slot is zero up to the rounding of the slice sums (~1e-10)
            per[name].append(d <= 2 * err + (1e-8 if name == "Q" else 1e-12))
            # an error bar means something only for series much longer than their tau_int
            ta, tb = A.tau_int(xa), A.tau_int(xb)
            taus[name] = max(ta, tb)
            resolved[name].append(min(len(xa), len(xb)) >= 50 * taus[name])
            if not per[name][-1]:
                detail[name].append([t, float(f"{xa.mean():.6g}"), float(f"{xb.mean():.6g}"),
                                     float(f"{2 * err:.3g}"), round(float(ta), 1), round(float(tb), 1)])
        for name, col, kind in (("C_v", 0, "cv"), ("chi", 1, "chi")):
            xa, xb = a[t, :, col], b[t, :, col]
            if col == 0:
                xa, xb = xa / N, xb / N
            va, ea = _jackknife_var_obs(xa, betas[t], N, kind)
            vb, eb = _jackknife_var_obs(xb, betas[t], N, kind)
            per[name].append(abs(va - vb) <= 2 * float(np.hypot(ea, eb)) + 1e-12)
            resolved[name].append(resolved["E" if col == 0 else "absM"][-1])
    within = {k: int(sum(v)) for k, v in per.items()}
    res = {k: {"resolved_slots": int(sum(resolved[k])),
               "within_2sigma_of_resolved": int(sum(1 for t in range(R) if resolved[k][t] and per[k][t]))}
           for k in per}
    for k in ("E", "absM", "Q"):
        res[k]["detail_outside"] = detail[k]
    return within, {k: [t for t in range(R) if not v[t]] for k, v in per.items()}, res


def learned_vs_plain(args, w):
    """Learned patch proposal against plain Metropolis on the C5 ensemble (SC L=96, 48 PT
    replicas, one exchange per sweep): thermalise one chain with plain sweeps, train the
    network on its windows, tune the patch step scales; then copy the state into a second
    mesh and run the two samplers as independent chains from that common state, in
    alternating segments: the plain arm (plain sweeps) and the learned arm (a plain sweep
    then one colour class of patch moves per step).  Reports tau_int and effective samples
    per second of Q and E per arm, and the per-slot agreement of E, |M|, Q, C_v and chi."""
    import numpy as np
    import torch

    import ising_b200 as ib
    from ising_b200 import _lib
    from ising_b200 import analysis as A

    L, R = w["L"], w["R"]
    N = L ** 3
    n_plain, n_learned = args.c5_plain, args.c5_learned
    stream = torch.cuda.current_stream()
    p = ib.params(J=w["J"], Dz=w["D"], B=w["B"], K=w["K"], dmi="bulk", include_Jp=False)
    betas = 1.0 / ib.temperature_ladder(w["tmin"], w["tmax"], R)
    meshes, pts = [], []
    for arm in range(2):
        m = ib.ChainMesh.simple_cubic(L, n_replicas=R)
        m.set_stream(stream.cuda_stream)
        m.init_uniform(0x15196 + 1000 * args.c5_seed, ensemble=arm)
        meshes.append(m)
        pts.append(ib.ParallelTempering(m, betas, p, seed=0x15196 + arm + 1000 * args.c5_seed, ensemble=arm,
                                        move=_lib.MOVE_BALL,
                                        r=w["r"], record=True, record_capacity=max(n_plain, n_learned) + 8))
    plain, learned = pts

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        t0 = time.perf_counter()
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3) / 1e3

    t_therm = timed(lambda: plain.relax(args.c5_therm))
    rng = np.random.default_rng(7 + args.c5_seed)
    net = ib.ProposalNet(max_batch=args.c5_batch, seed=1 + args.c5_seed)

    def jump_stats(steps=8):
        """per slot: acceptance and squared spin displacement per site per proposal (ESJD)"""
        p0, a0 = plain.patch_stats()
        j0 = plain.patch_jump()
        for i in range(steps):
            plain.patch_step(net, i % 8, tuple(int(v) for v in rng.integers(0, 8, 3)))
        p1, a1 = plain.patch_stats()
        j1 = plain.patch_jump()
        n = np.maximum(p1 - p0, 1).astype(float)
        return (a1 - a0) / n, (j1 - j0) / n / 64.0

    # the network as initialised (mu ~ 0, sigma = 0.3 everywhere) with its own tuned step scale
    plain.patch_tune_scale(net, target=0.25, iters=args.c5_tune, seed=1, drift=1.0)
    acc_untrained, esjd_untrained = jump_stats()
    # training set: windows of plain-PT states, targets from local equilibration of the patch
    ws, ts = [], []
    n_have = 0
    while n_have < args.c5_train:
        plain.relax(20)
        wi, ti = plain.patch_samples(int(rng.integers(0, 8)), tuple(int(v) for v in rng.integers(0, 8, 3)),
                                     n_local=args.c5_nlocal)
        ws.append(wi)
        ts.append(ti)
        n_have += wi.shape[0]
    W = torch.cat(ws)[: args.c5_train]
    T = torch.cat(ts)[: args.c5_train]
    del ws, ts
    losses = []

    def train():
        bs = 512
        for ep in range(args.c5_epochs):
            perm = torch.randperm(W.shape[0], device=W.device)
            for b0 in range(0, W.shape[0] - bs + 1, bs):
                j = perm[b0:b0 + bs]
                losses.append(net.train_step(W[j], T[j], lr=1e-3))

    t_train = timed(train)
    del W, T
    # the trained network at three drift weights, each with its own tuned step scale; the
    # learned arm uses the one with the largest mean ESJD
    trained = {}
    for lam in (0.0, 0.25, 1.0):
        sc = plain.patch_tune_scale(net, target=0.25, iters=args.c5_tune, seed=2, drift=lam)
        acc, ej = jump_stats()
        trained[lam] = (sc, acc, ej)
    best_lam = max(trained, key=lambda l: float(np.mean(trained[l][2])))
    scale_trained, acc_trained, esjd_trained = trained[best_lam]
    learned.patch_set_scale(scale_trained, best_lam)
    plain.relax(200)
    # the common starting state: slot t of the plain chain -> replica t of the learned mesh
    t2r = plain.permutation()
    for t in range(R):
        meshes[1].set_spins(meshes[0].get_spins(int(t2r[t])), t)
    learned.resync()
    # alternating segments; both arms record every sweep
    seg = max(1, min(500, n_plain, n_learned))
    t_plain = t_learned = 0.0
    done_p = done_l = 0
    step = [0]

    def learned_steps(n):
        for _ in range(n):
            learned.run(1, 1)
            learned.patch_step(net, step[0] % 8, tuple(int(v) for v in rng.integers(0, 8, 3)), slots=args.c5_slots)
            step[0] += 1

    while done_p < n_plain or done_l < n_learned:
        if done_p < n_plain:
            n = min(seg, n_plain - done_p)
            t_plain += timed(lambda: plain.run(1, n))
            done_p += n
        if done_l < n_learned:
            n = min(seg, n_learned - done_l)
            t_learned += timed(lambda: learned_steps(n))
            done_l += n
    sp, sl = plain.series(), learned.series()
    # the running FP64 accumulators of both arms against a device recomputation of E and M
    acc_check = {}
    for name, q, m in (("plain", plain, meshes[0]), ("learned", learned, meshes[1])):
        e_run, m_run = q.energies()
        e_dev, m_dev = ib.observables(m, p)
        acc_check[name] = {"max_abs_dE_per_site": float(np.max(np.abs(e_run - e_dev)) / N),
                           "max_abs_dM_per_site": float(np.max(np.abs(m_run - m_dev)) / N)}
    # the samplers' own cost per step, without the per-sweep recording of E, |M| and the
    # winding numbers (measurement overhead shared by both arms): relax sweeps record nothing
    c_plain = timed(lambda: plain.relax(100)) / 100
    c_patch = timed(lambda: [plain.patch_step(net, i % 8, tuple(int(v) for v in rng.integers(0, 8, 3)),
                                              slots=args.c5_slots) for i in range(40)]) / 40

    def arm(x, secs, cost):
        out = []
        for t in range(R):
            q, e = x[t, :, 3], x[t, :, 0]
            tq, te = A.tau_int(q), A.tau_int(e)
            out.append({"tau_Q": tq, "tau_E": te, "ess_Q_per_s": len(q) / (2 * tq) / secs,
                        "ess_E_per_s": len(e) / (2 * te) / secs, "ess_Q_per_sampler_s": 1.0 / (2 * tq * cost),
                        "q_var": float(np.var(q))})
        return out

    ap, al = arm(sp, t_plain, c_plain), arm(sl, t_learned, c_plain + c_patch)
    live = [t for t in range(R) if ap[t]["q_var"] > 1e-12 and al[t]["q_var"] > 1e-12]
    qp = float(np.mean([ap[t]["ess_Q_per_s"] for t in live])) if live else 0.0
    ql = float(np.mean([al[t]["ess_Q_per_s"] for t in live])) if live else 0.0
    qp_s = float(np.mean([ap[t]["ess_Q_per_sampler_s"] for t in live])) if live else 0.0
    ql_s = float(np.mean([al[t]["ess_Q_per_sampler_s"] for t in live])) if live else 0.0
    ratios = [al[t]["ess_Q_per_s"] / ap[t]["ess_Q_per_s"] for t in live if ap[t]["ess_Q_per_s"] > 0]
    within, outside, resolved = compare_arms(sp, sl, betas, N)
    reliable = {"plain": sum(1 for t in live if n_plain >= 50 * ap[t]["tau_Q"]),
                "learned": sum(1 for t in live if n_learned >= 50 * al[t]["tau_Q"]), "of": len(live)}
    q_ess = {
        "metric": "Q-ESS/s (mean over the temperature slots where Q fluctuates in both arms)",
        "plain": qp, "learned": ql, "learned_over_plain": ql / qp if qp > 0 else None,
        "per_sampler_second": {"plain": qp_s, "learned": ql_s, "learned_over_plain": ql_s / qp_s if qp_s > 0 else None,
                               "plain_sweep_s": c_plain, "patch_step_s": c_patch,
                               "note": "cost per step without the per-sweep recording of E, |M| and Q"},
        "learned_over_plain_per_slot": {"median": float(np.median(ratios)) if ratios else None,
                                        "slots_learned_better": sum(1 for r in ratios if r > 1.0),
                                        "of": len(ratios)},
        "slots_used": live, "slots_with_N_ge_50_tauQ": reliable,
        "plain_sweeps": n_plain, "learned_steps": n_learned, "plain_s": t_plain, "learned_s": t_learned,
        "tau_Q_plain": [round(x["tau_Q"], 2) for x in ap], "tau_Q_learned": [round(x["tau_Q"], 2) for x in al],
        "E_ess_per_s": {"plain": float(np.mean([x["ess_E_per_s"] for x in ap])),
                        "learned": float(np.mean([x["ess_E_per_s"] for x in al]))},
        "observables_within_2sigma": {"slots": R, **within, "outside": outside,
                                      "resolved": resolved,
                                      "design": "two independent chains from one thermalised state, "
                                                "binning errors (means) and blocked jackknife (C_v, chi)"},
        "exchange_every": 1, "thermalisation_sweeps": args.c5_therm, "thermalisation_s": t_therm,
        "accumulators_vs_recomputed": acc_check,
    }
    training = {"seconds": t_train, "steps": len(losses), "windows": args.c5_train, "epochs": args.c5_epochs,
                "loss_first": losses[0] if losses else None, "loss_last": losses[-1] if losses else None,
                "untrained": {"acceptance_mean": float(np.mean(acc_untrained)),
                              "esjd_mean": float(np.mean(esjd_untrained))},
                "trained": {str(l): {"acceptance_mean": float(np.mean(v[1])), "esjd_mean": float(np.mean(v[2]))}
                            for l, v in trained.items()},
                "drift_used": best_lam, "n_local": args.c5_nlocal,
                "esjd_trained_over_untrained_mean": float(np.mean(esjd_trained) / max(np.mean(esjd_untrained), 1e-30))}
    net.close()
    for q in pts:
        q.close()
    for m in meshes:
        m.close()
    return q_ess, training


def run_c5(args, w):
    """--learned: the learned-vs-plain comparison on its own, as one JSON line."""
    q_ess, training = learned_vs_plain(args, w)
    line = {"metric": "Q-ESS/s", "value": q_ess["learned"], "unit": "effective Q samples/s", "n_gpus": 1,
            "higher_is_better": True, "vs_baseline": None, "dtype": "f32 (network bf16)",
            "data": "synthetic (uniform random initial spins from Philox, seed 0x15196)",
            "config": {"workload": "c5", "desc": w["desc"], "L": w["L"], "replicas": w["R"]},
            "q_ess": q_ess, "training": training}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c5", choices=sorted(WORKLOADS))
    ap.add_argument("--L", type=int, default=0, help="override lattice size (profiling)")
    ap.add_argument("--replicas", type=int, default=0, help="override replica count (profiling)")
    ap.add_argument("--engine", default="ensembles", choices=["ensembles", "pt"])
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--schedule", default="", help="engine schedule 'threads,chunk_pairs,loader' (no autotuner)")
    ap.add_argument("--l2-group", type=int, default=0, help="--engine pt: replicas per sweep group (0 = auto)")
    ap.add_argument("--sweep-kernel", type=int, default=0,
                    help="--engine pt: 0 auto; checkerboard 1 register / 2 TMA; octant 3 persistent engine")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--learned", action="store_true", help="c5: learned patch proposal vs plain Metropolis")
    ap.add_argument("--patch-probe", action="store_true", help="time learned patch steps (C5 Hamiltonian)")
    ap.add_argument("--c1-therm", type=int, default=1000)
    ap.add_argument("--c1-meas", type=int, default=5000)
    ap.add_argument("--c1-every", type=int, default=10)
    ap.add_argument("--c1-gpu-chains", type=int, default=32)
    ap.add_argument("--c1-cpu-chains", type=int, default=8)
    ap.add_argument("--c5-plain", type=int, default=3000)
    ap.add_argument("--c5-learned", type=int, default=3000,
                    help="learned steps; equal to --c5-plain so both tau estimates see chains of one length")
    ap.add_argument("--c5-therm", type=int, default=20000)
    ap.add_argument("--c5-tune", type=int, default=10)
    ap.add_argument("--c5-nlocal", type=int, default=20)
    ap.add_argument("--c5-train", type=int, default=100000)
    ap.add_argument("--c5-epochs", type=int, default=3)
    ap.add_argument("--c5-batch", type=int, default=8192)
    ap.add_argument("--c5-slots", type=int, default=0)
    ap.add_argument("--c5-seed", type=int, default=0, help="c5 comparison: offset of every seed (independent repeats)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="c5: skip the learned-vs-plain q_ess block")
    ap.add_argument("--resync-every", type=int, default=10,
                    help="engine rounds between FP64 accumulator resyncs inside the timed region (0 = none)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w)
    elif args.patch_probe:
        run_patch_probe(args, WORKLOADS["c5"])
    elif args.learned:
        run_c5(args, WORKLOADS["c5"])
    elif args.workload == "c1":
        run_c1(args)
    elif args.workload == "stats":
        run_stats(args, w)
    elif args.workload == "setup":
        run_setup(args, w)
    elif args.workload == "demag":
        run_demag(args, w)
    else:
        run_gpu(args, w)


if __name__ == "__main__":
    main()
