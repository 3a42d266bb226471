#!/usr/bin/env python3
"""Benchmark: gate application on a 30-qubit ket on B200.

Workload (one rank per GPU, each rank its own replica -- weak scaling, no
collective on the data path): a 2^30-amplitude complex128 ket (16 GiB),
i.i.d. complex Gaussian from a seeded Philox stream, normalised; a random
layered circuit of depth 40 (every layer: a Haar 1-qubit gate on each of the
30 qubits, then a Haar 2-qubit gate on each pair of a random perfect
matching: 45 gates, 1800 in all). A "step" is one layer applied in the plain
form: each gate in complex128, in place, one read and one write of the state
per gate (2 * 16 B * 2^30 = 34.36 GB of algorithmic traffic per gate). The
state is 136x the L2, so no flush is needed between iterations.

value   = algorithmic gate bytes of all ranks / max-over-ranks device time
          (CUDA events on the library's stream), GB/s.
e2e     = the same metric through the public C ABI from a pinned host ket:
          upload, the whole depth-40 circuit, download (one e2e step = one
          circuit, so 16 GiB each way per step).
roofline= the dominant kernel (k_qubit_1q, 30 of 45 launches per layer):
          34.36 GB per launch / its mean CUDA-event duration, against the
          measured HBM copy bandwidth.
cpu_baseline = the CPU restatement of qpp's qubit kernels (oracle/, OpenMP on
          all host cores, qpp's copy-per-call semantics) on a bounded sample
          of the same gates on the same 2^30 ket.

--impl reference times that CPU restatement alone (qpp itself needs Eigen,
absent here) on the same metric, one gate per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "30q gate GB/s vs HBM peak; served circuits/s, p50/p99 vs plain, fid≥1-1e-6"
UNIT = "GB/s"
N_QUBITS = 30
DEPTH = 40
SEED = 1234


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--qubits", type=int, default=N_QUBITS)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-fused", action="store_true", help="skip the fused complex64 leg")
    return ap.parse_args()


def fused_leg(args, qb, torch, ctx, stream, psi, layers, n, rank, plain_ms, dist):
    """The fused form on the same depth-40 circuit from the same input: gates
    merged into <= 6-qubit blocks, each block one pass of a complex64 state on
    the tensor cores (tcgen05 kind::tf32, split-TF32 products, FP32
    accumulation). Reports its time, the speed-up over the plain complex128
    circuit time, and the infidelity against the plain complex128 result
    (when the timed plain run covered exactly the circuit)."""
    circ = qb.Circuit(n)
    for lay in layers:
        for U, t in lay:
            circ.gate(U, t)
    passes = circ.fused_passes(6)
    f64 = qb.State(ctx, qb.KET, [2] * n, qb.C64)
    f64.fill_gaussian(SEED + 77)
    circ.run(f64, qb.FUSED)  # warm-up: builds the plan and its device matrices
    src = qb.State(ctx, qb.KET, [2] * n, qb.C128).fill_gaussian(SEED + rank)
    f64.convert_from(src)
    src.free()
    ctx.synchronize()
    if dist:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    circ.run(f64, qb.FUSED)
    b.record(stream)
    torch.cuda.synchronize()
    f_ms = a.elapsed_time(b)
    if dist:
        t = torch.tensor([f_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        f_ms = float(t.item())
    plain_circuit_ms = plain_ms / args.steps * DEPTH
    out = {"form": "complex64 state, gates fused into <= 6-qubit blocks, 64x64 complex blocks on "
                   "tcgen05 (kind::tf32, 3xTF32 split products, FP32 accumulation)",
           "gates": sum(len(lay) for lay in layers), "passes": passes, "ms": f_ms,
           "plain_c128_circuit_ms": plain_circuit_ms,
           "speedup_vs_plain_c128": plain_circuit_ms / f_ms,
           "pass_bytes": 2 * 8 * 2 ** n,
           "pass_GBps": passes * 2 * 8 * 2 ** n / (f_ms / 1e3) / 1e9,
           "gate_GBps_c128_equivalent": sum(len(lay) for lay in layers) * wl_gate_bytes(n)
           / (f_ms / 1e3) / 1e9}
    if args.steps == DEPTH:
        tmp = qb.State(ctx, qb.KET, [2] * n, qb.C128).convert_from(f64)
        ov = psi.inner(tmp)
        fid = abs(ov) ** 2 / (psi.norm2() * tmp.norm2())
        out["infidelity_vs_plain_c128"] = 1.0 - fid
        tmp.free()
    f64.free()
    return out


def wl_gate_bytes(n):
    return 2 * 16 * 2 ** n


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dram_traffic(kernel):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            return json.load(f).get(kernel, {}).get("bytes_per_launch")
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.p = None
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(dev), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def reduce_over_ranks(dist, ms_local, bytes_local, device=None):
    """Replicas: the job time is the slowest rank's device time and the job
    work is the sum of every rank's work. Returns (max ms, total bytes)."""
    if dist is None or not dist.is_initialized():
        return ms_local, bytes_local
    import torch
    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    b = torch.tensor([float(bytes_local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    return float(t.item()), float(b.item())


def cpu_sample_gates(layers, count):
    """The first `count` gates of the circuit in layer order, taking 1q and
    2q gates in the circuit's 2:1 ratio."""
    ones = [g for g in layers[0] if len(g[1]) == 1]
    twos = [g for g in layers[0] if len(g[1]) == 2]
    out = []
    while len(out) < count:
        k = len(out)
        out.append(twos[k // 3] if k % 3 == 2 else ones[k - k // 3])
    return out


def cpu_baseline(n, layers, n_gates):
    """Time the oracle's restatement of qpp's qubit kernels (apply.hpp:57-265:
    full copy of the state, then the OpenMP pair/quad sweep into a fresh
    result) on `n_gates` gates of the circuit on a 2^n ket."""
    from oracle import oracle as orc
    import ctypes as ct
    L = orc.lib()
    D = 2 ** n
    psi = np.empty(D, dtype=np.complex128)
    L.oracle_fill_gaussian(psi.ctypes.data_as(ct.POINTER(ct.c_double)), ct.c_uint64(D),
                           ct.c_uint64(SEED))
    dims = [2] * n
    gates = cpu_sample_gates(layers, n_gates)
    t_total, b_total = 0.0, 0
    for U, t in gates:
        t0 = time.perf_counter()
        out = orc.apply(psi, U, t, dims, path=1)
        t_total += time.perf_counter() - t0
        b_total += 2 * 16 * D
        psi = out
        del out
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": b_total / t_total / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(gates)} gates of layer 0 (1q:2q = 2:1) on the 2^{n} complex128 "
                      f"ket, qpp copy-per-call semantics, {t_total:.2f} s"}


def run_reference(args):
    """--impl reference: the CPU restatement (qpp needs Eigen, absent here)
    on all host cores, one gate of the circuit per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from qpp_b200 import workloads as wl
    from oracle import oracle as orc
    import ctypes as ct
    os.environ.setdefault("OMP_PROC_BIND", "close")
    n = args.qubits
    layers = wl.layered_circuit(n, DEPTH, SEED)
    gates = [g for layer in layers for g in layer]
    L = orc.lib()
    D = 2 ** n
    psi = np.empty(D, dtype=np.complex128)
    L.oracle_fill_gaussian(psi.ctypes.data_as(ct.POINTER(ct.c_double)), ct.c_uint64(D),
                           ct.c_uint64(SEED))
    dims = [2] * n
    times = []
    for i in range(args.warmup + args.steps):
        U, t = gates[i % len(gates)]
        t0 = time.perf_counter()
        psi = orc.apply(psi, U, t, dims, path=1)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    tot = sum(times)
    val = args.steps * 2 * 16 * D / tot / 1e9
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": f"{n}-qubit ket, layered depth-{DEPTH} circuit, plain complex128, "
                               "one gate per step", "qubits": n, "depth": DEPTH},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"one gate of the layered circuit per step on the 2^{n} "
                                   "complex128 ket (qpp restatement, Eigen unavailable)"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import qpp_b200 as qb
    from qpp_b200 import workloads as wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    n = args.qubits
    D = 2 ** n
    gbytes = wl.gate_bytes(n)
    layers = wl.layered_circuit(n, DEPTH, SEED)
    ctx = qb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream())
    psi = qb.State(ctx, qb.KET, [2] * n, qb.C128)
    psi.fill_gaussian(SEED + rank)
    ctx.synchronize()

    def layer(i, events=None):
        for U, t in layers[i % DEPTH]:
            if events is not None:
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                psi.apply(U, t)
                b.record(stream)
                events.append((len(t), a, b))
            else:
                psi.apply(U, t)

    for w in range(args.warmup):
        layer(w)
    # timed steps start from the seeded input at layer 0, so steps == DEPTH
    # runs exactly the depth-40 circuit (the fused form's reference)
    psi.fill_gaussian(SEED + rank)
    ctx.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev = []
    l0 = ctx.launches()
    start.record(stream)
    for s in range(args.steps):
        layer(s, ev)
    end.record(stream)
    torch.cuda.synchronize()
    ctx.synchronize()
    launches = ctx.launches() - l0
    clk = clocks.stop()
    n_gates = sum(len(layers[s % DEPTH]) for s in range(args.steps))
    ms, job_bytes = reduce_over_ranks(dist, start.elapsed_time(end), n_gates * gbytes,
                                      device="cuda")
    if dist:
        dist.barrier()
    value = job_bytes / (ms / 1e3) / 1e9
    d1 = [a.elapsed_time(b) for k, a, b in ev if k == 1]
    d2 = [a.elapsed_time(b) for k, a, b in ev if k == 2]
    peak, peak_kind = peaks()
    ach1 = gbytes / (statistics.mean(d1) / 1e3) / 1e9
    ach2 = gbytes / (statistics.mean(d2) / 1e3) / 1e9
    norm_err = abs(psi.norm2() - 1.0)

    fused = None
    if not args.no_fused:
        fused = fused_leg(args, qb, torch, ctx, stream, psi, layers, n, rank, ms, dist)

    e2e = None
    if not args.no_e2e:
        # public ABI, host -> device -> depth-40 circuit -> host
        host = torch.empty(2 * D, dtype=torch.float64, pin_memory=True)
        lib = qb.lib()
        qb.check(lib.qgpu_state_download(psi.h, qb.vp(host.data_ptr())))
        e2e_ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        if dist:
            dist.barrier()
        e2e_ev[0].record(stream)
        qb.check(lib.qgpu_state_upload(psi.h, qb.vp(host.data_ptr())))
        for i in range(DEPTH):
            layer(i)
        qb.check(lib.qgpu_state_download(psi.h, qb.vp(host.data_ptr())))
        e2e_ev[1].record(stream)
        torch.cuda.synchronize()
        e_ms = e2e_ev[0].elapsed_time(e2e_ev[1])
        if dist:
            t = torch.tensor([e_ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
        e_gates = sum(len(lay) for lay in layers)
        e2e = {"value": world * e_gates * gbytes / (e_ms / 1e3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 16 * D, "d2h_bytes_per_step": 16 * D,
               "ms_per_step": e_ms,
               "step": f"one depth-{DEPTH} circuit ({e_gates} gates) from a pinned host ket: "
                       "qgpu_state_upload, qgpu_apply per gate, qgpu_state_download"}
        del host

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        psi.free()
        cpu = cpu_baseline(n, layers, n_gates=3)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"{n}-qubit ket (2^{n} complex128, {16 * D / 2**30:g} GiB), layered depth-{DEPTH} "
                                   "random circuit, plain form: one in-place pass per gate; "
                                   "step = one layer (30 1q + 15 2q gates)",
                       "qubits": n, "depth": DEPTH, "gates_per_step": len(layers[0]),
                       "parallelism": f"replicas x{world}",
                       "l2": f"state is {16 * D / 2**30:g} GiB, {16 * D / (126 * 2**20):.0f}x the 126 MB L2: no flush needed"},
            "roofline": {"bound": "hbm", "kernel": "k_qubit_1q", "achieved": ach1, "peak": peak,
                         "unit": "GB/s", "frac": ach1 / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": gbytes, "mean_launch_ms": statistics.mean(d1),
                         "launches": len(d1), "traffic": dram_traffic("k_qubit_1q"),
                         "k_qubit_2q": {"achieved": ach2, "frac": ach2 / peak,
                                        "mean_launch_ms": statistics.mean(d2),
                                        "launches": len(d2)}},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "fused": fused,
            "gpu_launches": launches,
            "clocks": clk,
            "check": {"norm_error_after_run": norm_err},
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
