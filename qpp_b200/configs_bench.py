"""Measurements of the other benchmark configurations (one GPU).

  config1  20-qubit Gaussian ket (16 MiB, L2-resident), 1000 Haar gates
           (70% 1-qubit, 30% 2-qubit on ordered pairs) then 100 applyCTRL
           with 1-3 controls; complex128, one pass per gate.
  config2  12-qubit density matrix (4096 x 4096, rank 64), 200 steps of
           {16-operator pair channel, ptrace over 6, ptranspose over 6,
           syspermute}; plus the mixed-dimension variant dims
           [3,3,2,2,3,2,2,3] with Haar 3x3 / 6x6 gates; complex128.
  config4  2048 kets of 10-22 qubits and 512 density matrices of 6-11
           qubits (rank 8), each with its own depth-20 layered circuit
           (density matrices: depolarising p=0.005 on every qubit after each
           layer), complex64: one CUDA-graph launch versus the plain loop of
           per-instance launches (and that loop in complex128).

  qft      QCircuit::QFT on n qubits executed by QEngine, as the reference's
           benchmarks/src/qft_bench.cpp and tfq_bench.cpp time it (engine
           reset, then execute); n = 20, 26, 30 in complex128 and n = 30 in
           complex64, against the same circuit run gate by gate (one pass per
           qpp gate) on the GPU.

Device times are CUDA events on the library's stream. Everything here runs
on the GPU through the library; the CPU baselines and the oracle checks of
these configurations are bench.py's (the oracle is test infrastructure).
Each function returns its JSON record and, where bench.py checks the result
against the oracle, the inputs and outputs it needs.
"""
from __future__ import annotations

import json
import math
import os
import sys
import time

import numpy as np

from . import (C64, C128, FUSED, KET, PLAIN, RHO, Circuit, Context, Engine, State,
               batch_last_phases, traj_fusion_width,
               run_batch, traj_tile_width)
from .workloads import haar_unitary, ket_gate_sequence


def _events(torch, stream):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return a, b


def _frac(gbps, peak):
    return None if not peak else gbps / peak


def config1(ctx, torch, stream, peak=None):
    """20-qubit Gaussian ket (seed 1), 1000 Haar gates + 100 applyCTRL, complex128.
    Returns (record, sequence, final states of the circuit and fused forms as
    numpy, keyed "circuit" and "fused")."""
    n = 20
    seq = ket_gate_sequence(n, seed=1)
    D = 2 ** n
    byts = sum(2 * 16 * D // (2 ** len(c)) for U, c, t in seq)
    s = State(ctx, KET, [2] * n, C128).fill_gaussian(1)
    for U, c, t in seq[:50]:  # warm-up
        s.apply_ctrl(U, c, t) if c else s.apply(U, t)
    a, b = _events(torch, stream)
    a.record(stream)
    for U, c, t in seq:
        s.apply_ctrl(U, c, t) if c else s.apply(U, t)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    out = {"workload": "20-qubit Gaussian ket (2^20 complex128, 16 MiB: L2-resident), 1000 Haar "
                       "gates (70% 1-qubit, 30% 2-qubit) then 100 applyCTRL with 1-3 controls",
           "gates": len(seq), "algorithmic_bytes": byts,
           "per_call": {"ms": ms, "gates_per_s": len(seq) / (ms / 1e3),
                        "GBps": byts / (ms / 1e3) / 1e9, "form": "one State.apply per gate"}}
    # the same gates as one circuit: one C call, the host loop in C++
    c = Circuit(n)
    for U, cs, t in seq:
        c.CTRL(U, cs, t) if cs else c.gate(U, t)
    c.run(s, PLAIN)  # warm-up
    times = []
    for _ in range(5):
        s.fill_gaussian(1)
        a, b = _events(torch, stream)
        a.record(stream)
        c.run(s, PLAIN)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ms2 = float(np.median(times))
    gbps = byts / (ms2 / 1e3) / 1e9
    out["circuit"] = {"ms": ms2, "gates_per_s": len(seq) / (ms2 / 1e3), "GBps": gbps,
                      "form": "qgpu_run_gates, plain complex128", "runs": len(times)}
    out["roofline"] = {"bound": "hbm", "achieved": gbps, "peak": peak, "unit": "GB/s",
                       "frac": _frac(gbps, peak),
                       "note": "algorithmic bytes over the measured HBM copy bandwidth; the "
                               "16 MiB state stays in the 126 MB L2, so the fraction can exceed 1"}
    finals = {"circuit": s.numpy()}
    # the fused form: the gates merged into blocks of <= 2 qubits (a 1-qubit
    # gate folded into a neighbouring block), list-scheduled into tile passes
    c.run(s, FUSED)  # warm-up: builds the plan
    times = []
    for _ in range(5):
        s.fill_gaussian(1)
        a, b = _events(torch, stream)
        a.record(stream)
        c.run(s, FUSED)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ms3 = float(np.median(times))
    out["fused"] = {"ms": ms3, "gates_per_s": len(seq) / (ms3 / 1e3),
                    "plan_entries": c.fused_passes(2), "runs": len(times),
                    "form": "qgpu_run_gates, fused complex128: gates merged into blocks of "
                            "<= 2 qubits (controlled gates with more controls as they are), "
                            "list-scheduled into tile passes"}
    finals["fused"] = s.numpy()
    s.free()
    return out, seq, finals


def qft(ctx, torch, stream, sizes=(20, 26, 30)):
    """QCircuit::QFT / TFQ on every qubit, QEngine reset + execute per
    iteration (benchmarks/src/qft_bench.cpp, tfq_bench.cpp). The engine runs
    the QFT block as ceil(n / 8) shared-memory passes; the bytes per
    iteration are that many reads and writes of the state."""
    rows = []
    for n in sizes:
        for prec, eb in ((C128, 16), (C64, 8)):
            if prec == C64 and n != max(sizes):
                continue
            for inverse in (False, True):
                c = Circuit(n)
                c.TFQ() if inverse else c.QFT()
                e = Engine(ctx, c, KET, prec)
                e.reset().execute()  # warm-up: state allocation
                ts, tx = [], []
                for _ in range(5):
                    a, m, b = (torch.cuda.Event(enable_timing=True) for _ in range(3))
                    a.record(stream)
                    e.reset()
                    m.record(stream)
                    e.execute()
                    b.record(stream)
                    torch.cuda.synchronize()
                    ts.append(a.elapsed_time(b))
                    tx.append(m.elapsed_time(b))
                ms, mx = float(np.median(ts)), float(np.median(tx))
                passes = -(-n // 8)
                byts = passes * 2 * eb * 2 ** n
                row = {"n": n, "prec": "c128" if prec == C128 else "c64",
                       "op": "TFQ" if inverse else "QFT", "steps": c.steps(),
                       "ms_reset_execute": ms, "ms_execute": mx, "passes": passes,
                       "GBps_execute": byts / (mx / 1e3) / 1e9}
                if n <= 26 and prec == C128:
                    s = State(ctx, KET, [2] * n, C128).fill_gaussian(1)
                    c.run(s, PLAIN)
                    a, b = _events(torch, stream)
                    a.record(stream)
                    c.run(s, PLAIN)
                    b.record(stream)
                    torch.cuda.synchronize()
                    row["gate_by_gate_ms"] = a.elapsed_time(b)
                    s.free()
                del e
                rows.append(row)
    out = {"rows": rows}
    return out


def _inv(p):
    q = [0] * len(p)
    for i, x in enumerate(p):
        q[x] = i
    return q


def config2(ctx, torch, stream, peak=None, steps=200):
    """12-qubit density matrix (rank 64), `steps` x {pair channel, ptrace(6),
    ptranspose(6), syspermute}, complex128, plus the mixed-dimension variant.
    Returns (record, check) where check holds the last step's input matrix, its
    targets and the three subsystem results, for a comparison with the oracle."""
    from .serving import pair_channel
    rng = np.random.default_rng(2)
    n, D = 12, 4096
    W = rng.standard_normal((D, 64)) + 1j * rng.standard_normal((D, 64))
    rho = W @ W.conj().T
    rho /= np.trace(rho).real
    s = State.from_numpy(ctx, rho, [2] * n)
    Ks = pair_channel()
    plan = []
    for _ in range(steps):
        plan.append(([int(x) for x in rng.choice(n, 2, replace=False)],
                     [int(x) for x in rng.choice(n, 6, replace=False)],
                     [int(x) for x in rng.choice(n, 6, replace=False)],
                     [int(x) for x in rng.permutation(n)]))
    t = {"channel": 0.0, "ptrace": 0.0, "ptranspose": 0.0, "syspermute": 0.0}
    check = None
    # the host enqueues the steps ahead of the device (outputs are freed in
    # stream order), as a resident sequence of ops runs; one synchronize at
    # the end, so each event pair brackets the op's device time
    all_ev = []
    a0, b0 = _events(torch, stream)
    for i, (pair, A, T, perm) in enumerate(plan):
        ev = [_events(torch, stream) for _ in range(4)]
        if i == 2:
            a0.record(stream)
        ev[0][0].record(stream)
        s.apply_kraus(Ks, pair)
        ev[0][1].record(stream)
        ev[1][0].record(stream)
        r = s.ptrace(A)
        ev[1][1].record(stream)
        ev[2][0].record(stream)
        p = s.ptranspose(T)
        ev[2][1].record(stream)
        ev[3][0].record(stream)
        s2 = s.syspermute(perm)
        ev[3][1].record(stream)
        if i >= 2:  # first two steps are warm-up
            all_ev.append(ev)
        if i == len(plan) - 1:
            b0.record(stream)
            check = {"dims": [2] * n, "rho": s.numpy(), "ptrace_target": A, "ptrace": r.numpy(),
                     "ptranspose_target": T, "ptranspose": p.numpy(), "perm": perm,
                     "syspermute": s2.numpy()}
        r.free()
        p.free()
        s.free()
        s = s2
    torch.cuda.synchronize()
    for ev in all_ev:
        for k, key in enumerate(t):
            t[key] += ev[k][0].elapsed_time(ev[k][1])
    m = steps - 2
    full = 2 * 16 * D * D
    out = {"workload": "12-qubit density matrix (4096 x 4096 complex128, rank 64); per step a "
                       "16-operator 2-qubit channel, ptrace over 6, ptranspose over 6, syspermute",
           "steps": steps, "ms_per_step": a0.elapsed_time(b0) / m,
           "timing": "ops enqueued ahead of the device, one synchronize at the end; "
                     "per-op CUDA events on the library stream"}
    for key, byts in (("channel", full), ("ptrace", 16 * 64 ** 3 + 16 * 64 * 64),
                      ("ptranspose", full), ("syspermute", full)):
        ms = t[key] / m
        gbps = byts / (ms / 1e3) / 1e9
        out[key] = {"ms": ms, "GBps": gbps, "bytes": byts, "frac": _frac(gbps, peak)}
    out["ptrace"]["note"] = "64 x 64 output: latency-bound, not an HBM figure"
    out["trace_error_after"] = abs(s.trace() - 1)
    s.free()
    # mixed dimensions
    dims = [3, 3, 2, 2, 3, 2, 2, 3]
    Dm = int(np.prod(dims))
    Wm = rng.standard_normal((Dm, 64)) + 1j * rng.standard_normal((Dm, 64))
    rm = Wm @ Wm.conj().T
    rm /= np.trace(rm).real
    sm = State.from_numpy(ctx, rm, dims)
    a, b = _events(torch, stream)
    a.record(stream)
    cur = list(dims)  # dims follow the permutations
    for _ in range(20):
        threes = [q for q in range(8) if cur[q] == 3]
        twos = [q for q in range(8) if cur[q] == 2]
        sm.apply(haar_unitary(rng, 3), [int(rng.choice(threes))])
        sm.apply(haar_unitary(rng, 6), [int(rng.choice(threes)), int(rng.choice(twos))])
        half = [int(x) for x in rng.choice(8, 4, replace=False)]
        sm.ptrace(half).free()
        sm.ptranspose(half).free()
        perm = [int(x) for x in rng.permutation(8)]
        nxt = sm.syspermute(perm)
        cur = [cur[p] for p in perm]
        sm.free()
        sm = nxt
    b.record(stream)
    torch.cuda.synchronize()
    out["mixed_dims"] = {"dims": dims, "steps": 20, "ms_per_step": a.elapsed_time(b) / 20,
                         "trace_error_after": abs(sm.trace() - 1)}
    sm.free()
    return out, check


def _layered(rng, n, depth, rho, bank1, bank2, chan):
    from .serving import c_channel
    c = Circuit(n)
    for _ in range(depth):
        for q in range(n):
            c.gate(bank1[int(rng.integers(len(bank1)))], [q])
        perm = rng.permutation(n)
        for i in range(n // 2):
            c.gate(bank2[int(rng.integers(len(bank2)))], [int(perm[2 * i]), int(perm[2 * i + 1])])
        if rho:
            for q in range(n):
                c_channel(c, chan, [q])
    return c


def _config4_accuracy(ctx, circs, states):
    """The chosen form (complex64, one graph) against the plain complex128 form from the
    same initial states: per ket the infidelity 1 - |<a|b>|^2 / (<a|a><b|b>), per density
    matrix the relative Hilbert-Schmidt distance ||A - B|| / ||B||; on the device (the
    complex64 result widened to complex128)."""
    s64, s128 = states(C64), states(C128)
    run_batch(ctx, circs, s64, FUSED)
    run_batch(ctx, circs, s128, PLAIN)
    ket_inf, rho_err = [], []
    for a64, b in zip(s64, s128):
        a = State(ctx, b.kind, b.dims, C128).convert_from(a64)
        ab, aa, bb = a.inner(b), a.inner(a).real, b.inner(b).real
        if b.kind == KET:
            ket_inf.append(max(0.0, 1.0 - abs(ab) ** 2 / (aa * bb)))
        else:
            rho_err.append(math.sqrt(max(0.0, aa + bb - 2 * ab.real) / bb))
        a.free()
    for s in s64 + s128:
        s.free()
    return {"kets_max_infidelity": max(ket_inf), "kets_median_infidelity": float(np.median(ket_inf)),
            "rho_max_rel_hs_error": max(rho_err),
            "rho_median_rel_hs_error": float(np.median(rho_err)),
            "compared": len(ket_inf) + len(rho_err)}


def config4(ctx, torch, stream, n_kets=2048, n_rho=512, depth=20):
    from .serving import _depol
    rng = np.random.default_rng(4)
    bank1 = [haar_unitary(rng, 2) for _ in range(64)]
    bank2 = [haar_unitary(rng, 4) for _ in range(64)]
    chan = _depol(0.005)
    ns = [int(x) for x in rng.integers(10, 23, size=n_kets)]
    nr = [int(x) for x in rng.integers(6, 12, size=n_rho)]
    circs = [_layered(rng, n, depth, False, bank1, bank2, chan) for n in ns] + \
            [_layered(rng, n, depth, True, bank1, bank2, chan) for n in nr]
    kinds = [KET] * n_kets + [RHO] * n_rho
    sizes = ns + nr

    def states(prec):
        out = []
        for i, (k, n) in enumerate(zip(kinds, sizes)):
            if k == KET:
                s = State(ctx, KET, [2] * n, prec).fill_gaussian(100 + i)
            else:
                # rank 8: W (2^n x 8 Gaussian, unit norm) as a ket over
                # [2]*n + [8]; tracing out the last subsystem gives W W^dagger
                w = State(ctx, KET, [2] * n + [8], prec).fill_gaussian(100 + i)
                s = w.ptrace([n])
                w.free()
            out.append(s)
        return out

    res = {"instances": {"kets": n_kets, "rho": n_rho, "depth": depth,
                         "ket_qubits": "10-22", "rho_qubits": "6-11"}}
    # one instance of every (kind, size) class: the warm-up run that also
    # lets the tile-width autotuner time each register size once
    firsts = {}
    for i, key in enumerate(zip(kinds, sizes)):
        firsts.setdefault(key, i)
    warm = sorted(firsts.values())
    for prec, name in ((C64, "c64"), (C128, "c128")):
        st = states(prec)
        ctx.synchronize()
        forms = (("graph", FUSED), ("plain_loop", PLAIN)) if prec == C64 else (("plain_loop", PLAIN),)
        for label, form in forms:
            t0 = time.perf_counter()
            run_batch(ctx, [circs[i] for i in warm], [st[i] for i in warm], form)  # warm-up
            res.setdefault("warmup_s", {})[f"{name}_{label}"] = time.perf_counter() - t0
            a, b = _events(torch, stream)
            a.record(stream)
            t0 = time.perf_counter()
            k = run_batch(ctx, circs, st, form)
            b.record(stream)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            res[f"{name}_{label}"] = {"s": wall, "device_ms": a.elapsed_time(b),
                                      "instances_per_s": len(circs) / wall,
                                      "graph_kernels": k}
            if label == "graph":
                res[f"{name}_{label}"]["phases"] = batch_last_phases(ctx)
        for s in st:
            s.free()
    res["graph_speedup_vs_plain_c64"] = res["c64_plain_loop"]["s"] / res["c64_graph"]["s"]
    res["accuracy_vs_plain_c128"] = _config4_accuracy(ctx, circs, states)
    # the tuned widths of the register sizes that ran on the tuned paths:
    # shared memory (10-14 bits) and layered tile passes (15-17); from 18
    # bits (kets of 18-22 qubits, density matrices of 9-11) the batch runs
    # block-layered at width 4, and the tuner is not consulted
    res["tile_widths"] = {n: traj_tile_width(ctx, n) for n in range(15, 18)}
    res["fusion_widths"] = {n: traj_fusion_width(ctx, n) for n in range(10, 18)}
    res["block_layered"] = {"register_bits": "18-22", "block_qubits": 4}
    return res


def config4_shard(ctx, torch, stream, dist=None, n_kets=2048, n_rho=512, depth=20):
    """Config 4 split across the ranks of a job by free HBM (sharding.assign on
    the instances' state bytes): every rank builds the same seeded instances,
    keeps its own share and runs it as one graph launch. Returns this rank's
    instance count and device milliseconds, and the job's slowest rank."""
    from .serving import _depol
    from .sharding import instance_bytes, shard_for_rank
    rng = np.random.default_rng(4)
    bank1 = [haar_unitary(rng, 2) for _ in range(64)]
    bank2 = [haar_unitary(rng, 4) for _ in range(64)]
    chan = _depol(0.005)
    ns = [int(x) for x in rng.integers(10, 23, size=n_kets)]
    nr = [int(x) for x in rng.integers(6, 12, size=n_rho)]
    circs = [_layered(rng, n, depth, False, bank1, bank2, chan) for n in ns] + \
            [_layered(rng, n, depth, True, bank1, bank2, chan) for n in nr]
    kinds = [KET] * n_kets + [RHO] * n_rho
    sizes = ns + nr
    nbytes = [instance_bytes(k == KET, n, 8) for k, n in zip(kinds, sizes)]
    free, _ = ctx.mem_info()
    mine = shard_for_rank(nbytes, free, dist)
    st = []
    for i in mine:
        if kinds[i] == KET:
            st.append(State(ctx, KET, [2] * sizes[i], C64).fill_gaussian(100 + i))
        else:
            w = State(ctx, KET, [2] * sizes[i] + [8], C64).fill_gaussian(100 + i)
            st.append(w.ptrace([sizes[i]]))
            w.free()
    my_circs = [circs[i] for i in mine]
    firsts = {}
    for j, i in enumerate(mine):
        firsts.setdefault((kinds[i], sizes[i]), j)
    warm = sorted(firsts.values())
    if warm:
        run_batch(ctx, [my_circs[j] for j in warm], [st[j] for j in warm], FUSED)
    ctx.synchronize()
    if dist is not None and dist.is_initialized():
        dist.barrier()
    a, b = _events(torch, stream)
    a.record(stream)
    if mine:
        run_batch(ctx, my_circs, st, FUSED)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    job_ms = ms
    if dist is not None and dist.is_initialized():
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        job_ms = float(t.item())
    for x in st:
        x.free()
    return {"instances": len(circs), "mine": len(mine),
            "my_state_bytes": int(sum(nbytes[i] for i in mine)), "my_ms": ms, "job_ms": job_ms,
            "instances_per_s": len(circs) / (job_ms / 1e3),
            "placement": "instances by state bytes over the ranks' free HBM (sharding.assign)"}


def main():
    import argparse

    import torch
    ap = argparse.ArgumentParser(description="configs 1, 2 and 4 and the QFT benchmark on one GPU "
                                             "(GPU only; bench.py adds the CPU baselines)")
    ap.add_argument("--only", choices=["config1", "config2", "config4", "qft"], action="append",
                    help="run only these configs (repeatable)")
    ap.add_argument("--no-cpu", action="store_true", help="accepted for compatibility (no-op)")
    ap.add_argument("--steps", type=int, default=200, help="config 2 steps")
    ap.add_argument("--kets", type=int, default=2048, help="config 4 kets")
    ap.add_argument("--rho", type=int, default=512, help="config 4 density matrices")
    ap.add_argument("--depth", type=int, default=20, help="config 4 circuit depth")
    ap.add_argument("--qft-n", type=int, action="append",
                    help="QFT benchmark qubit counts (repeatable; default 20, 26, 30)")
    a = ap.parse_args()
    run = set(a.only or ["config1", "config2", "config4", "qft"])
    ctx = Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream())
    out = {}
    if "config1" in run:
        out["config1"] = config1(ctx, torch, stream)[0]
    if "config2" in run:
        out["config2"] = config2(ctx, torch, stream, steps=max(a.steps, 3))[0]
    if "qft" in run:
        out["qft"] = qft(ctx, torch, stream, sizes=tuple(a.qft_n or (20, 26, 30)))
    if "config4" in run:
        out["config4"] = config4(ctx, torch, stream, n_kets=a.kets, n_rho=a.rho, depth=a.depth)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
