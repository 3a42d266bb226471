"""Serving benchmark: Poisson request streams through the batched server,
against the plain form one request at a time.

    python -m qpp_b200.serve_bench --rates 100,1000,10000 --duration 2

Prints one JSON object: per arrival rate the batched server's completed
circuits/s and p50/p99 latency; the plain form's circuits/s with every request
queued at once (one request at a time on the resident engine, complex128,
one launch per gate); and the ratio of the batched server's saturated
throughput to the plain form's.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import serving as sv


def closed_loop(server, pool, count, seed=11):
    t0 = time.perf_counter()
    ids = [server.submit(r.circuit, r.kind, r.p, r.shots, seed + k)
           for k, r in enumerate(pool[:count])]
    lat = [server.wait(i)[0] for i in ids]
    wall = time.perf_counter() - t0
    return np.array(lat), len(lat), wall


def run(rates, duration, pool_size, plain_requests, seed=2025, device=0, max_per_rate=400):
    pool = sv.request_pool(pool_size, seed=seed)
    out = {"pool": {"requests": pool_size,
                    "ket_fraction": float(np.mean([r.kind == sv.KET for r in pool])),
                    "mean_shots": float(np.mean([r.shots for r in pool])),
                    "qubits": [int(r.n) for r in pool]}}
    srv = sv.Server(device, mode=sv.BATCHED)
    # warm-up: every template once (programs compiled, allocator pools warm)
    closed_loop(srv, pool, len(pool), seed=1)
    sweep = []
    for rate in rates:
        # at most max_per_rate arrivals per point, so an overloaded rate
        # cannot build an unbounded backlog
        lat, done, wall = sv.run_open_loop(srv, pool, rate, duration,
                                           max_requests=max_per_rate)
        sweep.append({"rate_req_s": rate, **sv.summarize(lat, done, wall)})
    lat, done, wall = closed_loop(srv, pool, len(pool))
    batched_sat = sv.summarize(lat, done, wall)
    out["batched"] = {"sweep": sweep, "saturated": batched_sat, "stats": srv.stats()}
    srv.close()
    plain = sv.Server(device, mode=sv.PLAIN)
    lat, done, wall = closed_loop(plain, pool, plain_requests)
    plain_sat = sv.summarize(lat, done, wall)
    out["plain"] = {"saturated": plain_sat, "requests": plain_requests}
    plain.close()
    # the same requests through the batched server, for a like-for-like ratio
    srv = sv.Server(device, mode=sv.BATCHED)
    closed_loop(srv, pool, plain_requests, seed=1)
    lat, done, wall = closed_loop(srv, pool, plain_requests)
    same = sv.summarize(lat, done, wall)
    srv.close()
    out["batched_same_requests"] = same
    out["speedup_circuits_per_s"] = same["circuits_per_s"] / max(plain_sat["circuits_per_s"], 1e-12)
    return out


def sequential(server, pool, count, seed=1000):
    """One request at a time: submit, wait, next. Latency = service time."""
    t0 = time.perf_counter()
    lat = []
    for k, r in enumerate(pool[:count]):
        rid = server.submit(r.circuit, r.kind, r.p, r.shots, seed + k)
        lat.append(server.wait(rid)[0])
    return np.array(lat), count, time.perf_counter() - t0


def measure(rates=(100, 300, 1000), duration=2.0, pool_size=64, same=24, seed=2025, device=0,
            max_per_rate=400):
    """The serving record of the benchmark line: the batched server's open-loop Poisson
    sweep (circuits/s, p50/p99 latency per offered rate) and its saturated throughput;
    then the first `same` requests of every arrival stream (the pool's first templates,
    seeds 1000 + k as in the sweep) through the plain form one request at a time and
    through the batched server, all at once and one at a time."""
    pool = sv.request_pool(pool_size, seed=seed)
    same = min(same, pool_size)
    out = {"workload": "Poisson QNoisyEngine requests: 90% kets of 12-28 qubits (P(n) ~ "
                       "2^-(n-12)), depth 10-60 layered circuits, depolarising p=1e-3 per qubit "
                       "per step by trajectories, shots log-uniform 1-1000, 20% with mid-circuit "
                       "Z measurements; 10% density matrices of 8-13 qubits with 16-operator "
                       f"2-qubit channels; seeded pool of {pool_size} templates",
           "pool": {"requests": pool_size,
                    "ket_fraction": float(np.mean([r.kind == sv.KET for r in pool])),
                    "mean_shots": float(np.mean([r.shots for r in pool])),
                    "max_qubits": int(max(r.n for r in pool))}}
    srv = sv.Server(device, mode=sv.BATCHED)
    closed_loop(srv, pool, len(pool), seed=1)  # warm-up: programs, pools, autotuner
    sweep = []
    for rate in rates:
        lat, done, wall = sv.run_open_loop(srv, pool, rate, duration, max_requests=max_per_rate)
        sweep.append({"rate_req_s": rate, **sv.summarize(lat, done, wall)})
    lat, done, wall = closed_loop(srv, pool, len(pool))
    out["batched"] = {"sweep": sweep, "saturated_all_templates": sv.summarize(lat, done, wall)}
    lat, done, wall = closed_loop(srv, pool, same, seed=1000)
    b_all = sv.summarize(lat, done, wall)
    lat, done, wall = sequential(srv, pool, same)
    b_seq = sv.summarize(lat, done, wall)
    out["batched"]["stats"] = srv.stats()
    srv.close()
    plain = sv.Server(device, mode=sv.PLAIN)
    sequential(plain, pool, 2)  # warm-up
    lat, done, wall = sequential(plain, pool, same)
    p_seq = sv.summarize(lat, done, wall)
    plain.close()
    out["same_requests"] = {
        "requests": same,
        "rho_requests": int(sum(r.kind != sv.KET for r in pool[:same])),
        "plain_one_at_a_time": p_seq,
        "batched_all_at_once": b_all,
        "batched_one_at_a_time": b_seq,
        "speedup_circuits_per_s": b_all["circuits_per_s"] / max(p_seq["circuits_per_s"], 1e-12),
        "plain_form": "resident engine in complex128, one request at a time, one launch per gate"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="100,300,1000,3000,10000,20000")
    ap.add_argument("--duration", type=float, default=2.0)
    ap.add_argument("--pool", type=int, default=64)
    ap.add_argument("--plain-requests", type=int, default=12)
    a = ap.parse_args()
    res = run([float(x) for x in a.rates.split(",")], a.duration, a.pool, a.plain_requests)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
