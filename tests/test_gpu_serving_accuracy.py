"""Accuracy of the serving loop's chosen form against the FP64 oracle.

The ket requests of the serving benchmark's pool that run in shared memory (12-14 qubits,
complex64 trajectories, depolarising p = 1e-3 before every step, some with mid-circuit Z
measurements) run a few shots through the trajectory kernel with their final states, noise
events and outcomes dumped. Each shot is replayed through the oracle in complex128 with the
same Paulis and forced outcomes (qpp's QNoisyEngine semantics, qnoisy_engine.hpp:105-121), and
the infidelity 1 - |<psi_gpu|psi_fp64>|^2 must stay below 1e-6."""
import numpy as np
import pytest

from tests.test_gpu_traj import replay, run_traj

pytestmark = pytest.mark.gpu


def test_serving_pool_shots_against_fp64_oracle(ctx):
    from qpp_b200 import serving as sv
    pool = sv.request_pool(64, seed=2025)
    small = [r for r in pool if r.kind == sv.KET and r.n <= 14][:6]
    assert len(small) >= 3
    infid = []
    for k, r in enumerate(small):
        shots = 2
        _, dits, states, events = run_traj(__import__("qpp_b200"), ctx, r.circuit, r.n, r.p,
                                           shots, seed=31 + k, max_events=256)
        for s in range(shots):
            ref, _ = replay(r.steps, r.n, dits[s], events[s])
            got = states[s]
            f = abs(np.vdot(ref, got)) ** 2 / (np.vdot(ref, ref).real * np.vdot(got, got).real)
            infid.append(1.0 - f)
    worst = max(infid)
    print(f"serving pool: {len(infid)} shots of {len(small)} requests (n = "
          f"{sorted(r.n for r in small)}), infidelity vs FP64 oracle: max {worst:.3g}, "
          f"median {np.median(infid):.3g}")
    assert worst < 1e-6
