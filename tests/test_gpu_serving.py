"""Serving loop: continuous batching keeps every request's result unchanged.

A request's trajectories draw from Philox streams keyed by its own seed and
shot index, and its state never shares memory with another request, so its
samples and measurement dits must be identical whether it runs alone or in
a mix that arrives while other work is on the GPU (tolerance: exact). The
same holds on the engine path (density matrices), and for requests with many
shots arriving among others (the batching lanes slice requests by shots and
keep two launches in flight). The plain mode serves the same requests one at
a time.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pool():
    from qpp_b200 import serving as sv
    return sv.request_pool(24, seed=31, max_ket_qubits=16, max_rho_qubits=9)


def _ket_request(n, shots=30):
    """A ket request of n qubits (16: the per-CTA global-slot lane)."""
    from qpp_b200 import serving as sv
    from qpp_b200.workloads import haar_unitary
    rng = np.random.default_rng(n)
    c = sv.Circuit(n, 2, 2)
    for layer in range(5):
        for q in range(n):
            c.gate(haar_unitary(rng, 2), [q])
        perm = rng.permutation(n)
        for i in range(n // 2):
            c.gate(haar_unitary(rng, 4), [int(perm[2 * i]), int(perm[2 * i + 1])])
        if layer == 2:
            c.measure([3], 0, destructive=False)
    return sv.Request(c, sv.KET, n, 1e-3, shots, 2)


def _rho_request():
    """A small density-matrix request on the engine path."""
    from qpp_b200 import serving as sv
    from qpp_b200.workloads import haar_unitary
    rng = np.random.default_rng(77)
    c = sv.Circuit(6, 2, 1)
    for layer in range(4):
        for q in range(6):
            c.gate(haar_unitary(rng, 2), [q])
        for a, b in ((0, 3), (1, 4), (2, 5)):
            c.gate(haar_unitary(rng, 4), [a, b])
            sv.c_channel(c, sv.pair_channel(), [a, b])
    return sv.Request(c, sv.RHO, 6, 0.0, 40, 1)


def test_result_same_alone_and_in_mix():
    from qpp_b200 import serving as sv
    pool = _pool()
    probe = [r for r in pool if r.kind == sv.KET and r.n <= 14][:1] + \
        [_ket_request(16)] + [_rho_request()] + [_ket_request(12, shots=900)] + \
        [_ket_request(16, shots=700)]
    srv = sv.Server(0, mode=sv.BATCHED)
    alone = []
    for k, r in enumerate(probe):
        rid = srv.submit(r.circuit, r.kind, r.p, r.shots, seed=500 + k)
        alone.append(srv.wait(rid, r.shots, r.nc))
    # the mix: fillers keep the GPU busy while the probes arrive
    ids = []
    for k, r in enumerate(pool):
        ids.append(("fill", srv.submit(r.circuit, r.kind, r.p, r.shots, seed=9000 + k), r))
        if k in (3, 9, 15, 18, 21):
            j = (3, 9, 15, 18, 21).index(k)
            pr = probe[j]
            ids.append(("probe", srv.submit(pr.circuit, pr.kind, pr.p, pr.shots, seed=500 + j), j))
        time.sleep(0.001)
    got = {}
    for tag, rid, x in ids:
        if tag == "probe":
            got[x] = srv.wait(rid, probe[x].shots, probe[x].nc)
        else:
            lat, s, d = srv.wait(rid, x.shots, x.nc)
            assert np.all(s < 2 ** x.n)
    st = srv.stats()
    srv.close()
    for j in range(len(probe)):
        assert np.array_equal(alone[j][1], got[j][1]), j  # samples
        assert np.array_equal(alone[j][2], got[j][2]), j  # dits
    assert st["batches"] >= 2 and st["trajectories"] > 0


def test_plain_mode_serves_requests():
    from qpp_b200 import serving as sv
    pool = [r for r in _pool() if r.shots <= 20][:3]
    srv = sv.Server(0, mode=sv.PLAIN)
    ids = [srv.submit(r.circuit, r.kind, r.p, r.shots, seed=7 + k) for k, r in enumerate(pool)]
    for rid, r in zip(ids, pool):
        lat, s, d = srv.wait(rid, r.shots, r.nc)
        assert lat > 0 and np.all(s < 2 ** r.n)
    assert srv.stats()["engine_runs"] == len(pool)
    srv.close()


@pytest.mark.parametrize("n", [9, 12])
def test_large_density_matrix_batched_matches_plain_mode(n):
    """Density matrices above 7 qubits of gates and channels only run on the
    engine lane in the fused superoperator form in complex64; their shots
    (samples of the final diagonal, same seed) match the plain mode's
    complex128 engine run in all but a boundary draw or two."""
    from qpp_b200 import serving as sv
    from qpp_b200.workloads import haar_unitary
    rng = np.random.default_rng(900 + n)
    c = sv.Circuit(n, 2, 1)
    for layer in range(3):
        for q in range(n):
            c.gate(haar_unitary(rng, 2), [q])
        perm = rng.permutation(n)
        for i in range(n // 2):
            a, b = int(perm[2 * i]), int(perm[2 * i + 1])
            c.gate(haar_unitary(rng, 4), [a, b])
            sv.c_channel(c, sv.pair_channel(), [a, b])
    shots = 400
    got = []
    for mode in (sv.BATCHED, sv.PLAIN):
        srv = sv.Server(0, mode=mode)
        rid = srv.submit(c, sv.RHO, 0.0, shots, seed=42)
        lat, s, d = srv.wait(rid, shots, 1)
        srv.close()
        assert np.all(s < 2 ** n) and np.all(d == 0)
        got.append(s)
    assert np.sum(got[0] == got[1]) >= shots - 2
