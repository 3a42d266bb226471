"""The distributed ket on one GPU: G = 2 and 4 ranks as threads of one process
(ThreadComm), each with its own context and its share of the ket resident in HBM, run a
seeded circuit through the library's gate kernels; half-state exchanges are device copies
after a host barrier (no kernel waits on another rank). The gathered ket matches the
full-state oracle within 1e-12 (complex128) / 2e-5 (complex64)."""
import threading

import numpy as np
import pytest

from tests.dist_helpers import oracle_run, random_program, run_program, start_ket

pytestmark = pytest.mark.gpu


def _run(world, n, seed, prec):
    import qpp_b200 as qb
    from qpp_b200.distributed import DistributedKet, GpuLocal, ThreadComm, ThreadHub
    hub = ThreadHub(world, timeout=120)
    g = world.bit_length() - 1
    psi = start_ket(n, seed)
    prog = random_program(n, seed + 1)
    res, errs = {}, []

    def rank_main(r):
        try:
            ctx = qb.Context(0)
            dk = DistributedKet(n, ThreadComm(hub, r), GpuLocal(ctx, n - g, prec))
            dk.scatter_from(psi)
            run_program(dk, prog)
            res[f"norm{r}"] = dk.norm2()
            res[f"ex{r}"] = dk.exchanges
            got = dk.gather_numpy(0)
            if r == 0:
                res["got"] = got
            dk.local.free()
            ctx.close()
        except BaseException as e:  # surfaced in the main thread
            errs.append(e)
            hub.bar.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    return res, oracle_run(psi, n, prog)


@pytest.mark.parametrize("world,n", [(2, 10), (4, 12)])
def test_distributed_ket_threads_c128(world, n):
    import qpp_b200 as qb
    res, ref = _run(world, n, 3 * world + n, qb.C128)
    err = float(np.max(np.abs(res["got"] - ref)) / np.max(np.abs(ref)))
    assert err < 1e-12, err
    assert all(abs(res[f"norm{r}"] - 1.0) < 1e-12 for r in range(world))
    assert all(res[f"ex{r}"] > 0 for r in range(world))


def test_distributed_ket_threads_c64():
    import qpp_b200 as qb
    res, ref = _run(2, 11, 5, qb.C64)
    err = float(np.max(np.abs(res["got"] - ref)) / np.max(np.abs(ref)))
    assert err < 2e-5, err
