"""The distributed ket (qpp_b200/distributed.py) on CPU: 2 and 4 gloo ranks, each holding
its share in host memory, run a seeded circuit whose gates hit global qubits (half-state
exchanges through torch.distributed send/recv) and global controls (no exchange); the
gathered ket matches the full-state oracle within 1e-12."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, seed, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from qpp_b200.distributed import DistributedKet, TorchComm
        from tests.dist_helpers import NumpyLocal, oracle_run, random_program, run_program, start_ket
        comm = TorchComm()
        g = world.bit_length() - 1
        dk = DistributedKet(n, comm, NumpyLocal(n - g))
        psi = start_ket(n, seed)
        dk.scatter_from(psi)
        prog = random_program(n, seed + 1)
        run_program(dk, prog)
        nrm = dk.norm2()
        got = dk.gather_numpy(0)
        if rank == 0:
            ref = oracle_run(psi, n, prog)
            out["err"] = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
            out["norm"] = nrm
        out[f"ex{rank}"] = dk.exchanges
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 6), (4, 7)])
def test_distributed_ket_gloo(world, n):
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, n, 11 * world, out), nprocs=world,
                       start_method="spawn")
    assert out["err"] < 1e-12, out["err"]
    assert abs(out["norm"] - 1.0) < 1e-12
    assert all(out[f"ex{r}"] > 0 for r in range(world))


def test_layout_rules():
    """Global controls of value 0 skip the gate; a non-power-of-two world is refused."""
    from qpp_b200.distributed import DistributedKet, ThreadComm, ThreadHub
    from tests.dist_helpers import NumpyLocal

    with pytest.raises(ValueError):
        DistributedKet(6, ThreadComm(ThreadHub(3), 0), NumpyLocal(4))
    dk = DistributedKet(5, ThreadComm(ThreadHub(2), 0), NumpyLocal(4))  # rank 0: qubit 0 = 0
    dk.local.amps[:] = 1.0
    X = np.array([[0, 1], [1, 0]], dtype=np.complex128) * 2
    dk.apply_ctrl(X, [0], [3])  # control is global and 0 on rank 0: nothing happens
    assert np.all(dk.local.amps == 1.0) and dk.exchanges == 0
