"""qgpu_ptrace_noalloc: the partial trace for callers that cannot allocate
device memory at the time of the call (an application whose memory pool
already owns the GPU's free memory, or a loop that cannot afford the device
synchronisation of cudaMalloc/cudaFree).

The test calls it through the C ABI with a caller-owned output buffer and
compares it with the allocating qgpu_ptrace on the same state, within the
path's complex128 tolerance (1e-12 relative, max-norm), on two calls in a
row with different traced subsystems, so the second call overwrites the
shared offset table left by the first. It also checks the size limit.
This file is collected last on purpose: if it fails, a run that stops at
the first failure has already run every other test.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _noalloc(qb, state, target, out_state):
    t = np.ascontiguousarray(np.asarray(target, dtype=np.uint64))
    rc = qb.lib().qgpu_ptrace_noalloc(state.h, t.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                      ct.c_uint32(len(target)), ct.c_void_p(out_state.device_ptr()))
    qb.check(rc)
    state.ctx.synchronize()
    return out_state.numpy()


@pytest.mark.parametrize("kind", ["rho", "ket"])
def test_noalloc_ptrace_matches_allocating_ptrace_twice(kind):
    import qpp_b200 as qb
    from tests.qpp_helpers import gaussian_ket, random_rho
    ctx = qb.Context(0)
    rng = np.random.default_rng(65536)
    dims = [2, 3, 2, 2, 3, 2, 2]
    D = int(np.prod(dims))
    host = random_rho(rng, D, 6) if kind == "rho" else gaussian_ket(rng, D)
    s = qb.State.from_numpy(ctx, host, dims)
    for target in ([1, 4, 6], [0, 2, 3, 5]):  # two calls in a row
        kept = [dims[q] for q in range(len(dims)) if q not in target]
        out = qb.State(ctx, qb.RHO, kept)  # the caller's own buffer
        got = _noalloc(qb, s, target, out)
        ref = s.ptrace(target).numpy()
        out.free()
        assert _relerr(got, ref) < 1e-12, (target, _relerr(got, ref))
    s.free()
    ctx.close()


def test_noalloc_ptrace_rejects_traced_dimension_above_limit():
    import qpp_b200 as qb
    ctx = qb.Context(0)
    n = 17  # tracing 17 qubits of a ket: 131072 traced offsets > 65536
    s = qb.State(ctx, qb.KET, [2] * n).fill_gaussian(3)
    out = qb.State(ctx, qb.RHO, [1])
    with pytest.raises(qb.NotSupported):
        _noalloc(qb, s, list(range(n)), out)
    out.free()
    s.free()
    ctx.close()
