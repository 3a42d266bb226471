"""qgpu_ptrace_noalloc: the partial trace for callers that cannot allocate
device memory at the time of the call (an application whose memory pool
already owns the GPU's free memory, or a loop that cannot afford the device
synchronisation of cudaMalloc/cudaFree).

The test calls it through the C ABI with a caller-owned output buffer and
compares it with the allocating qgpu_ptrace on the same state, within the
path's complex128 tolerance (1e-12 relative, max-norm), on two calls in a
row with different traced subsystems, so the second call overwrites the
shared offset table left by the first; once with the two calls queued back
to back on the stream before a single synchronise (stream order keeps the
shared table safe for one caller), once against the FP64 oracle directly,
once in complex64 (1e-5) and once tracing every subsystem (the 1 x 1 trace).
It also checks the size limit and the error location.
This file is collected last on purpose: if it fails, a run that stops at
the first failure has already run every other test.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _queue(qb, state, target, out_state):
    t = np.ascontiguousarray(np.asarray(target, dtype=np.uint64))
    rc = qb.lib().qgpu_ptrace_noalloc(state.h, t.ctypes.data_as(ct.POINTER(ct.c_uint64)),
                                      ct.c_uint32(len(target)), ct.c_void_p(out_state.device_ptr()))
    qb.check(rc)


def _noalloc(qb, state, target, out_state):
    _queue(qb, state, target, out_state)
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


def test_noalloc_ptrace_queued_calls_and_oracle():
    """Two calls queued on the stream before one synchronise, each into its
    own buffer: both match the allocating path, and one matches the oracle."""
    import qpp_b200 as qb
    from oracle import oracle as orc
    from tests.qpp_helpers import random_rho
    ctx = qb.Context(0)
    rng = np.random.default_rng(7)
    dims = [2, 2, 3, 2, 2, 2]
    D = int(np.prod(dims))
    host = random_rho(rng, D, 5)
    s = qb.State.from_numpy(ctx, host, dims)
    targets = ([0, 3], [1, 2, 5])
    outs = []
    for target in targets:
        kept = [dims[q] for q in range(len(dims)) if q not in target]
        outs.append(qb.State(ctx, qb.RHO, kept))
        _queue(qb, s, target, outs[-1])
    ctx.synchronize()
    for target, out in zip(targets, outs):
        got = out.numpy()
        assert _relerr(got, s.ptrace(target).numpy()) < 1e-12
        assert _relerr(got, orc.ptrace(host, target, dims)) < 1e-12
        out.free()
    s.free()
    ctx.close()


def test_noalloc_ptrace_complex64_and_full_trace():
    import qpp_b200 as qb
    from tests.qpp_helpers import gaussian_ket
    ctx = qb.Context(0)
    rng = np.random.default_rng(8)
    n = 12
    host = gaussian_ket(rng, 2 ** n)
    s64 = qb.State.from_numpy(ctx, host, [2] * n, qb.C64)
    out = qb.State(ctx, qb.RHO, [2] * 5, qb.C64)
    target = [0, 2, 4, 5, 7, 9, 11]
    got = _noalloc(qb, s64, target, out)
    assert _relerr(got, s64.ptrace(target).numpy()) < 1e-5
    out.free()
    # every subsystem traced: the 1 x 1 result is the squared norm
    s = qb.State.from_numpy(ctx, host, [2] * n)
    one = qb.State(ctx, qb.RHO, [1])
    got = _noalloc(qb, s, list(range(n)), one)
    ref = s.ptrace(list(range(n))).numpy()
    assert got.shape == ref.shape and _relerr(got, ref) < 1e-12
    assert abs(got.reshape(-1)[0] - s.norm2()) < 1e-12
    one.free()
    s.free()
    s64.free()
    ctx.close()


def test_noalloc_ptrace_reports_its_own_name():
    import qpp_b200 as qb
    ctx = qb.Context(0)
    s = qb.State(ctx, qb.KET, [2] * 4).fill_gaussian(1)
    out = qb.State(ctx, qb.RHO, [2] * 3)
    with pytest.raises(qb.SubsysMismatchDims) as e:
        _noalloc(qb, s, [7], out)
    assert e.value.where == "qgpu_ptrace_noalloc()"
    out.free()
    s.free()
    ctx.close()
