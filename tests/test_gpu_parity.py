"""GPU parity of every op on the path against the CPU oracle.

Seeded random inputs, run through the C ABI (value-semantics qgpu_host_*
entry points and the resident qgpu_state ops). Tolerances: complex128 agrees
within 1e-12 relative in the max-norm; complex64 within 2e-5; ptranspose and
syspermute are bit-exact (pure data movement).
"""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import (amplitude_damping_kraus, depolarizing_kraus, gaussian_ket,
                               haar_unitary, random_rho)

pytestmark = pytest.mark.gpu

TOL128 = 1e-12
TOL64 = 2e-5


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _rand_targets(rng, n, k):
    return [int(x) for x in rng.choice(n, size=k, replace=False)]


MIXED = [3, 3, 2, 2, 3, 2, 2, 3]


@pytest.mark.parametrize("dims,k", [([2] * 1, 1), ([2] * 6, 1), ([2] * 6, 2), ([2] * 7, 3),
                                    ([2] * 8, 4), ([2] * 9, 5), (MIXED, 1), (MIXED, 2),
                                    ([3, 4, 5], 2), ([5, 2, 7], 1)])
def test_apply_ket(ctx, dims, k):
    import qpp_b200 as qb
    rng = np.random.default_rng(hash((tuple(dims), k)) % 2**32)
    D = int(np.prod(dims))
    for _ in range(4):
        t = _rand_targets(rng, len(dims), k)
        DA = int(np.prod([dims[i] for i in t]))
        U = haar_unitary(rng, DA)
        psi = gaussian_ket(rng, D)
        got = qb.apply(psi, U, t, dims, ctx=ctx)
        ref = orc.apply(psi, U, t, dims)
        assert relerr(got, ref) < TOL128, (t, relerr(got, ref))


@pytest.mark.parametrize("dims,k", [([2] * 1, 1), ([2] * 5, 1), ([2] * 5, 2), ([2] * 5, 3),
                                    ([3, 2, 3], 1), ([3, 2, 3], 2), ([2, 3, 2, 2], 2)])
def test_apply_rho(ctx, dims, k):
    import qpp_b200 as qb
    rng = np.random.default_rng(7 + k + len(dims))
    D = int(np.prod(dims))
    for _ in range(3):
        t = _rand_targets(rng, len(dims), k)
        DA = int(np.prod([dims[i] for i in t]))
        U = haar_unitary(rng, DA)
        rho = random_rho(rng, D, 3)
        got = qb.apply(rho, U, t, dims, ctx=ctx)
        ref = orc.apply(rho, U, t, dims)
        assert relerr(got, ref) < TOL128


@pytest.mark.parametrize("kind", ["ket", "rho"])
@pytest.mark.parametrize("dims,nc,k", [([2] * 7, 1, 1), ([2] * 7, 3, 1), ([2] * 7, 2, 2),
                                       ([3] * 4, 2, 1), ([3, 2, 3, 3], 2, 1)])
def test_apply_ctrl(ctx, kind, dims, nc, k):
    import qpp_b200 as qb
    rng = np.random.default_rng(11 * nc + k + len(dims))
    D = int(np.prod(dims))
    n = len(dims)
    for trial in range(3):
        for _ in range(100):
            sub = _rand_targets(rng, n, nc + k)
            ctrl, t = sub[:nc], sub[nc:]
            if len({dims[c] for c in ctrl}) == 1:
                break
        DA = int(np.prod([dims[i] for i in t]))
        U = haar_unitary(rng, DA)
        d = dims[ctrl[0]]
        shift = None if trial == 0 else [int(x) for x in rng.integers(0, d, size=nc)]
        st = gaussian_ket(rng, D) if kind == "ket" else random_rho(rng, D, 2)
        if kind == "rho" and D > 64:
            st = random_rho(rng, D, 2)
        got = qb.applyCTRL(st, U, ctrl, t, dims, shift, ctx=ctx)
        ref = orc.applyCTRL(st, U, ctrl, t, dims, shift, path=1 if set(dims) == {2} else 0)
        assert relerr(got, ref) < 1e-11, (ctrl, t, shift)


@pytest.mark.parametrize("kind", ["ket", "rho"])
def test_apply_ctrl_fan(ctx, kind):
    import qpp_b200 as qb
    rng = np.random.default_rng(961)
    for dims in ([2] * 6, [3] * 4):
        n = len(dims)
        D = int(np.prod(dims))
        sub = _rand_targets(rng, n, 4)
        ctrl, t = sub[:2], sub[2:]
        U = haar_unitary(rng, dims[0])
        st = gaussian_ket(rng, D) if kind == "ket" else random_rho(rng, D, 2)
        for shift in (None, [1, 0]):
            got = qb.applyCTRL_fan(st, U, ctrl, t, dims, shift, ctx=ctx)
            ref = orc.applyCTRL_fan(st, U, ctrl, t, dims, shift)
            assert relerr(got, ref) < 1e-11


@pytest.mark.parametrize("dims,t", [([2] * 6, [1, 4]), ([2] * 6, [5, 0]), ([2] * 5, [3]),
                                    (MIXED[:5], [0, 2]), ([3, 2, 2], [1])])
def test_apply_kraus(ctx, dims, t):
    import qpp_b200 as qb
    rng = np.random.default_rng(476 + len(t))
    D = int(np.prod(dims))
    rho = random_rho(rng, D, 4)
    if all(dims[i] == 2 for i in t) and len(t) == 2:
        Ks = [np.kron(a, b) for a in depolarizing_kraus(0.01) for b in amplitude_damping_kraus(0.02)]
    else:
        DA = int(np.prod([dims[i] for i in t]))
        Ks = [haar_unitary(rng, DA) * np.sqrt(0.5), haar_unitary(rng, DA) * np.sqrt(0.5)]
    got = qb.apply_kraus(rho, Ks, t, dims, ctx=ctx)
    ref = orc.apply_kraus(rho, Ks, t, dims)
    assert relerr(got, ref) < TOL128


@pytest.mark.parametrize("kind", ["ket", "rho"])
@pytest.mark.parametrize("dims,t", [([2] * 6, [1, 4]), ([2] * 6, []), ([2] * 6, list(range(6))),
                                    ([2] * 8, [0, 1, 2, 5, 6, 7]), ([2] * 8, [7]),
                                    (MIXED[:6], [0, 3, 5]), ([3, 4, 2], [1])])
def test_ptrace(ctx, kind, dims, t):
    import qpp_b200 as qb
    rng = np.random.default_rng(1908 + len(t))
    D = int(np.prod(dims))
    st = gaussian_ket(rng, D) if kind == "ket" else random_rho(rng, D, 5)
    got = qb.ptrace(st, t, dims, ctx=ctx)
    ref = orc.ptrace(st, t, dims)
    assert relerr(got, ref) < TOL128


@pytest.mark.parametrize("kind", ["ket", "rho"])
@pytest.mark.parametrize("dims,t", [([2] * 6, [1, 4]), ([2] * 6, []), ([2] * 6, list(range(6))),
                                    ([2] * 7, [0, 2, 3]), (MIXED[:6], [0, 3, 5]), ([3, 4, 2], [2])])
def test_ptranspose(ctx, kind, dims, t):
    import qpp_b200 as qb
    rng = np.random.default_rng(2167 + len(t))
    D = int(np.prod(dims))
    st = gaussian_ket(rng, D) if kind == "ket" else random_rho(rng, D, 5)
    got = qb.ptranspose(st, t, dims, ctx=ctx)
    ref = orc.ptranspose(st, t, dims)
    if kind == "rho":
        assert np.array_equal(got, ref)  # bit-exact data movement
    else:
        assert relerr(got, ref) < TOL128


@pytest.mark.parametrize("kind", ["ket", "rho"])
@pytest.mark.parametrize("dims", [[2] * 7, MIXED[:6], [3, 4, 2, 5], [2]])
def test_syspermute(ctx, kind, dims):
    import qpp_b200 as qb
    rng = np.random.default_rng(2386 + len(dims))
    D = int(np.prod(dims))
    for _ in range(3):
        perm = [int(x) for x in rng.permutation(len(dims))]
        st = gaussian_ket(rng, D) if kind == "ket" else random_rho(rng, D, 4)
        got = qb.syspermute(st, perm, dims, ctx=ctx)
        ref = orc.syspermute(st, perm, dims)
        assert np.array_equal(got, ref)  # bit-exact


@pytest.mark.parametrize("call", [
    ("apply", dict(target=[], dims=[2, 2])),
    ("apply", dict(target=[0, 0], dims=[2, 2])),
    ("apply", dict(target=[2], dims=[2, 2])),
    ("apply", dict(target=[0], dims=[2, 3])),
    ("apply", dict(target=[0], dims=[2, 0])),
    ("apply", dict(target=[0, 1], dims=[2, 2])),
    ("ptrace", dict(target=[5], dims=[2, 2])),
    ("ptranspose", dict(target=[0], dims=[3])),
    ("syspermute", dict(perm=[0, 0], dims=[2, 2])),
    ("syspermute", dict(perm=[1, 0, 2], dims=[2, 2])),
    ("ctrl", dict(ctrl=[0], target=[0], dims=[2, 2])),
    ("ctrl", dict(ctrl=[0, 1], target=[2], dims=[2, 3, 2])),
    ("ctrl", dict(ctrl=[0], target=[1], dims=[2, 2], shift=[2])),
    ("ctrl", dict(ctrl=[], target=[1], dims=[2, 2])),
])
def test_error_parity(ctx, call):
    """The first error matches qpp's exception type and (where, what)."""
    import qpp_b200 as qb
    name, kw = call
    psi = np.zeros(4, dtype=np.complex128)
    psi[0] = 1
    X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    fns = {
        "apply": (lambda m: m.apply(psi, X, kw["target"], kw["dims"])),
        "ptrace": (lambda m: m.ptrace(psi, kw["target"], kw["dims"])),
        "ptranspose": (lambda m: m.ptranspose(psi, kw["target"], kw["dims"])),
        "syspermute": (lambda m: m.syspermute(psi, kw["perm"], kw["dims"])),
        "ctrl": (lambda m: m.applyCTRL(psi if kw["dims"] != [2, 3, 2] else np.ones(12),
                                       X, kw["ctrl"], kw["target"], kw["dims"], kw.get("shift"))),
    }
    with pytest.raises(orc.OracleError) as eo:
        fns[name](orc)
    with pytest.raises(qb.QppError) as eg:
        fns[name](qb)
    assert (eg.value.code, eg.value.where, eg.value.what) == \
        (eo.value.code, eo.value.where, eo.value.what)


def test_resident_chain_c128_and_c64(ctx):
    """A chain of resident ops on one device state matches the oracle chain."""
    import qpp_b200 as qb
    rng = np.random.default_rng(99)
    dims = [2] * 10
    psi = gaussian_ket(rng, 2 ** 10)
    ref = psi.copy()
    s128 = qb.State.from_numpy(ctx, psi, dims, qb.C128)
    s64 = qb.State.from_numpy(ctx, psi, dims, qb.C64)
    for i in range(60):
        k = 1 + (i % 3)
        t = _rand_targets(rng, 10, k)
        U = haar_unitary(rng, 2 ** k)
        ref = orc.apply(ref, U, t, dims)
        s128.apply(U, t)
        s64.apply(U, t)
    assert relerr(s128.numpy(), ref) < TOL128
    assert relerr(s64.numpy(), ref) < 1e-4
    assert abs(s128.norm2() - 1) < 1e-12
    rho_ref = orc.ptrace(ref, [0, 3, 9], dims)
    assert relerr(s128.ptrace([0, 3, 9]).numpy(), rho_ref) < TOL128


def test_config1_ket_gates(ctx):
    """20-qubit Gaussian ket, 1000 Haar gates (70% 1q, 30% 2q on ordered
    pairs) then 100 applyCTRL with 1-3 controls; vs qpp within 1e-12."""
    import qpp_b200 as qb
    rng = np.random.default_rng(20)
    n = 20
    dims = [2] * n
    psi = gaussian_ket(rng, 2 ** n)
    ref = psi.copy()
    s = qb.State.from_numpy(ctx, psi, dims)
    for _ in range(1000):
        if rng.random() < 0.7:
            t = [int(rng.integers(n))]
        else:
            t = _rand_targets(rng, n, 2)
        U = haar_unitary(rng, 2 ** len(t))
        s.apply(U, t)
        ref = orc.apply(ref, U, t, dims, path=1)
    for _ in range(100):
        nc = int(rng.integers(1, 4))
        sub = _rand_targets(rng, n, nc + 1)
        U = haar_unitary(rng, 2)
        s.apply_ctrl(U, sub[:nc], sub[nc:])
        ref = orc.applyCTRL(ref, U, sub[:nc], sub[nc:], dims, path=1)
    assert relerr(s.numpy(), ref) < TOL128


def test_states_outlive_a_closed_context():
    """Destroying a context while states are alive defers the teardown to the
    last state's destruction (no use after free)."""
    import qpp_b200 as qb
    c = qb.Context(0)
    a = qb.State(c, qb.KET, [2] * 10).fill_gaussian(1)
    b = a.ptrace([0, 1])
    c.close()
    assert abs(a.norm2() - 1) < 1e-12
    del a
    assert b.numpy().shape == (256, 256)
    del b


def test_plain_gates_with_64_bit_indices():
    """A 31-qubit complex64 ket (16 GiB): a one-qubit gate's grid, one pair
    per thread over the whole state, has a last loop step past 2^32, so the
    kernel indexes in 64 bits; the same gate as U (x) I on a two-qubit group
    (whose kernel stays in 32 bits) must give the same state."""
    import qpp_b200 as qb
    ctx = qb.Context(0)
    n = 31
    rng = np.random.default_rng(31)
    s = qb.State(ctx, qb.KET, [2] * n, qb.C64)
    s.fill_gaussian(3)
    s.normalize()
    t = s.clone()
    for q, p in ((0, 5), (17, 30), (30, 0)):
        U = haar_unitary(rng, 2)
        s.apply(U, [q])
        t.apply(np.kron(U, np.eye(2)), [q, p])
    ov = s.inner(t)
    assert abs(abs(ov) - 1.0) < 1e-5, ov
    assert abs(s.norm2() - 1.0) < 1e-5
    s.free()
    t.free()
    ctx.close()
