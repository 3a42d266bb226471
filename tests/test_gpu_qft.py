"""GPU parity of qpp::applyQFT / applyTFQ / QFT / TFQ and QCircuit::QFT / TFQ
against the CPU oracle (oracle/oracle.py, qpp's gate sequence through the
oracle's apply / applyCTRL). Complex128 agrees within 1e-12 relative in the
max-norm; complex64 within 2e-5."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.qpp_helpers import gaussian_ket, random_rho

pytestmark = pytest.mark.gpu

TOL128 = 1e-12
TOL64 = 2e-5


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _targets(rng, n, k, ordered):
    t = [int(x) for x in rng.permutation(n)[:k]]
    return sorted(t) if ordered else t


@pytest.mark.parametrize("d,n", [(2, 1), (2, 2), (2, 5), (2, 9), (2, 12), (3, 4), (3, 6),
                                 (4, 3), (5, 3), (16, 2), (17, 2)])
def test_apply_qft_ket(ctx, d, n):
    """Kets: every target subset shape (all digits in order, random subsets in
    random order), swap on and off, forward and inverse; d = 17 takes qpp's
    gate sequence on the gate kernels."""
    import qpp_b200 as qb
    rng = np.random.default_rng(1000 * d + n)
    D = d ** n
    for rep in range(4):
        k = n if rep == 0 else int(rng.integers(1, n + 1))
        t = _targets(rng, n, k, rep == 0)
        psi = gaussian_ket(rng, D)
        for swap in (True, False):
            got = qb.applyQFT(psi, t, d, swap, ctx=ctx)
            ref = orc.applyQFT(psi, t, d, swap)
            assert relerr(got, ref) < TOL128, (t, swap, relerr(got, ref))
            got = qb.applyTFQ(psi, t, d, swap, ctx=ctx)
            ref = orc.applyTFQ(psi, t, d, swap)
            assert relerr(got, ref) < TOL128, (t, swap, "tfq", relerr(got, ref))


@pytest.mark.parametrize("d,n", [(2, 1), (2, 3), (2, 6), (3, 3)])
def test_apply_qft_rho(ctx, d, n):
    import qpp_b200 as qb
    rng = np.random.default_rng(77 + d + n)
    D = d ** n
    for rep in range(3):
        k = n if rep == 0 else int(rng.integers(1, n + 1))
        t = _targets(rng, n, k, rep == 0)
        rho = random_rho(rng, D, 3)
        for swap in (True, False):
            got = qb.applyQFT(rho, t, d, swap, ctx=ctx)
            ref = orc.applyQFT(rho, t, d, swap)
            assert relerr(got, ref) < TOL128, (t, swap, relerr(got, ref))
            got = qb.applyTFQ(rho, t, d, swap, ctx=ctx)
            ref = orc.applyTFQ(rho, t, d, swap)
            assert relerr(got, ref) < TOL128, (t, swap, "tfq", relerr(got, ref))


def test_whole_qft_tfq(ctx):
    import qpp_b200 as qb
    rng = np.random.default_rng(3)
    for d, n in [(2, 10), (3, 5)]:
        psi = gaussian_ket(rng, d ** n)
        for swap in (True, False):
            assert relerr(qb.QFT(psi, d, swap, ctx=ctx), orc.QFT(psi, d, swap)) < TOL128
            assert relerr(qb.TFQ(psi, d, swap, ctx=ctx), orc.TFQ(psi, d, swap)) < TOL128


def test_resident_qft_c128_c64_and_pass_count(ctx):
    """The resident op: 20 qubits in 3 passes (4 + 8 + 8 targets, the
    reversal riding on the last), matching numpy's DFT; complex64 too."""
    import qpp_b200 as qb
    rng = np.random.default_rng(11)
    n = 20
    psi = gaussian_ket(rng, 2 ** n)
    ref = np.fft.ifft(psi) * np.sqrt(2 ** n)
    s = qb.State.from_numpy(ctx, psi, [2] * n)
    ctx.synchronize()
    before = ctx.launches()
    s.qft()
    ctx.synchronize()
    assert ctx.launches() - before == 3
    assert relerr(s.numpy(), ref) < TOL128
    s.qft(inverse=True)
    assert relerr(s.numpy(), psi) < TOL128
    s64 = qb.State.from_numpy(ctx, psi, [2] * n, prec=qb.C64)
    s64.apply_qft(list(range(n)))
    assert relerr(s64.numpy(), ref) < TOL64


@pytest.mark.parametrize("n", [14, 22])
def test_pass_shapes_compiled_and_runtime(ctx, n):
    """The passes of full transforms: 14 = 6 + 8 and 22 = 6 + 8 + 8 targets
    (the 8-target pass that reverses the targets reads one buffer and writes
    another), 6- and 8-target passes of 2^11 (complex128) and 2^12
    (complex64) amplitudes; forward against numpy's DFT, inverse back to the
    input, both precisions."""
    import qpp_b200 as qb
    rng = np.random.default_rng(100 + n)
    psi = gaussian_ket(rng, 2 ** n)
    ref = np.fft.ifft(psi) * np.sqrt(2 ** n)
    for prec, tol in ((qb.C128, TOL128), (qb.C64, TOL64)):
        s = qb.State.from_numpy(ctx, psi, [2] * n, prec=prec)
        s.apply_qft(list(range(n)))
        assert relerr(s.numpy(), ref) < tol, (prec, "qft")
        s.apply_tfq(list(range(n)))
        assert relerr(s.numpy(), psi) < tol, (prec, "tfq")
        s.free()


def test_transforms_without_reversal(ctx):
    """swap = false: the pass on the lowest digits keeps the shared-memory
    rounds, the others run in register rounds. 14 qubits against the oracle
    in both precisions, 22 qubits as a QFT-then-TFQ round trip."""
    import qpp_b200 as qb
    rng = np.random.default_rng(1414)
    for n in (14, 22):
        psi = gaussian_ket(rng, 2 ** n)
        ref = orc.applyQFT(psi, list(range(n)), 2, False) if n == 14 else None
        for prec, tol in ((qb.C128, TOL128), (qb.C64, TOL64)):
            s = qb.State.from_numpy(ctx, psi, [2] * n, prec=prec)
            s.apply_qft(list(range(n)), swap=False)
            if ref is not None:
                assert relerr(s.numpy(), ref) < tol, (n, prec)
            s.apply_tfq(list(range(n)), swap=False)
            assert relerr(s.numpy(), psi) < tol, (n, prec, "round trip")
            s.free()


def test_complex64_density_matrix_passes(ctx):
    """A complex64 density matrix of 8 qubits: U on the row digits and
    conj(U) on the column digits, each an 8-step pass, against the oracle."""
    import qpp_b200 as qb
    rng = np.random.default_rng(808)
    n = 8
    rho = random_rho(rng, 2 ** n, 4)
    for inverse in (False, True):
        s = qb.State.from_numpy(ctx, rho, [2] * n, prec=qb.C64)
        if inverse:
            s.apply_tfq(list(range(n)))
            ref = orc.applyTFQ(rho, list(range(n)), 2, True)
        else:
            s.apply_qft(list(range(n)))
            ref = orc.applyQFT(rho, list(range(n)), 2, True)
        assert relerr(s.numpy(), ref) < TOL64, inverse
        s.free()


def test_round_trip_26_qubits(ctx):
    """Size-independent property at 26 qubits (1 GiB complex128): TFQ after
    QFT on a random subset gives the input back, and the norm is kept."""
    import qpp_b200 as qb
    rng = np.random.default_rng(26)
    n = 26
    s = qb.State(ctx, qb.KET, [2] * n)
    s.fill_gaussian(5)
    s.normalize()
    psi = s.numpy()
    t = _targets(rng, n, 19, False)
    s.apply_qft(t)
    assert abs(s.norm2() - 1.0) < 1e-12
    s.apply_tfq(t)
    assert relerr(s.numpy(), psi) < TOL128


def test_qft_on_grouped_dims(ctx):
    """qpp views the state as n digits of dimension d whatever dims it was
    built with: a state over dims [4, 2] is three qubits for d = 2."""
    import qpp_b200 as qb
    rng = np.random.default_rng(8)
    psi = gaussian_ket(rng, 8)
    s = qb.State.from_numpy(ctx, psi, [4, 2])
    s.apply_qft([2, 0], d=2)
    assert relerr(s.numpy(), orc.applyQFT(psi, [2, 0], 2)) < TOL128
    assert s.dims == [4, 2]


@pytest.mark.parametrize("call", [
    ("applyQFT", dict(a=np.zeros(0), t=[0])),
    ("applyQFT", dict(a=np.ones(4), t=[0], d=1)),
    ("applyQFT", dict(a=np.ones(4), t=[2])),
    ("applyQFT", dict(a=np.ones(4), t=[0, 0])),
    ("applyTFQ", dict(a=np.ones(6), t=[0])),
    ("applyQFT", dict(a=np.ones((6, 6)), t=[0])),
    ("applyQFT", dict(a=np.ones((4, 2)), t=[0])),
    ("TFQ", dict(a=np.ones(6))),
    ("TFQ", dict(a=np.ones(4), d=1)),
])
def test_error_parity(ctx, call):
    import qpp_b200 as qb
    name, kw = call
    d = kw.get("d", 2)

    def run(m):
        if name in ("QFT", "TFQ"):
            return getattr(m, name)(kw["a"], d)
        return getattr(m, name)(kw["a"], kw["t"], d)
    with pytest.raises(orc.OracleError) as eo:
        run(orc)
    with pytest.raises(qb.QppError) as eg:
        run(qb)
    assert (eg.value.code, eg.value.where, eg.value.what) == \
        (eo.value.code, eo.value.where, eo.value.what)


@pytest.mark.parametrize("inverse", [False, True])
def test_circuit_qft_block(ctx, inverse):
    """QCircuit::QFT / TFQ appends qpp's gate sequence; the noiseless engine
    runs the block as one transform, the noisy engine (identity noise) steps
    through the gates; both match the oracle."""
    import qpp_b200 as qb
    rng = np.random.default_rng(21 + inverse)
    n = 9
    psi = gaussian_ket(rng, 2 ** n)
    t = [4, 1, 7, 0, 8, 2]
    c = qb.Circuit(n)
    (c.TFQ if inverse else c.QFT)(t)
    assert c.steps() == len(t) + len(t) * (len(t) - 1) // 2 + len(t) // 2
    ref = (orc.applyTFQ if inverse else orc.applyQFT)(psi, t, 2)
    e = qb.Engine(ctx, c).set_state(qb.State.from_numpy(ctx, psi, [2] * n))
    ctx.synchronize()
    before = ctx.launches()
    e.execute()
    ctx.synchronize()
    assert ctx.launches() - before <= 2
    assert relerr(e.get_state().numpy(), ref) < TOL128
    en = qb.Engine(ctx, c).set_noise([np.eye(2)], [1.0])
    en.set_state(qb.State.from_numpy(ctx, psi, [2] * n)).execute()
    assert relerr(en.get_state().numpy(), ref) < TOL128


def test_circuit_qft_all_unmeasured(ctx):
    """QFT() with no target takes the qudits not measured so far."""
    import qpp_b200 as qb
    c = qb.Circuit(3, nc=1)
    c.measure([1], 0)
    c.QFT()
    assert c.steps() == 1 + 2 + 1 + 1
