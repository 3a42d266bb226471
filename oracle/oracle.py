"""ctypes front-end of the CPU oracle (oracle/qpp_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py. The product package (qpp_b200) never imports it.

Each function mirrors the Quantum++ 7.0.3 free function of the same name
(include/qpp/operations.hpp, instruments.hpp) with value semantics: numpy
complex128 arrays in (kets as 1-D arrays or (D, 1) columns, density matrices
as (D, D)), a fresh numpy array out. Errors raise OracleError carrying qpp's
(where, what) pair and the shared status code of include/qpp_b200.h.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

u64p = ct.POINTER(ct.c_uint64)
dp = ct.POINTER(ct.c_double)


class OracleError(RuntimeError):
    def __init__(self, code, where, what):
        super().__init__(f"{where}: {what} (status {code})")
        self.code, self.where, self.what = code, where, what


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ct.CDLL(_LIB_PATH)
        L.oracle_last_where.restype = ct.c_char_p
        L.oracle_last_what.restype = ct.c_char_p
        _lib = L
    return _lib


def _u64(v):
    if v is None:
        return None, None
    a = np.ascontiguousarray(np.asarray(v, dtype=np.uint64).reshape(-1))
    return a, a.ctypes.data_as(u64p)


def _cplx(a):
    a = np.asarray(a, dtype=np.complex128)
    return a


def _state(a):
    a = _cplx(a)
    if a.ndim == 1:
        rows, cols = a.shape[0], 1
        buf = np.ascontiguousarray(a)
    else:
        rows, cols = a.shape
        buf = np.asfortranarray(a)
    return buf, rows, cols


def _check(rc):
    if rc != 0:
        L = lib()
        raise OracleError(rc, L.oracle_last_where().decode(), L.oracle_last_what().decode())


def _out_like(rows, cols, shape_1d):
    if cols == 1 and shape_1d:
        return np.zeros(rows, dtype=np.complex128)
    return np.zeros((rows, cols), dtype=np.complex128, order="F")


def _dp(a):
    return a.ctypes.data_as(dp)


def apply(state, A, target, dims, path=0):
    """qpp::apply(state, A, target, dims), operations.hpp:72-372.
    path=1 takes the qubit-kernel loops (apply.hpp) for 1q/2q kets."""
    buf, rows, cols = _state(state)
    Am = np.asfortranarray(_cplx(A))
    ar, ac = (Am.shape + (1,))[:2] if Am.ndim == 2 else (Am.shape[0], 1)
    t, tp = _u64(target)
    d, dpp = _u64(dims)
    out = _out_like(rows, cols, np.asarray(state).ndim == 1)
    _check(lib().oracle_apply(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols), _dp(Am),
                              ct.c_uint64(ar), ct.c_uint64(ac), tp, ct.c_uint32(len(t)),
                              dpp, ct.c_uint32(len(d)), _dp(out), ct.c_int(path)))
    return out


def applyCTRL(state, A, ctrl, target, dims, shift=None, path=0, fan=False):
    """qpp::applyCTRL / applyCTRL_fan, operations.hpp:616-1234."""
    buf, rows, cols = _state(state)
    Am = np.asfortranarray(_cplx(A))
    c, cp = _u64(ctrl)
    t, tp = _u64(target)
    d, dpp = _u64(dims)
    s, sp = _u64(shift)
    out = _out_like(rows, cols, np.asarray(state).ndim == 1)
    _check(lib().oracle_apply_ctrl(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols), _dp(Am),
                                   ct.c_uint64(Am.shape[0]), ct.c_uint64(Am.shape[1]),
                                   cp, ct.c_uint32(len(c)), tp, ct.c_uint32(len(t)),
                                   dpp, ct.c_uint32(len(d)), sp, ct.c_int(1 if fan else 0),
                                   _dp(out), ct.c_int(path)))
    return out


def applyCTRL_fan(state, A, ctrl, target, dims, shift=None, path=0):
    return applyCTRL(state, A, ctrl, target, dims, shift, path, fan=True)


def apply_kraus(rho, Ks, target, dims):
    """qpp::apply(A, Ks, target, dims), operations.hpp:476-560."""
    buf, rows, cols = _state(rho)
    Ks = [np.asfortranarray(_cplx(K)) for K in Ks]
    kr, kc = Ks[0].shape if Ks else (0, 0)
    packed = np.concatenate([K.reshape(-1, order="F") for K in Ks]) if Ks else np.zeros(1, np.complex128)
    packed = np.ascontiguousarray(packed)
    t, tp = _u64(target)
    d, dpp = _u64(dims)
    out = np.zeros((rows, cols), dtype=np.complex128, order="F")
    _check(lib().oracle_apply_kraus(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols), _dp(packed),
                                    ct.c_uint32(len(Ks)), ct.c_uint64(kr), ct.c_uint64(kc),
                                    tp, ct.c_uint32(len(t)), dpp, ct.c_uint32(len(d)), _dp(out)))
    return out


def ptrace(state, target, dims):
    """qpp::ptrace(A, target, dims), operations.hpp:1908-2114."""
    buf, rows, cols = _state(state)
    t, tp = _u64(target)
    d, dpp = _u64(dims)
    DS = 1
    for i in target:
        if 0 <= int(i) < len(dims):
            DS *= int(dims[int(i)])
    Db = rows // DS if rows % DS == 0 else 1
    out = np.zeros((max(Db, 1), max(Db, 1)), dtype=np.complex128, order="F")
    _check(lib().oracle_ptrace(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols), tp,
                               ct.c_uint32(len(t)), dpp, ct.c_uint32(len(d)), _dp(out)))
    return out


def ptranspose(state, target, dims, compat=False):
    """qpp::ptranspose(A, target, dims), operations.hpp:2167-2335.
    compat=True reproduces internal/kernels/qubit/ptranspose.hpp."""
    buf, rows, cols = _state(state)
    t, tp = _u64(target)
    d, dpp = _u64(dims)
    out = np.zeros((rows, rows), dtype=np.complex128, order="F")
    _check(lib().oracle_ptranspose(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols), tp,
                                   ct.c_uint32(len(t)), dpp, ct.c_uint32(len(d)), _dp(out),
                                   ct.c_int(1 if compat else 0)))
    return out


def syspermute(state, perm, dims, compat=False):
    """qpp::syspermute(A, perm, dims), operations.hpp:2386-2514.
    compat=True reproduces internal/kernels/qubit/syspermute.hpp."""
    buf, rows, cols = _state(state)
    p, pp = _u64(perm)
    d, dpp = _u64(dims)
    out = _out_like(rows, cols, np.asarray(state).ndim == 1)
    _check(lib().oracle_syspermute(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols), pp,
                                   ct.c_uint32(len(p)), dpp, ct.c_uint32(len(d)), _dp(out),
                                   ct.c_int(1 if compat else 0)))
    return out


def normalize(state):
    """qpp::normalize(A), functions.hpp:304-333."""
    buf, rows, cols = _state(state)
    buf = buf.copy(order="F" if cols > 1 else "C")
    _check(lib().oracle_normalize(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols)))
    return buf


def measure_seq(state, target, dims, destructive=True, forced=None, seed=0):
    """qpp::measure_seq(A, target, dims, destructive), instruments.hpp:985-1111.
    forced: outcome dits to take instead of sampling (replay mode).
    Returns (results, probs, post-measurement state, its dims)."""
    buf, rows, cols = _state(state)
    t, tp = _u64(target)
    d, dpp = _u64(dims)
    f, fp = _u64(forced)
    k = len(t)
    res = np.zeros(max(k, 1), dtype=np.uint64)
    probs = np.zeros(max(k, 1), dtype=np.float64)
    out = np.zeros(rows * cols, dtype=np.complex128)
    od = np.zeros(max(len(d), 1), dtype=np.uint64)
    ond = ct.c_uint32(0)
    _check(lib().oracle_measure_seq(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols), tp,
                                    ct.c_uint32(k), dpp, ct.c_uint32(len(d)),
                                    ct.c_int(1 if destructive else 0), fp, ct.c_uint64(seed),
                                    res.ctypes.data_as(u64p), _dp(probs), _dp(out),
                                    od.ctypes.data_as(u64p), ct.byref(ond)))
    nd = [int(x) for x in od[: ond.value]]
    Dn = int(np.prod(nd)) if nd else 1
    if cols == 1:
        st = out[:Dn].copy()
    else:
        st = out[: Dn * Dn].reshape((Dn, Dn), order="F").copy()
    return [int(x) for x in res[:k]], [float(x) for x in probs[:k]], st, nd


def sample(state, target, dims, num_samples, seed=0):
    """qpp::sample(num_samples, A, target, dims), instruments.hpp:856-940, with
    std::mt19937(seed): the target digits of every draw, in draw order
    (num_samples x len(target))."""
    buf, rows, cols = _state(state)
    t, tp = _u64(target)
    d, dpp = _u64(dims)
    k = len(t)
    out = np.zeros(max(num_samples * k, 1), dtype=np.uint64)
    _check(lib().oracle_sample(_dp(buf), ct.c_uint64(rows), ct.c_uint64(cols), tp,
                               ct.c_uint32(k), dpp, ct.c_uint32(len(d)),
                               ct.c_uint64(num_samples), ct.c_uint64(seed),
                               out.ctypes.data_as(u64p)))
    return out[: num_samples * k].reshape(num_samples, k).astype(np.int64)


def discrete_draw(weights, seed=0):
    """One std::discrete_distribution draw from std::mt19937(seed)."""
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
    L = lib()
    L.oracle_discrete_draw.restype = ct.c_uint64
    return int(L.oracle_discrete_draw(_dp(w), ct.c_uint64(w.size), ct.c_uint64(seed)))


def _is_ket(a):
    a = np.asarray(a)
    return a.ndim == 1 or a.shape[1] == 1


def measure_kraus(state, Ks, target, dims, destructive=True, seed=0):
    """qpp::measure(A, Ks, target, dims, destructive), instruments.hpp:371-494:
    every Kraus operator applied on the targets (K psi, or K rho K^dagger),
    its probability, the normalised post-measurement state (targets traced
    out when destructive: a density matrix even for a ket), then one draw.
    Returns (result, probs, states with None where the probability is 0)."""
    ket = _is_ket(state)
    probs, outs = [], []
    for K in Ks:
        tmp = apply(state, K, target, dims)
        if ket:
            p = float(np.linalg.norm(tmp)) ** 2
            out = None
            if p > 0:
                tmp = tmp / np.sqrt(p)
                out = ptrace(tmp, target, dims) if destructive else tmp
        else:
            if destructive:
                tmp = ptrace(tmp, target, dims)
            p = abs(np.trace(tmp))
            out = tmp / p if p > 0 else None
        probs.append(p)
        outs.append(out)
    return discrete_draw(probs, seed), probs, outs


def _ip(v, psi, target, dims):
    """qpp::ip(phi, psi, subsys, dims): sum over the target digits of
    conj(phi) psi, the other digits kept in their order."""
    n = len(dims)
    x = np.asarray(psi).reshape([int(d) for d in dims])
    vv = np.conj(np.asarray(v).reshape([int(dims[t]) for t in target]))
    rest = [q for q in range(n) if q not in target]
    x = np.transpose(x, list(target) + rest)
    out = np.tensordot(vv, x, axes=(list(range(len(target))), list(range(len(target)))))
    return out.reshape(-1)


def measure_basis(state, V, target, dims, destructive=True, seed=0):
    """qpp::measure(A, V, target, dims, destructive), instruments.hpp:587-712:
    the columns of V as rank-1 projectors; a ket measured destructively keeps
    <v_i| psi> over the targets (a ket), otherwise prj(v_i) is applied; a
    density matrix goes through measure_kraus with K_i = v_i v_i^dagger."""
    V = np.asarray(V, dtype=np.complex128)
    if not _is_ket(state):
        return measure_kraus(state, [np.outer(V[:, i], V[:, i].conj()) for i in range(V.shape[1])],
                             target, dims, destructive, seed)
    psi = np.asarray(state).reshape(-1)
    probs, outs = [], []
    for i in range(V.shape[1]):
        v = V[:, i]
        o = _ip(v, psi, target, dims) if destructive else \
            apply(psi, np.outer(v, v.conj()), target, dims)
        nrm = float(np.linalg.norm(o))
        p = nrm * nrm
        probs.append(p)
        outs.append(o / nrm if p > 0 else None)
    return discrete_draw(probs, seed), probs, outs


def _xd_power(d, k):
    X = np.zeros((d, d), dtype=np.complex128)
    for j in range(d):
        X[(j + 1) % d, j] = 1
    return np.linalg.matrix_power(X, k)


def reset(state, target, dims, seed=0):
    """qpp::reset(A, target, dims), instruments.hpp:1148-1206: measure_seq
    without destruction, then Xd^(d - result) on each target; d is dims[i]
    for the i-th target (qpp indexes dims by the target's position)."""
    res, _, out, nd = measure_seq(state, target, dims, destructive=False, seed=seed)
    for i, t in enumerate(target):
        d = int(dims[i])
        out = apply(out, _xd_power(d, d - res[i]), [t], dims)
    return out


def discard(state, target, dims, seed=0):
    """qpp::discard(A, target, dims), instruments.hpp:1243-1292: measure_seq
    with destruction, the post-measurement state only."""
    return measure_seq(state, target, dims, destructive=True, seed=seed)[2]


# ------------------------------------------------------- Fourier transforms
def _fd(d):
    """qpp::Gates::Fd(d), gates.hpp:260-285: H for d = 2, else
    F(i, j) = omega^(i j) / sqrt(d) with omega = exp(2 pi i / d)."""
    if d == 2:
        h = 1.0 / np.sqrt(2.0)
        return np.array([[h, h], [h, -h]], dtype=np.complex128)
    om = np.exp(2.0 * np.pi * 1j / d)
    F = np.empty((d, d), dtype=np.complex128)
    for j in range(d):
        for i in range(d):
            F[i, j] = 1.0 / np.sqrt(d) * om ** (i * j)
    return F


def _swapd(d):
    """qpp::Gates::SWAPd(d): |a b> -> |b a>."""
    S = np.zeros((d * d, d * d), dtype=np.complex128)
    for a in range(d):
        for b in range(d):
            S[b * d + a, a * d + b] = 1
    return S


def _rj(d, j, sign):
    """R_j = diag(exp(sign 2 pi i m / d^j)), operations.hpp:2616-2618, :2641-2646."""
    return np.diag([np.exp(sign * 2.0 * np.pi * m * 1j / float(d) ** j) for m in range(d)])


_QFT_CODES = dict(ZeroSize=1, MatrixNotSquareNorCvector=3, DimsInvalid=5,
                  DimsMismatchMatrix=7, DimsMismatchCvector=8, SubsysMismatchDims=9)


def _check_qft(where, a, target, d, whole):
    """The checks of applyQFT / applyTFQ (operations.hpp:2569-2605,
    :2684-2720) and of QFT / TFQ (:2793-2826, :2845-2878, whose dims checks
    both name qpp::QFT()), in qpp's order. Returns dims = n x d."""
    def err(kind, w, what):
        raise OracleError(_QFT_CODES[kind], w, what)
    rows = a.shape[0]
    cols = 1 if a.ndim == 1 else a.shape[1]
    if rows * cols == 0:
        err("ZeroSize", where, "A")
    if d < 2:
        err("DimsInvalid", where, "d")
    n = int(np.rint(np.log2(rows) / np.log2(d)))  # get_num_subsys, util.hpp:389-397
    dims = [d] * n
    if not whole:
        if len(target) > n or len(set(target)) != len(target) or any(t >= n for t in target):
            err("SubsysMismatchDims", where, "dims/target")
    wd = "qpp::QFT()" if whole else where
    if cols == 1:
        if n == 0 or d ** n != rows:
            err("DimsMismatchCvector", wd, "A/dims")
    elif rows == cols:
        if n == 0 or d ** n != rows:
            err("DimsMismatchMatrix", wd, "A/dims")
    else:
        err("MatrixNotSquareNorCvector", wd, "A")
    return dims


def applyQFT(state, target, d=2, swap=True, _where="qpp::applyQFT()", _whole=False):
    """qpp::applyQFT(A, target, d, swap), operations.hpp:2565-2676: for each
    target i, Fd (H for qubits) on it, then controlled R_j (control
    target[i + j - 1], j = 2..k-i) on it; with swap, SWAPs reverse the
    targets at the end. Every gate goes through this oracle's apply /
    applyCTRL."""
    a = _cplx(state)
    dims = _check_qft(_where, a, list(target), d, _whole)
    if _whole:
        target = list(range(len(dims)))
    out = a
    k = len(target)
    for i in range(k):
        out = apply(out, _fd(d), [target[i]], dims)
        for j in range(2, k - i + 1):
            out = applyCTRL(out, _rj(d, j, 1.0), [target[i + j - 1]], [target[i]], dims)
    if swap:
        for i in range(k // 2):
            out = apply(out, _swapd(d), [target[i], target[k - i - 1]], dims)
    return out


def applyTFQ(state, target, d=2, swap=True, _where="qpp::applyTFQ()", _whole=False):
    """qpp::applyTFQ(A, target, d, swap), operations.hpp:2680-2787: the
    adjoint of applyQFT, gate by gate in the reverse order (SWAPs first)."""
    a = _cplx(state)
    dims = _check_qft(_where, a, list(target), d, _whole)
    if _whole:
        target = list(range(len(dims)))
    out = a
    k = len(target)
    if swap:
        for i in reversed(range(k // 2)):
            out = apply(out, _swapd(d), [target[i], target[k - i - 1]], dims)
    for i in reversed(range(k)):
        for j in reversed(range(2, k - i + 1)):
            out = applyCTRL(out, _rj(d, j, -1.0), [target[i + j - 1]], [target[i]], dims)
        out = apply(out, _fd(d).conj().T, [target[i]], dims)
    return out


def QFT(state, d=2, swap=True):
    """qpp::QFT(A, d, swap), operations.hpp:2792-2826: applyQFT on every
    subsystem in order."""
    return applyQFT(state, [], d, swap, _where="qpp::QFT()", _whole=True)


def TFQ(state, d=2, swap=True):
    """qpp::TFQ(A, d, swap), operations.hpp:2844-2878."""
    return applyTFQ(state, [], d, swap, _where="qpp::TFQ()", _whole=True)
