"""qpp_b200 -- B200-native Quantum++ gate-application and subsystem path.

Python host mirror of the C ABI in include/qpp_b200.h (libqpp_b200.so,
built in-tree for sm_100a). The free functions keep Quantum++'s names,
argument meaning and value semantics (include/qpp/operations.hpp):

    apply(state, A, target, dims)                       operations.hpp:72
    applyCTRL(state, A, ctrl, target, dims, shift)      operations.hpp:616
    applyCTRL_fan(state, A, ctrl, target, dims, shift)  operations.hpp:961
    apply_kraus(rho, Ks, target, dims)                  operations.hpp:476
    ptrace(state, target, dims)                         operations.hpp:1908
    ptranspose(state, target, dims)                     operations.hpp:2167
    syspermute(state, perm, dims)                       operations.hpp:2386

Errors raise the qpp exception type of the same name (ZeroSize,
DimsInvalid, SubsysMismatchDims, ...) with qpp's (where, what) text.
`State` is the resident form: a ket or density matrix kept in HBM, mutated
in place by its methods. There is no CPU fallback: importing on a machine
without the built library raises, and every op needs a B200.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqpp_b200.so")

u64p = ct.POINTER(ct.c_uint64)
dp = ct.POINTER(ct.c_double)
vp = ct.c_void_p

KET, RHO = 0, 1
C128, C64 = 0, 1

_STATUS = {
    1: "ZeroSize", 2: "MatrixNotSquare", 3: "MatrixNotSquareNorCvector",
    4: "MatrixMismatchSubsys", 5: "DimsInvalid", 6: "DimsNotEqual",
    7: "DimsMismatchMatrix", 8: "DimsMismatchCvector", 9: "SubsysMismatchDims",
    10: "PermInvalid", 11: "PermMismatchDims", 12: "OutOfRange",
    13: "TypeMismatch", 14: "SizeMismatch", 15: "QuditAlreadyMeasured",
    16: "MatrixNotSquareNorVector", 17: "DivisionByZero", 18: "Duplicates", 100: "CudaError",
    101: "OutOfMemory", 102: "Timeout", 103: "InvalidHandle",
    104: "NotSupported", 105: "InvalidArgument",
}


class QppError(RuntimeError):
    """Base of the qpp exception mirror (include/qpp/classes/exception.hpp)."""

    def __init__(self, code, where, what):
        super().__init__(f"{where}: {what}")
        self.code, self.where, self.what = code, where, what


_EXC = {code: type(name, (QppError,), {}) for code, name in _STATUS.items()}
globals().update({cls.__name__: cls for cls in _EXC.values()})

_lib = None


def lib():
    """The loaded libqpp_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`make -C qpp_b200` (nvcc, sm_100a)")
        L = ct.CDLL(LIB_PATH)
        L.qgpu_last_error_where.restype = ct.c_char_p
        L.qgpu_last_error_what.restype = ct.c_char_p
        L.qgpu_version.restype = ct.c_char_p
        L.qgpu_status_name.restype = ct.c_char_p
        L.qgpu_ctx_launch_count.restype = ct.c_uint64
        L.qgpu_ctx_stream.restype = vp
        L.qgpu_state_device_ptr.restype = vp
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        L = lib()
        where = L.qgpu_last_error_where().decode()
        what = L.qgpu_last_error_what().decode()
        raise _EXC.get(rc, QppError)(rc, where, what)


def _u64(v):
    if v is None:
        return None, None, 0
    a = np.ascontiguousarray(np.asarray(list(v), dtype=np.uint64).reshape(-1))
    if a.size == 0:
        a = np.zeros(1, dtype=np.uint64)
        return a, a.ctypes.data_as(u64p), 0
    return a, a.ctypes.data_as(u64p), a.size


def _mat(A):
    A = np.asfortranarray(np.asarray(A, dtype=np.complex128))
    if A.ndim == 1:
        A = A.reshape(-1, 1, order="F")
    return A


def _host_state(state):
    a = np.asarray(state, dtype=np.complex128)
    if a.ndim == 1:
        return np.ascontiguousarray(a), a.shape[0], 1, True
    return np.asfortranarray(a), a.shape[0], a.shape[1], False


def _dp(a):
    return a.ctypes.data_as(dp)


class Context:
    """A CUDA device plus the stream all ops on it are issued on."""

    def __init__(self, device=0):
        self.h = vp()
        check(lib().qgpu_ctx_create(ct.c_int(device), ct.byref(self.h)))
        self.device = device

    def synchronize(self):
        check(lib().qgpu_ctx_synchronize(self.h))

    def launches(self):
        return int(lib().qgpu_ctx_launch_count(self.h))

    def stream(self):
        return lib().qgpu_ctx_stream(self.h)

    def mem_info(self):
        f, t = ct.c_uint64(), ct.c_uint64()
        check(lib().qgpu_ctx_mem_info(self.h, ct.byref(f), ct.byref(t)))
        return f.value, t.value

    def close(self):
        if self.h:
            check(lib().qgpu_ctx_destroy(self.h))
            self.h = None


_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class State:
    """A ket (kind=KET) or density matrix (kind=RHO) resident in HBM."""

    def __init__(self, ctx, kind, dims, prec=C128, handle=None):
        self.ctx = ctx
        if handle is None:
            handle = vp()
            d, dpp, nd = _u64(dims)
            check(lib().qgpu_state_create(ctx.h, ct.c_int(kind), ct.c_int(prec), dpp,
                                          ct.c_uint32(nd), ct.byref(handle)))
        self.h = handle
        self._info()

    def _info(self):
        k, p, n, D = ct.c_int(), ct.c_int(), ct.c_uint32(), ct.c_uint64()
        check(lib().qgpu_state_info(self.h, ct.byref(k), ct.byref(p), ct.byref(n), None,
                                    ct.byref(D)))
        dims = np.zeros(max(n.value, 1), dtype=np.uint64)
        check(lib().qgpu_state_info(self.h, None, None, None, dims.ctypes.data_as(u64p), None))
        self.kind, self.prec, self.D = k.value, p.value, D.value
        self.dims = [int(x) for x in dims[: n.value]]

    @classmethod
    def from_numpy(cls, ctx, arr, dims, prec=C128):
        a = np.asarray(arr, dtype=np.complex128)
        kind = KET if a.ndim == 1 or (a.ndim == 2 and a.shape[1] == 1) else RHO
        s = cls(ctx, kind, dims, prec)
        s.upload(a)
        return s

    def upload(self, arr):
        a = np.asarray(arr, dtype=np.complex128)
        a = np.ascontiguousarray(a.reshape(-1)) if self.kind == KET else np.asfortranarray(a)
        check(lib().qgpu_state_upload_c128(self.h, _dp(a)))

    def numpy(self):
        n = self.D if self.kind == KET else self.D * self.D
        out = np.zeros(n, dtype=np.complex128)
        check(lib().qgpu_state_download_c128(self.h, _dp(out)))
        if self.kind == KET:
            return out
        return out.reshape((self.D, self.D), order="F")

    def device_ptr(self):
        return lib().qgpu_state_device_ptr(self.h)

    def fill_gaussian(self, seed):
        """i.i.d. complex Gaussian entries (Philox4x32-10 keyed by seed),
        normalised."""
        check(lib().qgpu_state_fill_gaussian(self.h, ct.c_uint64(seed)))
        return self

    def convert_from(self, other):
        check(lib().qgpu_state_convert(other.h, self.h))
        return self

    # resident (in-place) ops
    def apply(self, A, target):
        A = _mat(A)
        t, tp, nt = _u64(target)
        check(lib().qgpu_apply(self.h, _dp(A), ct.c_uint64(A.shape[0]), tp, ct.c_uint32(nt)))
        return self

    def apply_ctrl(self, A, ctrl, target, shift=None, fan=False):
        A = _mat(A)
        c, cp, nc = _u64(ctrl)
        t, tp, nt = _u64(target)
        s, sp, _ = _u64(shift)
        fn = lib().qgpu_apply_ctrl_fan if fan else lib().qgpu_apply_ctrl
        check(fn(self.h, _dp(A), ct.c_uint64(A.shape[0]), cp, ct.c_uint32(nc), tp,
                 ct.c_uint32(nt), sp))
        return self

    def apply_kraus(self, Ks, target):
        packed, DA = _pack_kraus(Ks)
        t, tp, nt = _u64(target)
        check(lib().qgpu_apply_kraus(self.h, _dp(packed), ct.c_uint32(len(Ks)),
                                     ct.c_uint64(DA), tp, ct.c_uint32(nt)))
        return self

    def ptrace(self, target):
        t, tp, nt = _u64(target)
        h = vp()
        check(lib().qgpu_ptrace(self.h, tp, ct.c_uint32(nt), ct.byref(h)))
        return State(self.ctx, RHO, None, handle=h)

    def ptranspose(self, target):
        t, tp, nt = _u64(target)
        h = vp()
        check(lib().qgpu_ptranspose(self.h, tp, ct.c_uint32(nt), ct.byref(h)))
        return State(self.ctx, RHO, None, handle=h)

    def syspermute(self, perm):
        p, pp, npm = _u64(perm)
        h = vp()
        check(lib().qgpu_syspermute(self.h, pp, ct.c_uint32(npm), ct.byref(h)))
        return State(self.ctx, self.kind, None, handle=h)

    def apply_qft(self, target, d=2, swap=True):
        """qpp::applyQFT on the resident state, in place."""
        t, tp, nt = _u64(target)
        check(lib().qgpu_apply_qft(self.h, tp, ct.c_uint32(nt), ct.c_uint64(d),
                                   ct.c_int(int(swap)), ct.c_int(0)))
        return self

    def apply_tfq(self, target, d=2, swap=True):
        """qpp::applyTFQ on the resident state, in place."""
        t, tp, nt = _u64(target)
        check(lib().qgpu_apply_qft(self.h, tp, ct.c_uint32(nt), ct.c_uint64(d),
                                   ct.c_int(int(swap)), ct.c_int(1)))
        return self

    def qft(self, d=2, swap=True, inverse=False):
        """qpp::QFT / TFQ (inverse) on every subsystem of the resident state."""
        check(lib().qgpu_qft(self.h, ct.c_uint64(d), ct.c_int(int(swap)),
                             ct.c_int(int(inverse))))
        return self

    def norm2(self):
        v = ct.c_double()
        check(lib().qgpu_norm2(self.h, ct.byref(v)))
        return v.value

    def trace(self):
        r, i = ct.c_double(), ct.c_double()
        check(lib().qgpu_trace(self.h, ct.byref(r), ct.byref(i)))
        return complex(r.value, i.value)

    def normalize(self):
        check(lib().qgpu_normalize(self.h))
        return self

    def inner(self, other):
        r, i = ct.c_double(), ct.c_double()
        check(lib().qgpu_inner(self.h, other.h, ct.byref(r), ct.byref(i)))
        return complex(r.value, i.value)

    def clone(self):
        h = vp()
        check(lib().qgpu_state_clone(self.h, ct.byref(h)))
        return State(self.ctx, self.kind, None, handle=h)

    def sample_draws(self, target, num_samples, seed=0, u=None):
        """qpp::sample(num_samples, ...) draws in order: an array of
        num_samples x len(target) digits (std::mt19937(seed), or the given
        uniforms u)."""
        t, tp, nt = _u64(target)
        out = np.zeros(max(num_samples * nt, 1), dtype=np.uint64)
        up = None
        if u is not None:
            u = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
            up = _dp(u)
        check(lib().qgpu_sample(self.h, tp, ct.c_uint32(nt), ct.c_uint64(num_samples),
                                ct.c_uint64(seed), up, out.ctypes.data_as(u64p)))
        return out[: num_samples * nt].reshape(num_samples, nt).astype(np.int64)

    def sample(self, target, num_samples, seed=0, u=None):
        """qpp::sample(num_samples, A, target, dims): {outcome tuple: count}."""
        res = {}
        for row in self.sample_draws(target, num_samples, seed, u):
            key = tuple(int(x) for x in row)
            res[key] = res.get(key, 0) + 1
        return res

    def _measure_out(self, fn, n, *args):
        res = ct.c_uint64()
        probs = np.zeros(max(n, 1), dtype=np.float64)
        outs = (vp * max(n, 1))()
        check(fn(*args, ct.byref(res), _dp(probs), outs))
        states = [State(self.ctx, KET, None, handle=vp(outs[i])) if outs[i] else None
                  for i in range(n)]
        return int(res.value), [float(x) for x in probs[:n]], states

    def measure_kraus(self, Ks, target, destructive=True, seed=0):
        """qpp::measure(A, Ks, target, dims, destructive): (result, probs,
        post-measurement States, None where the probability is 0)."""
        packed, DA = _pack_kraus(Ks)
        t, tp, nt = _u64(target)
        return self._measure_out(lib().qgpu_measure_kraus, len(Ks), self.h, _dp(packed),
                                 ct.c_uint32(len(Ks)), ct.c_uint64(DA), tp, ct.c_uint32(nt),
                                 ct.c_int(1 if destructive else 0), ct.c_uint64(seed))

    def measure_basis(self, V, target, destructive=True, seed=0):
        """qpp::measure(A, V, target, dims, destructive) with the columns of V."""
        V = _mat(V)
        t, tp, nt = _u64(target)
        return self._measure_out(lib().qgpu_measure_basis, V.shape[1], self.h, _dp(V),
                                 ct.c_uint64(V.shape[0]), ct.c_uint64(V.shape[1]), tp,
                                 ct.c_uint32(nt), ct.c_int(1 if destructive else 0),
                                 ct.c_uint64(seed))

    def reset(self, target, seed=0):
        """qpp::reset(A, target, dims): a new State."""
        t, tp, nt = _u64(target)
        h = vp()
        check(lib().qgpu_reset(self.h, tp, ct.c_uint32(nt), ct.c_uint64(seed), ct.byref(h)))
        return State(self.ctx, self.kind, None, handle=h)

    def discard(self, target, seed=0):
        """qpp::discard(A, target, dims): a new State."""
        t, tp, nt = _u64(target)
        h = vp()
        check(lib().qgpu_discard(self.h, tp, ct.c_uint32(nt), ct.c_uint64(seed), ct.byref(h)))
        return State(self.ctx, self.kind, None, handle=h)

    def measure_seq(self, target, destructive=True, seed=0, forced=None):
        """qpp::measure_seq(A, target, dims, destructive): (results, probs,
        post-measurement State); this state is unchanged."""
        t, tp, nt = _u64(target)
        f, fp, _ = _u64(forced)
        res = np.zeros(max(nt, 1), dtype=np.uint64)
        probs = np.zeros(max(nt, 1), dtype=np.float64)
        h = vp()
        check(lib().qgpu_measure_seq(self.h, tp, ct.c_uint32(nt), ct.c_int(1 if destructive else 0),
                                     ct.c_uint64(seed), fp, res.ctypes.data_as(u64p), _dp(probs),
                                     ct.byref(h)))
        return ([int(x) for x in res[:nt]], [float(x) for x in probs[:nt]],
                State(self.ctx, self.kind, None, handle=h))

    def free(self):
        if self.h:
            check(lib().qgpu_state_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            if self.h and lib() is not None:
                lib().qgpu_state_destroy(self.h)
                self.h = None
        except Exception:
            pass


def _pack_kraus(Ks):
    Ks = [_mat(K) for K in Ks]
    if not Ks:
        return np.zeros(1, dtype=np.complex128), 0
    packed = np.ascontiguousarray(np.concatenate([K.reshape(-1, order="F") for K in Ks]))
    return packed, Ks[0].shape[0]


# ------------------------------------------ value-semantics free functions
def apply(state, A, target, dims, ctx=None):
    """qpp::apply(state, A, target, dims) (operations.hpp:72-372)."""
    ctx = ctx or default_context()
    s, rows, cols, one_d = _host_state(state)
    A = _mat(A)
    t, tp, nt = _u64(target)
    d, dpp, nd = _u64(dims)
    out = np.zeros(s.shape, dtype=np.complex128, order="F")
    check(lib().qgpu_host_apply(ctx.h, _dp(s), ct.c_uint64(rows), ct.c_uint64(cols), _dp(A),
                                ct.c_uint64(A.shape[0]), ct.c_uint64(A.shape[1]), tp,
                                ct.c_uint32(nt), dpp, ct.c_uint32(nd), _dp(out)))
    return out


def applyCTRL(state, A, ctrl, target, dims, shift=None, ctx=None, fan=False):
    """qpp::applyCTRL(state, A, ctrl, target, dims, shift) (operations.hpp:616)."""
    ctx = ctx or default_context()
    s, rows, cols, one_d = _host_state(state)
    A = _mat(A)
    c, cp, nc = _u64(ctrl)
    t, tp, nt = _u64(target)
    d, dpp, nd = _u64(dims)
    sh, sp, _ = _u64(shift)
    out = np.zeros(s.shape, dtype=np.complex128, order="F")
    check(lib().qgpu_host_apply_ctrl(ctx.h, _dp(s), ct.c_uint64(rows), ct.c_uint64(cols),
                                     _dp(A), ct.c_uint64(A.shape[0]), ct.c_uint64(A.shape[1]),
                                     cp, ct.c_uint32(nc), tp, ct.c_uint32(nt), dpp,
                                     ct.c_uint32(nd), sp, ct.c_int(1 if fan else 0), _dp(out)))
    return out


def applyCTRL_fan(state, A, ctrl, target, dims, shift=None, ctx=None):
    """qpp::applyCTRL_fan(state, A, ctrl, target, dims, shift) (operations.hpp:961)."""
    return applyCTRL(state, A, ctrl, target, dims, shift, ctx=ctx, fan=True)


def apply_kraus(rho, Ks, target, dims, ctx=None):
    """qpp::apply(A, Ks, target, dims) (operations.hpp:476-560)."""
    ctx = ctx or default_context()
    s, rows, cols, one_d = _host_state(rho)
    Kl = [_mat(K) for K in Ks]
    packed, _ = _pack_kraus(Kl)
    kr, kc = (Kl[0].shape if Kl else (0, 0))
    t, tp, nt = _u64(target)
    d, dpp, nd = _u64(dims)
    out = np.zeros((rows, cols), dtype=np.complex128, order="F")
    check(lib().qgpu_host_apply_kraus(ctx.h, _dp(s), ct.c_uint64(rows), ct.c_uint64(cols),
                                      _dp(packed), ct.c_uint32(len(Kl)), ct.c_uint64(kr),
                                      ct.c_uint64(kc), tp, ct.c_uint32(nt), dpp,
                                      ct.c_uint32(nd), _dp(out)))
    return out


def ptrace(state, target, dims, ctx=None):
    """qpp::ptrace(A, target, dims) (operations.hpp:1908-2114)."""
    ctx = ctx or default_context()
    s, rows, cols, one_d = _host_state(state)
    t, tp, nt = _u64(target)
    d, dpp, nd = _u64(dims)
    DS = 1
    for i in (target or []):
        if 0 <= int(i) < len(dims):
            DS *= int(dims[int(i)])
    Db = max(rows // DS, 1) if rows % DS == 0 else 1
    out = np.zeros((Db, Db), dtype=np.complex128, order="F")
    check(lib().qgpu_host_ptrace(ctx.h, _dp(s), ct.c_uint64(rows), ct.c_uint64(cols), tp,
                                 ct.c_uint32(nt), dpp, ct.c_uint32(nd), _dp(out)))
    return out


def ptranspose(state, target, dims, ctx=None):
    """qpp::ptranspose(A, target, dims) (operations.hpp:2167-2335)."""
    ctx = ctx or default_context()
    s, rows, cols, one_d = _host_state(state)
    t, tp, nt = _u64(target)
    d, dpp, nd = _u64(dims)
    out = np.zeros((rows, rows), dtype=np.complex128, order="F")
    check(lib().qgpu_host_ptranspose(ctx.h, _dp(s), ct.c_uint64(rows), ct.c_uint64(cols), tp,
                                     ct.c_uint32(nt), dpp, ct.c_uint32(nd), _dp(out)))
    return out


def syspermute(state, perm, dims, ctx=None):
    """qpp::syspermute(A, perm, dims) (operations.hpp:2386-2514)."""
    ctx = ctx or default_context()
    s, rows, cols, one_d = _host_state(state)
    p, pp, npm = _u64(perm)
    d, dpp, nd = _u64(dims)
    out = np.zeros(s.shape, dtype=np.complex128, order="F")
    check(lib().qgpu_host_syspermute(ctx.h, _dp(s), ct.c_uint64(rows), ct.c_uint64(cols), pp,
                                     ct.c_uint32(npm), dpp, ct.c_uint32(nd), _dp(out)))
    return out


def _host_qft(state, target, d, swap, inverse, ctx):
    ctx = ctx or default_context()
    s, rows, cols, one_d = _host_state(state)
    out = np.zeros(s.shape, dtype=np.complex128, order="F")
    if target is None:
        check(lib().qgpu_host_qft(ctx.h, _dp(s), ct.c_uint64(rows), ct.c_uint64(cols),
                                  ct.c_uint64(d), ct.c_int(int(swap)), ct.c_int(int(inverse)),
                                  _dp(out)))
    else:
        t, tp, nt = _u64(target)
        check(lib().qgpu_host_apply_qft(ctx.h, _dp(s), ct.c_uint64(rows), ct.c_uint64(cols), tp,
                                        ct.c_uint32(nt), ct.c_uint64(d), ct.c_int(int(swap)),
                                        ct.c_int(int(inverse)), _dp(out)))
    return out


def applyQFT(state, target, d=2, swap=True, ctx=None):
    """qpp::applyQFT(A, target, d, swap) (operations.hpp:2565-2676)."""
    return _host_qft(state, target, d, swap, False, ctx)


def applyTFQ(state, target, d=2, swap=True, ctx=None):
    """qpp::applyTFQ(A, target, d, swap) (operations.hpp:2680-2787)."""
    return _host_qft(state, target, d, swap, True, ctx)


def QFT(state, d=2, swap=True, ctx=None):
    """qpp::QFT(A, d, swap) (operations.hpp:2792-2826)."""
    return _host_qft(state, None, d, swap, False, ctx)


def TFQ(state, d=2, swap=True, ctx=None):
    """qpp::TFQ(A, d, swap) (operations.hpp:2844-2878)."""
    return _host_qft(state, None, d, swap, True, ctx)


# ------------------------------------------------------------------ circuits
PLAIN, FUSED = 0, 1


class Circuit:
    """Step list of qpp::QCircuit (include/qpp/classes/qcircuit.hpp): gates,
    fan gates, (classically) controlled gates and Z-basis measurements."""

    def __init__(self, nq, d=2, nc=0):
        self.h = vp()
        check(lib().qgpu_circuit_create(ct.c_uint32(nq), ct.c_uint64(d), ct.c_uint32(nc),
                                        ct.byref(self.h)))
        self.nq, self.d, self.nc = nq, d, nc

    def gate(self, U, target):
        U = _mat(U)
        t, tp, nt = _u64(target)
        check(lib().qgpu_circuit_gate(self.h, _dp(U), ct.c_uint64(U.shape[0]), tp, ct.c_uint32(nt)))
        return self

    def gate_fan(self, U, target):
        U = _mat(U)
        t, tp, nt = _u64(target)
        check(lib().qgpu_circuit_gate_fan(self.h, _dp(U), ct.c_uint64(U.shape[0]), tp,
                                          ct.c_uint32(nt)))
        return self

    def CTRL(self, U, ctrl, target, shift=None, fan=False):
        U = _mat(U)
        c, cp, nc = _u64(ctrl)
        t, tp, nt = _u64(target)
        s, sp, _ = _u64(shift)
        check(lib().qgpu_circuit_ctrl(self.h, _dp(U), ct.c_uint64(U.shape[0]), cp, ct.c_uint32(nc),
                                      tp, ct.c_uint32(nt), sp, ct.c_int(1 if fan else 0)))
        return self

    def cCTRL(self, U, ctrl_dits, target, shift=None, fan=False):
        U = _mat(U)
        c, cp, nc = _u64(ctrl_dits)
        t, tp, nt = _u64(target)
        s, sp, _ = _u64(shift)
        check(lib().qgpu_circuit_cctrl(self.h, _dp(U), ct.c_uint64(U.shape[0]), cp,
                                       ct.c_uint32(nc), tp, ct.c_uint32(nt), sp,
                                       ct.c_int(1 if fan else 0)))
        return self

    @classmethod
    def from_qasm(cls, source):
        """qpp::qasm::read_from_string: an OpenQASM 2.0 program as a Circuit."""
        h = vp()
        check(lib().qgpu_qasm_read(source.encode(), ct.byref(h)))
        return cls._wrap(h)

    @classmethod
    def from_qasm_file(cls, path):
        """qpp::qasm::read_from_file."""
        h = vp()
        check(lib().qgpu_qasm_read_file(str(path).encode(), ct.byref(h)))
        return cls._wrap(h)

    @classmethod
    def _wrap(cls, h):
        c = cls.__new__(cls)
        c.h = h
        nq, d, nc = ct.c_uint32(), ct.c_uint64(), ct.c_uint32()
        check(lib().qgpu_circuit_shape(h, ct.byref(nq), ct.byref(d), ct.byref(nc)))
        c.nq, c.d, c.nc = nq.value, d.value, nc.value
        return c

    def reset(self, target):
        t, tp, nt = _u64(target if isinstance(target, (list, tuple)) else [target])
        check(lib().qgpu_circuit_reset(self.h, tp, ct.c_uint32(nt)))
        return self

    def cond_if(self, dits, value):
        """Steps until cond_end() run only when the dits (dits[0] the least
        significant bit) spell `value`."""
        d, dp_, nd = _u64(dits)
        check(lib().qgpu_circuit_cond_if(self.h, dp_, ct.c_uint32(nd), ct.c_uint64(value)))
        return self

    def QFT(self, target=None, swap=True):
        """QCircuit::QFT(target, swap); target None = every qudit not yet measured."""
        if target is None:
            check(lib().qgpu_circuit_qft(self.h, None, ct.c_uint32(0), ct.c_int(int(swap)),
                                         ct.c_int(0)))
        else:
            t, tp, nt = _u64(target)
            check(lib().qgpu_circuit_qft(self.h, tp, ct.c_uint32(nt), ct.c_int(int(swap)),
                                         ct.c_int(0)))
        return self

    def TFQ(self, target=None, swap=True):
        """QCircuit::TFQ(target, swap)."""
        if target is None:
            check(lib().qgpu_circuit_qft(self.h, None, ct.c_uint32(0), ct.c_int(int(swap)),
                                         ct.c_int(1)))
        else:
            t, tp, nt = _u64(target)
            check(lib().qgpu_circuit_qft(self.h, tp, ct.c_uint32(nt), ct.c_int(int(swap)),
                                         ct.c_int(1)))
        return self

    def cond_end(self):
        check(lib().qgpu_circuit_cond_end(self.h))
        return self

    def measure(self, target, c_reg=0, destructive=True):
        t, tp, nt = _u64(target if isinstance(target, (list, tuple)) else [target])
        check(lib().qgpu_circuit_measure(self.h, tp, ct.c_uint32(nt), ct.c_uint64(c_reg),
                                         ct.c_int(1 if destructive else 0)))
        return self

    def steps(self):
        n = ct.c_uint64()
        check(lib().qgpu_circuit_info(self.h, None, ct.byref(n)))
        return n.value

    def fused_passes(self, max_k=6):
        """Entries of the fused plan with blocks of <= max_k qubits: the
        merged blocks and the steps left as they are (host planning only)."""
        n = ct.c_uint64()
        check(lib().qgpu_circuit_fuse(self.h, ct.c_uint32(max_k), ct.byref(n)))
        return n.value

    def run(self, state, form=PLAIN):
        """Apply the unitary steps to a resident State (in place). PLAIN keeps
        qpp's arithmetic per gate. FUSED merges gates into blocks: on a
        complex64 qubit ket of <= 6 qubits each (the tensor cores from 13
        qubits), on a complex128 qubit ket of <= 2 qubits run as tile passes
        (up to 22 qubits) or <= 3 qubits as dense passes (above); on a
        complex64 qubit density matrix, gates and channels as superoperator
        blocks of <= 4 virtual qubits (6 on the tensor cores from 11
        qubits)."""
        check(lib().qgpu_run_gates(state.h, self.h, ct.c_int(form)))
        return state

    def __del__(self):
        try:
            if self.h:
                lib().qgpu_circuit_destroy(self.h)
                self.h = None
        except Exception:
            pass


def apply_tc(state, U, target):
    """One <= 6-qubit gate on a complex64 ket as a 64 x 64 tensor-core block."""
    U = _mat(U)
    t, tp, nt = _u64(target)
    check(lib().qgpu_apply_tc(state.h, _dp(U), tp, ct.c_uint32(nt)))
    return state


def batch_last_phases(ctx):
    """Milliseconds of the last run_batch on ctx: compile, build (upload +
    graph capture), graph device time, plain-form instances."""
    out = (ct.c_double * 6)()
    check(lib().qgpu_batch_last_phases(ctx.h, out))
    return {"compile_ms": out[0], "build_ms": out[1], "graph_device_ms": out[2],
            "plain_ms": out[3], "check_ms": out[4], "teardown_ms": out[5]}


def traj_fusion_width(ctx, n, w=None):
    """Fusion width (2-4) of batched registers of n qubits: the tuned choice,
    or pin w (w=-2 drops the choice so it is timed again)."""
    out = ct.c_int()
    check(lib().qgpu_traj_fusion_width(ctx.h, ct.c_uint32(n), ct.c_int(-1 if w is None else w),
                                       ct.byref(out)))
    return out.value


def traj_tile_width(ctx, n, T=None):
    """Tile width of the trajectory kernel for n-qubit registers (15-22):
    T=None queries (tuned on first use), 0 pins the untiled form, 9..14
    pins a width, -2 drops the choice. Returns the width in force."""
    out = ct.c_int()
    check(lib().qgpu_traj_tile_width(ctx.h, ct.c_uint32(n), ct.c_int(-1 if T is None else T),
                                     ct.byref(out)))
    return out.value


def run_batch(ctx, circuits, states, form=FUSED):
    """Independent instances circuits[i] on states[i] (in place): FUSED runs
    every complex64 instance that compiles as one CUDA-graph launch, PLAIN
    loops with one launch per gate. Returns the kernels in the graph."""
    n = len(circuits)
    C = (vp * n)(*[c.h for c in circuits])
    S = (vp * n)(*[s.h for s in states])
    k = ct.c_uint64()
    check(lib().qgpu_run_batch(ctx.h, ct.c_uint32(n), C, S, ct.c_int(form), ct.byref(k)))
    return k.value


def layered_circuit(n, depth, seed):
    """The seeded layered circuit of qpp_b200.workloads as a Circuit."""
    from . import workloads
    c = Circuit(n)
    for layer in workloads.layered_circuit(n, depth, seed):
        for U, t in layer:
            c.gate(U, t)
    return c


# ------------------------------------------------------------------- engines
class Engine:
    """QEngine (kind=KET) / QDensityEngine (kind=RHO) / QNoisyEngine (after
    set_noise) over a Circuit, state resident in HBM
    (include/qpp/classes/qengine.hpp, qnoisy_engine.hpp)."""

    def __init__(self, ctx, circuit, kind=KET, prec=C128):
        self.h = vp()
        self.ctx, self.circuit = ctx, circuit
        check(lib().qgpu_engine_create(ctx.h, circuit.h, ct.c_int(kind), ct.c_int(prec),
                                       ct.byref(self.h)))

    def set_seed(self, seed):
        check(lib().qgpu_engine_set_seed(self.h, ct.c_uint64(seed)))
        return self

    def set_noise(self, Ks, probs=None):
        """A Kraus list (+ probabilities; None: state-dependent), or one of
        the models of qpp_b200.noise."""
        if hasattr(Ks, "Ks"):
            Ks, probs = Ks.Ks, Ks.probs
        packed, d = _pack_kraus(Ks)
        pr = None if probs is None else np.ascontiguousarray(np.asarray(probs, dtype=np.float64))
        check(lib().qgpu_engine_set_noise(self.h, _dp(packed), ct.c_uint32(len(Ks)),
                                          ct.c_uint64(d), None if pr is None else _dp(pr)))
        return self

    def set_state(self, state):
        check(lib().qgpu_engine_set_state(self.h, state.h))
        return self

    def set_replay(self, outcomes=None, noise=None):
        o, op, no = _u64(outcomes) if outcomes is not None else (None, None, 0)
        k, kp, nk = _u64(noise) if noise is not None else (None, None, 0)
        check(lib().qgpu_engine_set_replay(self.h, op, ct.c_uint64(no), kp, ct.c_uint64(nk)))
        return self

    def reset(self, reset_stats=True):
        """State back to |0...0>, registers cleared (statistics too unless
        reset_stats is False)."""
        check(lib().qgpu_engine_reset(self.h, ct.c_int(1 if reset_stats else 0)))
        return self

    def execute(self, reps=1):
        """qpp's execute(reps): from the engine's current state; the engine
        keeps the first repetition's state and dits; statistics accumulate
        until reset()."""
        check(lib().qgpu_engine_execute(self.h, ct.c_uint64(reps)))
        return self

    def get_dits(self):
        nc = self.circuit.nc
        d = np.zeros(max(nc, 1), dtype=np.uint64)
        p = np.zeros(max(nc, 1), dtype=np.float64)
        check(lib().qgpu_engine_get_dits(self.h, d.ctypes.data_as(u64p), _dp(p)))
        return [int(x) for x in d[:nc]], [float(x) for x in p[:nc]]

    def get_state(self):
        h = vp()
        check(lib().qgpu_engine_get_state(self.h, ct.byref(h)))
        return State(self.ctx, KET, None, handle=h)

    def get_stats(self):
        n = ct.c_uint64()
        check(lib().qgpu_engine_get_stats(self.h, ct.byref(n), None, None))
        nc = self.circuit.nc
        counts = np.zeros(max(n.value, 1), dtype=np.uint64)
        outs = np.zeros(max(n.value * nc, 1), dtype=np.uint64)
        check(lib().qgpu_engine_get_stats(self.h, None, counts.ctypes.data_as(u64p),
                                          outs.ctypes.data_as(u64p)))
        return {tuple(int(x) for x in outs[i * nc:(i + 1) * nc]): int(counts[i])
                for i in range(n.value)}

    def get_record(self):
        no, nn = ct.c_uint64(), ct.c_uint64()
        check(lib().qgpu_engine_get_record(self.h, ct.byref(no), None, ct.byref(nn), None))
        o = np.zeros(max(no.value, 1), dtype=np.uint64)
        k = np.zeros(max(nn.value, 1), dtype=np.uint64)
        check(lib().qgpu_engine_get_record(self.h, None, o.ctypes.data_as(u64p), None,
                                           k.ctypes.data_as(u64p)))
        return [int(x) for x in o[:no.value]], [int(x) for x in k[:nn.value]]

    def __del__(self):
        try:
            if self.h:
                lib().qgpu_engine_destroy(self.h)
                self.h = None
        except Exception:
            pass
