// qpp_oracle.cpp -- CPU restatement of Quantum++ 7.0.3's gate-application and
// subsystem-manipulation path.
//
// TEST INFRASTRUCTURE ONLY. This file is the correctness oracle and the timed
// CPU baseline ("qpp-restatement (Eigen unavailable)"): Quantum++ itself needs
// Eigen >= 5.0 (cmake/qpp_eigen.cmake:9), which is absent on the build and GPU
// machines, so the reference cannot be compiled. Only tests/, the smoke check
// and the CPU-baseline leg of bench.py load this library; the product
// (qpp_b200/, libqpp_b200.so) never links or calls it.
//
// Parity is pinned by the known-answer tests of the reference's own suite
// (unit_tests/tests/operations.cpp:16-397, classes/gates.cpp:170-207,
// entropies.cpp:103-108, qasm/qasm.cpp:82-94), restated in
// tests/test_kats.py, and by dense Kronecker-expansion cross-checks.
//
// Layout: complex<double> interleaved, column-major, big-endian mixed radix
// (include/qpp/internal/util.hpp:58-116). Every function cites the reference
// code whose semantics (and, where it matters for timing, loop structure and
// OpenMP pragmas) it restates.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../include/qpp_b200.h"

using cplx = std::complex<double>;
using idx = uint64_t;

namespace {

constexpr idx kMaxN = 64; // internal::maxn, options.hpp:437

thread_local std::string g_where, g_what;

struct Fail {
    qgpu_status code;
    const char* where;
    const char* what;
};

int fail(const Fail& f) {
    g_where = f.where;
    g_what = f.what;
    return f.code;
}

// ---------------------------------------------------------------- helpers
// n2multiidx / multiidx2n: big-endian mixed radix (util.hpp:58-116).
inline void to_digits(idx v, idx n, const idx* dims, idx* out) {
    for (idx i = n; i-- > 0;) {
        out[i] = v % dims[i];
        v /= dims[i];
    }
}
inline idx from_digits(const idx* dig, idx n, const idx* dims) {
    idx r = 0, s = 1;
    for (idx i = n; i-- > 0;) {
        r += dig[i] * s;
        s *= dims[i];
    }
    return r;
}

// check_dims (util.hpp:158-166)
bool dims_ok(const std::vector<idx>& dims) {
    if (dims.empty()) return false;
    return std::find(dims.begin(), dims.end(), idx{0}) == dims.end();
}
idx prod(const std::vector<idx>& v) {
    idx p = 1;
    for (idx x : v) p *= x;
    return p;
}
// check_subsys_match_dims (util.hpp:233-252)
bool subsys_ok(const std::vector<idx>& s, const std::vector<idx>& dims) {
    if (s.size() > dims.size()) return false;
    std::vector<idx> t = s;
    std::sort(t.begin(), t.end());
    if (std::adjacent_find(t.begin(), t.end()) != t.end()) return false;
    for (idx x : s)
        if (x + 1 > dims.size()) return false;
    return true;
}
// check_perm (util.hpp:278-287)
bool perm_ok(const std::vector<idx>& p) {
    if (p.empty()) return false;
    std::vector<idx> t = p;
    std::sort(t.begin(), t.end());
    for (idx i = 0; i < t.size(); ++i)
        if (t[i] != i) return false;
    return true;
}
// complement(target, n), functions.hpp:1953: ascending order
std::vector<idx> complement_of(const std::vector<idx>& t, idx n) {
    std::vector<idx> r;
    for (idx i = 0; i < n; ++i)
        if (std::find(t.begin(), t.end(), i) == t.end()) r.push_back(i);
    return r;
}
bool all_two(const std::vector<idx>& dims) {
    for (idx d : dims)
        if (d != 2) return false;
    return true;
}

std::vector<idx> vec(const uint64_t* p, uint32_t n) {
    return p ? std::vector<idx>(p, p + n) : std::vector<idx>();
}
const cplx* C(const double* p) { return reinterpret_cast<const cplx*>(p); }
cplx* C(double* p) { return reinterpret_cast<cplx*>(p); }

// Dense matrix helpers (column-major).
using Mat = std::vector<cplx>;
Mat matmul(const Mat& a, const Mat& b, idx m) {
    Mat r(m * m, 0.0);
    for (idx j = 0; j < m; ++j)
        for (idx l = 0; l < m; ++l) {
            cplx blj = b[l + j * m];
            for (idx i = 0; i < m; ++i) r[i + j * m] += a[i + l * m] * blj;
        }
    return r;
}
// powm(A, k) (functions.hpp:838): A^0 = identity, repeated products.
Mat powm(const Mat& a, idx m, idx k) {
    Mat r(m * m, 0.0);
    for (idx i = 0; i < m; ++i) r[i + i * m] = 1.0;
    for (idx e = 0; e < k; ++e) r = matmul(r, a, m);
    return r;
}

// -------------------------------------------------------- shape validation
// The state-shape block shared by apply/ptrace/ptranspose/... :
// check_cvector -> dims match; square -> dims match; else NotSquareNorCvector.
int check_state_shape(idx rows, idx cols, const std::vector<idx>& dims,
                      const char* where, const char* what_cv,
                      const char* what_m, const char* what_nsq) {
    if (cols == 1) {
        if (prod(dims) != rows)
            return fail({QGPU_ERR_DIMS_MISMATCH_CVECTOR, where, what_cv});
    } else if (rows == cols) {
        if (prod(dims) != cols)
            return fail({QGPU_ERR_DIMS_MISMATCH_MATRIX, where, what_m});
    } else {
        return fail({QGPU_ERR_MATRIX_NOT_SQUARE_NOR_CVECTOR, where, what_nsq});
    }
    return 0;
}

// ------------------------------------------------ generic apply (qudits)
// operations.hpp:182-371: for every gate row m and complement index r, the
// output amplitude at (m, r) is sum_n A(m, n) * psi(n, r).
void generic_apply_ket(const cplx* psi, cplx* out, const cplx* A, idx DA,
                       const std::vector<idx>& target,
                       const std::vector<idx>& dims) {
    idx n = dims.size();
    idx D = prod(dims);
    std::vector<idx> bar = complement_of(target, n);
    idx k = target.size(), nb = bar.size();
    std::vector<idx> dA(k), dB(nb);
    for (idx i = 0; i < k; ++i) dA[i] = dims[target[i]];
    for (idx i = 0; i < nb; ++i) dB[i] = dims[bar[i]];
    idx DB = D / DA;
    std::memcpy(static_cast<void*>(out), psi, D * sizeof(cplx));
#pragma omp parallel for collapse(2)
    for (idx m = 0; m < DA; ++m)
        for (idx r = 0; r < DB; ++r) {
            idx mi[kMaxN], ma[kMaxN], mb[kMaxN];
            to_digits(r, nb, dB.data(), mb);
            for (idx t = 0; t < nb; ++t) mi[bar[t]] = mb[t];
            to_digits(m, k, dA.data(), ma);
            for (idx t = 0; t < k; ++t) mi[target[t]] = ma[t];
            idx dst = from_digits(mi, n, dims.data());
            cplx acc = 0;
            for (idx c = 0; c < DA; ++c) {
                to_digits(c, k, dA.data(), ma);
                for (idx t = 0; t < k; ++t) mi[target[t]] = ma[t];
                acc += A[m + c * DA] * psi[from_digits(mi, n, dims.data())];
            }
            out[dst] = acc;
        }
}

// operations.hpp:340-371: rho' = A rho A^dagger restricted to the target
// digits of both the row and the column index.
void generic_apply_rho(const cplx* rho, cplx* out, const cplx* A, idx DA,
                       const std::vector<idx>& target,
                       const std::vector<idx>& dims) {
    idx n = dims.size();
    idx D = prod(dims);
    std::vector<idx> bar = complement_of(target, n);
    idx k = target.size(), nb = bar.size();
    std::vector<idx> dA(k), dB(nb);
    for (idx i = 0; i < k; ++i) dA[i] = dims[target[i]];
    for (idx i = 0; i < nb; ++i) dB[i] = dims[bar[i]];
    idx DB = D / DA;
    std::memcpy(static_cast<void*>(out), rho, D * D * sizeof(cplx));
#pragma omp parallel for collapse(4)
    for (idx m1 = 0; m1 < DA; ++m1)
        for (idx r1 = 0; r1 < DB; ++r1)
            for (idx m2 = 0; m2 < DA; ++m2)
                for (idx r2 = 0; r2 < DB; ++r2) {
                    idx mr[kMaxN], mc[kMaxN], t1[kMaxN], t2[kMaxN];
                    to_digits(r1, nb, dB.data(), t1);
                    to_digits(r2, nb, dB.data(), t2);
                    for (idx t = 0; t < nb; ++t) {
                        mr[bar[t]] = t1[t];
                        mc[bar[t]] = t2[t];
                    }
                    to_digits(m1, k, dA.data(), t1);
                    to_digits(m2, k, dA.data(), t2);
                    for (idx t = 0; t < k; ++t) {
                        mr[target[t]] = t1[t];
                        mc[target[t]] = t2[t];
                    }
                    idx row = from_digits(mr, n, dims.data());
                    idx col = from_digits(mc, n, dims.data());
                    cplx acc = 0;
                    for (idx a = 0; a < DA; ++a) {
                        to_digits(a, k, dA.data(), t1);
                        for (idx t = 0; t < k; ++t) mr[target[t]] = t1[t];
                        idx rr = from_digits(mr, n, dims.data());
                        cplx lhs = A[m1 + a * DA];
                        for (idx b = 0; b < DA; ++b) {
                            to_digits(b, k, dA.data(), t2);
                            for (idx t = 0; t < k; ++t) mc[target[t]] = t2[t];
                            idx cc = from_digits(mc, n, dims.data());
                            // adjoint(A)(b, m2) = conj(A(m2, b))
                            cplx rhs = std::conj(A[m2 + b * DA]);
                            acc += lhs * rho[rr + cc * D] * rhs;
                        }
                    }
                    out[row + col * D] = acc;
                }
}

// ------------------------------------------- qubit kernels (timing paths)
// apply_psi_1q, internal/kernels/qubit/apply.hpp:57-126: copy, then pairs
// (k0, k0 + 2^j) with j = n - 1 - i, outer block loop parallel.
void qubit_apply_psi_1q(const cplx* psi, cplx* out, const cplx* A, idx i,
                        idx n) {
    idx D = idx{1} << n;
    std::memcpy(static_cast<void*>(out), psi, D * sizeof(cplx));
    idx j = n - 1 - i, step = idx{1} << j, jump = step << 1;
    cplx a00 = A[0], a10 = A[1], a01 = A[2], a11 = A[3];
#pragma omp parallel for
    for (idx L = 0; L < D; L += jump)
        for (idx R = 0; R < step; ++R) {
            idx k0 = L + R, k1 = k0 + step;
            cplx p0 = psi[k0], p1 = psi[k1];
            out[k0] = a00 * p0 + a01 * p1;
            out[k1] = a10 * p0 + a11 * p1;
        }
}

// apply_psi_2q, apply.hpp:139-265: copy, then 2^(n-2) groups; the base index
// is rebuilt bit by bit from the group index (skipping both target bits).
void qubit_apply_psi_2q(const cplx* psi, cplx* out, const cplx* A, idx qi,
                        idx qj, idx n) {
    idx D = idx{1} << n;
    std::memcpy(static_cast<void*>(out), psi, D * sizeof(cplx));
    idx pi = n - 1 - qi, pj = n - 1 - qj; // bit positions (LSB = 0)
    idx si = idx{1} << pi, sj = idx{1} << pj;
    idx Drem = D >> 2;
    cplx a[16];
    for (int t = 0; t < 16; ++t) a[t] = A[t];
#pragma omp parallel for
    for (idx b = 0; b < Drem; ++b) {
        idx k00 = 0, cur = 0;
        for (idx p = 0; p < n; ++p) {
            if (p == pi || p == pj) continue;
            if ((b >> cur) & 1) k00 |= idx{1} << p;
            ++cur;
        }
        idx k01 = k00 + sj, k10 = k00 + si, k11 = k00 + si + sj;
        cplx v0 = psi[k00], v1 = psi[k01], v2 = psi[k10], v3 = psi[k11];
        out[k00] = a[0] * v0 + a[4] * v1 + a[8] * v2 + a[12] * v3;
        out[k01] = a[1] * v0 + a[5] * v1 + a[9] * v2 + a[13] * v3;
        out[k10] = a[2] * v0 + a[6] * v1 + a[10] * v2 + a[14] * v3;
        out[k11] = a[3] * v0 + a[7] * v1 + a[11] * v2 + a[15] * v3;
    }
}

// ----------------------------------------------------- controlled gates
// Generic applyCTRL for kets, operations.hpp:777-821: for every r in [0, d),
// project on the control digits equal to (shift_inv + r) mod d, apply A^r on
// the target, and add the complement (psi / d - projection).
void generic_ctrl_ket(const cplx* psi, cplx* out, const std::vector<Mat>& Ak,
                      idx DA, const std::vector<idx>& ctrl,
                      const std::vector<idx>& target,
                      const std::vector<idx>& dims,
                      const std::vector<idx>& shift_inv, idx d, bool fan) {
    idx n = dims.size(), D = prod(dims);
    std::vector<cplx> result(D, 0.0), chopped(D), tmp(D);
    for (idx r = 0; r < d; ++r) {
        bool nonzero = false;
        for (idx i = 0; i < D; ++i) {
            idx dig[kMaxN];
            to_digits(i, n, dims.data(), dig);
            bool match = true;
            for (idx c = 0; c < ctrl.size(); ++c)
                if (dig[ctrl[c]] != (shift_inv[c] + r) % d) {
                    match = false;
                    break;
                }
            chopped[i] = match ? psi[i] : cplx(0.0);
            if (chopped[i] != cplx(0.0)) nonzero = true;
        }
        std::vector<cplx> bar(D);
        for (idx i = 0; i < D; ++i) bar[i] = psi[i] / static_cast<double>(d) - chopped[i];
        if (nonzero) {
            if (fan) {
                for (idx t : target) {
                    generic_apply_ket(chopped.data(), tmp.data(), Ak[r].data(),
                                      d, {t}, dims);
                    chopped.swap(tmp);
                }
            } else {
                generic_apply_ket(chopped.data(), tmp.data(), Ak[r].data(), DA,
                                  target, dims);
                chopped.swap(tmp);
            }
        }
        for (idx i = 0; i < D; ++i) result[i] += chopped[i] + bar[i];
    }
    std::memcpy(static_cast<void*>(out), result.data(), D * sizeof(cplx));
}

// Qubit-kernel semantics of applyCTRL on kets (apply_ctrl.hpp:63-509): a
// group whose control bits match (bit == 1 for shift 0, bit == 0 for shift 1)
// gets A; all other amplitudes are unchanged.
void qubit_ctrl_ket(const cplx* psi, cplx* out, const cplx* A, idx DA,
                    const std::vector<idx>& ctrl,
                    const std::vector<idx>& target,
                    const std::vector<idx>& shift_inv, idx n, bool fan) {
    idx D = idx{1} << n;
    idx ones = 0, zeros = 0;
    for (idx c = 0; c < ctrl.size(); ++c) {
        idx bit = idx{1} << (n - 1 - ctrl[c]);
        if (shift_inv[c] == 0) ones |= bit;
        else zeros |= bit;
    }
    std::memcpy(static_cast<void*>(out), psi, D * sizeof(cplx));
    std::vector<std::vector<idx>> tl;
    if (fan) {
        for (idx t : target) tl.push_back({t});
    } else {
        tl.push_back(target);
    }
    std::vector<cplx> cur(out, out + D);
    for (auto& tg : tl) {
        idx k = tg.size(), G = idx{1} << k;
        idx tmask = 0;
        for (idx t : tg) tmask |= idx{1} << (n - 1 - t);
#pragma omp parallel for
        for (idx base = 0; base < D; ++base) {
            if (base & tmask) continue;
            if ((base & ones) != ones || (base & zeros) != 0) continue;
            cplx v[64], w[64];
            idx off[64];
            for (idx m = 0; m < G; ++m) {
                idx o = 0;
                for (idx t = 0; t < k; ++t)
                    if ((m >> (k - 1 - t)) & 1) o |= idx{1} << (n - 1 - tg[t]);
                off[m] = o;
                v[m] = cur[base + o];
            }
            idx dm = fan ? 2 : DA;
            for (idx m = 0; m < G; ++m) {
                cplx acc = 0;
                for (idx c = 0; c < G; ++c) acc += A[m + c * dm] * v[c];
                w[m] = acc;
            }
            for (idx m = 0; m < G; ++m) out[base + off[m]] = w[m];
        }
        cur.assign(out, out + D);
    }
}

// ------------------------------------------------------------- ptrace
// operations.hpp:1908-2114: result(i, j) = sum_a A(i (+) a, j (+) a) over the
// traced digits a; for a ket, A(x, y) = psi(x) conj(psi(y)).
void generic_ptrace(const cplx* A, bool ket, cplx* out,
                    const std::vector<idx>& target,
                    const std::vector<idx>& dims) {
    idx n = dims.size(), D = prod(dims);
    idx k = target.size();
    std::vector<idx> bar = complement_of(target, n);
    idx nb = bar.size();
    std::vector<idx> dS(k), dB(nb);
    idx DS = 1;
    for (idx i = 0; i < k; ++i) {
        dS[i] = dims[target[i]];
        DS *= dS[i];
    }
    for (idx i = 0; i < nb; ++i) dB[i] = dims[bar[i]];
    idx DB = D / DS;
    if (k == n) {
        cplx s = 0;
        if (ket)
            for (idx i = 0; i < D; ++i) s += std::conj(A[i]) * A[i];
        else
            for (idx i = 0; i < D; ++i) s += A[i + i * D];
        out[0] = s;
        return;
    }
    if (k == 0) {
        if (ket)
            for (idx j = 0; j < D; ++j)
                for (idx i = 0; i < D; ++i) out[i + j * D] = A[i] * std::conj(A[j]);
        else
            std::memcpy(static_cast<void*>(out), A, D * D * sizeof(cplx));
        return;
    }
    for (idx j = 0; j < DB; ++j) {
        idx cb[kMaxN];
        to_digits(j, nb, dB.data(), cb);
#pragma omp parallel for
        for (idx i = 0; i < DB; ++i) {
            idx mr[kMaxN], mc[kMaxN], rb[kMaxN], sa[kMaxN];
            to_digits(i, nb, dB.data(), rb);
            for (idx t = 0; t < nb; ++t) {
                mr[bar[t]] = rb[t];
                mc[bar[t]] = cb[t];
            }
            cplx s = 0;
            for (idx a = 0; a < DS; ++a) {
                to_digits(a, k, dS.data(), sa);
                for (idx t = 0; t < k; ++t) mr[target[t]] = mc[target[t]] = sa[t];
                idx r = from_digits(mr, n, dims.data());
                idx c = from_digits(mc, n, dims.data());
                if (ket) s += A[r] * std::conj(A[c]);
                else s += A[r + c * D];
            }
            out[i + j * DB] = s;
        }
    }
}

// ---------------------------------------------------------- ptranspose
// operations.hpp:2167-2335: result(i, j) = A(i', j') where the target digits
// of i and j are exchanged; a ket input stands for |psi><psi|.
void generic_ptranspose(const cplx* A, bool ket, cplx* out,
                        const std::vector<idx>& target,
                        const std::vector<idx>& dims) {
    idx n = dims.size(), D = prod(dims);
    for (idx j = 0; j < D; ++j) {
        idx cj[kMaxN];
        to_digits(j, n, dims.data(), cj);
#pragma omp parallel for
        for (idx i = 0; i < D; ++i) {
            idx ri[kMaxN], cc[kMaxN];
            to_digits(i, n, dims.data(), ri);
            std::memcpy(cc, cj, n * sizeof(idx));
            for (idx t : target) std::swap(ri[t], cc[t]);
            idx r = from_digits(ri, n, dims.data());
            idx c = from_digits(cc, n, dims.data());
            out[i + j * D] = ket ? A[r] * std::conj(A[c]) : A[r + c * D];
        }
    }
}

// Qubit-kernel variant (internal/kernels/qubit/ptranspose.hpp:59-219): the
// mask is built little-endian (bit k for subsystem k), the density-matrix
// kernel reads rho(j_T, i_T) and the ket kernel conj(psi(i_T)) psi(j_T).
void compat_ptranspose(const cplx* A, bool ket, cplx* out,
                       const std::vector<idx>& target, idx n) {
    idx D = idx{1} << n;
    if (target.empty()) {
        if (ket)
            for (idx j = 0; j < D; ++j)
                for (idx i = 0; i < D; ++i) out[i + j * D] = A[i] * std::conj(A[j]);
        else
            std::memcpy(static_cast<void*>(out), A, D * D * sizeof(cplx));
        return;
    }
    if (target.size() == n) {
        for (idx j = 0; j < D; ++j)
            for (idx i = 0; i < D; ++i)
                out[i + j * D] = ket ? A[j] * std::conj(A[i]) : A[j + i * D];
        return;
    }
    idx M = 0;
    for (idx t : target) M |= idx{1} << t;
#pragma omp parallel for collapse(2)
    for (idx i = 0; i < D; ++i)
        for (idx j = 0; j < D; ++j) {
            idx iT = (i & ~M) | (j & M), jT = (j & ~M) | (i & M);
            out[i + j * D] = ket ? std::conj(A[iT]) * A[jT] : A[jT + iT * D];
        }
}

// ---------------------------------------------------------- syspermute
// operations.hpp:2386-2514: the element at linear index i (a multi-index over
// n digits for a ket, 2n digits [column digits, row digits] for a
// column-major density matrix) moves to the index whose digit k is old digit
// perm[k].
void generic_syspermute(const cplx* A, bool ket, cplx* out,
                        const std::vector<idx>& perm,
                        const std::vector<idx>& dims) {
    idx n = dims.size(), D = prod(dims);
    idx mult = ket ? 1 : 2, tot = n * mult, N = ket ? D : D * D;
    std::vector<idx> cd(tot), cp(tot);
    for (idx i = 0; i < n; ++i) {
        cd[i] = dims[i];
        cp[i] = perm[i];
        if (!ket) {
            cd[i + n] = dims[i];
            cp[i + n] = perm[i] + n;
        }
    }
#pragma omp parallel for
    for (idx i = 0; i < N; ++i) {
        idx mi[2 * kMaxN], mt[2 * kMaxN], pd[2 * kMaxN];
        to_digits(i, tot, cd.data(), mi);
        for (idx k = 0; k < tot; ++k) {
            pd[k] = cd[cp[k]];
            mt[k] = mi[cp[k]];
        }
        out[from_digits(mt, tot, pd)] = A[i];
    }
}

// Qubit-kernel variant (internal/kernels/qubit/syspermute.hpp:58-180): new bit
// k (little-endian) takes old bit inv_perm[k]; for a density matrix the same
// map is applied to both halves of the linear index.
void compat_syspermute(const cplx* A, bool ket, cplx* out,
                       const std::vector<idx>& perm, idx n) {
    idx D = idx{1} << n;
    std::vector<idx> inv(n);
    for (idx k = 0; k < n; ++k) inv[perm[k]] = k;
    auto pb = [&](idx old) {
        idx r = 0;
        for (idx k = 0; k < n; ++k) r |= ((old >> inv[k]) & 1) << k;
        return r;
    };
    if (ket) {
#pragma omp parallel for
        for (idx i = 0; i < D; ++i) out[pb(i)] = A[i];
    } else {
#pragma omp parallel for
        for (idx i = 0; i < D * D; ++i) {
            idx hi = i / D, lo = i % D;
            out[pb(hi) * D + pb(lo)] = A[i];
        }
    }
}

} // namespace

// ===================================================================== C ABI
extern "C" {

const char* oracle_last_where() { return g_where.c_str(); }
const char* oracle_last_what() { return g_what.c_str(); }

// qpp::apply(state, A, target, dims), operations.hpp:72-372.
// path: 0 = generic mixed-radix loops, 1 = qubit kernels where qpp has them
// (QPP_QUBIT_OPTIMIZATIONS, apply.hpp) for 1- and 2-qubit kets, else generic.
int oracle_apply(const double* state, idx rows, idx cols, const double* A,
                 idx A_rows, idx A_cols, const uint64_t* target_p, uint32_t k,
                 const uint64_t* dims_p, uint32_t nd, double* result,
                 int path) {
    const char* W = "qpp::apply()";
    std::vector<idx> target = vec(target_p, k), dims = vec(dims_p, nd);
    if (A_rows * A_cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "state"});
    if (target.empty()) return fail({QGPU_ERR_ZERO_SIZE, W, "target"});
    if (A_rows != A_cols) return fail({QGPU_ERR_MATRIX_NOT_SQUARE, W, "A"});
    if (!dims_ok(dims)) return fail({QGPU_ERR_DIMS_INVALID, W, "dims"});
    if (!subsys_ok(target, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target"});
    if (int e = check_state_shape(rows, cols, dims, W, "dims/state",
                                  "dims/state", "state"))
        return e;
    idx DA = 1;
    for (idx t : target) DA *= dims[t];
    if (DA != A_cols)
        return fail({QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, "A/dims/target"});
    idx D = rows;
    bool ket = cols == 1;
    if (D == 1) {
        std::memcpy(result, state, (ket ? 1 : 1) * sizeof(cplx));
        return 0;
    }
    idx n = dims.size();
    if (path == 1 && ket && all_two(dims) && target.size() == 1) {
        qubit_apply_psi_1q(C(state), C(result), C(A), target[0], n);
        return 0;
    }
    if (path == 1 && ket && all_two(dims) && target.size() == 2) {
        qubit_apply_psi_2q(C(state), C(result), C(A), target[0], target[1], n);
        return 0;
    }
    if (ket)
        generic_apply_ket(C(state), C(result), C(A), DA, target, dims);
    else
        generic_apply_rho(C(state), C(result), C(A), DA, target, dims);
    return 0;
}

// qpp::applyCTRL / applyCTRL_fan, operations.hpp:616-936 and :961-1234.
// path: 0 = generic (A^r table over the d control values), 1 = qubit-kernel
// mask semantics when all dims are 2. shift may be NULL.
int oracle_apply_ctrl(const double* state, idx rows, idx cols, const double* A,
                      idx A_rows, idx A_cols, const uint64_t* ctrl_p,
                      uint32_t nc, const uint64_t* target_p, uint32_t k,
                      const uint64_t* dims_p, uint32_t nd,
                      const uint64_t* shift_p, int fan, double* result,
                      int path) {
    const char* W = fan ? "qpp::applyCTRL_fan()" : "qpp::applyCTRL()";
    std::vector<idx> ctrl = vec(ctrl_p, nc), target = vec(target_p, k),
                     dims = vec(dims_p, nd);
    if (A_rows * A_cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "state"});
    if (ctrl.empty()) return fail({QGPU_ERR_ZERO_SIZE, W, "ctrl"});
    if (target.empty()) return fail({QGPU_ERR_ZERO_SIZE, W, "target"});
    if (A_rows != A_cols) return fail({QGPU_ERR_MATRIX_NOT_SQUARE, W, "A"});
    if (int e = check_state_shape(rows, cols, dims, W, "dims/state",
                                  "dims/state", "state"))
        return e;
    if (!subsys_ok(ctrl, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "ctrl/dims"});
    idx d = dims[ctrl[0]];
    for (idx i = 1; i < ctrl.size(); ++i)
        if (dims[ctrl[i]] != d) return fail({QGPU_ERR_DIMS_NOT_EQUAL, W, "ctrl"});
    if (!dims_ok(dims)) return fail({QGPU_ERR_DIMS_INVALID, W, "dims"});
    if (!subsys_ok(target, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target"});
    if (fan) {
        for (idx i = 1; i < target.size(); ++i)
            if (dims[target[i]] != d)
                return fail({QGPU_ERR_DIMS_NOT_EQUAL, W, "target"});
    }
    for (idx c : ctrl)
        for (idx t : target)
            if (c == t) return fail({QGPU_ERR_OUT_OF_RANGE, W, "ctrl/target"});
    idx DA = 1;
    if (fan) {
        if (A_rows != d)
            return fail({QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, "A/target"});
        DA = d;
    } else {
        for (idx t : target) DA *= dims[t];
        if (DA != A_cols)
            return fail({QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, "A/target"});
    }
    std::vector<idx> cg = ctrl;
    cg.insert(cg.end(), target.begin(), target.end());
    std::sort(cg.begin(), cg.end());
    if (!subsys_ok(cg, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/ctrl/target"});
    std::vector<idx> shift(ctrl.size(), 0);
    if (shift_p) {
        shift = vec(shift_p, nc);
        for (idx& s : shift) {
            if (s >= d) return fail({QGPU_ERR_OUT_OF_RANGE, W, "shift"});
            s = (d - s) % d; // operations.hpp:727-735
        }
    }
    idx n = dims.size(), D = rows;
    bool ket = cols == 1;
    if (D == 1) {
        result[0] = state[0];
        result[1] = state[1];
        return 0;
    }
    Mat Am(C(A), C(A) + DA * DA);
    std::vector<Mat> Ak;
    for (idx r = 0; r < d; ++r) Ak.push_back(powm(Am, DA, r));
    auto ket_op = [&](const cplx* in, cplx* outp) {
        if (path == 1 && all_two(dims))
            qubit_ctrl_ket(in, outp, C(A), DA, ctrl, target, shift, n, fan);
        else
            generic_ctrl_ket(in, outp, Ak, DA, ctrl, target, dims, shift, d, fan);
    };
    if (ket) {
        ket_op(C(state), C(result));
        return 0;
    }
    // density matrix, operations.hpp:846-882: rho = sum_i |i><row_i|, so
    // result = sum_i CTRL|i> (CTRL row_i^dagger)^dagger.
    const cplx* R = C(state);
    std::vector<cplx> out(D * D, 0.0);
    std::vector<cplx> e(D), ce(D), ph(D), cph(D);
    for (idx i = 0; i < D; ++i) {
        std::fill(e.begin(), e.end(), cplx(0.0));
        e[i] = 1.0;
        for (idx c = 0; c < D; ++c) ph[c] = std::conj(R[i + c * D]);
        ket_op(e.data(), ce.data());
        ket_op(ph.data(), cph.data());
        for (idx c = 0; c < D; ++c) {
            cplx bra = std::conj(cph[c]);
            for (idx r = 0; r < D; ++r) out[r + c * D] += ce[r] * bra;
        }
    }
    std::memcpy(result, out.data(), D * D * sizeof(cplx));
    return 0;
}

// qpp::apply(A, Ks, target, dims), operations.hpp:476-560.
int oracle_apply_kraus(const double* state, idx rows, idx cols,
                       const double* Ks, uint32_t nK, idx K_rows, idx K_cols,
                       const uint64_t* target_p, uint32_t k,
                       const uint64_t* dims_p, uint32_t nd, double* result) {
    const char* W = "qpp::apply()";
    std::vector<idx> target = vec(target_p, k), dims = vec(dims_p, nd);
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    if (target.empty()) return fail({QGPU_ERR_ZERO_SIZE, W, "target"});
    if (rows != cols) return fail({QGPU_ERR_MATRIX_NOT_SQUARE, W, "A"});
    if (!dims_ok(dims)) return fail({QGPU_ERR_DIMS_INVALID, W, "dims"});
    if (!subsys_ok(target, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target"});
    if (int e = check_state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A"))
        return e;
    idx DA = 1;
    for (idx t : target) DA *= dims[t];
    if (nK == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "Ks"});
    if (K_rows != K_cols) return fail({QGPU_ERR_MATRIX_NOT_SQUARE, W, "Ks[0]"});
    if (K_cols != DA)
        return fail({QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, "dims/Ks[0]/target"});
    idx D = rows;
    std::vector<cplx> acc(D * D, 0.0), tmp(D * D);
    for (uint32_t i = 0; i < nK; ++i) {
        generic_apply_rho(C(state), tmp.data(), C(Ks) + i * DA * DA, DA, target,
                          dims);
        for (idx t = 0; t < D * D; ++t) acc[t] += tmp[t];
    }
    std::memcpy(result, acc.data(), D * D * sizeof(cplx));
    return 0;
}

// qpp::ptrace(A, target, dims), operations.hpp:1908-2114.
int oracle_ptrace(const double* state, idx rows, idx cols,
                  const uint64_t* target_p, uint32_t k, const uint64_t* dims_p,
                  uint32_t nd, double* result) {
    const char* W = "qpp::ptrace()";
    std::vector<idx> target = vec(target_p, k), dims = vec(dims_p, nd);
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    if (!dims_ok(dims)) return fail({QGPU_ERR_DIMS_INVALID, W, "dims"});
    if (!subsys_ok(target, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target"});
    if (int e = check_state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A"))
        return e;
    generic_ptrace(C(state), cols == 1, C(result), target, dims);
    return 0;
}

// qpp::ptranspose(A, target, dims), operations.hpp:2167-2335.
// compat = 1 reproduces the qubit kernel (ptranspose.hpp) for all-qubit dims.
int oracle_ptranspose(const double* state, idx rows, idx cols,
                      const uint64_t* target_p, uint32_t k,
                      const uint64_t* dims_p, uint32_t nd, double* result,
                      int compat) {
    const char* W = "qpp::ptranspose()";
    std::vector<idx> target = vec(target_p, k), dims = vec(dims_p, nd);
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    if (!dims_ok(dims)) return fail({QGPU_ERR_DIMS_INVALID, W, "dims"});
    if (!subsys_ok(target, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target"});
    if (int e = check_state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A"))
        return e;
    if (compat && all_two(dims))
        compat_ptranspose(C(state), cols == 1, C(result), target, dims.size());
    else
        generic_ptranspose(C(state), cols == 1, C(result), target, dims);
    return 0;
}

// qpp::syspermute(A, perm, dims), operations.hpp:2386-2514.
int oracle_syspermute(const double* state, idx rows, idx cols,
                      const uint64_t* perm_p, uint32_t np,
                      const uint64_t* dims_p, uint32_t nd, double* result,
                      int compat) {
    const char* W = "qpp::syspermute()";
    std::vector<idx> perm = vec(perm_p, np), dims = vec(dims_p, nd);
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    if (!dims_ok(dims)) return fail({QGPU_ERR_DIMS_INVALID, W, "dims"});
    if (!perm_ok(perm)) return fail({QGPU_ERR_PERM_INVALID, W, "perm"});
    if (perm.size() != dims.size())
        return fail({QGPU_ERR_PERM_MISMATCH_DIMS, W, "dims/perm"});
    if (int e = check_state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A"))
        return e;
    if (compat && all_two(dims))
        compat_syspermute(C(state), cols == 1, C(result), perm, dims.size());
    else
        generic_syspermute(C(state), cols == 1, C(result), perm, dims);
    return 0;
}

// qpp::normalize(A), functions.hpp:304-333 (ket / norm, rho / trace).
int oracle_normalize(double* state, idx rows, idx cols) {
    const char* W = "qpp::normalize()";
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    cplx* s = C(state);
    if (cols == 1 || rows == 1) {
        double nn = 0;
        for (idx i = 0; i < rows * cols; ++i) nn += std::norm(s[i]);
        double nrm = std::sqrt(nn);
        if (nrm == 0) return fail({QGPU_ERR_DIVISION_BY_ZERO, W, "Division by zero!"});
        for (idx i = 0; i < rows * cols; ++i) s[i] /= nrm;
    } else if (rows == cols) {
        cplx tr = 0;
        for (idx i = 0; i < rows; ++i) tr += s[i + i * rows];
        if (std::abs(tr) == 0)
            return fail({QGPU_ERR_DIVISION_BY_ZERO, W, "Division by zero!"});
        for (idx i = 0; i < rows * cols; ++i) s[i] /= tr;
    } else {
        return fail({QGPU_ERR_MATRIX_NOT_SQUARE_NOR_VECTOR, W, "A"});
    }
    return 0;
}

// qpp::measure_seq(A, target, dims, destructive), instruments.hpp:985-1111,
// with the Z-basis sample() of instruments.hpp:746-818.
// forced: if non-NULL, the outcome dits to take (replay mode) instead of
// sampling with std::mt19937(seed) + std::discrete_distribution over the full
// basis, as sample() does. Writes results[k], probs[k], the post-measurement
// state to out_state and its dims to out_dims (count in *out_nd).
int oracle_measure_seq(const double* state, idx rows, idx cols,
                       const uint64_t* target_p, uint32_t k,
                       const uint64_t* dims_p, uint32_t nd, int destructive,
                       const uint64_t* forced, uint64_t seed,
                       uint64_t* results, double* probs, double* out_state,
                       uint64_t* out_dims, uint32_t* out_nd) {
    const char* W = "qpp::measure_seq()";
    std::vector<idx> target = vec(target_p, k), dims = vec(dims_p, nd);
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    if (!dims_ok(dims)) return fail({QGPU_ERR_DIMS_INVALID, W, "dims"});
    if (int e = check_state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A"))
        return e;
    if (!subsys_ok(target, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target"});
    bool ket = cols == 1;
    idx D = rows;
    std::vector<cplx> A(C(state), C(state) + (ket ? D : D * D));
    std::vector<idx> res(k);
    if (forced) {
        for (idx i = 0; i < k; ++i) res[i] = forced[i];
    } else {
        std::vector<double> pbs(D);
        for (idx i = 0; i < D; ++i)
            pbs[i] = ket ? std::norm(A[i]) : A[i + i * D].real();
        std::mt19937 gen(static_cast<uint32_t>(seed));
        std::discrete_distribution<idx> dd(pbs.begin(), pbs.end());
        idx s = dd(gen);
        idx dg[kMaxN];
        to_digits(s, dims.size(), dims.data(), dg);
        for (idx i = 0; i < k; ++i) res[i] = dg[target[i]];
    }
    // Density matrices of at most 10 subsystems take the "small" path
    // (instruments.hpp:1027-1047): targets in the given order, the traced
    // subsystems removed at the end. Everything else takes the shrink path
    // (instruments.hpp:1052-1108): when destructive, targets in descending
    // order, each removed right after its projection.
    bool small_rho = !ket && dims.size() <= 10;
    std::vector<idx> order(k);
    std::iota(order.begin(), order.end(), 0);
    if (destructive && !small_rho)
        std::sort(order.begin(), order.end(),
                  [&](idx a, idx b) { return target[a] > target[b]; });
    std::vector<idx> cd = dims;
    bool shrink_each = destructive && !small_rho;
    for (idx cnt = 0; cnt < k; ++cnt) {
        idx ip = order[cnt];
        idx t = target[ip];
        idx n = cd.size();
        idx Dc = prod(cd);
        // project the current state on digit res[ip] of subsystem t
        double p = 0;
        for (idx i = 0; i < Dc; ++i) {
            idx dg[kMaxN];
            to_digits(i, n, cd.data(), dg);
            bool keep_r = dg[t] == res[ip];
            if (ket) {
                if (!keep_r) A[i] = 0;
                else p += std::norm(A[i]);
            } else {
                for (idx j = 0; j < Dc; ++j) {
                    idx dj[kMaxN];
                    to_digits(j, n, cd.data(), dj);
                    if (!keep_r || dj[t] != res[ip]) A[i + j * Dc] = 0;
                }
                p += A[i + i * Dc].real();
            }
        }
        probs[ip] = p;
        if (p == 0) return fail({QGPU_ERR_DIVISION_BY_ZERO, W, "probability zero"});
        double sc = ket ? 1.0 / std::sqrt(p) : 1.0 / p;
        for (auto& v : A) v *= sc;
        if (shrink_each) {
            std::vector<idx> nd2 = cd;
            nd2.erase(nd2.begin() + static_cast<std::ptrdiff_t>(t));
            idx Dn = prod(nd2);
            std::vector<cplx> B(ket ? Dn : Dn * Dn);
            if (ket) {
                for (idx i = 0; i < Dc; ++i) {
                    idx dg[kMaxN] = {}, dn[kMaxN];
                    to_digits(i, n, cd.data(), dg);
                    if (dg[t] != res[ip]) continue;
                    idx m = 0;
                    for (idx q = 0; q < n; ++q)
                        if (q != t) dn[m++] = dg[q];
                    B[from_digits(dn, n - 1, nd2.data())] = A[i];
                }
            } else {
                std::vector<idx> tt{t};
                generic_ptrace(A.data(), false, B.data(), tt, cd);
            }
            A.swap(B);
            cd = nd2;
        }
    }
    if (destructive && small_rho) {
        std::vector<idx> bar = complement_of(target, dims.size());
        std::vector<idx> nd2;
        for (idx q : bar) nd2.push_back(dims[q]);
        idx Dn = prod(nd2);
        std::vector<cplx> B(Dn * Dn);
        generic_ptrace(A.data(), false, B.data(), target, dims);
        A.swap(B);
        cd = nd2;
    }
    for (idx i = 0; i < k; ++i) results[i] = res[i];
    std::memcpy(out_state, A.data(), A.size() * sizeof(cplx));
    for (idx i = 0; i < cd.size(); ++i) out_dims[i] = cd[i];
    *out_nd = static_cast<uint32_t>(cd.size());
    return 0;
}

// qpp::sample(num_samples, A, target, dims), instruments.hpp:856-940:
// num_samples draws of one std::discrete_distribution over the full basis
// (|A_i|^2 for a ket, Re A(i, i) for a density matrix) from
// std::mt19937(seed); results[i * k + j] = digit target[j] of draw i.
int oracle_sample(const double* state, idx rows, idx cols, const uint64_t* target_p,
                  uint32_t k, const uint64_t* dims_p, uint32_t nd, uint64_t num_samples,
                  uint64_t seed, uint64_t* results) {
    const char* W = "qpp::sample()";
    std::vector<idx> target = vec(target_p, k), dims = vec(dims_p, nd);
    if (rows * cols == 0) return fail({QGPU_ERR_ZERO_SIZE, W, "A"});
    if (!dims_ok(dims)) return fail({QGPU_ERR_DIMS_INVALID, W, "dims"});
    if (int e = check_state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A"))
        return e;
    if (!subsys_ok(target, dims))
        return fail({QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target"});
    if (num_samples == 0) return fail({QGPU_ERR_OUT_OF_RANGE, W, "num_samples"});
    const bool ket = cols == 1;
    const idx D = rows;
    const cplx* A = C(state);
    std::vector<double> pbs(D);
    for (idx i = 0; i < D; ++i) pbs[i] = ket ? std::norm(A[i]) : A[i + i * D].real();
    std::mt19937 gen(static_cast<uint32_t>(seed));
    std::discrete_distribution<idx> dd(pbs.begin(), pbs.end());
    for (uint64_t r = 0; r < num_samples; ++r) {
        idx dg[kMaxN];
        to_digits(dd(gen), dims.size(), dims.data(), dg);
        for (uint32_t j = 0; j < k; ++j) results[r * k + j] = dg[target[j]];
    }
    return 0;
}

} // extern "C"

// ------------------------------------------------------------------ inputs
// Philox4x32-10 (Salmon et al., SC'11) + Box-Muller, the same counter-based
// stream the product uses for qgpu_state_fill_gaussian, so the CPU baseline
// and the GPU start from the same seeded input. Not normalised here.
// One std::discrete_distribution draw over w[0..n) from std::mt19937(seed):
// the sampling step of qpp::measure (instruments.hpp:289-292, :488-491).
extern "C" uint64_t oracle_discrete_draw(const double* w, uint64_t n, uint64_t seed) {
    std::mt19937 gen(static_cast<uint32_t>(seed));
    std::discrete_distribution<uint64_t> dd(w, w + n);
    return dd(gen);
}

extern "C" void oracle_fill_gaussian(double* out, uint64_t n, uint64_t seed) {
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t c[4] = {uint32_t(i), uint32_t(i >> 32), 0u, 0u};
        uint32_t k0 = uint32_t(seed), k1 = uint32_t(seed >> 32);
        for (int r = 0; r < 10; ++r) {
            uint64_t p0 = uint64_t(0xD2511F53u) * c[0];
            uint64_t p1 = uint64_t(0xCD9E8D57u) * c[2];
            uint32_t n0 = uint32_t(p1 >> 32) ^ c[1] ^ k0;
            uint32_t n2 = uint32_t(p0 >> 32) ^ c[3] ^ k1;
            c[1] = uint32_t(p1);
            c[3] = uint32_t(p0);
            c[0] = n0;
            c[2] = n2;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t a = (uint64_t(c[0]) << 21) ^ (uint64_t(c[1]) >> 11);
        uint64_t b = (uint64_t(c[2]) << 21) ^ (uint64_t(c[3]) >> 11);
        double u1 = (double(a & ((1ull << 53) - 1)) + 1.0) * 0x1.0p-53;
        double u2 = double(b & ((1ull << 53) - 1)) * 0x1.0p-53;
        double r = std::sqrt(-2.0 * std::log(u1));
        double th = 2.0 * M_PI * u2;
        out[2 * i] = r * std::cos(th);
        out[2 * i + 1] = r * std::sin(th);
    }
}
