// qpp_b200.hpp -- C++17 drop-in layer over the C ABI (qpp_b200.h).
//
// Mirrors the Quantum++ 7.0.3 free functions of the gate-application and
// subsystem path with the same names, argument meaning, value semantics and
// exception types (include/qpp/operations.hpp, classes/exception.hpp):
//
//   qpp_b200::apply(state, A, target, dims)                 operations.hpp:72
//   qpp_b200::apply(state, A, target, d)                    operations.hpp:386
//   qpp_b200::applyCTRL(state, A, ctrl, target, dims, shift) operations.hpp:616
//   qpp_b200::applyCTRL_fan(...)                            operations.hpp:961
//   qpp_b200::apply(rho, Ks, target, dims)                  operations.hpp:476
//   qpp_b200::ptrace(A, target, dims)                       operations.hpp:1908
//   qpp_b200::ptranspose(A, target, dims)                   operations.hpp:2167
//   qpp_b200::syspermute(A, perm, dims)                     operations.hpp:2386
//   qpp_b200::sample(num_samples, A, target, dims, seed)    instruments.hpp:856
//   qpp_b200::measure_seq(A, target, dims, destructive, seed) instruments.hpp:985
//   qpp_b200::measure(A, Ks | V, target, dims, destructive, seed) instruments.hpp:371, :587
//   qpp_b200::reset(A, target, dims, seed), discard(...)    instruments.hpp:1148, :1243
//   qpp_b200::applyQFT / applyTFQ(A, target, d, swap)       operations.hpp:2565, :2680
//   qpp_b200::QFT / TFQ(A, d, swap)                         operations.hpp:2792, :2844
//
// Matrices are qpp_b200::cmat (column-major std::complex<double>, rows x
// cols; a ket is D x 1). When <Eigen/Dense> is on the include path, every
// function listed above also accepts Eigen matrices (Eigen::MatrixBase
// expressions) and returns Eigen::MatrixXcd in place of cmat, so code
// written against qpp:: compiles against qpp_b200:: unchanged. Errors throw
// qpp_b200::exception::<QppName> carrying qpp's (where, what) strings.
// Header-only; link with libqpp_b200.so.
#ifndef QPP_B200_HPP_
#define QPP_B200_HPP_

#include <cmath>
#include <complex>
#include <map>
#include <tuple>
#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "qpp_b200.h"

#if defined(__has_include)
#if __has_include(<Eigen/Dense>)
#include <Eigen/Dense>
#define QPP_B200_HAS_EIGEN 1
#endif
#endif

namespace qpp_b200 {

using idx = std::size_t;
using cplx = std::complex<double>;

struct cmat {
    idx rows_ = 0, cols_ = 0;
    std::vector<cplx> data_; // column-major
    cmat() = default;
    cmat(idx r, idx c) : rows_(r), cols_(c), data_(r * c, cplx(0.0)) {}
    idx rows() const { return rows_; }
    idx cols() const { return cols_; }
    cplx& operator()(idx r, idx c) { return data_[r + c * rows_]; }
    const cplx& operator()(idx r, idx c) const { return data_[r + c * rows_]; }
    cplx& operator()(idx i) { return data_[i]; }
    const cplx& operator()(idx i) const { return data_[i]; }
    const double* raw() const { return reinterpret_cast<const double*>(data_.data()); }
    double* raw() { return reinterpret_cast<double*>(data_.data()); }
};
using ket = cmat;

namespace exception {
// qpp::exception::Exception (classes/exception.hpp:68-127): what() is
// "IN " + where + ": Exception <type>! " + description.
class Exception : public std::runtime_error {
  public:
    Exception(std::string type, std::string where, std::string what)
        : std::runtime_error("IN " + where + ": Exception " + type + "! " + what),
          type_(std::move(type)), where_(std::move(where)), what_(std::move(what)) {}
    const std::string& type_description() const { return type_; }
    const std::string& where() const { return where_; }
    const std::string& detail() const { return what_; }

  private:
    std::string type_, where_, what_;
};
#define QPP_B200_EXC(Name)                                                    \
    class Name : public Exception {                                          \
      public:                                                                \
        Name(std::string where, std::string what)                            \
            : Exception(#Name, std::move(where), std::move(what)) {}         \
    };
QPP_B200_EXC(ZeroSize)
QPP_B200_EXC(MatrixNotSquare)
QPP_B200_EXC(MatrixNotSquareNorCvector)
QPP_B200_EXC(MatrixMismatchSubsys)
QPP_B200_EXC(DimsInvalid)
QPP_B200_EXC(DimsNotEqual)
QPP_B200_EXC(DimsMismatchMatrix)
QPP_B200_EXC(DimsMismatchCvector)
QPP_B200_EXC(SubsysMismatchDims)
QPP_B200_EXC(PermInvalid)
QPP_B200_EXC(PermMismatchDims)
QPP_B200_EXC(OutOfRange)
QPP_B200_EXC(TypeMismatch)
QPP_B200_EXC(SizeMismatch)
QPP_B200_EXC(QuditAlreadyMeasured)
QPP_B200_EXC(MatrixNotSquareNorVector)
QPP_B200_EXC(Duplicates)
QPP_B200_EXC(DeviceError)
#undef QPP_B200_EXC
} // namespace exception

namespace detail {

[[noreturn]] inline void throw_status(qgpu_status s) {
    std::string w = qgpu_last_error_where(), m = qgpu_last_error_what();
    using namespace exception;
    switch (s) {
        case QGPU_ERR_ZERO_SIZE: throw ZeroSize(w, m);
        case QGPU_ERR_MATRIX_NOT_SQUARE: throw MatrixNotSquare(w, m);
        case QGPU_ERR_MATRIX_NOT_SQUARE_NOR_CVECTOR: throw MatrixNotSquareNorCvector(w, m);
        case QGPU_ERR_MATRIX_MISMATCH_SUBSYS: throw MatrixMismatchSubsys(w, m);
        case QGPU_ERR_DIMS_INVALID: throw DimsInvalid(w, m);
        case QGPU_ERR_DIMS_NOT_EQUAL: throw DimsNotEqual(w, m);
        case QGPU_ERR_DIMS_MISMATCH_MATRIX: throw DimsMismatchMatrix(w, m);
        case QGPU_ERR_DIMS_MISMATCH_CVECTOR: throw DimsMismatchCvector(w, m);
        case QGPU_ERR_SUBSYS_MISMATCH_DIMS: throw SubsysMismatchDims(w, m);
        case QGPU_ERR_PERM_INVALID: throw PermInvalid(w, m);
        case QGPU_ERR_PERM_MISMATCH_DIMS: throw PermMismatchDims(w, m);
        case QGPU_ERR_OUT_OF_RANGE: throw OutOfRange(w, m);
        case QGPU_ERR_TYPE_MISMATCH: throw TypeMismatch(w, m);
        case QGPU_ERR_SIZE_MISMATCH: throw SizeMismatch(w, m);
        case QGPU_ERR_QUDIT_ALREADY_MEASURED: throw QuditAlreadyMeasured(w, m);
        case QGPU_ERR_MATRIX_NOT_SQUARE_NOR_VECTOR: throw MatrixNotSquareNorVector(w, m);
        case QGPU_ERR_DUPLICATES: throw Duplicates(w, m);
        case QGPU_ERR_DIVISION_BY_ZERO: throw std::overflow_error(w + ": " + m);
        default: throw DeviceError(w, std::string(qgpu_status_name(s)) + ": " + m);
    }
}

inline void check(qgpu_status s) {
    if (s != QGPU_OK) throw_status(s);
}

// One context per thread on device 0 unless set_device() chose another.
inline int& device_slot() {
    static thread_local int dev = 0;
    return dev;
}
struct CtxHolder {
    qgpu_ctx* c = nullptr;
    int dev = -1;
    ~CtxHolder() {
        if (c) qgpu_ctx_destroy(c);
    }
};
inline qgpu_ctx* ctx() {
    static thread_local CtxHolder h;
    if (!h.c || h.dev != device_slot()) {
        if (h.c) qgpu_ctx_destroy(h.c);
        h.c = nullptr;
        check(qgpu_ctx_create(device_slot(), &h.c));
        h.dev = device_slot();
    }
    return h.c;
}

inline std::vector<uint64_t> u64(const std::vector<idx>& v) {
    return std::vector<uint64_t>(v.begin(), v.end());
}
inline const uint64_t* ptr(const std::vector<uint64_t>& v) {
    return v.empty() ? nullptr : v.data();
}

// get_num_subsys (internal/util.hpp:389-397)
inline std::vector<idx> dims_of(idx D, idx d) {
    idx n = static_cast<idx>(std::llround(std::log2(static_cast<double>(D)) /
                                          std::log2(static_cast<double>(d))));
    return std::vector<idx>(n, d);
}

} // namespace detail

// Select the CUDA device used by the calling thread.
inline void set_device(int device) { detail::device_slot() = device; }

inline cmat apply(const cmat& state, const cmat& A, const std::vector<idx>& target,
                  const std::vector<idx>& dims) {
    auto t = detail::u64(target), d = detail::u64(dims);
    cmat out(state.rows(), state.cols());
    detail::check(qgpu_host_apply(detail::ctx(), state.raw(), state.rows(), state.cols(),
                                  A.raw(), A.rows(), A.cols(), detail::ptr(t),
                                  uint32_t(t.size()), detail::ptr(d), uint32_t(d.size()),
                                  out.raw()));
    return out;
}

inline cmat apply(const cmat& state, const cmat& A, const std::vector<idx>& target,
                  idx d = 2) {
    if (state.rows() * state.cols() == 0)
        throw exception::ZeroSize("qpp::apply()", "state");
    if (d < 2) throw exception::DimsInvalid("qpp::apply()", "d");
    return apply(state, A, target, detail::dims_of(state.rows(), d));
}

inline cmat applyCTRL(const cmat& state, const cmat& A, const std::vector<idx>& ctrl,
                      const std::vector<idx>& target, const std::vector<idx>& dims,
                      std::optional<std::vector<idx>> shift = std::nullopt) {
    auto c = detail::u64(ctrl), t = detail::u64(target), d = detail::u64(dims);
    std::vector<uint64_t> s;
    if (shift) s = detail::u64(*shift);
    cmat out(state.rows(), state.cols());
    detail::check(qgpu_host_apply_ctrl(
        detail::ctx(), state.raw(), state.rows(), state.cols(), A.raw(), A.rows(), A.cols(),
        detail::ptr(c), uint32_t(c.size()), detail::ptr(t), uint32_t(t.size()),
        detail::ptr(d), uint32_t(d.size()), shift ? s.data() : nullptr, 0, out.raw()));
    return out;
}

inline cmat applyCTRL_fan(const cmat& state, const cmat& A, const std::vector<idx>& ctrl,
                          const std::vector<idx>& target, const std::vector<idx>& dims,
                          std::optional<std::vector<idx>> shift = std::nullopt) {
    auto c = detail::u64(ctrl), t = detail::u64(target), d = detail::u64(dims);
    std::vector<uint64_t> s;
    if (shift) s = detail::u64(*shift);
    cmat out(state.rows(), state.cols());
    detail::check(qgpu_host_apply_ctrl(
        detail::ctx(), state.raw(), state.rows(), state.cols(), A.raw(), A.rows(), A.cols(),
        detail::ptr(c), uint32_t(c.size()), detail::ptr(t), uint32_t(t.size()),
        detail::ptr(d), uint32_t(d.size()), shift ? s.data() : nullptr, 1, out.raw()));
    return out;
}

inline cmat apply(const cmat& rho, const std::vector<cmat>& Ks,
                  const std::vector<idx>& target, const std::vector<idx>& dims) {
    auto t = detail::u64(target), d = detail::u64(dims);
    std::vector<cplx> packed;
    idx kr = Ks.empty() ? 0 : Ks[0].rows(), kc = Ks.empty() ? 0 : Ks[0].cols();
    for (auto& K : Ks) {
        if (K.rows() != kr || K.cols() != kc)
            throw exception::DimsNotEqual("qpp::apply()", "K");
        packed.insert(packed.end(), K.data_.begin(), K.data_.end());
    }
    cmat out(rho.rows(), rho.cols());
    detail::check(qgpu_host_apply_kraus(
        detail::ctx(), rho.raw(), rho.rows(), rho.cols(),
        reinterpret_cast<const double*>(packed.data()), uint32_t(Ks.size()), kr, kc,
        detail::ptr(t), uint32_t(t.size()), detail::ptr(d), uint32_t(d.size()), out.raw()));
    return out;
}

inline cmat ptrace(const cmat& A, const std::vector<idx>& target, const std::vector<idx>& dims) {
    auto t = detail::u64(target), d = detail::u64(dims);
    idx DS = 1;
    for (idx x : target)
        if (x < dims.size()) DS *= dims[x];
    idx Db = (DS && A.rows() % DS == 0) ? A.rows() / DS : 1;
    cmat out(Db, Db);
    detail::check(qgpu_host_ptrace(detail::ctx(), A.raw(), A.rows(), A.cols(), detail::ptr(t),
                                   uint32_t(t.size()), detail::ptr(d), uint32_t(d.size()),
                                   out.raw()));
    return out;
}

inline cmat ptranspose(const cmat& A, const std::vector<idx>& target,
                       const std::vector<idx>& dims) {
    auto t = detail::u64(target), d = detail::u64(dims);
    cmat out(A.rows(), A.rows());
    detail::check(qgpu_host_ptranspose(detail::ctx(), A.raw(), A.rows(), A.cols(),
                                       detail::ptr(t), uint32_t(t.size()), detail::ptr(d),
                                       uint32_t(d.size()), out.raw()));
    return out;
}

inline cmat syspermute(const cmat& A, const std::vector<idx>& perm, const std::vector<idx>& dims) {
    auto p = detail::u64(perm), d = detail::u64(dims);
    cmat out(A.rows(), A.cols());
    detail::check(qgpu_host_syspermute(detail::ctx(), A.raw(), A.rows(), A.cols(),
                                       detail::ptr(p), uint32_t(p.size()), detail::ptr(d),
                                       uint32_t(d.size()), out.raw()));
    return out;
}

namespace detail {
// qpp's state checks for sample / measure_seq (instruments.hpp:757-781,
// :996-1017), then the state uploaded as a resident handle
struct StateHolder {
    qgpu_state* s = nullptr;
    ~StateHolder() {
        if (s) qgpu_state_destroy(s);
    }
};
inline void upload_checked(const cmat& A, const std::vector<idx>& dims, const char* W,
                           StateHolder& h) {
    using namespace exception;
    if (A.rows() * A.cols() == 0) throw ZeroSize(W, "A");
    idx D = 1;
    bool ok = !dims.empty();
    for (idx x : dims) {
        ok = ok && x != 0;
        D *= x;
    }
    if (!ok) throw DimsInvalid(W, "dims");
    const bool is_ket = A.cols() == 1;
    if (is_ket) {
        if (D != A.rows()) throw DimsMismatchCvector(W, "A/dims");
    } else if (A.rows() == A.cols()) {
        if (D != A.rows()) throw DimsMismatchMatrix(W, "A/dims");
    } else {
        throw MatrixNotSquareNorCvector(W, "A");
    }
    auto d = u64(dims);
    check(qgpu_state_create(ctx(), is_ket ? QGPU_KET : QGPU_RHO, QGPU_C128, ptr(d),
                            uint32_t(d.size()), &h.s));
    check(qgpu_state_upload_c128(h.s, A.raw()));
}
} // namespace detail

// qpp::sample(num_samples, A, target, dims) (instruments.hpp:856-940), with
// the draws of a std::mt19937 seeded with `seed`.
inline std::map<std::vector<idx>, idx> sample(idx num_samples, const cmat& A,
                                              const std::vector<idx>& target,
                                              const std::vector<idx>& dims, uint64_t seed = 0) {
    detail::StateHolder h;
    detail::upload_checked(A, dims, "qpp::sample()", h);
    auto t = detail::u64(target);
    std::vector<uint64_t> r(num_samples * t.size() + 1);
    detail::check(qgpu_sample(h.s, detail::ptr(t), uint32_t(t.size()), num_samples, seed,
                              nullptr, r.data()));
    std::map<std::vector<idx>, idx> out;
    for (idx i = 0; i < num_samples; ++i)
        ++out[std::vector<idx>(r.begin() + i * t.size(), r.begin() + (i + 1) * t.size())];
    return out;
}

// qpp::measure_seq(A, target, dims, destructive) (instruments.hpp:985-1111):
// (outcomes, probabilities, post-measurement state).
inline std::tuple<std::vector<idx>, std::vector<double>, cmat>
measure_seq(const cmat& A, const std::vector<idx>& target, const std::vector<idx>& dims,
            bool destructive = true, uint64_t seed = 0) {
    detail::StateHolder h, o;
    detail::upload_checked(A, dims, "qpp::measure_seq()", h);
    auto t = detail::u64(target);
    std::vector<uint64_t> res(t.size() + 1);
    std::vector<double> ps(t.size() + 1);
    detail::check(qgpu_measure_seq(h.s, detail::ptr(t), uint32_t(t.size()), destructive ? 1 : 0,
                                   seed, nullptr, res.data(), ps.data(), &o.s));
    uint64_t D = 0;
    detail::check(qgpu_state_info(o.s, nullptr, nullptr, nullptr, nullptr, &D));
    cmat out(D, A.cols() == 1 ? 1 : D);
    detail::check(qgpu_state_download_c128(o.s, out.raw()));
    return {std::vector<idx>(res.begin(), res.begin() + t.size()),
            std::vector<double>(ps.begin(), ps.begin() + t.size()), out};
}

// qpp::applyQFT / applyTFQ (operations.hpp:2565-2787), qpp::QFT / TFQ
// (:2792-2899): A viewed as qudits of dimension d.
inline cmat applyQFT(const cmat& A, const std::vector<idx>& target, idx d = 2,
                     bool swap = true) {
    auto t = detail::u64(target);
    cmat out(A.rows(), A.cols());
    detail::check(qgpu_host_apply_qft(detail::ctx(), A.raw(), A.rows(), A.cols(),
                                      detail::ptr(t), uint32_t(t.size()), d, swap ? 1 : 0, 0,
                                      out.raw()));
    return out;
}
inline cmat applyTFQ(const cmat& A, const std::vector<idx>& target, idx d = 2,
                     bool swap = true) {
    auto t = detail::u64(target);
    cmat out(A.rows(), A.cols());
    detail::check(qgpu_host_apply_qft(detail::ctx(), A.raw(), A.rows(), A.cols(),
                                      detail::ptr(t), uint32_t(t.size()), d, swap ? 1 : 0, 1,
                                      out.raw()));
    return out;
}
inline cmat QFT(const cmat& A, idx d = 2, bool swap = true) {
    cmat out(A.rows(), A.cols());
    detail::check(qgpu_host_qft(detail::ctx(), A.raw(), A.rows(), A.cols(), d, swap ? 1 : 0, 0,
                                out.raw()));
    return out;
}
inline cmat TFQ(const cmat& A, idx d = 2, bool swap = true) {
    cmat out(A.rows(), A.cols());
    detail::check(qgpu_host_qft(detail::ctx(), A.raw(), A.rows(), A.cols(), d, swap ? 1 : 0, 1,
                                out.raw()));
    return out;
}

namespace detail {
inline cmat download(qgpu_state* s) {
    qgpu_kind kind = QGPU_KET;
    uint64_t D = 0;
    check(qgpu_state_info(s, &kind, nullptr, nullptr, nullptr, &D));
    cmat out(D, kind == QGPU_KET ? 1 : D);
    check(qgpu_state_download_c128(s, out.raw()));
    return out;
}
inline std::tuple<idx, std::vector<double>, std::vector<cmat>>
collect(uint64_t r, const std::vector<double>& probs, std::vector<qgpu_state*>& outs) {
    std::vector<cmat> states(outs.size());
    for (size_t i = 0; i < outs.size(); ++i)
        if (outs[i]) {
            StateHolder h;
            h.s = outs[i];
            states[i] = download(outs[i]);
        }
    return {idx(r), probs, states};
}
} // namespace detail

// qpp::measure(A, Ks, target, dims, destructive) (instruments.hpp:371-494):
// (result, probabilities, post-measurement states; empty where a probability
// is 0), the result drawn from a std::mt19937 seeded with `seed`.
inline std::tuple<idx, std::vector<double>, std::vector<cmat>>
measure(const cmat& A, const std::vector<cmat>& Ks, const std::vector<idx>& target,
        const std::vector<idx>& dims, bool destructive = true, uint64_t seed = 0) {
    detail::StateHolder h;
    detail::upload_checked(A, dims, "qpp::measure()", h);
    auto t = detail::u64(target);
    const idx DK = Ks.empty() ? 0 : Ks[0].rows();
    std::vector<cplx> packed;
    for (const cmat& K : Ks) {
        if (K.rows() != DK || K.cols() != DK)
            throw exception::DimsNotEqual("qpp::measure()", "K");
        packed.insert(packed.end(), K.data_.begin(), K.data_.end());
    }
    std::vector<double> probs(Ks.size() + 1);
    std::vector<qgpu_state*> outs(Ks.size() + 1, nullptr);
    uint64_t r = 0;
    detail::check(qgpu_measure_kraus(h.s, reinterpret_cast<const double*>(packed.data()),
                                     uint32_t(Ks.size()), DK, detail::ptr(t), uint32_t(t.size()),
                                     destructive ? 1 : 0, seed, &r, probs.data(), outs.data()));
    probs.resize(Ks.size());
    outs.resize(Ks.size());
    return detail::collect(r, probs, outs);
}

// qpp::measure(A, V, target, dims, destructive) (instruments.hpp:587-712).
inline std::tuple<idx, std::vector<double>, std::vector<cmat>>
measure(const cmat& A, const cmat& V, const std::vector<idx>& target,
        const std::vector<idx>& dims, bool destructive = true, uint64_t seed = 0) {
    detail::StateHolder h;
    detail::upload_checked(A, dims, "qpp::measure()", h);
    auto t = detail::u64(target);
    std::vector<double> probs(V.cols() + 1);
    std::vector<qgpu_state*> outs(V.cols() + 1, nullptr);
    uint64_t r = 0;
    detail::check(qgpu_measure_basis(h.s, V.raw(), V.rows(), V.cols(), detail::ptr(t),
                                     uint32_t(t.size()), destructive ? 1 : 0, seed, &r,
                                     probs.data(), outs.data()));
    probs.resize(V.cols());
    outs.resize(V.cols());
    return detail::collect(r, probs, outs);
}

// qpp::reset(A, target, dims) (instruments.hpp:1148-1206), seeded.
inline cmat reset(const cmat& A, const std::vector<idx>& target, const std::vector<idx>& dims,
                  uint64_t seed = 0) {
    detail::StateHolder h, o;
    detail::upload_checked(A, dims, "qpp::reset()", h);
    auto t = detail::u64(target);
    detail::check(qgpu_reset(h.s, detail::ptr(t), uint32_t(t.size()), seed, &o.s));
    return detail::download(o.s);
}

// qpp::discard(A, target, dims) (instruments.hpp:1243-1292), seeded.
inline cmat discard(const cmat& A, const std::vector<idx>& target, const std::vector<idx>& dims,
                    uint64_t seed = 0) {
    detail::StateHolder h, o;
    detail::upload_checked(A, dims, "qpp::discard()", h);
    auto t = detail::u64(target);
    detail::check(qgpu_discard(h.s, detail::ptr(t), uint32_t(t.size()), seed, &o.s));
    return detail::download(o.s);
}

#ifdef QPP_B200_HAS_EIGEN
// Eigen adapters: every function above also takes Eigen matrices (any
// Eigen::MatrixBase expression of complex or real scalars) and returns
// Eigen::MatrixXcd where qpp returns a matrix, so code written against
// qpp:: compiles against qpp_b200:: unchanged. Each adapter converts to a
// column-major cmat, calls the function above and converts back.
namespace detail {
template <typename D>
cmat from_eigen(const Eigen::MatrixBase<D>& m) {
    Eigen::MatrixXcd e = m.template cast<cplx>();
    cmat r(idx(e.rows()), idx(e.cols()));
    for (idx j = 0; j < r.cols(); ++j)
        for (idx i = 0; i < r.rows(); ++i) r(i, j) = e(Eigen::Index(i), Eigen::Index(j));
    return r;
}
inline Eigen::MatrixXcd to_eigen(const cmat& m) {
    Eigen::MatrixXcd e(Eigen::Index(m.rows()), Eigen::Index(m.cols()));
    for (idx j = 0; j < m.cols(); ++j)
        for (idx i = 0; i < m.rows(); ++i) e(Eigen::Index(i), Eigen::Index(j)) = m(i, j);
    return e;
}
template <typename M>
std::vector<cmat> from_eigen_list(const std::vector<M>& Ks) {
    std::vector<cmat> r;
    r.reserve(Ks.size());
    for (const auto& K : Ks) r.push_back(from_eigen(K));
    return r;
}
inline std::vector<Eigen::MatrixXcd> to_eigen_list(const std::vector<cmat>& v) {
    std::vector<Eigen::MatrixXcd> r;
    r.reserve(v.size());
    for (const auto& m : v) r.push_back(to_eigen(m));
    return r;
}
} // namespace detail

// apply (operations.hpp:72, :386)
template <typename D1, typename D2>
Eigen::MatrixXcd apply(const Eigen::MatrixBase<D1>& s, const Eigen::MatrixBase<D2>& A,
                       const std::vector<idx>& target, const std::vector<idx>& dims) {
    return detail::to_eigen(apply(detail::from_eigen(s), detail::from_eigen(A), target, dims));
}
template <typename D1, typename D2>
Eigen::MatrixXcd apply(const Eigen::MatrixBase<D1>& s, const Eigen::MatrixBase<D2>& A,
                       const std::vector<idx>& target, idx d = 2) {
    return detail::to_eigen(apply(detail::from_eigen(s), detail::from_eigen(A), target, d));
}
// applyCTRL / applyCTRL_fan (operations.hpp:616, :961)
template <typename D1, typename D2>
Eigen::MatrixXcd applyCTRL(const Eigen::MatrixBase<D1>& s, const Eigen::MatrixBase<D2>& A,
                           const std::vector<idx>& ctrl, const std::vector<idx>& target,
                           const std::vector<idx>& dims,
                           std::optional<std::vector<idx>> shift = std::nullopt) {
    return detail::to_eigen(
        applyCTRL(detail::from_eigen(s), detail::from_eigen(A), ctrl, target, dims, shift));
}
template <typename D1, typename D2>
Eigen::MatrixXcd applyCTRL_fan(const Eigen::MatrixBase<D1>& s, const Eigen::MatrixBase<D2>& A,
                               const std::vector<idx>& ctrl, const std::vector<idx>& target,
                               const std::vector<idx>& dims,
                               std::optional<std::vector<idx>> shift = std::nullopt) {
    return detail::to_eigen(
        applyCTRL_fan(detail::from_eigen(s), detail::from_eigen(A), ctrl, target, dims, shift));
}
// apply with Kraus operators (operations.hpp:476)
template <typename D, typename M>
Eigen::MatrixXcd apply(const Eigen::MatrixBase<D>& rho, const std::vector<M>& Ks,
                       const std::vector<idx>& target, const std::vector<idx>& dims) {
    return detail::to_eigen(
        apply(detail::from_eigen(rho), detail::from_eigen_list(Ks), target, dims));
}
// ptrace / ptranspose / syspermute (operations.hpp:1908, :2167, :2386)
template <typename D>
Eigen::MatrixXcd ptrace(const Eigen::MatrixBase<D>& A, const std::vector<idx>& target,
                        const std::vector<idx>& dims) {
    return detail::to_eigen(ptrace(detail::from_eigen(A), target, dims));
}
template <typename D>
Eigen::MatrixXcd ptranspose(const Eigen::MatrixBase<D>& A, const std::vector<idx>& target,
                            const std::vector<idx>& dims) {
    return detail::to_eigen(ptranspose(detail::from_eigen(A), target, dims));
}
template <typename D>
Eigen::MatrixXcd syspermute(const Eigen::MatrixBase<D>& A, const std::vector<idx>& perm,
                            const std::vector<idx>& dims) {
    return detail::to_eigen(syspermute(detail::from_eigen(A), perm, dims));
}
// sample / measure_seq (instruments.hpp:856, :985)
template <typename D>
std::map<std::vector<idx>, idx> sample(idx num_samples, const Eigen::MatrixBase<D>& A,
                                       const std::vector<idx>& target,
                                       const std::vector<idx>& dims, uint64_t seed = 0) {
    return sample(num_samples, detail::from_eigen(A), target, dims, seed);
}
template <typename D>
std::tuple<std::vector<idx>, std::vector<double>, Eigen::MatrixXcd>
measure_seq(const Eigen::MatrixBase<D>& A, const std::vector<idx>& target,
            const std::vector<idx>& dims, bool destructive = true, uint64_t seed = 0) {
    auto r = measure_seq(detail::from_eigen(A), target, dims, destructive, seed);
    return {std::get<0>(r), std::get<1>(r), detail::to_eigen(std::get<2>(r))};
}
// measure with Kraus operators / in a basis (instruments.hpp:371, :587)
template <typename D, typename M>
std::tuple<idx, std::vector<double>, std::vector<Eigen::MatrixXcd>>
measure(const Eigen::MatrixBase<D>& A, const std::vector<M>& Ks, const std::vector<idx>& target,
        const std::vector<idx>& dims, bool destructive = true, uint64_t seed = 0) {
    auto r = measure(detail::from_eigen(A), detail::from_eigen_list(Ks), target, dims,
                     destructive, seed);
    return {std::get<0>(r), std::get<1>(r), detail::to_eigen_list(std::get<2>(r))};
}
template <typename D1, typename D2>
std::tuple<idx, std::vector<double>, std::vector<Eigen::MatrixXcd>>
measure(const Eigen::MatrixBase<D1>& A, const Eigen::MatrixBase<D2>& V,
        const std::vector<idx>& target, const std::vector<idx>& dims, bool destructive = true,
        uint64_t seed = 0) {
    auto r = measure(detail::from_eigen(A), detail::from_eigen(V), target, dims, destructive,
                     seed);
    return {std::get<0>(r), std::get<1>(r), detail::to_eigen_list(std::get<2>(r))};
}
// reset / discard (instruments.hpp:1148, :1243)
template <typename D>
Eigen::MatrixXcd reset(const Eigen::MatrixBase<D>& A, const std::vector<idx>& target,
                       const std::vector<idx>& dims, uint64_t seed = 0) {
    return detail::to_eigen(reset(detail::from_eigen(A), target, dims, seed));
}
template <typename D>
Eigen::MatrixXcd discard(const Eigen::MatrixBase<D>& A, const std::vector<idx>& target,
                         const std::vector<idx>& dims, uint64_t seed = 0) {
    return detail::to_eigen(discard(detail::from_eigen(A), target, dims, seed));
}
// applyQFT / applyTFQ / QFT / TFQ (operations.hpp:2565, :2680, :2792, :2844)
template <typename D>
Eigen::MatrixXcd applyQFT(const Eigen::MatrixBase<D>& A, const std::vector<idx>& target,
                          idx d = 2, bool swap = true) {
    return detail::to_eigen(applyQFT(detail::from_eigen(A), target, d, swap));
}
template <typename D>
Eigen::MatrixXcd applyTFQ(const Eigen::MatrixBase<D>& A, const std::vector<idx>& target,
                          idx d = 2, bool swap = true) {
    return detail::to_eigen(applyTFQ(detail::from_eigen(A), target, d, swap));
}
template <typename D>
Eigen::MatrixXcd QFT(const Eigen::MatrixBase<D>& A, idx d = 2, bool swap = true) {
    return detail::to_eigen(QFT(detail::from_eigen(A), d, swap));
}
template <typename D>
Eigen::MatrixXcd TFQ(const Eigen::MatrixBase<D>& A, idx d = 2, bool swap = true) {
    return detail::to_eigen(TFQ(detail::from_eigen(A), d, swap));
}
#endif

} // namespace qpp_b200

#endif // QPP_B200_HPP_
