// C++17 drop-in check: the qpp_b200:: functions with qpp's signatures on the
// known answers of the reference suite (unit_tests/tests/operations.cpp:16-74,
// :101-162) and qpp's exception types. Built and run by tests/test_cpp_shim.py.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "qpp_b200.hpp"

using namespace qpp_b200;

static int fails = 0;
#define EXPECT(c)                                                          \
    do {                                                                   \
        if (!(c)) {                                                        \
            std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c);        \
            ++fails;                                                       \
        }                                                                  \
    } while (0)

static cmat ket_bits(const char* s) {
    idx n = 0;
    while (s[n]) ++n;
    idx i = 0;
    for (idx k = 0; k < n; ++k) i = 2 * i + idx(s[k] - '0');
    cmat v(idx(1) << n, 1);
    v(i) = 1;
    return v;
}
static cmat lin(double a, const cmat& x, double b, const cmat& y) {
    cmat r(x.rows(), x.cols());
    for (idx i = 0; i < x.data_.size(); ++i) r.data_[i] = a * x.data_[i] + b * y.data_[i];
    return r;
}
static double dist(const cmat& a, const cmat& b) {
    double s = 0;
    for (idx i = 0; i < a.data_.size(); ++i) s += std::norm(a.data_[i] - b.data_[i]);
    return std::sqrt(s);
}

int main() {
    cmat X(2, 2), Z(2, 2), CNOT(4, 4);
    X(0, 1) = X(1, 0) = 1;
    Z(0, 0) = 1;
    Z(1, 1) = -1;
    CNOT(0, 0) = CNOT(1, 1) = CNOT(2, 3) = CNOT(3, 2) = 1;
    // operations.cpp:30-40
    cmat psi = lin(0.8, ket_bits("00"), 0.6, ket_bits("11"));
    EXPECT(dist(apply(psi, X, {1}, {2, 2}), lin(0.8, ket_bits("01"), 0.6, ket_bits("10"))) == 0);
    EXPECT(dist(apply(psi, Z, {1}, {2, 2}), lin(0.8, ket_bits("00"), -0.6, ket_bits("11"))) == 0);
    EXPECT(dist(apply(psi, CNOT, {0, 1}, {2, 2}), lin(0.8, ket_bits("00"), 0.6, ket_bits("10"))) == 0);
    EXPECT(dist(apply(psi, CNOT, {1, 0}), lin(0.8, ket_bits("00"), 0.6, ket_bits("01"))) == 0);
    // applyCTRL on qubits: CNOT as CTRL-X
    EXPECT(dist(applyCTRL(psi, X, {0}, {1}, {2, 2}), apply(psi, CNOT, {0, 1}, {2, 2})) < 1e-15);
    // ptrace of |00><00| + |11><11| mixture -> diag(0.64, 0.36)
    cmat rho(4, 4);
    for (idx r = 0; r < 4; ++r)
        for (idx c = 0; c < 4; ++c) rho(r, c) = psi(r) * std::conj(psi(c));
    cmat red = ptrace(rho, {1}, {2, 2});
    EXPECT(std::abs(red(0, 0) - 0.64) < 1e-15 && std::abs(red(1, 1) - 0.36) < 1e-15);
    EXPECT(dist(syspermute(rho, {1, 0}, {2, 2}), rho) == 0);
    // exceptions carry qpp's types and (where, what)
    bool caught = false;
    try {
        apply(psi, X, {2}, {2, 2});
    } catch (const exception::SubsysMismatchDims& e) {
        caught = e.where() == "qpp::apply()" && e.detail() == "dims/target";
    }
    EXPECT(caught);
    caught = false;
    try {
        syspermute(rho, {0, 0}, {2, 2});
    } catch (const exception::PermInvalid&) {
        caught = true;
    }
    EXPECT(caught);
    // sampling and sequential measurement of the Bell state (|00> + |11>)/sqrt2
    cmat bell(4, 1);
    bell(0) = bell(3) = 1 / std::sqrt(2.0);
    auto counts = sample(200, bell, {0, 1}, {2, 2}, 7);
    idx total = 0;
    for (auto& kv : counts) {
        EXPECT(kv.first.size() == 2 && kv.first[0] == kv.first[1]);
        total += kv.second;
    }
    EXPECT(total == 200 && counts.size() == 2);
    auto [res, probs, post] = measure_seq(bell, {0}, {2, 2}, true, 3);
    EXPECT(res.size() == 1 && std::abs(probs[0] - 0.5) < 1e-15);
    EXPECT(post.rows() == 2 && post.cols() == 1 && std::abs(std::abs(post(res[0])) - 1) < 1e-15);
    caught = false;
    try {
        sample(0, bell, {0}, {2, 2});
    } catch (const exception::OutOfRange& e) {
        caught = e.where() == "qpp::sample()" && e.detail() == "num_samples";
    }
    EXPECT(caught);
    // measuring the first qubit of the Bell state with projectors / a basis
    cmat P0(2, 2), P1(2, 2);
    P0(0, 0) = 1;
    P1(1, 1) = 1;
    auto [mr, mp, ms] = measure(bell, std::vector<cmat>{P0, P1}, {0}, {2, 2}, true, 5);
    EXPECT(mp.size() == 2 && std::abs(mp[0] - 0.5) < 1e-15 && std::abs(mp[1] - 0.5) < 1e-15);
    EXPECT(ms[mr].rows() == 2 && ms[mr].cols() == 2 && std::abs(ms[mr](mr, mr) - 1.0) < 1e-15);
    cmat I2(2, 2);
    I2(0, 0) = I2(1, 1) = 1;
    auto [br, bp, bs] = measure(bell, I2, {1}, {2, 2}, true, 5);
    EXPECT(bs[br].rows() == 2 && bs[br].cols() == 1 && std::abs(std::abs(bs[br](br)) - 1.0) < 1e-15);
    cmat z = reset(bell, {0, 1}, {2, 2}, 9);
    EXPECT(std::abs(std::abs(z(0)) - 1.0) < 1e-15);
    cmat dsc = discard(bell, {0}, {2, 2}, 9);
    EXPECT(dsc.rows() == 2 && dsc.cols() == 1);
    // QFT of |1> on 3 qubits: amplitudes exp(2 pi i y / 8) / sqrt(8); TFQ
    // brings it back; applyQFT on one qubit is H
    cmat one(8, 1);
    one(1) = 1;
    cmat f = QFT(one);
    double qerr = 0;
    for (idx y = 0; y < 8; ++y)
        qerr = std::max(qerr, std::abs(f(y) - std::polar(1.0 / std::sqrt(8.0), 2 * M_PI * y / 8.0)));
    EXPECT(qerr < 1e-15);
    EXPECT(dist(TFQ(f), one) < 1e-15);
    cmat H(2, 2);
    H(0, 0) = H(0, 1) = H(1, 0) = 1 / std::sqrt(2.0);
    H(1, 1) = -1 / std::sqrt(2.0);
    EXPECT(dist(applyQFT(one, {2}), apply(one, H, {2}, {2, 2, 2})) < 1e-15);
    caught = false;
    try {
        applyQFT(one, {3});
    } catch (const exception::SubsysMismatchDims& e) {
        caught = e.where() == "qpp::applyQFT()" && e.detail() == "dims/target";
    }
    EXPECT(caught);
    std::printf(fails ? "shim FAILED (%d)\n" : "shim ok\n", fails);
    return fails ? 1 : 0;
}
