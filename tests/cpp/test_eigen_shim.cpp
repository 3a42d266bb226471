// Eigen-typed calls of the C++ drop-in layer (include/qpp_b200.hpp): every
// adapter compiles against the Eigen interface (here the stand-in under
// tests/cpp/eigen_standin, built with QPP_B200_HAS_EIGEN) and returns exactly
// what the same call on qpp_b200::cmat returns. Run on a GPU by
// tests/test_eigen_adapters.py; on the CPU the same file is only compiled.
#include <cmath>
#include <cstdio>
#include <random>

#include <Eigen/Dense>

#include "qpp_b200.hpp"

#ifndef QPP_B200_HAS_EIGEN
#error "the adapters need <Eigen/Dense> on the include path"
#endif

using namespace qpp_b200;

static int fails = 0;
#define EXPECT(c)                                                          \
    do {                                                                   \
        try {                                                              \
            if (!(c)) {                                                    \
                std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c);    \
                ++fails;                                                   \
            }                                                              \
        } catch (const std::exception& e) {                                \
            std::printf("FAIL %s:%d %s: %s\n", __FILE__, __LINE__, #c, e.what()); \
            ++fails;                                                       \
        }                                                                  \
    } while (0)

static std::mt19937_64 rng(5);

static Eigen::MatrixXcd rand_mat(idx r, idx c) {
    std::normal_distribution<double> nd;
    Eigen::MatrixXcd m(static_cast<Eigen::Index>(r), static_cast<Eigen::Index>(c));
    for (idx j = 0; j < c; ++j)
        for (idx i = 0; i < r; ++i) m(Eigen::Index(i), Eigen::Index(j)) = cplx(nd(rng), nd(rng));
    return m;
}

// a Haar-free unitary: the Cayley transform of a random anti-Hermitian matrix
// is enough here (the adapters are checked against the cmat calls)
static Eigen::MatrixXcd unitary(idx D) {
    cmat H = detail::from_eigen(rand_mat(D, D));
    cmat A(D, D);
    for (idx i = 0; i < D; ++i)
        for (idx j = 0; j < D; ++j) A(i, j) = 0.5 * (H(i, j) - std::conj(H(j, i)));
    // U = (I - A)^-1 (I + A) by Gauss-Jordan on [I - A | I + A]
    std::vector<std::vector<cplx>> M(D, std::vector<cplx>(2 * D));
    for (idx i = 0; i < D; ++i)
        for (idx j = 0; j < D; ++j) {
            M[i][j] = (i == j ? 1.0 : 0.0) - A(i, j);
            M[i][D + j] = (i == j ? 1.0 : 0.0) + A(i, j);
        }
    for (idx c = 0; c < D; ++c) {
        idx p = c;
        for (idx r = c + 1; r < D; ++r)
            if (std::abs(M[r][c]) > std::abs(M[p][c])) p = r;
        std::swap(M[c], M[p]);
        const cplx piv = M[c][c];
        for (auto& x : M[c]) x /= piv;
        for (idx r = 0; r < D; ++r)
            if (r != c) {
                const cplx f = M[r][c];
                for (idx k = 0; k < 2 * D; ++k) M[r][k] -= f * M[c][k];
            }
    }
    Eigen::MatrixXcd U(static_cast<Eigen::Index>(D), static_cast<Eigen::Index>(D));
    for (idx i = 0; i < D; ++i)
        for (idx j = 0; j < D; ++j) U(Eigen::Index(i), Eigen::Index(j)) = M[i][D + j];
    return U;
}

static bool same(const Eigen::MatrixXcd& e, const cmat& c) {
    if (idx(e.rows()) != c.rows() || idx(e.cols()) != c.cols()) return false;
    for (idx j = 0; j < c.cols(); ++j)
        for (idx i = 0; i < c.rows(); ++i)
            if (e(Eigen::Index(i), Eigen::Index(j)) != c(i, j)) return false;
    return true;
}

static int run() {
    const std::vector<idx> dims = {2, 3, 2, 2};
    const idx D = 24;
    Eigen::MatrixXcd psi = rand_mat(D, 1), rho = rand_mat(D, D);
    const cmat cpsi = detail::from_eigen(psi), crho = detail::from_eigen(rho);
    const Eigen::MatrixXcd U2 = unitary(2), U6 = unitary(6);
    const cmat cU2 = detail::from_eigen(U2), cU6 = detail::from_eigen(U6);

    EXPECT(same(apply(psi, U6, {1, 2}, dims), apply(cpsi, cU6, {1, 2}, dims)));
    EXPECT(same(apply(rho, U2, {3}, dims), apply(crho, cU2, {3}, dims)));
    Eigen::MatrixXcd q = rand_mat(8, 1);
    EXPECT(same(apply(q, U2, {1}), apply(detail::from_eigen(q), cU2, {1})));
    EXPECT(same(applyCTRL(psi, U2, {0}, {2}, dims), applyCTRL(cpsi, cU2, {0}, {2}, dims)));
    EXPECT(same(applyCTRL(rho, U2, {2}, {3}, dims, std::vector<idx>{1}),
                applyCTRL(crho, cU2, {2}, {3}, dims, std::vector<idx>{1})));
    EXPECT(same(applyCTRL_fan(psi, U2, {2}, {0, 3}, dims),
                applyCTRL_fan(cpsi, cU2, {2}, {0, 3}, dims)));
    // Kraus operators: an amplitude-damping pair on qubit 3
    const double g = 0.3;
    Eigen::MatrixXcd K0(2, 2), K1(2, 2);
    K0(0, 0) = 1.0; K0(0, 1) = 0.0; K0(1, 0) = 0.0; K0(1, 1) = std::sqrt(1 - g);
    K1(0, 0) = 0.0; K1(0, 1) = std::sqrt(g); K1(1, 0) = 0.0; K1(1, 1) = 0.0;
    std::vector<Eigen::MatrixXcd> Ks = {K0, K1};
    EXPECT(same(apply(rho, Ks, {3}, dims),
                apply(crho, detail::from_eigen_list(Ks), {3}, dims)));
    EXPECT(same(ptrace(rho, {1, 3}, dims), ptrace(crho, {1, 3}, dims)));
    EXPECT(same(ptrace(psi, {0}, dims), ptrace(cpsi, {0}, dims)));
    EXPECT(same(ptranspose(rho, {0, 1}, dims), ptranspose(crho, {0, 1}, dims)));
    EXPECT(same(syspermute(rho, {2, 0, 3, 1}, dims), syspermute(crho, {2, 0, 3, 1}, dims)));
    EXPECT(same(syspermute(psi, {3, 1, 0, 2}, dims), syspermute(cpsi, {3, 1, 0, 2}, dims)));
    // instruments, seeded
    EXPECT(sample(50, psi, {0, 1}, dims, 3) == sample(50, cpsi, {0, 1}, dims, 3));
    {
        auto a = measure_seq(psi, {1, 3}, dims, true, 9);
        auto b = measure_seq(cpsi, {1, 3}, dims, true, 9);
        EXPECT(std::get<0>(a) == std::get<0>(b) && std::get<1>(a) == std::get<1>(b));
        EXPECT(same(std::get<2>(a), std::get<2>(b)));
    }
    {
        auto a = measure(rho, Ks, {2}, dims, false, 4);
        auto b = measure(crho, detail::from_eigen_list(Ks), {2}, dims, false, 4);
        EXPECT(std::get<0>(a) == std::get<0>(b) && std::get<1>(a) == std::get<1>(b));
        EXPECT(std::get<2>(a).size() == std::get<2>(b).size());
        for (size_t i = 0; i < std::get<2>(a).size(); ++i)
            EXPECT(same(std::get<2>(a)[i], std::get<2>(b)[i]));
    }
    {
        auto a = measure(psi, U2, {0}, dims, true, 2);
        auto b = measure(cpsi, cU2, {0}, dims, true, 2);
        EXPECT(std::get<0>(a) == std::get<0>(b) && std::get<1>(a) == std::get<1>(b));
        for (size_t i = 0; i < std::get<2>(a).size(); ++i)
            EXPECT(same(std::get<2>(a)[i], std::get<2>(b)[i]));
    }
    EXPECT(same(reset(psi, {2}, dims, 6), reset(cpsi, {2}, dims, 6)));
    // qpp's reset takes the i-th target's dimension from dims[i]
    // (instruments.hpp:1190-1192), so a qutrit target in first place throws
    bool reset_thrown = false;
    try {
        reset(psi, {1}, dims, 6);
    } catch (const exception::MatrixMismatchSubsys& e) {
        reset_thrown = e.where() == "qpp::apply()";
    }
    EXPECT(reset_thrown);
    EXPECT(same(discard(rho, {0, 2}, dims, 6), discard(crho, {0, 2}, dims, 6)));
    Eigen::MatrixXcd k = rand_mat(16, 1);
    const cmat ck = detail::from_eigen(k);
    EXPECT(same(applyQFT(k, {0, 2, 3}), applyQFT(ck, {0, 2, 3})));
    EXPECT(same(applyTFQ(k, {3, 1}), applyTFQ(ck, {3, 1})));
    EXPECT(same(QFT(k), QFT(ck)));
    EXPECT(same(TFQ(k, 2, false), TFQ(ck, 2, false)));
    // qpp's exception types come through the adapters as well
    bool thrown = false;
    try {
        ptrace(rho, {7}, dims);
    } catch (const exception::SubsysMismatchDims& e) {
        thrown = e.where() == "qpp::ptrace()";
    }
    EXPECT(thrown);
    if (fails) {
        std::printf("%d failures\n", fails);
        return 1;
    }
    std::printf("eigen adapters ok\n");
    return 0;
}

int main() {
    try {
        return run();
    } catch (const std::exception& e) {
        std::printf("unexpected exception: %s\n", e.what());
        return 1;
    }
}
