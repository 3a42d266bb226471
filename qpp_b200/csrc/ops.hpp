// ops.hpp -- device ops on qgpu_state handles (validated inputs assumed).
//
// Planning maps each Quantum++ op onto the virtual-ket kernels:
//   ket  over dims[0..n)            : virtual subsystems = dims
//   rho  (column-major D x D)       : virtual [col digits 0..n, row digits]
// A gate on rho is the superoperator conj(U) (x) U on (col t, row t) in one
// pass when DA <= 4, else U on the row digits then conj(U) on the columns;
// controlled gates fix the control digits so only the matching subspace is
// touched; a Kraus channel is its superoperator sum_i conj(K_i) (x) K_i.
#pragma once

#include <complex>
#include <cstdint>
#include <utility>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace qgpu {

using cd = std::complex<double>;

struct VSpace {
    std::vector<uint64_t> dims;    // big-endian: index 0 most significant
    std::vector<uint64_t> strides; // element stride of each subsystem
};

VSpace vspace_ket(const std::vector<uint64_t>& dims);
VSpace vspace_rho(const std::vector<uint64_t>& dims);
VSpace vspace_of(const qgpu_state* s);

// Groups over the subsystems not in `excluded`, merged into runs.
SegPlan plan_free(const VSpace& vs, const std::vector<int>& excluded,
                  uint64_t fixed_off);
// Dense gather: output digits (big-endian dims) with a source stride each.
SegPlan plan_gather(const std::vector<uint64_t>& out_dims,
                    const std::vector<uint64_t>& src_strides,
                    uint64_t fixed_off);
// off[m] = sum_j digit_j(m) * stride[target_j], big-endian over `targets`.
std::vector<uint64_t> target_offsets(const VSpace& vs,
                                     const std::vector<int>& targets);

// In-place gate on virtual targets with fixed digits elsewhere.
void vapply(qgpu_state* s, const VSpace& vs, const std::vector<int>& vt,
            const std::vector<std::pair<int, uint64_t>>& fixed, const cd* A,
            uint64_t DA);

std::vector<cd> conj_mat(const std::vector<cd>& A);
std::vector<cd> kron_mat(const std::vector<cd>& A, uint64_t da,
                         const std::vector<cd>& B, uint64_t db);
std::vector<cd> mat_pow(const std::vector<cd>& A, uint64_t m, uint64_t k);

qgpu_state* new_state(qgpu_ctx* ctx, qgpu_kind kind, qgpu_prec prec,
                      const std::vector<uint64_t>& dims, bool zero);
void free_state(qgpu_state* s);

void op_apply(qgpu_state* s, const cd* A, uint64_t DA,
              const std::vector<uint64_t>& target);
// shift_inv: qpp's inverted shift ((d - s) % d); fan applies a d x d A to
// each target.
void op_apply_ctrl(qgpu_state* s, const cd* A, uint64_t DA,
                   const std::vector<uint64_t>& ctrl,
                   const std::vector<uint64_t>& target,
                   const std::vector<uint64_t>& shift_inv, bool fan);
void op_apply_kraus(qgpu_state* s, const cd* Ks, uint32_t nK, uint64_t DA,
                    const std::vector<uint64_t>& target);
qgpu_state* op_ptrace(const qgpu_state* s, const std::vector<uint64_t>& target);
qgpu_state* op_ptranspose(const qgpu_state* s,
                          const std::vector<uint64_t>& target);
qgpu_state* op_syspermute(const qgpu_state* s,
                          const std::vector<uint64_t>& perm);
// The gates of qpp's QFT circuits, column-major: Fd(d) as qpp::Gates::Fd
// builds it (gates.hpp:260-285: H for d = 2, else pow(omega, i j) / sqrt(d),
// omega = exp(2 pi i / d)); R_j = diag(exp(+-2 pi i m / d^j))
// (operations.hpp:2616-2618, :2641-2646); SWAPd |a b> -> |b a>.
std::vector<cd> fourier_gate(uint64_t d);
std::vector<cd> qft_phase(uint64_t d, size_t j, bool inverse);
std::vector<cd> swap_gate(uint64_t d);
// qpp::applyQFT (inverse = false) / applyTFQ (true) on the state viewed as
// qudits of dimension d; in place (the state's buffer may be replaced).
void op_apply_qft(qgpu_state* s, const std::vector<uint64_t>& target, uint64_t d, bool swap,
                  bool inverse);
double op_norm2(const qgpu_state* s);
cd op_trace(const qgpu_state* s);
// qpp::normalize: ket / norm, rho / trace; returns false on a zero divisor.
bool op_normalize(qgpu_state* s);

} // namespace qgpu
