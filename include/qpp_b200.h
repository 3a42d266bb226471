/*
 * qpp_b200.h -- C ABI of the B200-native Quantum++ gate-application and
 * subsystem-manipulation path.
 *
 * Conventions (identical to Quantum++ 7.0.3, include/qpp/types.hpp:127-178):
 *   - complex numbers are interleaved (re, im) pairs of double (c128) or
 *     float (c64); gate matrices passed to this ABI are always c128;
 *   - a ket is a D x 1 column, a density matrix is a D x D matrix stored
 *     column-major (element (r, c) at r + c * D);
 *   - multi-indices are big-endian mixed radix: subsystem 0 is the most
 *     significant digit (include/qpp/internal/util.hpp:58-116);
 *   - a gate on k target subsystems is a DA x DA matrix, DA = prod dims[t],
 *     whose row/column index is the big-endian multi-index over `target`
 *     in the order given.
 *
 * Ownership: host arrays are borrowed for the duration of a call. Device
 * states are owned by qgpu_state handles; ops on a handle work in place in
 * HBM (the resident path). The qgpu_host_* entry points keep Quantum++'s
 * value semantics: the input is const, the result is written to a caller
 * buffer.
 *
 * Errors: every entry point returns a qgpu_status. Validation follows the
 * order of the corresponding qpp function, so the first error reported is
 * the one qpp would throw; qgpu_last_error_where()/what() return qpp's
 * (where, what) strings, e.g. ("qpp::apply()", "dims/target").
 *
 * Threading: a context may be used from several threads; a state handle may
 * not be used by two threads at once. A circuit keeps the plans of its fused
 * forms (built by the first qgpu_run_gates in that form, again after steps
 * are added): run it in a fused form from one thread at a time, or run it
 * once before sharing it. Errors are recorded per thread.
 */
#ifndef QPP_B200_H_
#define QPP_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One value per qpp::exception type used on this path
 * (include/qpp/classes/exception.hpp:129-655), plus device-side codes. */
typedef enum qgpu_status {
    QGPU_OK = 0,
    QGPU_ERR_ZERO_SIZE = 1,                     /* exception::ZeroSize */
    QGPU_ERR_MATRIX_NOT_SQUARE = 2,             /* exception::MatrixNotSquare */
    QGPU_ERR_MATRIX_NOT_SQUARE_NOR_CVECTOR = 3, /* MatrixNotSquareNorCvector */
    QGPU_ERR_MATRIX_MISMATCH_SUBSYS = 4,        /* MatrixMismatchSubsys */
    QGPU_ERR_DIMS_INVALID = 5,                  /* DimsInvalid */
    QGPU_ERR_DIMS_NOT_EQUAL = 6,                /* DimsNotEqual */
    QGPU_ERR_DIMS_MISMATCH_MATRIX = 7,          /* DimsMismatchMatrix */
    QGPU_ERR_DIMS_MISMATCH_CVECTOR = 8,         /* DimsMismatchCvector */
    QGPU_ERR_SUBSYS_MISMATCH_DIMS = 9,          /* SubsysMismatchDims */
    QGPU_ERR_PERM_INVALID = 10,                 /* PermInvalid */
    QGPU_ERR_PERM_MISMATCH_DIMS = 11,           /* PermMismatchDims */
    QGPU_ERR_OUT_OF_RANGE = 12,                 /* OutOfRange */
    QGPU_ERR_TYPE_MISMATCH = 13,                /* TypeMismatch */
    QGPU_ERR_SIZE_MISMATCH = 14,                /* SizeMismatch */
    QGPU_ERR_QUDIT_ALREADY_MEASURED = 15,       /* QuditAlreadyMeasured */
    QGPU_ERR_MATRIX_NOT_SQUARE_NOR_VECTOR = 16, /* MatrixNotSquareNorVector */
    QGPU_ERR_DIVISION_BY_ZERO = 17, /* std::overflow_error in normalize() */
    QGPU_ERR_DUPLICATES = 18,       /* exception::Duplicates */
    /* device-side and library codes (no qpp counterpart) */
    QGPU_ERR_CUDA = 100,         /* a CUDA runtime call failed */
    QGPU_ERR_OUT_OF_MEMORY = 101, /* device allocation or admission refused */
    QGPU_ERR_TIMEOUT = 102,      /* a bounded device wait gave up */
    QGPU_ERR_INVALID_HANDLE = 103,
    QGPU_ERR_NOT_SUPPORTED = 104, /* size or form outside what is built */
    QGPU_ERR_INVALID_ARGUMENT = 105
} qgpu_status;

typedef enum qgpu_kind { QGPU_KET = 0, QGPU_RHO = 1 } qgpu_kind;
typedef enum qgpu_prec { QGPU_C128 = 0, QGPU_C64 = 1 } qgpu_prec;

typedef struct qgpu_ctx qgpu_ctx;
typedef struct qgpu_state qgpu_state;

/* ---------------------------------------------------------------- errors */
const char* qgpu_last_error_where(void);
const char* qgpu_last_error_what(void);
const char* qgpu_status_name(qgpu_status s);
/* Library version string. */
const char* qgpu_version(void);

/* --------------------------------------------------------------- context */
/* A context binds one CUDA device and owns the stream every op runs on. */
qgpu_status qgpu_ctx_create(int device, qgpu_ctx** out);
qgpu_status qgpu_ctx_destroy(qgpu_ctx* ctx);
qgpu_status qgpu_ctx_synchronize(qgpu_ctx* ctx);
/* Device bytes currently free / total (cudaMemGetInfo on the ctx device). */
qgpu_status qgpu_ctx_mem_info(qgpu_ctx* ctx, uint64_t* free_bytes,
                              uint64_t* total_bytes);
/* Number of kernels this library launched on the context since creation. */
uint64_t qgpu_ctx_launch_count(const qgpu_ctx* ctx);
/* The cudaStream_t every op of this context is issued on, as void*. */
void* qgpu_ctx_stream(qgpu_ctx* ctx);
/* Bounded-wait controls of the fused tensor-core passes (no counterpart in
 * Quantum++, which has no device waits). spin_limit: iterations of each wait
 * for the tensor cores (0 restores the default, 2^26). stall_next != 0: the
 * next fused pass on this context first waits on a barrier that nothing
 * completes, so that wait runs out: the pass records the timeout, lets its
 * own tensor-core work finish, frees its tensor memory and returns, and the
 * call reports QGPU_ERR_TIMEOUT; the context stays usable. For tests of the
 * timeout path; one-shot. */
qgpu_status qgpu_ctx_set_wait_test(qgpu_ctx* ctx, uint32_t spin_limit, int stall_next);
/* Largest tile, in state bits (5..14), of the tile passes that run the plain
 * form of qgpu_run_gates on qubit kets (runs of 1- and 2-qubit gates, each run
 * one read and one write of the state); 0 restores the default, which is
 * also the cap: 13 for complex128 and 14 for complex64 (128 KB of shared
 * memory per tile). No counterpart
 * in Quantum++, which applies one gate per pass. */
qgpu_status qgpu_ctx_set_tile_bits(qgpu_ctx* ctx, int bits);

/* ---------------------------------------------------------------- states */
/* Allocate a ket (D x 1) or density matrix (D x D) over `dims` in HBM,
 * zero-initialised. Fails with QGPU_ERR_DIMS_INVALID for empty dims or a
 * zero dimension (internal::check_dims, util.hpp:158-166). */
qgpu_status qgpu_state_create(qgpu_ctx* ctx, qgpu_kind kind, qgpu_prec prec,
                              const uint64_t* dims, uint32_t n,
                              qgpu_state** out);
qgpu_status qgpu_state_destroy(qgpu_state* s);
qgpu_status qgpu_state_clone(const qgpu_state* s, qgpu_state** out);
/* Copy host data in the state's own precision (interleaved, column-major). */
qgpu_status qgpu_state_upload(qgpu_state* s, const void* host);
qgpu_status qgpu_state_download(const qgpu_state* s, void* host);
/* Copy c128 host data, converting on the device for c64 states. */
qgpu_status qgpu_state_upload_c128(qgpu_state* s, const double* host);
qgpu_status qgpu_state_download_c128(const qgpu_state* s, double* host);
qgpu_status qgpu_state_info(const qgpu_state* s, qgpu_kind* kind,
                            qgpu_prec* prec, uint32_t* n, uint64_t* dims,
                            uint64_t* D);
/* Device pointer of the amplitudes (c128: double2*, c64: float2*). */
void* qgpu_state_device_ptr(qgpu_state* s);
/* Fill with i.i.d. complex Gaussian entries (re, im ~ N(0, 1)) from the
 * counter-based Philox4x32-10 generator keyed by `seed` (element index as
 * the counter), then normalise as qpp::normalize does. The same stream is
 * reproducible on the host. */
qgpu_status qgpu_state_fill_gaussian(qgpu_state* s, uint64_t seed);
/* Copy a state into another of the same kind and dims, converting the
 * precision on the device (c128 <-> c64). */
qgpu_status qgpu_state_convert(const qgpu_state* src, qgpu_state* dst);

/* ------------------------------------------------- resident ops (in HBM) */
/* qpp::apply(state, A, target, dims), operations.hpp:72-372; in place. */
qgpu_status qgpu_apply(qgpu_state* s, const double* A, uint64_t DA,
                       const uint64_t* target, uint32_t k);
/* qpp::applyCTRL(state, A, ctrl, target, dims, shift), operations.hpp:616-887.
 * shift may be NULL (std::nullopt). */
qgpu_status qgpu_apply_ctrl(qgpu_state* s, const double* A, uint64_t DA,
                            const uint64_t* ctrl, uint32_t nc,
                            const uint64_t* target, uint32_t k,
                            const uint64_t* shift);
/* qpp::applyCTRL_fan(...), operations.hpp:961-1234 (A is d x d). */
qgpu_status qgpu_apply_ctrl_fan(qgpu_state* s, const double* A, uint64_t DA,
                                const uint64_t* ctrl, uint32_t nc,
                                const uint64_t* target, uint32_t k,
                                const uint64_t* shift);
/* qpp::apply(A, Ks, target, dims), operations.hpp:476-560: the channel
 * sum_i K_i rho K_i^dagger on the subsystems `target`, in place.
 * Ks holds nK consecutive DA x DA column-major c128 matrices. */
qgpu_status qgpu_apply_kraus(qgpu_state* s, const double* Ks, uint32_t nK,
                             uint64_t DA, const uint64_t* target, uint32_t k);
/* qpp::ptrace(A, target, dims), operations.hpp:1908-2114: writes a new
 * density-matrix state over the complement of `target`. */
qgpu_status qgpu_ptrace(const qgpu_state* s, const uint64_t* target,
                        uint32_t k, qgpu_state** out);
/* qpp::ptranspose(A, target, dims), operations.hpp:2167-2335: a new
 * D x D density-matrix state (a ket input gives (|psi><psi|)^{T_target}). */
qgpu_status qgpu_ptranspose(const qgpu_state* s, const uint64_t* target,
                            uint32_t k, qgpu_state** out);
/* qpp::syspermute(A, perm, dims), operations.hpp:2386-2514: subsystem
 * perm[i] moves to position i; writes a new state of the same kind. */
qgpu_status qgpu_syspermute(const qgpu_state* s, const uint64_t* perm,
                            uint32_t n, qgpu_state** out);
/* qpp::applyQFT(A, target, d, swap) (inverse = 0, operations.hpp:2565-2676)
 * and qpp::applyTFQ (inverse = 1, :2680-2787), in place: the qudit quantum
 * Fourier transform (or its adjoint) on the targets of the state viewed as
 * n = round(log2 D / log2 d) qudits of dimension d (a density matrix gets
 * U rho U^dagger). target[0] is the most significant digit of the
 * transformed register; swap reverses the targets at the end (QFT) or the
 * start (TFQ), as qpp's SWAP gates do. The steps of up to 8 consecutive
 * targets run as one pass over the state in shared memory, so the transform
 * costs ceil(k / 8) passes (qubits; fewer targets per pass for d > 2)
 * instead of qpp's k (k + 1) / 2 gate passes; with swap the reversal rides
 * on the last pass, which writes a new buffer (the state's device pointer
 * changes). Results match qpp's gate sequence to rounding (the butterflies
 * sum the same terms). d above 16 runs qpp's gate sequence on the gate
 * kernels. */
qgpu_status qgpu_apply_qft(qgpu_state* s, const uint64_t* target, uint32_t k, uint64_t d,
                           int swap, int inverse);
/* qpp::QFT(A, d, swap) / qpp::TFQ (operations.hpp:2792-2899): every digit
 * is a target, in order. */
qgpu_status qgpu_qft(qgpu_state* s, uint64_t d, int swap, int inverse);
/* Partial trace that allocates nothing. No counterpart in the reference:
 * Quantum++ always returns a freshly allocated matrix. This entry point is
 * for callers that cannot allocate device memory when they need the trace --
 * an application whose own memory pool holds all of the GPU's free memory, or
 * a latency-critical loop that cannot afford the device-wide synchronisation
 * of cudaMalloc / cudaFree. The result (the Dbar x Dbar density matrix over
 * the kept subsystems, column-major, in the state's precision, Dbar = D /
 * prod dims[target]) is written to d_out, device memory the caller owns.
 * The table of traced offsets lives in a fixed array of 65536 entries
 * (512 KB) that the library keeps on every GPU that loads it until the
 * process exits; a traced dimension prod dims[target] above 65536 is
 * rejected with QGPU_ERR_NOT_SUPPORTED. The first call on a device, and the
 * first one after each qgpu_ctx_create on that device (a cudaDeviceReset in
 * between can move the array), looks up the array's device address, so that
 * call should come before any stream capture. Invalid targets are reported
 * with where = "qgpu_ptrace_noalloc()". Every call shares that one array:
 * calls whose
 * work overlaps on the GPU (different streams, different contexts of the
 * same device) race on it, so serialise them. The work is queued on the
 * state's context stream; synchronise that stream before reading d_out
 * elsewhere. */
qgpu_status qgpu_ptrace_noalloc(const qgpu_state* s, const uint64_t* target,
                                uint32_t k, void* d_out);
/* Squared norm (ket) or trace (rho, real and imaginary parts), FP64
 * accumulation. */
qgpu_status qgpu_norm2(const qgpu_state* s, double* out);
qgpu_status qgpu_trace(const qgpu_state* s, double* re, double* im);
/* qpp::normalize(A), functions.hpp:304-333, in place (ket / norm,
 * rho / trace). */
qgpu_status qgpu_normalize(qgpu_state* s);
/* <a|b> for two kets over the same dims, or tr(A^dagger B) for two density
 * matrices (FP64 accumulation; no qpp counterpart). */
qgpu_status qgpu_inner(const qgpu_state* a, const qgpu_state* b, double* re,
                       double* im);

/* ----------------------------------------- Z-basis sampling and measurement
 * Replaces qpp::sample(num_samples, A, target, dims)
 * (instruments.hpp:856-940): num_samples full-basis draws of |A_i|^2 (ket)
 * or Re A(i, i) (density matrix); results[i * k + j] = digit of target[j] in
 * draw i. The draws are std::discrete_distribution's: u = the caller's
 * uniforms in [0, 1) when u != NULL, else generate_canonical<double, 53> of a
 * std::mt19937 seeded with `seed` (qpp's generator, seeded); index = the first
 * whose FP64 prefix sum reaches u * total. One pass over the state plus one
 * 4096-weight chunk scanned per draw. */
qgpu_status qgpu_sample(const qgpu_state* s, const uint64_t* target, uint32_t k,
                        uint64_t num_samples, uint64_t seed, const double* u,
                        uint64_t* results);
/* Replaces qpp::measure_seq(A, target, dims, destructive)
 * (instruments.hpp:985-1111), value semantics: one full-basis draw (seeded
 * as above; forced != NULL gives the outcomes instead), then each target is
 * projected and renormalised (probs = qpp's conditional probabilities);
 * destructive drops the measured subsystems. *out is a new state; `s` is
 * unchanged. */
qgpu_status qgpu_measure_seq(const qgpu_state* s, const uint64_t* target, uint32_t k,
                             int destructive, uint64_t seed, const uint64_t* forced,
                             uint64_t* results, double* probs, qgpu_state** out);
/* Replaces qpp::measure(A, Ks, target, dims, destructive)
 * (instruments.hpp:371-494): each of the nK Kraus operators (DK x DK,
 * consecutive, column-major, DK = the targets' dimension) is applied on the
 * targets (K psi, or K rho K^dagger); probs[i] = ||K psi||^2 or |tr|, outs[i]
 * = the normalised post-measurement state (a new handle; the targets traced
 * out when destructive, which makes a ket's result a density matrix; NULL
 * where probs[i] == 0); *result = one std::discrete_distribution draw of a
 * std::mt19937 seeded with `seed`. outs may be NULL. All probabilities zero:
 * QGPU_ERR_DIVISION_BY_ZERO. */
qgpu_status qgpu_measure_kraus(const qgpu_state* s, const double* Ks, uint32_t nK,
                               uint64_t DK, const uint64_t* target, uint32_t k,
                               int destructive, uint64_t seed, uint64_t* result,
                               double* probs, qgpu_state** outs);
/* Replaces qpp::measure(A, V, target, dims, destructive)
 * (instruments.hpp:587-712): the M columns of V (rows x M, rows = the
 * targets' dimension) as rank-1 projectors; a ket measured destructively
 * keeps <v_i|psi> over the targets (a ket of the other subsystems). Outputs
 * as qgpu_measure_kraus. */
qgpu_status qgpu_measure_basis(const qgpu_state* s, const double* V, uint64_t rows,
                               uint64_t M, const uint64_t* target, uint32_t k,
                               int destructive, uint64_t seed, uint64_t* result,
                               double* probs, qgpu_state** outs);
/* Replaces qpp::reset(A, target, dims) (instruments.hpp:1148-1206): a seeded
 * non-destructive measure_seq, then Xd^(d - result_i) on each target, with
 * d = dims[i] (qpp indexes dims by the target's position). New handle. */
qgpu_status qgpu_reset(const qgpu_state* s, const uint64_t* target, uint32_t k,
                       uint64_t seed, qgpu_state** out);
/* Replaces qpp::discard(A, target, dims) (instruments.hpp:1243-1292): a seeded
 * destructive measure_seq; the post-measurement state as a new handle. */
qgpu_status qgpu_discard(const qgpu_state* s, const uint64_t* target, uint32_t k,
                         uint64_t seed, qgpu_state** out);

/* ------------------------------------- value-semantics entry points (host)
 * These mirror qpp's free functions exactly: the state is a host array with
 * `rows` x `cols` (cols == 1 for a ket, rows == cols for a density matrix),
 * the result goes to a host buffer. Each call uploads, runs the device op
 * and downloads; they exist so that a caller binding qpp's signatures can
 * switch without keeping states resident. */
qgpu_status qgpu_host_apply(qgpu_ctx* ctx, const double* state, uint64_t rows,
                            uint64_t cols, const double* A, uint64_t A_rows,
                            uint64_t A_cols, const uint64_t* target,
                            uint32_t k, const uint64_t* dims, uint32_t n,
                            double* result);
qgpu_status qgpu_host_apply_ctrl(qgpu_ctx* ctx, const double* state,
                                 uint64_t rows, uint64_t cols, const double* A,
                                 uint64_t A_rows, uint64_t A_cols,
                                 const uint64_t* ctrl, uint32_t nc,
                                 const uint64_t* target, uint32_t k,
                                 const uint64_t* dims, uint32_t n,
                                 const uint64_t* shift, int fan,
                                 double* result);
qgpu_status qgpu_host_apply_kraus(qgpu_ctx* ctx, const double* state,
                                  uint64_t rows, uint64_t cols,
                                  const double* Ks, uint32_t nK,
                                  uint64_t K_rows, uint64_t K_cols,
                                  const uint64_t* target, uint32_t k,
                                  const uint64_t* dims, uint32_t n,
                                  double* result);
/* result is Dbar x Dbar, Dbar = D / prod dims[target]. */
qgpu_status qgpu_host_ptrace(qgpu_ctx* ctx, const double* state, uint64_t rows,
                             uint64_t cols, const uint64_t* target, uint32_t k,
                             const uint64_t* dims, uint32_t n, double* result);
/* result is D x D. */
qgpu_status qgpu_host_ptranspose(qgpu_ctx* ctx, const double* state,
                                 uint64_t rows, uint64_t cols,
                                 const uint64_t* target, uint32_t k,
                                 const uint64_t* dims, uint32_t n,
                                 double* result);
/* result has the input's shape. */
qgpu_status qgpu_host_syspermute(qgpu_ctx* ctx, const double* state,
                                 uint64_t rows, uint64_t cols,
                                 const uint64_t* perm, uint32_t nperm,
                                 const uint64_t* dims, uint32_t n,
                                 double* result);

/* qpp::applyQFT / applyTFQ (inverse = 1) on a host array; result has the
 * input's shape. */
qgpu_status qgpu_host_apply_qft(qgpu_ctx* ctx, const double* state, uint64_t rows,
                                uint64_t cols, const uint64_t* target, uint32_t k,
                                uint64_t d, int swap, int inverse, double* result);
/* qpp::QFT / TFQ (inverse = 1) on a host array. */
qgpu_status qgpu_host_qft(qgpu_ctx* ctx, const double* state, uint64_t rows, uint64_t cols,
                          uint64_t d, int swap, int inverse, double* result);

/* --------------------------------------------------------------- circuits
 * The step list of qpp::QCircuit (include/qpp/classes/qcircuit.hpp) over nq
 * qudits of dimension d with nc classical dits. Step checks follow
 * QCircuit's (qcircuit.hpp:1166-1483), with "Step <i>: <what>" messages. */
typedef struct qgpu_circuit qgpu_circuit;
qgpu_status qgpu_circuit_create(uint32_t nq, uint64_t d, uint32_t nc,
                                qgpu_circuit** out);
qgpu_status qgpu_circuit_destroy(qgpu_circuit* c);
/* QCircuit::gate(U, target), qcircuit.hpp:1166-1483 (U is d^k x d^k). */
qgpu_status qgpu_circuit_gate(qgpu_circuit* c, const double* U, uint64_t DU,
                              const uint64_t* target, uint32_t k);
/* QCircuit::gate_fan(U, target): the d x d U on every target. */
qgpu_status qgpu_circuit_gate_fan(qgpu_circuit* c, const double* U,
                                  uint64_t DU, const uint64_t* target,
                                  uint32_t k);
/* QCircuit::CTRL / CTRL_fan(U, ctrl, target, shift), qcircuit.hpp:1985-2322;
 * shift may be NULL. */
qgpu_status qgpu_circuit_ctrl(qgpu_circuit* c, const double* U, uint64_t DU,
                              const uint64_t* ctrl, uint32_t nc,
                              const uint64_t* target, uint32_t k,
                              const uint64_t* shift, int fan);
/* QCircuit::cCTRL / cCTRL_fan: controlled on classical dits ctrl_dits. */
qgpu_status qgpu_circuit_cctrl(qgpu_circuit* c, const double* U, uint64_t DU,
                               const uint64_t* ctrl_dits, uint32_t nc,
                               const uint64_t* target, uint32_t k,
                               const uint64_t* shift, int fan);
/* QCircuit::measure / measure_many in the Z basis (qcircuit.hpp:2983):
 * the first outcome goes to classical dit c_reg. */
qgpu_status qgpu_circuit_measure(qgpu_circuit* c, const uint64_t* target,
                                 uint32_t k, uint64_t c_reg, int destructive);
/* QCircuit::reset / reset_many: RESET steps; an engine applies qpp::reset
 * (instruments.hpp:1148-1206) on them with its own generator. */
qgpu_status qgpu_circuit_reset(qgpu_circuit* c, const uint64_t* target, uint32_t k);
/* QCircuit::cond_if / cond_end: the steps added between the two run only
 * when the classical dits (dits[0] the least significant bit) spell `value`
 * (a runtime IF, qengine.hpp:837-861; a false IF skips its block and its
 * END). Not nested. Circuits with conditionals run on engines only. */
qgpu_status qgpu_circuit_cond_if(qgpu_circuit* c, const uint64_t* dits, uint32_t n,
                                 uint64_t value);
qgpu_status qgpu_circuit_cond_end(qgpu_circuit* c);
/* QCircuit::QFT(target, swap) (inverse = 0, qcircuit.hpp:1514-1617) and
 * QCircuit::TFQ (inverse = 1, :1628-1732): appends qpp's gate sequence as
 * steps (H or Fd on target i followed by CTRL R_j from target i + j - 1,
 * then the SWAPs; the adjoint sequence in reverse for TFQ). target == NULL
 * takes every qudit not measured so far. Noiseless engines run the appended
 * block as one transform (qgpu_apply_qft); noisy engines step through it. */
qgpu_status qgpu_circuit_qft(qgpu_circuit* c, const uint64_t* target, uint32_t k, int swap,
                             int inverse);
/* OpenQASM 2.0 reader (replaces qpp::qasm::read_from_string /
 * read_from_file, qasm/qasm.hpp:781-820): registers in declaration order,
 * non-destructive measurements, resets, runtime conditionals for `if`, and
 * qelib1.inc's gates as single steps with qpp's matrices (u3/u2/u1 as U; the
 * gates qpp expands into several U/CX steps -- cu1, cu3, crx, cry, cswap,
 * rxx, rzz, sx, ... -- as one step with the same matrix). Parse errors are
 * QGPU_ERR_INVALID_ARGUMENT with "line L, column C: ..." in the message. */
qgpu_status qgpu_qasm_read(const char* source, qgpu_circuit** out);
qgpu_status qgpu_qasm_read_file(const char* path, qgpu_circuit** out);
/* A Kraus channel sum_i K_i . K_i^+ on `target` (nK consecutive DK x DK
 * operators). No QCircuit counterpart: density-matrix engines apply it
 * exactly (qpp::apply(rho, Ks, target, dims), operations.hpp:476-560); ket
 * engines draw one branch with probability ||K_i psi||^2 and renormalise. */
qgpu_status qgpu_circuit_channel(qgpu_circuit* c, const double* Ks,
                                 uint32_t nK, uint64_t DK,
                                 const uint64_t* target, uint32_t k);
qgpu_status qgpu_circuit_info(const qgpu_circuit* c, uint32_t* nq,
                              uint64_t* n_steps);
/* Qudits, their dimension and the classical dits of a circuit. */
qgpu_status qgpu_circuit_shape(const qgpu_circuit* c, uint32_t* nq, uint64_t* d, uint32_t* nc);
/* Number of state passes of the fused plan with blocks of <= max_k qubits
 * (host-side planning only). */
qgpu_status qgpu_circuit_fuse(qgpu_circuit* c, uint32_t max_k,
                              uint64_t* n_passes);

/* Execution forms of the unitary steps of a circuit on a resident state. */
typedef enum qgpu_form {
    QGPU_FORM_PLAIN = 0, /* one pass per qpp call, in the state precision */
    QGPU_FORM_FUSED = 1  /* fused blocks: c64 -> 6-qubit tcgen05 split-FP16 */
} qgpu_form;
/* Kets: the unitary steps (measurements and classical control need an
 * engine). QGPU_FORM_FUSED on a qubit ket merges gates into blocks: of <= 6
 * qubits in complex64 (on the tensor cores from 13 qubits); in complex128,
 * of <= 2 qubits run as tile passes up to 22 qubits and of <= 3 qubits as
 * dense passes above. QGPU_FORM_FUSED on a complex64 qubit density matrix of <= 15
 * qubits whose circuit holds only gates and 1- or 2-qubit channels:
 * superoperators on the 2n virtual qubits (column digits, row digits) merged
 * into blocks of <= 4 virtual qubits, one pass over the matrix per block
 * (a layer's gates and pair channel on one qubit pair become one 16 x 16
 * block); other density matrices return QGPU_ERR_NOT_SUPPORTED in that form.
 * No reference counterpart for the fused forms. */
qgpu_status qgpu_run_gates(qgpu_state* s, qgpu_circuit* c, int form);
/* One gate of k <= 6 qubits on a complex64 qubit ket of >= 13 qubits, as a
 * 64 x 64 block on the tensor cores (split-FP16, FP32 accumulation). */
qgpu_status qgpu_apply_tc(qgpu_state* s, const double* U,
                          const uint64_t* target, uint32_t k);

/* ---------------------------------------------------------------- engines
 * QEngine / QDensityEngine / QNoisyEngine over a qgpu_circuit
 * (include/qpp/classes/qengine.hpp:1271-1405, qnoisy_engine.hpp:105-139).
 * The state stays in HBM across gates, measurements and noise; kind
 * QGPU_KET runs a QEngine, QGPU_RHO a QDensityEngine. Randomness is one
 * std::mt19937 per engine drawn in qpp's order (one full-basis index per
 * measurement step, one Kraus index per non-measured qudit before every step
 * when noisy); every draw is recorded and can be replayed. */
typedef struct qgpu_engine qgpu_engine;
qgpu_status qgpu_engine_create(qgpu_ctx* ctx, qgpu_circuit* c, qgpu_kind kind,
                               qgpu_prec prec, qgpu_engine** out);
qgpu_status qgpu_engine_destroy(qgpu_engine* e);
qgpu_status qgpu_engine_set_seed(qgpu_engine* e, uint64_t seed);
/* QNoisyEngine noise model (noise.hpp:75-380): nK Kraus operators on one
 * qudit (d x d each, consecutive, column-major); probs != NULL gives a
 * state-independent model (e.g. QubitDepolarizingNoise {1-p, p/3, p/3,
 * p/3}), probs == NULL a state-dependent one (p_i = tr(K_i rho_q K_i^+)).
 * nK == 0 removes the noise. */
qgpu_status qgpu_engine_set_noise(qgpu_engine* e, const double* Ks,
                                  uint32_t nK, uint64_t d,
                                  const double* probs);
/* QEngineT::set_state (qengine.hpp:1191-1214): replaces the engine's
 * current state (a copy); its dimension must be d^(qudits not measured
 * destructively), else QGPU_ERR_DIMS_NOT_EQUAL; a density matrix for a ket
 * engine (or the reverse) is QGPU_ERR_TYPE_MISMATCH. */
qgpu_status qgpu_engine_set_state(qgpu_engine* e, const qgpu_state* s);
/* QEngineT::reset / QNoisyEngineT::reset (qengine.hpp:1251-1260): the state
 * back to |0...0>, dits / probabilities / measured qudits cleared; the
 * statistics too when reset_stats != 0. */
qgpu_status qgpu_engine_reset(qgpu_engine* e, int reset_stats);
/* Force the random choices: measurement outcome dits in execution order and
 * Kraus indices step by step, qudit by qudit (NULL, 0 to stop replaying). */
qgpu_status qgpu_engine_set_replay(qgpu_engine* e, const uint64_t* outcomes,
                                   uint64_t n_out, const uint64_t* noise,
                                   uint64_t n_noise);
/* QEngineT::execute(reps) (qengine.hpp:1341-1405). A noiseless engine
 * starts from its current state (which must be full size), clears the dits,
 * and for reps > 1 reorders the circuit as qpp's canonical_form (classical
 * controls, then measurements, pushed to the end past steps they commute
 * with); the steps before the first measurement run once, the rest reps
 * times from that point. When the rest holds only measurements, one run
 * gives the engine state and the other reps - 1 are full-basis samples of
 * the pre-measurement state (qengine.hpp:374-481), drawn in qpp's RNG order.
 * A noisy engine (qnoisy_engine.hpp:129-139) runs every step reps times from
 * its current engine state. Either way the engine keeps the FIRST
 * repetition's state, dits and probabilities, and the statistics accumulate
 * across calls until a reset. reps == 0: QGPU_ERR_OUT_OF_RANGE. */
qgpu_status qgpu_engine_execute(qgpu_engine* e, uint64_t reps);
qgpu_status qgpu_engine_get_dits(const qgpu_engine* e, uint64_t* dits,
                                 double* probs);
/* A new state handle holding a copy of the engine's current state. */
qgpu_status qgpu_engine_get_state(const qgpu_engine* e, qgpu_state** out);
/* Outcome statistics since the last reset (QEngineStatistics): the number of
 * distinct dit vectors, then their counts and the vectors (nc dits each). */
qgpu_status qgpu_engine_get_stats(const qgpu_engine* e, uint64_t* n_distinct,
                                  uint64_t* counts, uint64_t* outcomes);
/* The random choices of the last execute (sizes first, arrays when given). */
qgpu_status qgpu_engine_get_record(const qgpu_engine* e, uint64_t* n_out,
                                   uint64_t* outcomes, uint64_t* n_noise,
                                   uint64_t* noise);

/* ------------------------------------------------ trajectory batches
 * All `shots` stochastic trajectories of a QNoisyEngine request (qubit
 * circuit of at most 22 qubits; 1- and 2-qubit gates, fan gates, controlled
 * 1-qubit gates, Z measurements) in one launch, one CTA per trajectory with
 * the state in shared memory (up to 14 qubits) or in a global slot, worked
 * through in cache-blocked tile passes of the tuned width (15-22 qubits).
 * No reference counterpart (qpp runs one trajectory per execute). Noise:
 * before every step each non-measured
 * qubit draws from the depolarising channel {I, X, Y, Z} with probabilities
 * {1 - p, p/3, p/3, p/3} (qnoisy_engine.hpp:105-121, noise.hpp:388-412).
 * Outputs (any may be NULL): samples[shots] = the final full-basis sample of
 * each shot; dits[shots * max(nc, 1)] = measurement outcomes; dump[shots * 2
 * * 2^n] = final states (complex64 widened to double, for parity checks);
 * events[shots * max_events * 2] = noise events as (instruction, bit |
 * pauli << 16), unused slots 0xffffffff. Draws come from Philox4x32-10
 * keyed by seed with counter (shot, instruction, qubit). */
qgpu_status qgpu_trajectories(qgpu_ctx* ctx, qgpu_circuit* c, double p_depol,
                              uint64_t shots, uint64_t seed,
                              uint64_t* samples, uint32_t* dits, double* dump,
                              uint32_t* events, uint32_t max_events);
/* Tile width of the trajectory kernel for registers of n qubits (15-22) on
 * this context's device: set_T = -1 queries (timing the candidates
 * {untiled (below 17 qubits), 10, 11, 12, 13} once on first use), 0 pins the
 * untiled form, 9..14 (< n) pins that width, -2 drops the choice so it is
 * timed again. No reference counterpart. *chosen (if not NULL) receives the
 * width now in force. */
qgpu_status qgpu_traj_tile_width(qgpu_ctx* ctx, uint32_t n, int set_T, int* chosen);
/* Fusion width of batched (noiseless) registers of n qubits (1-22): the gates
 * of a batched instance merge into dense blocks of at most this many qubits
 * (2, 3 or 4; 8 x 8 and 16 x 16 blocks for 3 and 4). set_w = -1 queries
 * (timing the widths on a two-layer random-matching program with the tuned
 * tile width once on first use), 2..4 pins a width, -2 drops the choice so
 * it is timed again. No reference counterpart. *chosen (if not NULL)
 * receives the width now in force. */
qgpu_status qgpu_traj_fusion_width(qgpu_ctx* ctx, uint32_t n, int set_w, int* chosen);

/* ------------------------------------------------------ batched instances
 * n_inst independent instances, instance i running circuits[i] on
 * states[i] in place (kets or density matrices of uneven sizes). form
 * QGPU_FORM_FUSED (1): every complex64 instance of <= 22 (virtual) qubits is
 * compiled into a trajectory program (a density matrix as a ket over 2n
 * virtual qubits: 1-qubit gates and 1-qubit channels as 4 x 4
 * superoperators, 2-qubit gates as U on the rows then conj(U) on the
 * columns) and all of them run as ONE CUDA-graph launch holding one
 * trajectory-kernel launch per register size; instances it cannot compile
 * run in the plain form afterwards. form QGPU_FORM_PLAIN (0): a loop over
 * the instances, one kernel launch per gate. graph_kernels (may be NULL)
 * receives the number of kernels in the graph. No reference counterpart. */
qgpu_status qgpu_run_batch(qgpu_ctx* ctx, uint32_t n_inst,
                           qgpu_circuit* const* circuits,
                           qgpu_state* const* states, int form,
                           uint64_t* graph_kernels);
/* Where the last qgpu_run_batch on ctx spent its time, in milliseconds
 * (phases_ms holds 6 values): [0] compiling and tiling the programs on the
 * host, [1] uploading them and capturing + instantiating the graph, [2] the
 * graph on the device (CUDA events), [3] the instances run in the plain
 * form, [4] the argument checks, [5] releasing the graph after it ran. No
 * reference counterpart. */
qgpu_status qgpu_batch_last_phases(qgpu_ctx* ctx, double* phases_ms);

/* ------------------------------------------------------------ serving loop
 * QNoisyEngine requests on one GPU, submitted from any thread.
 * mode 0 (batched): kets of up to 20 qubits and density matrices of up to 7
 * run as trajectories; waiting requests are admitted in arrival order, a
 * slice of their shots at a time, into the next launch of their register
 * size while their estimated HBM footprint fits hbm_budget. Each register
 * size has its own stream with up to two launches in flight, so sizes run
 * side by side and a request finishes when its last shot lands. Requests the
 * trajectory kernel cannot run (larger density matrices, kets above 20
 * qubits, wider gates) run one at a time on each of two engine workers with
 * high-priority streams, density matrices of gates and channels in the fused
 * superoperator form. mode 1 (plain): one request at a time on the resident
 * engine in complex128, one launch per gate. Results do not depend on what
 * else is in flight. A request's circuit must stay alive until its wait
 * returns. */
typedef struct qgpu_server qgpu_server;
qgpu_status qgpu_server_create(int device, uint64_t hbm_budget, int mode,
                               qgpu_server** out);
/* kind QGPU_KET: `shots` trajectories with depolarising probability p per
 * qubit per step; kind QGPU_RHO: one exact density-matrix run (noise from
 * the circuit's channels), then `shots` samples of the final diagonal. */
qgpu_status qgpu_server_submit(qgpu_server* s, qgpu_circuit* c,
                               qgpu_kind kind, double p, uint64_t shots,
                               uint64_t seed, uint64_t* id);
/* Blocks until request `id` finished (timeout_s < 0: no limit); latency is
 * submit -> result on the host; samples[shots] and dits[shots * max(nc, 1)]
 * are copied when given. The request is released afterwards. */
qgpu_status qgpu_server_wait(qgpu_server* s, uint64_t id, double timeout_s,
                             double* latency_s, uint64_t* samples,
                             uint32_t* dits);
qgpu_status qgpu_server_stats(qgpu_server* s, uint64_t* batches,
                              uint64_t* trajectories, uint64_t* engine_runs,
                              double* busy_s);
qgpu_status qgpu_server_destroy(qgpu_server* s);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* QPP_B200_H_ */
