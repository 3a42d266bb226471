// circuit.hpp -- circuit description, gate fusion and execution forms.
//
// A qgpu_circuit mirrors the steps of qpp::QCircuit that the engines execute
// (include/qpp/classes/qcircuit.hpp: gate :1166-1444, CTRL :1985-2322,
// measure :2983; step kinds internal/classes/qcircuit_gate_step.hpp and
// qcircuit_measurement_step.hpp). Gate matrices are stored once per step on
// the host and uploaded on use.
//
// Fusion (no reference counterpart): consecutive unitary steps on qubit
// circuits are merged greedily into dense blocks of at most k qubits. Open
// blocks act on disjoint qubits, so they commute; a gate joins (and merges)
// the open blocks it touches while the union stays within k qubits,
// otherwise those blocks are emitted first. Non-unitary steps flush every
// open block.
#pragma once

#include <complex>
#include <cstdint>
#include <memory>
#include <vector>

#include "internal.hpp"

namespace qgpu {

using cd = std::complex<double>;
struct TProgram;
struct FusedTiles;

enum class StepKind {
    Gate,      // apply(U, target)           GType SINGLE/TWO/THREE/JOINT
    Fan,       // apply(U, {t}) for each t   GType FAN
    Ctrl,      // applyCTRL                  GType CTRL
    CtrlFan,   // applyCTRL_fan              GType CTRL_FAN
    CCtrl,     // classically controlled     GType cCTRL
    CCtrlFan,  // classically controlled fan GType cCTRL_FAN
    Measure,   // Z-basis measure_seq        MType MEASURE / MEASURE_MANY (+ _ND)
    Reset,     // reset targets to |0>
    Channel,   // Kraus channel sum_i K_i . K_i^+ on the targets (no QCircuit step:
               // exact on density matrices, one sampled branch on kets)
    CondIf,    // runtime IF (qengine.hpp:837-861): ctrl = the dits (LSB first),
               // c_reg = the value they must spell; nK = the steps to skip when
               // false (the block and its CondEnd)
    CondEnd,   // runtime ENDIF
    Nop
};

struct Step {
    StepKind kind = StepKind::Nop;
    std::vector<cd> U; // Channel: nK consecutive DU x DU Kraus operators
    uint64_t DU = 0;
    uint32_t nK = 0;
    std::vector<uint64_t> target, ctrl, shift;
    bool has_shift = false;
    uint64_t c_reg = 0;
    bool destructive = true;
    // first step of a QCircuit::QFT / TFQ block: the block's step count, its
    // targets and flags, so that noiseless engines can run the block as one
    // transform (the steps themselves are qpp's gate sequence)
    uint32_t block_len = 0;
    bool block_inverse = false, block_swap = false;
    std::vector<uint64_t> block_target;
};

struct Block {
    std::vector<int> qubits; // big-endian order of the block index
    std::vector<cd> U;       // 2^k x 2^k, column-major
    int step = -1;           // >= 0: not fused, run step `step` as is
};

} // namespace qgpu

struct qgpu_circuit {
    uint32_t nq = 0;
    uint64_t d = 2;
    uint32_t nc = 0; // classical dits
    std::vector<qgpu::Step> steps;
    // fused plan cache
    uint32_t plan_k = 0;
    std::vector<qgpu::Block> plan;
    // device images of the tensor-core block matrices (65536 bytes each:
    // fp16 hi and lo halves in the kernel's shared-memory layout)
    qgpu_ctx* plan_ctx = nullptr;
    unsigned char* dB = nullptr;
    int dB_dev = -1; // the device holding dB
    std::vector<int64_t> block_slot; // plan index -> image slot in dB, or -1
    // fused density-matrix program (superoperator blocks), built for the
    // first rho_steps steps (steps are only ever appended)
    uint64_t rho_steps = ~uint64_t(0);
    std::shared_ptr<qgpu::TProgram> rho_prog; // null: the form does not apply
    // fused complex128 ket form as tile passes (blocks of <= 2 qubits),
    // planned for the first ftiles->nsteps steps
    std::shared_ptr<qgpu::FusedTiles> ftiles;
    // fused density-matrix form on the tensor cores (complex64, 2n >= 13
    // virtual qubits): superoperator blocks of <= 6 virtual qubits, built for
    // the first rho_tc_steps steps
    uint64_t rho_tc_steps = ~uint64_t(0);
    bool rho_tc_ok = false;
    std::vector<qgpu::Block> rho_plan;
    unsigned char* rho_dB = nullptr;
    int rho_dB_dev = -1; // the device holding rho_dB
    std::vector<int64_t> rho_slot;
    ~qgpu_circuit();
};

namespace qgpu {

// Dense matrix of the step on its qubits (ctrl + target order), for steps
// that can be fused; false if the step is not unitary or too wide.
bool step_dense(const Step& s, uint32_t max_k, std::vector<int>& qubits,
                std::vector<cd>& U);
std::vector<cd> embed(const std::vector<cd>& G, const std::vector<int>& gq,
                      const std::vector<int>& bq);
std::vector<Block> fuse(const std::vector<Step>& steps, uint32_t nq,
                        uint32_t max_k);

// Runs the unitary steps [first, first + count) of `c` on `s`:
// form 0 = plain (one pass per qpp call), form 1 = fused blocks.
void run_gates(qgpu_state* s, qgpu_circuit* c, int form, uint64_t first,
               uint64_t count);
// The fused form of a whole circuit in two parts, so that the launches can be
// captured into a CUDA graph: fused_prepare does the host planning and the
// one-time uploads (synchronous; raises QGPU_ERR_NOT_SUPPORTED where
// run_gates' fused form would), fused_launch only enqueues kernels on
// s->ctx->stream; the caller checks fused_error(ctx) once they have run.
void fused_prepare(qgpu_state* s, qgpu_circuit* c);
// The superoperator program of a complex64 density-matrix circuit (blocks of
// <= 4 virtual qubits, c->rho_prog), as the batched block-layered launches
// use it; raises QGPU_ERR_NOT_SUPPORTED when the circuit does not compile.
void rho_program_prepare(qgpu_state* s, qgpu_circuit* c);
void fused_launch(qgpu_state* s, qgpu_circuit* c);
// One pass per instruction of a program of dense blocks (G1-G4 only) on a
// complex64 qubit state: bit b of the program is qubit n - 1 - b of a ket,
// or virtual qubit 2n - 1 - b (column digits, then row digits) of a density
// matrix. Launches only.
void launch_program(qgpu_state* s, const TProgram& P);
void apply_step(qgpu_state* s, const Step& st);

} // namespace qgpu
