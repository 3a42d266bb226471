// traj.hpp -- compiled trajectory programs for the shared-memory kernel.
#pragma once

#include <complex>
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "internal.hpp"

namespace qgpu {

// kTG3: 8 x 8 on three bits (b0, b1, cmask & 255), row index 4 b0 + 2 b1 + b2
// kTG4: 16 x 16 on four bits (b0, b1, cmask & 255, cmask >> 8 & 255)
// kTTile: tile-pass header: the next `cmask` instructions act on the b0 = T
// bits listed (one 32-bit word each, ascending, bits 0..4 first) at float2
// offset `mat` of the matrix pool, with their bit positions renumbered
// within that list
enum : uint8_t { kTG1 = 1, kTG2 = 2, kTCG1 = 3, kTMeas = 4, kTG4 = 5, kTTile = 6, kTG3 = 7 };
enum : uint8_t { kTNewStep = 1, kTDestructive = 2 };

// One instruction; qubits are bit positions (LSB = 0) of the full register.
struct TInstr {
    uint8_t op;
    uint8_t b0, b1; // targets (G2: row index = 2 * bit(b0) + bit(b1))
    uint8_t flags;  // kTNewStep: noise is drawn before this instruction
    uint32_t mat;   // gate: float2 offset of the column-major matrix; meas: c_reg
    uint32_t cmask; // controlled gate: control bits
    uint32_t cval;  // controlled gate: required values of the control bits
};

// One trajectory (shot) of one request.
struct TWork {
    const TInstr* prog;
    const float2* mats;
    uint32_t nins;
    uint8_t n;
    uint8_t inplace; // 1: run directly in `fin` (== init, HBM), no copies
    uint16_t pad1;
    float p_noise;  // depolarising probability per qubit per step
    uint32_t shot;  // trajectory index inside its request (Philox counter)
    uint32_t out;   // global output slot
    uint64_t seed;  // request seed (Philox key)
    const float2* init; // initial register (null: |0...0>)
    float2* fin;        // where the final register goes (null: nowhere)
    double* diag;       // density-matrix run: Re rho(i, i) of the final state
                        // (2^(n/2) values; no basis sample is drawn)
};

// Recorded noise event: before instruction `ins`, Pauli `pauli` (1 X, 2 Y,
// 3 Z) on bit `bit`.
struct TEvent {
    uint32_t ins;
    uint16_t bit;
    uint16_t pauli;
};

// Largest register held in shared memory (2^14 complex64 = 128 KB); up to
// kTrajMaxGlobalQubits a CTA works on its own slot of a global scratch
// buffer instead (traj_global_grid(ctx, nwork) slots of 2^n amplitudes).
constexpr int kTrajMaxQubits = 14;
constexpr int kTrajMaxGlobalQubits = 22;
// Largest ket the serving loop sends to the global-slot lane.
constexpr int kServeMaxSlotQubits = 20;
// CTAs (= scratch slots) for a launch of nwork trajectories of n qubits:
// at most 8 per SM and at most 4 GiB of slots.
int traj_global_grid(qgpu_ctx* ctx, int nwork, int n);
// Resident CTAs of a launch of shared-memory trajectories of n <=
// kTrajMaxQubits qubits: one wave of the device.
int traj_resident_slots(qgpu_ctx* ctx, int n);
// Raises the kernel's shared-memory limit once (outside any stream capture).
void traj_prepare();

struct TProgram {
    uint32_t n = 0;
    uint32_t ncreg = 0;
    std::vector<TInstr> ins;
    std::vector<float> mats; // interleaved complex64
};

// Appends complex64 copies of gate matrices to a program's pool, each
// distinct matrix once (a layered circuit drawn from a gate bank stores the
// bank, not one copy per gate); returns the float2 offset, always even (the
// matrix starts on a 16-byte boundary of the pool).
struct MatPool {
    explicit MatPool(TProgram& p) : P(p) {}
    uint32_t add(const std::vector<std::complex<double>>& U);
    TProgram& P;
    std::unordered_map<std::string, uint32_t> seen;
};

// Registers above kTrajMaxQubits run either in a slot of `gscratch` or, when
// every work item of the launch has `inplace` set (gscratch null), directly
// in the item's own state. `stream` null: the context's stream.
// `tile_bits`: the largest T of the tile passes in the launch's programs
// (0: none); such a launch reserves a 2^T-amplitude shared-memory tile.
void launch_traj(qgpu_ctx* ctx, const TWork* dwork, int nwork, int nmax, uint32_t* ddits,
                 int maxcreg, uint64_t* dsamples, float2* ddump, TEvent* devents,
                 int max_events, float2* gscratch, cudaStream_t stream = nullptr,
                 int tile_bits = 0);
// Cache blocking for registers above 2^14 amplitudes (no reference
// counterpart): runs of consecutive gate instructions whose bits outside
// 0..4 number at most T - 5 become one tile pass (kTTile) of 2^T-amplitude
// tiles, so the register is read and written once per run instead of once
// per gate. Noise and measurement draws keep their untiled instruction
// counters, so a tiled program gives bit-identical results.
// Noiseless programs only (folding moves gates across step boundaries, where
// noise would be drawn): every 1-qubit gate is folded into the next gate on
// its qubit when that gate is a 1- or 2-qubit gate (it commutes past the
// gates in between, which act on other qubits); products in FP64, rounded
// to complex64 once. No reference counterpart.
void fold_1q_gates(TProgram& P);
// Noiseless programs only: consecutive dense gates (G1-G4) merge greedily into
// dense blocks of at most w bits (open blocks act on disjoint bits, so they
// commute; a gate joins the blocks it touches while their union stays within
// w bits, otherwise those blocks are emitted first), emitted as G1-G4.
// Products in FP64, rounded to complex64 once. Fusion width w = 2 holds 1- and
// 2-qubit gates; wider blocks trade arithmetic for register passes.
constexpr int kFuseMaxWidth = 4;
void fuse_blocks(TProgram& P, int w);
// The fusion width (2..kFuseMaxWidth) for batched registers of n qubits on
// this device, chosen once per (device, n) by timing the calibration program
// (two layers on random matchings) fused at each width with the tuned tile
// width; call outside stream capture.
int fusion_width(qgpu_ctx* ctx, int n);
void set_fusion_width(qgpu_ctx* ctx, int n, int w);
// min_run: the shortest run that becomes a pass (2 by default; 1 turns
// every gate into a pass, as the layer-synchronous batches need).
void plan_tiles(TProgram& P, int T, size_t min_run = 2);

// One register's tile pass in a layer-synchronous launch: items
// [first_item, first_item + ceil(2^(n-T) / tiles_per_item)) of the launch
// run tiles_per_item tiles each; `ins` = the pass's nins gate instructions
// (bits renumbered within the tile), tile bits at float2 offset tb_off of
// `mats` (one 32-bit word each).
struct PassInst {
    float2* psi;
    const float2* mats;
    const TInstr* ins;
    uint32_t nins;
    uint32_t tb_off;
    uint32_t first_item;
    uint32_t tiles_per_item;
    uint8_t n, T;
    uint16_t pad;
};
// One launch of k_pass_batch over `ninst` registers (sorted by first_item,
// nitems items in total) with two 2^tile_bits-amplitude tile buffers
// (tile_bits >= every T, <= 13). Every register must start on a 16-byte
// boundary. A bounded wait that gives up sets *err (the context's device
// error word).
void launch_pass_batch(qgpu_ctx* ctx, const PassInst* dinsts, int ninst, uint32_t nitems,
                       int tile_bits, int* err, cudaStream_t stream);
// One dense block of one register in a block-layered launch (no reference
// counterpart): every group of 2^k amplitudes of the 2^n-amplitude register
// at psi that differ only in bits b[0..k-1] (b[0] the most significant digit
// of the block's index, 1 <= k <= 4) is replaced by m times it (column-major
// 2^k x 2^k complex64, 16-byte aligned). Items [first_item, first_item +
// ceil(2^(n-k) / 512)) of the launch are this block's, 512 groups each.
struct BlockInst {
    float2* psi;
    const float2* m;
    uint32_t first_item;
    uint8_t n, k;
    uint8_t b[4];
    uint8_t pad[6];
};
// One launch over `ninst` blocks of distinct registers (sorted by
// first_item, nitems items in total); one thread per group, in place.
void launch_block_batch(qgpu_ctx* ctx, const BlockInst* dinsts, int ninst, uint32_t nitems,
                        cudaStream_t stream);
// The context's device error word (allocated on first use: call outside
// stream capture), and whether a kernel set it (reading clears it).
int* ctx_error_flag(qgpu_ctx* ctx);
int fused_error(qgpu_ctx* ctx);
// The fused tensor-core pass (kernels_fused.cu): one 64 x 64 complex block on
// six bits `tbits` (block index big-endian over them) of a complex64 ket of
// 2^nbits amplitudes, in place; img is the block's 64 KB shared-memory image
// (fused6_images) and norm2 a device word holding |psi|^2, written by
// fused_norm_prepare earlier on the same stream.
void launch_fused6_tc(qgpu_ctx* ctx, void* data, int nbits, const int* tbits,
                      const void* img, const double* norm2);
// Images of nblocks consecutive 128 x 128 fp32 block matrices (fused6_matrix
// layout) at dB into dimg (65536 bytes each), on the context stream.
void fused6_images(qgpu_ctx* ctx, const float* dB, void* dimg, int nblocks);
const double* fused_norm_prepare(qgpu_ctx* ctx, const void* data, uint64_t n);
// The tile width T (0: untiled) for registers of n qubits on this device,
// chosen once per (device, n) by timing calibration programs for T in
// {untiled (below 17 qubits), 10, 11, 12, 13} on a two-layer program;
// call outside stream capture.
int tile_width(qgpu_ctx* ctx, int n);
// Pin the width for (device, n) (T >= 0), or drop the choice (T < 0) so the
// next tile_width() times it again.
void set_tile_width(qgpu_ctx* ctx, int n, int T);
bool compile_traj(const qgpu_circuit* c, TProgram& P);
// A density-matrix run of `c` as a ket over 2n virtual qubits [column
// digits, row digits]: 1-qubit gates and 1-qubit channels become 4 x 4
// superoperators on (column t, row t); 2-qubit gates become U on the row
// digits and conj(U) on the column digits. False for anything else, and
// above max_nv virtual qubits (at most 31: instruction bit masks are 32-bit).
bool compile_traj_rho(const qgpu_circuit* c, TProgram& P, int max_nv = kTrajMaxGlobalQubits);

} // namespace qgpu
