// tile_gates.hpp -- planning and execution of gate runs as tile passes
// (tile_gates.cpp, kernels_tile.cu).
#pragma once

#include <complex>
#include <utility>
#include <vector>

#include "internal.hpp"
#include "kernels.hpp"

namespace qgpu {

struct Step;

// One 1- or 2-qubit gate of a qubit ket: state bits b0 (and b1 for op 2; the
// matrix's row index is 2 * b(b0) + b(b1)), controls as (state bit, value),
// the matrix column-major.
struct GateDesc {
    int op = 1;
    int b0 = 0, b1 = 0;
    std::vector<std::pair<int, int>> ctrl;
    cd A[16];
};

// Appends the gates of step `st` on an nbits-qubit ket and returns true, or
// returns false (appending nothing) when the step is not a 1- or 2-qubit
// unitary, fan or controlled gate.
bool gate_desc_of(const Step& st, int nbits, std::vector<GateDesc>& out);
// Splits `gates` (in order) into tile passes of at most Tmax tile bits: the
// low min(nbits, 5) state bits and the targets above them; each pass into
// sweeps of consecutive gates on at most three tile bits. `dev` gets one
// entry per gate with tile-local bits, `sweeps` the sweeps, `mats` the
// row-major matrices.
void plan_gate_tiles(const std::vector<GateDesc>& gates, int nbits, int Tmax,
                     std::vector<TilePassParams>& passes, std::vector<TileGate>& dev,
                     std::vector<TileSweep>& sweeps, std::vector<cd>& mats);
// The gates reordered for fewer tile passes and sweeps (list scheduling):
// every gate still follows the earlier gates it shares a bit with (target or
// control), so the product is the same up to rounding, but each pass takes
// every ready gate whose targets fit the tile, those that extend the current
// sweep first. For forms that do not promise the gate-by-gate arithmetic.
std::vector<GateDesc> schedule_gates(const std::vector<GateDesc>& gates, int nbits, int Tmax);
// Largest tile (bits) for this context and precision: 13 for complex128 and
// 14 for complex64 (128 KB of shared memory), or qgpu_ctx_set_tile_bits's.
int tile_bits_max(const qgpu_ctx* ctx, qgpu_prec prec);
// A run of gates planned as tile passes on an nbits-qubit ket (host side;
// uploaded by run_tile_program each time it runs).
struct TileProgram {
    int nbits = 0, Tmax = 0;
    std::vector<GateDesc> gates; // in pass order
    std::vector<TilePassParams> passes;
    std::vector<TileGate> dev;
    std::vector<TileSweep> sweeps;
    std::vector<cd> mats;
};
void plan_tile_program(const std::vector<GateDesc>& gates, int nbits, int Tmax, TileProgram& P);
// Uploads P's tables and launches its passes on s (stream order).
void run_tile_program(qgpu_state* s, const TileProgram& P);
// Runs `gates` on the qubit ket s as planned tile passes (stream order).
void run_tiled_gates(qgpu_state* s, const std::vector<GateDesc>& gates);

// The fused complex128 tile form of a circuit, planned once: list-scheduled
// tile programs and the unfused steps between them, for the circuit's first
// nsteps steps and tiles of at most Tmax bits.
struct FusedTiles {
    uint64_t nsteps = 0;
    int Tmax = 0;
    std::vector<std::pair<int64_t, TileProgram>> runs; // first >= 0: that step as it is
};

// A piece of a fused complex128 ket plan: a run of gate descriptors for the
// tile passes (step < 0; possibly empty), or one step run as it is.
struct TiledRun {
    std::vector<GateDesc> gates;
    int64_t step = -1;
};
// The circuit's fused plan (blocks of <= 2 qubits, c->plan) and its unfused
// steps, in circuit order, as tile-pass runs and steps.
void tiled_runs(const qgpu_circuit* c, std::vector<TiledRun>& out);

} // namespace qgpu
