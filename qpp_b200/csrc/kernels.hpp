// kernels.hpp -- host-callable launchers of the sm_100a kernels.
//
// All launchers enqueue on the context stream and return immediately; they
// throw qgpu::Exc on a launch error. Matrices are c128 column-major; the
// launcher converts them to the state precision.
#pragma once

#include <complex>
#include <cstdint>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace qgpu {

using cd = std::complex<double>;

// Number of SMs and resident blocks of 256 threads used to size grids.
int grid_blocks(qgpu_ctx* ctx, int blocks_per_sm);

// --- gate application (kernels_gate.cu), all in place -------------------
// Qubit ket, one target at bit position `bit` (LSB = 0) of a 2^nbits state.
void launch_qubit_1q(qgpu_ctx* ctx, qgpu_prec prec, void* data, int nbits,
                     int bit, const cd* A);
// Qubit ket, two targets: A's row index is 2 * b(bit0) + b(bit1).
void launch_qubit_2q(qgpu_ctx* ctx, qgpu_prec prec, void* data, int nbits,
                     int bit0, int bit1, const cd* A);
// Generic: for every group g of `outer`, the DA amplitudes at
// base(g) + off[m] are replaced by A * (those amplitudes).
void launch_apply_generic(qgpu_ctx* ctx, qgpu_prec prec, void* data,
                          const SegPlan& outer,
                          const std::vector<uint64_t>& off, const cd* A,
                          uint64_t DA);

// Generic 16 x 16 that factors as A (x) B (both 4 x 4, column-major): the
// group's element (i, j) at base(g) + off[4 i + j] becomes
// sum A[i, i'] B[j, j'] x(i', j').
void launch_apply_kron4(qgpu_ctx* ctx, qgpu_prec prec, void* data, const SegPlan& outer,
                        const std::vector<uint64_t>& off, const cd* A, const cd* B);

// --- tile passes (kernels_tile.cu) -----------------------------------------
// One gate of a tile pass on a qubit ket: op 1 = 2 x 2 on tile bit t0, op 2 =
// 4 x 4 on tile bits (t0, t1) with row index 2 * b(t0) + b(t1); the matrix is
// row-major at mats + mat (state precision). It acts on the amplitudes i of
// the tile with (i & lmask) == lval, in tiles whose base offset b has
// (b & gmask) == gval (controls on bits outside the tile). k0 / k1: the
// positions of t0 / t1 in its sweep's bit list.
struct TileGate {
    uint32_t op;
    int32_t t0, t1;
    uint32_t lmask, lval;
    uint32_t mat;
    uint64_t gmask, gval;
    uint32_t k0, k1;
};
// A sweep: consecutive gates of a pass whose targets lie in nb <= 3 tile bits
// b[0..nb): every thread takes groups of 2^nb amplitudes (group element bit k
// <-> tile bit b[k]) from shared memory into registers, applies the sweep's
// gates in order there and writes the group back. Group numbers spell the
// other tile bits in ascending order.
struct TileSweep {
    uint32_t nb;
    int32_t b[3];
    uint32_t first, ngates;
};
// A pass: tiles of 2^T amplitudes, tile bits = state bits 0..L-1 and hi[0..T-L)
// (ascending); sweeps[first_sweep, first_sweep + nsweeps) in order; their
// gates' matrices are the mat_elems entries from mats + mat_first.
struct TilePassParams {
    uint64_t ntiles;
    int T, L;
    int hi[16];
    uint32_t first, ngates;
    uint32_t first_sweep, nsweeps;
    uint32_t mat_first, mat_elems;
};
size_t tile_pass_smem(qgpu_prec prec, const TilePassParams& p);
// Drops the cached device address of qgpu_ptrace_noalloc's offset table for
// `device` (kernels_subsys.cu); the next call looks it up again.
void noalloc_forget(int device);
void launch_tile_pass(qgpu_ctx* ctx, qgpu_prec prec, void* data, const TilePassParams& p,
                      const TileGate* gates, const TileSweep* sweeps, const void* mats);

// --- subsystem kernels (kernels_subsys.cu) --------------------------------
// out[o] = in[map(o)], o over map.count.
// Tiled bit permutation (see kernels_subsys.cu): when every output digit's
// dimension is a power of two, out[o] = in[foff + sum_j bit_j(o) *
// in_stride[j]]; tiles of 2^tb elements are staged in shared memory so that
// both the reads and the writes are coalesced.
struct PermPlan {
    uint64_t in_stride[64];  // input offset of output bit j
    uint64_t foff;
    int nb, tb, nrest;
    uint8_t tbits[16];   // tile bits, ascending (write order)
    uint8_t tin[16];     // the same bits by ascending input stride (read order)
    uint8_t tin_pos[16]; // position of tin[j] within tbits
    uint8_t rest[64];    // output bits outside the tile, ascending
    // shared-memory swizzle of tile positions, linear over GF(2): position p
    // is stored at the XOR of swz_bit[q] over p's set bits q. It is p with
    // some high bits folded into the bank-selecting low bits, chosen per plan
    // so that the warp's scattered stores (read order) and its row reads
    // (write order) both touch every bank group equally.
    uint16_t swz_bit[16];
};
constexpr int kPermTileBits = 10; // the smallest tile
// false when a dimension is not a power of two or there are <= tile_bits
// bits. The tile holds the out_low lowest output bits and then the bits of
// smallest input stride up to tile_bits (10-12); elem_bytes (8 or 16) sets
// how many low position bits select a bank group.
bool plan_permute(const std::vector<uint64_t>& out_dims, const std::vector<uint64_t>& src,
                  uint64_t fixed_off, PermPlan& P, int elem_bytes = 16,
                  int tile_bits = kPermTileBits, int out_low = 5);
// the tiled form of launch_gather(plan_gather(out_dims, src, fixed_off));
// false (nothing launched) when plan_permute does not apply
bool launch_permute_tiled(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                          const std::vector<uint64_t>& out_dims,
                          const std::vector<uint64_t>& src, uint64_t fixed_off);
void launch_gather(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                   const SegPlan& map);
// out[o] = in[mapA(o)] * conj(in[mapB(o)]) (ket -> density-matrix forms).
void launch_gather_outer(qgpu_ctx* ctx, qgpu_prec prec, const void* in,
                         void* out, const SegPlan& mapA, const SegPlan& mapB);
// Partial trace: out[o] = sum_a in[mapA(o) + toff[a]] (rho), or
// sum_a in[mapA(o) + toff[a]] * conj(in[mapB(o) + toff[a]]) (ket, is_ket).
void launch_ptrace(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                   const SegPlan& mapA, const SegPlan& mapB,
                   const std::vector<uint64_t>& toff, bool is_ket);

// --- quantum Fourier transform passes (kernels_qft.cu) --------------------
// One pass applies the QFT (or TFQ) steps of targets [a, a + M) of a k-target
// transform to every tile. The tile index is mixed radix over the tile
// digits in tile order: first the nr run digits (the lowest other digits in
// memory, Rsize values together), then the group digits with step M - 1
// lowest and step 0 highest, so that a step's phase index is a plain shift
// and mask of the tile index. The run digits that are later targets (nz of
// them, CZ values) come first: the per-tile step constants are tabulated over
// their values. Loads and stores walk the tile in memory order
// (rperm / wperm: tile digits by ascending read / write stride, with pitches
// rpitch / wpitch in that order). Outer digits enumerate the tiles (tile
// number = sum digit * opitch); ozw / tzw are a digit's weight in the integer
// spelled by the targets after the group (0 for other digits).
constexpr int kQftMaxTile = 16;
constexpr int kQftMaxOuter = 64;
constexpr int kQftMaxD = 16;
struct QftPlan {
    uint64_t ntiles;
    uint64_t dpow[65]; // d^e for e <= k
    uint64_t odim[kQftMaxOuter], opitch[kQftMaxOuter];
    uint64_t ors[kQftMaxOuter], ows[kQftMaxOuter], ozw[kQftMaxOuter];
    uint64_t trs[kQftMaxTile], tws[kQftMaxTile], tzw[kQftMaxTile];
    uint32_t tdim[kQftMaxTile], tpitch[kQftMaxTile];
    int rperm[kQftMaxTile], wperm[kQftMaxTile];
    uint32_t rpitch[kQftMaxTile], wpitch[kQftMaxTile];
    uint8_t oshift[kQftMaxOuter];
    uint32_t E, Rsize, CZ, Glo, Flo, wmul, nW;
    int ntd, nr, nz, nod, M, a, k, d, sigma, inverse, pow2, glo_shift, flo_shift;
    double scale; // qubit passes: 2^(-M/2)
    // complex64 8- and 6-step passes (k_qft_pass8): the tile bits that a
    // base index's bits select in round A (the tile bits outside that
    // round's, by ascending read stride) and in round B (by ascending write
    // stride); set by the launcher
    uint8_t q8a[12], q8b[12];
};
size_t qft_smem_bytes(const QftPlan& p, size_t elem_bytes);
// The passes of one transform (qft.cpp): fold[i] = pass i reads the state
// buffer and writes a second one with the targets reversed (fold = true
// asks for that on the last pass of a forward transform, the first of an
// inverse one). false when the kernel does not apply (d > kQftMaxD, or a
// pass outside its table limits).
struct QftSchedule {
    std::vector<QftPlan> plans;
    std::vector<char> fold;
    int Mmax = 0;
    uint64_t nW = 0; // d^Mmax
};
bool plan_qft(bool rho, uint64_t D, uint64_t d, size_t elem_bytes,
              const std::vector<uint64_t>& target, bool inverse, bool fold, QftSchedule& S);
// exp(2 pi i e / nW), e < nW
std::vector<std::complex<double>> qft_roots(uint64_t nW);
// W: exp(2 pi i e / nW), e < nW = d^Mmax (state precision; p.wmul = d^(Mmax-M));
// F: the d x d Fourier matrix of the pass, column-major (qudits only).
void launch_qft_pass(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                     const QftPlan& p, const void* W, const void* F);
// The register-round qubit passes (k_qft_pass8, which launch_qft_pass takes
// when they apply): log2 of their tile (12 complex64, 11 complex128); whether
// a plan is one of theirs (8 or 6 steps over a whole tile; in place, or
// into another buffer); and the thread-to-base maps the launcher sets
// (q8a, q8b) for a tile of 2^EB amplitudes.
int qft_pass8_tile_bits(qgpu_prec prec);
bool qft_pass8_applies(qgpu_prec prec, const void* in, const void* out, const QftPlan& p);
void qft_pass8_maps(QftPlan& p, int EB);

// --- reductions and elementwise (kernels_reduce.cu) ----------------------
// sum |x|^2 over n elements, FP64 accumulation; result to *host_out.
double reduce_norm2(qgpu_ctx* ctx, qgpu_prec prec, const void* data,
                    uint64_t n);
// The same sum left on the device at dev_out (stream order, no host wait).
void reduce_norm2_device(qgpu_ctx* ctx, qgpu_prec prec, const void* data, uint64_t n,
                         double* dev_out);
// sum_i x[i * stride] (complex, FP64 accumulation): the trace for stride D+1.
cd reduce_strided_sum(qgpu_ctx* ctx, qgpu_prec prec, const void* data,
                      uint64_t n, uint64_t stride);
// sum conj(a[i]) b[i], FP64 accumulation.
cd reduce_inner(qgpu_ctx* ctx, qgpu_prec prec, const void* a, const void* b,
                uint64_t n);
// x[i] *= s
void launch_scale(qgpu_ctx* ctx, qgpu_prec prec, void* data, uint64_t n,
                  cd s);
// Marginal probabilities over the target digits of a ket (|x|^2) or of the
// diagonal of a density matrix: p[m] = sum_g w(base(g) + off[m]), FP64.
std::vector<double> reduce_marginals(qgpu_ctx* ctx, qgpu_prec prec,
                                     const void* data, const SegPlan& outer,
                                     const std::vector<uint64_t>& off,
                                     bool diag_of_rho, uint64_t D);
// Index of the first element whose inclusive prefix sum of weights reaches
// fraction * (sum of all weights) (FP64); weights are |x_i|^2 (ket) or
// Re rho(i, i). This is std::discrete_distribution's draw for a uniform u
// = fraction.
uint64_t prefix_search(qgpu_ctx* ctx, qgpu_prec prec, const void* data,
                       uint64_t D, bool diag_of_rho, double fraction,
                       double* total_out);
// The same search for many fractions at once: one pass over the weights
// (sums of 4096-weight chunks, prefix on the host), then one block per draw
// scans its chunk.
std::vector<uint64_t> prefix_search_many(qgpu_ctx* ctx, qgpu_prec prec, const void* data,
                                         uint64_t D, bool diag_of_rho,
                                         const std::vector<double>& fractions);
// Keep the elements whose digit (index / dig_stride) % dig_dim equals
// dig_val (for rho: in both the row and the column index), scale them by
// `scale`, zero the rest.
void launch_project(qgpu_ctx* ctx, qgpu_prec prec, void* data, uint64_t n,
                    uint64_t D, bool is_rho, uint64_t dig_stride,
                    uint64_t dig_dim, uint64_t dig_val, double scale);
// Philox4x32-10 counter-based normal samples: x = (N(0,1), N(0,1)).
void launch_fill_gaussian(qgpu_ctx* ctx, qgpu_prec prec, void* data,
                          uint64_t n, uint64_t seed);
// c128 <-> c64 conversion on the device.
void launch_convert(qgpu_ctx* ctx, const void* in, qgpu_prec in_prec,
                    void* out, qgpu_prec out_prec, uint64_t n);

} // namespace qgpu
