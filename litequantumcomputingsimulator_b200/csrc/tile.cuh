// tile.cuh — operation records of the shared-memory tile passes (tile_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace lqcs_b200 {

constexpr uint32_t kTileThreads = 256;
constexpr uint32_t kTileMinBits = 8;             // a tile holds at least one amplitude per thread
constexpr uint32_t kTileMaxBits = 13;            // 2^13 amplitudes = 128 KiB of shared memory
constexpr uint32_t kTileMaxHigh = 8;             // at most 8 high qubits per tile
constexpr uint32_t kTileMaxK = 4;                // widest dense operation inside a tile
constexpr uint32_t kTileMaxOps = 128;            // operations per pass (staged in shared memory)
constexpr uint32_t kTileMaxIters = 32;           // 2^kTileMaxBits / kTileThreads
constexpr size_t kTileMaxSmem = 200 * 1024;      // tile + staged operation records

// kTilePauli: a Pauli rotation exp(-i theta/2 P) inside a register pass (planner only; the
// shared-memory kernel has no such operation).
enum : uint8_t { kTileDense = 0, kTileDiag = 1, kTilePhase = 2, kTilePauli = 3 };

// Shared-memory slot of tile element i: the low 3 bits are XOR-ed with a fold of the
// higher bits so that power-of-two strides spread over the 8 16-byte positions of a
// 128-byte wavefront.  The map is linear over GF(2): sw(a ^ b) == sw(a) ^ sw(b).
__host__ __device__ __forceinline__ uint32_t tile_swizzle(uint32_t i) {
    return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9) ^ (i >> 12)) & 7u);
}

// One operation on a tile, in tile-local bit positions (local bit j < L is qubit j, local
// bit L + i is the i-th high qubit of the tile).  Groups (of 2^k amplitudes, or single
// amplitudes of a phase) are numbered g = t + kTileThreads * j for thread t; because both
// the zero-insertion that spreads g over the free bit positions and the swizzle are linear
// over GF(2), the slot of member l of group g is
//     sw(deposit(t)) ^ dhi[j] ^ soff[l],
// with sw(deposit(t)) computed once per thread and operation and dhi, soff precomputed.
struct TileOp {
    uint64_t gcmask;      // qubits outside the tile that must all be 1 (controls / phase bits)
    uint32_t mat_off;     // matrix (dense), diagonal (diag) or phase factor (phase), in double2
    uint16_t n_groups;    // groups (dense, diag) or amplitudes (phase) to visit
    uint16_t iters;       // ceil(n_groups / kTileThreads)
    uint16_t soff[16];    // sw(local offset of member l), matrix local order
    uint16_t dhi[kTileMaxIters];   // sw(deposit(j * kTileThreads) | local control bits)
    uint8_t kind;
    uint8_t k;
    uint8_t n_fixed;      // positions inserted as zeros when spreading a group index
    uint8_t pad;
    uint8_t fixed[8];     // those positions, ascending
};

struct TilePass {
    uint64_t n_tiles;
    uint64_t batch_stride;
    uint32_t m;           // tile bits
    uint32_t L;           // low qubits 0..L-1 always in the tile
    uint32_t h;           // number of high tile qubits (m - L)
    uint32_t n_ops;
    uint32_t kmax;        // widest dense/diagonal operation of the pass
    uint32_t hbits[kTileMaxHigh];   // ascending
};

static_assert(sizeof(TileOp) % 4 == 0, "TileOp is copied to shared memory as 32-bit words");

void launch_tile_pass(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                      const TilePass& pass, const TileOp* d_ops, const double2* d_mats);
size_t tile_smem_bytes(const TilePass& pass);
void cuda_check_launch_attr(cudaError_t e);

// ------------------------------------------------------------------ register tile passes
//
// The same passes with the tile held in registers: each of the 2^(m-4) threads of a CTA
// owns 16 amplitudes.  A layout assigns 4 tile bits to the register index (amplitude u of
// a thread has bit i of u at tile bit rpos[i]) and the other m-4 tile bits to the thread
// index.  Dense operations whose targets are register bits run without shared memory;
// diagonal and phase operations run in any layout; a remap operation moves the tile to the
// next layout through shared memory.  Every remap, tile load and tile store is one pass of
// the tile through shared memory or HBM, so a pass costs (remaps + 2) tile transfers
// instead of (operations + 2).
constexpr uint32_t kRegBits = 4;                // amplitudes per thread: 16
constexpr uint32_t kRegMinBits = 9;             // a tile spans at least one warp
constexpr uint32_t kRegMaxBits = 13;
constexpr uint32_t kRegMaxK = 3;                // widest dense operation
constexpr uint32_t kRegMaxRecords = 256;        // operations + remaps per pass
constexpr uint32_t kRegMaxLayouts = 128;
constexpr uint32_t kRegMaxMatrix = 2048;        // double2 of matrices staged per pass (32 KiB)
constexpr uint32_t kRegMaxSelect = 2;           // out-of-tile selector qubits per operation
constexpr uint32_t kRegMaxDiag = 6;             // widest diagonal operation (64 entries)
constexpr uint32_t kRegMaxDyn = 8;              // per-tile diagonals per pass
constexpr uint32_t kRegMaxDynEntries = 512;     // their table entries per pass
constexpr uint32_t kRegMaxDynTerms = 48;        // gated phase terms of one per-tile diagonal
constexpr uint32_t kRegPauliMaxFlips = 9;       // X/Y qubits of a Pauli rotation in a pass:
                                                // register bits and lanes

// kRegDiagDyn: a diagonal whose table is built at the start of every tile from a base table
// and gated phase terms (the matrices hold the 2^k base entries, then per term its factor and
// a word pair {out-of-tile mask, entry mask}); it is applied like kRegDiag.
// kRegMma: a two-qubit dense block whose targets are the tile bits on lanes 0 and 1 (matrix
// bit 0 on lane 0), applied with mma.sync.m8n8k4.f64 by the whole warp: over the reals the
// 4 x 4 complex block is an 8 x 8 real matrix, each register index u of the warp's 32 lanes
// a set of 8 groups (lanes 2..4) of 4 amplitudes (lanes 0..1), and two k = 4 steps (real
// parts, then imaginary parts) give every lane its own new amplitude.  Its tile controls are
// register bits (rcmask) or warp bits (tcmask), never lanes.
// kRegPauli: exp(-i theta/2 P), a'_i = cos(theta/2) a_i + y (-1)^parity(i & zy) a_(i ^ x) with
// y = -i sin(theta/2) i^(n_Y) (-1)^parity(x & zy) (kernels::apply_pauli_rotation,
// src/backend/kernels/gate_kernels.cpp:191-225, x and zy formed as in
// statevector_simulator.cpp:36-46): its flip bits x are register bits (code = their register
// mask) or lanes (loc[0] = their lane mask: the partner comes by shuffle), its Z-type bits zy
// are register bits (rcmask), thread bits (tcmask) or out-of-tile qubits (a 64-bit mask among
// its matrices: (cos, 0), y, then the mask as two exact 32-bit halves).
enum : uint8_t { kRegDense = 0, kRegDiag = 1, kRegPhase = 2, kRegSwapX = 3, kRegRemap = 4,
                 kRegDiagDyn = 5, kRegMma = 6, kRegPauli = 7 };

struct RegLayout {
    uint16_t rsw[kRegBits];   // tile_swizzle(1 << rpos[i])
    uint16_t tsw[9];          // tile_swizzle(1 << tpos[i])
    uint8_t rpos[kRegBits];   // tile bit of register-index bit i
    uint8_t tpos[9];          // tile bit of thread-index bit i
    uint8_t pad[1];
};

struct RegOp {
    uint64_t gcmask;          // qubits outside the tile that must all be 1
    uint32_t mat_off;         // double2 offset in the pass's staged matrices
    uint8_t kind;
    uint8_t code;             // dense / swap: register target mask; remap: new layout index
    uint8_t k;                // dense / diag: number of targets; remap: 1 = warp-local
    uint8_t rcmask;           // register-index bits that must be 1 (controls, phase bits)
    uint16_t tcmask;          // thread-index bits that must be 1
    uint8_t loc[kRegMaxDiag]; // diag: target j at register bit loc, or thread bit loc & 0x7f
                              // when loc & 0x80
    uint8_t nsel;             // dense / diag: the tile's bits at qubits selq[0..nsel) pick
    uint8_t selq[kRegMaxSelect];   // one of 2^nsel consecutive matrices
    uint8_t nterm;            // per-tile diagonal: gated phase terms
    uint16_t dyn_off;         // per-tile diagonal: first entry in the per-tile tables
    uint8_t pad[2];
};

struct RegPass {
    uint64_t n_tiles;
    uint64_t batch_stride;
    uint32_t m, L, h;
    uint32_t n_ops, n_layouts, n_mat;
    uint32_t mat_stride;      // double2 between the matrices of consecutive states (0: shared)
    uint32_t sync_tiles;      // barrier between a CTA's tiles
    uint32_t cta_remaps;      // some remap changes the warp bits (every warp's slot set)
    uint32_t hbits[kTileMaxHigh];
    uint32_t n_dyn;           // per-tile diagonals: their record indices and table entries
    uint32_t dyn_entries;
    uint8_t dyn_rec[kRegMaxDyn];
    uint32_t relabel;         // SWAPs relabelled tile bits: tile bit b is stored to the place
    uint8_t store_qubit[kRegMaxBits];   // of qubit store_qubit[b]
    uint32_t load_barrier;    // a barrier between the tile's loads and stores is needed and no
                              // other barrier provides it (relabelled stores, in place)
    uint32_t fma_dense;       // some record is a dense op on register bits (kRegDense)
    uint32_t mma_ops;         // some record is a tensor-path block (kRegMma)
    uint32_t pauli_ops;       // some record is a Pauli rotation (kRegPauli)
};

static_assert(sizeof(RegLayout) % 4 == 0 && sizeof(RegOp) == 32, "staged as 32-bit words");

void launch_reg_pass(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                     const RegPass& pass, const RegOp* d_ops, const RegLayout* d_layouts,
                     const double2* d_mats);
// Shared memory of a register pass holding `tiles` tile buffers (2: double-buffered kernel).
size_t reg_smem_bytes(const RegPass& pass, uint32_t tiles = 1);
constexpr size_t kRegPipeMaxSmem = 220 * 1024;   // double-buffered kernel, one CTA per SM at m = 12

}  // namespace lqcs_b200
