// tile.cuh — operation records of the shared-memory tile passes (tile_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace lqcs_b200 {

constexpr uint32_t kTileThreads = 256;
constexpr uint32_t kTileMaxBits = 13;            // 2^13 amplitudes = 128 KiB of shared memory
constexpr uint32_t kTileMaxHigh = 8;             // at most 8 high qubits per tile
constexpr uint32_t kTileMaxK = 4;                // widest dense operation inside a tile
constexpr uint32_t kTileMaxOps = 512;            // operations per pass (staged in shared memory)
constexpr size_t kTileMaxSmem = 200 * 1024;      // tile + staged operation records

enum : uint8_t { kTileDense = 0, kTileDiag = 1, kTilePhase = 2 };

// One operation on a tile, in tile-local bit positions (local bit j < L is qubit j, local
// bit L + i is the i-th high qubit of the tile).
struct TileOp {
    uint64_t gcmask;      // qubits outside the tile that must all be 1 (controls / phase bits)
    uint32_t lcmask;      // dense/diag: local control bits; phase: local phase bits
    uint32_t mat_off;     // matrix (dense), diagonal (diag) or phase factor (phase), in double2
    uint16_t loff[16];    // local offsets of the 2^k members of a group (matrix local order)
    uint8_t kind;
    uint8_t k;
    uint8_t n_fixed;      // number of local positions inserted as zeros when enumerating groups
    uint8_t n_lctrl;      // popcount(lcmask) for dense/diag
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

}  // namespace lqcs_b200
