// tile_plan.hpp — planning and lowering of shared-memory tile passes.
#pragma once

#include <vector>

#include "gates.hpp"
#include "tile.cuh"

namespace lqcs_b200 {

struct TileConfig {
    uint32_t m = 12;       // tile bits (2^m amplitudes in shared memory)
    uint32_t L = 5;        // low qubits always in the tile
    uint32_t inner = 2;    // widest dense operation fused inside a pass
    bool reg = true;       // register tile kernel where the pass fits it
    bool search = true;    // local search over each pass's high qubits (LQCS_TILE_SEARCH=0: off)
    bool mma = false;      // register passes: one- and two-qubit blocks on the FP64 tensor
                           // path (mma.sync m8n8k4) instead of FP64 FMAs over register bits
                           // (LQCS_REG_MMA=1)
    bool pauli = true;     // register passes: Pauli rotations whose X/Y qubits (at most
                           // kRegPauliMaxFlips) are tile qubits run inside the pass
                           // (LQCS_TILE_PAULI=0: only those of at most kTileMaxK qubits, as
                           // dense blocks)
};

// Whether gate g runs as a native Pauli rotation inside a register pass (cfg.reg, cfg.pauli,
// an uncontrolled rotation with at most kRegPauliMaxFlips X/Y qubits — on register bits and
// lanes; its Z qubits need not be in the tile).  A pass holding one that does not fit the
// register kernel is split at it.
bool native_pauli(const GateDesc& g, const TileConfig& cfg);
TileConfig default_tile_config(uint32_t n);

// A pass (hbits + gates applied in program order) or one gate run on its own.
struct PlanItem {
    bool is_pass = false;
    uint32_t gate = 0;
    std::vector<uint32_t> hbits;
    std::vector<uint32_t> gates;
};

std::vector<PlanItem> plan_tiles(const std::vector<GateDesc>& gates, uint32_t n,
                                 const TileConfig& cfg);

// A phase factor f on the amplitudes whose tile-local bits lbits are all 1, applied only in
// tiles whose out-of-tile qubits gcmask are all 1: one term of a diagonal whose table is
// built per tile.
struct DynTerm {
    uint64_t gcmask = 0;
    uint32_t lbits = 0;
    cd f{1, 0};
};

// One operation of a pass in tile-local bits, before it is encoded for a kernel.
struct LocalOp {
    uint8_t kind = kTileDense;      // kTileDense, kTileDiag or kTilePhase
    std::vector<uint32_t> lt;       // targets, matrix local order (none for a phase)
    uint32_t lmask = 0;             // local controls, or the local bits of a phase
    uint64_t gcmask = 0;            // controls / phase bits outside the tile
    std::vector<uint32_t> sel;      // out-of-tile qubits selecting one of 2^|sel| matrices
    bool variant = false;           // contains a noise slot: the matrices differ per state
    std::vector<cd> m;              // dense: 2^k x 2^k, diagonal: 2^k, phase: the factor;
                                    // with sel, one such block per selector value
    std::vector<DynTerm> dyn;       // diagonal: gated phase terms multiplied into m per tile
    // kTilePauli: lt = the flip (X/Y) bits, lmask = the Z-type (Z/Y) tile bits, pz_out = the
    // Z-type qubits outside the tile, m = {(cos, 0), y} (see kRegPauli)
    uint64_t pz_out = 0;
};

// The operations of one pass in program order, neighbouring gates fused into blocks of at
// most cfg.inner local qubits.  A block may take gates controlled by up to max_select
// qubits outside the tile: those bits are constant over a tile, so the block becomes one
// matrix per value of them, picked per tile.
// Runs of commuting diagonal work merge into diagonals of at most max_diag tile bits; with
// dyn_terms, phases gated by other out-of-tile qubits join them as per-tile terms.  With
// store_qubits, SWAPs of two tile qubits become relabellings (no operation) and
// store_qubits[b] receives the qubit whose place tile bit b is stored to.
std::vector<LocalOp> pass_local_ops(const PlanItem& item, const std::vector<GateDesc>& gates,
                                    const TileConfig& cfg, uint32_t max_select,
                                    const std::vector<std::array<cd, 4>>* slot_mats = nullptr,
                                    uint32_t max_diag = kTileMaxK, bool dyn_terms = false,
                                    std::vector<uint32_t>* store_qubits = nullptr,
                                    bool native_rotations = false);

// Append the tile operations of one pass to ops_out (matrices to arena) and fill `pass`.
void lower_pass(const PlanItem& item, const std::vector<GateDesc>& gates, const TileConfig& cfg,
                TilePass& pass, std::vector<TileOp>& ops_out, std::vector<cd>& arena,
                double* flops_per_amp = nullptr);

// Register-tile encoding of one pass: the operations scheduled over a sequence of register
// layouts (greedy: each layout applies every pending operation it can, the next one is the
// register set that applies the most), with a remap record between layouts.  Returns false
// when the pass does not fit the register kernel (tile size, a dense operation of more than
// kRegMaxK targets, record / layout / matrix limits); nothing is appended then.
// With state_slots (one table of noise-slot matrices per state of a batch) the records are
// shared and the matrices are stored once per state, n_mat apart (pass.mat_stride).
bool lower_pass_reg(const PlanItem& item, const std::vector<GateDesc>& gates,
                    const TileConfig& cfg, RegPass& pass, std::vector<RegOp>& ops_out,
                    std::vector<RegLayout>& layouts_out, std::vector<cd>& mats_out,
                    double* flops_per_amp = nullptr,
                    const std::vector<std::vector<std::array<cd, 4>>>* state_slots = nullptr);

// FP64 flops per state amplitude one pass operation executes (op_flops_per_amp's
// conventions); x_free: an uncontrolled-by-selector X runs as a register swap.
double local_op_flops(const LocalOp& o, bool x_free);

}  // namespace lqcs_b200
