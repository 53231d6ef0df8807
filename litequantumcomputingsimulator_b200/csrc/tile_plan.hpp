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
};
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

// Append the tile operations of one pass to ops_out (matrices to arena) and fill `pass`.
void lower_pass(const PlanItem& item, const std::vector<GateDesc>& gates, const TileConfig& cfg,
                TilePass& pass, std::vector<TileOp>& ops_out, std::vector<cd>& arena);

}  // namespace lqcs_b200
