// gates.hpp — host-side gate model of the engine: decoding of lqcs_instruction records,
// gate matrices, lowering to device operations, and the fusion planner.
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lqcs_b200.h"

namespace lqcs_b200 {

using cd = std::complex<double>;

// Error carrying one of the lqcs_status codes; the C ABI turns it into a status code and
// the message returned by lqcs_last_error().
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] inline void invalid(const std::string& m) { throw Error(LQCS_ERR_INVALID_ARGUMENT, m); }
[[noreturn]] inline void out_of_range(const std::string& m) { throw Error(LQCS_ERR_OUT_OF_RANGE, m); }
[[noreturn]] inline void logic(const std::string& m) { throw Error(LQCS_ERR_LOGIC, m); }

// A decoded instruction: lqcs::Instruction + lqcs::Gate
// (include/lqcs/circuit/instruction.hpp:9-13, include/lqcs/circuit/gate.hpp:30-68).
struct GateDesc {
    int type = LQCS_GATE_I;
    uint32_t n_controls = 0;
    std::vector<uint32_t> qubits;        // controls first, then targets
    std::vector<double> params;
    std::vector<cd> mat;                 // UNITARY
    std::vector<uint64_t> perm;          // PERMUTATION
    std::string pauli;                   // PAULI_ROTATION
    uint32_t clbit = 0;                  // MEASURE
    std::vector<std::array<cd, 4>> kraus;  // KRAUS
    // Engine-internal: a noise slot of a trajectory batch — a one-qubit UNITARY whose 2x2
    // matrix differs per state (slot_id indexes the per-state tables); never specialised
    // as a phase, diagonal or X.
    bool slot = false;
    uint32_t slot_id = 0;

    uint32_t base_qubits() const;        // Gate::base_qubits (src/circuit/gate.cpp:27-49)
    bool is_unitary() const;             // not Measure / Reset / Barrier / Kraus
    std::string name() const;            // Gate::name (src/circuit/gate.cpp:283-317)
    // Gate::base_matrix (src/circuit/gate.cpp:94-201): 2^k x 2^k row-major, no controls.
    std::vector<cd> base_matrix() const;
    // Matrix on all of `qubits` (controls in the low local bits) — Gate::matrix
    // (src/circuit/gate.cpp:203-226).
    std::vector<cd> full_matrix() const;
    const uint32_t* controls() const { return qubits.data(); }
    const uint32_t* targets() const { return qubits.data() + n_controls; }
};

struct PauliMasks {
    uint64_t x = 0, zy = 0;
    uint32_t n_y = 0;
};
// Gate::pauli_masks (src/circuit/gate.cpp:51-68): local bit j <-> pauli[k-1-j].
PauliMasks pauli_local_masks(const std::string& pauli);
// Pauli string over all n qubits, leftmost character = highest qubit
// (src/backend/statevector.cpp:44-60).
PauliMasks pauli_global_masks(const char* pauli, uint32_t n, const char* who);

// Decode and validate one C record against an n-qubit register.
GateDesc decode(const lqcs_instruction& in, uint32_t n_qubits);
std::vector<GateDesc> decode_all(const lqcs_instruction* insts, uint64_t n_insts,
                                 uint32_t n_qubits);

// ------------------------------------------------------------------ device operations
enum class OpKind { K1Q, PHASE, DENSE, DIAG, PERM, PAULI, TILE };

struct DevOp {
    OpKind kind = OpKind::DENSE;
    uint32_t k = 0;                      // number of targets
    std::vector<uint32_t> targets;       // local bit j <-> targets[j]
    uint64_t cmask = 0;
    // K1Q
    std::array<cd, 4> m1{};
    bool diag1 = false;
    // PHASE
    uint64_t phase_mask = 0;
    cd phase{1.0, 0.0};
    // DENSE / DIAG: matrix (2^k x 2^k) or diagonal (2^k)
    std::vector<cd> mat;
    // PERM: cycles over local indices
    std::vector<uint32_t> cycles, cycle_len;
    // PAULI
    uint64_t x = 0, zy = 0;
    uint32_t n_y = 0;
    double cos_h = 1.0, sin_h = 0.0;
    // TILE: index of the pass in the program's shared-memory or register pass list
    uint32_t pass_index = 0;
    bool reg_tile = false;
    double tile_flops = 0.0;             // TILE: FP64 flops per state amplitude of the pass
    // bookkeeping
    uint32_t src_gates = 1;              // source gates merged into this op
    double alg_fraction = 1.0;           // fraction of amplitudes it can change
};

// FP64 flops per state amplitude an op executes: 8 per complex multiply-add of a dense
// 2^k block row (8 * 2^k), 6 per complex multiply of a diagonal or phase, none for
// permutations; scaled by the fraction of amplitudes the op touches.
double op_flops_per_amp(const DevOp& op);

// Kind number of an op in profiles and cost-model features: the OpKind, or 7 for a tile
// pass run by the register kernel.
inline uint32_t profile_kind(const DevOp& op) {
    return op.kind == OpKind::TILE && op.reg_tile ? 7u : static_cast<uint32_t>(op.kind);
}

// Lower one unitary gate to a device op following the dispatch of apply_instruction
// (src/backend/statevector_simulator.cpp:22-85) — plus a PHASE fast path for diagonal
// gates with d0 == 1.  States with n < 5 use DENSE/DIAG/PERM only.
DevOp lower_gate(const GateDesc& g, uint32_t n);

// ------------------------------------------------------------------ fusion
struct FusedBlock {
    std::vector<uint32_t> qubits;        // sorted ascending
    std::vector<uint32_t> gates;         // indices into the gate list, program order
};

// Greedy block fusion: gates join an open block while the union of qubits stays within
// max_width; a gate that would overflow closes the blocks it touches.  Gates wider than
// max_width stand alone.  Correct for any order because open blocks act on disjoint qubits.
std::vector<FusedBlock> plan_greedy(const std::vector<GateDesc>& gates, uint32_t n,
                                    uint32_t max_width);

// Merge neighbouring blocks of an emission order while their qubit union fits max_width.
std::vector<FusedBlock> pack_consecutive(const std::vector<FusedBlock>& blocks,
                                         uint32_t max_width);

// Dense matrix of a block (block-local bit j <-> qubits[j]).
std::vector<cd> block_matrix(const FusedBlock& b, const std::vector<GateDesc>& gates);

// Turn a plan into device ops (single-gate blocks keep their specialised kernel).
std::vector<DevOp> lower_plan(const std::vector<FusedBlock>& plan,
                              const std::vector<GateDesc>& gates, uint32_t n);

// Fraction of amplitudes a gate can change (32 N f algorithmic bytes per gate).
double gate_alg_fraction(const GateDesc& g);

}  // namespace lqcs_b200
