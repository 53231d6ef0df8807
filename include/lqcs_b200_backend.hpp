// lqcs_b200_backend.hpp — header-only drop-in backend for LiteQuantumComputingSimulator.
//
// CudaStatevectorSimulator is an lqcs::Backend (include/lqcs/backend/backend.hpp:11-17)
// with the public surface of lqcs::StatevectorSimulator
// (include/lqcs/backend/statevector_simulator.hpp:17-42): the same Options
// {seed, fuse_gates, num_threads, noise}, run(circuit, shots = 1024) -> Result,
// run_statevector(circuit) -> host Statevector, name().  It flattens the reference's own
// QuantumCircuit into lqcs_instruction records and calls the engine's C ABI
// (lqcs_b200.h); engine status codes come back as the exception types the reference
// throws (std::invalid_argument, std::out_of_range, std::logic_error) with the same text.
//
// Include it in a program that already builds against the reference (include/lqcs/...)
// and link liblqcs_b200.so.
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include <lqcs/backend/backend.hpp>
#include <lqcs/backend/statevector.hpp>
#include <lqcs/backend/statevector_simulator.hpp>

#include "lqcs_b200.h"

namespace lqcs_b200 {

inline void rethrow(int status) {
    if (status == LQCS_OK) return;
    const std::string msg = lqcs_last_error();
    switch (status) {
        case LQCS_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
        case LQCS_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
        case LQCS_ERR_LOGIC: throw std::logic_error(msg);
        default: throw std::runtime_error(msg);
    }
}

// The records point into the circuit's own storage: the circuit must outlive them.
inline std::vector<lqcs_instruction> flatten(const lqcs::QuantumCircuit& circuit) {
    static_assert(sizeof(lqcs::qubit_t) == sizeof(uint32_t), "qubit_t must be 32-bit");
    static_assert(sizeof(std::size_t) == sizeof(uint64_t), "size_t must be 64-bit");
    static_assert(sizeof(lqcs::complex_t) == 2 * sizeof(double), "complex_t must be 2 doubles");
    std::vector<lqcs_instruction> out;
    out.reserve(circuit.num_instructions());
    for (const lqcs::Instruction& inst : circuit.instructions()) {
        const lqcs::Gate& g = inst.gate;
        lqcs_instruction r{};
        r.gate_type = static_cast<int32_t>(g.type);
        r.n_controls = static_cast<uint32_t>(g.n_controls);
        r.n_qubits = static_cast<uint32_t>(inst.qubits.size());
        r.n_params = static_cast<uint32_t>(g.params.size() < 3 ? g.params.size() : 3);
        for (uint32_t k = 0; k < r.n_params; ++k) r.params[k] = g.params[k];
        r.clbit = inst.clbits.empty() ? 0 : inst.clbits[0];
        r.qubits = inst.qubits.data();
        r.matrix = g.mat.empty() ? nullptr : reinterpret_cast<const double*>(g.mat.data());
        r.perm = g.perm.empty() ? nullptr : reinterpret_cast<const uint64_t*>(g.perm.data());
        r.pauli = g.pauli.empty() ? nullptr : g.pauli.c_str();
        out.push_back(r);
    }
    return out;
}

class CudaStatevectorSimulator final : public lqcs::Backend {
public:
    using Options = lqcs::StatevectorSimulator::Options;

    CudaStatevectorSimulator() = default;
    explicit CudaStatevectorSimulator(Options options) : options_(std::move(options)) {}

    lqcs::Result run(const lqcs::QuantumCircuit& circuit, std::size_t shots = 1024) override {
        const std::vector<lqcs_instruction> recs = flatten(circuit);
        std::vector<std::vector<double>> ops;
        std::vector<lqcs_kraus_channel> chans;
        lqcs_sim_options o = options();
        for (const lqcs::KrausChannel& ch : options_.noise.channels()) {
            std::vector<double> flat;
            for (const auto& k : ch.ops)
                for (const auto& z : k) {
                    flat.push_back(z.real());
                    flat.push_back(z.imag());
                }
            ops.push_back(std::move(flat));
        }
        for (size_t c = 0; c < ops.size(); ++c)
            chans.push_back({options_.noise.channels()[c].ops.size(), ops[c].data()});
        o.n_channels = chans.size();
        o.channels = chans.empty() ? nullptr : chans.data();
        std::vector<uint64_t> regs(shots ? shots : 1);
        rethrow(lqcs_run(static_cast<uint32_t>(circuit.num_qubits()),
                         static_cast<uint32_t>(circuit.num_clbits()), recs.data(), recs.size(),
                         shots, &o, regs.data()));
        const std::size_t nc = circuit.num_clbits();
        std::map<std::string, std::size_t> counts;
        std::string key(nc, '0');
        for (std::size_t s = 0; s < shots; ++s) {
            for (std::size_t c = 0; c < nc; ++c) key[nc - 1 - c] = ((regs[s] >> c) & 1) ? '1' : '0';
            ++counts[key];
        }
        return lqcs::Result(std::move(counts), shots);
    }

    std::string name() const override { return "statevector_simulator"; }

    // The final state copied into host memory as an lqcs::Statevector (the reference's
    // 30-qubit host cap applies to this return type).
    lqcs::Statevector run_statevector(const lqcs::QuantumCircuit& circuit) const {
        if (!options_.noise.empty()) {
            throw std::invalid_argument(
                "run_statevector: noisy simulation is stochastic (one trajectory is not the "
                "quantum state); use run() or DensityMatrixSimulator");
        }
        lqcs::Statevector sv(circuit.num_qubits());
        lqcs_state* st = nullptr;
        const std::vector<lqcs_instruction> recs = flatten(circuit);
        const lqcs_sim_options o = options();
        rethrow(lqcs_run_statevector(static_cast<uint32_t>(circuit.num_qubits()), recs.data(),
                                     recs.size(), &o, nullptr, &st));
        const int rc = lqcs_state_store(st, reinterpret_cast<double*>(sv.data()), sv.size());
        lqcs_state_destroy(st);
        rethrow(rc);
        return sv;
    }

private:
    lqcs_sim_options options() const {
        lqcs_sim_options o{};
        o.has_seed = options_.seed.has_value() ? 1 : 0;
        o.seed = options_.seed.value_or(0);
        o.fuse_gates = options_.fuse_gates ? 1 : 0;
        o.num_threads = options_.num_threads;
        return o;
    }

    Options options_;
};

}  // namespace lqcs_b200
