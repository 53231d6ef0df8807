// ref_shim.cpp — ORACLE (test infrastructure only; never part of the product path).
//
// A C entry layer over the reference implementation itself, compiled together with the
// reference's own sources (see oracle/Makefile) into oracle/_ref/liblqcs_ref.so.  Tests
// and bench.py's CPU-baseline leg call it through ctypes to obtain the reference's
// amplitudes, counts, expectations, gradients and density-matrix probabilities, and to
// time the reference's OpenMP kernels.  Circuits arrive as the engine's lqcs_instruction
// records (include/lqcs_b200.h) and are rebuilt here as lqcs::QuantumCircuit objects with
// the reference's public API.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include <lqcs/lqcs.hpp>

#include "backend/kernels/kernels.hpp"
#include "lqcs_b200.h"

using namespace lqcs;

namespace {

thread_local std::string g_err;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return 1;
    } catch (const std::out_of_range& e) {
        g_err = e.what();
        return 2;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 3;
    }
}

Gate to_gate(const lqcs_instruction& in) {
    const auto type = static_cast<GateType>(in.gate_type);
    std::vector<double> params(in.params, in.params + in.n_params);
    const std::size_t k = in.n_qubits - in.n_controls;
    std::vector<complex_t> mat;
    std::vector<std::size_t> perm;
    std::string pauli;
    if (type == GateType::Unitary) {
        const std::size_t dim = std::size_t{1} << k;
        for (std::size_t i = 0; i < dim * dim; ++i)
            mat.emplace_back(in.matrix[2 * i], in.matrix[2 * i + 1]);
    }
    if (type == GateType::Permutation) {
        const std::size_t dim = std::size_t{1} << k;
        perm.assign(in.perm, in.perm + dim);
    }
    if (type == GateType::PauliRotation) pauli = in.pauli;
    return Gate{type, params, in.n_controls, mat, perm, pauli};
}

Instruction to_inst(const lqcs_instruction& in) {
    Instruction inst{to_gate(in), std::vector<qubit_t>(in.qubits, in.qubits + in.n_qubits), {}};
    if (in.gate_type == LQCS_GATE_MEASURE) inst.clbits = {in.clbit};
    return inst;
}

QuantumCircuit to_circuit(uint32_t n, uint32_t nclbits, const lqcs_instruction* insts,
                          uint64_t n_insts) {
    QuantumCircuit qc(n, nclbits);
    for (uint64_t i = 0; i < n_insts; ++i) {
        if (insts[i].gate_type == LQCS_GATE_KRAUS) throw std::invalid_argument("kraus instruction");
        if (insts[i].gate_type == LQCS_GATE_RESET) qc.reset(insts[i].qubits[0]);
        else if (insts[i].gate_type == LQCS_GATE_BARRIER) qc.barrier();
        else qc.append(to_inst(insts[i]));
    }
    return qc;
}

KrausChannel to_channel(const lqcs_kraus_channel& c) {
    std::vector<std::array<complex_t, 4>> ops(c.n_ops);
    for (uint64_t o = 0; o < c.n_ops; ++o)
        for (int e = 0; e < 4; ++e) ops[o][e] = complex_t{c.ops[8 * o + 2 * e], c.ops[8 * o + 2 * e + 1]};
    return KrausChannel(ops);
}

KrausChannel kraus_of(const lqcs_instruction& in) {
    lqcs_kraus_channel c{in.n_kraus, in.matrix};
    return to_channel(c);
}

uint64_t key_to_register(const std::string& key) {
    uint64_t r = 0;
    const std::size_t n = key.size();
    for (std::size_t c = 0; c < n; ++c)
        if (key[n - 1 - c] == '1') r |= uint64_t{1} << c;
    return r;
}

void write_counts(const Result& res, uint64_t* keys, uint64_t* counts, uint64_t cap,
                  uint64_t* n_out) {
    uint64_t i = 0;
    for (const auto& [k, v] : res.counts()) {
        if (i < cap) {
            keys[i] = key_to_register(k);
            counts[i] = v;
        }
        ++i;
    }
    *n_out = i;
}

// The instruction dispatch of the reference's statevector backend restated over the
// reference's own kernels, so a circuit can start from any given state.
void apply_with_kernels(complex_t* s, std::size_t n_amps, const Instruction& inst) {
    const Gate& g = inst.gate;
    const std::size_t nc = g.n_controls;
    const std::size_t k = g.base_qubits();
    const qubit_t* controls = inst.qubits.data();
    const qubit_t* targets = inst.qubits.data() + nc;
    if (g.type == GateType::Permutation) {
        kernels::apply_controlled_permutation(s, n_amps, controls, nc, targets, k, g.perm.data());
        return;
    }
    if (g.type == GateType::PauliRotation && nc == 0) {
        const auto pm = g.pauli_masks();
        std::size_t xg = 0, zyg = 0;
        for (std::size_t j = 0; j < k; ++j) {
            if (pm.x & (std::size_t{1} << j)) xg |= std::size_t{1} << targets[j];
            if (pm.zy & (std::size_t{1} << j)) zyg |= std::size_t{1} << targets[j];
        }
        kernels::apply_pauli_rotation(s, n_amps, xg, zyg, pm.n_y, g.params.at(0));
        return;
    }
    if (nc == 0 && k == 1) {
        const auto m = g.base_matrix();
        if (g.is_diagonal()) kernels::apply_diagonal_single_qubit(s, n_amps, targets[0], m[0], m[3]);
        else kernels::apply_single_qubit(s, n_amps, targets[0], m.data());
        return;
    }
    if (nc == 0 && g.type == GateType::SWAP) {
        kernels::apply_swap(s, n_amps, targets[0], targets[1]);
        return;
    }
    if (nc == 0 && k == 2) {
        const auto m = g.base_matrix();
        kernels::apply_two_qubit(s, n_amps, targets[0], targets[1], m.data());
        return;
    }
    if (nc == 1 && k == 1) {
        const auto m = g.base_matrix();
        kernels::apply_controlled_single_qubit(s, n_amps, controls[0], targets[0], m.data());
        return;
    }
    const auto m = g.base_matrix();
    kernels::apply_controlled_unitary(s, n_amps, controls, nc, targets, k, m.data());
}

}  // namespace

extern "C" {

const char* lqcsref_last_error(void) { return g_err.c_str(); }

void lqcsref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int lqcsref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// StatevectorSimulator::run_statevector
int lqcsref_run_statevector(uint32_t n, const lqcs_instruction* insts, uint64_t n_insts,
                            int fuse, double* out) {
    return guarded([&] {
        StatevectorSimulator sim({.fuse_gates = fuse != 0});
        const Statevector sv = sim.run_statevector(to_circuit(n, 0, insts, n_insts));
        std::memcpy(out, sv.data(), sizeof(complex_t) * sv.size());
    });
}

// StatevectorSimulator::run with an all-qubit noise model; counts as (register, count)
int lqcsref_run(uint32_t n, uint32_t nclbits, const lqcs_instruction* insts, uint64_t n_insts,
                uint64_t shots, int has_seed, uint64_t seed, int fuse, uint64_t n_channels,
                const lqcs_kraus_channel* channels, uint64_t* keys, uint64_t* counts,
                uint64_t cap, uint64_t* n_out) {
    return guarded([&] {
        NoiseModel noise;
        for (uint64_t c = 0; c < n_channels; ++c) noise.add_all_qubit_channel(to_channel(channels[c]));
        StatevectorSimulator::Options o;
        if (has_seed) o.seed = seed;
        o.fuse_gates = fuse != 0;
        o.noise = noise;
        StatevectorSimulator sim(o);
        const Result r = sim.run(to_circuit(n, nclbits, insts, n_insts), shots);
        write_counts(r, keys, counts, cap, n_out);
    });
}

// DensityMatrixSimulator::run (src/backend/density_matrix_simulator.cpp:26-80): counts of
// the final density matrix's diagonal, noise model after every unitary.
int lqcsref_dm_run(uint32_t n, uint32_t nclbits, const lqcs_instruction* insts, uint64_t n_insts,
                   uint64_t shots, int has_seed, uint64_t seed, uint64_t n_channels,
                   const lqcs_kraus_channel* channels, uint64_t* keys, uint64_t* counts,
                   uint64_t cap, uint64_t* n_out) {
    return guarded([&] {
        DensityMatrixSimulator::Options o;
        if (has_seed) o.seed = seed;
        for (uint64_t c = 0; c < n_channels; ++c) o.noise.add_all_qubit_channel(to_channel(channels[c]));
        DensityMatrixSimulator sim(o);
        const Result r = sim.run(to_circuit(n, nclbits, insts, n_insts), shots);
        write_counts(r, keys, counts, cap, n_out);
    });
}

// io::to_qasm(io::from_qasm(src)) (src/io/qasm.cpp) into out (capacity cap, NUL-terminated).
int lqcsref_qasm_roundtrip(const char* src, char* out, uint64_t cap) {
    return guarded([&] {
        const std::string text = io::to_qasm(io::from_qasm(src));
        if (text.size() + 1 > cap) throw std::invalid_argument("qasm_roundtrip: buffer too small");
        std::memcpy(out, text.c_str(), text.size() + 1);
    });
}

// Evolve a given state by the unitary instructions with the reference kernels.
int lqcsref_evolve_from(uint32_t n, const double* in, const lqcs_instruction* insts,
                        uint64_t n_insts, double* out) {
    return guarded([&] {
        Statevector sv(n);
        std::memcpy(sv.data(), in, sizeof(complex_t) * sv.size());
        for (uint64_t i = 0; i < n_insts; ++i) {
            const Instruction inst = to_inst(insts[i]);
            if (inst.gate.is_unitary()) apply_with_kernels(sv.data(), sv.size(), inst);
        }
        std::memcpy(out, sv.data(), sizeof(complex_t) * sv.size());
    });
}

// Time the reference kernels: apply the unitary instructions `reps` times to a state of
// n qubits (allocated and touched once, outside the timed region).  Seconds per pass over
// the instruction list.
int lqcsref_time_apply(uint32_t n, const lqcs_instruction* insts, uint64_t n_insts,
                       uint32_t reps, double* seconds) {
    return guarded([&] {
        // one host state per register size, allocated and first-touched once
        static std::unique_ptr<Statevector> cached;
        if (!cached || cached->num_qubits() != n) {
            cached.reset();
            cached = std::make_unique<Statevector>(n);
        }
        Statevector& sv = *cached;
        std::vector<Instruction> list;
        for (uint64_t i = 0; i < n_insts; ++i) list.push_back(to_inst(insts[i]));
        const auto t0 = std::chrono::steady_clock::now();
        for (uint32_t r = 0; r < reps; ++r)
            for (const Instruction& inst : list)
                if (inst.gate.is_unitary()) apply_with_kernels(sv.data(), sv.size(), inst);
        const auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count() / reps;
    });
}

int lqcsref_expectation(uint32_t n, const double* amps, const char* pauli, double* out) {
    return guarded([&] {
        Statevector sv(n);
        std::memcpy(sv.data(), amps, sizeof(complex_t) * sv.size());
        *out = sv.expectation_value(pauli);
    });
}

int lqcsref_hamiltonian(uint32_t n, const double* amps, uint64_t n_terms, const double* coeffs,
                        const char* const* paulis, double* out) {
    return guarded([&] {
        Statevector sv(n);
        std::memcpy(sv.data(), amps, sizeof(complex_t) * sv.size());
        algorithms::Hamiltonian h;
        for (uint64_t t = 0; t < n_terms; ++t) h.push_back({coeffs[t], paulis[t]});
        *out = algorithms::expectation(sv, h);
    });
}

// algorithms::parameter_shift_gradient on a ParametricCircuit rebuilt from the template.
int lqcsref_parameter_shift(uint32_t n, const lqcs_instruction* insts, uint64_t n_insts,
                            const uint64_t* param_inst, uint64_t n_params, uint64_t n_terms,
                            const double* coeffs, const char* const* paulis,
                            const double* params, double* grad) {
    return guarded([&] {
        ParametricCircuit pc(n);
        std::vector<bool> is_param(n_insts, false);
        for (uint64_t p = 0; p < n_params; ++p) is_param[param_inst[p]] = true;
        for (uint64_t i = 0; i < n_insts; ++i) {
            const lqcs_instruction& in = insts[i];
            const qubit_t* q = in.qubits;
            const auto type = static_cast<GateType>(in.gate_type);
            if (is_param[i]) {
                switch (type) {
                    case GateType::RX: pc.rx(q[0]); break;
                    case GateType::RY: pc.ry(q[0]); break;
                    case GateType::RZ: pc.rz(q[0]); break;
                    case GateType::PauliRotation:
                        pc.rp(in.pauli, std::span<const qubit_t>(q, in.n_qubits));
                        break;
                    default: throw std::invalid_argument("unsupported parameterised gate");
                }
                continue;
            }
            const bool ctl = in.n_controls > 0;
            switch (type) {
                case GateType::X:
                    if (in.n_controls == 2) pc.ccx(q[0], q[1], q[2]);
                    else if (ctl) pc.cx(q[0], q[1]);
                    else pc.x(q[0]);
                    break;
                case GateType::Y: ctl ? pc.cy(q[0], q[1]) : pc.y(q[0]); break;
                case GateType::Z: ctl ? pc.cz(q[0], q[1]) : pc.z(q[0]); break;
                case GateType::H: pc.h(q[0]); break;
                case GateType::S: pc.s(q[0]); break;
                case GateType::Sdg: pc.sdg(q[0]); break;
                case GateType::T: pc.t(q[0]); break;
                case GateType::SX: pc.sx(q[0]); break;
                case GateType::SWAP: pc.swap(q[0], q[1]); break;
                case GateType::Barrier: pc.barrier(); break;
                default: throw std::invalid_argument("unsupported fixed gate in ParametricCircuit");
            }
        }
        algorithms::Hamiltonian h;
        for (uint64_t t = 0; t < n_terms; ++t) h.push_back({coeffs[t], paulis[t]});
        const auto g = algorithms::parameter_shift_gradient(
            h, pc, std::span<const double>(params, n_params));
        std::memcpy(grad, g.data(), sizeof(double) * g.size());
    });
}

// DensityMatrix probabilities after the circuit: unitary instructions followed by every
// all-qubit channel on the touched qubits (density_matrix_simulator.cpp semantics), plus
// explicit Kraus instructions applied where they stand.
int lqcsref_dm_probabilities(uint32_t n, const lqcs_instruction* insts, uint64_t n_insts,
                             uint64_t n_channels, const lqcs_kraus_channel* channels,
                             double* probs) {
    return guarded([&] {
        DensityMatrix rho(n);
        std::vector<KrausChannel> chs;
        for (uint64_t c = 0; c < n_channels; ++c) chs.push_back(to_channel(channels[c]));
        for (uint64_t i = 0; i < n_insts; ++i) {
            const lqcs_instruction& in = insts[i];
            if (in.gate_type == LQCS_GATE_KRAUS) {
                rho.apply_channel(kraus_of(in), in.qubits[0]);
                continue;
            }
            if (in.gate_type == LQCS_GATE_MEASURE || in.gate_type == LQCS_GATE_BARRIER) continue;
            if (in.gate_type == LQCS_GATE_RESET) throw std::invalid_argument("reset");
            const Instruction inst = to_inst(in);
            rho.apply_instruction(inst);
            for (const auto& ch : chs)
                for (qubit_t q : inst.qubits) rho.apply_channel(ch, q);
        }
        const auto p = rho.probabilities();
        std::memcpy(probs, p.data(), sizeof(double) * p.size());
    });
}

// Trajectory driver with the reference's per-shot semantics
// (statevector_simulator.cpp:122-190) that also honours explicit Kraus instructions:
// one uniform per Measure / Reset / Kraus instruction and per (unitary x channel x qubit).
int lqcsref_trajectories(uint32_t n, uint32_t nclbits, const lqcs_instruction* insts,
                         uint64_t n_insts, uint64_t shots, uint64_t seed, uint64_t n_channels,
                         const lqcs_kraus_channel* channels, uint64_t* regs) {
    return guarded([&] {
        std::vector<KrausChannel> chs;
        for (uint64_t c = 0; c < n_channels; ++c) chs.push_back(to_channel(channels[c]));
        Rng rng(seed);
        auto branch = [&](Statevector& sv, const KrausChannel& ch, qubit_t q) {
            const double r = rng.uniform();
            double cum = 0.0;
            const std::array<complex_t, 4>* chosen = nullptr;
            double chosen_p = 0.0;
            for (const auto& k : ch.ops) {
                const double p = kernels::kraus_probability(sv.data(), sv.size(), q, k.data());
                if (p <= 0.0) continue;
                chosen = &k;
                chosen_p = p;
                cum += p;
                if (r < cum) break;
            }
            if (!chosen) return;
            const double inv = 1.0 / std::sqrt(chosen_p);
            const complex_t m[4] = {(*chosen)[0] * inv, (*chosen)[1] * inv, (*chosen)[2] * inv,
                                    (*chosen)[3] * inv};
            kernels::apply_single_qubit(sv.data(), sv.size(), q, m);
        };
        std::vector<Instruction> list;
        std::vector<int> kinds;
        std::vector<KrausChannel> kraus;
        std::vector<int> kraus_idx;
        for (uint64_t i = 0; i < n_insts; ++i) {
            kinds.push_back(insts[i].gate_type);
            if (insts[i].gate_type == LQCS_GATE_KRAUS) {
                kraus_idx.push_back(static_cast<int>(kraus.size()));
                kraus.push_back(kraus_of(insts[i]));
                list.push_back(Instruction{Gate{GateType::Barrier}, {insts[i].qubits[0]}, {}});
            } else {
                kraus_idx.push_back(-1);
                if (insts[i].gate_type == LQCS_GATE_RESET)
                    list.push_back(Instruction{Gate{GateType::Reset}, {insts[i].qubits[0]}, {}});
                else
                    list.push_back(to_inst(insts[i]));
            }
        }
        for (uint64_t s = 0; s < shots; ++s) {
            Statevector sv(n);
            uint64_t creg = 0;
            for (uint64_t i = 0; i < n_insts; ++i) {
                const int kind = kinds[i];
                const Instruction& inst = list[i];
                if (kind == LQCS_GATE_MEASURE) {
                    const bool o = kernels::collapse_qubit(sv.data(), sv.size(), inst.qubits[0], rng.uniform());
                    if (o) creg |= uint64_t{1} << inst.clbits[0];
                    else creg &= ~(uint64_t{1} << inst.clbits[0]);
                } else if (kind == LQCS_GATE_RESET) {
                    kernels::reset_qubit(sv.data(), sv.size(), inst.qubits[0], rng.uniform());
                } else if (kind == LQCS_GATE_BARRIER) {
                } else if (kind == LQCS_GATE_KRAUS) {
                    branch(sv, kraus[kraus_idx[i]], inst.qubits[0]);
                } else {
                    apply_with_kernels(sv.data(), sv.size(), inst);
                    for (const auto& ch : chs)
                        for (qubit_t q : inst.qubits) branch(sv, ch, q);
                }
            }
            regs[s] = creg;
        }
        (void)nclbits;
    });
}

// Period-finding register of algorithms::modular_exponentiation
// (src/algorithms/arithmetic.cpp): work register |1>, H on every counting qubit, then the
// controlled modular multiplications; the amplitudes of run_statevector.
int lqcsref_modexp_statevector(uint64_t a, uint64_t N, uint32_t n_count, uint32_t n_work,
                               double* out) {
    return guarded([&] {
        QuantumCircuit qc(n_count + n_work);
        qc.x(static_cast<qubit_t>(n_count));
        for (uint32_t j = 0; j < n_count; ++j) qc.h(static_cast<qubit_t>(j));
        qc.compose(algorithms::modular_exponentiation(a, N, n_count, n_work));
        StatevectorSimulator sim;
        const Statevector sv = sim.run_statevector(qc);
        std::memcpy(out, sv.data(), sizeof(complex_t) * sv.size());
    });
}

// algorithms::shor (src/algorithms/shor.cpp): info = {success, factor1, factor2, a, period,
// attempts}; the counts of the successful round as (register, count).
int lqcsref_shor(uint64_t N, uint64_t shots, uint64_t max_attempts, int has_seed, uint64_t seed,
                 uint64_t* info, uint64_t* keys, uint64_t* counts, uint64_t cap,
                 uint64_t* n_out) {
    return guarded([&] {
        algorithms::ShorOptions o;
        o.shots = shots;
        o.max_attempts = max_attempts;
        if (has_seed) o.seed = seed;
        const algorithms::ShorResult r = algorithms::shor(N, o);
        info[0] = r.success ? 1 : 0;
        info[1] = r.factor1;
        info[2] = r.factor2;
        info[3] = r.a;
        info[4] = r.period;
        info[5] = r.attempts;
        Result res(r.counts, shots);
        write_counts(res, keys, counts, cap, n_out);
    });
}

// Draw `count` uniforms from lqcs::Rng(seed) (include/lqcs/core/random.hpp).
void lqcsref_uniforms(uint64_t seed, uint64_t count, double* out) {
    Rng rng(seed);
    for (uint64_t i = 0; i < count; ++i) out[i] = rng.uniform();
}

}  // extern "C"
