// capi.cpp — the extern "C" boundary (include/lqcs_b200.h).  Every entry point runs its
// body under `guarded`, which turns engine errors into status codes and keeps the message
// for lqcs_last_error().
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "costmodel.hpp"
#include "engine.hpp"

namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return LQCS_OK;
    } catch (const lqcs_b200::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "out of host memory";
        return LQCS_ERR_OUT_OF_MEMORY;
    } catch (const std::logic_error& e) {
        g_last_error = e.what();
        return LQCS_ERR_LOGIC;
    } catch (const std::runtime_error& e) {
        g_last_error = e.what();
        return LQCS_ERR_CUDA;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return LQCS_ERR_INTERNAL;
    } catch (...) {
        g_last_error = "unknown error";
        return LQCS_ERR_INTERNAL;
    }
}

void need(const void* p, const char* what) {
    if (p == nullptr) lqcs_b200::invalid(std::string(what) + " is null");
}

lqcs_b200::FusionConfig fusion_of(int32_t fuse, int32_t width, int32_t mode) {
    lqcs_b200::FusionConfig fc;
    fc.fuse = fuse != 0;
    if (width < 0 || width > lqcs_b200::kMaxDense) lqcs_b200::invalid("fusion width must be in [1, 6]");
    fc.max_width = static_cast<uint32_t>(width);
    fc.mode = mode;
    return fc;
}

}  // namespace

extern "C" {

const char* lqcs_last_error(void) { return g_last_error.c_str(); }

const char* lqcs_version(void) { return "lqcs_b200 0.1.0 sm_100a"; }

uint64_t lqcs_kernel_launch_count(void) { return lqcs_b200::launch_count(); }

int lqcs_debug_emulate_register_passes(uint32_t n_qubits, const lqcs_instruction* insts,
                                       uint64_t n_insts, uint64_t grid, int32_t sync_tiles,
                                       double* state, uint64_t race_ctas, uint64_t* n_passes,
                                       uint64_t* n_races, char* report, uint64_t report_cap) {
    return guarded([&] {
        need(n_passes, "n_passes");
        need(n_races, "n_races");
        if (n_qubits < lqcs_b200::kRegMinBits || n_qubits > 26)
            lqcs_b200::invalid("register tile emulation: n_qubits must be in [9, 26]");
        const int mode = sync_tiles & 7, drop = sync_tiles & 8;
        if (mode > 3 || (sync_tiles & ~15))
            lqcs_b200::invalid("register tile emulation: sync_tiles must be 0..3, optionally + 8");
        std::string first;
        lqcs_b200::emulate_register_program(n_qubits, insts, n_insts, grid, mode == 3 ? 1 : mode,
                                            mode == 3, drop != 0,
                                            reinterpret_cast<lqcs_b200::cd*>(state), race_ctas,
                                            n_passes, n_races, &first);
        if (report && report_cap) {
            const size_t k = std::min<size_t>(first.size(), report_cap - 1);
            std::memcpy(report, first.data(), k);
            report[k] = 0;
        }
    });
}

int lqcs_state_create(uint32_t n_qubits, void* stream, lqcs_state** out) {
    return guarded([&] {
        need(out, "out");
        auto st = lqcs_b200::new_state(n_qubits, 1, static_cast<cudaStream_t>(stream));
        st->sync();
        *out = st.release();
    });
}

int lqcs_state_create_batch(uint32_t n_qubits, uint32_t batch, void* stream, lqcs_state** out) {
    return guarded([&] {
        need(out, "out");
        auto st = lqcs_b200::new_state(n_qubits, batch, static_cast<cudaStream_t>(stream));
        st->sync();
        *out = st.release();
    });
}

int lqcs_state_destroy(lqcs_state* st) {
    return guarded([&] {
        if (!st) return;
        cudaStreamSynchronize(st->stream);
        delete st;
    });
}

int lqcs_state_num_qubits(const lqcs_state* st, uint32_t* out) {
    return guarded([&] {
        need(st, "state");
        need(out, "out");
        *out = st->n;
    });
}

int lqcs_state_device_ptr(const lqcs_state* st, void** out) {
    return guarded([&] {
        need(st, "state");
        need(out, "out");
        *out = st->amps.ptr;
    });
}

int lqcs_state_set_zero(lqcs_state* st) {
    return guarded([&] {
        need(st, "state");
        lqcs_b200::launch_set_basis(st->ctx, st->d(), st->n, st->batch, 0);
        st->sync();
    });
}

int lqcs_state_load(lqcs_state* st, const double* host_amps, uint64_t n_amps) {
    return guarded([&] {
        need(st, "state");
        need(host_amps, "host_amps");
        if (n_amps != st->len() && n_amps != st->len() * st->batch)
            lqcs_b200::invalid("state_load: amplitude count must be 2^n (or 2^n * batch)");
        lqcs_b200::cuda_check(cudaMemcpyAsync(st->amps.ptr, host_amps, n_amps * sizeof(double2),
                                              cudaMemcpyHostToDevice, st->stream),
                              "H2D amplitudes");
        st->sync();
    });
}

int lqcs_state_store(const lqcs_state* st, double* host_amps, uint64_t n_amps) {
    return guarded([&] {
        need(st, "state");
        need(host_amps, "host_amps");
        if (n_amps != st->len() && n_amps != st->len() * st->batch)
            lqcs_b200::invalid("state_store: amplitude count must be 2^n (or 2^n * batch)");
        lqcs_b200::cuda_check(cudaMemcpyAsync(host_amps, st->amps.ptr, n_amps * sizeof(double2),
                                              cudaMemcpyDeviceToHost, st->stream),
                              "D2H amplitudes");
        st->sync();
    });
}

int lqcs_state_apply(lqcs_state* st, const lqcs_instruction* insts, uint64_t n_insts,
                     int32_t fuse_gates, int32_t max_fusion_width, int32_t fusion_mode) {
    return guarded([&] {
        need(st, "state");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, st->n);
        lqcs_b200::apply_circuit(*st, gates, fusion_of(fuse_gates, max_fusion_width, fusion_mode));
    });
}

int lqcs_program_create(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                        int32_t fuse_gates, int32_t max_fusion_width, int32_t fusion_mode,
                        lqcs_program** out) {
    return guarded([&] {
        need(out, "out");
        if (n_qubits == 0) lqcs_b200::invalid("QuantumCircuit: num_qubits must be >= 1");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, n_qubits);
        *out = lqcs_b200::program_create(n_qubits, gates,
                                         fusion_of(fuse_gates, max_fusion_width, fusion_mode))
                   .release();
    });
}

int lqcs_program_destroy(lqcs_program* prog) {
    return guarded([&] { delete prog; });
}

int lqcs_program_info(const lqcs_program* prog, uint64_t* n_ops, uint64_t* n_gates) {
    return guarded([&] {
        need(prog, "program");
        if (n_ops) *n_ops = prog->prog.ops.size();
        if (n_gates) *n_gates = prog->prog.source_gates;
    });
}

int lqcs_program_apply(lqcs_state* st, const lqcs_program* prog) {
    return guarded([&] {
        need(st, "state");
        need(prog, "program");
        if (prog->n != st->n) lqcs_b200::invalid("program_apply: qubit count mismatch");
        prog->prog.launch(st->ctx, st->d(), st->n, st->batch);
        st->sync();
    });
}

int lqcs_program_apply_profiled(lqcs_state* st, const lqcs_program* prog, uint64_t cap,
                                lqcs_op_profile* out, uint64_t* n_out) {
    return guarded([&] {
        need(st, "state");
        need(prog, "program");
        need(n_out, "n_out");
        if (prog->n != st->n) lqcs_b200::invalid("program_apply: qubit count mismatch");
        lqcs_b200::program_profile(*st, *prog, cap, out, n_out);
    });
}

int lqcs_run_statevector(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                         const lqcs_sim_options* opts, void* stream, lqcs_state** out) {
    return guarded([&] {
        need(out, "out");
        if (opts && opts->n_channels > 0) {
            lqcs_b200::invalid(
                "run_statevector: noisy simulation is stochastic (one trajectory is not the "
                "quantum state); use run() or DensityMatrixSimulator");
        }
        if (n_qubits == 0) lqcs_b200::invalid("QuantumCircuit: num_qubits must be >= 1");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, n_qubits);
        auto st = lqcs_b200::new_state(n_qubits, 1, static_cast<cudaStream_t>(stream));
        const int32_t fuse = opts ? opts->fuse_gates : 1;
        const int32_t width = opts ? opts->max_fusion_width : 0;
        const int32_t mode = opts ? opts->fusion_mode : 0;
        lqcs_b200::apply_circuit(*st, gates, fusion_of(fuse, width, mode));
        *out = st.release();
    });
}

int lqcs_run(uint32_t n_qubits, uint32_t n_clbits, const lqcs_instruction* insts,
             uint64_t n_insts, uint64_t shots, const lqcs_sim_options* opts,
             uint64_t* shot_registers) {
    return guarded([&] {
        if (n_qubits == 0) lqcs_b200::invalid("QuantumCircuit: num_qubits must be >= 1");
        if (shots > 0) need(shot_registers, "shot_registers");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, n_qubits);
        lqcs_b200::run_shots(n_qubits, n_clbits, gates, shots, opts, shot_registers);
    });
}

int lqcs_dm_create(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                   const lqcs_sim_options* opts, lqcs_state** out) {
    return guarded([&] {
        need(out, "out");
        *out = nullptr;
        if (n_qubits == 0) lqcs_b200::invalid("DensityMatrix: num_qubits must be >= 1");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, n_qubits);
        *out = lqcs_b200::dm_evolve(n_qubits, gates, opts).release();
    });
}

int lqcs_dm_probabilities(const lqcs_state* rho, double* probs) {
    return guarded([&] {
        need(rho, "rho");
        need(probs, "probs");
        if (rho->n % 2 != 0 || rho->batch != 1) lqcs_b200::invalid("dm_probabilities: not a density matrix");
        lqcs_b200::dm_probabilities(const_cast<lqcs_state&>(*rho), rho->n / 2, probs);
    });
}

int lqcs_dm_run(uint32_t n_qubits, uint32_t n_clbits, const lqcs_instruction* insts,
                uint64_t n_insts, uint64_t shots, const lqcs_sim_options* opts,
                uint64_t* shot_registers) {
    return guarded([&] {
        if (n_qubits == 0) lqcs_b200::invalid("QuantumCircuit: num_qubits must be >= 1");
        if (shots > 0) need(shot_registers, "shot_registers");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, n_qubits);
        lqcs_b200::dm_run_shots(n_qubits, n_clbits, gates, shots, opts, shot_registers);
    });
}

int lqcs_state_read_range(const lqcs_state* st, uint64_t first, uint64_t count, double* host) {
    return guarded([&] {
        need(st, "state");
        if (count == 0) return;
        need(host, "host");
        if (first >= st->len() * st->batch || count > st->len() * st->batch - first)
            lqcs_b200::out_of_range("state_read_range: index out of range");
        lqcs_b200::cuda_check(cudaMemcpyAsync(host, st->d() + first, count * sizeof(double2),
                                              cudaMemcpyDeviceToHost, st->stream),
                              "D2H amplitudes");
        st->sync();
    });
}

int lqcs_gate_matrix(const lqcs_instruction* inst, int32_t with_controls, double* out,
                     uint64_t cap_doubles, uint64_t* dim_out) {
    return guarded([&] {
        need(inst, "instruction");
        need(dim_out, "dim_out");
        uint32_t max_q = 0;
        for (uint32_t i = 0; i < inst->n_qubits; ++i) max_q = std::max(max_q, inst->qubits[i] + 1);
        const lqcs_b200::GateDesc g = lqcs_b200::decode(*inst, std::max<uint32_t>(max_q, 1));
        const std::vector<lqcs_b200::cd> m = with_controls ? g.full_matrix() : g.base_matrix();
        uint64_t dim = 1;
        while (dim * dim < m.size()) dim <<= 1;
        *dim_out = dim;
        if (out == nullptr) return;
        if (cap_doubles < 2 * m.size()) lqcs_b200::invalid("gate_matrix: output buffer too small");
        for (size_t i = 0; i < m.size(); ++i) {
            out[2 * i] = m[i].real();
            out[2 * i + 1] = m[i].imag();
        }
    });
}

int lqcs_state_probabilities(const lqcs_state* st, double* host_out) {
    return guarded([&] {
        need(st, "state");
        need(host_out, "host_out");
        lqcs_b200::DeviceBuffer p;
        p.ensure(sizeof(double) * st->len());
        lqcs_b200::launch_probabilities(st->ctx, st->d(), st->n, p.as<double>());
        lqcs_b200::cuda_check(cudaMemcpyAsync(host_out, p.ptr, sizeof(double) * st->len(),
                                              cudaMemcpyDeviceToHost, st->stream),
                              "D2H probabilities");
        st->sync();
    });
}

int lqcs_state_norm(const lqcs_state* st, double* out) {
    return guarded([&] {
        need(st, "state");
        need(out, "out");
        *out = std::sqrt(lqcs_b200::state_norm2(*const_cast<lqcs_state*>(st)));
    });
}

int lqcs_state_sample(const lqcs_state* st, const double* uniforms, uint64_t shots,
                      uint64_t* idx_out, double* min_margin) {
    return guarded([&] {
        need(st, "state");
        if (shots > 0) {
            need(uniforms, "uniforms");
            need(idx_out, "idx_out");
        }
        lqcs_b200::sample(*const_cast<lqcs_state*>(st), uniforms, shots, idx_out, min_margin);
    });
}

int lqcs_state_expectation_pauli(const lqcs_state* st, const char* pauli, double* out) {
    return guarded([&] {
        need(st, "state");
        need(out, "out");
        const auto m = lqcs_b200::pauli_global_masks(pauli, st->n, "expectation_value");
        *out = lqcs_b200::expectation_terms(*const_cast<lqcs_state*>(st), {m})[0];
    });
}

int lqcs_state_expectation_terms(const lqcs_state* st, const char* const* paulis,
                                 const double* coeffs, uint64_t n_terms, double* per_term,
                                 double* total) {
    return guarded([&] {
        need(st, "state");
        if (n_terms > 0) {
            need(paulis, "paulis");
            need(coeffs, "coeffs");
        }
        std::vector<lqcs_b200::PauliMasks> terms;
        for (uint64_t t = 0; t < n_terms; ++t)
            terms.push_back(lqcs_b200::pauli_global_masks(paulis[t], st->n, "expectation_value"));
        const auto v = lqcs_b200::expectation_terms(*const_cast<lqcs_state*>(st), terms);
        double e = 0.0;
        for (uint64_t t = 0; t < n_terms; ++t) {
            if (per_term) per_term[t] = v[t];
            e += coeffs[t] * v[t];
        }
        if (total) *total = e;
    });
}

int lqcs_expectation_terms_noalloc(const void* d_amps, uint32_t n_qubits,
                                   const char* const* paulis, uint64_t n_terms,
                                   double* host_values, void* stream) {
    return guarded([&] {
        lqcs_b200::expectation_terms_static(d_amps, n_qubits, paulis, n_terms, host_values,
                                            static_cast<cudaStream_t>(stream));
    });
}

int lqcs_state_collapse(lqcs_state* st, uint32_t qubit, double uniform, int32_t* outcome) {
    return guarded([&] {
        need(st, "state");
        const int o = lqcs_b200::collapse(*st, qubit, uniform);
        st->sync();
        if (outcome) *outcome = o;
    });
}

int lqcs_state_reset_qubit(lqcs_state* st, uint32_t qubit, double uniform) {
    return guarded([&] {
        need(st, "state");
        if (qubit >= st->n) lqcs_b200::out_of_range("reset: qubit index out of range");
        lqcs_b200::reset_qubit(*st, qubit, uniform);
        st->sync();
    });
}

int lqcs_state_kraus_probability(const lqcs_state* st, uint32_t qubit, const double* k,
                                 double* out) {
    return guarded([&] {
        need(st, "state");
        need(k, "k");
        need(out, "out");
        const std::array<lqcs_b200::cd, 4> kk{lqcs_b200::cd{k[0], k[1]}, lqcs_b200::cd{k[2], k[3]},
                                              lqcs_b200::cd{k[4], k[5]}, lqcs_b200::cd{k[6], k[7]}};
        *out = lqcs_b200::kraus_probability(*const_cast<lqcs_state*>(st), qubit, kk);
    });
}

int lqcs_parameter_shift_gradient(const lqcs_parametric_circuit* pc, const lqcs_hamiltonian* h,
                                  const double* params, double* grad_out) {
    return guarded([&] {
        need(pc, "parametric circuit");
        if (pc->n_params > 0) {
            need(params, "params");
            need(grad_out, "grad_out");
        }
        const auto ham = lqcs_b200::decode_hamiltonian(h, pc->n_qubits);
        lqcs_b200::parameter_shift(pc, ham, params, grad_out);
    });
}

int lqcs_adjoint_gradient(const lqcs_parametric_circuit* pc, const lqcs_hamiltonian* h,
                          const double* params, uint64_t batch, uint32_t max_resident,
                          double* energy_out, double* grad_out) {
    return guarded([&] {
        need(pc, "parametric circuit");
        const auto ham = lqcs_b200::decode_hamiltonian(h, pc->n_qubits);
        lqcs_b200::adjoint_batched(pc, ham, params, batch, max_resident, energy_out, grad_out);
    });
}

int lqcs_adjoint_gradient_multi(uint64_t n_problems, const lqcs_parametric_circuit* const* pcs,
                                const lqcs_hamiltonian* const* hs, const double* const* params,
                                const uint64_t* batches, double* const* energy_out,
                                double* const* grad_out) {
    return guarded([&] {
        lqcs_b200::adjoint_batched_multi(n_problems, pcs, hs, params, batches, energy_out, grad_out);
    });
}

int lqcs_release_caches(void) {
    return guarded([&] {
        lqcs_b200::release_adjoint_plans();
        lqcs_b200::clear_autotune_cache();
        lqcs_b200::clear_program_cache();
        lqcs_b200::clear_state_pool();
        lqcs_b200::forget_static_scratch_addresses();
    });
}

int lqcs_batched_energy(const lqcs_parametric_circuit* pc, const lqcs_hamiltonian* h,
                        const double* params, uint64_t batch, uint32_t max_resident,
                        double* energy_out) {
    return guarded([&] {
        need(pc, "parametric circuit");
        need(energy_out, "energy_out");
        const auto ham = lqcs_b200::decode_hamiltonian(h, pc->n_qubits);
        lqcs_b200::adjoint_batched(pc, ham, params, batch, max_resident, energy_out, nullptr);
    });
}

int lqcs_costmodel_features(uint32_t kind, uint32_t width, uint32_t min_target,
                            uint32_t max_target, uint32_t n_gates, uint32_t n_qubits,
                            double flops_per_amp, float* out) {
    return guarded([&] {
        need(out, "out");
        const auto f = lqcs_b200::op_features(kind, width, min_target, max_target, n_gates, n_qubits,
                                              flops_per_amp);
        for (int i = 0; i < lqcs_b200::kCostFeatures; ++i) out[i] = f[i];
    });
}

int lqcs_costmodel_train(const float* features, const float* targets, uint64_t n,
                         uint32_t epochs, float learning_rate, uint64_t seed, float* loss_out) {
    return guarded([&] {
        need(features, "features");
        need(targets, "targets");
        const float loss = lqcs_b200::costmodel_train(features, targets, n, epochs, learning_rate, seed);
        if (loss_out) *loss_out = loss;
    });
}

int lqcs_costmodel_predict(const float* features, uint64_t n, float* out) {
    return guarded([&] {
        if (n > 0) {
            need(features, "features");
            need(out, "out");
        }
        lqcs_b200::costmodel_predict(features, n, out);
    });
}

int lqcs_costmodel_grad(const float* features, const float* targets, uint64_t n,
                        float* loss_out, float* grad_out, uint64_t grad_cap,
                        uint64_t* n_params_out) {
    return guarded([&] {
        need(features, "features");
        need(targets, "targets");
        if (n_params_out) *n_params_out = lqcs_b200::kCostParams;
        if (grad_cap < static_cast<uint64_t>(lqcs_b200::kCostParams))
            lqcs_b200::invalid("costmodel_grad: gradient buffer too small");
        need(grad_out, "grad_out");
        const float loss = lqcs_b200::costmodel_grad(features, targets, n, grad_out);
        if (loss_out) *loss_out = loss;
    });
}

int lqcs_costmodel_get_weights(float* out, uint64_t cap, uint64_t* n_out) {
    return guarded([&] {
        const std::vector<float> w = lqcs_b200::costmodel_weights();
        if (n_out) *n_out = w.size();
        if (out == nullptr) return;
        if (cap < w.size()) lqcs_b200::invalid("costmodel_get_weights: buffer too small");
        std::copy(w.begin(), w.end(), out);
    });
}

int lqcs_costmodel_set_weights(const float* w, uint64_t n) {
    return guarded([&] {
        need(w, "weights");
        lqcs_b200::costmodel_set_weights(w, n);
    });
}

int lqcs_costmodel_clear(void) {
    return guarded([&] { lqcs_b200::costmodel_clear(); });
}

int lqcs_costmodel_plan_ms(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                           int32_t max_fusion_width, int32_t fusion_mode, double* ms_out) {
    return guarded([&] {
        need(ms_out, "ms_out");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, n_qubits);
        auto prog = lqcs_b200::program_create(n_qubits, gates,
                                              fusion_of(1, max_fusion_width, fusion_mode));
        *ms_out = lqcs_b200::predict_ops_ms(prog->prog.ops, n_qubits);
    });
}

int lqcs_rng_uniforms(uint64_t seed, uint64_t count, double* out) {
    return guarded([&] {
        if (count > 0) need(out, "out");
        lqcs_b200::Rng rng(seed);
        for (uint64_t i = 0; i < count; ++i) out[i] = lqcs_b200::rng_uniform(rng);
    });
}

int lqcs_rng_u64(uint64_t seed, uint64_t skip, uint64_t count, uint64_t* out) {
    return guarded([&] {
        if (count > 0) need(out, "out");
        lqcs_b200::Rng rng(seed);
        rng.discard(skip);
        for (uint64_t i = 0; i < count; ++i) out[i] = rng();
    });
}

int lqcs_fusion_plan(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                     int32_t max_fusion_width, int32_t fusion_mode, uint64_t cap,
                     uint32_t* block_width, uint32_t* block_gates, uint64_t* n_blocks) {
    return guarded([&] {
        need(n_blocks, "n_blocks");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, n_qubits);
        if (fusion_mode == lqcs_b200::kFuseTile) {
            // passes: width = number of high tile qubits, gates = gates applied by the pass
            const auto items = lqcs_b200::plan_tiles(gates, n_qubits,
                                                     lqcs_b200::default_tile_config(n_qubits));
            *n_blocks = items.size();
            for (uint64_t i = 0; i < items.size() && i < cap; ++i) {
                const bool pass = items[i].is_pass;
                if (block_width)
                    block_width[i] = pass ? static_cast<uint32_t>(items[i].hbits.size())
                                          : gates[items[i].gate].base_qubits();
                if (block_gates) block_gates[i] = pass ? static_cast<uint32_t>(items[i].gates.size()) : 1;
            }
            return;
        }
        const auto p = lqcs_b200::plan(gates, n_qubits, fusion_of(1, max_fusion_width, fusion_mode));
        *n_blocks = p.size();
        for (uint64_t i = 0; i < p.size() && i < cap; ++i) {
            if (block_width) block_width[i] = static_cast<uint32_t>(p[i].qubits.size());
            if (block_gates) block_gates[i] = static_cast<uint32_t>(p[i].gates.size());
        }
    });
}

int lqcs_autotune(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                  uint64_t cap, lqcs_tune_entry* out, uint64_t* n_out) {
    return guarded([&] {
        need(n_out, "n_out");
        const auto gates = lqcs_b200::decode_all(insts, n_insts, n_qubits);
        size_t best = 0;
        const auto t = lqcs_b200::autotune(gates, n_qubits, &best);
        *n_out = t.size();
        for (size_t i = 0; i < t.size() && i < cap && out; ++i) {
            lqcs_tune_entry& e = out[i];
            e = lqcs_tune_entry{};
            e.planner = t[i].cand.planner;
            e.tile_bits = t[i].cand.planner == 2 ? 0 : t[i].cand.cfg.m;
            e.tile_low = t[i].cand.planner == 2 ? 0 : t[i].cand.cfg.L;
            e.inner = t[i].cand.planner == 2 ? 0 : t[i].cand.cfg.inner;
            e.width = t[i].cand.width;
            e.chosen = i == best ? 1u : 0u;
            e.n_ops = t[i].n_ops;
            e.device_ms = t[i].ms;
        }
    });
}

}  // extern "C"
