// dm.cpp — the density-matrix backend on the device.
//
// DensityMatrixSimulator (src/backend/density_matrix_simulator.cpp, density_matrix.cpp)
// keeps rho of n qubits as a vector of 2n qubits: element rho_{rc} at (c << n) | r, so the
// ket (row) bits are the circuit's qubits and the bra (column) bits are qubits + n.  A gate
// U on qubits Q is U on Q and conj(U) on Q + n (rho -> U rho U^dagger); a one-qubit channel
// {K_i} on q is the 4x4 superoperator S = sum_i K_i (x) conj(K_i) on (q, q + n).  Here that
// 2n-qubit gate list is compiled like any circuit — fused into register tile passes — and
// run on a 2n-qubit device state; probabilities are the diagonal rho_ii, and shots sample
// it with the statevector path's prefix sum and upper_bound rule.
#include <algorithm>
#include <cmath>

#include "engine.hpp"

namespace lqcs_b200 {

namespace {

using Kraus = std::array<cd, 4>;

// The bra-side copy of a unitary gate: conj(U) on qubits + n.  Permutations are real;
// exp(-i theta/2 P)* = exp(-i theta'/2 P) with theta' = theta for an odd number of Y
// factors (P* = -P) and -theta otherwise; every other gate becomes its conjugated matrix.
GateDesc bra_gate(const GateDesc& g, uint32_t n) {
    GateDesc b = g;
    for (uint32_t& q : b.qubits) q += n;
    if (g.type == LQCS_GATE_PERMUTATION) return b;
    if (g.type == LQCS_GATE_PAULI_ROTATION) {
        const PauliMasks m = pauli_local_masks(g.pauli);
        if (m.n_y % 2 == 0) b.params[0] = -g.params[0];
        return b;
    }
    std::vector<cd> mat = g.base_matrix();
    for (cd& z : mat) z = std::conj(z);
    b.type = LQCS_GATE_UNITARY;
    b.params.clear();
    b.mat = std::move(mat);
    return b;
}

// sum_i K_i (x) conj(K_i) on (q, q + n): local bit 0 is the ket bit, bit 1 the bra bit.
GateDesc superoperator(const std::vector<Kraus>& ops, uint32_t q, uint32_t n) {
    GateDesc g;
    g.type = LQCS_GATE_UNITARY;
    g.qubits = {q, q + n};
    g.mat.assign(16, cd{0, 0});
    for (const Kraus& k : ops)
        for (uint32_t ro = 0; ro < 2; ++ro)
            for (uint32_t bo = 0; bo < 2; ++bo)
                for (uint32_t ri = 0; ri < 2; ++ri)
                    for (uint32_t bi = 0; bi < 2; ++bi)
                        g.mat[(ro | bo << 1) * 4 + (ri | bi << 1)] +=
                            k[ro * 2 + ri] * std::conj(k[bo * 2 + bi]);
    return g;
}

}  // namespace

std::vector<GateDesc> dm_gates(const std::vector<GateDesc>& gates, uint32_t n,
                               const std::vector<std::vector<Kraus>>& noise) {
    std::vector<GateDesc> out;
    for (const GateDesc& g : gates) {
        if (g.type == LQCS_GATE_RESET) invalid("DensityMatrixSimulator: Reset is not supported yet");
        if (g.type == LQCS_GATE_KRAUS) {   // explicit channel (engine extension) where it stands
            out.push_back(superoperator(std::vector<Kraus>(g.kraus.begin(), g.kraus.end()),
                                        g.qubits[0], n));
            continue;
        }
        if (!g.is_unitary()) continue;   // Measure / Barrier
        out.push_back(g);
        out.push_back(bra_gate(g, n));
        for (const auto& ch : noise)
            for (uint32_t q : g.qubits) out.push_back(superoperator(ch, q, n));
    }
    return out;
}

std::unique_ptr<lqcs_state> dm_evolve(uint32_t n, const std::vector<GateDesc>& gates,
                                      const lqcs_sim_options* opts) {
    if (n == 0) invalid("DensityMatrix: num_qubits must be >= 1");
    if (2 * n > static_cast<uint32_t>(kMaxQubits)) invalid("DensityMatrix: too many qubits");
    std::vector<std::vector<Kraus>> noise;
    for (const auto& c : decode_channels(opts)) noise.emplace_back(c.begin(), c.end());
    const std::vector<GateDesc> g2 = dm_gates(gates, n, noise);
    auto st = new_state(2 * n, 1, nullptr);   // vec(|0><0|) = e_0
    FusionConfig fc;
    if (opts) {
        fc.max_width = static_cast<uint32_t>(std::max(0, opts->max_fusion_width));
        fc.mode = opts->fusion_mode;
    }
    apply_circuit(*st, g2, fc);
    return st;
}

void dm_probabilities(lqcs_state& rho, uint32_t n, double* host) {
    DeviceBuffer p;
    p.ensure(sizeof(double) << n);
    launch_dm_diagonal(rho.ctx, rho.d(), n, p.as<double>());
    cuda_check(cudaMemcpyAsync(host, p.ptr, sizeof(double) << n, cudaMemcpyDeviceToHost,
                               rho.stream),
               "D2H probabilities");
    rho.sync();
}

void dm_run_shots(uint32_t n, uint32_t n_clbits, const std::vector<GateDesc>& gates,
                  uint64_t shots, const lqcs_sim_options* opts, uint64_t* regs) {
    if (shots == 0) invalid("run: shots must be >= 1");
    if (n_clbits > 64) invalid("run: this engine reports at most 64 classical bits");
    // terminal measurements only (density_matrix_simulator.cpp:32-46)
    bool seen_measure = false;
    std::vector<int64_t> src(n_clbits, -1);
    for (const GateDesc& g : gates) {
        if (g.type == LQCS_GATE_MEASURE) {
            if (g.clbit >= n_clbits) {
                out_of_range("clbit index " + std::to_string(g.clbit) +
                             " out of range (num_clbits = " + std::to_string(n_clbits) + ")");
            }
            seen_measure = true;
            src[g.clbit] = g.qubits[0];
        } else if (seen_measure && (g.is_unitary() || g.type == LQCS_GATE_KRAUS)) {
            invalid("DensityMatrixSimulator: mid-circuit measurement is not supported");
        }
    }
    if (!seen_measure) invalid("run: circuit has no measurements; use run_density_matrix()");
    auto rho = dm_evolve(n, gates, opts);
    Rng rng = make_rng(opts);
    const uint64_t len = uint64_t{1} << n;
    DeviceBuffer tpref, seg, du, didx, dmargin;
    tpref.ensure(sizeof(double) * scan_thread_count(n));
    seg.ensure(sizeof(double) * (scan_block_count(n) + 1));
    launch_dm_diag_scan(rho->ctx, rho->d(), n, tpref.as<double>(), seg.as<double>());
    std::vector<double> u(shots);
    if (opts && opts->shot_offset) rng.discard(opts->shot_offset);   // one uniform per shot
    for (uint64_t s = 0; s < shots; ++s) u[s] = rng_uniform(rng);
    du.ensure(sizeof(double) * shots);
    didx.ensure(sizeof(uint64_t) * shots);
    dmargin.ensure(sizeof(double) * shots);
    cuda_check(cudaMemcpyAsync(du.ptr, u.data(), sizeof(double) * shots, cudaMemcpyHostToDevice,
                               rho->stream),
               "H2D uniforms");
    launch_dm_sample_search(rho->ctx, rho->d(), n, tpref.as<double>(), seg.as<double>(),
                            du.as<double>(), shots, didx.as<uint64_t>(), dmargin.as<double>());
    std::vector<uint64_t> idx(shots);
    cuda_check(cudaMemcpyAsync(idx.data(), didx.ptr, sizeof(uint64_t) * shots,
                               cudaMemcpyDeviceToHost, rho->stream),
               "D2H sample indices");
    rho->sync();
    for (uint64_t s = 0; s < shots; ++s) {
        uint64_t reg = 0;
        for (uint32_t c = 0; c < n_clbits; ++c)
            if (src[c] >= 0 && ((idx[s] >> src[c]) & 1u)) reg |= uint64_t{1} << c;
        regs[s] = reg;
    }
}

}  // namespace lqcs_b200
