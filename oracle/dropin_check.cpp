// dropin_check.cpp — ORACLE (test infrastructure only).
//
// Builds circuits with the reference's own API (lqcs::QuantumCircuit, algorithms::qft,
// NoiseModel), runs them through the reference's StatevectorSimulator and through
// lqcs_b200::CudaStatevectorSimulator (include/lqcs_b200_backend.hpp), and compares:
// amplitudes within 1e-12, counts identical for the same seed, error types identical.
// Prints one JSON line and exits non-zero on any mismatch.  Built by oracle/Makefile into
// oracle/_ref/dropin_check against the reference library and the engine library.
#include <cmath>
#include <cstdio>
#include <random>
#include <string>

#include <lqcs/lqcs.hpp>

#include "lqcs_b200_backend.hpp"

using namespace lqcs;

namespace {

int failures = 0;

void check(bool ok, const std::string& what) {
    if (!ok) {
        ++failures;
        std::fprintf(stderr, "MISMATCH: %s\n", what.c_str());
    }
}

QuantumCircuit brick(std::size_t n, std::size_t depth, std::uint64_t seed, bool measure) {
    std::mt19937_64 eng(seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    QuantumCircuit qc(n, measure ? n : 0);
    for (std::size_t l = 0; l < depth; ++l) {
        for (qubit_t q = 0; q < n; ++q) qc.u(6.283 * u(eng), 6.283 * u(eng), 6.283 * u(eng), q);
        std::vector<qubit_t> order(n);
        for (qubit_t q = 0; q < n; ++q) order[q] = q;
        std::shuffle(order.begin(), order.end(), eng);
        for (std::size_t k = 0; k + 1 < n; k += 2) qc.cx(order[k], order[k + 1]);
    }
    qc.rp(0.4, "XYZ", {0, 1, 2}).ccx(0, 1, 2).swap(1, n - 1).iswap(0, 2).rzz(0.3, 1, 2);
    if (measure) qc.measure_all();
    return qc;
}

double max_diff(const Statevector& a, const Statevector& b) {
    double m = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i) m = std::max(m, std::abs(a[i] - b[i]));
    return m;
}

}  // namespace

int main() {
    double worst = 0.0;
    for (std::size_t n : {3, 8, 12, 16}) {
        const QuantumCircuit qc = brick(n, 6, 100 + n, false);
        for (bool fuse : {false, true}) {
            StatevectorSimulator ref({.fuse_gates = fuse});
            lqcs_b200::CudaStatevectorSimulator gpu({.fuse_gates = fuse});
            const double d = max_diff(ref.run_statevector(qc), gpu.run_statevector(qc));
            worst = std::max(worst, d);
            check(d < 1e-12, "amplitudes n=" + std::to_string(n));
        }
    }
    {
        QuantumCircuit qft(10);
        qft.x(3).x(7).compose(algorithms::qft(10));
        const double d = max_diff(StatevectorSimulator().run_statevector(qft),
                                  lqcs_b200::CudaStatevectorSimulator().run_statevector(qft));
        worst = std::max(worst, d);
        check(d < 1e-12, "qft");
    }
    for (std::uint64_t seed : {1ull, 42ull, 2024ull}) {
        const QuantumCircuit qc = brick(10, 5, seed, true);
        const auto a = StatevectorSimulator({.seed = seed}).run(qc, 4096).counts();
        const auto b = lqcs_b200::CudaStatevectorSimulator({.seed = seed}).run(qc, 4096).counts();
        check(a == b, "counts seed " + std::to_string(seed));
    }
    {
        QuantumCircuit qc(2, 2);
        qc.h(0).measure(0, 0).cx(0, 1).reset(1).h(1).measure(1, 1);
        check(StatevectorSimulator({.seed = 5}).run(qc, 500).counts() ==
                  lqcs_b200::CudaStatevectorSimulator({.seed = 5}).run(qc, 500).counts(),
              "mid-circuit counts");
        NoiseModel noise;
        noise.add_all_qubit_channel(KrausChannel::depolarizing(0.1));
        noise.add_all_qubit_channel(KrausChannel::amplitude_damping(0.05));
        QuantumCircuit nq(3, 3);
        nq.h(0).cx(0, 1).cx(1, 2).measure_all();
        check(StatevectorSimulator({.seed = 8, .noise = noise}).run(nq, 300).counts() ==
                  lqcs_b200::CudaStatevectorSimulator({.seed = 8, .noise = noise}).run(nq, 300).counts(),
              "trajectory counts");
    }
    {
        int same = 0;
        QuantumCircuit qc(2);
        qc.h(0);
        try { lqcs_b200::CudaStatevectorSimulator().run(qc, 10); } catch (const std::invalid_argument&) { ++same; }
        try { lqcs_b200::CudaStatevectorSimulator().run(qc, 0); } catch (const std::invalid_argument&) { ++same; }
        check(same == 2, "exception types");
    }
    std::printf("{\"dropin_failures\": %d, \"max_amp_diff\": %.3e}\n", failures, worst);
    return failures == 0 ? 0 : 1;
}
