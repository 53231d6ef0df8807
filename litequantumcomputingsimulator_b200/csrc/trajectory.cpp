// trajectory.cpp — per-shot evolution with many shots resident on the device.
//
// Semantics of run_per_shot (src/backend/statevector_simulator.cpp:156-190): every shot
// starts from |0...0>; a Measure collapses with one uniform; a Reset collapses and moves a
// |1> back to |0> with one uniform; after every unitary instruction each channel of the
// noise model samples one branch per touched qubit (channel-major order, one uniform
// each, statevector_simulator.cpp:146-153); an explicit Kraus instruction samples one
// branch.  The number of uniforms per shot is therefore fixed by the circuit, and shot s
// consumes draws [s*K, (s+1)*K) of the single seeded stream — the reference's order.
// All uniforms are drawn up front and uploaded; a batch of R shots then runs without any
// host synchronisation until its registers are read back.
#include <algorithm>
#include <cmath>

#include "engine.hpp"
#include "traj.cuh"

namespace lqcs_b200 {

namespace {

using Kraus = std::array<cd, 4>;
using Channel = std::vector<Kraus>;

enum ItemKind { kUnitary, kMeasure, kReset, kKrausTable, kKrausGeneral };

struct Item {
    ItemKind kind;
    size_t prog = 0;          // kUnitary
    uint32_t q = 0;
    uint32_t clbit = 0;
    uint32_t uidx = 0;        // index of the event's uniform within a shot
    size_t channel = 0;       // index into the channel list
};

// Every operator proportional to a unitary (K^dagger K = |c|^2 I): the branch probabilities
// |c_i|^2 ||psi||^2 do not depend on the state, and ||psi|| = 1 up to rounding.
bool unitary_mixture(const Channel& ch, std::vector<double>& weights) {
    weights.clear();
    for (const Kraus& k : ch) {
        const cd a = std::conj(k[0]) * k[0] + std::conj(k[2]) * k[2];
        const cd d = std::conj(k[1]) * k[1] + std::conj(k[3]) * k[3];
        const cd off = std::conj(k[0]) * k[1] + std::conj(k[2]) * k[3];
        if (std::abs(a - d) > 1e-14 * std::max(1.0, std::abs(a)) || std::abs(off) > 1e-14) return false;
        weights.push_back(a.real());
    }
    return true;
}

bool is_identity_scaled(const Kraus& m) {
    constexpr double tol = 1e-14;
    return std::abs(m[1]) < tol && std::abs(m[2]) < tol && std::abs(m[0] - cd{1, 0}) < tol &&
           std::abs(m[3] - cd{1, 0}) < tol;
}

}  // namespace

void run_per_shot_batched(uint32_t n, const std::vector<GateDesc>& gates, uint64_t shots,
                          const std::vector<Channel>& model, const FusionConfig& fc_in, Rng& rng,
                          uint32_t max_resident, uint64_t* regs) {
    const bool noisy = !model.empty();
    FusionConfig fc = fc_in;
    if (noisy) fc.fuse = false;

    // ---- events in program order
    std::vector<Channel> channels = model;   // explicit Kraus instructions appended below
    std::vector<Item> items;
    std::vector<GateDesc> stretch;
    std::vector<std::vector<GateDesc>> stretches;
    uint32_t K = 0;
    auto flush = [&]() {
        if (stretch.empty()) return;
        stretches.push_back(stretch);
        Item it{kUnitary};
        it.prog = stretches.size() - 1;
        items.push_back(it);
        stretch.clear();
    };
    for (const GateDesc& g : gates) {
        if (g.type == LQCS_GATE_BARRIER) continue;
        if (g.type == LQCS_GATE_MEASURE || g.type == LQCS_GATE_RESET) {
            flush();
            Item it{g.type == LQCS_GATE_MEASURE ? kMeasure : kReset};
            it.q = g.qubits[0];
            it.clbit = g.clbit;
            it.uidx = K++;
            items.push_back(it);
            continue;
        }
        if (g.type == LQCS_GATE_KRAUS) {
            flush();
            channels.emplace_back(g.kraus.begin(), g.kraus.end());
            Item it{kKrausGeneral};
            it.q = g.qubits[0];
            it.channel = channels.size() - 1;
            it.uidx = K++;
            items.push_back(it);
            continue;
        }
        stretch.push_back(g);
        if (noisy) {
            flush();
            for (size_t c = 0; c < model.size(); ++c) {
                for (uint32_t q : g.qubits) {
                    Item it{kKrausGeneral};
                    it.q = q;
                    it.channel = c;
                    it.uidx = K++;
                    items.push_back(it);
                }
            }
        }
    }
    flush();

    // ---- uniforms, in the reference's consumption order
    std::vector<double> u(static_cast<size_t>(shots) * K);
    for (double& v : u) v = rng_uniform(rng);

    // ---- channels: unitary mixtures get a per-shot branch table chosen here
    struct ChanDev {
        bool table = false;
        std::vector<int> unused;
        DeviceBuffer ops;        // general: raw operators; table: normalised operators
        std::vector<Kraus> norm;
        std::vector<double> weights;
    };
    std::vector<ChanDev> cdev(channels.size());
    for (size_t c = 0; c < channels.size(); ++c) {
        ChanDev& d = cdev[c];
        d.table = unitary_mixture(channels[c], d.weights);
        std::vector<double2> buf;
        if (d.table) {
            for (size_t i = 0; i < channels[c].size(); ++i) {
                const double inv = d.weights[i] > 0 ? 1.0 / std::sqrt(d.weights[i]) : 0.0;
                Kraus m{};
                for (int e = 0; e < 4; ++e) m[e] = channels[c][i][e] * inv;
                d.norm.push_back(m);
                for (int e = 0; e < 4; ++e) buf.push_back(make_double2(m[e].real(), m[e].imag()));
            }
        } else {
            for (const Kraus& k : channels[c])
                for (int e = 0; e < 4; ++e) buf.push_back(make_double2(k[e].real(), k[e].imag()));
        }
        d.ops.ensure(sizeof(double2) * buf.size());
        cuda_check(cudaMemcpy(d.ops.ptr, buf.data(), sizeof(double2) * buf.size(),
                              cudaMemcpyHostToDevice), "H2D Kraus operators");
    }
    // per table item: branch per shot (-1 = identity, nothing to apply)
    std::vector<DeviceBuffer> choice(items.size());
    for (size_t i = 0; i < items.size(); ++i) {
        Item& it = items[i];
        if (it.kind != kKrausGeneral || !cdev[it.channel].table) continue;
        it.kind = kKrausTable;
        const ChanDev& d = cdev[it.channel];
        std::vector<int> ch(shots);
        for (uint64_t s = 0; s < shots; ++s) {
            const double r = u[s * K + it.uidx];
            double cum = 0.0;
            int chosen = -1;
            for (size_t k = 0; k < d.weights.size(); ++k) {
                if (d.weights[k] <= 0.0) continue;
                chosen = static_cast<int>(k);
                cum += d.weights[k];
                if (r < cum) break;
            }
            ch[s] = (chosen >= 0 && !is_identity_scaled(d.norm[chosen])) ? chosen : -1;
        }
        choice[i].ensure(sizeof(int) * shots);
        cuda_check(cudaMemcpy(choice[i].ptr, ch.data(), sizeof(int) * shots, cudaMemcpyHostToDevice),
                   "H2D branch table");
    }

    // ---- resident batch
    size_t free_b = 0, total_b = 0;
    cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const uint64_t state_bytes = uint64_t{16} << n;
    const uint64_t fit = std::max<uint64_t>(1, static_cast<uint64_t>(free_b * 0.85) / state_bytes);
    const uint32_t R = static_cast<uint32_t>(std::min<uint64_t>(
        {shots, fit, max_resident ? max_resident : uint64_t{1024}}));
    auto st = new_state(n, R, nullptr);
    const LaunchCtx ctx = st->ctx;

    std::vector<Program> progs;
    for (const auto& s : stretches) progs.push_back(compile(s, n, fc, nullptr));

    DeviceBuffer d_u, part, mats, flag, scale, dregs;
    d_u.ensure(sizeof(double) * std::max<size_t>(1, u.size()));
    if (!u.empty())
        cuda_check(cudaMemcpy(d_u.ptr, u.data(), sizeof(double) * u.size(), cudaMemcpyHostToDevice),
                   "H2D uniforms");
    part.ensure(sizeof(double) * R * 4 * kTrajMaxBlocks);
    mats.ensure(sizeof(double2) * R * 4);
    flag.ensure(sizeof(int) * R);
    scale.ensure(sizeof(double) * R);
    dregs.ensure(sizeof(uint64_t) * R);
    TrajScratch scr{part.as<double>(), mats.as<double2>(), flag.as<int>(), scale.as<double>(),
                    dregs.as<uint64_t>()};

    for (uint64_t first = 0; first < shots; first += R) {
        const uint32_t nb = static_cast<uint32_t>(std::min<uint64_t>(R, shots - first));
        launch_set_basis(ctx, st->d(), n, nb, 0);
        cuda_check(cudaMemsetAsync(dregs.ptr, 0, sizeof(uint64_t) * nb, ctx.stream), "memset");
        for (size_t i = 0; i < items.size(); ++i) {
            const Item& it = items[i];
            TrajDecide d{};
            d.uniform_index = it.uidx;
            switch (it.kind) {
                case kUnitary:
                    progs[it.prog].launch(ctx, st->d(), n, nb);
                    break;
                case kKrausTable:
                    launch_traj_table(ctx, st->d(), n, nb, it.q, cdev[it.channel].ops.as<double2>(),
                                      choice[i].as<int>() + first);
                    break;
                case kKrausGeneral:
                    d.mode = 0;
                    d.n_ops = static_cast<uint32_t>(channels[it.channel].size());
                    d.ops = cdev[it.channel].ops.as<double2>();
                    launch_traj_kraus(ctx, st->d(), n, nb, it.q, d, d_u.as<double>(), first, K, scr);
                    break;
                case kMeasure:
                case kReset:
                    d.mode = 1;
                    d.is_measure = it.kind == kMeasure ? 1 : 0;
                    d.clbit = it.clbit;
                    launch_traj_measure(ctx, st->d(), n, nb, it.q, d, d_u.as<double>(), first, K,
                                        it.kind == kReset ? 1 : 0, scr);
                    break;
            }
        }
        cuda_check(cudaMemcpyAsync(regs + first, dregs.ptr, sizeof(uint64_t) * nb,
                                   cudaMemcpyDeviceToHost, ctx.stream), "D2H registers");
        cuda_check(cudaStreamSynchronize(ctx.stream), "trajectory batch");
    }
}

}  // namespace lqcs_b200
