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
#include <cstdlib>

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

int env_int_or(const char* name, int dflt) {
    const char* e = std::getenv(name);
    return e ? std::atoi(e) : dflt;
}

bool use_fused(uint32_t n) {
    if (n < kRegMinBits) return false;
    const char* e = std::getenv("LQCS_TRAJ_FUSED");
    return !(e && e[0] == '0');
}

// lambda_min(K^dagger K): for every state, Tr(K rho K^dagger) / Tr(rho) >= this bound.
double min_eig_kdk(const Kraus& k) {
    const double a = std::norm(k[0]) + std::norm(k[2]), d = std::norm(k[1]) + std::norm(k[3]);
    const double b = std::abs(std::conj(k[0]) * k[1] + std::conj(k[2]) * k[3]);
    return 0.5 * (a + d) - std::sqrt(0.25 * (a - d) * (a - d) + b * b);
}

GateDesc matrix_gate(uint32_t q, const Kraus& m) {
    GateDesc g;
    g.type = LQCS_GATE_UNITARY;
    g.qubits = {q};
    g.mat.assign(m.begin(), m.end());
    return g;
}

struct FusedRun {
    uint32_t n;
    const std::vector<Item>& items;
    const std::vector<std::vector<GateDesc>>& stretches;
    const std::vector<Channel>& channels;
    const std::vector<std::vector<Kraus>>& norm;        // unitary mixtures: normalised ops
    const std::vector<const DeviceBuffer*>& ops_dev;     // raw operators on the device
    const std::vector<std::vector<int>>& choice;         // unitary-mixture items: branch per shot
    const std::vector<double>& u;
    uint32_t K;
    uint64_t shots;
    uint32_t max_resident;
};

// Fused batches.  Every noise event whose branch is fixed before the run is a matrix in
// the gate stream: a unitary-mixture branch (chosen from its uniform alone) and the first
// operator K0 of a general channel when u < lambda_min(K0^dagger K0) - 1e-12, because then
// u < Tr(K0 rho K0^dagger) / Tr(rho) for every state, so the reference's first-branch rule
// picks K0 whatever the state.  K0 is applied without its 1/sqrt(p0): states stay
// unnormalised until a state-dependent event, which takes probabilities relative to the
// state's norm and renormalises.  A branch fixed for all states of the batch is one shared
// gate; one that differs is a noise slot (per-state 2x2).  Only events whose branch depends
// on the state (some uncertain general channel, Measure, Reset) cut the batch's gate stream;
// between cuts the stream runs as register tile passes over the whole batch.
void run_fused(const FusedRun& f, uint64_t* regs) {
    const uint32_t n = f.n;
    std::vector<double> lam(f.channels.size(), 0.0);
    for (size_t c = 0; c < f.channels.size(); ++c) lam[c] = min_eig_kdk(f.channels[c][0]);
    // batch work on its own stream; program uploads on another, so the host compiles the next
    // segment while the device runs the current one
    cudaStream_t cs = nullptr, us = nullptr;
    cuda_check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate");
    struct Streams {
        cudaStream_t a = nullptr, b = nullptr;
        ~Streams() {
            if (a) cudaStreamDestroy(a);
            if (b) cudaStreamDestroy(b);
        }
    } guard;
    guard.a = cs;
    cuda_check(cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking), "cudaStreamCreate");
    guard.b = us;

    size_t free_b = 0, total_b = 0;
    cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const uint64_t state_bytes = uint64_t{16} << n;
    const uint64_t fit = std::max<uint64_t>(1, static_cast<uint64_t>(free_b * 0.85) / state_bytes);
    const uint32_t R = static_cast<uint32_t>(std::min<uint64_t>(
        {f.shots, fit, f.max_resident ? f.max_resident : uint64_t{1024}}));
    auto st = new_state(n, R, cs);
    const LaunchCtx ctx = st->ctx;

    // Shot order.  A general channel's event cuts the batch's gate stream only where some
    // state's uniform is at or above the certainty bound, and then it cuts it for every state
    // of the batch.  Shots whose events are all certain ("clean") therefore run together in
    // batches of R without cuts; the others run in small batches that cut only where their
    // own few states need it.  Batch position p holds shot order[p]; the device sees the
    // uniforms in that order, and the registers go back to shot order at the end.
    std::vector<uint64_t> order;
    uint64_t n_clean = 0;
    {
        std::vector<char> dirty(f.shots, 0);
        for (const Item& it : f.items) {
            if (it.kind != kKrausGeneral) continue;
            const double bound = lam[it.channel] - 1e-12;
            for (uint64_t sh = 0; sh < f.shots; ++sh)
                dirty[sh] |= f.u[sh * f.K + it.uidx] < bound ? 0 : 1;
        }
        order.reserve(f.shots);
        for (uint64_t sh = 0; sh < f.shots; ++sh)
            if (!dirty[sh]) order.push_back(sh);
        n_clean = order.size();
        for (uint64_t sh = 0; sh < f.shots; ++sh)
            if (dirty[sh]) order.push_back(sh);
    }
    const uint32_t R_dirty = std::max<uint32_t>(1, std::min<uint32_t>(
        R, static_cast<uint32_t>(env_int_or("LQCS_TRAJ_DIRTY_BATCH", 4))));
    std::vector<double> u_perm(f.u.size());
    for (uint64_t p = 0; p < f.shots; ++p)
        std::copy(f.u.begin() + order[p] * f.K, f.u.begin() + (order[p] + 1) * f.K,
                  u_perm.begin() + p * f.K);
    std::vector<uint64_t> regs_perm(f.shots);

    DeviceBuffer d_u, part, mats, flag, scale, dregs;
    d_u.ensure(sizeof(double) * std::max<size_t>(1, u_perm.size()));
    if (!u_perm.empty())
        cuda_check(cudaMemcpy(d_u.ptr, u_perm.data(), sizeof(double) * u_perm.size(),
                              cudaMemcpyHostToDevice),
                   "H2D uniforms");
    part.ensure(sizeof(double) * R * 4 * kTrajMaxBlocks);
    mats.ensure(sizeof(double2) * R * 4);
    flag.ensure(sizeof(int) * R);
    scale.ensure(sizeof(double) * R);
    dregs.ensure(sizeof(uint64_t) * R);
    TrajScratch scr{part.as<double>(), mats.as<double2>(), flag.as<int>(), scale.as<double>(),
                    dregs.as<uint64_t>()};
    const Kraus ident{cd{1, 0}, cd{0, 0}, cd{0, 0}, cd{1, 0}};
    // Terminal measurements (nothing but Measures of distinct qubits up to the end) need no
    // collapse: each outcome follows from the amplitudes consistent with the earlier ones.
    size_t tail = f.items.size();
    {
        std::vector<char> seen(n, 0);
        while (tail > 0 && f.items[tail - 1].kind == kMeasure && !seen[f.items[tail - 1].q]) {
            seen[f.items[tail - 1].q] = 1;
            --tail;
        }
    }
    DeviceBuffer d_vals;
    d_vals.ensure(sizeof(uint64_t) * R);

    for (uint64_t first = 0; first < f.shots;) {   // first: batch start position in `order`
        const uint32_t nb = static_cast<uint32_t>(
            first < n_clean ? std::min<uint64_t>(R, n_clean - first)
                            : std::min<uint64_t>(R_dirty, f.shots - first));
        auto shot = [&](uint32_t b) { return order[first + b]; };
        launch_set_basis(ctx, st->d(), n, nb, 0);
        cuda_check(cudaMemsetAsync(dregs.ptr, 0, sizeof(uint64_t) * nb, cs), "memset");
        cuda_check(cudaMemsetAsync(d_vals.ptr, 0, sizeof(uint64_t) * nb, cs), "memset");
        BitList tail_fixed{};
        std::vector<Program> keep;          // alive until the batch is done
        std::vector<DeviceBuffer> bufs;
        std::vector<GateDesc> seg;
        std::vector<std::vector<Kraus>> slots(nb);
        auto upload = [&](const void* src, size_t bytes) {
            DeviceBuffer b;
            b.ensure(bytes);
            cuda_check(cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice, us), "H2D batch data");
            cuda_check(cudaStreamSynchronize(us), "H2D batch data");
            bufs.push_back(std::move(b));
            return bufs.back().ptr;
        };
        auto flush = [&]() {
            if (seg.empty()) return;
            Program p;
            if (compile_slots(seg, n, slots, us, p)) {
                p.launch(ctx, st->d(), n, nb);
                keep.push_back(std::move(p));
            } else {
                // gate by gate: shared gates as programs, noise slots as per-state 2x2 tables
                FusionConfig none;
                none.fuse = false;
                for (const GateDesc& g : seg) {
                    if (!g.slot) {
                        keep.push_back(compile({g}, n, none, us));
                        keep.back().launch(ctx, st->d(), n, nb);
                        continue;
                    }
                    std::vector<double2> tab(4 * static_cast<size_t>(nb));
                    std::vector<int> idx(nb);
                    for (uint32_t b = 0; b < nb; ++b) {
                        for (int e = 0; e < 4; ++e) {
                            const cd z = slots[b][g.slot_id][e];
                            tab[4 * b + e] = make_double2(z.real(), z.imag());
                        }
                        idx[b] = static_cast<int>(b);
                    }
                    const void* dt = upload(tab.data(), sizeof(double2) * tab.size());
                    const void* di = upload(idx.data(), sizeof(int) * idx.size());
                    launch_traj_table(ctx, st->d(), n, nb, g.qubits[0],
                                      static_cast<const double2*>(dt), static_cast<const int*>(di));
                }
            }
            seg.clear();
            for (auto& s : slots) s.clear();
        };
        for (size_t i = 0; i < f.items.size(); ++i) {
            const Item& it = f.items[i];
            switch (it.kind) {
                case kUnitary:
                    seg.insert(seg.end(), f.stretches[it.prog].begin(), f.stretches[it.prog].end());
                    break;
                case kKrausTable: {
                    const std::vector<int>& ch = f.choice[i];
                    const int c0 = ch[shot(0)];
                    bool any = false, same = true;
                    for (uint32_t b = 0; b < nb; ++b) {
                        any |= ch[shot(b)] >= 0;
                        same &= ch[shot(b)] == c0;
                    }
                    if (!any) break;
                    if (same) {
                        seg.push_back(matrix_gate(it.q, f.norm[it.channel][c0]));
                        break;
                    }
                    GateDesc g = matrix_gate(it.q, ident);
                    g.slot = true;
                    g.slot_id = static_cast<uint32_t>(slots[0].size());
                    for (uint32_t b = 0; b < nb; ++b) {
                        const int c = ch[shot(b)];
                        slots[b].push_back(c < 0 ? ident : f.norm[it.channel][c]);
                    }
                    seg.push_back(std::move(g));
                    break;
                }
                case kKrausGeneral: {
                    const double bound = lam[it.channel] - 1e-12;
                    std::vector<int> forced(nb);
                    bool all = true;
                    for (uint32_t b = 0; b < nb; ++b) {
                        forced[b] = f.u[shot(b) * f.K + it.uidx] < bound ? 0 : -1;
                        all &= forced[b] == 0;
                    }
                    if (all) {
                        seg.push_back(matrix_gate(it.q, f.channels[it.channel][0]));
                        break;
                    }
                    flush();
                    TrajDecide d{};
                    d.mode = 0;
                    d.uniform_index = it.uidx;
                    d.n_ops = static_cast<uint32_t>(f.channels[it.channel].size());
                    d.ops = f.ops_dev[it.channel]->as<double2>();
                    d.forced = static_cast<const int*>(upload(forced.data(), sizeof(int) * nb));
                    launch_traj_kraus(ctx, st->d(), n, nb, it.q, d, d_u.as<double>(), first, f.K, scr);
                    // the states whose branch was known take K0 as the first gate of the next
                    // segment (identity for the states decided here)
                    GateDesc g = matrix_gate(it.q, ident);
                    g.slot = true;
                    g.slot_id = static_cast<uint32_t>(slots[0].size());
                    for (uint32_t b = 0; b < nb; ++b)
                        slots[b].push_back(forced[b] == 0 ? f.channels[it.channel][0] : ident);
                    seg.push_back(std::move(g));
                    break;
                }
                case kMeasure:
                    if (i >= tail) {   // terminal: Born rule on the consistent subspace
                        flush();
                        launch_traj_tail_measure(ctx, st->d(), n, nb, it.q, tail_fixed,
                                                 d_vals.as<uint64_t>(), it.clbit, it.uidx,
                                                 d_u.as<double>(), first, f.K, scr);
                        tail_fixed.pos[tail_fixed.n++] = it.q;
                        std::sort(tail_fixed.pos, tail_fixed.pos + tail_fixed.n);
                        break;
                    }
                    [[fallthrough]];
                case kReset: {
                    flush();
                    TrajDecide d{};
                    d.mode = 1;
                    d.is_measure = it.kind == kMeasure ? 1 : 0;
                    d.clbit = it.clbit;
                    d.uniform_index = it.uidx;
                    launch_traj_measure(ctx, st->d(), n, nb, it.q, d, d_u.as<double>(), first, f.K,
                                        it.kind == kReset ? 1 : 0, scr);
                    break;
                }
            }
        }
        flush();
        cuda_check(cudaMemcpyAsync(regs_perm.data() + first, dregs.ptr, sizeof(uint64_t) * nb,
                                   cudaMemcpyDeviceToHost, cs), "D2H registers");
        cuda_check(cudaStreamSynchronize(cs), "trajectory batch");
        first += nb;
    }
    for (uint64_t p = 0; p < f.shots; ++p) regs[order[p]] = regs_perm[p];
}

uint64_t stretch_qubits(const std::vector<GateDesc>& s) {
    uint64_t m = 0;
    for (const GateDesc& g : s)
        for (uint32_t q : g.qubits) m |= uint64_t{1} << q;
    return m;
}

// Shared deterministic prefix.  When nothing before the final measurements is random (no
// noise model, no Kraus instruction, no Reset, no earlier Measure), every shot reaches them
// in the same state.  Unitaries between those measurements are moved ahead of them when
// they touch no qubit measured before them (a unitary and a projective measurement on
// disjoint qubits commute) and dropped when no measurement follows them (they cannot change
// a recorded outcome); the reference's one-qubit fusion leaves such gates there, because a
// Measure flushes only its own qubit's pending product (src/transpiler/gate_fusion.cpp:
// 58-62), and they send the reference down its per-shot path.  One state is evolved, the
// joint distribution of the measured qubits is tabulated once, and each shot walks its
// measurements with its own uniforms: outcome 1 iff u < P(bit = 1 | earlier outcomes) —
// the Born rule on the subspace consistent with the earlier outcomes, as the terminal
// measurements of the batched path decide.  Returns false (nothing done) when the circuit
// does not have this form or the table would exceed 2^24 entries.
bool run_shared_prefix(uint32_t n, const std::vector<Item>& items,
                       const std::vector<std::vector<GateDesc>>& stretches, const FusionConfig& fc,
                       const std::vector<double>& u, uint32_t K, uint64_t shots, uint64_t* regs) {
    // tail: the longest suffix of Measures (distinct qubits) and unitaries
    size_t b = items.size();
    {
        uint64_t seen = 0;
        while (b > 0) {
            const Item& it = items[b - 1];
            if (it.kind == kMeasure) {
                if ((seen >> it.q) & 1) break;
                seen |= uint64_t{1} << it.q;
            } else if (it.kind != kUnitary) {
                break;
            }
            --b;
        }
    }
    // shrink until every unitary of the tail commutes with the measurements before it
    std::vector<size_t> hoist;
    while (true) {
        hoist.clear();
        uint64_t measured = 0;
        size_t bad = items.size();
        for (size_t i = b; i < items.size(); ++i) {
            const Item& it = items[i];
            if (it.kind == kMeasure) {
                measured |= uint64_t{1} << it.q;
                continue;
            }
            bool later = false;
            for (size_t j = i + 1; j < items.size(); ++j) later |= items[j].kind == kMeasure;
            if (!later) continue;   // dropped
            if ((stretch_qubits(stretches[it.prog]) & measured) == 0) {
                hoist.push_back(i);
                continue;
            }
            bad = i;
            break;
        }
        if (bad == items.size()) break;
        b = bad + 1;
    }
    for (size_t i = 0; i < b; ++i)
        if (items[i].kind != kUnitary) return false;
    std::vector<uint32_t> mq, clb, uid;
    for (size_t i = b; i < items.size(); ++i)
        if (items[i].kind == kMeasure) {
            mq.push_back(items[i].q);
            clb.push_back(items[i].clbit);
            uid.push_back(items[i].uidx);
        }
    const uint32_t m = static_cast<uint32_t>(mq.size());
    if (m == 0 || m > 24) return false;

    std::vector<GateDesc> prefix;
    for (size_t i = 0; i < b; ++i)
        prefix.insert(prefix.end(), stretches[items[i].prog].begin(), stretches[items[i].prog].end());
    for (size_t i : hoist)
        prefix.insert(prefix.end(), stretches[items[i].prog].begin(), stretches[items[i].prog].end());

    auto st = new_state(n, 1, nullptr);
    const LaunchCtx ctx = st->ctx;
    launch_set_basis(ctx, st->d(), n, 1, 0);
    Program prog;
    if (!prefix.empty()) {
        prog = compile(prefix, n, fc, nullptr);
        prog.launch(ctx, st->d(), n, 1);
    }
    const uint64_t entries = uint64_t{1} << m;
    DeviceBuffer partial, table;
    partial.ensure(sizeof(double) * entries * marginal_chunks(n, m));
    table.ensure(sizeof(double) * entries);
    launch_marginal_table(ctx, st->d(), n, mq.data(), m, partial.as<double>(), table.as<double>());
    // level sums: lev[j][o] = total over the entries whose low j bits equal o
    std::vector<std::vector<double>> lev(m + 1);
    lev[m].resize(entries);
    cuda_check(cudaMemcpyAsync(lev[m].data(), table.ptr, sizeof(double) * entries,
                               cudaMemcpyDeviceToHost, ctx.stream), "D2H marginal table");
    cuda_check(cudaStreamSynchronize(ctx.stream), "marginal table");
    for (uint32_t j = m; j-- > 0;) {
        lev[j].resize(uint64_t{1} << j);
        for (uint64_t o = 0; o < (uint64_t{1} << j); ++o)
            lev[j][o] = lev[j + 1][o] + lev[j + 1][o | (uint64_t{1} << j)];
    }
    for (uint64_t s = 0; s < shots; ++s) {
        uint64_t o = 0, reg = 0;
        for (uint32_t j = 0; j < m; ++j) {
            const double r0 = lev[j + 1][o], r1 = lev[j + 1][o | (uint64_t{1} << j)];
            const int outcome = u[s * K + uid[j]] < r1 / (r0 + r1) ? 1 : 0;
            o |= static_cast<uint64_t>(outcome) << j;
            const uint64_t bit = uint64_t{1} << clb[j];
            reg = outcome ? (reg | bit) : (reg & ~bit);
        }
        regs[s] = reg;
    }
    return true;
}

}  // namespace

void run_per_shot_batched(uint32_t n, const std::vector<GateDesc>& gates, uint64_t shots,
                          const std::vector<Channel>& model, const FusionConfig& fc_in, Rng& rng,
                          uint32_t max_resident, uint64_t* regs, uint64_t shot_offset) {
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
    rng.discard(shot_offset * K);   // the draws of the shots before this call's first
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
    std::vector<std::vector<int>> choice_host(items.size());
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
        choice_host[i] = std::move(ch);
    }

    if (!noisy && run_shared_prefix(n, items, stretches, fc, u, K, shots, regs)) return;

    if (fc_in.fuse && use_fused(n)) {
        std::vector<std::vector<Kraus>> norm(channels.size());
        std::vector<const DeviceBuffer*> ops_dev(channels.size());
        for (size_t c = 0; c < channels.size(); ++c) {
            norm[c] = cdev[c].norm;
            ops_dev[c] = &cdev[c].ops;
        }
        const FusedRun fr{n, items, stretches, channels, norm, ops_dev, choice_host, u, K, shots,
                          max_resident};
        run_fused(fr, regs);
        return;
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
