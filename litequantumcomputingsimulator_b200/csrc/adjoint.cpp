// adjoint.cpp — batched adjoint-state gradients of <psi(theta)|H|psi(theta)>.
//
// Engine extension: the reference differentiates by the parameter-shift rule, two full
// circuit evaluations per parameter (algorithms::parameter_shift_gradient,
// src/algorithms/vqe.cpp:68-94).  Every parameterised gate here is exp(-i theta/2 P) for a
// Pauli string P (RX, RY, RZ, rp), so with psi_k the state after gate k and
// lambda_k = U_{k+1}^dagger ... U_N^dagger H psi_N,
//     dE/dtheta_k = 2 Re <lambda_k| (-i/2) P_k |psi_k> = Im <lambda_k| P_k |psi_k>.
// One forward pass, one Hamiltonian application and one backward pass (undoing each gate
// on psi and lambda) give all gradients.  Up to `max_resident` parameter sets advance
// together: every kernel launch walks the whole resident batch (gridDim.y), the
// parameterised rotations read one (cos, sin) per state.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>

#include "engine.hpp"

namespace lqcs_b200 {

void launch_batched_inner_re_p(const LaunchCtx& ctx, const double2* a, const double2* b,
                               uint32_t n, uint32_t batch, double* d_partials, double* d_out);
void launch_batched_pauli_im_p(const LaunchCtx& ctx, const double2* a, const double2* b,
                               uint32_t n, uint32_t batch, uint64_t x, uint64_t zy,
                               uint32_t n_y, double* d_partials, double* d_out,
                               uint64_t out_stride);

namespace {

struct GateStep {
    int param = -1;            // parameter index, -1 for a fixed gate
    PauliMasks gen;            // generator of a parameterised gate (global masks)
    Program fwd, inv;          // fixed gate and its inverse (one op each)
};

PauliMasks generator(const GateDesc& g) {
    PauliMasks m;
    const uint64_t t = uint64_t{1} << g.targets()[0];
    switch (g.type) {
        case LQCS_GATE_RX: m.x = t; break;
        case LQCS_GATE_RY: m.x = t; m.zy = t; m.n_y = 1; break;
        case LQCS_GATE_RZ: m.zy = t; break;
        default: {
            const PauliMasks loc = pauli_local_masks(g.pauli);
            for (uint32_t j = 0; j < g.pauli.size(); ++j) {
                if ((loc.x >> j) & 1) m.x |= uint64_t{1} << g.targets()[j];
                if ((loc.zy >> j) & 1) m.zy |= uint64_t{1} << g.targets()[j];
            }
            m.n_y = loc.n_y;
        }
    }
    return m;
}

// Inverse of one device op (conjugate transpose, inverse permutation).
DevOp invert(const DevOp& op) {
    DevOp r = op;
    switch (op.kind) {
        case OpKind::K1Q:
            r.m1 = {std::conj(op.m1[0]), std::conj(op.m1[2]), std::conj(op.m1[1]),
                    std::conj(op.m1[3])};
            break;
        case OpKind::PHASE:
            r.phase = std::conj(op.phase);
            break;
        case OpKind::DIAG:
            for (cd& z : r.mat) z = std::conj(z);
            break;
        case OpKind::DENSE: {
            const uint64_t dim = uint64_t{1} << op.k;
            for (uint64_t i = 0; i < dim; ++i)
                for (uint64_t j = 0; j < dim; ++j) r.mat[j * dim + i] = std::conj(op.mat[i * dim + j]);
            break;
        }
        case OpKind::PERM: {
            // reverse every cycle
            size_t s = 0;
            for (uint32_t len : op.cycle_len) {
                std::reverse(r.cycles.begin() + s, r.cycles.begin() + s + len);
                s += len;
            }
            break;
        }
        case OpKind::PAULI:
            r.sin_h = -op.sin_h;
            break;
    }
    return r;
}

}  // namespace

// Terms as c_t i^{n_y} with their masks, grouped by the bits of x above the kernel's tile
// (stable within a group, groups by first appearance).
void HamiltonianDev::upload(const Hamiltonian& h, uint32_t n) {
    static const cd ipow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    const uint32_t ml = ham_tile_bits(n);
    std::vector<uint64_t> keys;
    std::vector<std::vector<PauliTermDev>> by_key;
    for (size_t t = 0; t < h.terms.size(); ++t) {
        const cd c = h.coeffs[t] * ipow[h.terms[t].n_y % 4];
        const uint64_t key = h.terms[t].x >> ml;
        size_t k = std::find(keys.begin(), keys.end(), key) - keys.begin();
        if (k == keys.size()) {
            keys.push_back(key);
            by_key.emplace_back();
        }
        by_key[k].push_back({h.terms[t].x, h.terms[t].zy, make_double2(c.real(), c.imag())});
    }
    std::vector<PauliTermDev> flat;
    std::vector<uint32_t> grp{static_cast<uint32_t>(keys.size())};
    for (uint64_t key : keys) grp.push_back(static_cast<uint32_t>(key));
    for (const auto& v : by_key) {
        grp.push_back(static_cast<uint32_t>(flat.size()));
        flat.insert(flat.end(), v.begin(), v.end());
    }
    grp.push_back(static_cast<uint32_t>(flat.size()));
    n_terms = static_cast<uint32_t>(flat.size());
    terms.ensure(sizeof(PauliTermDev) * std::max<size_t>(1, flat.size()));
    groups.ensure(sizeof(uint32_t) * grp.size());
    if (!flat.empty())
        cuda_check(cudaMemcpy(terms.ptr, flat.data(), sizeof(PauliTermDev) * flat.size(),
                              cudaMemcpyHostToDevice),
                   "H2D terms");
    cuda_check(cudaMemcpy(groups.ptr, grp.data(), sizeof(uint32_t) * grp.size(),
                          cudaMemcpyHostToDevice),
               "H2D term groups");
}

namespace {

// Resident sets per launch batch: as many as fit (two states per set), at most 256.  With
// the rotation tile passes a launch is compute-heavy and larger batches amortise it better
// (16 qubits: 7960 gradients/s with 256 sets, 7570 with 32).  One launch per step (fixed
// gates, LQCS_ADJ_TILES=0) streams every state per step, and there a batch that stays in L2
// is faster (32 sets: 4230 against 3210) — max_resident picks that size.
uint32_t default_resident(uint32_t n, uint64_t batch) {
    size_t free_b = 0, total_b = 0;
    cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const uint64_t per_set = 2 * (uint64_t{16} << n);
    const uint64_t fit = std::max<uint64_t>(1, (free_b / 2) / per_set);
    return static_cast<uint32_t>(std::min<uint64_t>({batch, fit, 256}));
}

}  // namespace

namespace {

// One launch of the forward or backward sweep: a rotation tile pass (step < 0; its ops at
// op_off in d_rot_ops) or one step launched on its own.
struct Segment {
    int step = -1;
    RotTilePass pass{};
    uint32_t op_off = 0;
};

// Rotation tile passes over a run of parameterised steps: a pass takes rotations while the
// X bits above L of its rotations fit the m - L free tile slots.
void plan_rotation_passes(const std::vector<const GateStep*>& run,
                          const std::vector<size_t>& index, uint32_t n, uint32_t m, uint32_t L,
                          std::vector<Segment>& segs, std::vector<RotTileOp>& all_ops) {
    const uint64_t low = (uint64_t{1} << L) - 1u;
    const uint32_t slots = m - L;
    uint64_t H = 0;
    std::vector<const GateStep*> cur;
    auto close = [&] {
        if (cur.empty()) return;
        for (uint32_t q = L; q < n && static_cast<uint32_t>(__builtin_popcountll(H)) < slots; ++q)
            H |= uint64_t{1} << q;
        Segment sg;
        sg.pass.m = m;
        sg.pass.L = L;
        sg.pass.h = slots;
        sg.pass.n_ops = static_cast<uint32_t>(cur.size());
        uint32_t loc[64] = {};
        for (uint32_t q = 0; q < L; ++q) loc[q] = q;
        uint32_t i = 0;
        for (uint32_t q = 0; q < n; ++q) {
            if ((H >> q) & 1) {
                sg.pass.hbits[i] = q;
                loc[q] = L + i;
                ++i;
            }
        }
        const uint64_t tile = H | low;
        auto local = [&](uint64_t mask) {
            uint32_t r = 0;
            for (uint32_t q = 0; q < n; ++q)
                if (((mask & tile) >> q) & 1) r |= 1u << loc[q];
            return r;
        };
        sg.op_off = static_cast<uint32_t>(all_ops.size());
        for (const GateStep* st : cur) {
            RotTileOp op{};
            op.x_loc = local(st->gen.x);
            op.zy_loc = local(st->gen.zy);
            op.zy_out = st->gen.zy & ~tile;
            op.param = static_cast<uint32_t>(st->param);
            op.n_y = st->gen.n_y;
            all_ops.push_back(op);
        }
        segs.push_back(sg);
        cur.clear();
        H = 0;
    };
    // Passes fill greedily over the pending rotations in order; a rotation may join ahead of
    // rotations left for a later pass when it commutes with every one of them (Pauli strings
    // commute when they anticommute on an even number of qubits), so the pass sequence is
    // one factorisation of the same product.  A rotation too wide for a tile runs on its own.
    auto commute = [](const PauliMasks& a, const PauliMasks& b) {
        return ((__builtin_popcountll(a.x & b.zy) + __builtin_popcountll(a.zy & b.x)) & 1) == 0;
    };
    std::vector<size_t> pend(run.size());
    for (size_t r = 0; r < run.size(); ++r) pend[r] = r;
    while (!pend.empty()) {
        const size_t f0 = pend.front();
        if (static_cast<uint32_t>(__builtin_popcountll(run[f0]->gen.x & ~low)) > slots) {
            Segment own;
            own.step = static_cast<int>(index[f0]);
            segs.push_back(own);
            pend.erase(pend.begin());
            continue;
        }
        std::vector<size_t> rest;
        for (size_t r : pend) {
            const uint64_t need = run[r]->gen.x & ~low;
            bool ok = static_cast<uint32_t>(__builtin_popcountll(H | need)) <= slots &&
                      cur.size() < kRotMaxOps;
            for (size_t k = 0; ok && k < rest.size(); ++k) ok = commute(run[r]->gen, run[rest[k]]->gen);
            if (ok) {
                H |= need;
                cur.push_back(run[r]);
            } else {
                rest.push_back(r);
            }
        }
        close();
        pend = std::move(rest);
    }
}

int env_or(const char* name, int dflt) {
    const char* e = std::getenv(name);
    return e ? std::atoi(e) : dflt;
}

// Everything one (circuit, Hamiltonian, resident batch) needs on the device, kept between
// calls: the fixed gates and their inverses, the two resident state batches, the Hamiltonian
// terms and the per-set buffers, on a stream of its own.  A call only uploads the new
// (cos, sin) tables, so the launch sequence of a batch of nb sets never changes: it is
// captured once as a CUDA graph and replayed (LQCS_GRAPHS=0: launched directly).
struct AdjointPlan {
    uint64_t key = 0;
    uint32_t n = 0, R = 0;
    uint64_t np = 0;
    std::vector<GateStep> steps;
    HamiltonianDev ham;
    std::unique_ptr<lqcs_state> psi, lam;
    DeviceBuffer d_cs, d_csi, d_part, d_energy, d_grad;
    // rotation tile passes (empty: one launch per step)
    std::vector<Segment> fwd_segs, bwd_segs;
    DeviceBuffer d_rot_ops, d_rot_part;
    cudaStream_t stream = nullptr;
    // (2 nb + with gradients) -> (graph, kernels)
    std::map<uint32_t, std::pair<cudaGraphExec_t, uint64_t>> graphs;

    AdjointPlan() = default;
    AdjointPlan(const AdjointPlan&) = delete;
    AdjointPlan& operator=(const AdjointPlan&) = delete;
    ~AdjointPlan() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.second.first);
        psi.reset();
        lam.reset();
        if (stream) cudaStreamDestroy(stream);
    }

    void forward_step(const GateStep& s, uint32_t nb) const {
        const LaunchCtx& ctx = psi->ctx;
        if (s.param >= 0) {
            launch_pauli_rotation_batched(ctx, psi->d(), n, nb, s.gen.x, s.gen.zy, s.gen.n_y,
                                          d_cs.as<double2>() + static_cast<uint64_t>(s.param) * R);
        } else {
            s.fwd.launch(ctx, psi->d(), n, nb);
        }
    }

    void backward_step(const GateStep& s, uint32_t nb) const {
        const LaunchCtx& ctx = psi->ctx;
        if (s.param >= 0) {
            launch_batched_pauli_im_p(ctx, lam->d(), psi->d(), n, nb, s.gen.x, s.gen.zy,
                                      s.gen.n_y, d_part.as<double>(),
                                      d_grad.as<double>() + s.param, np);
            const double2* inv = d_csi.as<double2>() + static_cast<uint64_t>(s.param) * R;
            launch_pauli_rotation_batched(ctx, psi->d(), n, nb, s.gen.x, s.gen.zy, s.gen.n_y, inv);
            launch_pauli_rotation_batched(ctx, lam->d(), n, nb, s.gen.x, s.gen.zy, s.gen.n_y, inv);
        } else {
            s.inv.launch(ctx, psi->d(), n, nb);
            s.inv.launch(ctx, lam->d(), n, nb);
        }
    }

    // The launch sequence of one batch of nb sets on this plan's stream; without gradients
    // (energies only) it ends after <psi|H|psi>.
    void enqueue(uint32_t nb, bool grads = true) const {
        const LaunchCtx& ctx = psi->ctx;
        const uint64_t len = uint64_t{1} << n;
        const RotTileOp* rot_ops = d_rot_ops.as<RotTileOp>();
        launch_set_basis(ctx, psi->d(), n, nb, 0);
        if (fwd_segs.empty()) {
            for (const GateStep& s : steps) forward_step(s, nb);
        } else {
            for (const Segment& sg : fwd_segs) {
                if (sg.step >= 0) forward_step(steps[sg.step], nb);
                else launch_rot_tile_fwd(ctx, psi->d(), n, nb, sg.pass, rot_ops + sg.op_off,
                                         d_cs.as<double2>(), R);
            }
        }
        if (ham.n_terms == 0) {
            cuda_check(cudaMemsetAsync(lam->d(), 0, sizeof(double2) * len * nb, ctx.stream), "memset");
        } else {
            launch_apply_hamiltonian(ctx, psi->d(), lam->d(), n, nb, ham.terms.as<PauliTermDev>(),
                                     ham.groups.as<uint32_t>());
        }
        launch_batched_inner_re_p(ctx, psi->d(), lam->d(), n, nb, d_part.as<double>(),
                                  d_energy.as<double>());
        if (!grads) return;
        if (bwd_segs.empty()) {
            for (size_t i = steps.size(); i-- > 0;) backward_step(steps[i], nb);
        } else {
            for (const Segment& sg : bwd_segs) {
                if (sg.step >= 0) backward_step(steps[sg.step], nb);
                else launch_rot_tile_bwd(ctx, psi->d(), lam->d(), n, nb, sg.pass, rot_ops + sg.op_off,
                                         d_cs.as<double2>(), R, d_rot_part.as<double>(),
                                         d_grad.as<double>(), np);
            }
        }
    }

    // Rotation tile passes for both sweeps: forward tiles of 2^min(n, 12) amplitudes (one
    // state in shared memory), backward 2^min(n, 11) (psi and lambda); qubits 0..2 stay in
    // every tile so tile rows are 128-byte lines.  LQCS_ADJ_TILES=0 keeps one launch per step.
    void plan_tiles() {
        if (env_or("LQCS_ADJ_TILES", 1) == 0) return;
        const uint32_t mf = std::min<uint32_t>(n, static_cast<uint32_t>(env_or("LQCS_ADJ_TILE_F", 12)));
        const uint32_t mb = std::min<uint32_t>(n, static_cast<uint32_t>(env_or("LQCS_ADJ_TILE_B", 11)));
        if (mf < 5 || mb < 5 || mf > kRotMaxBits || mb > kRotMaxBits) return;
        const uint32_t L = 3;
        std::vector<RotTileOp> ops;
        std::vector<const GateStep*> run;
        std::vector<size_t> idx;
        auto flush = [&](std::vector<Segment>& segs, uint32_t m) {
            plan_rotation_passes(run, idx, n, m, L, segs, ops);
            run.clear();
            idx.clear();
        };
        for (size_t i = 0; i < steps.size(); ++i) {
            if (steps[i].param >= 0) {
                run.push_back(&steps[i]);
                idx.push_back(i);
                continue;
            }
            flush(fwd_segs, mf);
            Segment own;
            own.step = static_cast<int>(i);
            fwd_segs.push_back(own);
        }
        flush(fwd_segs, mf);
        for (size_t i = steps.size(); i-- > 0;) {
            if (steps[i].param >= 0) {
                run.push_back(&steps[i]);
                idx.push_back(i);
                continue;
            }
            flush(bwd_segs, mb);
            Segment own;
            own.step = static_cast<int>(i);
            bwd_segs.push_back(own);
        }
        flush(bwd_segs, mb);
        uint32_t max_ops = 1;
        for (const Segment& sg : bwd_segs)
            if (sg.step < 0) max_ops = std::max(max_ops, sg.pass.n_ops);
        d_rot_ops.ensure(sizeof(RotTileOp) * std::max<size_t>(1, ops.size()));
        if (!ops.empty())
            cuda_check(cudaMemcpy(d_rot_ops.ptr, ops.data(), sizeof(RotTileOp) * ops.size(),
                                  cudaMemcpyHostToDevice),
                       "H2D rotation passes");
        d_rot_part.ensure(sizeof(double) * max_ops * R * (uint64_t{1} << (n - mb)));
    }

    void run(uint32_t nb, bool grads = true) {
        const char* e = std::getenv("LQCS_GRAPHS");
        if (e && e[0] == '0') {
            enqueue(nb, grads);
            return;
        }
        const uint32_t key = 2 * nb + (grads ? 1u : 0u);
        auto it = graphs.find(key);
        bool fresh = false;
        if (it == graphs.end()) {
            // capture once; a failed capture falls back to direct launches (which rethrow any
            // real launch error)
            const uint64_t k0 = launch_count();
            cudaGraph_t g = nullptr;
            cudaGraphExec_t exec = nullptr;
            bool ok = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                try {
                    enqueue(nb, grads);
                } catch (...) {
                    ok = false;
                }
                cudaGraph_t done = nullptr;
                const bool ended = cudaStreamEndCapture(stream, &done) == cudaSuccess;
                g = done;
                ok = ok && ended && g;
            }
            if (ok) ok = cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
            if (!ok) {
                cudaGetLastError();
                enqueue(nb, grads);
                return;
            }
            it = graphs.emplace(key, std::make_pair(exec, launch_count() - k0)).first;
            fresh = true;   // the capture already counted this batch's kernels
        }
        cuda_check(cudaGraphLaunch(it->second.first, stream), "cudaGraphLaunch");
        if (!fresh) count_launch(it->second.second);   // the graph's kernels, each replay
    }
};

uint64_t plan_key(const std::vector<GateDesc>& tmpl, const std::vector<int>& param_of,
                  const Hamiltonian& h, uint32_t n, uint32_t R) {
    uint64_t k = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t len) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < len; ++i) k = (k ^ b[i]) * 1099511628211ull;
    };
    mix(&n, sizeof n);
    mix(&R, sizeof R);
    for (size_t i = 0; i < tmpl.size(); ++i) {
        const GateDesc& g = tmpl[i];
        mix(&g.type, sizeof g.type);
        mix(&g.n_controls, sizeof g.n_controls);
        mix(g.qubits.data(), g.qubits.size() * sizeof(uint32_t));
        mix(&param_of[i], sizeof(int));
        if (param_of[i] < 0) {   // fixed gates: their values are part of the plan
            mix(g.params.data(), g.params.size() * sizeof(double));
            mix(g.mat.data(), g.mat.size() * sizeof(cd));
            mix(g.perm.data(), g.perm.size() * sizeof(uint64_t));
        }
        mix(g.pauli.data(), g.pauli.size());
    }
    for (size_t t = 0; t < h.terms.size(); ++t) {
        mix(&h.terms[t].x, sizeof(uint64_t));
        mix(&h.terms[t].zy, sizeof(uint64_t));
        mix(&h.coeffs[t], sizeof(double));
    }
    return k;
}

// The most recent plans (resident memory: two state batches each), newest last.
std::mutex g_plan_mu;
std::vector<std::unique_ptr<AdjointPlan>> g_plans;
constexpr size_t kKeptPlans = 2;

std::unique_ptr<AdjointPlan> build_plan(const std::vector<GateDesc>& tmpl,
                                        const std::vector<int>& param_of, const Hamiltonian& h,
                                        uint32_t n, uint64_t np, uint32_t R, uint64_t dkey);

AdjointPlan& adjoint_plan(const std::vector<GateDesc>& tmpl, const std::vector<int>& param_of,
                          const Hamiltonian& h, uint32_t n, uint64_t np, uint64_t batch,
                          uint32_t max_resident) {
    const uint32_t R = max_resident ? static_cast<uint32_t>(std::min<uint64_t>(max_resident, batch))
                                    : default_resident(n, batch);
    const uint64_t key = plan_key(tmpl, param_of, h, n, R);
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    const uint64_t dkey = key ^ (static_cast<uint64_t>(dev) << 56);
    std::lock_guard<std::mutex> lk(g_plan_mu);
    for (auto& p : g_plans)
        if (p->key == dkey) return *p;
    auto plan = build_plan(tmpl, param_of, h, n, np, R, dkey);
    if (g_plans.size() >= kKeptPlans) g_plans.erase(g_plans.begin());
    g_plans.push_back(std::move(plan));
    return *g_plans.back();
}

std::unique_ptr<AdjointPlan> build_plan(const std::vector<GateDesc>& tmpl,
                                        const std::vector<int>& param_of, const Hamiltonian& h,
                                        uint32_t n, uint64_t np, uint32_t R, uint64_t dkey) {
    auto plan = std::make_unique<AdjointPlan>();
    plan->key = dkey;
    plan->n = n;
    plan->R = R;
    plan->np = np;
    cuda_check(cudaStreamCreateWithFlags(&plan->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    // the fixed gates (and their inverses); barrier / measure are skipped
    for (size_t i = 0; i < tmpl.size(); ++i) {
        const GateDesc& g = tmpl[i];
        if (g.type == LQCS_GATE_RESET) invalid("run_statevector: Reset is non-deterministic; use run() instead");
        if (!g.is_unitary()) continue;
        GateStep s;
        s.param = param_of[i];
        if (s.param >= 0) {
            s.gen = generator(g);
        } else {
            const DevOp op = lower_gate(g, n);
            s.fwd.build({op}, plan->stream);
            s.inv.build({invert(op)}, plan->stream);
        }
        plan->steps.push_back(std::move(s));
    }
    plan->psi = new_state(n, R, plan->stream);
    plan->lam = new_state(n, R, plan->stream);
    plan->ham.upload(h, n);
    plan->plan_tiles();
    plan->d_cs.ensure(sizeof(double2) * std::max<uint64_t>(1, np) * R);
    plan->d_csi.ensure(sizeof(double2) * std::max<uint64_t>(1, np) * R);
    plan->d_part.ensure(sizeof(double) * 64 * R);
    plan->d_energy.ensure(sizeof(double) * R);
    plan->d_grad.ensure(sizeof(double) * std::max<uint64_t>(1, np) * R);
    return plan;
}

}  // namespace

void adjoint_batched(const lqcs_parametric_circuit* pc, const Hamiltonian& h,
                     const double* params, uint64_t batch, uint32_t max_resident,
                     double* energy_out, double* grad_out) {
    std::vector<GateDesc> tmpl;
    std::vector<uint64_t> pinst;
    check_pc(pc, tmpl, pinst);
    if (batch == 0) return;
    if (!params && !pinst.empty()) invalid("adjoint_gradient: params is null");
    const uint32_t n = pc->n_qubits;
    const uint64_t np = pinst.size();
    const uint64_t len = uint64_t{1} << n;

    std::vector<int> param_of(tmpl.size(), -1);
    for (uint64_t p = 0; p < np; ++p) param_of[pinst[p]] = static_cast<int>(p);

    // States smaller than one lane chunk use the per-set dense path: bind and evolve.
    if (n < 5) {
        auto st = new_state(n, 1, nullptr);
        auto lam = new_state(n, 1, nullptr);
        FusionConfig none;
        none.fuse = false;
        DeviceBuffer part, d_out;
        HamiltonianDev ham;
        ham.upload(h, n);
        for (uint64_t b = 0; b < batch; ++b) {
            const double* th = params + b * np;
            std::vector<GateDesc> bound = bind_params(tmpl, pinst, th);
            launch_set_basis(st->ctx, st->d(), n, 1, 0);
            apply_circuit(*st, bound, none);
            // lambda = H psi
            if (ham.n_terms == 0) cuda_check(cudaMemset(lam->d(), 0, sizeof(double2) * len), "memset");
            else launch_apply_hamiltonian(st->ctx, st->d(), lam->d(), n, 1,
                                          ham.terms.as<PauliTermDev>(), ham.groups.as<uint32_t>());
            part.ensure(sizeof(double) * 128);
            d_out.ensure(sizeof(double) * (np + 1));
            launch_batched_inner_re_p(st->ctx, st->d(), lam->d(), n, 1, part.as<double>(),
                                      d_out.as<double>() + np);
            for (size_t i = grad_out ? tmpl.size() : 0; i-- > 0;) {
                const GateDesc& g = bound[i];
                if (!g.is_unitary()) continue;
                if (param_of[i] >= 0) {
                    const PauliMasks m = generator(g);
                    launch_batched_pauli_im_p(st->ctx, lam->d(), st->d(), n, 1, m.x, m.zy, m.n_y,
                                              part.as<double>(), d_out.as<double>() + param_of[i], 1);
                }
                Program inv;
                std::vector<DevOp> ops{invert(lower_gate(g, n))};
                inv.build(std::move(ops), nullptr);
                inv.launch(st->ctx, st->d(), n, 1);
                inv.launch(st->ctx, lam->d(), n, 1);
            }
            std::vector<double> out(np + 1);
            cuda_check(cudaMemcpy(out.data(), d_out.ptr, sizeof(double) * (np + 1),
                                  cudaMemcpyDeviceToHost), "D2H gradients");
            if (energy_out) energy_out[b] = out[np];
            if (grad_out) std::copy(out.begin(), out.begin() + np, grad_out + b * np);
        }
        return;
    }

    AdjointPlan& plan = adjoint_plan(tmpl, param_of, h, n, np, batch, max_resident);
    const uint32_t R = plan.R;
    std::vector<double2> cs(np * R), csi(np * R);
    std::vector<double> h_energy(R), h_grad(np * R);
    for (uint64_t b0 = 0; b0 < batch; b0 += R) {
        const uint32_t nb = static_cast<uint32_t>(std::min<uint64_t>(R, batch - b0));
        // (cos, sin) of theta/2 per parameter and set; layout [param][set]
        for (uint64_t p = 0; p < np; ++p) {
            for (uint32_t b = 0; b < nb; ++b) {
                const double hh = params[(b0 + b) * np + p] / 2;
                cs[p * R + b] = make_double2(std::cos(hh), std::sin(hh));
                csi[p * R + b] = make_double2(std::cos(hh), -std::sin(hh));
            }
        }
        if (np) {
            cuda_check(cudaMemcpyAsync(plan.d_cs.ptr, cs.data(), sizeof(double2) * np * R,
                                       cudaMemcpyHostToDevice, plan.stream), "H2D");
            cuda_check(cudaMemcpyAsync(plan.d_csi.ptr, csi.data(), sizeof(double2) * np * R,
                                       cudaMemcpyHostToDevice, plan.stream), "H2D");
        }
        plan.run(nb, grad_out != nullptr);
        cuda_check(cudaMemcpyAsync(h_energy.data(), plan.d_energy.ptr, sizeof(double) * nb,
                                   cudaMemcpyDeviceToHost, plan.stream), "D2H energies");
        if (np && grad_out)
            cuda_check(cudaMemcpyAsync(h_grad.data(), plan.d_grad.ptr, sizeof(double) * np * nb,
                                       cudaMemcpyDeviceToHost, plan.stream), "D2H gradients");
        cuda_check(cudaStreamSynchronize(plan.stream), "adjoint");
        for (uint32_t b = 0; b < nb; ++b) {
            if (energy_out) energy_out[b0 + b] = h_energy[b];
            if (grad_out)
                std::copy(h_grad.begin() + b * np, h_grad.begin() + (b + 1) * np,
                          grad_out + (b0 + b) * np);
        }
    }
}

// ------------------------------------------------------------------ ragged batches

namespace {

// Problems of different qubit counts (each its own ansatz, Hamiltonian and parameter sets)
// in one CUDA graph: every problem keeps its plan and stream; the capture forks from an
// origin stream to all of them and joins back, so a call is one graph launch whose
// branches run concurrently — small states that leave most of the GPU idle on their own
// fill it together.
struct MultiPlan {
    uint64_t key = 0;
    std::vector<std::unique_ptr<AdjointPlan>> plans;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    bool direct = false;   // capture failed: launch the branches without a graph

    MultiPlan() = default;
    MultiPlan(const MultiPlan&) = delete;
    MultiPlan& operator=(const MultiPlan&) = delete;
    ~MultiPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        for (cudaEvent_t e : joins) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        plans.clear();
        if (origin) cudaStreamDestroy(origin);
    }

    void enqueue_all() {
        cuda_check(cudaEventRecord(fork, origin), "cudaEventRecord");
        for (size_t i = 0; i < plans.size(); ++i) {
            cuda_check(cudaStreamWaitEvent(plans[i]->stream, fork, 0), "cudaStreamWaitEvent");
            plans[i]->enqueue(plans[i]->R);
            cuda_check(cudaEventRecord(joins[i], plans[i]->stream), "cudaEventRecord");
            cuda_check(cudaStreamWaitEvent(origin, joins[i], 0), "cudaStreamWaitEvent");
        }
    }

    void run() {
        const char* e = std::getenv("LQCS_GRAPHS");
        if (direct || (e && e[0] == '0')) {
            enqueue_all();
            return;
        }
        if (!exec) {
            const uint64_t k0 = launch_count();
            cudaGraph_t g = nullptr;
            bool ok = cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                try {
                    enqueue_all();
                } catch (...) {
                    ok = false;
                }
                cudaGraph_t done = nullptr;
                const bool ended = cudaStreamEndCapture(origin, &done) == cudaSuccess;
                g = done;
                ok = ok && ended && g;
            }
            if (ok) ok = cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
            if (!ok) {
                cudaGetLastError();
                exec = nullptr;
                direct = true;
                enqueue_all();
                return;
            }
            kernels = launch_count() - k0;
            cuda_check(cudaGraphLaunch(exec, origin), "cudaGraphLaunch");
            return;   // the capture counted this call's kernels
        }
        cuda_check(cudaGraphLaunch(exec, origin), "cudaGraphLaunch");
        count_launch(kernels);
    }
};

std::mutex g_multi_mu;
std::vector<std::unique_ptr<MultiPlan>> g_multi;

struct Problem {
    std::vector<GateDesc> tmpl;
    std::vector<uint64_t> pinst;
    std::vector<int> param_of;
    Hamiltonian h;
    uint32_t n = 0;
};

}  // namespace

void adjoint_batched_multi(uint64_t n_problems, const lqcs_parametric_circuit* const* pcs,
                           const lqcs_hamiltonian* const* hs, const double* const* params,
                           const uint64_t* batches, double* const* energy_out,
                           double* const* grad_out) {
    if (n_problems == 0) return;
    if (!pcs || !hs || !params || !batches) invalid("adjoint_gradient_multi: null arrays");
    std::vector<Problem> probs(n_problems);
    double need = 0.0;
    bool fused = true;
    for (uint64_t p = 0; p < n_problems; ++p) {
        if (!pcs[p]) invalid("adjoint_gradient_multi: parametric circuit is null");
        Problem& q = probs[p];
        check_pc(pcs[p], q.tmpl, q.pinst);
        q.n = pcs[p]->n_qubits;
        q.h = decode_hamiltonian(hs[p], q.n);
        q.param_of.assign(q.tmpl.size(), -1);
        for (uint64_t i = 0; i < q.pinst.size(); ++i) q.param_of[q.pinst[i]] = static_cast<int>(i);
        if (batches[p] > 0 && !params[p] && !q.pinst.empty()) invalid("adjoint_gradient_multi: params is null");
        need += 2.0 * static_cast<double>(batches[p]) * 16.0 * std::ldexp(1.0, static_cast<int>(q.n));
        fused &= q.n >= 5 && batches[p] > 0;
    }
    size_t free_b = 0, total_b = 0;
    cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    if (!fused || need > 0.5 * static_cast<double>(free_b)) {
        // one problem after another (each still batched)
        for (uint64_t p = 0; p < n_problems; ++p)
            adjoint_batched(pcs[p], probs[p].h, params[p], batches[p], 0,
                            energy_out ? energy_out[p] : nullptr, grad_out ? grad_out[p] : nullptr);
        return;
    }
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::vector<uint64_t> keys(n_problems);
    uint64_t mkey = 1469598103934665603ull ^ (static_cast<uint64_t>(dev) << 56);
    for (uint64_t p = 0; p < n_problems; ++p) {
        keys[p] = plan_key(probs[p].tmpl, probs[p].param_of, probs[p].h, probs[p].n,
                           static_cast<uint32_t>(batches[p])) ^ (static_cast<uint64_t>(dev) << 56);
        mkey = (mkey ^ keys[p]) * 1099511628211ull;
    }
    std::lock_guard<std::mutex> lk(g_multi_mu);
    MultiPlan* mp = nullptr;
    for (auto& m : g_multi)
        if (m->key == mkey) mp = m.get();
    if (!mp) {
        auto m = std::make_unique<MultiPlan>();
        m->key = mkey;
        cuda_check(cudaStreamCreateWithFlags(&m->origin, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_check(cudaEventCreateWithFlags(&m->fork, cudaEventDisableTiming), "cudaEventCreate");
        for (uint64_t p = 0; p < n_problems; ++p) {
            m->plans.push_back(build_plan(probs[p].tmpl, probs[p].param_of, probs[p].h, probs[p].n,
                                          probs[p].pinst.size(), static_cast<uint32_t>(batches[p]),
                                          keys[p]));
            cudaEvent_t ev = nullptr;
            cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
            m->joins.push_back(ev);
        }
        if (g_multi.size() >= kKeptPlans) g_multi.erase(g_multi.begin());
        g_multi.push_back(std::move(m));
        mp = g_multi.back().get();
    }
    // (cos, sin) tables of every problem, uploaded in order on the origin stream
    std::vector<std::vector<double2>> tabs(2 * n_problems);
    for (uint64_t p = 0; p < n_problems; ++p) {
        const AdjointPlan& pl = *mp->plans[p];
        const uint64_t np = pl.np, R = pl.R;
        std::vector<double2>& cs = tabs[2 * p];
        std::vector<double2>& csi = tabs[2 * p + 1];
        cs.resize(np * R);
        csi.resize(np * R);
        for (uint64_t k = 0; k < np; ++k) {
            for (uint64_t b = 0; b < R; ++b) {
                const double hh = params[p][b * np + k] / 2;
                cs[k * R + b] = make_double2(std::cos(hh), std::sin(hh));
                csi[k * R + b] = make_double2(std::cos(hh), -std::sin(hh));
            }
        }
        if (np) {
            cuda_check(cudaMemcpyAsync(pl.d_cs.ptr, cs.data(), sizeof(double2) * np * R,
                                       cudaMemcpyHostToDevice, mp->origin), "H2D");
            cuda_check(cudaMemcpyAsync(pl.d_csi.ptr, csi.data(), sizeof(double2) * np * R,
                                       cudaMemcpyHostToDevice, mp->origin), "H2D");
        }
    }
    mp->run();
    for (uint64_t p = 0; p < n_problems; ++p) {
        const AdjointPlan& pl = *mp->plans[p];
        if (energy_out && energy_out[p])
            cuda_check(cudaMemcpyAsync(energy_out[p], pl.d_energy.ptr, sizeof(double) * pl.R,
                                       cudaMemcpyDeviceToHost, mp->origin), "D2H energies");
        if (grad_out && grad_out[p] && pl.np)
            cuda_check(cudaMemcpyAsync(grad_out[p], pl.d_grad.ptr, sizeof(double) * pl.np * pl.R,
                                       cudaMemcpyDeviceToHost, mp->origin), "D2H gradients");
    }
    cuda_check(cudaStreamSynchronize(mp->origin), "adjoint_gradient_multi");
}

void release_adjoint_plans() {
    {
        std::lock_guard<std::mutex> lk(g_multi_mu);
        g_multi.clear();
    }
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plans.clear();
}

}  // namespace lqcs_b200
