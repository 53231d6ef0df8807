// tile_plan.cpp — planning of shared-memory tile passes.
//
// A pass is a set H of high qubits plus the gates it applies.  First-fit over the gates in
// program order: a gate joins the pass when its targets above bit L fit into H (growing H up
// to h qubits) and none of its qubits is blocked; otherwise it is deferred and its qubits
// become blocked, so every later gate on them is deferred too and program order on each
// qubit is kept.  Controls and phase bits need no tile slot (they are constant over a tile
// or select the amplitudes a phase multiplies).  Inside a pass, neighbouring gates on tile
// qubits are fused into dense operations of at most `inner` qubits.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <tuple>

#include "tile_plan.hpp"

namespace lqcs_b200 {

namespace {

bool is_phase_gate(const GateDesc& g) {
    if (g.slot || !g.is_unitary() || g.base_qubits() != 1) return false;
    if (g.type == LQCS_GATE_PAULI_ROTATION) return false;
    const std::vector<cd> m = g.base_matrix();
    return m[1] == cd{0, 0} && m[2] == cd{0, 0} && m[0] == cd{1, 0};
}

int env_int(const char* name, int dflt) {
    if (const char* e = std::getenv(name)) return std::atoi(e);
    return dflt;
}

}  // namespace

TileConfig default_tile_config(uint32_t n) {
    TileConfig c;
    c.m = static_cast<uint32_t>(env_int("LQCS_TILE_BITS", 12));
    c.L = static_cast<uint32_t>(env_int("LQCS_TILE_LOW", 5));
    c.inner = static_cast<uint32_t>(env_int("LQCS_TILE_INNER", 2));
    c.reg = env_int("LQCS_TILE_REG", 1) != 0;
    c.search = env_int("LQCS_TILE_SEARCH", 1) != 0;
    c.mma = env_int("LQCS_REG_MMA", 0) != 0;
    c.pauli = env_int("LQCS_TILE_PAULI", 1) != 0;
    c.m = std::max<uint32_t>(kTileMinBits, std::min<uint32_t>(std::min<uint32_t>(c.m, kTileMaxBits), n));
    c.L = std::min<uint32_t>(std::min(c.L, c.m), kTileMinBits);   // column bits come from the thread index
    if (c.m - c.L > kTileMaxHigh) c.L = c.m - kTileMaxHigh;
    c.inner = std::max<uint32_t>(1, std::min<uint32_t>(c.inner, kTileMaxK));
    return c;
}

bool native_pauli(const GateDesc& g, const TileConfig& cfg) {
    if (!cfg.reg || !cfg.pauli || g.type != LQCS_GATE_PAULI_ROTATION || g.n_controls != 0 || g.slot)
        return false;
    uint32_t flips = 0;
    for (char ch : g.pauli) flips += ch == 'X' || ch == 'Y';
    return flips <= kRegPauliMaxFlips;
}

// Qubits a gate needs inside the tile, or false if it cannot run in a tile at all.  A native
// Pauli rotation needs only its X/Y qubits there (its Z-type qubits act through parities).
static bool tile_requirements(const GateDesc& g, const TileConfig& c, std::vector<uint32_t>& need) {
    need.clear();
    if (native_pauli(g, c)) {
        const uint32_t k = g.base_qubits();
        for (uint32_t j = 0; j < k; ++j) {
            const char ch = g.pauli[k - 1 - j];   // local bit j <-> pauli[k-1-j] (Gate::pauli_masks)
            if (ch == 'X' || ch == 'Y') need.push_back(g.targets()[j]);
        }
        return true;
    }
    if (is_phase_gate(g)) return g.qubits.size() <= 8;   // at most 8 local phase bits
    const uint32_t k = g.base_qubits();
    if (k == 0 || k > kTileMaxK) return false;
    if (g.type == LQCS_GATE_PERMUTATION && k > kTileMaxK) return false;
    if (k + g.n_controls > 8) return false;
    for (uint32_t j = 0; j < k; ++j) need.push_back(g.targets()[j]);
    (void)c;
    return true;
}

// First-fit picks the high tile qubits in the order gates ask for them, which is often not
// the set that takes the most gates.  Local search: swap one high qubit of the pass for one
// outside it while that lets the pass take more gates (same rules as the first-fit scan:
// program order per qubit, barriers end the pass, at most kTileMaxOps gates).  On the
// 30-qubit brickwork this cuts 75 passes to about 50.
static void improve_high_bits(const std::vector<GateDesc>& gates, uint32_t n, const TileConfig& cfg,
                              const std::vector<uint32_t>& remaining, std::vector<uint32_t>& hset,
                              std::vector<uint32_t>& taken, std::vector<uint32_t>& deferred) {
    struct G {
        uint64_t qubits, need;   // all qubits; high qubits the gate needs in the tile
        bool ok, barrier;
    };
    std::vector<G> gs;
    gs.reserve(remaining.size());
    std::vector<uint32_t> need;
    for (uint32_t gi : remaining) {
        const GateDesc& g = gates[gi];
        G e{0, 0, false, g.type == LQCS_GATE_BARRIER};
        for (uint32_t q : g.qubits) e.qubits |= uint64_t{1} << q;
        if (!e.barrier && tile_requirements(g, cfg, need)) {
            e.ok = true;
            for (uint32_t q : need)
                if (q >= cfg.L) e.need |= uint64_t{1} << q;
        }
        gs.push_back(e);
    }
    auto count = [&](uint64_t hmask) {
        uint64_t blocked = 0;
        size_t got = 0;
        for (const G& e : gs) {
            if (e.barrier || got >= kTileMaxOps) break;
            if (!(e.qubits & blocked) && e.ok && !(e.need & ~hmask)) ++got;
            else blocked |= e.qubits;
        }
        return got;
    };
    uint64_t hmask = 0;
    for (uint32_t q : hset) hmask |= uint64_t{1} << q;
    // with the padded set fixed the scan takes every gate first-fit took (and maybe more)
    size_t best = count(hmask);
    for (int round = 0; round < 8; ++round) {
        bool better = false;
        for (uint32_t out = cfg.L; out < n; ++out) {
            if (!((hmask >> out) & 1)) continue;
            for (uint32_t in = cfg.L; in < n; ++in) {
                if ((hmask >> in) & 1) continue;
                const uint64_t cand = (hmask & ~(uint64_t{1} << out)) | (uint64_t{1} << in);
                const size_t c = count(cand);
                if (c > best) {
                    best = c;
                    hmask = cand;
                    better = true;
                    break;
                }
            }
        }
        if (!better) break;
    }
    hset.clear();
    for (uint32_t q = cfg.L; q < n; ++q)
        if ((hmask >> q) & 1) hset.push_back(q);
    taken.clear();
    deferred.clear();
    uint64_t blocked = 0;
    bool stop = false;
    for (size_t i = 0; i < gs.size(); ++i) {
        const G& e = gs[i];
        if (stop || e.barrier || taken.size() >= kTileMaxOps) {
            stop = true;
            deferred.push_back(remaining[i]);
            continue;
        }
        if (!(e.qubits & blocked) && e.ok && !(e.need & ~hmask)) {
            taken.push_back(remaining[i]);
        } else {
            deferred.push_back(remaining[i]);
            blocked |= e.qubits;
        }
    }
}

std::vector<PlanItem> plan_tiles(const std::vector<GateDesc>& gates, uint32_t n,
                                 const TileConfig& cfg) {
    std::vector<PlanItem> items;
    const uint32_t h = cfg.m - cfg.L;
    std::vector<uint32_t> remaining;
    for (uint32_t i = 0; i < gates.size(); ++i) {
        if (gates[i].type == LQCS_GATE_BARRIER) {
            remaining.push_back(i);
            continue;
        }
        if (gates[i].is_unitary()) remaining.push_back(i);
    }
    std::vector<uint32_t> need;
    std::vector<char> blocked(n, 0);
    while (!remaining.empty()) {
        // a barrier at the front closes nothing (there is no open pass): drop it
        if (gates[remaining.front()].type == LQCS_GATE_BARRIER) {
            remaining.erase(remaining.begin());
            continue;
        }
        std::vector<uint32_t> hset;
        std::vector<uint32_t> taken, deferred;
        std::fill(blocked.begin(), blocked.end(), 0);
        bool stop = false;
        for (uint32_t gi : remaining) {
            const GateDesc& g = gates[gi];
            if (stop || g.type == LQCS_GATE_BARRIER || taken.size() >= kTileMaxOps) {
                // a barrier ends the pass: everything from here waits for the next one
                stop = true;
                deferred.push_back(gi);
                continue;
            }
            bool blk = false;
            for (uint32_t q : g.qubits) blk |= blocked[q] != 0;
            bool ok = !blk && tile_requirements(g, cfg, need);
            if (ok) {
                std::vector<uint32_t> add;
                for (uint32_t q : need)
                    if (q >= cfg.L && std::find(hset.begin(), hset.end(), q) == hset.end() &&
                        std::find(add.begin(), add.end(), q) == add.end())
                        add.push_back(q);
                ok = hset.size() + add.size() <= h;
                if (ok) hset.insert(hset.end(), add.begin(), add.end());
            }
            if (ok) {
                taken.push_back(gi);
            } else {
                deferred.push_back(gi);
                for (uint32_t q : g.qubits) blocked[q] = 1;
            }
        }
        if (taken.empty()) {
            // the first gate cannot run in a tile: run it on its own
            PlanItem it;
            it.is_pass = false;
            it.gate = remaining.front();
            items.push_back(std::move(it));
            remaining.erase(remaining.begin());
            continue;
        }
        // every pass gets the full tile size: pad H with unused high qubits
        for (uint32_t q = cfg.L; q < n && hset.size() < h; ++q)
            if (std::find(hset.begin(), hset.end(), q) == hset.end()) hset.push_back(q);
        if (cfg.search && n <= 64) improve_high_bits(gates, n, cfg, remaining, hset, taken, deferred);
        PlanItem it;
        it.is_pass = true;
        std::sort(hset.begin(), hset.end());
        it.hbits = hset;
        it.gates = taken;
        items.push_back(std::move(it));
        remaining = std::move(deferred);
    }
    return items;
}

// ------------------------------------------------------------------ lowering

namespace {

struct LocalMap {
    uint32_t L;
    std::vector<uint32_t> hbits;
    // tile bit of qubit q, where a relabelling (virtual SWAP) has moved it; -1: none
    std::vector<std::pair<uint32_t, uint32_t>> moved;
    int home(uint32_t q) const {   // tile bit at load, -1 if outside the tile
        if (q < L) return static_cast<int>(q);
        const auto it = std::find(hbits.begin(), hbits.end(), q);
        return it == hbits.end() ? -1 : static_cast<int>(L + (it - hbits.begin()));
    }
    int local(uint32_t q) const {   // -1 if outside the tile
        for (const auto& [qq, b] : moved)
            if (qq == q) return static_cast<int>(b);
        return home(q);
    }
    void swap_bits(uint32_t a, uint32_t b) {
        const uint32_t la = static_cast<uint32_t>(local(a)), lb = static_cast<uint32_t>(local(b));
        auto set = [&](uint32_t q, uint32_t bit) {
            for (auto& e : moved)
                if (e.first == q) {
                    e.second = bit;
                    return;
                }
            moved.emplace_back(q, bit);
        };
        set(a, lb);
        set(b, la);
    }
};

uint32_t deposit(uint32_t v, const std::vector<uint32_t>& sorted_pos) {
    for (uint32_t p : sorted_pos) {
        const uint32_t low = (1u << p) - 1u;
        v = ((v & ~low) << 1) | (v & low);
    }
    return v;
}

bool is_diagonal(const std::vector<cd>& m, uint64_t dim) {
    for (uint64_t r = 0; r < dim; ++r)
        for (uint64_t c = 0; c < dim; ++c)
            if (r != c && m[r * dim + c] != cd{0, 0}) return false;
    return true;
}

// Dense or diagonal op of matrix m on local targets lt, local controls lcmask.
LocalOp matrix_op(const std::vector<cd>& m, const std::vector<uint32_t>& lt, uint32_t lcmask,
                  uint64_t gcmask, bool variant) {
    LocalOp op;
    const uint64_t dim = uint64_t{1} << lt.size();
    op.lt = lt;
    op.lmask = lcmask;
    op.gcmask = gcmask;
    op.variant = variant;
    if (!variant && is_diagonal(m, dim)) {
        op.kind = kTileDiag;
        for (uint64_t i = 0; i < dim; ++i) op.m.push_back(m[i * dim + i]);
    } else {
        op.kind = kTileDense;
        op.m = m;
    }
    return op;
}

// Group enumeration of an op on a 2^m tile: the positions spread over (ascending), the
// group count, and the per-iteration slot parts sw(deposit(j * threads) | lcmask).
void set_groups(TileOp& op, std::vector<uint32_t> pos, uint32_t lcmask, uint32_t m) {
    std::sort(pos.begin(), pos.end());
    op.n_fixed = static_cast<uint8_t>(pos.size());
    for (size_t i = 0; i < pos.size(); ++i) op.fixed[i] = static_cast<uint8_t>(pos[i]);
    const uint32_t groups = (1u << m) >> pos.size();
    op.n_groups = static_cast<uint16_t>(groups);
    op.iters = static_cast<uint16_t>(std::max<uint32_t>(1, groups / kTileThreads));
    for (uint32_t j = 0; j < op.iters; ++j)
        op.dhi[j] = static_cast<uint16_t>(tile_swizzle(deposit(j * kTileThreads, pos) | lcmask));
}

bool is_x(const std::vector<cd>& m) {
    return m.size() == 4 && m[0] == cd{0, 0} && m[1] == cd{1, 0} && m[2] == cd{1, 0} &&
           m[3] == cd{0, 0};
}

}  // namespace

double local_op_flops(const LocalOp& o, bool x_free) {
    if (o.kind == kTilePauli) return o.lt.empty() ? 6.0 : 16.0;   // op_flops_per_amp of PAULI
    const double frac = std::ldexp(1.0, -(__builtin_popcount(o.lmask) + __builtin_popcountll(o.gcmask)));
    if (o.kind != kTileDense) return 6.0 * frac;
    if (x_free && !o.variant && o.lt.size() == 1 && o.sel.empty() && is_x(o.m)) return 0.0;
    return 8.0 * std::ldexp(1.0, static_cast<int>(o.lt.size())) * frac;
}

// Matrix of a 2^k dense op with a one-qubit matrix applied first on its target bit j:
// M' = M (I (x) .. u .. (x) I).  Both sides may carry selector blocks: `ms` / `us` give the
// bit of each op's selector qubit within the merged selector set.
static void fold_into(LocalOp& q, const LocalOp& p, uint32_t j, const std::vector<uint32_t>& sel,
                      bool after = false) {
    const uint32_t k = static_cast<uint32_t>(q.lt.size());
    const uint64_t D = uint64_t{1} << k;
    const uint32_t nsel = static_cast<uint32_t>(sel.size());
    auto index_of = [&](const std::vector<uint32_t>& own, uint32_t sv) {
        uint32_t idx = 0;
        for (size_t i = 0; i < own.size(); ++i) {
            const uint32_t pos = static_cast<uint32_t>(std::find(sel.begin(), sel.end(), own[i]) - sel.begin());
            if ((sv >> pos) & 1) idx |= 1u << i;
        }
        return idx;
    };
    std::vector<cd> out;
    for (uint32_t sv = 0; sv < (1u << nsel); ++sv) {
        const cd* m = q.m.data() + static_cast<size_t>(index_of(q.sel, sv)) * D * D;
        std::array<cd, 4> u{};
        const uint32_t pi = index_of(p.sel, sv);
        if (p.kind == kTileDiag) {
            u = {p.m[2 * pi], cd{0, 0}, cd{0, 0}, p.m[2 * pi + 1]};
        } else {
            for (int e = 0; e < 4; ++e) u[e] = p.m[4 * pi + e];
        }
        for (uint64_t r = 0; r < D; ++r) {
            for (uint64_t c = 0; c < D; ++c) {
                cd acc{0, 0};
                if (after) {
                    // (U M)[r][c] = sum_x U[r_j][x] M[r with bit j = x][c]
                    const uint64_t rj = (r >> j) & 1, r0 = r & ~(uint64_t{1} << j);
                    for (uint64_t xj = 0; xj < 2; ++xj)
                        acc += u[rj * 2 + xj] * m[(r0 | xj << j) * D + c];
                } else {
                    // (M U)[r][c] = sum_x M[r][x] U[x][c]; U acts on bit j only
                    const uint64_t cj = (c >> j) & 1, c0 = c & ~(uint64_t{1} << j);
                    for (uint64_t xj = 0; xj < 2; ++xj)
                        acc += m[r * D + (c0 | xj << j)] * u[xj * 2 + cj];
                }
                out.push_back(acc);
            }
        }
    }
    q.m = std::move(out);
    q.sel = sel;
}

// Diagonal form of a phase or diagonal op without local controls: local bits (ascending)
// and the 2^k entries.  A phase multiplies where all its bits are 1.
static bool diagonal_form(const LocalOp& o, std::vector<uint32_t>& bits, std::vector<cd>& d) {
    if (o.variant || !o.sel.empty() || !o.dyn.empty()) return false;
    if (o.kind == kTilePhase) {
        bits.clear();
        for (uint32_t b = 0; b < 32; ++b)
            if ((o.lmask >> b) & 1) bits.push_back(b);
        d.assign(size_t{1} << bits.size(), cd{1, 0});
        d.back() = o.m[0];
        return true;
    }
    if (o.kind != kTileDiag || o.lmask) return false;
    // entries in local order (bit j <-> lt[j]); re-index to ascending bits
    std::vector<uint32_t> order(o.lt.size());
    for (size_t j = 0; j < order.size(); ++j) order[j] = static_cast<uint32_t>(j);
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return o.lt[a] < o.lt[b]; });
    bits.clear();
    for (uint32_t j : order) bits.push_back(o.lt[j]);
    const size_t D = size_t{1} << bits.size();
    d.assign(D, cd{1, 0});
    for (size_t e = 0; e < D; ++e) {
        size_t src = 0;
        for (size_t q = 0; q < order.size(); ++q)
            if ((e >> q) & 1) src |= size_t{1} << order[q];
        d[e] = o.m[src];
    }
    return true;
}

// Product of two diagonals given over ascending tile bits: the table over the union.
static void mul_tables(std::vector<uint32_t>& bi, std::vector<cd>& di, const std::vector<uint32_t>& bj,
                       const std::vector<cd>& dj) {
    uint32_t uni = 0;
    for (uint32_t b : bi) uni |= 1u << b;
    for (uint32_t b : bj) uni |= 1u << b;
    std::vector<uint32_t> ub;
    for (uint32_t b = 0; b < 32; ++b)
        if ((uni >> b) & 1) ub.push_back(b);
    std::vector<cd> du(size_t{1} << ub.size());
    for (size_t e = 0; e < du.size(); ++e) {
        size_t ei = 0, ej = 0;
        for (size_t q = 0; q < ub.size(); ++q) {
            if (!((e >> q) & 1)) continue;
            const auto pi = std::find(bi.begin(), bi.end(), ub[q]);
            if (pi != bi.end()) ei |= size_t{1} << (pi - bi.begin());
            const auto pj = std::find(bj.begin(), bj.end(), ub[q]);
            if (pj != bj.end()) ej |= size_t{1} << (pj - bj.begin());
        }
        du[e] = di[ei] * dj[ej];
    }
    bi = std::move(ub);
    di = std::move(du);
}

// Runs of diagonal work (phases such as the controlled phases of a QFT, diagonal blocks)
// become one diagonal table over the union of their tile bits: an op joins an earlier
// diagonal op when every op in between commutes with it (no dense target on its bits) and
// the union stays within max_bits.  Ops with the same out-of-tile predicate merge into the
// table itself.  With dyn_terms a phase gated by other out-of-tile qubits joins as a term
// that the kernel multiplies into the table at the start of each tile where those qubits are
// all 1 (a group whose own predicate differs turns into such terms when it is made of phases
// only).  Each merge removes a pass over the tile's amplitudes for a table entry lookup.
static void merge_diagonal_runs(std::vector<LocalOp>& ops, uint32_t max_bits, bool dyn_terms) {
    std::vector<char> dead(ops.size(), 0);
    std::vector<uint32_t> bi, bj;
    std::vector<cd> di, dj;
    uint32_t dyn_groups = 0, dyn_entries = 0;
    auto mask_of = [](const std::vector<uint32_t>& bits) {
        uint32_t mk = 0;
        for (uint32_t b : bits) mk |= 1u << b;
        return mk;
    };
    for (size_t i = 0; i < ops.size(); ++i) {
        if (dead[i] || !diagonal_form(ops[i], bi, di)) continue;
        uint64_t gc = ops[i].gcmask;
        std::vector<DynTerm> dyn;
        std::vector<DynTerm> phases;   // the group as phase terms while it is made of phases
        bool only_phases = ops[i].kind == kTilePhase;
        if (only_phases) phases.push_back({gc, ops[i].lmask, ops[i].m[0]});
        uint32_t merged = 0;
        uint32_t blocked = 0;   // tile bits a dense op between i and j targets
        for (size_t j = i + 1; j < ops.size(); ++j) {
            if (dead[j]) continue;
            const LocalOp& q = ops[j];
            if (diagonal_form(q, bj, dj)) {
                const uint32_t mj = mask_of(bj);
                const uint32_t uni = mask_of(bi) | mj;
                const uint32_t width = static_cast<uint32_t>(__builtin_popcount(uni));
                const bool fits = !(mj & blocked) && width <= max_bits &&
                                  (dyn.empty() || dyn_entries + (1u << width) <= kRegMaxDynEntries);
                if (fits && q.gcmask == gc) {
                    mul_tables(bi, di, bj, dj);
                    if (q.kind == kTilePhase) phases.push_back({q.gcmask, q.lmask, q.m[0]});
                    else only_phases = false;
                    dead[j] = 1;
                    ++merged;
                    continue;
                }
                // a gated phase as a per-tile term (table entries within the pass's budget)
                const bool room = dyn_entries + (1u << width) <= kRegMaxDynEntries &&
                                  (!dyn.empty() || dyn_groups < kRegMaxDyn) &&
                                  dyn.size() + (gc ? phases.size() : 0) < kRegMaxDynTerms;
                if (fits && dyn_terms && q.kind == kTilePhase && room && (gc == 0 || only_phases)) {
                    if (gc != 0) {   // the group so far becomes terms over an identity table
                        dyn = phases;
                        std::fill(di.begin(), di.end(), cd{1, 0});
                        gc = 0;
                    }
                    const std::vector<cd> ones(size_t{1} << bj.size(), cd{1, 0});
                    mul_tables(bi, di, bj, ones);
                    if (q.gcmask) dyn.push_back({q.gcmask, q.lmask, q.m[0]});
                    else mul_tables(bi, di, bj, dj);
                    phases.push_back({q.gcmask, q.lmask, q.m[0]});
                    dead[j] = 1;
                    ++merged;
                    continue;
                }
            }
            // q stays: later diagonal work may pass it only on bits it does not target
            if (q.kind == kTileDense || q.kind == kTilePauli)
                for (uint32_t b : q.lt) blocked |= 1u << b;
        }
        if (!merged) continue;   // a lone op keeps its own (cheaper) form
        LocalOp& o = ops[i];
        o.kind = kTileDiag;
        o.lt = bi;
        o.lmask = 0;
        o.gcmask = gc;
        o.m = di;
        o.dyn = std::move(dyn);
        if (!o.dyn.empty()) {
            ++dyn_groups;
            dyn_entries += 1u << o.lt.size();
        }
    }
    size_t w = 0;
    for (size_t i = 0; i < ops.size(); ++i) {
        if (dead[i]) continue;
        if (w != i) ops[w] = std::move(ops[i]);
        ++w;
    }
    ops.resize(w);
}

// Peephole after inner fusion: a one-qubit dense or diagonal op (no controls) moves into the
// next op touching its qubit — or, failing that, the previous one — when that op is a dense
// block on it without controls (the ops in between do not touch the qubit, so they commute
// with it): the block's matrix absorbs it at no extra cost per amplitude and one operation
// disappears.  A noise slot (per-state matrix) folds too: the block becomes per-state.
static void fold_single_qubit_ops(std::vector<LocalOp>& ops, uint32_t max_select) {
    std::vector<char> dead(ops.size(), 0);
    for (size_t i = 0; i < ops.size(); ++i) {
        // a phase on one tile bit (such as K0 of amplitude damping) folds as the diagonal
        // (1, f); if it does not fold it keeps its phase form
        LocalOp as_diag;
        const bool one_bit_phase = ops[i].kind == kTilePhase && !ops[i].gcmask &&
                                   ops[i].sel.empty() && __builtin_popcount(ops[i].lmask) == 1;
        if (one_bit_phase) {
            as_diag.kind = kTileDiag;
            as_diag.lt = {static_cast<uint32_t>(__builtin_ctz(ops[i].lmask))};
            as_diag.m = {cd{1, 0}, ops[i].m[0]};
        }
        const LocalOp& p = one_bit_phase ? as_diag : ops[i];
        if (p.kind == kTilePhase || p.kind == kTilePauli || p.lt.size() != 1 || p.lmask ||
            p.gcmask || !p.dyn.empty())
            continue;
        const uint32_t a = p.lt[0];
        for (size_t j = i + 1; j < ops.size(); ++j) {
            if (dead[j]) continue;
            LocalOp& q = ops[j];
            const bool touches = ((q.lmask >> a) & 1) ||
                                 std::find(q.lt.begin(), q.lt.end(), a) != q.lt.end();
            if (!touches) continue;
            const auto it = std::find(q.lt.begin(), q.lt.end(), a);
            if (q.kind == kTileDense && it != q.lt.end() && !q.lmask && !q.gcmask) {
                std::vector<uint32_t> sel = q.sel;
                for (uint32_t s : p.sel)
                    if (std::find(sel.begin(), sel.end(), s) == sel.end()) sel.push_back(s);
                std::sort(sel.begin(), sel.end());
                if (sel.size() <= max_select || (p.sel.empty() && q.sel.size() <= max_select)) {
                    fold_into(q, p, static_cast<uint32_t>(it - q.lt.begin()), sel);
                    q.variant = q.variant || p.variant;
                    dead[i] = 1;
                }
            }
            break;   // only the next op on the qubit
        }
        if (dead[i]) continue;
        for (size_t j = i; j-- > 0;) {
            if (dead[j]) continue;
            LocalOp& q = ops[j];
            const bool touches = ((q.lmask >> a) & 1) ||
                                 std::find(q.lt.begin(), q.lt.end(), a) != q.lt.end();
            if (!touches) continue;
            const auto it = std::find(q.lt.begin(), q.lt.end(), a);
            if (q.kind == kTileDense && it != q.lt.end() && !q.lmask && !q.gcmask) {
                std::vector<uint32_t> sel = q.sel;
                for (uint32_t s : p.sel)
                    if (std::find(sel.begin(), sel.end(), s) == sel.end()) sel.push_back(s);
                std::sort(sel.begin(), sel.end());
                if (sel.size() <= max_select || (p.sel.empty() && q.sel.size() <= max_select)) {
                    fold_into(q, p, static_cast<uint32_t>(it - q.lt.begin()), sel, true);
                    q.variant = q.variant || p.variant;
                    dead[i] = 1;
                }
            }
            break;   // only the previous op on the qubit
        }
    }
    size_t w = 0;
    for (size_t i = 0; i < ops.size(); ++i) {
        if (dead[i]) continue;
        if (w != i) ops[w] = std::move(ops[i]);
        ++w;
    }
    ops.resize(w);
}

std::vector<LocalOp> pass_local_ops(const PlanItem& item, const std::vector<GateDesc>& gates,
                                    const TileConfig& cfg, uint32_t max_select,
                                    const std::vector<std::array<cd, 4>>* slot_mats,
                                    uint32_t max_diag, bool dyn_terms,
                                    std::vector<uint32_t>* store_qubits, bool native_rotations) {
    LocalMap lm{cfg.L, item.hbits, {}};
    std::vector<LocalOp> out;
    // a noise slot takes this state's matrix (identity when no table is given)
    auto resolved = [&](const GateDesc& g) {
        GateDesc r = g;
        if (g.slot) {
            r.type = LQCS_GATE_UNITARY;
            r.mat.assign(4, cd{0, 0});
            r.mat[0] = r.mat[3] = 1.0;
            if (slot_mats) r.mat.assign((*slot_mats)[g.slot_id].begin(), (*slot_mats)[g.slot_id].end());
        }
        return r;
    };
    // inner fusion: greedy blocks of at most cfg.inner local qubits (targets and local
    // controls) and at most max_select out-of-tile controls; any other gate closes the
    // blocks it touches and is emitted on its own
    struct Open {
        std::vector<uint32_t> qubits;   // local part, global numbering, sorted
        std::vector<uint32_t> sel;      // out-of-tile controls, sorted
        std::vector<uint32_t> gates;
        bool alive = true;
    };
    std::vector<Open> open;
    std::vector<int> owner(64, -1);
    auto emit_single = [&](const GateDesc& g) {
        if (is_phase_gate(g)) {
            LocalOp op;
            op.kind = kTilePhase;
            for (uint32_t q : g.qubits) {
                const int l = lm.local(q);
                if (l >= 0) op.lmask |= 1u << l;
                else op.gcmask |= uint64_t{1} << q;
            }
            op.m.push_back(g.base_matrix()[3]);
            out.push_back(std::move(op));
            return;
        }
        std::vector<uint32_t> lt;
        for (uint32_t j = 0; j < g.base_qubits(); ++j)
            lt.push_back(static_cast<uint32_t>(lm.local(g.targets()[j])));
        uint32_t lc = 0;
        uint64_t gc = 0;
        for (uint32_t c = 0; c < g.n_controls; ++c) {
            const uint32_t q = g.controls()[c];
            const int l = lm.local(q);
            if (l >= 0) lc |= 1u << l;
            else gc |= uint64_t{1} << q;
        }
        out.push_back(matrix_op(resolved(g).base_matrix(), lt, lc, gc, g.slot));
    };
    auto emit_block = [&](Open& b) {
        if (!b.alive) return;
        b.alive = false;
        for (uint32_t q : b.qubits) owner[q] = -1;
        if (b.gates.size() == 1) {   // keeps the cheaper single-gate encodings (controls, X)
            emit_single(gates[b.gates[0]]);
            return;
        }
        std::vector<uint32_t> lt;
        for (uint32_t q : b.qubits) lt.push_back(static_cast<uint32_t>(lm.local(q)));
        FusedBlock fb;
        fb.qubits = b.qubits;
        bool variant = false;
        for (uint32_t gi : b.gates) variant |= gates[gi].slot;
        if (b.sel.empty()) {
            std::vector<GateDesc> res;
            for (uint32_t gi : b.gates) {
                fb.gates.push_back(static_cast<uint32_t>(res.size()));
                res.push_back(resolved(gates[gi]));
            }
            out.push_back(matrix_op(block_matrix(fb, res), lt, 0, 0, variant));
            return;
        }
        // one matrix per value s of the out-of-tile controls (bit i of s = qubit sel[i]): a
        // gate acts, without those controls, where all of its own are 1 and is the identity
        // elsewhere
        const uint32_t c = static_cast<uint32_t>(b.sel.size());
        const uint64_t dim = uint64_t{1} << lt.size();
        std::vector<std::vector<cd>> mats;
        bool diag = true;
        for (uint32_t sv = 0; sv < (1u << c); ++sv) {
            std::vector<GateDesc> red;
            for (uint32_t gi : b.gates) {
                const GateDesc g = resolved(gates[gi]);
                GateDesc r = g;
                r.qubits.clear();
                r.n_controls = 0;
                bool on = true;
                for (uint32_t k = 0; k < g.n_controls; ++k) {
                    const uint32_t q = g.controls()[k];
                    if (lm.local(q) >= 0) {
                        r.qubits.push_back(q);
                        ++r.n_controls;
                    } else {
                        const auto it = std::find(b.sel.begin(), b.sel.end(), q);
                        on &= ((sv >> (it - b.sel.begin())) & 1u) != 0;
                    }
                }
                for (uint32_t j = 0; j < g.base_qubits(); ++j) r.qubits.push_back(g.targets()[j]);
                if (on) red.push_back(std::move(r));
            }
            fb.gates.clear();
            for (uint32_t i = 0; i < red.size(); ++i) fb.gates.push_back(i);
            mats.push_back(block_matrix(fb, red));
            diag &= !variant && is_diagonal(mats.back(), dim);
        }
        LocalOp op;
        op.kind = diag ? kTileDiag : kTileDense;
        op.lt = lt;
        op.sel = b.sel;
        op.variant = variant;
        for (const std::vector<cd>& m : mats) {
            if (diag) {
                for (uint64_t i = 0; i < dim; ++i) op.m.push_back(m[i * dim + i]);
            } else {
                op.m.insert(op.m.end(), m.begin(), m.end());
            }
        }
        out.push_back(std::move(op));
    };

    for (uint32_t gi : item.gates) {
        const GateDesc& g = gates[gi];
        // a native Pauli rotation: closes the blocks on its tile qubits and runs on its own
        if (native_rotations && native_pauli(g, cfg)) {
            for (uint32_t q : g.qubits)
                if (lm.local(q) >= 0 && owner[q] >= 0) emit_block(open[owner[q]]);
            const PauliMasks pm = pauli_local_masks(g.pauli);
            LocalOp op;
            op.kind = kTilePauli;
            uint64_t xg = 0, zg = 0;
            for (uint32_t j = 0; j < g.base_qubits(); ++j) {
                const uint32_t q = g.targets()[j];
                const int l = lm.local(q);
                if ((pm.x >> j) & 1) {
                    if (l < 0) logic("tile lowering: a Pauli rotation flips a qubit outside the tile");
                    op.lt.push_back(static_cast<uint32_t>(l));
                    xg |= uint64_t{1} << q;
                }
                if ((pm.zy >> j) & 1) {
                    zg |= uint64_t{1} << q;
                    if (l >= 0) op.lmask |= 1u << l;
                    else op.pz_out |= uint64_t{1} << q;
                }
            }
            std::sort(op.lt.begin(), op.lt.end());
            // y = (-i sin) i^n_Y, as apply_pauli_rotation forms it, times (-1)^parity(x & zy)
            const double h = g.params.at(0) / 2;
            static const cd kIPow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
            cd y = cd{0.0, -std::sin(h)} * kIPow[pm.n_y % 4];
            if (__builtin_popcountll(xg & zg) & 1) y = -y;
            op.m = {cd{std::cos(h), 0.0}, y};
            out.push_back(std::move(op));
            continue;
        }
        // a SWAP of two tile qubits moves no data: the two tile bits trade qubits for the rest
        // of the pass, and the store writes each tile bit to its qubit's place
        if (store_qubits && g.type == LQCS_GATE_SWAP && g.n_controls == 0 && !g.slot &&
            g.qubits.size() == 2 && lm.local(g.qubits[0]) >= 0 && lm.local(g.qubits[1]) >= 0) {
            for (uint32_t q : g.qubits)
                if (owner[q] >= 0) emit_block(open[owner[q]]);
            lm.swap_bits(g.qubits[0], g.qubits[1]);
            continue;
        }
        std::vector<uint32_t> part, sel;   // local qubits; out-of-tile controls
        for (uint32_t q : g.qubits) (lm.local(q) >= 0 ? part : sel).push_back(q);
        std::sort(part.begin(), part.end());
        std::sort(sel.begin(), sel.end());
        if (cfg.inner < 2 || is_phase_gate(g) || part.size() > cfg.inner || sel.size() > max_select) {
            for (uint32_t q : part)
                if (owner[q] >= 0) emit_block(open[owner[q]]);
            emit_single(g);
            continue;
        }
        std::vector<int> touched;
        for (uint32_t q : part)
            if (owner[q] >= 0 && std::find(touched.begin(), touched.end(), owner[q]) == touched.end())
                touched.push_back(owner[q]);
        std::vector<uint32_t> uni = part, usel = sel;
        for (int b : touched) {
            uni.insert(uni.end(), open[b].qubits.begin(), open[b].qubits.end());
            usel.insert(usel.end(), open[b].sel.begin(), open[b].sel.end());
        }
        std::sort(uni.begin(), uni.end());
        uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
        std::sort(usel.begin(), usel.end());
        usel.erase(std::unique(usel.begin(), usel.end()), usel.end());
        Open nb;
        if (uni.size() > cfg.inner || usel.size() > max_select) {
            for (int b : touched) emit_block(open[b]);
            nb.qubits = part;
            nb.sel = sel;
            nb.gates = {gi};
        } else {
            nb.qubits = uni;
            nb.sel = usel;
            for (int b : touched) {
                nb.gates.insert(nb.gates.end(), open[b].gates.begin(), open[b].gates.end());
                open[b].alive = false;
            }
            std::sort(nb.gates.begin(), nb.gates.end());
            nb.gates.push_back(gi);
        }
        const int id = static_cast<int>(open.size());
        for (uint32_t q : nb.qubits) owner[q] = id;
        open.push_back(std::move(nb));
    }
    for (Open& b : open) emit_block(b);
    // one-qubit ops first go into the dense blocks on their qubits (free); the diagonal
    // work left over then merges into tables
    fold_single_qubit_ops(out, max_select);
    merge_diagonal_runs(out, max_diag, dyn_terms);
    if (store_qubits) {   // qubit each tile bit holds at the end of the pass
        const uint32_t m = cfg.L + static_cast<uint32_t>(item.hbits.size());
        store_qubits->assign(m, 0);
        for (uint32_t b = 0; b < m; ++b) {
            const uint32_t q = b < cfg.L ? b : item.hbits[b - cfg.L];
            (*store_qubits)[static_cast<uint32_t>(lm.local(q))] = q;
        }
    }
    return out;
}

void lower_pass(const PlanItem& item, const std::vector<GateDesc>& gates, const TileConfig& cfg,
                TilePass& pass, std::vector<TileOp>& ops_out, std::vector<cd>& arena,
                double* flops_per_amp) {
    pass = TilePass{};
    pass.L = cfg.L;
    pass.h = static_cast<uint32_t>(item.hbits.size());
    pass.m = cfg.L + pass.h;
    for (uint32_t i = 0; i < pass.h; ++i) pass.hbits[i] = item.hbits[i];
    const size_t first = ops_out.size();
    double flops = 0.0;
    for (const LocalOp& lo : pass_local_ops(item, gates, cfg, 0)) {
        flops += local_op_flops(lo, false);
        TileOp op{};
        op.kind = lo.kind;
        op.gcmask = lo.gcmask;
        op.mat_off = static_cast<uint32_t>(arena.size());
        arena.insert(arena.end(), lo.m.begin(), lo.m.end());
        if (lo.kind == kTilePhase) {
            std::vector<uint32_t> fixed;
            for (uint32_t b = 0; b < 32; ++b)
                if ((lo.lmask >> b) & 1) fixed.push_back(b);
            set_groups(op, fixed, lo.lmask, pass.m);
        } else {
            const uint32_t k = static_cast<uint32_t>(lo.lt.size());
            op.k = static_cast<uint8_t>(k);
            for (uint32_t l = 0; l < (1u << k); ++l) {
                uint32_t o = 0;
                for (uint32_t j = 0; j < k; ++j)
                    if ((l >> j) & 1) o |= 1u << lo.lt[j];
                op.soff[l] = static_cast<uint16_t>(tile_swizzle(o));
            }
            std::vector<uint32_t> fixed = lo.lt;
            for (uint32_t b = 0; b < 32; ++b)
                if ((lo.lmask >> b) & 1) fixed.push_back(b);
            set_groups(op, fixed, lo.lmask, pass.m);
        }
        ops_out.push_back(op);
    }
    pass.n_ops = static_cast<uint32_t>(ops_out.size() - first);
    if (flops_per_amp) *flops_per_amp = flops;
    pass.kmax = 1;
    for (size_t i = first; i < ops_out.size(); ++i)
        if (ops_out[i].kind != kTilePhase) pass.kmax = std::max<uint32_t>(pass.kmax, ops_out[i].k);
}

// ------------------------------------------------------------------ register passes

namespace {

constexpr uint32_t kLaneBits = 5;

uint32_t target_mask(const LocalOp& o) {
    uint32_t t = 0;
    for (uint32_t b : o.lt) t |= 1u << b;
    return t;
}

// Tile bits an op uses off the diagonal (dense targets) and on it (controls, phase bits,
// diagonal targets).  Two ops commute when every bit they share is diagonal in both.
struct Use {
    uint32_t nd = 0, dg = 0;
};
Use op_use(const LocalOp& o) {
    Use u;
    if (o.kind == kTileDense || o.kind == kTilePauli) u.nd = target_mask(o);
    else if (o.kind == kTileDiag) u.dg = target_mask(o);
    u.dg |= o.lmask;
    return u;
}

// A layout as the scheduler sees it: register set S, warp bits W and the pair P of tile
// bits on lanes 0 and 1 (0: none), where the two-qubit blocks of a tensor-core pass run.
struct Lay {
    uint32_t S = 0, W = 0, P = 0;
};

// Whether op o runs in layout ly: a dense op on the tensor path (mma) needs its targets
// (two, or one) on the lane pair and its tile controls on register or warp bits (every lane
// of a warp takes part in the instruction); any other dense op needs its targets on
// register bits.
bool fits(const LocalOp& o, bool mma, const Lay& ly) {
    if (o.kind == kTilePauli) return (target_mask(o) & ly.W) == 0;   // flips on registers, lanes
    if (o.kind != kTileDense) return true;
    if (mma) return ly.P != 0 && (target_mask(o) & ~ly.P) == 0 && (o.lmask & ~(ly.S | ly.W)) == 0;
    return (target_mask(o) & ~ly.S) == 0;
}

// Scan of the pending ops under layout ly: every op that commutes with all skipped ops
// before it and fits the layout is applied.  Returns the count; with `emitted` the applied
// ops move there (in order) and `pending` keeps the rest.  mma[i]: op i is a tensor-path op.
size_t scan(const std::vector<LocalOp>& ops, const std::vector<Use>& use,
            const std::vector<uint8_t>& mma, std::vector<uint32_t>& pending, const Lay& ly,
            std::vector<uint32_t>* emitted) {
    uint32_t busy_nd = 0, busy_dg = 0;
    size_t cnt = 0;
    std::vector<uint32_t> rest;
    for (uint32_t i : pending) {
        const Use& u = use[i];
        const bool blocked = (u.nd & (busy_nd | busy_dg)) != 0 || (u.dg & busy_nd) != 0;
        if (!blocked && fits(ops[i], mma[i] != 0, ly)) {
            ++cnt;
            if (emitted) emitted->push_back(i);
        } else {
            busy_nd |= u.nd;
            busy_dg |= u.dg;
            if (emitted) rest.push_back(i);
        }
    }
    if (emitted) pending = std::move(rest);
    return cnt;
}

// Register-path dense ops of `pending` whose targets all lie in S (a tie-break: later use
// of a layout).
size_t covered(const std::vector<LocalOp>& ops, const std::vector<uint8_t>& mma,
               const std::vector<uint32_t>& pending, uint32_t S) {
    size_t c = 0;
    for (uint32_t i : pending)
        if ((ops[i].kind == kTileDense || ops[i].kind == kTilePauli) && !mma[i] &&
            (target_mask(ops[i]) & ~S) == 0)
            ++c;
    return c;
}

// Layout of register set S, warp bits W and lane pair P on an m-bit tile.  Thread-index bits
// 0..4 (the lanes) take the tile bits outside S and W, bits 5.. (the warps) take W in
// ascending order.  With a pair, lanes 0 and 1 take its lower and higher bit and lane 2 a
// bit of the third residue mod 3 where one exists; otherwise lanes ascending, except that
// when they are not tile bits 0..4 the first three are picked with distinct residues mod 3:
// tile_swizzle sends 1 << b to slot bit (b mod 3), so then the 8 lanes of a quarter warp hit
// 8 different 16-byte bank groups in a remap.  A remap that keeps W keeps every warp on the
// same tile indices, hence on its own shared-memory slots: it needs only a warp-level
// barrier.
RegLayout make_layout(uint32_t S, uint32_t W, uint32_t m, uint32_t P = 0) {
    RegLayout ly{};
    std::vector<uint32_t> rb, lanes, warps;
    for (uint32_t b = 0; b < m; ++b) {
        if ((S >> b) & 1) rb.push_back(b);
        else if ((W >> b) & 1) warps.push_back(b);
        else if (!((P >> b) & 1)) lanes.push_back(b);
    }
    if (P != 0) {
        const uint32_t p0 = static_cast<uint32_t>(__builtin_ctz(P));
        const uint32_t p1 = 31u - static_cast<uint32_t>(__builtin_clz(P));
        const uint32_t seen = (1u << (p0 % 3)) | (1u << (p1 % 3));
        for (size_t i = 0; i < lanes.size(); ++i)
            if (!((seen >> (lanes[i] % 3)) & 1)) {
                std::rotate(lanes.begin(), lanes.begin() + static_cast<long>(i),
                            lanes.begin() + static_cast<long>(i) + 1);
                break;
            }
        lanes.insert(lanes.begin(), {p0, p1});
    } else if (lanes.size() >= 3 && lanes[0] + lanes.size() - 1 != lanes.back()) {
        std::vector<uint32_t> first, rest;
        uint32_t seen = 0;
        for (uint32_t b : lanes) {
            if (first.size() < 3 && !((seen >> (b % 3)) & 1)) {
                first.push_back(b);
                seen |= 1u << (b % 3);
            } else {
                rest.push_back(b);
            }
        }
        lanes = first;
        lanes.insert(lanes.end(), rest.begin(), rest.end());
    }
    std::vector<uint32_t> tb = lanes;
    tb.insert(tb.end(), warps.begin(), warps.end());
    for (uint32_t i = 0; i < kRegBits; ++i) {
        ly.rpos[i] = static_cast<uint8_t>(rb[i]);
        ly.rsw[i] = static_cast<uint16_t>(tile_swizzle(1u << rb[i]));
    }
    for (uint32_t i = 0; i < tb.size(); ++i) {
        ly.tpos[i] = static_cast<uint8_t>(tb[i]);
        ly.tsw[i] = static_cast<uint16_t>(tile_swizzle(1u << tb[i]));
    }
    return ly;
}

// Whether the tile bits in `lanes` cover all three residues mod 3 (see make_layout).
bool residues_spread(uint32_t lanes) {
    uint32_t seen = 0;
    for (uint32_t b = 0; b < 32; ++b)
        if ((lanes >> b) & 1) seen |= 1u << (b % 3);
    return seen == 7u;
}

// `count` warp bits out of `avail`: the tile bits the pending dense operations target least
// (ties: the higher bit), so that few later operations need a bit that is a warp bit.
uint32_t pick_warp_bits(const std::vector<LocalOp>& ops, const std::vector<uint32_t>& pending,
                        uint32_t avail, uint32_t count, uint32_t pair = 0) {
    uint32_t usage[32] = {};
    for (uint32_t i : pending)
        if (ops[i].kind == kTileDense || ops[i].kind == kTilePauli)
            for (uint32_t b : ops[i].lt) ++usage[b];
    uint32_t W = 0;
    for (uint32_t k = 0; k < count; ++k) {
        int best = -1;
        for (int b = 31; b >= 0; --b) {
            if (!((avail >> b) & 1) || ((W >> b) & 1)) continue;
            if (best < 0 || usage[b] < usage[best]) best = b;
        }
        if (best >= 0) W |= 1u << best;
    }
    // lanes (the rest of avail and the lane pair) without a residue mod 3: trade a warp bit
    // for a lane bit as little used
    if (!residues_spread((avail & ~W) | pair)) {
        for (uint32_t w = 0; w < 32; ++w) {
            if (!((W >> w) & 1)) continue;
            for (uint32_t l = 0; l < 32; ++l) {
                const uint32_t W2 = (W & ~(1u << w)) | (1u << l);
                if (((avail & ~W) >> l) & 1 && usage[l] <= usage[w] &&
                    residues_spread((avail & ~W2) | pair))
                    return W2;
            }
        }
    }
    return W;
}

// Register sets of size kRegBits inside `allowed` that contain `must`, best first by
// (ops applied now with warp bits W and lane pair P, register-path dense ops covered later,
// usable as the final layout, and — when the warp bits are known, `lane_pool` being the
// tile bits outside them — lanes that take all three residues mod 3, which keeps the remaps
// free of bank conflicts).
uint32_t choose_set(const std::vector<LocalOp>& ops, const std::vector<Use>& use,
                    const std::vector<uint8_t>& mma, std::vector<uint32_t>& pending,
                    uint32_t must, uint32_t allowed, uint32_t m, uint32_t lane_pool = 0,
                    uint32_t P = 0, uint32_t W = 0) {
    uint32_t best = 0;
    size_t best_now = 0, best_later = 0;
    bool best_final = false, best_spread = false, have = false;
    const uint32_t lanes = (1u << kLaneBits) - 1u;
    for (uint32_t S = 0; S < (1u << m); ++S) {
        if (__builtin_popcount(S) != static_cast<int>(kRegBits) || (S & must) != must ||
            (S & ~allowed) != 0)
            continue;
        const size_t now = scan(ops, use, mma, pending, Lay{S, W, P}, nullptr);
        const size_t later = covered(ops, mma, pending, S);
        const bool fin = (S & lanes) == 0;
        const bool spread = lane_pool != 0 && residues_spread(lane_pool & ~S);
        const auto key = std::make_tuple(now, later, fin, spread);
        if (!have || key > std::make_tuple(best_now, best_later, best_final, best_spread)) {
            have = true;
            best = S;
            best_now = now;
            best_later = later;
            best_final = fin;
            best_spread = spread;
        }
    }
    return best;
}

}  // namespace

namespace {

// Matrix data of op o in layout (ly, S): dense matrices re-indexed so that matrix bit q is
// the q-th lowest register target (one block per selector value), diagonals and phase
// factors as they are.  X operations (swaps) have none.
// A tensor-path op (mma) instead: matrix bit 0 is the tile bit on lane 0, bit 1 the one on
// lane 1.
void append_matrices(const LocalOp& o, const RegLayout& ly, uint32_t S, std::vector<cd>& mats,
                     bool mma = false) {
    if (mma) {
        std::vector<cd> pm(16);
        if (o.lt.size() == 1) {   // one target: the 2 x 2 matrix on its lane, identity on the other
            const uint32_t j = o.lt[0] == ly.tpos[0] ? 0u : 1u;
            for (size_t blk = 0; blk < o.m.size(); blk += 4) {
                for (uint32_t rr = 0; rr < 4; ++rr)
                    for (uint32_t cc = 0; cc < 4; ++cc)
                        pm[rr * 4 + cc] = ((rr ^ cc) >> (1u - j)) & 1u
                                              ? cd{0, 0}
                                              : o.m[blk + ((rr >> j) & 1u) * 2 + ((cc >> j) & 1u)];
                mats.insert(mats.end(), pm.begin(), pm.end());
            }
            return;
        }
        const bool swap = o.lt[0] != ly.tpos[0];   // matrix bit 0 is on lane 1
        auto sw = [&](uint32_t l) { return swap ? ((l & 1u) << 1) | (l >> 1) : l; };
        for (size_t blk = 0; blk < o.m.size(); blk += 16) {
            for (uint32_t rr = 0; rr < 4; ++rr)
                for (uint32_t cc = 0; cc < 4; ++cc) pm[sw(rr) * 4 + sw(cc)] = o.m[blk + rr * 4 + cc];
            mats.insert(mats.end(), pm.begin(), pm.end());
        }
        return;
    }
    if (o.kind == kTilePauli) {   // (cos, 0), y, the out-of-tile Z-type qubits as two halves
        mats.insert(mats.end(), o.m.begin(), o.m.end());
        mats.emplace_back(static_cast<double>(o.pz_out & 0xffffffffu),
                          static_cast<double>(o.pz_out >> 32));
        return;
    }
    if (o.kind == kTilePhase || o.kind == kTileDiag) {
        mats.insert(mats.end(), o.m.begin(), o.m.end());
        // per-tile terms: the factor, then {gcmask low 32 bits, gcmask high 32 bits * 64 +
        // entry mask} as exact integers
        for (const DynTerm& t : o.dyn) {
            uint64_t em = 0;
            for (size_t j = 0; j < o.lt.size(); ++j)
                if ((t.lbits >> o.lt[j]) & 1) em |= uint64_t{1} << j;
            mats.push_back(t.f);
            mats.emplace_back(static_cast<double>(t.gcmask & 0xffffffffu),
                              static_cast<double>((t.gcmask >> 32) * 64u + em));
        }
        return;
    }
    const uint32_t k = static_cast<uint32_t>(o.lt.size());
    if (k == 1 && !o.variant && o.sel.empty() && is_x(o.m)) return;
    int ridx[32];
    for (uint32_t i = 0; i < kRegBits; ++i) ridx[ly.rpos[i]] = static_cast<int>(i);
    uint32_t tm = 0;
    for (uint32_t b : o.lt) tm |= 1u << ridx[b];
    (void)S;
    std::vector<uint32_t> pos(k);
    for (uint32_t j = 0; j < k; ++j) {
        const uint32_t rb = static_cast<uint32_t>(ridx[o.lt[j]]);
        pos[j] = static_cast<uint32_t>(__builtin_popcount(tm & ((1u << rb) - 1u)));
    }
    const uint32_t D = 1u << k;
    std::vector<uint32_t> perm(D);
    for (uint32_t l = 0; l < D; ++l) {
        uint32_t p = 0;
        for (uint32_t j = 0; j < k; ++j)
            if ((l >> j) & 1) p |= 1u << pos[j];
        perm[l] = p;
    }
    std::vector<cd> pm(D * D);
    for (size_t blk = 0; blk < o.m.size(); blk += D * D) {   // per selector value
        for (uint32_t rr = 0; rr < D; ++rr)
            for (uint32_t cc = 0; cc < D; ++cc) pm[perm[rr] * D + perm[cc]] = o.m[blk + rr * D + cc];
        mats.insert(mats.end(), pm.begin(), pm.end());
    }
}

// The record of op o in layout (ly, S); its matrices start at mat_off.  mma: a two-qubit
// block on the lane pair (tensor path), its controls on register or warp bits.
RegOp make_record(const LocalOp& o, const RegLayout& ly, uint32_t S, uint32_t m, uint32_t mat_off,
                  bool mma = false) {
    int ridx[32], tidx[32];
    for (uint32_t i = 0; i < kRegBits; ++i) ridx[ly.rpos[i]] = static_cast<int>(i);
    for (uint32_t i = 0; i < m - kRegBits; ++i) tidx[ly.tpos[i]] = static_cast<int>(i);
    RegOp r{};
    r.gcmask = o.gcmask;
    r.mat_off = mat_off;
    r.nsel = static_cast<uint8_t>(o.sel.size());
    for (size_t i = 0; i < o.sel.size(); ++i) r.selq[i] = static_cast<uint8_t>(o.sel[i]);
    for (uint32_t b = 0; b < m; ++b) {
        if (!((o.lmask >> b) & 1)) continue;
        if ((S >> b) & 1) r.rcmask = static_cast<uint8_t>(r.rcmask | (1u << ridx[b]));
        else r.tcmask = static_cast<uint16_t>(r.tcmask | (1u << tidx[b]));
    }
    const uint32_t k = static_cast<uint32_t>(o.lt.size());
    r.k = static_cast<uint8_t>(k);
    if (mma) {
        if (r.tcmask & ((1u << kLaneBits) - 1u))
            logic("register tile lowering: a tensor-path block is controlled by a lane bit");
        r.kind = kRegMma;
        r.k = 2;   // always a 4 x 4 block (a one-target op with the identity on the other lane)
    } else if (o.kind == kTilePauli) {   // Z-type tile bits went to rcmask / tcmask above
        r.kind = kRegPauli;
        r.k = 0;
        for (uint32_t b : o.lt) {
            if ((S >> b) & 1) {
                r.code = static_cast<uint8_t>(r.code | (1u << ridx[b]));
            } else {
                if (tidx[b] >= static_cast<int>(kLaneBits))
                    logic("register tile lowering: a Pauli rotation flips a warp bit");
                r.loc[0] = static_cast<uint8_t>(r.loc[0] | (1u << tidx[b]));
            }
        }
    } else if (o.kind == kTilePhase) {
        r.kind = kRegPhase;
    } else if (o.kind == kTileDiag) {
        r.kind = o.dyn.empty() ? kRegDiag : kRegDiagDyn;
        r.nterm = static_cast<uint8_t>(o.dyn.size());
        for (uint32_t j = 0; j < k; ++j) {
            const uint32_t b = o.lt[j];
            r.loc[j] = static_cast<uint8_t>((S >> b) & 1 ? ridx[b] : (0x80 | tidx[b]));
        }
    } else {
        uint32_t tm = 0;
        for (uint32_t b : o.lt) tm |= 1u << ridx[b];
        r.code = static_cast<uint8_t>(tm);
        r.kind = (k == 1 && !o.variant && o.sel.empty() && is_x(o.m)) ? kRegSwapX : kRegDense;
    }
    return r;
}

bool same_shape(const LocalOp& a, const LocalOp& b) {
    return a.kind == b.kind && a.lt == b.lt && a.lmask == b.lmask && a.gcmask == b.gcmask &&
           a.sel == b.sel && a.m.size() == b.m.size() && a.variant == b.variant &&
           a.dyn.size() == b.dyn.size();
}

bool lower_pass_reg_sel(const PlanItem& item, const std::vector<GateDesc>& gates,
                        const TileConfig& cfg, uint32_t max_select, RegPass& pass,
                        std::vector<RegOp>& ops_out, std::vector<RegLayout>& layouts_out,
                        std::vector<cd>& mats_out, double* flops_per_amp,
                        const std::vector<std::vector<std::array<cd, 4>>>* state_slots) {
    const uint32_t m = cfg.L + static_cast<uint32_t>(item.hbits.size());
    const std::vector<std::array<cd, 4>>* slots0 =
        state_slots && !state_slots->empty() ? &(*state_slots)[0] : nullptr;
    std::vector<uint32_t> store_q;
    const std::vector<LocalOp> ops =
        pass_local_ops(item, gates, cfg, max_select, slots0, kRegMaxDiag, true, &store_q, true);
    for (const LocalOp& o : ops)
        if (o.kind != kTilePhase && o.kind != kTilePauli &&
            o.lt.size() > (o.kind == kTileDense ? kRegMaxK : kRegMaxDiag))
            return false;
    std::vector<Use> use;
    for (const LocalOp& o : ops) use.push_back(op_use(o));
    // One- and two-target dense blocks run on the FP64 tensor path (lane pair) when cfg.mma
    // is set — all but X operations, which stay register swaps; their tile controls must fit
    // on the register bits, which at most kRegBits can.
    std::vector<uint8_t> mma(ops.size(), 0);
    for (size_t i = 0; i < ops.size(); ++i) {
        const LocalOp& o = ops[i];
        const size_t k = o.lt.size();
        const bool swapx = k == 1 && !o.variant && o.sel.empty() && is_x(o.m);
        mma[i] = cfg.mma && o.kind == kTileDense && (k == 2 || (k == 1 && !swapx)) &&
                 __builtin_popcount(o.lmask) <= static_cast<int>(kRegBits);
    }

    std::vector<RegLayout> lays;
    std::vector<Lay> lay_keys;
    auto layout_index = [&](uint32_t S, uint32_t W, uint32_t P) {
        if ((P != 0 && __builtin_popcount(P) != 2) || (P & (S | W)) != 0 || (S & W) != 0)
            logic("register tile lowering: inconsistent layout");
        for (size_t i = 0; i < lay_keys.size(); ++i)
            if (lay_keys[i].S == S && lay_keys[i].W == W && lay_keys[i].P == P)
                return static_cast<uint32_t>(i);
        lay_keys.push_back(Lay{S, W, P});
        lays.push_back(make_layout(S, W, m, P));
        return static_cast<uint32_t>(lay_keys.size() - 1);
    };
    // schedule: (op, layout) in application order, remaps as (-1 warp-local / -2 CTA-wide,
    // new layout)
    std::vector<std::pair<int, uint32_t>> seq;
    const uint32_t all = (1u << m) - 1u;
    const uint32_t lanes = (1u << kLaneBits) - 1u;
    const uint32_t high = all & ~lanes;
    const uint32_t nwarp = m - kRegBits - kLaneBits;
    std::vector<uint32_t> pending(ops.size());
    for (uint32_t i = 0; i < ops.size(); ++i) pending[i] = i;
    // Lane pair for tensor-path op i out of the tile bits `pool` (0: none there): its two
    // targets; for one target, the targets of a pending two-target block that contains it,
    // else the target and the lowest free bit of pool (one of `prefer` if there is one).
    auto pair_for = [&](uint32_t i, uint32_t pool, uint32_t prefer) -> uint32_t {
        const uint32_t t = target_mask(ops[i]);
        if ((t & ~pool) != 0) return 0u;
        if (ops[i].lt.size() == 2) return t;
        for (uint32_t j : pending) {
            const uint32_t tj = target_mask(ops[j]);
            if (mma[j] && ops[j].lt.size() == 2 && (tj & t) && !(tj & ~pool) && !(tj & ops[i].lmask))
                return tj;
        }
        const uint32_t free = pool & ~t & ~ops[i].lmask;
        if (free == 0) return 0u;
        const uint32_t pick = (free & prefer) ? (free & prefer) : free;
        return t | (1u << __builtin_ctz(pick));
    };
    // lane pair for a layout whose lanes are `pool`: that of the first pending tensor-path
    // block that has one there
    auto next_pair = [&](uint32_t pool) -> uint32_t {
        for (uint32_t i : pending)
            if (mma[i])
                if (const uint32_t pr = pair_for(i, pool, pool)) return pr;
        return 0u;
    };
    // the first layout loads the tile: lanes on tile bits 0..4 keep the loads coalesced
    uint32_t P = next_pair(lanes);
    uint32_t S = choose_set(ops, use, mma, pending, 0, high, m, 0, P, 0);
    uint32_t W = pick_warp_bits(ops, pending, high & ~S, nwarp, P);
    uint32_t cur = layout_index(S, W, P);
    bool sync_tiles = false;
    while (true) {
        std::vector<uint32_t> applied;
        scan(ops, use, mma, pending, Lay{S, W, P}, &applied);
        for (uint32_t i : applied) seq.emplace_back(static_cast<int>(i), cur);
        if (pending.empty()) break;
        const LocalOp& f = ops[pending.front()];
        if (mma[pending.front()]) {   // a tensor-path block: its targets become the lane pair
            P = pair_for(pending.front(), all, all & ~W);
            if ((P & W) == 0) {       // warp-local: the warp bits stay
                S = choose_set(ops, use, mma, pending, f.lmask & ~W, all & ~W & ~P, m, all & ~W,
                               P, W);
                cur = layout_index(S, W, P);
                seq.emplace_back(-1, cur);
            } else {                  // a target is a warp bit: new warp bits, CTA-wide remap
                S = choose_set(ops, use, mma, pending, f.lmask, all & ~P, m, 0, P, 0);
                W = pick_warp_bits(ops, pending, all & ~S & ~P, nwarp, P);
                cur = layout_index(S, W, P);
                seq.emplace_back(-2, cur);
                sync_tiles = true;
            }
            continue;
        }
        if (f.kind == kTilePauli) {   // its flips on warp bits: new warp bits outside them
            W = pick_warp_bits(ops, pending, all & ~target_mask(f), nwarp);
            S = choose_set(ops, use, mma, pending, 0, all & ~W, m, all & ~W, 0, W);
            P = next_pair(all & ~W & ~S);
            cur = layout_index(S, W, P);
            seq.emplace_back(-2, cur);
            sync_tiles = true;
            continue;
        }
        const uint32_t must = target_mask(f);
        if ((must & W) == 0) {   // warp-local: the warp bits stay
            S = choose_set(ops, use, mma, pending, must, all & ~W, m, all & ~W, 0, W);
            P = next_pair(all & ~W & ~S);
            cur = layout_index(S, W, P);
            seq.emplace_back(-1, cur);
        } else {                 // a target is a warp bit: new warp bits, CTA-wide remap
            S = choose_set(ops, use, mma, pending, must, all, m);
            P = next_pair(all & ~S);
            W = pick_warp_bits(ops, pending, all & ~S & ~P, nwarp, P);
            cur = layout_index(S, W, P);
            seq.emplace_back(-2, cur);
            sync_tiles = true;
        }
    }
    // The store wants the lanes on the tile bits that hold qubits of tile bits 0..4 at the
    // load (the same bits unless a relabelling moved those qubits).
    uint32_t slanes = 0;
    for (uint32_t l = 0; l < kLaneBits; ++l) {
        const uint32_t q = l < cfg.L ? l : item.hbits[l - cfg.L];
        for (uint32_t b = 0; b < m; ++b)
            if (store_q[b] == q) slanes |= 1u << b;
    }
    const uint32_t shigh = all & ~slanes;
    if (((S | W) & slanes) != 0) {
        if ((W & slanes) == 0) {
            seq.emplace_back(-1, layout_index(shigh & ~W, W, 0));
        } else {
            uint32_t Sf = 0;   // the four highest tile bits outside the store lanes
            for (int b = static_cast<int>(m) - 1; b >= 0 && __builtin_popcount(Sf) < static_cast<int>(kRegBits); --b)
                if ((shigh >> b) & 1) Sf |= 1u << b;
            W = pick_warp_bits(ops, pending, shigh & ~Sf, nwarp);
            seq.emplace_back(-2, layout_index(Sf, W, 0));
            sync_tiles = true;
        }
    }

    // records and the first state's matrices
    std::vector<RegOp> rec;
    std::vector<cd> mats;
    std::vector<uint32_t> dyn_rec;
    uint32_t dyn_entries = 0;
    for (const auto& [i, l] : seq) {
        if (i < 0) {
            RegOp r{};
            r.kind = kRegRemap;
            r.code = static_cast<uint8_t>(l);
            r.k = i == -1 ? 1 : 0;   // 1: warp-local
            rec.push_back(r);
            continue;
        }
        RegOp r = make_record(ops[i], lays[l], lay_keys[l].S, m, static_cast<uint32_t>(mats.size()),
                              mma[i] != 0);
        if (r.kind == kRegDiagDyn) {
            r.dyn_off = static_cast<uint16_t>(dyn_entries);
            dyn_entries += 1u << r.k;
            dyn_rec.push_back(static_cast<uint32_t>(rec.size()));
        }
        rec.push_back(r);
        append_matrices(ops[i], lays[l], lay_keys[l].S, mats, mma[i] != 0);
    }
    if (rec.size() > kRegMaxRecords || lays.size() > kRegMaxLayouts || mats.size() > kRegMaxMatrix ||
        dyn_rec.size() > kRegMaxDyn || dyn_entries > kRegMaxDynEntries)
        return false;
    const size_t n_mat = mats.size();
    // every further state: same records, its own slot matrices
    if (state_slots) {
        for (size_t b = 1; b < state_slots->size(); ++b) {
            std::vector<uint32_t> store_b;
            const std::vector<LocalOp> ob = pass_local_ops(item, gates, cfg, max_select,
                                                           &(*state_slots)[b], kRegMaxDiag, true,
                                                           &store_b, true);
            if (ob.size() != ops.size() || store_b != store_q) return false;
            for (size_t i = 0; i < ops.size(); ++i)
                if (!same_shape(ops[i], ob[i])) return false;
            const size_t before = mats.size();
            for (const auto& [i, l] : seq)
                if (i >= 0) append_matrices(ob[i], lays[l], lay_keys[l].S, mats, mma[i] != 0);
            if (mats.size() - before != n_mat) return false;
        }
    }
    pass = RegPass{};
    pass.L = cfg.L;
    pass.h = static_cast<uint32_t>(item.hbits.size());
    pass.m = m;
    for (uint32_t i = 0; i < pass.h; ++i) pass.hbits[i] = item.hbits[i];
    pass.n_ops = static_cast<uint32_t>(rec.size());
    pass.n_layouts = static_cast<uint32_t>(lays.size());
    pass.n_mat = static_cast<uint32_t>(n_mat);
    pass.mat_stride = state_slots ? static_cast<uint32_t>(n_mat) : 0u;
    // A barrier between a CTA's tiles only where the last layout's warp bits differ from the
    // first's: then a warp's shared-memory slots at the end of one tile are not its slots at
    // the start of the next.  The slots a warp touches in a layout depend only on the warp
    // bits and the warp's index (tile_swizzle is a linear bijection, and a layout only permutes
    // the other bits among lanes and registers), so where they agree each warp meets only its
    // own slots across the tile boundary — up to the next tile's first CTA-wide remap, whose
    // barrier every warp reaches only after finishing this tile.  The host emulation
    // (reg_emulate.cpp) checks this against the barrier model.
    uint32_t last_layout = 0;
    for (const auto& [i, l] : seq)
        if (i < 0) last_layout = l;
    pass.cta_remaps = sync_tiles ? 1u : 0u;
    pass.sync_tiles = sync_tiles && lay_keys[last_layout].W != lay_keys[0].W ? 1u : 0u;
    for (uint32_t b = 0; b < m; ++b) {
        pass.store_qubit[b] = static_cast<uint8_t>(store_q[b]);
        const uint32_t home = b < cfg.L ? b : item.hbits[b - cfg.L];
        if (store_q[b] != home) pass.relabel = 1;
    }
    pass.n_dyn = static_cast<uint32_t>(dyn_rec.size());
    pass.dyn_entries = dyn_entries;
    // A relabelling pass stores amplitudes, in place, to places that other threads (of other
    // warps) load: every load of the tile must come before any store.  A CTA-wide remap or
    // the per-tile table barrier, both after the loads, order them; otherwise the kernel
    // adds a barrier after the loads.
    pass.load_barrier = pass.relabel && !sync_tiles && dyn_rec.empty() ? 1u : 0u;
    pass.fma_dense = pass.mma_ops = pass.pauli_ops = 0;
    for (const RegOp& r : rec) {
        if (r.kind == kRegDense) pass.fma_dense = 1;
        if (r.kind == kRegMma) pass.mma_ops = 1;
        if (r.kind == kRegPauli) pass.pauli_ops = 1;
    }
    for (size_t d = 0; d < dyn_rec.size(); ++d) pass.dyn_rec[d] = static_cast<uint8_t>(dyn_rec[d]);
    ops_out.insert(ops_out.end(), rec.begin(), rec.end());
    layouts_out.insert(layouts_out.end(), lays.begin(), lays.end());
    mats_out.insert(mats_out.end(), mats.begin(), mats.end());
    if (flops_per_amp) {
        *flops_per_amp = 0.0;
        for (const LocalOp& o : ops) *flops_per_amp += local_op_flops(o, true);
    }
    return true;
}

}  // namespace

bool lower_pass_reg(const PlanItem& item, const std::vector<GateDesc>& gates,
                    const TileConfig& cfg, RegPass& pass, std::vector<RegOp>& ops_out,
                    std::vector<RegLayout>& layouts_out, std::vector<cd>& mats_out,
                    double* flops_per_amp,
                    const std::vector<std::vector<std::array<cd, 4>>>* state_slots) {
    const uint32_t m = cfg.L + static_cast<uint32_t>(item.hbits.size());
    if (m < kRegMinBits || m > kRegMaxBits || item.hbits.size() > kTileMaxHigh) return false;
    // fewer selector qubits when the matrices of a pass outgrow their shared-memory stage
    for (int sel = static_cast<int>(kRegMaxSelect); sel >= 0; --sel)
        if (lower_pass_reg_sel(item, gates, cfg, static_cast<uint32_t>(sel), pass, ops_out,
                               layouts_out, mats_out, flops_per_amp, state_slots))
            return true;
    return false;
}

}  // namespace lqcs_b200
