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

#include "tile_plan.hpp"

namespace lqcs_b200 {

namespace {

bool is_phase_gate(const GateDesc& g) {
    if (!g.is_unitary() || g.base_qubits() != 1) return false;
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
    c.m = std::max<uint32_t>(kTileMinBits, std::min<uint32_t>(std::min<uint32_t>(c.m, kTileMaxBits), n));
    c.L = std::min<uint32_t>(std::min(c.L, c.m), kTileMinBits);   // column bits come from the thread index
    if (c.m - c.L > kTileMaxHigh) c.L = c.m - kTileMaxHigh;
    c.inner = std::max<uint32_t>(1, std::min<uint32_t>(c.inner, kTileMaxK));
    return c;
}

// Qubits a gate needs inside the tile, or false if it cannot run in a tile at all.
static bool tile_requirements(const GateDesc& g, const TileConfig& c, std::vector<uint32_t>& need) {
    need.clear();
    if (is_phase_gate(g)) return g.qubits.size() <= 8;   // at most 8 local phase bits
    const uint32_t k = g.base_qubits();
    if (k == 0 || k > kTileMaxK) return false;
    if (g.type == LQCS_GATE_PERMUTATION && k > kTileMaxK) return false;
    if (k + g.n_controls > 8) return false;
    for (uint32_t j = 0; j < k; ++j) need.push_back(g.targets()[j]);
    (void)c;
    return true;
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
    int local(uint32_t q) const {   // -1 if outside the tile
        if (q < L) return static_cast<int>(q);
        const auto it = std::find(hbits.begin(), hbits.end(), q);
        return it == hbits.end() ? -1 : static_cast<int>(L + (it - hbits.begin()));
    }
};

uint32_t deposit(uint32_t v, const std::vector<uint32_t>& sorted_pos) {
    for (uint32_t p : sorted_pos) {
        const uint32_t low = (1u << p) - 1u;
        v = ((v & ~low) << 1) | (v & low);
    }
    return v;
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

// Dense or diagonal op of matrix m on local target positions lt (matrix local order).
TileOp make_matrix_op(const std::vector<cd>& m, const std::vector<uint32_t>& lt, uint32_t lcmask,
                      uint64_t gcmask, std::vector<cd>& arena, uint32_t tile_bits) {
    TileOp op{};
    const uint32_t k = static_cast<uint32_t>(lt.size());
    const uint64_t dim = uint64_t{1} << k;
    bool diag = true;
    for (uint64_t r = 0; r < dim && diag; ++r)
        for (uint64_t c = 0; c < dim; ++c)
            if (r != c && m[r * dim + c] != cd{0, 0}) { diag = false; break; }
    op.kind = diag ? kTileDiag : kTileDense;
    op.k = static_cast<uint8_t>(k);
    op.gcmask = gcmask;
    for (uint64_t l = 0; l < dim; ++l) {
        uint32_t o = 0;
        for (uint32_t j = 0; j < k; ++j)
            if ((l >> j) & 1) o |= 1u << lt[j];
        op.soff[l] = static_cast<uint16_t>(tile_swizzle(o));
    }
    std::vector<uint32_t> fixed = lt;
    for (uint32_t b = 0; b < 32; ++b)
        if ((lcmask >> b) & 1) fixed.push_back(b);
    set_groups(op, fixed, lcmask, tile_bits);
    op.mat_off = static_cast<uint32_t>(arena.size());
    if (diag) {
        for (uint64_t i = 0; i < dim; ++i) arena.push_back(m[i * dim + i]);
    } else {
        arena.insert(arena.end(), m.begin(), m.end());
    }
    return op;
}

}  // namespace

void lower_pass(const PlanItem& item, const std::vector<GateDesc>& gates, const TileConfig& cfg,
                TilePass& pass, std::vector<TileOp>& ops_out, std::vector<cd>& arena) {
    LocalMap lm{cfg.L, item.hbits};
    pass = TilePass{};
    pass.L = cfg.L;
    pass.h = static_cast<uint32_t>(item.hbits.size());
    pass.m = cfg.L + pass.h;
    for (uint32_t i = 0; i < pass.h; ++i) pass.hbits[i] = item.hbits[i];
    const size_t first = ops_out.size();

    // inner fusion: greedy blocks over gates whose qubits are all local; any other gate
    // closes the blocks it touches and is emitted on its own
    struct Open {
        std::vector<uint32_t> qubits;   // global, sorted
        std::vector<uint32_t> gates;
        bool alive = true;
    };
    std::vector<Open> open;
    std::vector<int> owner(64, -1);
    auto emit_block = [&](Open& b) {
        if (!b.alive) return;
        b.alive = false;
        for (uint32_t q : b.qubits) owner[q] = -1;
        std::vector<uint32_t> lt;
        for (uint32_t q : b.qubits) lt.push_back(static_cast<uint32_t>(lm.local(q)));
        FusedBlock fb;
        fb.qubits = b.qubits;
        fb.gates = b.gates;
        const std::vector<cd> m = block_matrix(fb, gates);
        ops_out.push_back(make_matrix_op(m, lt, 0, 0, arena, pass.m));
    };
    auto emit_single = [&](const GateDesc& g) {
        if (is_phase_gate(g)) {
            TileOp op{};
            op.kind = kTilePhase;
            std::vector<uint32_t> fixed;
            uint32_t lmask = 0;
            for (uint32_t q : g.qubits) {
                const int l = lm.local(q);
                if (l >= 0) {
                    lmask |= 1u << l;
                    fixed.push_back(static_cast<uint32_t>(l));
                } else {
                    op.gcmask |= uint64_t{1} << q;
                }
            }
            set_groups(op, fixed, lmask, pass.m);
            op.mat_off = static_cast<uint32_t>(arena.size());
            arena.push_back(g.base_matrix()[3]);
            ops_out.push_back(op);
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
        ops_out.push_back(make_matrix_op(g.base_matrix(), lt, lc, gc, arena, pass.m));
    };

    for (uint32_t gi : item.gates) {
        const GateDesc& g = gates[gi];
        bool all_local = !is_phase_gate(g);
        for (uint32_t q : g.qubits) all_local &= lm.local(q) >= 0;
        if (cfg.inner < 2 || !all_local || g.qubits.size() > cfg.inner) {
            for (uint32_t q : g.qubits)
                if (owner[q] >= 0) emit_block(open[owner[q]]);
            emit_single(g);
            continue;
        }
        std::vector<int> touched;
        for (uint32_t q : g.qubits)
            if (owner[q] >= 0 && std::find(touched.begin(), touched.end(), owner[q]) == touched.end())
                touched.push_back(owner[q]);
        std::vector<uint32_t> uni(g.qubits.begin(), g.qubits.end());
        for (int b : touched) uni.insert(uni.end(), open[b].qubits.begin(), open[b].qubits.end());
        std::sort(uni.begin(), uni.end());
        uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
        Open nb;
        if (uni.size() > cfg.inner) {
            for (int b : touched) emit_block(open[b]);
            nb.qubits.assign(g.qubits.begin(), g.qubits.end());
            std::sort(nb.qubits.begin(), nb.qubits.end());
            nb.gates = {gi};
        } else {
            nb.qubits = uni;
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
    pass.n_ops = static_cast<uint32_t>(ops_out.size() - first);
    pass.kmax = 1;
    for (size_t i = first; i < ops_out.size(); ++i)
        if (ops_out[i].kind != kTilePhase) pass.kmax = std::max<uint32_t>(pass.kmax, ops_out[i].k);
}

}  // namespace lqcs_b200
