// gates.cpp — host-side gate model: decoding, matrices, lowering and fusion planning.
#include "gates.hpp"

#include <algorithm>
#include <cmath>
#include <numbers>
#include <numeric>
#include <unordered_set>

namespace lqcs_b200 {

namespace {

constexpr cd kI{0.0, 1.0};

cd unit(double theta) { return {std::cos(theta), std::sin(theta)}; }

const char* base_name(int type) {
    switch (type) {
        case LQCS_GATE_I: return "id";
        case LQCS_GATE_X: return "x";
        case LQCS_GATE_Y: return "y";
        case LQCS_GATE_Z: return "z";
        case LQCS_GATE_H: return "h";
        case LQCS_GATE_S: return "s";
        case LQCS_GATE_SDG: return "sdg";
        case LQCS_GATE_T: return "t";
        case LQCS_GATE_TDG: return "tdg";
        case LQCS_GATE_SX: return "sx";
        case LQCS_GATE_RX: return "rx";
        case LQCS_GATE_RY: return "ry";
        case LQCS_GATE_RZ: return "rz";
        case LQCS_GATE_P: return "p";
        case LQCS_GATE_U: return "u";
        case LQCS_GATE_SWAP: return "swap";
        case LQCS_GATE_ISWAP: return "iswap";
        case LQCS_GATE_RXX: return "rxx";
        case LQCS_GATE_RYY: return "ryy";
        case LQCS_GATE_RZZ: return "rzz";
        case LQCS_GATE_PAULI_ROTATION: return "rp";
        case LQCS_GATE_UNITARY: return "unitary";
        case LQCS_GATE_PERMUTATION: return "perm";
        case LQCS_GATE_MEASURE: return "measure";
        case LQCS_GATE_RESET: return "reset";
        case LQCS_GATE_BARRIER: return "barrier";
        case LQCS_GATE_KRAUS: return "kraus";
        default: return "?";
    }
}

double param(const GateDesc& g, size_t i) {
    if (i >= g.params.size()) invalid(g.name() + ": missing parameter");
    return g.params[i];
}

// Apply a dense gate (matrix f on local positions pos[0..m-1] of a k-bit space) to a
// small host vector v of 2^k entries.
void apply_small(std::vector<cd>& v, uint32_t k, const std::vector<uint32_t>& pos,
                 const std::vector<cd>& f) {
    const uint32_t m = static_cast<uint32_t>(pos.size());
    const uint64_t dim = uint64_t{1} << m;
    std::vector<uint32_t> sorted = pos;
    std::sort(sorted.begin(), sorted.end());
    std::vector<uint64_t> off(dim, 0);
    for (uint64_t l = 0; l < dim; ++l)
        for (uint32_t j = 0; j < m; ++j)
            if ((l >> j) & 1) off[l] |= uint64_t{1} << pos[j];
    const uint64_t groups = (uint64_t{1} << k) >> m;
    std::vector<cd> a(dim);
    for (uint64_t g = 0; g < groups; ++g) {
        uint64_t base = g;
        for (uint32_t p : sorted) {
            const uint64_t low = (uint64_t{1} << p) - 1;
            base = ((base & ~low) << 1) | (base & low);
        }
        for (uint64_t l = 0; l < dim; ++l) a[l] = v[base | off[l]];
        for (uint64_t r = 0; r < dim; ++r) {
            cd s{0.0, 0.0};
            for (uint64_t c = 0; c < dim; ++c) s += f[r * dim + c] * a[c];
            v[base | off[r]] = s;
        }
    }
}

bool is_diag_matrix(const std::vector<cd>& m, uint64_t dim) {
    for (uint64_t r = 0; r < dim; ++r)
        for (uint64_t c = 0; c < dim; ++c)
            if (r != c && m[r * dim + c] != cd{0.0, 0.0}) return false;
    return true;
}

void perm_cycles(const std::vector<uint64_t>& perm, std::vector<uint32_t>& cycles,
                 std::vector<uint32_t>& lens) {
    std::vector<bool> seen(perm.size(), false);
    for (uint64_t s = 0; s < perm.size(); ++s) {
        if (seen[s] || perm[s] == s) { seen[s] = true; continue; }
        uint32_t len = 0;
        uint64_t c = s;
        while (!seen[c]) {
            seen[c] = true;
            cycles.push_back(static_cast<uint32_t>(c));
            ++len;
            c = perm[c];
        }
        lens.push_back(len);
    }
}

}  // namespace

uint32_t GateDesc::base_qubits() const {
    switch (type) {
        case LQCS_GATE_SWAP:
        case LQCS_GATE_ISWAP:
        case LQCS_GATE_RXX:
        case LQCS_GATE_RYY:
        case LQCS_GATE_RZZ:
            return 2;
        case LQCS_GATE_UNITARY: {
            uint64_t dim = 1;
            uint32_t k = 0;
            while (dim * dim < mat.size()) { dim <<= 1; ++k; }
            return k;
        }
        case LQCS_GATE_PERMUTATION: {
            uint32_t k = 0;
            while ((uint64_t{1} << k) < perm.size()) ++k;
            return k;
        }
        case LQCS_GATE_PAULI_ROTATION:
            return static_cast<uint32_t>(pauli.size());
        case LQCS_GATE_BARRIER:
            return 0;
        default:
            return 1;
    }
}

bool GateDesc::is_unitary() const {
    return type != LQCS_GATE_MEASURE && type != LQCS_GATE_RESET && type != LQCS_GATE_BARRIER &&
           type != LQCS_GATE_KRAUS;
}

std::string GateDesc::name() const {
    std::string base = base_name(type);
    if (type == LQCS_GATE_PAULI_ROTATION) base = "rp(" + pauli + ")";
    if (n_controls == 0) return base;
    if (n_controls == 1) return "c" + base;
    if (n_controls == 2) return "cc" + base;
    return "mc" + base;
}

PauliMasks pauli_local_masks(const std::string& pauli) {
    PauliMasks m;
    const size_t k = pauli.size();
    for (size_t j = 0; j < k; ++j) {
        const char c = pauli[k - 1 - j];
        const uint64_t bit = uint64_t{1} << j;
        switch (c) {
            case 'I': break;
            case 'X': m.x |= bit; break;
            case 'Y': m.x |= bit; m.zy |= bit; ++m.n_y; break;
            case 'Z': m.zy |= bit; break;
            default: invalid("PauliRotation: pauli must contain only I/X/Y/Z");
        }
    }
    return m;
}

PauliMasks pauli_global_masks(const char* pauli, uint32_t n, const char* who) {
    if (pauli == nullptr) invalid(std::string(who) + ": pauli string is null");
    const size_t len = std::char_traits<char>::length(pauli);
    if (len != n) invalid(std::string(who) + ": pauli string length must equal num_qubits");
    PauliMasks m;
    for (size_t j = 0; j < len; ++j) {
        const uint64_t bit = uint64_t{1} << (n - 1 - j);
        switch (pauli[j]) {
            case 'I': break;
            case 'X': m.x |= bit; break;
            case 'Z': m.zy |= bit; break;
            case 'Y': m.x |= bit; m.zy |= bit; ++m.n_y; break;
            default: invalid(std::string(who) + ": pauli must contain only I/X/Y/Z");
        }
    }
    return m;
}

std::vector<cd> GateDesc::base_matrix() const {
    if (!is_unitary()) logic("Gate::base_matrix: " + name() + " has no matrix");
    const double s2 = std::numbers::sqrt2 / 2.0;
    switch (type) {
        case LQCS_GATE_I: return {1, 0, 0, 1};
        case LQCS_GATE_X: return {0, 1, 1, 0};
        case LQCS_GATE_Y: return {0, -kI, kI, 0};
        case LQCS_GATE_Z: return {1, 0, 0, -1};
        case LQCS_GATE_H: return {s2, s2, s2, -s2};
        case LQCS_GATE_S: return {1, 0, 0, kI};
        case LQCS_GATE_SDG: return {1, 0, 0, -kI};
        case LQCS_GATE_T: return {1, 0, 0, unit(std::numbers::pi / 4)};
        case LQCS_GATE_TDG: return {1, 0, 0, unit(-std::numbers::pi / 4)};
        case LQCS_GATE_SX: return {cd{0.5, 0.5}, cd{0.5, -0.5}, cd{0.5, -0.5}, cd{0.5, 0.5}};
        case LQCS_GATE_RX: {
            const double h = param(*this, 0) / 2;
            return {std::cos(h), -kI * std::sin(h), -kI * std::sin(h), std::cos(h)};
        }
        case LQCS_GATE_RY: {
            const double h = param(*this, 0) / 2;
            return {std::cos(h), -std::sin(h), std::sin(h), std::cos(h)};
        }
        case LQCS_GATE_RZ: {
            const double h = param(*this, 0) / 2;
            return {unit(-h), 0, 0, unit(h)};
        }
        case LQCS_GATE_P: return {1, 0, 0, unit(param(*this, 0))};
        case LQCS_GATE_U: {
            // U(theta, phi, lambda) = [[cos, -e^{i lambda} sin], [e^{i phi} sin, e^{i(phi+lambda)} cos]]
            const double h = param(*this, 0) / 2;
            const double phi = param(*this, 1), lam = param(*this, 2);
            return {std::cos(h), -unit(lam) * std::sin(h), unit(phi) * std::sin(h),
                    unit(phi + lam) * std::cos(h)};
        }
        case LQCS_GATE_SWAP:
            return {1, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 1};
        case LQCS_GATE_ISWAP:
            return {1, 0, 0, 0, 0, 0, kI, 0, 0, kI, 0, 0, 0, 0, 0, 1};
        case LQCS_GATE_RXX: {
            const double h = param(*this, 0) / 2;
            const cd c = std::cos(h), is = kI * std::sin(h);
            return {c, 0, 0, -is, 0, c, -is, 0, 0, -is, c, 0, -is, 0, 0, c};
        }
        case LQCS_GATE_RYY: {
            const double h = param(*this, 0) / 2;
            const cd c = std::cos(h), is = kI * std::sin(h);
            return {c, 0, 0, is, 0, c, -is, 0, 0, -is, c, 0, is, 0, 0, c};
        }
        case LQCS_GATE_RZZ: {
            const double h = param(*this, 0) / 2;
            return {unit(-h), 0, 0, 0, 0, unit(h), 0, 0, 0, 0, unit(h), 0, 0, 0, 0, unit(-h)};
        }
        case LQCS_GATE_PAULI_ROTATION: {
            // exp(-i theta/2 P) = cos(theta/2) I - i sin(theta/2) P,
            // P|col> = i^{n_y} (-1)^{popcount(col & zy)} |col ^ x>
            const uint64_t dim = uint64_t{1} << pauli.size();
            const PauliMasks pm = pauli_local_masks(pauli);
            const double h = param(*this, 0) / 2;
            const cd c = std::cos(h);
            const cd mis{0.0, -std::sin(h)};
            static const cd ipow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
            const cd yph = ipow[pm.n_y % 4];
            std::vector<cd> out(dim * dim, cd{0, 0});
            for (uint64_t col = 0; col < dim; ++col) {
                out[col * dim + col] += c;
                const uint64_t row = col ^ pm.x;
                const double sign = (__builtin_popcountll(col & pm.zy) % 2 == 0) ? 1.0 : -1.0;
                out[row * dim + col] += mis * yph * sign;
            }
            return out;
        }
        case LQCS_GATE_UNITARY:
            return mat;
        case LQCS_GATE_PERMUTATION: {
            const uint64_t dim = perm.size();
            std::vector<cd> m(dim * dim, cd{0, 0});
            for (uint64_t l = 0; l < dim; ++l) m[perm[l] * dim + l] = 1;
            return m;
        }
        default:
            logic("Gate::base_matrix: unhandled gate type");
    }
}

std::vector<cd> GateDesc::full_matrix() const {
    const std::vector<cd> base = base_matrix();
    if (n_controls == 0) return base;
    const uint32_t k = base_qubits();
    const uint64_t bdim = uint64_t{1} << k;
    const uint64_t dim = uint64_t{1} << (n_controls + k);
    const uint64_t cm = (uint64_t{1} << n_controls) - 1;
    std::vector<cd> m(dim * dim, cd{0, 0});
    for (uint64_t col = 0; col < dim; ++col) {
        if ((col & cm) != cm) {
            m[col * dim + col] = 1;
            continue;
        }
        const uint64_t tcol = col >> n_controls;
        for (uint64_t trow = 0; trow < bdim; ++trow) {
            const uint64_t row = (trow << n_controls) | cm;
            m[row * dim + col] = base[trow * bdim + tcol];
        }
    }
    return m;
}

GateDesc decode(const lqcs_instruction& in, uint32_t n_qubits) {
    GateDesc g;
    g.type = in.gate_type;
    const bool known = (in.gate_type >= LQCS_GATE_I && in.gate_type <= LQCS_GATE_BARRIER) ||
                       in.gate_type == LQCS_GATE_KRAUS;
    if (!known) invalid("instruction: unknown gate type " + std::to_string(in.gate_type));
    g.n_controls = in.n_controls;
    if (in.n_qubits > 0 && in.qubits == nullptr) invalid("instruction: qubits pointer is null");
    g.qubits.assign(in.qubits, in.qubits + in.n_qubits);
    if (in.n_params > 3) invalid("instruction: at most 3 parameters");
    g.params.assign(in.params, in.params + in.n_params);
    g.clbit = in.clbit;
    if (g.type == LQCS_GATE_PAULI_ROTATION) {
        if (in.pauli == nullptr) invalid("rp: pauli string is null");
        g.pauli = in.pauli;
        if (g.pauli.empty()) invalid("rp: pauli length must equal qubit count and be non-empty");
        for (char c : g.pauli)
            if (c != 'I' && c != 'X' && c != 'Y' && c != 'Z')
                invalid("rp: pauli must contain only I/X/Y/Z");
    }
    if (g.type == LQCS_GATE_UNITARY) {
        const uint32_t k = in.n_qubits - in.n_controls;
        if (in.n_qubits < in.n_controls || k > 20) invalid("unitary: bad qubit count");
        const uint64_t dim = uint64_t{1} << k;
        if (in.matrix == nullptr) invalid("unitary: matrix pointer is null");
        g.mat.resize(dim * dim);
        for (uint64_t i = 0; i < dim * dim; ++i) g.mat[i] = cd{in.matrix[2 * i], in.matrix[2 * i + 1]};
    }
    if (g.type == LQCS_GATE_PERMUTATION) {
        const uint32_t k = in.n_qubits - in.n_controls;
        if (in.n_qubits < in.n_controls || k > 24) invalid("permutation: bad qubit count");
        const uint64_t dim = uint64_t{1} << k;
        if (in.perm == nullptr) invalid("permutation: table pointer is null");
        g.perm.assign(in.perm, in.perm + dim);
        std::vector<bool> hit(dim, false);
        for (uint64_t v : g.perm) {
            if (v >= dim || hit[v]) invalid("permutation: table is not a bijection");
            hit[v] = true;
        }
    }
    if (g.type == LQCS_GATE_KRAUS) {
        if (in.n_kraus == 0 || in.matrix == nullptr)
            invalid("KrausChannel: needs at least one operator");
        g.kraus.resize(in.n_kraus);
        for (uint32_t o = 0; o < in.n_kraus; ++o)
            for (int e = 0; e < 4; ++e)
                g.kraus[o][e] = cd{in.matrix[8 * o + 2 * e], in.matrix[8 * o + 2 * e + 1]};
        if (g.qubits.size() != 1 || g.n_controls != 0) invalid("kraus: expects 1 qubit");
    }
    // arity: Measure/Reset one qubit; Barrier none; gates n_controls + base_qubits
    uint32_t expect;
    if (g.type == LQCS_GATE_BARRIER) expect = 0;
    else if (g.type == LQCS_GATE_MEASURE || g.type == LQCS_GATE_RESET || g.type == LQCS_GATE_KRAUS) expect = 1;
    else expect = g.n_controls + g.base_qubits();
    if (g.type != LQCS_GATE_BARRIER && g.qubits.size() != expect) {
        invalid(g.name() + ": expects " + std::to_string(expect) + " qubits, got " +
                std::to_string(g.qubits.size()));
    }
    if (g.type == LQCS_GATE_MEASURE && g.n_controls != 0) invalid("append: malformed measure instruction");
    std::unordered_set<uint32_t> seen;
    for (uint32_t q : g.qubits) {
        if (q >= n_qubits) {
            out_of_range("qubit index " + std::to_string(q) + " out of range (num_qubits = " +
                         std::to_string(n_qubits) + ")");
        }
        if (!seen.insert(q).second) invalid(g.name() + ": duplicate qubit " + std::to_string(q));
    }
    return g;
}

std::vector<GateDesc> decode_all(const lqcs_instruction* insts, uint64_t n_insts,
                                 uint32_t n_qubits) {
    if (n_insts > 0 && insts == nullptr) invalid("instructions pointer is null");
    std::vector<GateDesc> out;
    out.reserve(n_insts);
    for (uint64_t i = 0; i < n_insts; ++i) out.push_back(decode(insts[i], n_qubits));
    return out;
}

double gate_alg_fraction(const GateDesc& g) {
    if (!g.is_unitary()) return 0.0;
    const double ctrl = std::ldexp(1.0, -static_cast<int>(g.n_controls));
    if (g.type == LQCS_GATE_SWAP) return 0.5 * ctrl;
    if (g.type == LQCS_GATE_PERMUTATION) {
        uint64_t moved = 0;
        for (uint64_t l = 0; l < g.perm.size(); ++l) moved += (g.perm[l] != l);
        return ctrl * static_cast<double>(moved) / static_cast<double>(g.perm.size());
    }
    if (g.base_qubits() == 1) {
        const std::vector<cd> m = g.base_matrix();
        if (m[1] == cd{0, 0} && m[2] == cd{0, 0}) {
            if (m[0] == cd{1, 0} && m[3] == cd{1, 0}) return 0.0;
            if (m[0] == cd{1, 0} || m[3] == cd{1, 0}) return 0.5 * ctrl;
        }
    }
    return ctrl;
}

double op_flops_per_amp(const DevOp& op) {
    switch (op.kind) {
        case OpKind::K1Q: return (op.diag1 ? 6.0 : 16.0) * op.alg_fraction;
        case OpKind::PHASE: return 6.0 * op.alg_fraction;
        case OpKind::DENSE: return 8.0 * std::ldexp(1.0, static_cast<int>(op.k)) * op.alg_fraction;
        case OpKind::DIAG: return 6.0 * op.alg_fraction;
        case OpKind::PERM: return 0.0;
        case OpKind::PAULI: return 16.0 * op.alg_fraction;
        case OpKind::TILE: return op.tile_flops;
    }
    return 0.0;
}

// ------------------------------------------------------------------ lowering

DevOp lower_gate(const GateDesc& g, uint32_t n) {
    if (!g.is_unitary()) logic("lower_gate: " + g.name() + " is not unitary");
    DevOp op;
    op.alg_fraction = gate_alg_fraction(g);
    const uint32_t nc = g.n_controls;
    const uint32_t k = g.base_qubits();
    op.k = k;
    op.targets.assign(g.targets(), g.targets() + k);
    for (uint32_t c = 0; c < nc; ++c) op.cmask |= uint64_t{1} << g.controls()[c];

    if (g.type == LQCS_GATE_PERMUTATION) {
        op.kind = OpKind::PERM;
        perm_cycles(g.perm, op.cycles, op.cycle_len);
        return op;
    }
    if (g.type == LQCS_GATE_SWAP) {
        op.kind = OpKind::PERM;
        op.cycles = {1, 2};
        op.cycle_len = {2};
        return op;
    }
    if (g.type == LQCS_GATE_PAULI_ROTATION && nc == 0 && n >= 5) {
        const PauliMasks pm = pauli_local_masks(g.pauli);
        op.kind = OpKind::PAULI;
        for (uint32_t j = 0; j < k; ++j) {
            if ((pm.x >> j) & 1) op.x |= uint64_t{1} << op.targets[j];
            if ((pm.zy >> j) & 1) op.zy |= uint64_t{1} << op.targets[j];
        }
        op.n_y = pm.n_y;
        const double h = param(g, 0) / 2;
        op.cos_h = std::cos(h);
        op.sin_h = std::sin(h);
        return op;
    }
    std::vector<cd> m = g.base_matrix();
    const uint64_t dim = uint64_t{1} << k;
    const bool diag = is_diag_matrix(m, dim);
    if (k == 1 && n >= 5) {
        if (diag && m[0] == cd{1.0, 0.0}) {
            op.kind = OpKind::PHASE;
            op.phase_mask = op.cmask | (uint64_t{1} << op.targets[0]);
            op.phase = m[3];
            return op;
        }
        op.kind = OpKind::K1Q;
        op.m1 = {m[0], m[1], m[2], m[3]};
        op.diag1 = diag;
        return op;
    }
    if (k > 6) invalid(g.name() + ": dense gates wider than 6 target qubits are not supported");
    if (diag) {
        op.kind = OpKind::DIAG;
        op.mat.resize(dim);
        for (uint64_t i = 0; i < dim; ++i) op.mat[i] = m[i * dim + i];
    } else {
        op.kind = OpKind::DENSE;
        op.mat = std::move(m);
    }
    return op;
}

// ------------------------------------------------------------------ fusion

std::vector<FusedBlock> plan_greedy(const std::vector<GateDesc>& gates, uint32_t n,
                                    uint32_t max_width) {
    std::vector<FusedBlock> out;
    std::vector<FusedBlock> open;
    std::vector<bool> alive;
    std::vector<int> owner(n, -1);
    auto close = [&](int b) {
        if (!alive[b]) return;
        alive[b] = false;
        for (uint32_t q : open[b].qubits) owner[q] = -1;
        out.push_back(std::move(open[b]));
    };
    for (uint32_t gi = 0; gi < gates.size(); ++gi) {
        const GateDesc& g = gates[gi];
        std::vector<int> touched;
        for (uint32_t q : g.qubits)
            if (owner[q] >= 0 && std::find(touched.begin(), touched.end(), owner[q]) == touched.end())
                touched.push_back(owner[q]);
        std::vector<uint32_t> uni(g.qubits.begin(), g.qubits.end());
        for (int b : touched) uni.insert(uni.end(), open[b].qubits.begin(), open[b].qubits.end());
        std::sort(uni.begin(), uni.end());
        uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
        FusedBlock nb;
        if (g.qubits.size() > max_width || uni.size() > max_width) {
            for (int b : touched) close(b);
            nb.qubits.assign(g.qubits.begin(), g.qubits.end());
            std::sort(nb.qubits.begin(), nb.qubits.end());
            nb.gates = {gi};
            if (g.qubits.size() > max_width) {
                out.push_back(std::move(nb));
                continue;
            }
        } else {
            nb.qubits = uni;
            for (int b : touched) {
                nb.gates.insert(nb.gates.end(), open[b].gates.begin(), open[b].gates.end());
                alive[b] = false;
            }
            std::sort(nb.gates.begin(), nb.gates.end());
            nb.gates.push_back(gi);
        }
        const int id = static_cast<int>(open.size());
        for (uint32_t q : nb.qubits) owner[q] = id;
        open.push_back(std::move(nb));
        alive.push_back(true);
    }
    for (int b = 0; b < static_cast<int>(open.size()); ++b) close(b);
    return pack_consecutive(out, max_width);
}

std::vector<FusedBlock> pack_consecutive(const std::vector<FusedBlock>& blocks,
                                         uint32_t max_width) {
    // Two blocks adjacent in a valid emission order can always be concatenated; their
    // gates keep program order within the merged block.
    std::vector<FusedBlock> out;
    for (const FusedBlock& b : blocks) {
        if (!out.empty()) {
            FusedBlock& last = out.back();
            std::vector<uint32_t> uni = last.qubits;
            uni.insert(uni.end(), b.qubits.begin(), b.qubits.end());
            std::sort(uni.begin(), uni.end());
            uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
            if (uni.size() <= max_width) {
                last.qubits = std::move(uni);
                last.gates.insert(last.gates.end(), b.gates.begin(), b.gates.end());
                std::sort(last.gates.begin(), last.gates.end());
                continue;
            }
        }
        out.push_back(b);
    }
    return out;
}

std::vector<cd> block_matrix(const FusedBlock& b, const std::vector<GateDesc>& gates) {
    const uint32_t k = static_cast<uint32_t>(b.qubits.size());
    const uint64_t dim = uint64_t{1} << k;
    std::vector<cd> m(dim * dim, cd{0, 0});
    // columns evolve independently: column c starts as e_c
    std::vector<std::vector<cd>> cols(dim, std::vector<cd>(dim, cd{0, 0}));
    for (uint64_t c = 0; c < dim; ++c) cols[c][c] = 1.0;
    for (uint32_t gi : b.gates) {
        const GateDesc& g = gates[gi];
        std::vector<uint32_t> pos;
        for (uint32_t q : g.qubits) {
            const auto it = std::find(b.qubits.begin(), b.qubits.end(), q);
            pos.push_back(static_cast<uint32_t>(it - b.qubits.begin()));
        }
        const std::vector<cd> f = g.full_matrix();
        for (uint64_t c = 0; c < dim; ++c) apply_small(cols[c], k, pos, f);
    }
    for (uint64_t c = 0; c < dim; ++c)
        for (uint64_t r = 0; r < dim; ++r) m[r * dim + c] = cols[c][r];
    return m;
}

std::vector<DevOp> lower_plan(const std::vector<FusedBlock>& plan,
                              const std::vector<GateDesc>& gates, uint32_t n) {
    std::vector<DevOp> ops;
    ops.reserve(plan.size());
    for (const FusedBlock& b : plan) {
        if (b.gates.size() == 1) {
            ops.push_back(lower_gate(gates[b.gates[0]], n));
            continue;
        }
        const uint32_t k = static_cast<uint32_t>(b.qubits.size());
        const uint64_t dim = uint64_t{1} << k;
        std::vector<cd> m = block_matrix(b, gates);
        DevOp op;
        op.k = k;
        op.targets = b.qubits;
        op.src_gates = static_cast<uint32_t>(b.gates.size());
        op.alg_fraction = 1.0;   // a fused block reads and writes every amplitude
        const bool diag = is_diag_matrix(m, dim);
        if (k == 1 && n >= 5) {
            if (diag && m[0] == cd{1.0, 0.0}) {
                op.kind = OpKind::PHASE;
                op.phase_mask = uint64_t{1} << b.qubits[0];
                op.phase = m[3];
            } else {
                op.kind = OpKind::K1Q;
                op.m1 = {m[0], m[1], m[2], m[3]};
                op.diag1 = diag;
            }
        } else if (diag) {
            op.kind = OpKind::DIAG;
            op.mat.resize(dim);
            for (uint64_t i = 0; i < dim; ++i) op.mat[i] = m[i * dim + i];
        } else {
            op.kind = OpKind::DENSE;
            op.mat = std::move(m);
        }
        ops.push_back(std::move(op));
    }
    return ops;
}

}  // namespace lqcs_b200
