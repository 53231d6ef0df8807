// reg_emulate.cpp — host emulation of the register tile kernel (k_regtile), for tests.
//
// Two checks of the records the planner lowers a circuit into, without a GPU:
//
// * Values: every thread of every tile is executed as k_regtile executes it (load through
//   layout 0, per-tile diagonal tables, operations and remaps, store through the last
//   layout and the relabelled store bits), out of place, so a tile that stores to an
//   amplitude it did not load (which in place, on the device, would race with the tile that
//   owns it), or an amplitude stored other than once, is found as well as a wrong record.
// * Races: every shared-memory access of the kernel (remap slots and per-tile diagonal
//   tables) is checked against the CUDA barrier model.  Warps run independently between
//   CTA-wide barriers (__syncthreads); threads of a warp run independently between warp
//   barriers (__syncwarp, or a CTA barrier).  Two accesses to one slot, at least one a write,
//   race when they fall in the same CTA-barrier interval and come from different warps, or
//   from different threads of one warp in the same warp-barrier interval.  Each emulated
//   CTA walks its tiles in the kernel's order (tile, tile + grid, ...), so accesses of
//   consecutive tiles of one CTA meet exactly as on the device.
//
// The emulation follows reg_tile_kernels.cu line for line in what it computes; its
// arithmetic is plain std::complex<double> (results agree with the device within rounding).
#include <algorithm>
#include <complex>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.hpp"
#include "tile_plan.hpp"

namespace lqcs_b200 {

namespace {

constexpr int kE = 1 << kRegBits;

uint32_t deposit4(uint32_t l, uint32_t mask) {
    uint32_t out = 0, j = 0;
    for (uint32_t b = 0; b < kRegBits; ++b)
        if ((mask >> b) & 1) {
            if ((l >> j) & 1) out |= 1u << b;
            ++j;
        }
    return out;
}

// Barrier-model bookkeeping of one shared-memory slot.
struct Slot {
    uint64_t epoch = ~uint64_t{0};   // CTA-barrier interval of the accesses below
    bool written = false;
    uint32_t w_warp = 0, w_thread = 0;
    uint64_t w_wepoch = 0;
    uint32_t read_warps = 0;                 // warps that read in this interval
    std::vector<uint64_t> r_wepoch;          // per warp: warp-barrier interval of its reads
    std::vector<int64_t> r_thread;           // the reading thread, -1 for several
};

struct RaceLog {
    uint64_t races = 0;
    std::string first;
};

class CtaModel {
  public:
    // warps 0 .. threads/32 - 1 are the CTA's; one more stands for the asynchronous copies
    // (cp.async), whose writes may land at any time before the waiting barrier
    CtaModel(uint32_t threads, size_t slots) : kT_(threads), warps_((threads + 31) / 32 + 1) {
        slot_.resize(slots);
        for (Slot& s : slot_) {
            s.r_wepoch.assign(warps_, ~uint64_t{0});
            s.r_thread.assign(warps_, -1);
        }
        wepoch_.assign(warps_, 0);
    }
    uint32_t async_thread() const { return (warps_ - 1) * 32; }
    void cta_barrier() {
        ++epoch_;
        for (uint64_t& w : wepoch_) ++w;
    }
    void warp_barrier(uint32_t warp) { ++wepoch_[warp]; }

    void access(size_t idx, uint32_t thread, bool write, const char* what, RaceLog& log,
                uint64_t tile, uint32_t pass) {
        Slot& s = slot_.at(idx);
        const uint32_t warp = thread / 32;
        const uint64_t we = wepoch_[warp];
        if (s.epoch != epoch_) {
            s.epoch = epoch_;
            s.written = false;
            s.read_warps = 0;
        }
        auto conflict = [&](uint32_t ow, uint64_t owe, int64_t ot) {
            if (ow != warp) return true;
            return owe == we && (ot < 0 || static_cast<uint32_t>(ot) != thread);
        };
        bool race = false;
        if (s.written && conflict(s.w_warp, s.w_wepoch, s.w_thread)) race = true;
        if (write) {
            for (uint32_t w = 0; w < warps_ && !race; ++w)
                if ((s.read_warps >> w) & 1u)
                    race = conflict(w, s.r_wepoch[w], s.r_thread[w]);
            s.written = true;
            s.w_warp = warp;
            s.w_thread = thread;
            s.w_wepoch = we;
        } else {
            const bool had = (s.read_warps >> warp) & 1u;
            if (had && s.r_wepoch[warp] == we) {
                if (s.r_thread[warp] != static_cast<int64_t>(thread)) s.r_thread[warp] = -1;
            } else {
                s.r_wepoch[warp] = we;
                s.r_thread[warp] = thread;
            }
            s.read_warps |= 1u << warp;
        }
        if (race) {
            if (log.races == 0) {
                std::ostringstream os;
                os << "pass " << pass << ", tile " << tile << ": " << what << " of shared slot "
                   << idx << " by thread " << thread << " (warp " << warp
                   << ") races with warp " << s.w_warp << " / earlier readers";
                log.first = os.str();
            }
            ++log.races;
        }
    }
    uint32_t threads() const { return kT_; }
    uint64_t epoch() const { return epoch_; }
    uint64_t wepoch(uint32_t warp) const { return wepoch_[warp]; }
    // Whether an access by `thread` now conflicts with an earlier one by (warp, wepoch,
    // thread) in CTA-barrier interval `epoch` (the barrier model above, for global memory).
    bool conflicts(uint64_t epoch, uint32_t warp, uint64_t wepoch, uint32_t other,
                   uint32_t thread) const {
        if (epoch != epoch_) return false;
        if (warp != thread / 32) return true;
        return wepoch == wepoch_[warp] && other != thread;
    }

  private:
    uint32_t kT_, warps_;
    uint64_t epoch_ = 0;
    std::vector<uint64_t> wepoch_;
    std::vector<Slot> slot_;
};

uint64_t insert_zero(uint64_t v, uint32_t pos) {
    const uint64_t low = (uint64_t{1} << pos) - 1;
    return ((v & ~low) << 1) | (v & low);
}

uint32_t thread_slot(const RegLayout& ly, uint32_t tbits, uint32_t t) {
    uint32_t s = 0;
    for (uint32_t i = 0; i < tbits; ++i)
        if ((t >> i) & 1u) s ^= ly.tsw[i];
    return s;
}

uint32_t reg_slot(const RegLayout& ly, uint32_t u) {
    uint32_t s = 0;
    for (uint32_t i = 0; i < kRegBits; ++i)
        if ((u >> i) & 1u) s ^= ly.rsw[i];
    return s;
}

uint64_t thread_goff(const RegLayout& ly, uint32_t tbits, const uint64_t* gbit, uint32_t t) {
    uint64_t g = 0;
    for (uint32_t i = 0; i < tbits; ++i)
        if ((t >> i) & 1u) g |= gbit[ly.tpos[i]];
    return g;
}

uint64_t reg_goff(const RegLayout& ly, const uint64_t* gbit, uint32_t u) {
    uint64_t g = 0;
    for (uint32_t i = 0; i < kRegBits; ++i)
        if ((u >> i) & 1u) g |= gbit[ly.rpos[i]];
    return g;
}

}  // namespace

// Amplitude bookkeeping of one emulated pass: how often each amplitude was stored, and
// which tile loaded it.
struct AmpLog {
    std::vector<uint8_t> written;
    std::vector<uint64_t> owner;
    // the load of each amplitude: CTA-barrier interval, warp, warp-barrier interval, thread
    std::vector<uint64_t> ld_epoch, ld_wepoch;
    std::vector<uint32_t> ld_thread;
};

// Emulate one register pass on `in` (read) / `out` (written; `amps` records stores and
// loading tiles) — values are skipped when in == nullptr — and check its shared-memory
// accesses for every CTA of a grid of `grid` CTAs (only the first `race_ctas` CTAs when
// values are skipped).  sync_tiles: 1 barrier between tiles, 0 none, 2 as the pass says
// (its sync_tiles: where the last layout's warp bits differ from the first's).
//
// pipe: the double-buffered kernel (k_regtile_pipe) instead: each tile's amplitudes arrive
// by asynchronous copies into one of two shared buffers (issued right after the previous
// tile's barrier), are read linearly through layout 0, and the remaps use that buffer; its
// per-tile tables are built before the tile's one barrier.  drop_load_barrier: leave out the
// barrier a relabelling pass puts between its loads and stores (to show that the in-place
// check finds the hazard it prevents).
void emulate_reg_pass(const RegPass& pass, const RegOp* ops, const RegLayout* lays, const cd* mats,
                      uint32_t n, const cd* in, cd* out, AmpLog* amps,
                      uint64_t grid, uint64_t race_ctas, int sync_tiles, bool pipe,
                      bool drop_load_barrier, uint32_t pass_index, RaceLog& log) {
    RegPass p = pass;
    if (sync_tiles != 2) p.sync_tiles = static_cast<uint32_t>(sync_tiles != 0);
    const uint32_t m = p.m;
    const uint32_t kTB = m - kRegBits;
    const uint32_t kT = 1u << kTB;
    const uint64_t n_tiles = (uint64_t{1} << n) >> m;
    uint64_t gbit[kRegMaxBits], sgbit[kRegMaxBits];
    for (uint32_t b = 0; b < m; ++b) {
        gbit[b] = uint64_t{1} << (b < p.L ? b : p.hbits[b - p.L]);
        sgbit[b] = uint64_t{1} << (p.relabel ? p.store_qubit[b] : (b < p.L ? b : p.hbits[b - p.L]));
    }
    const size_t tile_slots = size_t{1} << m;
    const size_t nbuf = pipe ? 2 : 1;
    const size_t dyn_base_slot = nbuf * tile_slots;
    grid = std::max<uint64_t>(1, std::min<uint64_t>(grid, n_tiles));
    const uint64_t ctas = in ? grid : std::min<uint64_t>(grid, std::max<uint64_t>(1, race_ctas));
    std::vector<cd> v(static_cast<size_t>(kT) * kE);
    std::vector<cd> dyn(2 * static_cast<size_t>(p.dyn_entries) + 1);
    std::vector<cd> smem(nbuf * tile_slots);
    auto tile_base = [&](uint64_t tile) {
        uint64_t b = tile << p.L;
        for (uint32_t i = 0; i < p.h; ++i) b = insert_zero(b, p.hbits[i]);
        return b;
    };
    // the double-buffered kernel's copy of a tile into buffer `which`: thread t copies
    // positions j * kT + t from base | (bits of t on tile bits 0..kTB-1) | (bits of j above)
    auto async_copy = [&](CtaModel& model, uint64_t tile, uint32_t which) {
        const uint64_t b = tile_base(tile);
        for (uint32_t t = 0; t < kT; ++t) {
            uint64_t toff = 0;
            for (uint32_t q = 0; q < kTB; ++q)
                if ((t >> q) & 1u) toff |= gbit[q];
            for (uint32_t j = 0; j < kE; ++j) {
                uint64_t a = b | toff;
                for (uint32_t q = 0; q < kRegBits; ++q)
                    if ((j >> q) & 1u) a |= gbit[kTB + q];
                const size_t at = which * tile_slots + j * kT + t;
                model.access(at, model.async_thread(), true, "asynchronous tile copy", log, tile,
                             pass_index);
                if (in) {
                    smem[at] = in[a];
                    if (amps) {
                        amps->owner[a] = tile;
                        amps->ld_epoch[a] = model.epoch();
                        amps->ld_wepoch[a] = model.wepoch(model.async_thread() / 32);
                        amps->ld_thread[a] = model.async_thread();
                    }
                }
            }
        }
    };
    for (uint64_t cta = 0; cta < ctas; ++cta) {
        CtaModel model(kT, nbuf * tile_slots + 2 * static_cast<size_t>(p.dyn_entries));
        model.cta_barrier();   // the prologue's barrier
        if (pipe) async_copy(model, cta, 0);
        uint32_t parity = 0;
        for (uint64_t tid = cta; tid < n_tiles; tid += grid, parity ^= 1u) {
            if (p.sync_tiles && !pipe) model.cta_barrier();
            const uint64_t base = tile_base(tid);
            const size_t boff = pipe ? parity * tile_slots : 0;   // this tile's buffer
            // load through layout 0
            if (in && !pipe) {
                const RegLayout& ly = lays[0];
                for (uint32_t t = 0; t < kT; ++t) {
                    const uint64_t g = base | thread_goff(ly, kTB, gbit, t);
                    for (uint32_t u = 0; u < kE; ++u) {
                        const uint64_t a = g | reg_goff(ly, gbit, u);
                        v[t * kE + u] = in[a];
                        if (amps) {
                            amps->owner[a] = tid;
                            amps->ld_epoch[a] = model.epoch();
                            amps->ld_wepoch[a] = model.wepoch(t / 32);
                            amps->ld_thread[a] = t;
                        }
                    }
                }
            }
            if (!pipe && p.load_barrier && !drop_load_barrier) model.cta_barrier();
            // per-tile diagonal tables
            const uint32_t dyn_base = parity * p.dyn_entries;
            if (p.n_dyn) {
                for (uint32_t t = 0; t < kT; ++t)
                    for (uint32_t w = t; w < p.n_dyn * 64u; w += kT) {
                        const RegOp& op = ops[p.dyn_rec[w >> 6]];
                        const uint32_t e = w & 63u;
                        if (e >= (1u << op.k)) continue;
                        const cd* src = mats + op.mat_off;
                        cd acc = src[e];
                        const cd* term = src + (1u << op.k);
                        for (uint32_t q = 0; q < op.nterm; ++q) {
                            const cd meta = term[2 * q + 1];
                            const uint64_t hi = static_cast<uint64_t>(meta.imag());
                            const uint64_t gc = static_cast<uint64_t>(meta.real()) | ((hi >> 6) << 32);
                            const uint32_t em = static_cast<uint32_t>(hi & 63u);
                            if ((base & gc) == gc && (e & em) == em) acc = term[2 * q] * acc;
                        }
                        const size_t at = dyn_base + op.dyn_off + e;
                        model.access(dyn_base_slot + at, t, true, "per-tile table write", log, tid, pass_index);
                        dyn[at] = acc;
                    }
                if (!pipe) model.cta_barrier();
            }
            if (pipe) {
                model.cta_barrier();   // copies waited for, tables published
                if (tid + grid < n_tiles) async_copy(model, tid + grid, parity ^ 1u);
                const RegLayout& ly = lays[0];
                for (uint32_t t = 0; t < kT; ++t) {
                    uint32_t tp = 0;
                    for (uint32_t i = 0; i < kTB; ++i)
                        if ((t >> i) & 1u) tp |= 1u << ly.tpos[i];
                    for (uint32_t u = 0; u < kE; ++u) {
                        uint32_t pos = tp;
                        for (uint32_t i = 0; i < kRegBits; ++i)
                            if ((u >> i) & 1u) pos |= 1u << ly.rpos[i];
                        model.access(boff + pos, t, false, "layout-0 read", log, tid, pass_index);
                        if (in) v[t * kE + u] = smem[boff + pos];
                    }
                }
                for (uint32_t w = 0; w < (kT + 31) / 32; ++w) model.warp_barrier(w);
            }
            // operations, thread by thread between barriers: a remap is a barrier point, so
            // each thread runs up to the next remap, then the remap's two phases follow; a
            // tensor-path block (warp barrier, then one instruction of the whole warp) is
            // such a point too
            std::vector<uint32_t> cur(kT, 0);
            uint32_t o = 0;
            while (o <= p.n_ops) {
                uint32_t end = o;
                auto warp_wide = [&](const RegOp& r) {
                    return r.kind == kRegRemap || r.kind == kRegMma ||
                           (r.kind == kRegPauli && r.loc[0] != 0);
                };
                while (end < p.n_ops &&
                       !(warp_wide(ops[end]) && (base & ops[end].gcmask) == ops[end].gcmask))
                    ++end;
                // [o, end): non-remap operations, each thread independently
                for (uint32_t t = 0; t < kT; ++t) {
                    cd* vt = &v[t * kE];
                    for (uint32_t i = o; i < end; ++i) {
                        const RegOp& op = ops[i];
                        if ((base & op.gcmask) != op.gcmask) continue;
                        if (op.kind == kRegPauli) {   // rcmask / tcmask: Z-type bits
                            if (!in) continue;
                            const cd c = mats[op.mat_off];
                            cd y = mats[op.mat_off + 1];
                            const cd zd = mats[op.mat_off + 2];
                            const uint64_t zg = static_cast<uint64_t>(zd.real()) |
                                                (static_cast<uint64_t>(zd.imag()) << 32);
                            if ((__builtin_popcountll(base & zg) + __builtin_popcount(t & op.tcmask)) & 1)
                                y = -y;
                            auto sign = [&](uint32_t u) {
                                return (__builtin_popcount(u & op.rcmask) & 1) ? -1.0 : 1.0;
                            };
                            const uint32_t xr = op.code;
                            if (xr == 0) {
                                for (uint32_t u = 0; u < kE; ++u) vt[u] *= c + sign(u) * y;
                                continue;
                            }
                            const uint32_t low = xr & (~xr + 1u);
                            for (uint32_t u = 0; u < kE; ++u) {
                                if (u & low) continue;
                                const uint32_t w = u ^ xr;
                                const cd a = vt[u], b = vt[w];
                                vt[u] = c * a + sign(u) * y * b;
                                vt[w] = c * b + sign(w) * y * a;
                            }
                            continue;
                        }
                        if ((t & op.tcmask) != op.tcmask) continue;
                        const uint32_t rc = op.rcmask;
                        uint32_t moff = op.mat_off;
                        if (op.nsel) {
                            uint32_t sel = 0;
                            for (uint32_t q = 0; q < op.nsel; ++q)
                                sel |= static_cast<uint32_t>((base >> op.selq[q]) & 1u) << q;
                            const uint32_t k2 =
                                op.kind == kRegDense || op.kind == kRegMma ? 2u * op.k : op.k;
                            moff += sel << k2;
                        }
                        if (op.kind == kRegDense) {
                            const uint32_t TM = op.code;
                            const uint32_t K = static_cast<uint32_t>(__builtin_popcount(TM));
                            const uint32_t D = 1u << K;
                            if (!in) continue;
                            for (uint32_t b = 0; b < kE; ++b) {
                                if (b & TM) continue;
                                if ((b & rc) != rc) continue;
                                cd y[8];
                                for (uint32_t r = 0; r < D; ++r) {
                                    cd acc = 0;
                                    for (uint32_t c = 0; c < D; ++c)
                                        acc += mats[moff + r * D + c] * vt[b | deposit4(c, TM)];
                                    y[r] = acc;
                                }
                                for (uint32_t r = 0; r < D; ++r) vt[b | deposit4(r, TM)] = y[r];
                            }
                        } else if (op.kind == kRegPhase) {
                            if (!in) continue;
                            const cd f = mats[moff];
                            for (uint32_t u = 0; u < kE; ++u)
                                if ((u & rc) == rc) vt[u] *= f;
                        } else if (op.kind == kRegSwapX) {
                            if (!in) continue;
                            const uint32_t I = op.code == 1 ? 0 : op.code == 2 ? 1 : op.code == 4 ? 2 : 3;
                            for (uint32_t b = 0; b < kE; ++b) {
                                if ((b >> I) & 1) continue;
                                if ((b & rc) != rc) continue;
                                std::swap(vt[b], vt[b | (1u << I)]);
                            }
                        } else {   // diagonal, fixed or per-tile table
                            uint32_t tpart = 0, rb[kRegBits] = {0, 0, 0, 0};
                            for (uint32_t j = 0; j < op.k; ++j) {
                                const uint32_t loc = op.loc[j];
                                if (loc & 0x80u) tpart |= ((t >> (loc & 0x7fu)) & 1u) << j;
                                else rb[loc] |= 1u << j;
                            }
                            for (uint32_t u = 0; u < kE; ++u) {
                                if ((u & rc) != rc) continue;
                                uint32_t e = tpart;
                                for (uint32_t i2 = 0; i2 < kRegBits; ++i2)
                                    if ((u >> i2) & 1u) e |= rb[i2];
                                cd f;
                                if (op.kind == kRegDiagDyn) {
                                    const size_t at = dyn_base + op.dyn_off + e;
                                    model.access(dyn_base_slot + at, t, false, "per-tile table read", log,
                                                 tid, pass_index);
                                    f = dyn[at];
                                } else {
                                    f = mats[moff + e];
                                }
                                if (in) vt[u] *= f;
                            }
                        }
                    }
                }
                if (end >= p.n_ops) break;
                if (ops[end].kind == kRegPauli) {
                    // flips on lanes: a lane reads its partner lane's registers (shuffles), so
                    // the warp's values are read before any is written
                    const RegOp& op = ops[end];
                    if (in) {
                        const std::vector<cd> snap = v;
                        const cd c = mats[op.mat_off];
                        const cd y0 = mats[op.mat_off + 1];
                        const cd zd = mats[op.mat_off + 2];
                        const uint64_t zg = static_cast<uint64_t>(zd.real()) |
                                            (static_cast<uint64_t>(zd.imag()) << 32);
                        for (uint32_t t = 0; t < kT; ++t) {
                            const uint32_t tp = t ^ op.loc[0];
                            for (uint32_t u = 0; u < kE; ++u) {
                                const int par = __builtin_popcountll(base & zg) +
                                                __builtin_popcount(t & op.tcmask) +
                                                __builtin_popcount(u & op.rcmask);
                                const cd y = (par & 1) ? -y0 : y0;
                                v[t * kE + u] = c * snap[t * kE + u] + y * snap[tp * kE + (u ^ op.code)];
                            }
                        }
                    }
                    o = end + 1;
                    continue;
                }
                if (ops[end].kind == kRegMma) {
                    // every lane of a warp whose warp-bit controls are all 1 (lane controls
                    // never occur: the lowering refuses them); register u's quad of lanes
                    // 4g..4g+3 holds members 0..3 of group g, matrix bit j on lane bit j
                    const RegOp& op = ops[end];
                    uint32_t moff = op.mat_off;
                    if (op.nsel) {
                        uint32_t sel = 0;
                        for (uint32_t q = 0; q < op.nsel; ++q)
                            sel |= static_cast<uint32_t>((base >> op.selq[q]) & 1u) << q;
                        moff += sel << (2u * op.k);
                    }
                    if (op.tcmask & 31u)
                        logic("register tile emulation: a tensor-path block is controlled by a lane bit");
                    for (uint32_t w = 0; w < (kT + 31) / 32; ++w) {
                        const uint32_t t0 = 32 * w;
                        if ((t0 & op.tcmask) != op.tcmask) continue;
                        model.warp_barrier(w);
                        if (!in) continue;
                        for (uint32_t u = 0; u < kE; ++u) {
                            if ((u & op.rcmask) != op.rcmask) continue;
                            for (uint32_t g = 0; g < 8; ++g) {
                                cd a[4], y[4];
                                for (uint32_t k = 0; k < 4; ++k) a[k] = v[(t0 + 4 * g + k) * kE + u];
                                for (uint32_t j = 0; j < 4; ++j) {
                                    y[j] = 0;
                                    for (uint32_t k = 0; k < 4; ++k) y[j] += mats[moff + 4 * j + k] * a[k];
                                }
                                for (uint32_t j = 0; j < 4; ++j) v[(t0 + 4 * g + j) * kE + u] = y[j];
                            }
                        }
                    }
                    o = end + 1;
                    continue;
                }
                // the remap at `end`: write under the current layout, barrier, read under the
                // new one, barrier
                const RegOp& rm = ops[end];
                const bool local = rm.k != 0;
                for (uint32_t t = 0; t < kT; ++t) {
                    const RegLayout& ly = lays[cur[t]];
                    const uint32_t ts = thread_slot(ly, kTB, t);
                    for (uint32_t u = 0; u < kE; ++u) {
                        const size_t sl = boff + (ts ^ reg_slot(ly, u));
                        model.access(sl, t, true, "remap write", log, tid, pass_index);
                        if (in) smem[sl] = v[t * kE + u];
                    }
                }
                if (local) {
                    for (uint32_t w = 0; w < (kT + 31) / 32; ++w) model.warp_barrier(w);
                } else {
                    model.cta_barrier();
                }
                for (uint32_t t = 0; t < kT; ++t) {
                    cur[t] = rm.code;
                    const RegLayout& ly = lays[cur[t]];
                    const uint32_t ts = thread_slot(ly, kTB, t);
                    for (uint32_t u = 0; u < kE; ++u) {
                        const size_t sl = boff + (ts ^ reg_slot(ly, u));
                        model.access(sl, t, false, "remap read", log, tid, pass_index);
                        if (in) v[t * kE + u] = smem[sl];
                    }
                }
                if (local) {
                    for (uint32_t w = 0; w < (kT + 31) / 32; ++w) model.warp_barrier(w);
                } else {
                    model.cta_barrier();
                }
                o = end + 1;
            }
            // store through the last layout and the (relabelled) store bits
            if (in) {
                for (uint32_t t = 0; t < kT; ++t) {
                    const RegLayout& ly = lays[cur[t]];
                    const uint64_t g = base | thread_goff(ly, kTB, sgbit, t);
                    for (uint32_t u = 0; u < kE; ++u) {
                        const uint64_t a = g | reg_goff(ly, sgbit, u);
                        out[a] = v[t * kE + u];
                        if (amps) {
                            ++amps->written[a];
                            // in place: a store may not overtake another thread's load of
                            // the same amplitude (a pass that relabels stores to places
                            // other warps load)
                            if (model.conflicts(amps->ld_epoch[a], amps->ld_thread[a] / 32,
                                                amps->ld_wepoch[a], amps->ld_thread[a], t)) {
                                if (log.races == 0) {
                                    std::ostringstream os;
                                    os << "pass " << pass_index << ", tile " << tid
                                       << ": store of amplitude " << a << " by thread " << t
                                       << " may overtake its load by thread " << amps->ld_thread[a]
                                       << " (no barrier between them)";
                                    log.first = os.str();
                                }
                                ++log.races;
                            }
                            if (amps->owner[a] != tid)
                                logic("register tile emulation: pass " + std::to_string(pass_index) +
                                      ", tile " + std::to_string(tid) + " stores amplitude " +
                                      std::to_string(a) + ", which tile " +
                                      std::to_string(amps->owner[a]) + " loaded");
                        }
                    }
                }
            }
        }
    }
}

// Plan and lower a circuit into register tile passes with the default tile configuration
// (environment overrides included) and emulate every pass; see lqcs_debug_emulate_register_passes.
void emulate_register_program(uint32_t n, const lqcs_instruction* insts, uint64_t n_insts,
                              uint64_t grid, int sync_tiles, bool pipe, bool drop_load_barrier,
                              cd* state, uint64_t race_ctas, uint64_t* n_passes,
                              uint64_t* n_races, std::string* report) {
    const auto gates = decode_all(insts, n_insts, n);
    const TileConfig cfg = default_tile_config(n);
    if (!cfg.reg) invalid("register tile emulation: register passes are switched off");
    const auto items = plan_tiles(gates, n, cfg);
    RaceLog log;
    uint64_t passes = 0;
    std::vector<cd> next;
    AmpLog amps;
    if (state) {
        next.resize(size_t{1} << n);
        amps.owner.resize(size_t{1} << n);
        amps.ld_epoch.resize(size_t{1} << n);
        amps.ld_wepoch.resize(size_t{1} << n);
        amps.ld_thread.resize(size_t{1} << n);
    }
    for (const PlanItem& it : items) {
        if (!it.is_pass)
            invalid("register tile emulation: gate " + std::to_string(it.gate) +
                    " runs on its own (not a register pass)");
        RegPass rp;
        std::vector<RegOp> ops;
        std::vector<RegLayout> lays;
        std::vector<cd> mats;
        if (!lower_pass_reg(it, gates, cfg, rp, ops, lays, mats))
            invalid("register tile emulation: a pass does not fit the register kernel");
        rp.batch_stride = uint64_t{1} << n;
        rp.n_tiles = (uint64_t{1} << n) >> rp.m;
        if (state) amps.written.assign(size_t{1} << n, 0);
        emulate_reg_pass(rp, ops.data(), lays.data(), mats.data(), n, state, state ? next.data() : nullptr,
                         state ? &amps : nullptr, grid, race_ctas, sync_tiles,
                         pipe && (rp.m == 11 || rp.m == 12), drop_load_barrier,
                         static_cast<uint32_t>(passes), log);
        if (state) {
            for (size_t a = 0; a < amps.written.size(); ++a)
                if (amps.written[a] != 1)
                    logic("register tile emulation: pass " + std::to_string(passes) +
                          " wrote amplitude " + std::to_string(a) + " " +
                          std::to_string(amps.written[a]) + " times");
            std::memcpy(state, next.data(), sizeof(cd) * next.size());
        }
        ++passes;
    }
    *n_passes = passes;
    *n_races = log.races;
    if (report) *report = log.first;
}

}  // namespace lqcs_b200
