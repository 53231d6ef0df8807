// traj_kernels.cu — batched per-shot evolution: many trajectories resident at once.
//
// The reference evolves shots one after another (run_per_shot,
// src/backend/statevector_simulator.cpp:156-190): per Measure a collapse
// (gate_kernels.cpp:227-247), per Reset a reset (:249-260), per noise point one uniform,
// a branch probability ||K_i psi||^2 per Kraus operator and K_i/sqrt(p_i) applied
// (statevector_simulator.cpp:122-144).  Here R trajectories advance together: state b of a
// batch is trajectory `first + b`; every random decision of trajectory t reads its own
// uniform u[t * per_shot + j], so decisions stay per trajectory while each kernel walks the
// whole batch.  No host round trip happens inside a batch.
#include <algorithm>
#include <stdexcept>
#include <string>

#include "traj.cuh"

namespace lqcs_b200 {

namespace {

void check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA launch failed in ") + what + ": " +
                                 cudaGetErrorString(e));
    }
    count_launch();
}

constexpr uint32_t kThreads = 256;

uint32_t blocks_per_state(const LaunchCtx& ctx, uint64_t work, uint32_t batch) {
    const uint64_t want = (work + kThreads - 1) / kThreads;
    const uint64_t cap = std::max<uint64_t>(1, static_cast<uint64_t>(ctx.num_sms) * 8 /
                                                   std::max(1u, batch));
    return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>({want, cap,
                                                                           kTrajMaxBlocks})));
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* out_row, uint32_t stride) {
    __shared__ double sh[NV][kThreads / 32];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0.0;
        for (int w = 0; w < static_cast<int>(kThreads / 32); ++w) t += sh[threadIdx.x][w];
        out_row[threadIdx.x * stride] = t;
    }
}

// Per state: rho of qubit q = {sum |a0|^2, sum |a1|^2, Re sum a0 conj(a1), Im ...}
// partials layout [state][value][block]
__global__ void __launch_bounds__(kThreads) k_b_rdm1(const double2* __restrict__ st, uint64_t len,
                                                     uint32_t q, double* __restrict__ partials,
                                                     const int* __restrict__ skip) {
    if (skip && skip[blockIdx.y] >= 0) return;   // branch known: no reduction needed
    const double2* s = st + static_cast<uint64_t>(blockIdx.y) * len;
    const uint64_t half = len >> 1, qb = uint64_t{1} << q;
    double v[4] = {0, 0, 0, 0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < half;
         g += stride) {
        const uint64_t i0 = insert_zero_bit(g, q);
        const double2 a0 = __ldg(s + i0), a1 = __ldg(s + (i0 | qb));
        v[0] += a0.x * a0.x + a0.y * a0.y;
        v[1] += a1.x * a1.x + a1.y * a1.y;
        v[2] += a0.x * a1.x + a0.y * a1.y;
        v[3] += a0.y * a1.x - a0.x * a1.y;
    }
    block_sum<4>(v, partials + static_cast<uint64_t>(blockIdx.y) * 4 * gridDim.x + blockIdx.x,
                 gridDim.x);
}

__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// One thread per state: sum the partials, then decide.
// The state need not be normalised: with t = Tr(rho) = rho00 + rho11,
// mode 0 (Kraus): probabilities p_i = Tr(K_i rho K_i^dagger) / t, first i with
//                 u < cumulative p (p <= 0 skipped, last non-zero branch as fallback),
//                 mats[b] = K_i / sqrt(p_i t), flag[b] = 1 (0 only when every probability is
//                 zero: nothing is applied).  A state with a forced branch (forced[b] >= 0)
//                 is left alone.
// mode 1 (measure/reset): p1 = rho11 / t, outcome = u < p1, scale 1/sqrt(rho_oo); the clbit
//                 of the register is set or cleared (measure only).
__global__ void k_b_decide(const double* __restrict__ partials, uint32_t nb, uint32_t batch,
                           TrajDecide d, const double* __restrict__ uniforms, uint64_t first,
                           uint64_t per_shot, double2* __restrict__ mats, int* __restrict__ flag,
                           double* __restrict__ scale, uint64_t* __restrict__ regs) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    if (d.mode == 0 && d.forced && d.forced[b] >= 0) {
        flag[b] = 0;   // branch known in advance: applied by the caller
        return;
    }
    double r[4] = {0, 0, 0, 0};
    const double* row = partials + static_cast<uint64_t>(b) * 4 * nb;
    for (int k = 0; k < 4; ++k)
        for (uint32_t j = 0; j < nb; ++j) r[k] += row[k * nb + j];
    const double u = uniforms[(first + b) * per_shot + d.uniform_index];
    const double tr = r[0] + r[1];
    if (d.mode == 1) {
        const double p1 = r[1] / tr;
        const int outcome = u < p1 ? 1 : 0;
        const double keep = outcome ? r[1] : r[0];
        flag[b] = outcome;
        scale[b] = 1.0 / sqrt(keep);
        if (d.is_measure) {
            const uint64_t bit = uint64_t{1} << d.clbit;
            regs[b] = outcome ? (regs[b] | bit) : (regs[b] & ~bit);
        }
        return;
    }
    const double2 rho00 = make_double2(r[0], 0.0), rho11 = make_double2(r[1], 0.0);
    const double2 rho01 = make_double2(r[2], r[3]), rho10 = make_double2(r[2], -r[3]);
    double cum = 0.0, chosen_p = 0.0;
    int chosen = -1;
    for (uint32_t i = 0; i < d.n_ops; ++i) {
        const double2* k = d.ops + 4 * i;
        double2 p = make_double2(0.0, 0.0);
        for (int row2 = 0; row2 < 2; ++row2) {
            const double2 k0 = k[2 * row2], k1 = k[2 * row2 + 1];
            p = cadd(p, cmul(cmul(k0, rho00), cconj(k0)));
            p = cadd(p, cmul(cmul(k0, rho01), cconj(k1)));
            p = cadd(p, cmul(cmul(k1, rho10), cconj(k0)));
            p = cadd(p, cmul(cmul(k1, rho11), cconj(k1)));
        }
        if (p.x <= 0.0) continue;
        chosen = static_cast<int>(i);
        chosen_p = p.x;   // unnormalised: Tr(K rho K^dagger)
        cum += p.x / tr;
        if (u < cum) break;
    }
    if (chosen < 0) {
        flag[b] = 0;
        return;
    }
    const double inv = 1.0 / sqrt(chosen_p);
    const double2* k = d.ops + 4 * chosen;
    for (int e = 0; e < 4; ++e) mats[4 * b + e] = cscale(k[e], inv);
    flag[b] = 1;
}

// Per-state 2x2 on qubit q (state b uses mats[4b..4b+3]); skipped where flag[b] == 0.
__global__ void __launch_bounds__(kThreads) k_b_apply_mats(double2* __restrict__ st, uint64_t len,
                                                           uint32_t q, const double2* __restrict__ mats,
                                                           const int* __restrict__ flag) {
    const uint32_t b = blockIdx.y;
    if (flag[b] == 0) return;
    double2* s = st + static_cast<uint64_t>(b) * len;
    const double2 m0 = mats[4 * b], m1 = mats[4 * b + 1], m2 = mats[4 * b + 2], m3 = mats[4 * b + 3];
    const uint64_t half = len >> 1, qb = uint64_t{1} << q;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < half;
         g += stride) {
        const uint64_t i0 = insert_zero_bit(g, q);
        const double2 a0 = s[i0], a1 = s[i0 | qb];
        s[i0] = cmad(m1, a1, cmul(m0, a0));
        s[i0 | qb] = cmad(m3, a1, cmul(m2, a0));
    }
}

// Collapse: keep bit q == outcome[b] scaled by scale[b]; with `reset`, a 1 outcome is then
// moved back to |0> (kernels::reset_qubit).
__global__ void __launch_bounds__(kThreads) k_b_project(double2* __restrict__ st, uint64_t len,
                                                        uint32_t q, const int* __restrict__ outcome,
                                                        const double* __restrict__ scale, int reset) {
    const uint32_t b = blockIdx.y;
    double2* s = st + static_cast<uint64_t>(b) * len;
    const int o = outcome[b];
    const double sc = scale[b];
    const uint64_t half = len >> 1, qb = uint64_t{1} << q;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < half;
         g += stride) {
        const uint64_t i0 = insert_zero_bit(g, q);
        const double2 a0 = s[i0], a1 = s[i0 | qb];
        const double2 z = make_double2(0.0, 0.0);
        if (o == 0) {
            s[i0] = cscale(a0, sc);
            s[i0 | qb] = z;
        } else if (reset) {
            s[i0] = cscale(a1, sc);
            s[i0 | qb] = z;
        } else {
            s[i0] = z;
            s[i0 | qb] = cscale(a1, sc);
        }
    }
}

// Unitary-mixture channels (every K_i proportional to a unitary): the branch does not
// depend on the state, so it is chosen for every trajectory of the whole run up front on
// the host; here each state applies its own (possibly identity-skipped) 2x2.
__global__ void __launch_bounds__(kThreads) k_b_apply_table(double2* __restrict__ st, uint64_t len,
                                                            uint32_t q, const double2* __restrict__ mats,
                                                            const int* __restrict__ choice) {
    const uint32_t b = blockIdx.y;
    const int c = choice[b];
    if (c < 0) return;
    double2* s = st + static_cast<uint64_t>(b) * len;
    const double2 m0 = mats[4 * c], m1 = mats[4 * c + 1], m2 = mats[4 * c + 2], m3 = mats[4 * c + 3];
    const uint64_t half = len >> 1, qb = uint64_t{1} << q;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < half;
         g += stride) {
        const uint64_t i0 = insert_zero_bit(g, q);
        const double2 a0 = s[i0], a1 = s[i0 | qb];
        s[i0] = cmad(m1, a1, cmul(m0, a0));
        s[i0 | qb] = cmad(m3, a1, cmul(m2, a0));
    }
}

// Sum of |a|^2 over the amplitudes of state b whose bits at `fixed` equal vals[b], split by
// bit q (values 0 and 1 of the partials row; 2 and 3 stay zero).
__global__ void __launch_bounds__(kThreads) k_b_tail_sum(const double2* __restrict__ st,
                                                         uint64_t len, uint32_t q, BitList fixed,
                                                         const uint64_t* __restrict__ vals,
                                                         double* __restrict__ partials) {
    const double2* s = st + static_cast<uint64_t>(blockIdx.y) * len;
    const uint64_t val = vals[blockIdx.y];
    const uint64_t count = len >> fixed.n;
    double v[4] = {0, 0, 0, 0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += stride) {
        const uint64_t x = expand_bits(i, fixed) | val;
        const double2 a = __ldg(s + x);
        v[(x >> q) & 1] += a.x * a.x + a.y * a.y;
    }
    block_sum<4>(v, partials + static_cast<uint64_t>(blockIdx.y) * 4 * gridDim.x + blockIdx.x,
                 gridDim.x);
}

__global__ void k_b_tail_decide(const double* __restrict__ partials, uint32_t nb, uint32_t batch,
                                const double* __restrict__ uniforms, uint64_t first,
                                uint64_t per_shot, uint32_t uidx, uint32_t q, uint32_t clbit,
                                uint64_t* __restrict__ vals, uint64_t* __restrict__ regs) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    double r0 = 0.0, r1 = 0.0;
    const double* row = partials + static_cast<uint64_t>(b) * 4 * nb;
    for (uint32_t j = 0; j < nb; ++j) {
        r0 += row[j];
        r1 += row[nb + j];
    }
    const double u = uniforms[(first + b) * per_shot + uidx];
    const int outcome = u < r1 / (r0 + r1) ? 1 : 0;
    if (outcome) vals[b] |= uint64_t{1} << q;
    const uint64_t bit = uint64_t{1} << clbit;
    regs[b] = outcome ? (regs[b] | bit) : (regs[b] & ~bit);
}

struct MarginalArgs {
    uint8_t mq[kMaxQubits];   // measured qubit of table bit j
    uint32_t m;
    uint32_t log_chunks;
    uint64_t free_mask;       // bits of the unmeasured qubits
    uint64_t chunk;           // free indices per chunk
};

// Thread (t, c): table entry t, chunk c of the free indices (enumerated in increasing order
// by the masked increment cur = ((cur | ~free) + 1) & free).  Consecutive threads take
// consecutive t, so measured low qubits give coalesced reads.
__global__ void __launch_bounds__(kThreads) k_marginal_partial(const double2* __restrict__ st,
                                                               MarginalArgs a,
                                                               double* __restrict__ partial) {
    const uint64_t entries = uint64_t{1} << a.m;
    const uint64_t gid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gid >= (entries << a.log_chunks)) return;
    const uint64_t t = gid & (entries - 1), c = gid >> a.m;
    uint64_t base = 0;
    for (uint32_t j = 0; j < a.m; ++j) base |= ((t >> j) & 1u) << a.mq[j];
    // deposit of the chunk's first free index c * chunk into the free bit positions
    uint64_t w = c * a.chunk, cur = 0, rest = a.free_mask;
    while (w != 0 && rest != 0) {
        const uint64_t low = rest & (~rest + 1);
        if (w & 1u) cur |= low;
        w >>= 1;
        rest &= rest - 1;
    }
    double sum = 0.0;
    for (uint64_t k = 0; k < a.chunk; ++k) {
        const double2 v = __ldg(st + (base | cur));
        sum += v.x * v.x + v.y * v.y;
        cur = ((cur | ~a.free_mask) + 1) & a.free_mask;
    }
    partial[c * entries + t] = sum;
}

__global__ void k_marginal_sum(const double* __restrict__ partial, uint64_t entries,
                               uint64_t chunks, double* __restrict__ table) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= entries) return;
    double s = 0.0;
    for (uint64_t c = 0; c < chunks; ++c) s += partial[c * entries + t];
    table[t] = s;
}

}  // namespace

uint64_t marginal_chunks(uint32_t n, uint32_t m) {
    // about 2^21 threads in all, at most one chunk per free index
    const uint32_t lc = m >= 21 ? 0u : std::min<uint32_t>(21u - m, n - m);
    return uint64_t{1} << lc;
}

void launch_marginal_table(const LaunchCtx& ctx, const double2* st, uint32_t n,
                           const uint32_t* mq, uint32_t m, double* partial, double* table) {
    MarginalArgs a{};
    uint64_t meas = 0;
    for (uint32_t j = 0; j < m; ++j) {
        a.mq[j] = static_cast<uint8_t>(mq[j]);
        meas |= uint64_t{1} << mq[j];
    }
    a.m = m;
    const uint64_t chunks = marginal_chunks(n, m);
    a.log_chunks = static_cast<uint32_t>(__builtin_ctzll(chunks));
    a.free_mask = ((uint64_t{1} << n) - 1) & ~meas;
    a.chunk = (uint64_t{1} << (n - m)) >> a.log_chunks;
    const uint64_t entries = uint64_t{1} << m, threads = entries * chunks;
    k_marginal_partial<<<static_cast<unsigned>((threads + kThreads - 1) / kThreads), kThreads, 0,
                         ctx.stream>>>(st, a, chunks == 1 ? table : partial);
    check_launch("marginal_partial");
    if (chunks > 1) {
        k_marginal_sum<<<static_cast<unsigned>((entries + 255) / 256), 256, 0, ctx.stream>>>(
            partial, entries, chunks, table);
        check_launch("marginal_sum");
    }
}

void launch_traj_kraus(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch, uint32_t q,
                       const TrajDecide& d, const double* d_uniforms, uint64_t first,
                       uint64_t per_shot, TrajScratch& s) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = blocks_per_state(ctx, len >> 1, batch);
    k_b_rdm1<<<dim3(nb, batch), kThreads, 0, ctx.stream>>>(st, len, q, s.partials, d.forced);
    check_launch("traj_rdm1");
    k_b_decide<<<(batch + 127) / 128, 128, 0, ctx.stream>>>(s.partials, nb, batch, d, d_uniforms,
                                                             first, per_shot, s.mats, s.flag,
                                                             s.scale, s.regs);
    check_launch("traj_decide");
    k_b_apply_mats<<<dim3(nb, batch), kThreads, 0, ctx.stream>>>(st, len, q, s.mats, s.flag);
    check_launch("traj_apply");
}

void launch_traj_measure(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                         uint32_t q, const TrajDecide& d, const double* d_uniforms,
                         uint64_t first, uint64_t per_shot, int reset, TrajScratch& s) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = blocks_per_state(ctx, len >> 1, batch);
    k_b_rdm1<<<dim3(nb, batch), kThreads, 0, ctx.stream>>>(st, len, q, s.partials, nullptr);
    check_launch("traj_rdm1");
    k_b_decide<<<(batch + 127) / 128, 128, 0, ctx.stream>>>(s.partials, nb, batch, d, d_uniforms,
                                                             first, per_shot, s.mats, s.flag,
                                                             s.scale, s.regs);
    check_launch("traj_decide");
    k_b_project<<<dim3(nb, batch), kThreads, 0, ctx.stream>>>(st, len, q, s.flag, s.scale, reset);
    check_launch("traj_project");
}

void launch_traj_table(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch, uint32_t q,
                       const double2* d_mats, const int* d_choice) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = blocks_per_state(ctx, len >> 1, batch);
    k_b_apply_table<<<dim3(nb, batch), kThreads, 0, ctx.stream>>>(st, len, q, d_mats, d_choice);
    check_launch("traj_table");
}

}  // namespace lqcs_b200

namespace lqcs_b200 {

void launch_traj_tail_measure(const LaunchCtx& ctx, const double2* st, uint32_t n,
                              uint32_t batch, uint32_t q, const BitList& fixed, uint64_t* vals,
                              uint32_t clbit, uint32_t uniform_index, const double* d_uniforms,
                              uint64_t first, uint64_t per_shot, TrajScratch& s) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = blocks_per_state(ctx, len >> fixed.n, batch);
    k_b_tail_sum<<<dim3(nb, batch), kThreads, 0, ctx.stream>>>(st, len, q, fixed, vals, s.partials);
    check_launch("traj_tail_sum");
    k_b_tail_decide<<<(batch + 127) / 128, 128, 0, ctx.stream>>>(s.partials, nb, batch, d_uniforms,
                                                                  first, per_shot, uniform_index, q,
                                                                  clbit, vals, s.regs);
    check_launch("traj_tail_decide");
}

}  // namespace lqcs_b200
