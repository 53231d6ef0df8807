// gate_kernels.cu — sm_100a gate-application kernels for complex128 statevectors.
//
// Memory-bound streaming kernels.  The common access pattern is the "lane chunk":
// the 32 lanes of a warp own 32 consecutive amplitudes (bits 0..4 of the basis index),
// so every warp-wide load is one fully coalesced 512-byte stretch.  Bits that an
// operation fixes above bit 4 (high targets, high controls) are inserted into the chunk
// index, so only chunks in the controlled subspace are read.  Targets below bit 5 are
// exchanged between lanes with warp shuffles instead of strided loads.
//
// Reference semantics: src/backend/kernels/gate_kernels.cpp (per-kernel citations below).
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "kernels.cuh"

namespace lqcs_b200 {

namespace {
std::atomic<uint64_t> g_launches{0};

constexpr uint32_t kThreads = 256;

uint32_t grid_for(const LaunchCtx& ctx, uint64_t threads_needed, uint32_t per_sm = 8) {
    const uint64_t blocks = (threads_needed + kThreads - 1) / kThreads;
    const uint64_t cap = static_cast<uint64_t>(ctx.num_sms) * per_sm;
    return static_cast<uint32_t>(std::max<uint64_t>(1, std::min(blocks, cap)));
}

void check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA launch failed in ") + what + ": " +
                                 cudaGetErrorString(e));
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

// Split a mask into the lane part (bits 0..4) and a sorted list of the bits >= 5.
BitList high_bits(uint64_t mask) {
    BitList bl{};
    for (uint32_t b = 5; b < 64; ++b) {
        if ((mask >> b) & 1) bl.pos[bl.n++] = b;
    }
    return bl;
}

BitList sorted_bits(uint64_t mask) {
    BitList bl{};
    for (uint32_t b = 0; b < 64; ++b) {
        if ((mask >> b) & 1) bl.pos[bl.n++] = b;
    }
    return bl;
}

__device__ __forceinline__ double parity_sign(uint64_t v) {
    return (__popcll(v) & 1) ? -1.0 : 1.0;
}

}  // namespace

uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ============================================================================ 1q gate
// kernels::apply_single_qubit / apply_diagonal_single_qubit /
// apply_controlled_single_qubit (src/backend/kernels/gate_kernels.cpp:26-69), generalised
// to any number of controls.

struct P1Q {
    double2 m0, m1, m2, m3;
    uint64_t cmask_hi;      // control bits >= 5, ORed into every chunk base
    uint64_t n_chunks;      // chunks of 32 amplitudes (pairs of chunks when t >= 5)
    uint64_t batch_stride;  // amplitudes between states of a batch
    uint64_t tbit;          // 1 << t
    uint32_t cmask_lo;      // control bits < 5 (lane predicate)
    uint32_t t;
    int diag;
    BitList fix;            // sorted bits >= 5 inserted into the chunk index
};

// Target t >= 5: lane l of chunk w owns the pair (base|l, base|l|2^t); both halves of the
// pair are read as coalesced 512-byte warp stretches.  Two chunks per iteration keep four
// 16-byte loads in flight per thread.
__global__ void __launch_bounds__(kThreads) k_apply_1q_hi(double2* __restrict__ st, P1Q p) {
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    const uint32_t lane = threadIdx.x & 31u;
    if ((lane & p.cmask_lo) != p.cmask_lo) return;
    const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t tb = p.tbit;
    for (; w + nw < p.n_chunks; w += 2 * nw) {
        const uint64_t i0 = expand_bits(w << 5, p.fix) | p.cmask_hi | lane;
        const uint64_t j0 = expand_bits((w + nw) << 5, p.fix) | p.cmask_hi | lane;
        const double2 a0 = ld_amp(s + i0), a1 = ld_amp(s + (i0 | tb));
        const double2 b0 = ld_amp(s + j0), b1 = ld_amp(s + (j0 | tb));
        if (p.diag) {
            s[i0] = cmul(p.m0, a0); s[i0 | tb] = cmul(p.m3, a1);
            s[j0] = cmul(p.m0, b0); s[j0 | tb] = cmul(p.m3, b1);
        } else {
            s[i0] = cmad(p.m1, a1, cmul(p.m0, a0));
            s[i0 | tb] = cmad(p.m3, a1, cmul(p.m2, a0));
            s[j0] = cmad(p.m1, b1, cmul(p.m0, b0));
            s[j0 | tb] = cmad(p.m3, b1, cmul(p.m2, b0));
        }
    }
    if (w < p.n_chunks) {
        const uint64_t i0 = expand_bits(w << 5, p.fix) | p.cmask_hi | lane;
        const double2 a0 = ld_amp(s + i0), a1 = ld_amp(s + (i0 | tb));
        if (p.diag) {
            s[i0] = cmul(p.m0, a0); s[i0 | tb] = cmul(p.m3, a1);
        } else {
            s[i0] = cmad(p.m1, a1, cmul(p.m0, a0));
            s[i0 | tb] = cmad(p.m3, a1, cmul(p.m2, a0));
        }
    }
}

// Target t < 5: each lane owns one amplitude; the partner amplitude comes from lane
// l ^ 2^t by shuffle.  Lanes failing a low-control predicate still shuffle, but do not store.
__global__ void __launch_bounds__(kThreads) k_apply_1q_lo(double2* __restrict__ st, P1Q p) {
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    const uint32_t lane = threadIdx.x & 31u;
    const bool active = (lane & p.cmask_lo) == p.cmask_lo;
    const bool upper = (lane >> p.t) & 1u;
    const double2 c_self = upper ? p.m3 : p.m0;
    const double2 c_part = upper ? p.m2 : p.m1;
    const int tm = 1 << p.t;
    const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    for (; w + nw < p.n_chunks; w += 2 * nw) {
        const uint64_t i = expand_bits(w << 5, p.fix) | p.cmask_hi | lane;
        const uint64_t j = expand_bits((w + nw) << 5, p.fix) | p.cmask_hi | lane;
        const double2 a = ld_amp(s + i), b = ld_amp(s + j);
        double2 ra, rb;
        if (p.diag) {
            ra = cmul(c_self, a); rb = cmul(c_self, b);
        } else {
            const double2 pa = shfl_xor_d2(a, tm), pb = shfl_xor_d2(b, tm);
            ra = cmad(c_part, pa, cmul(c_self, a));
            rb = cmad(c_part, pb, cmul(c_self, b));
        }
        if (active) { s[i] = ra; s[j] = rb; }
    }
    if (w < p.n_chunks) {
        const uint64_t i = expand_bits(w << 5, p.fix) | p.cmask_hi | lane;
        const double2 a = ld_amp(s + i);
        double2 ra;
        if (p.diag) {
            ra = cmul(c_self, a);
        } else {
            const double2 pa = shfl_xor_d2(a, tm);
            ra = cmad(c_part, pa, cmul(c_self, a));
        }
        if (active) s[i] = ra;
    }
}

void launch_apply_1q(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                     const Apply1QOp& op) {
    if (n < 5) throw std::logic_error("launch_apply_1q: needs n >= 5");
    P1Q p{};
    p.m0 = op.m[0]; p.m1 = op.m[1]; p.m2 = op.m[2]; p.m3 = op.m[3];
    p.t = op.t;
    p.tbit = uint64_t{1} << op.t;
    p.diag = op.diag;
    p.cmask_lo = static_cast<uint32_t>(op.cmask & 31u);
    p.cmask_hi = op.cmask & ~uint64_t{31};
    uint64_t fixmask = p.cmask_hi;
    if (op.t >= 5) fixmask |= p.tbit;
    p.fix = high_bits(fixmask);
    p.n_chunks = (uint64_t{1} << n) >> (5 + p.fix.n);
    p.batch_stride = uint64_t{1} << n;
    dim3 grid(grid_for(ctx, p.n_chunks * 32), batch);
    if (op.t >= 5) k_apply_1q_hi<<<grid, kThreads, 0, ctx.stream>>>(st, p);
    else k_apply_1q_lo<<<grid, kThreads, 0, ctx.stream>>>(st, p);
    check_launch("apply_1q");
}

// ============================================================================ phase
// Diagonal gates with d0 == 1 (T, S, Z, P and their controlled forms) only change the
// amplitudes whose target and control bits are all 1: a streaming multiply of that subspace
// (kernels::apply_diagonal_single_qubit touches all 2^n, gate_kernels.cpp:41-47).

struct PPhase {
    double2 ph;
    uint64_t mask_hi;
    uint64_t n_chunks;
    uint64_t batch_stride;
    uint32_t mask_lo;
    BitList fix;
};

__global__ void __launch_bounds__(kThreads) k_phase(double2* __restrict__ st, PPhase p) {
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    const uint32_t lane = threadIdx.x & 31u;
    if ((lane & p.mask_lo) != p.mask_lo) return;
    const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    for (; w + nw < p.n_chunks; w += 2 * nw) {
        const uint64_t i = expand_bits(w << 5, p.fix) | p.mask_hi | lane;
        const uint64_t j = expand_bits((w + nw) << 5, p.fix) | p.mask_hi | lane;
        const double2 a = ld_amp(s + i), b = ld_amp(s + j);
        s[i] = cmul(p.ph, a);
        s[j] = cmul(p.ph, b);
    }
    if (w < p.n_chunks) {
        const uint64_t i = expand_bits(w << 5, p.fix) | p.mask_hi | lane;
        s[i] = cmul(p.ph, ld_amp(s + i));
    }
}

void launch_phase(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                  uint64_t mask, double2 ph) {
    if (n < 5) throw std::logic_error("launch_phase: needs n >= 5");
    PPhase p{};
    p.ph = ph;
    p.mask_lo = static_cast<uint32_t>(mask & 31u);
    p.mask_hi = mask & ~uint64_t{31};
    p.fix = high_bits(p.mask_hi);
    p.n_chunks = (uint64_t{1} << n) >> (5 + p.fix.n);
    p.batch_stride = uint64_t{1} << n;
    dim3 grid(grid_for(ctx, p.n_chunks * 32), batch);
    k_phase<<<grid, kThreads, 0, ctx.stream>>>(st, p);
    check_launch("phase");
}

// ============================================================================ dense k
// kernels::apply_two_qubit / apply_controlled_unitary
// (src/backend/kernels/gate_kernels.cpp:86-106, 143-167): one thread per group of 2^k
// amplitudes, the group index expanded over the sorted fixed bits, consecutive threads
// on consecutive groups so each of the 2^k loads is coalesced whenever the lowest fixed
// bit is >= 5.  The matrix sits in shared memory and is read as a warp-wide broadcast.

template <int K>
struct PDense {
    uint64_t off[1 << K];   // local index l -> address offset (bit j of l <-> targets[j])
    uint64_t cmask;
    uint64_t n_groups;
    uint64_t batch_stride;
    const double2* mat;
    BitList fixed;          // sorted controls and targets
};

template <int K>
__global__ void __launch_bounds__(kThreads) k_dense(double2* __restrict__ st, PDense<K> p) {
    constexpr int D = 1 << K;
    extern __shared__ double2 sm_mat[];
    for (int i = threadIdx.x; i < D * D; i += blockDim.x) sm_mat[i] = p.mat[i];
    __syncthreads();
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         g < p.n_groups; g += stride) {
        const uint64_t base = expand_bits(g, p.fixed) | p.cmask;
        double2 a[D];
#pragma unroll
        for (int l = 0; l < D; ++l) a[l] = ld_amp(s + (base | p.off[l]));
#pragma unroll
        for (int r = 0; r < D; ++r) {
            double2 acc = cmul(sm_mat[r * D], a[0]);
#pragma unroll
            for (int c = 1; c < D; ++c) acc = cmad(sm_mat[r * D + c], a[c], acc);
            s[base | p.off[r]] = acc;
        }
    }
}

template <int K>
static void dense_impl(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                       const uint32_t* targets, uint64_t cmask, const double2* d_mat) {
    PDense<K> p{};
    uint64_t fixmask = cmask;
    for (int j = 0; j < K; ++j) fixmask |= uint64_t{1} << targets[j];
    for (int l = 0; l < (1 << K); ++l) {
        uint64_t o = 0;
        for (int j = 0; j < K; ++j)
            if ((l >> j) & 1) o |= uint64_t{1} << targets[j];
        p.off[l] = o;
    }
    p.cmask = cmask;
    p.fixed = sorted_bits(fixmask);
    p.n_groups = (uint64_t{1} << n) >> p.fixed.n;
    p.batch_stride = uint64_t{1} << n;
    p.mat = d_mat;
    const size_t smem = sizeof(double2) * (1u << K) * (1u << K);
    if (smem > 48 * 1024) {
        cudaFuncSetAttribute(k_dense<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
    }
    dim3 grid(grid_for(ctx, p.n_groups, K >= 5 ? 2 : 8), batch);
    k_dense<K><<<grid, kThreads, smem, ctx.stream>>>(st, p);
    check_launch("dense");
}

void launch_dense(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                  const uint32_t* targets, uint32_t k, uint64_t cmask,
                  const double2* d_mat) {
    if (dense_mma_enabled(k)) {   // wide blocks on the FP64 tensor path
        launch_dense_mma(ctx, st, n, batch, targets, k, cmask, d_mat);
        return;
    }
    switch (k) {
        case 1: dense_impl<1>(ctx, st, n, batch, targets, cmask, d_mat); break;
        case 2: dense_impl<2>(ctx, st, n, batch, targets, cmask, d_mat); break;
        case 3: dense_impl<3>(ctx, st, n, batch, targets, cmask, d_mat); break;
        case 4: dense_impl<4>(ctx, st, n, batch, targets, cmask, d_mat); break;
        case 5: dense_impl<5>(ctx, st, n, batch, targets, cmask, d_mat); break;
        case 6: dense_impl<6>(ctx, st, n, batch, targets, cmask, d_mat); break;
        default: throw std::logic_error("launch_dense: k out of range");
    }
}

// ============================================================================ diagonal k
template <int K>
struct PDiag {
    uint64_t off[1 << K];
    uint64_t cmask;
    uint64_t n_groups;
    uint64_t batch_stride;
    const double2* diag;
    BitList fixed;
};

template <int K>
__global__ void __launch_bounds__(kThreads) k_diag(double2* __restrict__ st, PDiag<K> p) {
    constexpr int D = 1 << K;
    __shared__ double2 sd[D];
    for (int i = threadIdx.x; i < D; i += blockDim.x) sd[i] = p.diag[i];
    __syncthreads();
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         g < p.n_groups; g += stride) {
        const uint64_t base = expand_bits(g, p.fixed) | p.cmask;
        double2 a[D];
#pragma unroll
        for (int l = 0; l < D; ++l) a[l] = ld_amp(s + (base | p.off[l]));
#pragma unroll
        for (int l = 0; l < D; ++l) s[base | p.off[l]] = cmul(sd[l], a[l]);
    }
}

template <int K>
static void diag_impl(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                      const uint32_t* targets, uint64_t cmask, const double2* d_diag) {
    PDiag<K> p{};
    uint64_t fixmask = cmask;
    for (int j = 0; j < K; ++j) fixmask |= uint64_t{1} << targets[j];
    for (int l = 0; l < (1 << K); ++l) {
        uint64_t o = 0;
        for (int j = 0; j < K; ++j)
            if ((l >> j) & 1) o |= uint64_t{1} << targets[j];
        p.off[l] = o;
    }
    p.cmask = cmask;
    p.fixed = sorted_bits(fixmask);
    p.n_groups = (uint64_t{1} << n) >> p.fixed.n;
    p.batch_stride = uint64_t{1} << n;
    p.diag = d_diag;
    dim3 grid(grid_for(ctx, p.n_groups), batch);
    k_diag<K><<<grid, kThreads, 0, ctx.stream>>>(st, p);
    check_launch("diag");
}

void launch_diag(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                 const uint32_t* targets, uint32_t k, uint64_t cmask,
                 const double2* d_diag) {
    switch (k) {
        case 1: diag_impl<1>(ctx, st, n, batch, targets, cmask, d_diag); break;
        case 2: diag_impl<2>(ctx, st, n, batch, targets, cmask, d_diag); break;
        case 3: diag_impl<3>(ctx, st, n, batch, targets, cmask, d_diag); break;
        case 4: diag_impl<4>(ctx, st, n, batch, targets, cmask, d_diag); break;
        case 5: diag_impl<5>(ctx, st, n, batch, targets, cmask, d_diag); break;
        case 6: diag_impl<6>(ctx, st, n, batch, targets, cmask, d_diag); break;
        default: throw std::logic_error("launch_diag: k out of range");
    }
}

// ============================================================================ permutation
// kernels::apply_controlled_permutation (src/backend/kernels/gate_kernels.cpp:169-189):
// |l> -> |perm[l]> per group.  The permutation is walked as cycles so a thread needs no
// per-group scratch for any k: along a cycle c0 -> c1 -> ... -> c_{m-1} -> c0 the new
// amplitude at c_{i+1} is the old one at c_i.

struct PPerm {
    uint64_t cmask;
    uint64_t n_groups;
    uint64_t batch_stride;
    const uint32_t* cycles;
    const uint32_t* cycle_len;
    uint32_t n_cycles;
    uint32_t total_len;
    uint32_t k;
    uint32_t targets[kMaxQubits];
    BitList fixed;
};

__device__ __forceinline__ uint64_t local_offset(uint32_t l, const PPerm& p) {
    uint64_t o = 0;
    for (uint32_t j = 0; j < p.k; ++j)
        if ((l >> j) & 1u) o |= uint64_t{1} << p.targets[j];
    return o;
}

// Each block converts the cycle table to state offsets once (shared memory); a thread then
// rotates every cycle of its group, eight elements per step: the eight source amplitudes of
// a step are all still unwritten when they are loaded together (a step writes positions
// i..i-7 and reads i-1..i-8), so eight loads are in flight instead of one.
// Off: uint32_t when every target is below bit 32, else uint64_t.  kShared = false (tables
// too large for shared memory, 2^15 entries and up): offsets computed from the global table.
template <typename Off, bool kShared>
__global__ void __launch_bounds__(kThreads) k_perm(double2* __restrict__ st, PPerm p) {
    extern __shared__ __align__(8) unsigned char sm_raw[];
    Off* sm_off = reinterpret_cast<Off*>(sm_raw);
    uint32_t* s_len = reinterpret_cast<uint32_t*>(sm_off + p.total_len);
    if constexpr (kShared) {
        for (uint32_t i = threadIdx.x; i < p.total_len; i += blockDim.x)
            sm_off[i] = static_cast<Off>(local_offset(p.cycles[i], p));
        for (uint32_t i = threadIdx.x; i < p.n_cycles; i += blockDim.x) s_len[i] = p.cycle_len[i];
        __syncthreads();
    }
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         g < p.n_groups; g += stride) {
        double2* __restrict__ sg = s + (expand_bits(g, p.fixed) | p.cmask);
        uint32_t start = 0;
        for (uint32_t c = 0; c < p.n_cycles; ++c) {
            const uint32_t len = kShared ? s_len[c] : p.cycle_len[c];
            auto off = [&](uint32_t i) -> uint64_t {
                if constexpr (kShared) return sm_off[start + i];
                else return local_offset(p.cycles[start + i], p);
            };
            const double2 last = sg[off(len - 1)];
            uint32_t i = len - 1;
            for (; i >= 8; i -= 8) {
                double2 t[8];
#pragma unroll
                for (uint32_t u = 0; u < 8; ++u) t[u] = sg[off(i - 1 - u)];
#pragma unroll
                for (uint32_t u = 0; u < 8; ++u) sg[off(i - u)] = t[u];
            }
            for (; i > 0; --i) sg[off(i)] = sg[off(i - 1)];
            sg[off(0)] = last;
            start += len;
        }
    }
}

void launch_perm(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                 const uint32_t* targets, uint32_t k, uint64_t cmask,
                 const uint32_t* d_cycles, const uint32_t* d_cycle_len, uint32_t n_cycles,
                 uint32_t total_len) {
    if (n_cycles == 0) return;
    PPerm p{};
    uint64_t fixmask = cmask;
    for (uint32_t j = 0; j < k; ++j) {
        fixmask |= uint64_t{1} << targets[j];
        p.targets[j] = targets[j];
    }
    p.k = k;
    p.cmask = cmask;
    p.fixed = sorted_bits(fixmask);
    p.n_groups = (uint64_t{1} << n) >> p.fixed.n;
    p.batch_stride = uint64_t{1} << n;
    p.cycles = d_cycles;
    p.cycle_len = d_cycle_len;
    p.n_cycles = n_cycles;
    p.total_len = total_len;
    uint32_t top = 0;
    for (uint32_t j = 0; j < k; ++j) top = std::max(top, targets[j]);
    const bool narrow = top < 32;
    const size_t smem = (narrow ? sizeof(uint32_t) : sizeof(uint64_t)) * total_len +
                        sizeof(uint32_t) * n_cycles;
    dim3 grid(grid_for(ctx, p.n_groups), batch);
    if (smem > 160 * 1024) {
        k_perm<uint64_t, false><<<grid, kThreads, 0, ctx.stream>>>(st, p);
    } else if (narrow) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_perm<uint32_t, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        k_perm<uint32_t, true><<<grid, kThreads, smem, ctx.stream>>>(st, p);
    } else {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_perm<uint64_t, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        k_perm<uint64_t, true><<<grid, kThreads, smem, ctx.stream>>>(st, p);
    }
    check_launch("perm");
}

// ============================================================================ Pauli rotation
// kernels::apply_pauli_rotation (src/backend/kernels/gate_kernels.cpp:191-225):
// new[i] = c a_i + yphase * sign(i ^ x) * a_{i ^ x}, sign(v) = (-1)^popcount(v & zy),
// yphase = -i sin(theta/2) * i^{n_y}.  x == 0 is the diagonal case
// new[i] = a_i (c + yphase sign(i)).  The partner of lane l is lane l ^ (x & 31); when x
// has bits >= 5 a warp owns a chunk A and its partner chunk A ^ (x & ~31).

struct PPauli {
    double2 c;
    double2 yph;
    uint64_t x_hi;
    uint64_t x;
    uint64_t zy;
    uint64_t n_units;
    uint64_t batch_stride;
    const double2* cos_sin;   // per-state (cos, sin) of theta/2, or null
    uint32_t x_lo;
    uint32_t hp;
    uint32_t n_y;
};

__device__ __forceinline__ void pauli_coeffs(const PPauli& p, double2& c, double2& yph) {
    if (p.cos_sin == nullptr) {
        c = p.c;
        yph = p.yph;
        return;
    }
    const double2 cs = p.cos_sin[blockIdx.y];
    c = make_double2(cs.x, 0.0);
    const double2 mis = make_double2(0.0, -cs.y);
    const uint32_t r = p.n_y & 3u;
    const double2 ip = (r == 0) ? make_double2(1, 0)
                     : (r == 1) ? make_double2(0, 1)
                     : (r == 2) ? make_double2(-1, 0) : make_double2(0, -1);
    yph = cmul(mis, ip);
}

template <int MODE>  // 0: diagonal, 1: partner in the same chunk, 2: partner chunk
__global__ void __launch_bounds__(kThreads) k_pauli(double2* __restrict__ st, PPauli p) {
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    double2 c, yph;
    pauli_coeffs(p, c, yph);
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
         w < p.n_units; w += nw) {
        if (MODE == 0) {
            const uint64_t i = (w << 5) | lane;
            const double sg = parity_sign(i & p.zy);
            const double2 f = make_double2(c.x + yph.x * sg, c.y + yph.y * sg);
            s[i] = cmul(ld_amp(s + i), f);
        } else if (MODE == 1) {
            const uint64_t i = (w << 5) | lane;
            const double2 a = ld_amp(s + i);
            const double2 b = shfl_xor_d2(a, static_cast<int>(p.x_lo));
            const double sj = parity_sign((i ^ p.x) & p.zy);
            s[i] = cmad(cscale(yph, sj), b, cmul(c, a));
        } else {
            const uint64_t ia = insert_zero_bit(w << 5, p.hp) | lane;
            const uint64_t ib = ia ^ p.x_hi;
            const double2 a = ld_amp(s + ia), b = ld_amp(s + ib);
            const double2 pa = shfl_xor_d2(b, static_cast<int>(p.x_lo));
            const double2 pb = shfl_xor_d2(a, static_cast<int>(p.x_lo));
            const double sa = parity_sign((ia ^ p.x) & p.zy);
            const double sb = parity_sign((ib ^ p.x) & p.zy);
            s[ia] = cmad(cscale(yph, sa), pa, cmul(c, a));
            s[ib] = cmad(cscale(yph, sb), pb, cmul(c, b));
        }
    }
}

static void pauli_launch(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                         PPauli& p) {
    if (n < 5) throw std::logic_error("launch_pauli_rotation: needs n >= 5");
    p.batch_stride = uint64_t{1} << n;
    p.x_lo = static_cast<uint32_t>(p.x & 31u);
    p.x_hi = p.x & ~uint64_t{31};
    const uint64_t chunks = (uint64_t{1} << n) >> 5;
    int mode;
    if (p.x == 0) {
        mode = 0;
        p.n_units = chunks;
    } else if (p.x_hi == 0) {
        mode = 1;
        p.n_units = chunks;
    } else {
        mode = 2;
        p.hp = static_cast<uint32_t>(__builtin_ctzll(p.x_hi));
        p.n_units = chunks / 2;
    }
    dim3 grid(grid_for(ctx, p.n_units * 32), batch);
    if (mode == 0) k_pauli<0><<<grid, kThreads, 0, ctx.stream>>>(st, p);
    else if (mode == 1) k_pauli<1><<<grid, kThreads, 0, ctx.stream>>>(st, p);
    else k_pauli<2><<<grid, kThreads, 0, ctx.stream>>>(st, p);
    check_launch("pauli_rotation");
}

void launch_pauli_rotation(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                           uint64_t x, uint64_t zy, uint32_t n_y, double cos_h,
                           double sin_h) {
    PPauli p{};
    p.x = x;
    p.zy = zy;
    p.n_y = n_y;
    p.c = make_double2(cos_h, 0.0);
    // yphase = (-i sin) * i^{n_y}, as the reference forms it
    const double2 mis = make_double2(0.0, -sin_h);
    const uint32_t r = n_y & 3u;
    const double2 ip = (r == 0) ? make_double2(1, 0)
                     : (r == 1) ? make_double2(0, 1)
                     : (r == 2) ? make_double2(-1, 0) : make_double2(0, -1);
    p.yph = make_double2(mis.x * ip.x - mis.y * ip.y, mis.x * ip.y + mis.y * ip.x);
    p.cos_sin = nullptr;
    pauli_launch(ctx, st, n, batch, p);
}

void launch_pauli_rotation_batched(const LaunchCtx& ctx, double2* st, uint32_t n,
                                   uint32_t batch, uint64_t x, uint64_t zy, uint32_t n_y,
                                   const double2* d_cos_sin) {
    PPauli p{};
    p.x = x;
    p.zy = zy;
    p.n_y = n_y;
    p.cos_sin = d_cos_sin;
    pauli_launch(ctx, st, n, batch, p);
}

// ============================================================================ utilities

__global__ void k_set_basis(double2* __restrict__ st, uint64_t len, uint64_t index) {
    double2* s = st + static_cast<uint64_t>(blockIdx.y) * len;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
         i += stride) {
        s[i] = make_double2(i == index ? 1.0 : 0.0, 0.0);
    }
}

void launch_set_basis(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                      uint64_t index) {
    const uint64_t len = uint64_t{1} << n;
    dim3 grid(grid_for(ctx, len), batch);
    k_set_basis<<<grid, kThreads, 0, ctx.stream>>>(st, len, index);
    check_launch("set_basis");
}

__global__ void k_scale(double2* __restrict__ st, uint64_t count, double sc) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += stride) {
        const double2 a = st[i];
        st[i] = make_double2(a.x * sc, a.y * sc);
    }
}

void launch_scale(const LaunchCtx& ctx, double2* st, uint64_t count, double s) {
    k_scale<<<grid_for(ctx, count), kThreads, 0, ctx.stream>>>(st, count, s);
    check_launch("scale");
}

__global__ void k_axpy(double2* __restrict__ out, const double2* __restrict__ b, double2 alpha,
                       uint64_t count) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += stride) {
        out[i] = cmad(alpha, b[i], out[i]);
    }
}

void launch_axpy(const LaunchCtx& ctx, double2* out, const double2* b, double2 alpha,
                 uint64_t count) {
    k_axpy<<<grid_for(ctx, count), kThreads, 0, ctx.stream>>>(out, b, alpha, count);
    check_launch("axpy");
}

}  // namespace lqcs_b200
