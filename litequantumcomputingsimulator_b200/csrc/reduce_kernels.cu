// reduce_kernels.cu — read-only passes over the statevector: norms, Born-rule
// probabilities, Kraus branch probabilities, Pauli expectations, prefix sums for shot
// sampling, and the projection kernels of mid-circuit measurement.
//
// Every reduction is deterministic: a fixed grid (reduce_grid), a fixed per-thread
// traversal, a butterfly warp reduction, a fixed-order block combine, and a one-block
// final pass over the per-block partials.  Two runs on the same input agree bit for bit.
#include <algorithm>
#include <stdexcept>
#include <string>

#include "kernels.cuh"

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

__device__ __forceinline__ double parity_sign(uint64_t v) {
    return (__popcll(v) & 1) ? -1.0 : 1.0;
}

// Sum NV values over the block; thread 0..NV-1 write the block totals to out[k*stride].
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double* out,
                                                uint64_t stride) {
    __shared__ double sh[NV][kReduceThreads / 32];
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
        for (int w = 0; w < static_cast<int>(kReduceThreads / 32); ++w) t += sh[threadIdx.x][w];
        out[threadIdx.x * stride] = t;
    }
}

// Final pass: out[k] = sum_b partials[k*nb + b], one block, fixed order.
template <int NV>
__global__ void __launch_bounds__(kReduceThreads) k_finalize(const double* __restrict__ partials,
                                                             uint32_t nb, double* __restrict__ out) {
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += partials[k * static_cast<uint64_t>(nb) + b];
    }
    block_sum_store<NV>(v, out, 1);
}

template <int NV>
void finalize(const LaunchCtx& ctx, const double* partials, uint32_t nb, double* out) {
    k_finalize<NV><<<1, kReduceThreads, 0, ctx.stream>>>(partials, nb, out);
    check_launch("finalize");
}

}  // namespace

uint32_t reduce_grid(const LaunchCtx& ctx, uint64_t work_items) {
    const uint64_t blocks = (work_items + kReduceThreads - 1) / kReduceThreads;
    const uint64_t cap = std::min<uint64_t>(kMaxReduceBlocks,
                                            static_cast<uint64_t>(ctx.num_sms) * 8);
    return static_cast<uint32_t>(std::max<uint64_t>(1, std::min(blocks, cap)));
}

// ---------------------------------------------------------------- norm^2
// Statevector::norm (src/backend/statevector.cpp:27-31)
__global__ void __launch_bounds__(kReduceThreads) k_norm2(const double2* __restrict__ s,
                                                          uint64_t len, double* partials) {
    double v[1] = {0.0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
         i += stride) {
        const double2 a = __ldg(s + i);
        v[0] += norm_rn(a);
    }
    block_sum_store<1>(v, partials + blockIdx.x, gridDim.x);
}

void launch_norm2(const LaunchCtx& ctx, const double2* st, uint32_t n, double* d_partials,
                  double* d_out) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = reduce_grid(ctx, len);
    k_norm2<<<nb, kReduceThreads, 0, ctx.stream>>>(st, len, d_partials);
    check_launch("norm2");
    finalize<1>(ctx, d_partials, nb, d_out);
}

// ---------------------------------------------------------------- P(bit q == 1)
// first loop of kernels::collapse_qubit (src/backend/kernels/gate_kernels.cpp:229-234)
__global__ void __launch_bounds__(kReduceThreads) k_bitprob(const double2* __restrict__ s,
                                                            uint64_t half, uint32_t q,
                                                            double* partials) {
    double v[1] = {0.0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t qb = uint64_t{1} << q;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < half;
         g += stride) {
        const uint64_t i = insert_zero_bit(g, q) | qb;
        v[0] += norm_rn(__ldg(s + i));
    }
    block_sum_store<1>(v, partials + blockIdx.x, gridDim.x);
}

void launch_bitprob(const LaunchCtx& ctx, const double2* st, uint32_t n, uint32_t q,
                    double* d_partials, double* d_out) {
    const uint64_t half = (uint64_t{1} << n) >> 1;
    const uint32_t nb = reduce_grid(ctx, half);
    k_bitprob<<<nb, kReduceThreads, 0, ctx.stream>>>(st, half, q, d_partials);
    check_launch("bitprob");
    finalize<1>(ctx, d_partials, nb, d_out);
}

// ---------------------------------------------------------------- reduced density matrix
// One read of the state gives rho_q = sum over pairs (a0, a1)(a0, a1)^dagger, from which
// every Kraus branch probability Tr(K rho K^dagger) follows on the host.
__global__ void __launch_bounds__(kReduceThreads) k_rdm1(const double2* __restrict__ s,
                                                         uint64_t half, uint32_t q,
                                                         double* partials) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t qb = uint64_t{1} << q;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < half;
         g += stride) {
        const uint64_t i0 = insert_zero_bit(g, q);
        const double2 a0 = __ldg(s + i0), a1 = __ldg(s + (i0 | qb));
        v[0] += a0.x * a0.x + a0.y * a0.y;
        v[1] += a1.x * a1.x + a1.y * a1.y;
        // a0 * conj(a1)
        v[2] += a0.x * a1.x + a0.y * a1.y;
        v[3] += a0.y * a1.x - a0.x * a1.y;
    }
    block_sum_store<4>(v, partials + blockIdx.x, gridDim.x);
}

void launch_rdm1(const LaunchCtx& ctx, const double2* st, uint32_t n, uint32_t q,
                 double* d_partials, double* d_out) {
    const uint64_t half = (uint64_t{1} << n) >> 1;
    const uint32_t nb = reduce_grid(ctx, half);
    k_rdm1<<<nb, kReduceThreads, 0, ctx.stream>>>(st, half, q, d_partials);
    check_launch("rdm1");
    finalize<4>(ctx, d_partials, nb, d_out);
}

// ---------------------------------------------------------------- Kraus probability
// kernels::kraus_probability (src/backend/kernels/gate_kernels.cpp:262-277)
struct PKraus {
    double2 k0, k1, k2, k3;
};
__global__ void __launch_bounds__(kReduceThreads) k_kraus_prob(const double2* __restrict__ s,
                                                               uint64_t half, uint32_t q,
                                                               PKraus k, double* partials) {
    double v[1] = {0.0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t qb = uint64_t{1} << q;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < half;
         g += stride) {
        const uint64_t i0 = insert_zero_bit(g, q);
        const double2 a0 = __ldg(s + i0), a1 = __ldg(s + (i0 | qb));
        const double2 b0 = cadd(cmul(k.k0, a0), cmul(k.k1, a1));
        const double2 b1 = cadd(cmul(k.k2, a0), cmul(k.k3, a1));
        v[0] += norm_rn(b0) + norm_rn(b1);
    }
    block_sum_store<1>(v, partials + blockIdx.x, gridDim.x);
}

void launch_kraus_prob(const LaunchCtx& ctx, const double2* st, uint32_t n, uint32_t q,
                       const double2 k[4], double* d_partials, double* d_out) {
    const uint64_t half = (uint64_t{1} << n) >> 1;
    const uint32_t nb = reduce_grid(ctx, half);
    PKraus pk{k[0], k[1], k[2], k[3]};
    k_kraus_prob<<<nb, kReduceThreads, 0, ctx.stream>>>(st, half, q, pk, d_partials);
    check_launch("kraus_prob");
    finalize<1>(ctx, d_partials, nb, d_out);
}

// ---------------------------------------------------------------- Pauli expectation
// Statevector::expectation_value (src/backend/statevector.cpp:39-78):
// <P> = Re( i^{n_y} sum_i (-1)^{popcount(i & zy)} a_i conj(a_{i ^ x}) ).
// Terms sharing an x mask share the one read of a_i and a_{i ^ x}.
struct PExpect {
    uint64_t x;
    uint64_t len;
    uint32_t n_terms;
    uint32_t n_y[kMaxTermsPerPass];
    uint64_t zy[kMaxTermsPerPass];
};

__global__ void __launch_bounds__(kReduceThreads) k_expect(const double2* __restrict__ s,
                                                           PExpect p, double* partials) {
    double v[2 * kMaxTermsPerPass];
#pragma unroll
    for (int k = 0; k < static_cast<int>(2 * kMaxTermsPerPass); ++k) v[k] = 0.0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    if (p.x == 0) {
        for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
             i < p.len; i += stride) {
            const double2 a = __ldg(s + i);
            const double wr = a.x * a.x + a.y * a.y;
#pragma unroll
            for (int t = 0; t < static_cast<int>(kMaxTermsPerPass); ++t) {
                if (t < static_cast<int>(p.n_terms)) v[2 * t] += parity_sign(i & p.zy[t]) * wr;
            }
        }
    } else {
        // each pair (i, i ^ x) once: the term at i ^ x is the conjugate of the one at i, with
        // its own sign, so every amplitude is read once
        const unsigned hb = 63u - static_cast<unsigned>(__clzll(p.x));
        for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
             g < p.len / 2; g += stride) {
            const uint64_t i = insert_zero_bit(g, hb), j = i ^ p.x;
            const double2 a = __ldg(s + i), b = __ldg(s + j);
            // a * conj(b) at i; b * conj(a) = its conjugate at j
            const double wr = a.x * b.x + a.y * b.y;
            const double wi = a.y * b.x - a.x * b.y;
#pragma unroll
            for (int t = 0; t < static_cast<int>(kMaxTermsPerPass); ++t) {
                if (t < static_cast<int>(p.n_terms)) {
                    const double si = parity_sign(i & p.zy[t]), sj = parity_sign(j & p.zy[t]);
                    v[2 * t] += (si + sj) * wr;
                    v[2 * t + 1] += (si - sj) * wi;
                }
            }
        }
    }
    block_sum_store<2 * kMaxTermsPerPass>(v, partials + blockIdx.x, gridDim.x);
}

__global__ void k_expect_combine(const double* __restrict__ sums, PExpect p,
                                 double* __restrict__ out) {
    const uint32_t t = threadIdx.x;
    if (t >= p.n_terms) return;
    const double re = sums[2 * t], im = sums[2 * t + 1];
    // Re(i^{n_y} (re + i im))
    double r;
    switch (p.n_y[t] & 3u) {
        case 0: r = re; break;
        case 1: r = -im; break;
        case 2: r = -re; break;
        default: r = im; break;
    }
    out[t] = r;
}

void launch_expect_xgroup(const LaunchCtx& ctx, const double2* st, uint32_t n, uint64_t x,
                          const uint64_t* zy, const uint32_t* n_y, uint32_t n_terms,
                          double* d_partials, double* d_out) {
    if (n_terms == 0 || n_terms > kMaxTermsPerPass)
        throw std::logic_error("launch_expect_xgroup: bad term count");
    PExpect p{};
    p.x = x;
    p.len = uint64_t{1} << n;
    p.n_terms = n_terms;
    for (uint32_t t = 0; t < n_terms; ++t) {
        p.zy[t] = zy[t];
        p.n_y[t] = n_y[t];
    }
    const uint32_t nb = reduce_grid(ctx, p.len);
    k_expect<<<nb, kReduceThreads, 0, ctx.stream>>>(st, p, d_partials);
    check_launch("expect");
    // reuse the tail of the partial buffer for the 2*kMaxTermsPerPass sums
    double* sums = d_partials + static_cast<uint64_t>(nb) * 2 * kMaxTermsPerPass;
    finalize<2 * kMaxTermsPerPass>(ctx, d_partials, nb, sums);
    k_expect_combine<<<1, 32, 0, ctx.stream>>>(sums, p, d_out);
    check_launch("expect_combine");
}

// ---------------------------------------------------------------- probabilities
// Statevector::probabilities (src/backend/statevector.cpp:33-37)
__global__ void k_probs(const double2* __restrict__ s, uint64_t len, double* __restrict__ p) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
         i += stride) {
        p[i] = norm_rn(__ldg(s + i));
    }
}

void launch_probabilities(const LaunchCtx& ctx, const double2* st, uint32_t n, double* d_p) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = static_cast<uint32_t>(std::min<uint64_t>(
        (len + kReduceThreads - 1) / kReduceThreads, static_cast<uint64_t>(ctx.num_sms) * 8));
    k_probs<<<std::max(1u, nb), kReduceThreads, 0, ctx.stream>>>(st, len, d_p);
    check_launch("probabilities");
}

// ---------------------------------------------------------------- prefix sum for sampling
// The reference forms the inclusive prefix sum of |a_i|^2 sequentially
// (std::partial_sum, src/backend/statevector_simulator.cpp:98-100).  Here each segment of
// kSegAmps amplitudes is summed sequentially per thread (kPerThread consecutive
// amplitudes), thread totals are combined by a sequential scan in fixed order, and the
// segment prefixes are added at the end.  The result differs from the sequential sum only
// in rounding; lqcs_state_sample reports how far each shot was from a bin edge.
//
// The prefix array itself is never stored: the scan keeps each thread chunk's exclusive
// prefix within its segment (tpref, one double per 16 amplitudes) and the segments'
// exclusive prefixes (block), and the search evaluates an element of the prefix array when
// its binary search probes it — re-adding at most 16 probabilities in the scan's own order,
// so every probed value is the one the full array would hold.
constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kPerThread = 16;
constexpr uint64_t kSegAmps = uint64_t{kScanThreads} * kPerThread;

uint64_t scan_block_count(uint32_t n) {
    const uint64_t len = uint64_t{1} << n;
    return (len + kSegAmps - 1) / kSegAmps;
}

uint64_t scan_thread_count(uint32_t n) { return scan_block_count(n) * kScanThreads; }

// Probability sources of the scan: |a_i|^2 of a statevector, or the diagonal rho_ii of a
// density matrix stored as a 2n-qubit vector (element (col << n) | row).
struct AmpSource {
    const double2* s;
    __device__ double operator()(uint64_t i) const { return norm_rn(__ldg(s + i)); }
};
struct DiagSource {
    const double2* rho;
    uint32_t n;
    __device__ double operator()(uint64_t i) const { return __ldg(rho + ((i << n) | i)).x; }
};

template <class Src>
__global__ void __launch_bounds__(kScanThreads) k_scan_seg(Src src, uint64_t len,
                                                           double* __restrict__ tpref_out,
                                                           double* __restrict__ seg_total) {
    __shared__ double tsum[kScanThreads];
    // the segment's probabilities, read coalesced; element e at e + e / kPerThread (one pad
    // slot per chunk, so the chunk-wise reads below hit distinct banks)
    __shared__ double sp[kSegAmps + kSegAmps / kPerThread];
    const uint64_t seg0 = static_cast<uint64_t>(blockIdx.x) * kSegAmps;
#pragma unroll
    for (uint32_t k = 0; k < kPerThread; ++k) {
        const uint32_t e = k * kScanThreads + threadIdx.x;
        const uint64_t i = seg0 + e;
        sp[e + e / kPerThread] = (i < len) ? src(i) : 0.0;
    }
    __syncthreads();
    double acc = 0.0;
#pragma unroll
    for (uint32_t k = 0; k < kPerThread; ++k) {
        const double p = sp[threadIdx.x * (kPerThread + 1) + k];
        acc = (k == 0) ? p : __dadd_rn(acc, p);
    }
    tsum[threadIdx.x] = acc;
    __syncthreads();
    // exclusive prefix of the thread totals, sequential in thread order
    if (threadIdx.x == 0) {
        double run = 0.0;
        double* tp = tpref_out + static_cast<uint64_t>(blockIdx.x) * kScanThreads;
        for (uint32_t t = 0; t < kScanThreads; ++t) {
            tp[t] = run;
            run = __dadd_rn(run, tsum[t]);
        }
        seg_total[blockIdx.x] = run;
    }
}

// Exclusive scan of the segment totals in place (one block, sequential per thread chunk).
__global__ void __launch_bounds__(1024) k_scan_top(double* __restrict__ seg, uint64_t nseg) {
    __shared__ double tsum[1024];
    const uint64_t per = (nseg + blockDim.x - 1) / blockDim.x;
    const uint64_t b0 = static_cast<uint64_t>(threadIdx.x) * per;
    double acc = 0.0;
    for (uint64_t k = 0; k < per; ++k) {
        const uint64_t b = b0 + k;
        if (b < nseg) acc = __dadd_rn(acc, seg[b]);
    }
    tsum[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double run = 0.0;
        for (uint32_t t = 0; t < blockDim.x; ++t) {
            const double v = tsum[t];
            tsum[t] = run;
            run = __dadd_rn(run, v);
        }
    }
    __syncthreads();
    double run = tsum[threadIdx.x];
    for (uint64_t k = 0; k < per; ++k) {
        const uint64_t b = b0 + k;
        if (b < nseg) {
            const double v = seg[b];
            seg[b] = run;
            run = __dadd_rn(run, v);
        }
    }
}

template <class Src>
void prob_scan(const LaunchCtx& ctx, Src src, uint32_t n, double* d_tpref, double* d_block) {
    const uint64_t len = uint64_t{1} << n;
    const uint64_t nseg = scan_block_count(n);
    k_scan_seg<Src><<<static_cast<uint32_t>(nseg), kScanThreads, 0, ctx.stream>>>(src, len, d_tpref,
                                                                                  d_block);
    check_launch("scan_seg");
    if (nseg > 1) {
        k_scan_top<<<1, 1024, 0, ctx.stream>>>(d_block, nseg);
        check_launch("scan_top");
    }
}

void launch_prob_scan(const LaunchCtx& ctx, const double2* st, uint32_t n, double* d_tpref,
                      double* d_block) {
    prob_scan(ctx, AmpSource{st}, n, d_tpref, d_block);
}

void launch_dm_diag_scan(const LaunchCtx& ctx, const double2* rho, uint32_t n, double* d_tpref,
                         double* d_block) {
    prob_scan(ctx, DiagSource{rho, n}, n, d_tpref, d_block);
}

__global__ void k_dm_diag(const double2* __restrict__ rho, uint32_t n, double* __restrict__ p) {
    const uint64_t len = uint64_t{1} << n;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
         i += stride)
        p[i] = __ldg(rho + ((i << n) | i)).x;
}

void launch_dm_diagonal(const LaunchCtx& ctx, const double2* rho, uint32_t n, double* d_p) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = static_cast<uint32_t>(std::min<uint64_t>(
        (len + 255) / 256, static_cast<uint64_t>(ctx.num_sms) * 8));
    k_dm_diag<<<std::max(1u, nb), 256, 0, ctx.stream>>>(rho, n, d_p);
    check_launch("dm_diag");
}

// Element j of the inclusive prefix array, evaluated as the scan would have stored it:
// the thread chunk's running sum up to j, plus the chunk's prefix in its segment (not for
// the first chunk), plus the segment's prefix (not for the first segment, and only when
// there is more than one).
template <class Src>
__device__ double cum_at(const Src& src, uint64_t j, const double* __restrict__ tpref,
                         const double* __restrict__ seg_prefix, uint64_t nseg) {
    const uint64_t b = j / kSegAmps;
    const uint32_t t = static_cast<uint32_t>((j % kSegAmps) / kPerThread);
    const uint64_t i0 = b * kSegAmps + static_cast<uint64_t>(t) * kPerThread;
    double local = src(i0);
    for (uint64_t i = i0 + 1; i <= j; ++i) local = __dadd_rn(local, src(i));
    const double c = (t == 0) ? local : __dadd_rn(tpref[b * kScanThreads + t], local);
    return (b > 0 && nseg > 1) ? __dadd_rn(seg_prefix[b], c) : c;
}

// std::upper_bound(cum, cum + N, u * total) for every shot
// (src/backend/statevector_simulator.cpp:105-109), probing cum through cum_at.
template <class Src>
__global__ void k_sample_search(Src src, uint64_t len, const double* __restrict__ tpref,
                                const double* __restrict__ seg_prefix, uint64_t nseg,
                                const double* __restrict__ u, uint64_t shots,
                                uint64_t* __restrict__ idx, double* __restrict__ margin) {
    const uint64_t s = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= shots) return;
    const double total = cum_at(src, len - 1, tpref, seg_prefix, nseg);
    const double r = u[s] * total;
    uint64_t lo = 0, count = len;
    while (count > 0) {
        const uint64_t half = count >> 1;
        if (!(r < cum_at(src, lo + half, tpref, seg_prefix, nseg))) {
            lo = lo + half + 1;
            count = count - half - 1;
        } else {
            count = half;
        }
    }
    idx[s] = lo;
    if (margin) {
        const double below = (lo > 0) ? cum_at(src, lo - 1, tpref, seg_prefix, nseg) : 0.0;
        const double above = (lo < len) ? cum_at(src, lo, tpref, seg_prefix, nseg) : total;
        margin[s] = fmin(r - below, above - r) / total;
    }
}

template <class Src>
void sample_search(const LaunchCtx& ctx, Src src, uint32_t n, const double* d_tpref,
                   const double* d_block, const double* d_u, uint64_t shots, uint64_t* d_idx,
                   double* d_margin) {
    if (shots == 0) return;
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = static_cast<uint32_t>((shots + 127) / 128);
    k_sample_search<Src><<<nb, 128, 0, ctx.stream>>>(src, len, d_tpref, d_block,
                                                     scan_block_count(n), d_u, shots, d_idx,
                                                     d_margin);
    check_launch("sample_search");
}

void launch_sample_search(const LaunchCtx& ctx, const double2* st, uint32_t n,
                          const double* d_tpref, const double* d_block, const double* d_u,
                          uint64_t shots, uint64_t* d_idx, double* d_margin) {
    sample_search(ctx, AmpSource{st}, n, d_tpref, d_block, d_u, shots, d_idx, d_margin);
}

void launch_dm_sample_search(const LaunchCtx& ctx, const double2* rho, uint32_t n,
                             const double* d_tpref, const double* d_block, const double* d_u,
                             uint64_t shots, uint64_t* d_idx, double* d_margin) {
    sample_search(ctx, DiagSource{rho, n}, n, d_tpref, d_block, d_u, shots, d_idx, d_margin);
}

// ---------------------------------------------------------------- projection
// second loop of kernels::collapse_qubit (src/backend/kernels/gate_kernels.cpp:236-246)
__global__ void k_project(double2* __restrict__ s, uint64_t len, uint32_t q, int outcome,
                          double scale) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
         i += stride) {
        if (static_cast<int>((i >> q) & 1u) == outcome) {
            const double2 a = s[i];
            s[i] = make_double2(a.x * scale, a.y * scale);
        } else {
            s[i] = make_double2(0.0, 0.0);
        }
    }
}

void launch_project(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t q, int outcome,
                    double scale) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = static_cast<uint32_t>(std::min<uint64_t>(
        (len + 255) / 256, static_cast<uint64_t>(ctx.num_sms) * 8));
    k_project<<<std::max(1u, nb), 256, 0, ctx.stream>>>(st, len, q, outcome, scale);
    check_launch("project");
}

// tail of kernels::reset_qubit (src/backend/kernels/gate_kernels.cpp:253-259)
__global__ void k_move_to_zero(double2* __restrict__ s, uint64_t half, uint32_t q) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t qb = uint64_t{1} << q;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < half;
         g += stride) {
        const uint64_t i0 = insert_zero_bit(g, q);
        s[i0] = s[i0 | qb];
        s[i0 | qb] = make_double2(0.0, 0.0);
    }
}

void launch_move_to_zero(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t q) {
    const uint64_t half = (uint64_t{1} << n) >> 1;
    const uint32_t nb = static_cast<uint32_t>(std::min<uint64_t>(
        (half + 255) / 256, static_cast<uint64_t>(ctx.num_sms) * 8));
    k_move_to_zero<<<std::max(1u, nb), 256, 0, ctx.stream>>>(st, half, q);
    check_launch("move_to_zero");
}

// ---------------------------------------------------------------- Hamiltonian apply
// (H psi)[i] = sum_t c_t i^{n_y,t} (-1)^{popcount((i ^ x_t) & zy_t)} psi[i ^ x_t]
// (the action of P on a basis state, src/backend/statevector.cpp:52-53).
//
// Tiled over the state: a CTA owns one output tile of 2^ml amplitudes (its index bits above
// ml fixed), and the terms come sorted by the bits of x above ml in groups: groups[0] = G,
// then G group keys g (x >> ml), then G + 1 term offsets.  For each group the CTA stages the
// one source tile all its terms read (output tile ^ g) in shared memory and gathers from
// there, so a source amplitude crosses L2 once per output tile and group instead of once per
// term.
uint32_t ham_tile_bits(uint32_t n) { return std::min<uint32_t>(n, 11); }

template <int PER>
__global__ void __launch_bounds__(256) k_apply_ham(const double2* __restrict__ in,
                                                   double2* __restrict__ out, uint32_t n,
                                                   uint32_t ml,
                                                   const PauliTermDev* __restrict__ terms,
                                                   const uint32_t* __restrict__ groups) {
    extern __shared__ double2 src_tile[];
    const uint64_t len = uint64_t{1} << n;
    const uint32_t T = 1u << ml;
    const double2* src = in + static_cast<uint64_t>(blockIdx.y) * len;
    double2* dst = out + static_cast<uint64_t>(blockIdx.y) * len;
    const uint64_t out_hi = blockIdx.x;
    const uint32_t n_groups = __ldg(groups);
    const uint32_t* keys = groups + 1;
    const uint32_t* offs = keys + n_groups;
    double2 acc[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) acc[j] = make_double2(0.0, 0.0);
    for (uint32_t k = 0; k < n_groups; ++k) {
        const uint64_t g = __ldg(keys + k);
        const uint32_t t0 = __ldg(offs + k), t1 = __ldg(offs + k + 1);
        __syncthreads();          // the previous group's gathers are done
        const double2* row = src + ((out_hi ^ g) << ml);
        for (uint32_t l = threadIdx.x; l < T; l += blockDim.x) src_tile[l] = __ldcg(row + l);
        __syncthreads();
        for (uint32_t t = t0; t < t1; ++t) {
            const uint64_t x = __ldg(&terms[t].x), zy = __ldg(&terms[t].zy);
            const double2 c = __ldg(&terms[t].coeff);
            const uint32_t xl = static_cast<uint32_t>(x) & (T - 1u);
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                const uint32_t l = threadIdx.x + j * blockDim.x;
                const uint64_t jj = ((out_hi << ml) | l) ^ x;
                const double sg = (__popcll(jj & zy) & 1) ? -1.0 : 1.0;
                acc[j] = cmad(make_double2(sg * c.x, sg * c.y), src_tile[l ^ xl], acc[j]);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < PER; ++j) dst[(out_hi << ml) | (threadIdx.x + j * blockDim.x)] = acc[j];
}

void launch_apply_hamiltonian(const LaunchCtx& ctx, const double2* in, double2* out,
                              uint32_t n, uint32_t batch, const PauliTermDev* d_terms,
                              const uint32_t* d_groups) {
    const uint32_t ml = ham_tile_bits(n);
    const uint32_t T = 1u << ml;
    const uint32_t threads = std::min<uint32_t>(256, T);
    const uint32_t per = T / threads;
    const dim3 grid(1u << (n - ml), batch);
    const size_t smem = sizeof(double2) * T;
    switch (per) {
        case 1: k_apply_ham<1><<<grid, threads, smem, ctx.stream>>>(in, out, n, ml, d_terms, d_groups); break;
        case 2: k_apply_ham<2><<<grid, threads, smem, ctx.stream>>>(in, out, n, ml, d_terms, d_groups); break;
        case 4: k_apply_ham<4><<<grid, threads, smem, ctx.stream>>>(in, out, n, ml, d_terms, d_groups); break;
        default: k_apply_ham<8><<<grid, threads, smem, ctx.stream>>>(in, out, n, ml, d_terms, d_groups); break;
    }
    check_launch("apply_hamiltonian");
}

// ---------------------------------------------------------------- batched inner products
// Re<a_b|b_b> per state b: one block row per state, partials then a per-state final sum.
__global__ void __launch_bounds__(kReduceThreads) k_inner_re(const double2* __restrict__ a,
                                                             const double2* __restrict__ b,
                                                             uint64_t len, double* partials) {
    const double2* pa = a + static_cast<uint64_t>(blockIdx.y) * len;
    const double2* pb = b + static_cast<uint64_t>(blockIdx.y) * len;
    double v[1] = {0.0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
         i += stride) {
        const double2 x = __ldg(pa + i), y = __ldg(pb + i);
        v[0] += x.x * y.x + x.y * y.y;
    }
    block_sum_store<1>(v, partials + static_cast<uint64_t>(blockIdx.y) * gridDim.x + blockIdx.x,
                       1);
}

// Im<a|P|b> = Im sum_i conj(a_i) i^{n_y} (-1)^{popcount((i^x) & zy)} b_{i^x}
__global__ void __launch_bounds__(kReduceThreads) k_pauli_im(const double2* __restrict__ a,
                                                             const double2* __restrict__ b,
                                                             uint64_t len, uint64_t x,
                                                             uint64_t zy, uint32_t n_y,
                                                             double* partials) {
    const double2* pa = a + static_cast<uint64_t>(blockIdx.y) * len;
    const double2* pb = b + static_cast<uint64_t>(blockIdx.y) * len;
    double v[2] = {0.0, 0.0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
         i += stride) {
        const uint64_t j = i ^ x;
        const double2 u = __ldg(pa + i), w = __ldg(pb + j);
        const double sg = parity_sign(j & zy);
        // conj(u) * w * sg
        v[0] += sg * (u.x * w.x + u.y * w.y);
        v[1] += sg * (u.x * w.y - u.y * w.x);
    }
    // multiply by i^{n_y} and keep the imaginary part
    double im;
    switch (n_y & 3u) {
        case 0: im = v[1]; break;
        case 1: im = v[0]; break;
        case 2: im = -v[1]; break;
        default: im = -v[0]; break;
    }
    double w1[1] = {im};
    block_sum_store<1>(w1, partials + static_cast<uint64_t>(blockIdx.y) * gridDim.x + blockIdx.x,
                       1);
}

__global__ void __launch_bounds__(kReduceThreads) k_rows_final(const double* __restrict__ partials,
                                                               uint32_t nb, double* __restrict__ out,
                                                               uint64_t out_stride) {
    const double* row = partials + static_cast<uint64_t>(blockIdx.x) * nb;
    double v[1] = {0.0};
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) v[0] += row[b];
    __shared__ double res[1];
    block_sum_store<1>(v, res, 1);
    __syncthreads();
    if (threadIdx.x == 0) out[static_cast<uint64_t>(blockIdx.x) * out_stride] = res[0];
}

static uint32_t per_state_blocks(const LaunchCtx& ctx, uint64_t len, uint32_t batch) {
    const uint64_t want = (len + kReduceThreads - 1) / kReduceThreads;
    const uint64_t cap = std::max<uint64_t>(1, static_cast<uint64_t>(ctx.num_sms) * 8 /
                                                   std::max(1u, batch));
    return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>({want, cap, 64})));
}

void launch_batched_inner_re_p(const LaunchCtx& ctx, const double2* a, const double2* b,
                               uint32_t n, uint32_t batch, double* d_partials, double* d_out) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = per_state_blocks(ctx, len, batch);
    k_inner_re<<<dim3(nb, batch), kReduceThreads, 0, ctx.stream>>>(a, b, len, d_partials);
    check_launch("inner_re");
    k_rows_final<<<batch, kReduceThreads, 0, ctx.stream>>>(d_partials, nb, d_out, 1);
    check_launch("rows_final");
}

void launch_batched_pauli_im_p(const LaunchCtx& ctx, const double2* a, const double2* b,
                               uint32_t n, uint32_t batch, uint64_t x, uint64_t zy,
                               uint32_t n_y, double* d_partials, double* d_out,
                               uint64_t out_stride) {
    const uint64_t len = uint64_t{1} << n;
    const uint32_t nb = per_state_blocks(ctx, len, batch);
    k_pauli_im<<<dim3(nb, batch), kReduceThreads, 0, ctx.stream>>>(a, b, len, x, zy, n_y,
                                                                   d_partials);
    check_launch("pauli_im");
    k_rows_final<<<batch, kReduceThreads, 0, ctx.stream>>>(d_partials, nb, d_out, out_stride);
    check_launch("rows_final");
}

}  // namespace lqcs_b200
