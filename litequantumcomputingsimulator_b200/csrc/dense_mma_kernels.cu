// dense_mma_kernels.cu — dense k-qubit blocks (k = 4..6) on the FP64 tensor path.
//
// A fused block is a 2^k x 2^k complex matrix M applied to every group of 2^k amplitudes
// whose non-target bits agree (controls all 1).  Over the reals it is a GEMM:
//     Y (R x G) = Mr (R x R) * X (R x G),   R = 2^(k+1),
// with X the groups' amplitudes as interleaved (re, im) rows — exactly the double2 layout
// of the state — and Mr the real embedding of M: Mr[2r+a][2c+b] = Re M[r][c] for a = b,
// -Im M[r][c] for (a, b) = (0, 1), Im M[r][c] for (1, 0).  A CTA gathers 64 groups into
// shared memory, each warp computes 8 groups (one n-tile) of all R output rows with
// mma.sync.m8n8k4.f64 (the FP64 tensor instruction of sm_100a; tcgen05 has no FP64 kind),
// and the results go back through shared memory to coalesced stores.
//
// Semantics: kernels::apply_matrix (src/backend/kernels/gate_kernels.cpp) for a k-qubit
// unitary with controls, as the FFMA kernel k_dense<K> (gate_kernels.cu).
#include <algorithm>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "kernels.cuh"

namespace lqcs_b200 {

namespace {

constexpr int kMmaThreads = 256;   // 8 warps
constexpr int kMmaGroups = 64;     // groups per CTA tile: one n-tile of 8 per warp

void check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA launch failed in ") + what + ": " +
                                 cudaGetErrorString(e));
    }
    count_launch();
}

template <int K>
struct PDenseMma {
    uint64_t off[1 << K];   // member l -> address offset (bit j of l <-> targets[j])
    uint64_t cmask;
    uint64_t n_groups;
    uint64_t batch_stride;
    const double2* mat;
    uint32_t n_fixed;
    uint32_t fixed[kMaxQubits];   // sorted controls and targets
};

// Row strides (in doubles) of the shared operands: = 4 (mod 16), so the 16 lanes of a
// half-warp reading an 8-byte fragment element (row = lane % 4 or lane / 4, column = the
// other) fall on 16 different 8-byte bank pairs.
template <int K> __host__ __device__ constexpr int mat_stride() { return (2 << K) + 4; }
constexpr int kXStride = kMmaGroups + 4;

template <int K>
constexpr size_t mma_smem_bytes() {
    return sizeof(double) * (static_cast<size_t>(2 << K) * mat_stride<K>() +
                             static_cast<size_t>(2 << K) * kXStride) +
           sizeof(uint64_t) * ((1u << K) + kMaxQubits + kMmaGroups);
}

__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

template <int K>
__global__ void __launch_bounds__(kMmaThreads) k_dense_mma(double2* __restrict__ st, PDenseMma<K> p) {
    constexpr int D = 1 << K;
    constexpr int R = 2 * D;          // real rows / columns of the embedded matrix
    constexpr int MT = R / 8;         // m-tiles
    constexpr int SM = mat_stride<K>();
    extern __shared__ __align__(16) double smd[];
    double* Ms = smd;                         // R x SM
    double* Xs = Ms + R * SM;                 // R x kXStride, then the results
    uint64_t* soff = reinterpret_cast<uint64_t*>(Xs + R * kXStride);
    uint64_t* sfix = soff + D;
    uint64_t* sbase = sfix + kMaxQubits;      // this tile's group bases
    for (int i = threadIdx.x; i < D * D; i += kMmaThreads) {
        const int r = i / D, c = i % D;
        const double2 m = p.mat[i];
        Ms[(2 * r) * SM + 2 * c] = m.x;
        Ms[(2 * r) * SM + 2 * c + 1] = -m.y;
        Ms[(2 * r + 1) * SM + 2 * c] = m.y;
        Ms[(2 * r + 1) * SM + 2 * c + 1] = m.x;
    }
    for (int i = threadIdx.x; i < D; i += kMmaThreads) soff[i] = p.off[i];
    for (uint32_t i = threadIdx.x; i < p.n_fixed; i += kMmaThreads) sfix[i] = p.fixed[i];
    __syncthreads();
    const uint32_t nf = p.n_fixed;
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t n_tiles = (p.n_groups + kMmaGroups - 1) / kMmaGroups;
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const uint64_t g0 = tile * kMmaGroups;
        if (threadIdx.x < kMmaGroups) {
            uint64_t g = g0 + threadIdx.x;
            for (uint32_t i = 0; i < nf; ++i) g = insert_zero_bit(g, static_cast<unsigned>(sfix[i]));
            sbase[threadIdx.x] = g | p.cmask;
        }
        __syncthreads();
        // gather: consecutive threads take consecutive groups of one member
        for (int i = threadIdx.x; i < kMmaGroups * D; i += kMmaThreads) {
            const int g = i % kMmaGroups, l = i / kMmaGroups;
            double2 a = make_double2(0.0, 0.0);
            if (g0 + g < p.n_groups) a = __ldcs(s + (sbase[g] | soff[l]));
            Xs[(2 * l) * kXStride + g] = a.x;
            Xs[(2 * l + 1) * kXStride + g] = a.y;
        }
        __syncthreads();
        double acc[MT][2];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
        const int ncol = 8 * warp + (lane >> 2);
#pragma unroll 2
        for (int kk = 0; kk < R; kk += 4) {
            const double b = Xs[(kk + (lane & 3)) * kXStride + ncol];
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
                mma_f64(acc[mt], Ms[(8 * mt + (lane >> 2)) * SM + kk + (lane & 3)], b);
        }
        __syncthreads();   // every warp has read X: the results may overwrite it
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            double* row = Xs + (8 * mt + (lane >> 2)) * kXStride + 8 * warp + 2 * (lane & 3);
            row[0] = acc[mt][0];
            row[1] = acc[mt][1];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kMmaGroups * D; i += kMmaThreads) {
            const int g = i % kMmaGroups, l = i / kMmaGroups;
            if (g0 + g < p.n_groups)
                __stcs(s + (sbase[g] | soff[l]),
                       make_double2(Xs[(2 * l) * kXStride + g], Xs[(2 * l + 1) * kXStride + g]));
        }
        __syncthreads();
    }
}

template <int K>
void mma_impl(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
              const uint32_t* targets, uint64_t cmask, const double2* d_mat) {
    PDenseMma<K> p{};
    uint64_t fixmask = cmask;
    for (int j = 0; j < K; ++j) fixmask |= uint64_t{1} << targets[j];
    for (int l = 0; l < (1 << K); ++l) {
        uint64_t o = 0;
        for (int j = 0; j < K; ++j)
            if ((l >> j) & 1) o |= uint64_t{1} << targets[j];
        p.off[l] = o;
    }
    for (uint32_t b = 0; b < 64; ++b)
        if ((fixmask >> b) & 1) p.fixed[p.n_fixed++] = b;
    p.cmask = cmask;
    p.n_groups = (uint64_t{1} << n) >> p.n_fixed;
    p.batch_stride = uint64_t{1} << n;
    p.mat = d_mat;
    constexpr size_t smem = mma_smem_bytes<K>();
    const cudaError_t e = cudaFuncSetAttribute(k_dense_mma<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(smem));
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    const uint64_t tiles = (p.n_groups + kMmaGroups - 1) / kMmaGroups;
    const uint32_t per_sm = static_cast<uint32_t>(std::max<size_t>(1, (227 * 1024) / (smem + 1024)));
    const uint64_t want = static_cast<uint64_t>(ctx.num_sms) * std::min<uint32_t>(per_sm, 4);
    const uint32_t grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(want, tiles)));
    k_dense_mma<K><<<dim3(grid, batch), kMmaThreads, smem, ctx.stream>>>(st, p);
    check_launch("dense_mma");
}

}  // namespace

// Default: 6-qubit blocks only, where the tensor path measured faster than FFMA (4.49 s vs
// 6.65 s on the 30-qubit brickwork fused to width 6; 4- and 5-qubit blocks were faster on
// FFMA).  LQCS_DENSE_MMA=1 takes every 4..6-qubit block to the tensor path, =0 none.
bool dense_mma_enabled(uint32_t k) {
    if (k < 4 || k > 6) return false;
    const char* e = std::getenv("LQCS_DENSE_MMA");   // read per launch: cheap next to one pass
    if (e && e[0] == '0') return false;
    if (e && e[0] == '1') return true;
    return k == 6;
}

void launch_dense_mma(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                      const uint32_t* targets, uint32_t k, uint64_t cmask, const double2* d_mat) {
    switch (k) {
        case 4: mma_impl<4>(ctx, st, n, batch, targets, cmask, d_mat); break;
        case 5: mma_impl<5>(ctx, st, n, batch, targets, cmask, d_mat); break;
        case 6: mma_impl<6>(ctx, st, n, batch, targets, cmask, d_mat); break;
        default: throw std::logic_error("launch_dense_mma: k must be 4..6");
    }
}

}  // namespace lqcs_b200
