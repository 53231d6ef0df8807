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

constexpr int kMmaThreads = 512;   // 16 warps
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

// X (the gathered groups) in shared memory as double2 [member][group], row stride kXStride
// double2: a B fragment (real row 4 ks + lane % 4 = member, re / im; column = group) reads
// two rows of 16 consecutive doubles, one wavefront each.  Two buffers: the next tile's
// groups arrive by cp.async while this tile computes.
constexpr int kXStride = kMmaGroups + 4;

template <int K>
constexpr size_t mma_smem_bytes() {
    return sizeof(double2) * 2 * static_cast<size_t>(1 << K) * kXStride;
}

__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Element (row, col) of the real embedding of the complex matrix m (D x D).
template <int D>
__device__ __forceinline__ double embedded(const double2* __restrict__ m, int row, int col) {
    const double2 z = __ldg(m + (row >> 1) * D + (col >> 1));
    const int a = row & 1, b = col & 1;
    return a == b ? z.x : (a == 0 ? -z.y : z.y);
}

// 16-byte asynchronous copy global -> shared; src_bytes = 0 writes zeros.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src, uint32_t src_bytes) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gmem_src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Work split of the R/8 m-tiles and the 8 n-tiles (of 8 groups) over the 16 warps: each warp
// keeps the A fragments of its m-tile in registers for the whole launch (the matrix is the
// same for every tile) and reads the B fragments of its NPW n-tiles from shared memory.
template <int K>
struct MmaSplit {
    static constexpr int R = 2 << K;
    static constexpr int MT = R / 8;                          // m-tiles (<= warps)
    static constexpr int WARPS = kMmaThreads / 32;
    static constexpr int NSPLIT = WARPS / MT;                 // warps sharing an m-tile
    static constexpr int NPW = 8 / NSPLIT;                    // n-tiles per warp
    static constexpr int KS = R / 4;                          // k-steps
    static_assert(MT <= WARPS && WARPS % MT == 0 && 8 % NSPLIT == 0, "m-tile split");
};

// A thread's group within a tile (g = tid % 64) and members l = tid / 64 + 8 r: one group
// base per tile, computed by the thread itself.
template <int K>
__device__ __forceinline__ uint64_t group_base(uint64_t g, const PDenseMma<K>& p) {
    for (uint32_t i = 0; i < p.n_fixed; ++i) g = insert_zero_bit(g, p.fixed[i]);
    return g | p.cmask;
}

template <int K>
__global__ void __launch_bounds__(kMmaThreads, 1) k_dense_mma(double2* __restrict__ st, PDenseMma<K> p) {
    using S = MmaSplit<K>;
    constexpr int D = 1 << K;
    constexpr int MPT = D * kMmaGroups / kMmaThreads;         // members per thread
    extern __shared__ __align__(16) double2 xs[];             // 2 buffers of D x kXStride
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = warp % S::MT, nset = warp / S::MT;
    const int g_t = threadIdx.x % kMmaGroups, l_t = threadIdx.x / kMmaGroups;
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    const uint64_t n_tiles = (p.n_groups + kMmaGroups - 1) / kMmaGroups;

    auto gather = [&](uint64_t tile, int buf) {
        const uint64_t g = tile * kMmaGroups + g_t;
        const bool ok = g < p.n_groups;
        const uint64_t base = ok ? group_base<K>(g, p) : 0;
        double2* x = xs + buf * D * kXStride;
#pragma unroll
        for (int r = 0; r < MPT; ++r) {
            const int l = l_t + r * (kMmaThreads / kMmaGroups);
            cp_async16(x + l * kXStride + g_t, ok ? s + (base | p.off[l]) : s, ok ? 16u : 0u);
        }
    };

    if (blockIdx.x < n_tiles) gather(blockIdx.x, 0);
    cp_async_commit();
    // A fragments: row 8 mt + lane / 4, column 4 ks + lane % 4 of the embedded matrix
    double af[S::KS];
#pragma unroll
    for (int ks = 0; ks < S::KS; ++ks) af[ks] = embedded<D>(p.mat, 8 * mt + (lane >> 2), 4 * ks + (lane & 3));

    int buf = 0;
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, buf ^= 1) {
        if (tile + gridDim.x < n_tiles) gather(tile + gridDim.x, buf ^ 1);
        cp_async_commit();
        cp_async_wait_prev();   // this tile's copies (all but the newest group) have landed
        __syncthreads();
        double2* x = xs + buf * D * kXStride;
        const double* xd = reinterpret_cast<const double*>(x);
        double acc[S::NPW][2];
#pragma unroll
        for (int j = 0; j < S::NPW; ++j) acc[j][0] = acc[j][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < S::KS; ++ks) {
            const int k = 4 * ks + (lane & 3);   // real row: member k / 2, re / im k % 2
#pragma unroll
            for (int j = 0; j < S::NPW; ++j) {
                const int n = 8 * (nset * S::NPW + j) + (lane >> 2);
                mma_f64(acc[j], af[ks], xd[((k >> 1) * kXStride + n) * 2 + (k & 1)]);
            }
        }
        __syncthreads();   // every warp has read X: the results may overwrite it
        {
            double* xo = reinterpret_cast<double*>(x);
            const int k = 8 * mt + (lane >> 2);
#pragma unroll
            for (int j = 0; j < S::NPW; ++j) {
                const int n = 8 * (nset * S::NPW + j) + 2 * (lane & 3);
                xo[((k >> 1) * kXStride + n) * 2 + (k & 1)] = acc[j][0];
                xo[((k >> 1) * kXStride + n + 1) * 2 + (k & 1)] = acc[j][1];
            }
        }
        __syncthreads();
        {
            const uint64_t g = tile * kMmaGroups + g_t;
            if (g < p.n_groups) {
                const uint64_t base = group_base<K>(g, p);
#pragma unroll
                for (int r = 0; r < MPT; ++r) {
                    const int l = l_t + r * (kMmaThreads / kMmaGroups);
                    __stcs(s + (base | p.off[l]), x[l * kXStride + g_t]);
                }
            }
        }
        __syncthreads();   // the store has read this buffer: the gather after next may refill it
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
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
    const uint64_t want = static_cast<uint64_t>(ctx.num_sms);   // one 16-warp CTA per SM
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
