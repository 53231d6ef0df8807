// tile_kernels.cu — multi-gate passes through shared memory.
//
// One launch applies a whole list of operations to the state in a single HBM read and
// write.  The state is cut into tiles of 2^M amplitudes: a tile holds every amplitude whose
// bits outside the tile-bit set {0..L-1} u H are fixed, H being up to M-L chosen high
// qubits.  A CTA copies a tile into shared memory (2^|H| runs of 2^L contiguous
// amplitudes, each run a coalesced stretch of at least 512 bytes), applies the operation
// list to it with a barrier between operations, and writes it back.  An operation may act
// only on tile bits through its targets; its controls (and the bits of a phase) may lie
// outside the tile, where they are constant for the whole tile and become a per-tile
// predicate.  Reference semantics of each operation: src/backend/kernels/gate_kernels.cpp.
//
// The pass's operation records are staged in shared memory once per CTA.  Slot arithmetic
// is XOR-only (see TileOp): per operation a thread spreads its index over the free bit
// positions once; each group then costs one XOR for its base and one per member.
#include <algorithm>
#include <stdexcept>
#include <string>

#include "kernels.cuh"
#include "tile.cuh"

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

__device__ __forceinline__ uint32_t insert0(uint32_t v, uint32_t pos) {
    const uint32_t low = (1u << pos) - 1u;
    return ((v & ~low) << 1) | (v & low);
}

// sw(deposit(t)) for this thread and operation.
__device__ __forceinline__ uint32_t thread_slot(const TileOp& op) {
    uint32_t v = threadIdx.x;
    const uint32_t nf = op.n_fixed;
    for (uint32_t i = 0; i < nf; ++i) v = insert0(v, op.fixed[i]);
    return tile_swizzle(v);
}

__device__ __forceinline__ void op_dense1(double2* __restrict__ t, const TileOp& op,
                                          const double2* __restrict__ mat) {
    if (threadIdx.x >= op.n_groups) return;
    const double2 m0 = __ldg(mat), m1 = __ldg(mat + 1), m2 = __ldg(mat + 2), m3 = __ldg(mat + 3);
    const uint32_t ts = thread_slot(op), o1 = op.soff[1];
    const uint32_t iters = op.iters;
    for (uint32_t j = 0; j < iters; ++j) {
        const uint32_t p0 = ts ^ op.dhi[j], p1 = p0 ^ o1;
        const double2 a0 = t[p0], a1 = t[p1];
        t[p0] = cmad(m1, a1, cmul(m0, a0));
        t[p1] = cmad(m3, a1, cmul(m2, a0));
    }
}

__device__ __forceinline__ void op_dense2(double2* __restrict__ t, const TileOp& op,
                                          const double2* __restrict__ mat) {
    if (threadIdx.x >= op.n_groups) return;
    double2 mm[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) mm[i] = __ldg(mat + i);
    const uint32_t ts = thread_slot(op);
    const uint32_t o1 = op.soff[1], o2 = op.soff[2], o3 = op.soff[3];
    const uint32_t iters = op.iters;
    for (uint32_t j = 0; j < iters; ++j) {
        const uint32_t p0 = ts ^ op.dhi[j];
        const uint32_t p1 = p0 ^ o1, p2 = p0 ^ o2, p3 = p0 ^ o3;
        const double2 a0 = t[p0], a1 = t[p1], a2 = t[p2], a3 = t[p3];
        double2 y[4];
#pragma unroll
        for (int row = 0; row < 4; ++row) {
            double2 acc = cmul(mm[4 * row], a0);
            acc = cmad(mm[4 * row + 1], a1, acc);
            acc = cmad(mm[4 * row + 2], a2, acc);
            y[row] = cmad(mm[4 * row + 3], a3, acc);
        }
        t[p0] = y[0];
        t[p1] = y[1];
        t[p2] = y[2];
        t[p3] = y[3];
    }
}

template <int K>
__device__ __forceinline__ void op_dense_wide(double2* __restrict__ t, const TileOp& op,
                                              const double2* __restrict__ mat) {
    constexpr int D = 1 << K;
    if (threadIdx.x >= op.n_groups) return;
    uint32_t off[D];
#pragma unroll
    for (int l = 0; l < D; ++l) off[l] = op.soff[l];
    const uint32_t ts = thread_slot(op);
    const uint32_t iters = op.iters;
    for (uint32_t j = 0; j < iters; ++j) {
        const uint32_t b = ts ^ op.dhi[j];
        double2 a[D];
#pragma unroll
        for (int l = 0; l < D; ++l) a[l] = t[b ^ off[l]];
#pragma unroll 1
        for (int row = 0; row < D; ++row) {
            double2 acc = cmul(__ldg(mat + row * D), a[0]);
#pragma unroll
            for (int c = 1; c < D; ++c) acc = cmad(__ldg(mat + row * D + c), a[c], acc);
            t[b ^ off[row]] = acc;
        }
    }
}

template <int K>
__device__ __forceinline__ void op_diag(double2* __restrict__ t, const TileOp& op,
                                        const double2* __restrict__ dg) {
    constexpr int D = 1 << K;
    if (threadIdx.x >= op.n_groups) return;
    double2 d[D];
    uint32_t off[D];
#pragma unroll
    for (int l = 0; l < D; ++l) {
        d[l] = __ldg(dg + l);
        off[l] = op.soff[l];
    }
    const uint32_t ts = thread_slot(op);
    const uint32_t iters = op.iters;
    for (uint32_t j = 0; j < iters; ++j) {
        const uint32_t b = ts ^ op.dhi[j];
#pragma unroll
        for (int l = 0; l < D; ++l) t[b ^ off[l]] = cmul(d[l], t[b ^ off[l]]);
    }
}

__device__ __forceinline__ void op_phase(double2* __restrict__ t, const TileOp& op, double2 ph) {
    if (threadIdx.x >= op.n_groups) return;
    const uint32_t ts = thread_slot(op);
    const uint32_t iters = op.iters;
    for (uint32_t j = 0; j < iters; ++j) {
        const uint32_t p = ts ^ op.dhi[j];
        t[p] = cmul(ph, t[p]);
    }
}

template <int M, int KMAX>
__global__ void __launch_bounds__(kTileThreads, 2) k_tile(double2* __restrict__ st, TilePass p,
                                                          const TileOp* __restrict__ ops,
                                                          const double2* __restrict__ mats) {
    constexpr uint32_t kSize = 1u << M;
    constexpr uint32_t kEpt = kSize / kTileThreads;      // elements per thread
    extern __shared__ __align__(16) unsigned char smem[];
    double2* __restrict__ tile = reinterpret_cast<double2*>(smem);
    TileOp* sops = reinterpret_cast<TileOp*>(smem + sizeof(double2) * kSize);
    __shared__ uint64_t rowoff[1u << kTileMaxHigh];
    const uint32_t L = p.L;
    const uint32_t rows = 1u << p.h;
    for (uint32_t r = threadIdx.x; r < rows; r += blockDim.x) {
        uint64_t off = 0;
        for (uint32_t i = 0; i < p.h; ++i)
            if ((r >> i) & 1u) off |= uint64_t{1} << p.hbits[i];
        rowoff[r] = off;
    }
    {
        const uint32_t words = p.n_ops * static_cast<uint32_t>(sizeof(TileOp) / sizeof(uint32_t));
        const uint32_t* src = reinterpret_cast<const uint32_t*>(ops);
        uint32_t* dst = reinterpret_cast<uint32_t*>(sops);
        for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
    }
    __syncthreads();
    // element e = tid + kTileThreads * u: column bits come from tid alone (L <= 8)
    const uint32_t col = threadIdx.x & ((1u << L) - 1u);
    const uint32_t row0 = threadIdx.x >> L;
    const uint32_t row_step = kTileThreads >> L;
    const uint32_t swt = tile_swizzle(threadIdx.x);
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    for (uint64_t tid = blockIdx.x; tid < p.n_tiles; tid += gridDim.x) {
        uint64_t base = tid << L;
        for (uint32_t i = 0; i < p.h; ++i) base = insert_zero_bit(base, p.hbits[i]);
        base |= col;
        {
            double2 v[kEpt];
#pragma unroll
            for (uint32_t u = 0; u < kEpt; ++u) v[u] = __ldcs(s + (base | rowoff[row0 + u * row_step]));
#pragma unroll
            for (uint32_t u = 0; u < kEpt; ++u) tile[swt ^ tile_swizzle(u * kTileThreads)] = v[u];
        }
        __syncthreads();
        for (uint32_t o = 0; o < p.n_ops; ++o) {
            const TileOp& op = sops[o];
            if ((base & op.gcmask) != op.gcmask) continue;   // uniform across the CTA
            const double2* mat = mats + op.mat_off;
            const uint32_t kind = op.kind, k = op.k;
            if (kind == kTileDense) {
                if (k == 1) op_dense1(tile, op, mat);
                else if (KMAX <= 2 || k == 2) op_dense2(tile, op, mat);
                else if (k == 3) op_dense_wide<(KMAX > 2 ? 3 : 1)>(tile, op, mat);
                else op_dense_wide<(KMAX > 2 ? 4 : 1)>(tile, op, mat);
            } else if (kind == kTileDiag) {
                if (k == 1) op_diag<1>(tile, op, mat);
                else if (KMAX <= 2 || k == 2) op_diag<2>(tile, op, mat);
                else if (k == 3) op_diag<(KMAX > 2 ? 3 : 1)>(tile, op, mat);
                else op_diag<(KMAX > 2 ? 4 : 1)>(tile, op, mat);
            } else {
                op_phase(tile, op, __ldg(mat));
            }
            __syncthreads();
        }
#pragma unroll
        for (uint32_t u = 0; u < kEpt; ++u)
            __stcs(s + (base | rowoff[row0 + u * row_step]), tile[swt ^ tile_swizzle(u * kTileThreads)]);
        __syncthreads();
    }
}

template <int M>
void launch_m(const LaunchCtx& ctx, double2* st, uint32_t batch, const TilePass& p, size_t smem,
              const TileOp* d_ops, const double2* d_mats) {
    auto kern = p.kmax <= 2 ? k_tile<M, 2> : k_tile<M, 4>;
    // per device and cheap: set on every launch so any device the caller switches to has it
    cuda_check_launch_attr(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(kTileMaxSmem)));
    const uint32_t per_sm = static_cast<uint32_t>(std::max<size_t>(1, (224 * 1024) / (smem + 3072)));
    const uint64_t want = static_cast<uint64_t>(ctx.num_sms) * std::min<uint32_t>(per_sm, 2);
    const uint32_t grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(want, p.n_tiles)));
    kern<<<dim3(grid, batch), kTileThreads, smem, ctx.stream>>>(st, p, d_ops, d_mats);
    check_launch("tile_pass");
}

}  // namespace

size_t tile_smem_bytes(const TilePass& pass) {
    return sizeof(double2) * (size_t{1} << pass.m) + sizeof(TileOp) * pass.n_ops;
}

void launch_tile_pass(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                      const TilePass& pass, const TileOp* d_ops, const double2* d_mats) {
    TilePass p = pass;
    p.batch_stride = uint64_t{1} << n;
    p.n_tiles = (uint64_t{1} << n) >> p.m;
    const size_t smem = tile_smem_bytes(p);
    if (smem > kTileMaxSmem || p.m < kTileMinBits || p.m > kTileMaxBits || p.L > kTileMinBits)
        throw std::logic_error("tile pass: unsupported shape");
    switch (p.m) {
        case 8: launch_m<8>(ctx, st, batch, p, smem, d_ops, d_mats); break;
        case 9: launch_m<9>(ctx, st, batch, p, smem, d_ops, d_mats); break;
        case 10: launch_m<10>(ctx, st, batch, p, smem, d_ops, d_mats); break;
        case 11: launch_m<11>(ctx, st, batch, p, smem, d_ops, d_mats); break;
        case 12: launch_m<12>(ctx, st, batch, p, smem, d_ops, d_mats); break;
        default: launch_m<13>(ctx, st, batch, p, smem, d_ops, d_mats); break;
    }
}

void cuda_check_launch_attr(cudaError_t e) {
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    }
}

}  // namespace lqcs_b200
