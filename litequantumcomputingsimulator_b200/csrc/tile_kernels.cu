// tile_kernels.cu — multi-gate passes through shared memory.
//
// One launch applies a whole list of operations to the state in a single HBM read and
// write.  The state is cut into tiles of 2^m amplitudes: a tile holds every amplitude whose
// bits outside the tile-bit set {0..L-1} u H are fixed, H being up to m-L chosen high
// qubits.  A CTA copies a tile into shared memory (2^|H| runs of 2^L contiguous
// amplitudes, each run a coalesced stretch of at least 512 bytes), applies the operation
// list to it with a barrier between operations, and writes it back.  An operation may act
// only on tile bits through its targets; its controls (and the bits of a phase) may lie
// outside the tile, where they are constant for the whole tile and become a per-tile
// predicate.  Reference semantics of each operation: src/backend/kernels/gate_kernels.cpp.
//
// Per CTA the pass's operation records are staged in shared memory once; per operation
// every thread copies the record's fields and (for k <= 2) the whole matrix into registers,
// so the inner loops over groups touch shared memory only for the amplitudes themselves.
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

// Shared-memory slot of tile element i.  A warp's 16-byte accesses are served in
// 128-byte wavefronts (8 slots); operations on low qubits access power-of-two strides,
// which would put many threads of a wavefront on the same banks.  XOR-ing the slot's low 3
// bits with a fold of its higher bits (a bijection) spreads every power-of-two stride over
// all 8 positions of a wavefront.
__device__ __forceinline__ uint32_t sw(uint32_t i) {
    return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9) ^ (i >> 12)) & 7u);
}

__device__ __forceinline__ uint32_t insert0(uint32_t v, uint32_t pos) {
    const uint32_t low = (1u << pos) - 1u;
    return ((v & ~low) << 1) | (v & low);
}

// The fields of one operation, held in registers while it is applied.
struct OpRegs {
    uint32_t kind, k, nf, lcmask, mat_off, n_lctrl;
    uint32_t f[8];
    uint32_t off[16];
};

__device__ __forceinline__ void read_op(const TileOp& s, OpRegs& r) {
    r.kind = s.kind;
    r.k = s.k;
    r.nf = s.n_fixed;
    r.lcmask = s.lcmask;
    r.mat_off = s.mat_off;
    r.n_lctrl = s.n_lctrl;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.f[i] = s.fixed[i];
}

__device__ __forceinline__ uint32_t group_base(uint32_t g, const OpRegs& r) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (i < static_cast<int>(r.nf)) g = insert0(g, r.f[i]);
    return g | r.lcmask;
}

__device__ __forceinline__ void op_dense1(double2* __restrict__ t, const TileOp& s, const OpRegs& r,
                                          const double2* __restrict__ mat, uint32_t m) {
    const double2 m0 = __ldg(mat), m1 = __ldg(mat + 1), m2 = __ldg(mat + 2), m3 = __ldg(mat + 3);
    const uint32_t o1 = s.loff[1];
    const uint32_t groups = (1u << m) >> (1 + r.n_lctrl);
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
        const uint32_t i0 = group_base(g, r);
        const uint32_t p0 = sw(i0), p1 = sw(i0 | o1);
        const double2 a0 = t[p0], a1 = t[p1];
        t[p0] = cmad(m1, a1, cmul(m0, a0));
        t[p1] = cmad(m3, a1, cmul(m2, a0));
    }
}

__device__ __forceinline__ void op_dense2(double2* __restrict__ t, const TileOp& s, const OpRegs& r,
                                          const double2* __restrict__ mat, uint32_t m) {
    double2 mm[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) mm[i] = __ldg(mat + i);
    const uint32_t o1 = s.loff[1], o2 = s.loff[2], o3 = s.loff[3];
    const uint32_t groups = (1u << m) >> (2 + r.n_lctrl);
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
        const uint32_t b = group_base(g, r);
        const uint32_t p0 = sw(b), p1 = sw(b | o1), p2 = sw(b | o2), p3 = sw(b | o3);
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
__device__ __forceinline__ void op_dense_wide(double2* __restrict__ t, const TileOp& s,
                                              const OpRegs& r, const double2* __restrict__ mat,
                                              uint32_t m) {
    constexpr int D = 1 << K;
    uint32_t off[D];
#pragma unroll
    for (int l = 0; l < D; ++l) off[l] = s.loff[l];
    const uint32_t groups = (1u << m) >> (K + r.n_lctrl);
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
        const uint32_t b = group_base(g, r);
        double2 a[D];
#pragma unroll
        for (int l = 0; l < D; ++l) a[l] = t[sw(b | off[l])];
#pragma unroll 1
        for (int row = 0; row < D; ++row) {
            double2 acc = cmul(__ldg(mat + row * D), a[0]);
#pragma unroll
            for (int c = 1; c < D; ++c) acc = cmad(__ldg(mat + row * D + c), a[c], acc);
            t[sw(b | off[row])] = acc;
        }
    }
}

template <int K>
__device__ __forceinline__ void op_diag(double2* __restrict__ t, const TileOp& s, const OpRegs& r,
                                        const double2* __restrict__ dg, uint32_t m) {
    constexpr int D = 1 << K;
    double2 d[D];
    uint32_t off[D];
#pragma unroll
    for (int l = 0; l < D; ++l) {
        d[l] = __ldg(dg + l);
        off[l] = s.loff[l];
    }
    const uint32_t groups = (1u << m) >> (K + r.n_lctrl);
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
        const uint32_t b = group_base(g, r);
#pragma unroll
        for (int l = 0; l < D; ++l) {
            const uint32_t p = sw(b | off[l]);
            t[p] = cmul(d[l], t[p]);
        }
    }
}

__device__ __forceinline__ void op_phase(double2* __restrict__ t, const OpRegs& r, double2 ph,
                                         uint32_t m) {
    const uint32_t n_amps = (1u << m) >> r.nf;
    for (uint32_t g = threadIdx.x; g < n_amps; g += blockDim.x) {
        const uint32_t idx = sw(group_base(g, r));
        t[idx] = cmul(ph, t[idx]);
    }
}

template <int KMAX>
__global__ void __launch_bounds__(kTileThreads, 2) k_tile(double2* __restrict__ st, TilePass p,
                                                          const TileOp* __restrict__ ops,
                                                          const double2* __restrict__ mats) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t m = p.m;
    const uint32_t L = p.L;
    const uint32_t run = 1u << L;
    const uint32_t rows = 1u << p.h;
    const uint32_t tsize = 1u << m;
    double2* __restrict__ tile = reinterpret_cast<double2*>(smem);
    TileOp* sops = reinterpret_cast<TileOp*>(smem + sizeof(double2) * tsize);
    __shared__ uint64_t rowoff[1u << kTileMaxHigh];
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
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    for (uint64_t tid = blockIdx.x; tid < p.n_tiles; tid += gridDim.x) {
        // base address of this tile: tile id spread over the non-tile bits >= L
        uint64_t base = tid << L;
        for (uint32_t i = 0; i < p.h; ++i) base = insert_zero_bit(base, p.hbits[i]);
        // load: element e = row * run + col; 4 independent loads in flight per thread
        for (uint32_t e0 = threadIdx.x; e0 < tsize; e0 += 4 * blockDim.x) {
            double2 v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t e = e0 + u * blockDim.x;
                if (e < tsize) v[u] = __ldcs(s + (base | rowoff[e >> L] | (e & (run - 1))));
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t e = e0 + u * blockDim.x;
                if (e < tsize) tile[sw(e)] = v[u];
            }
        }
        __syncthreads();
        for (uint32_t o = 0; o < p.n_ops; ++o) {
            const TileOp& so = sops[o];
            if ((base & so.gcmask) != so.gcmask) continue;   // uniform across the CTA
            OpRegs r;
            read_op(so, r);
            const double2* mat = mats + r.mat_off;
            if (r.kind == kTileDense) {
                if (r.k == 1) op_dense1(tile, so, r, mat, m);
                else if (KMAX <= 2 || r.k == 2) op_dense2(tile, so, r, mat, m);
                else if (r.k == 3) op_dense_wide<(KMAX > 2 ? 3 : 1)>(tile, so, r, mat, m);
                else op_dense_wide<(KMAX > 2 ? 4 : 1)>(tile, so, r, mat, m);
            } else if (r.kind == kTileDiag) {
                if (r.k == 1) op_diag<1>(tile, so, r, mat, m);
                else if (KMAX <= 2 || r.k == 2) op_diag<2>(tile, so, r, mat, m);
                else if (r.k == 3) op_diag<(KMAX > 2 ? 3 : 1)>(tile, so, r, mat, m);
                else op_diag<(KMAX > 2 ? 4 : 1)>(tile, so, r, mat, m);
            } else {
                op_phase(tile, r, __ldg(mat), m);
            }
            __syncthreads();
        }
        for (uint32_t e = threadIdx.x; e < tsize; e += blockDim.x)
            __stcs(s + (base | rowoff[e >> L] | (e & (run - 1))), tile[sw(e)]);
        __syncthreads();
    }
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
    if (smem > kTileMaxSmem) throw std::logic_error("tile pass: shared memory budget exceeded");
    auto kern = pass.kmax <= 2 ? k_tile<2> : k_tile<4>;
    // per device and cheap: set on every launch so any device the caller switches to has it
    cuda_check_launch_attr(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(kTileMaxSmem)));
    const uint32_t per_sm = static_cast<uint32_t>(std::max<size_t>(1, (224 * 1024) / (smem + 3072)));
    const uint64_t want = static_cast<uint64_t>(ctx.num_sms) * std::min<uint32_t>(per_sm, 2);
    const uint32_t grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(want, p.n_tiles)));
    kern<<<dim3(grid, batch), kTileThreads, smem, ctx.stream>>>(st, p, d_ops, d_mats);
    check_launch("tile_pass");
}

void cuda_check_launch_attr(cudaError_t e) {
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    }
}

}  // namespace lqcs_b200
