// rot_tile_kernels.cu — runs of Pauli rotations on shared-memory tiles (batched adjoint).
//
// The adjoint gradient (adjoint.cpp) walks an ansatz of Pauli rotations exp(-i theta/2 P)
// forward over a batch of states, then backward over two batches (psi and lambda), taking
// Im<lambda|P|psi> before undoing each rotation.  One launch per rotation reads and writes
// every state once per rotation; here a run of rotations whose X masks lie inside a tile of
// 2^m amplitudes (qubits 0..L-1 plus up to m-L others) is applied to each tile in shared
// memory in one launch, so a pass costs one read and one write of the states however many
// rotations it holds.  A rotation acts on a tile by the same formulas as the one-rotation
// kernel (k_pauli, gate_kernels.cpp's launch_pauli_rotation_batched; the reference's
// apply_pauli_rotation, src/backend/kernels/gate_kernels.cpp:191-225):
//     psi'[i] = cos * psi[i] + (-i sin) i^{n_y} (-1)^{popcount((i ^ x) & zy)} psi[i ^ x].
// Z / Y bits outside the tile only flip the sign, uniformly over a tile.  Backward passes
// write one partial Im<lambda|P|psi> per (rotation, state, tile); a second launch sums the
// tiles in a fixed order into the gradient.
#include <algorithm>
#include <stdexcept>
#include <string>

#include "common.cuh"
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

__device__ __forceinline__ double sign_of(uint32_t parity) { return parity ? -1.0 : 1.0; }

// (-i sin) i^{n_y}, formed as the one-rotation kernel forms it
__device__ __forceinline__ double2 y_phase(double sin_h, uint32_t n_y) {
    const double2 mis = make_double2(0.0, -sin_h);
    const uint32_t r = n_y & 3u;
    const double2 ip = (r == 0) ? make_double2(1, 0)
                     : (r == 1) ? make_double2(0, 1)
                     : (r == 2) ? make_double2(-1, 0) : make_double2(0, -1);
    return cmul(mis, ip);
}

__device__ __forceinline__ uint32_t insert_zero32(uint32_t v, uint32_t pos) {
    const uint32_t low = (1u << pos) - 1u;
    return ((v & ~low) << 1) | (v & low);
}

// A rotation as the tile loop reads it: staged in shared memory at the start of a launch,
// with this state's cos and (-i sin) i^{n_y} (the inverse's for a backward pass) and the
// tile-uniform sign parity of the Z / Y bits outside the tile.
struct RotStaged {
    double2 c;
    double2 yph;
    uint32_t x_loc, zy_loc, tpar, n_y;
};

// Stages ops[0 .. n_ops) for state blockIdx.y; the caller synchronises.
__device__ __forceinline__ void stage_ops(RotStaged* so, const RotTileOp* ops, uint32_t n_ops,
                                          const double2* cs, uint32_t R, uint64_t base,
                                          bool inverse) {
    for (uint32_t k = threadIdx.x; k < n_ops; k += blockDim.x) {
        const RotTileOp op = ops[k];
        const double2 csv = __ldg(cs + static_cast<uint64_t>(op.param) * R + blockIdx.y);
        RotStaged r;
        r.c = make_double2(csv.x, 0.0);
        r.yph = y_phase(inverse ? -csv.y : csv.y, op.n_y);
        r.x_loc = op.x_loc;
        r.zy_loc = op.zy_loc;
        r.tpar = __popcll(base & op.zy_out) & 1u;
        r.n_y = op.n_y;
        so[k] = r;
    }
}

// Tile base of tile t (zero at every tile bit) and the global offset of each tile bit.
__device__ __forceinline__ uint64_t tile_base(uint64_t t, const RotTilePass& p,
                                              const uint32_t* hb) {
    uint64_t base = t << p.L;
    for (uint32_t i = 0; i < p.h; ++i) base = insert_zero_bit(base, hb[i]);
    return base;
}

__device__ __forceinline__ uint64_t tile_offset(uint32_t l, const RotTilePass& p,
                                                const uint32_t* hb) {
    uint64_t g = l & ((1u << p.L) - 1u);
    for (uint32_t i = 0; i < p.h; ++i)
        if ((l >> (p.L + i)) & 1u) g |= uint64_t{1} << hb[i];
    return g;
}

// One rotation on a tile in shared memory (pairs split over the CTA's threads).
__device__ __forceinline__ void rotate_tile(double2* sv, uint32_t T, const RotStaged& op) {
    const double2 c = op.c, yph = op.yph;
    if (op.x_loc == 0) {
        for (uint32_t l = threadIdx.x; l < T; l += blockDim.x) {
            const double sg = sign_of((__popc(l & op.zy_loc) ^ op.tpar) & 1u);
            const double2 f = make_double2(c.x + yph.x * sg, c.y + yph.y * sg);
            sv[l] = cmul(sv[l], f);
        }
        return;
    }
    const uint32_t hb = 31u - __clz(op.x_loc);
    for (uint32_t q = threadIdx.x; q < T / 2; q += blockDim.x) {
        const uint32_t l0 = insert_zero32(q, hb), l1 = l0 ^ op.x_loc;
        const double2 a = sv[l0], b = sv[l1];
        const double s0 = sign_of((__popc(l1 & op.zy_loc) ^ op.tpar) & 1u);   // (l0 ^ x) = l1
        const double s1 = sign_of((__popc(l0 & op.zy_loc) ^ op.tpar) & 1u);
        sv[l0] = cmad(cscale(yph, s0), b, cmul(c, a));
        sv[l1] = cmad(cscale(yph, s1), a, cmul(c, b));
    }
}

__global__ void __launch_bounds__(kRotThreads) k_rot_tile_fwd(double2* __restrict__ st,
                                                              uint64_t len, RotTilePass p,
                                                              const RotTileOp* __restrict__ ops,
                                                              const double2* __restrict__ cs,
                                                              uint32_t R) {
    extern __shared__ __align__(16) double2 sv[];
    __shared__ uint32_t hb[kRotMaxHigh];
    __shared__ RotStaged so[kRotMaxOps];
    if (threadIdx.x < kRotMaxHigh) hb[threadIdx.x] = p.hbits[threadIdx.x < p.h ? threadIdx.x : 0];
    __syncthreads();
    double2* s = st + static_cast<uint64_t>(blockIdx.y) * len;
    const uint32_t T = 1u << p.m;
    const uint64_t base = tile_base(blockIdx.x, p, hb);
    // local index l = threadIdx.x + j * blockDim.x: its offset is the OR of both parts'
    __shared__ uint64_t offj[kRotMaxRows];
    const uint32_t rows = T / blockDim.x;
    if (threadIdx.x < rows) offj[threadIdx.x] = tile_offset(threadIdx.x * blockDim.x, p, hb);
    stage_ops(so, ops, p.n_ops, cs, R, base, false);
    const uint64_t off_t = base | tile_offset(threadIdx.x, p, hb);
    __syncthreads();
    for (uint32_t j = 0; j < rows; ++j) sv[threadIdx.x + j * blockDim.x] = __ldcg(s + (off_t | offj[j]));
    __syncthreads();
    for (uint32_t k = 0; k < p.n_ops; ++k) {
        rotate_tile(sv, T, so[k]);
        __syncthreads();
    }
    for (uint32_t j = 0; j < rows; ++j) s[off_t | offj[j]] = sv[threadIdx.x + j * blockDim.x];
}

// Backward: for each rotation, Im<lambda|P|psi> over the tile, then the inverse rotation on
// both tiles.  partials[(k * nb + state) * n_tiles + tile].
__global__ void __launch_bounds__(kRotThreads) k_rot_tile_bwd(double2* __restrict__ psi,
                                                              double2* __restrict__ lam,
                                                              uint64_t len, RotTilePass p,
                                                              const RotTileOp* __restrict__ ops,
                                                              const double2* __restrict__ cs,
                                                              uint32_t R,
                                                              double* __restrict__ partials) {
    extern __shared__ __align__(16) double2 sv[];
    __shared__ uint32_t hb[kRotMaxHigh];
    __shared__ double red[2][kRotThreads / 32];
    __shared__ RotStaged so[kRotMaxOps];
    if (threadIdx.x < kRotMaxHigh) hb[threadIdx.x] = p.hbits[threadIdx.x < p.h ? threadIdx.x : 0];
    __syncthreads();
    const uint32_t T = 1u << p.m;
    double2* sp = sv;
    double2* sl = sv + T;
    double2* gp = psi + static_cast<uint64_t>(blockIdx.y) * len;
    double2* gl = lam + static_cast<uint64_t>(blockIdx.y) * len;
    const uint64_t base = tile_base(blockIdx.x, p, hb);
    __shared__ uint64_t offj[kRotMaxRows];
    const uint32_t rows = T / blockDim.x;
    if (threadIdx.x < rows) offj[threadIdx.x] = tile_offset(threadIdx.x * blockDim.x, p, hb);
    stage_ops(so, ops, p.n_ops, cs, R, base, true);   // the inverse rotations
    const uint64_t off_t = base | tile_offset(threadIdx.x, p, hb);
    __syncthreads();
    for (uint32_t j = 0; j < rows; ++j) {
        const uint64_t g = off_t | offj[j];
        sp[threadIdx.x + j * blockDim.x] = __ldcg(gp + g);
        sl[threadIdx.x + j * blockDim.x] = __ldcg(gl + g);
    }
    __syncthreads();
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t k = 0; k < p.n_ops; ++k) {
        const RotStaged& op = so[k];
        const uint32_t tpar = op.tpar;
        const double2 c = op.c;
        const double2 yinv = op.yph;
        double v0 = 0.0, v1 = 0.0;   // sum of sign * conj(lambda_i) * psi_{i ^ x}
        if (op.x_loc == 0) {
            for (uint32_t l = threadIdx.x; l < T; l += blockDim.x) {
                const double sg = sign_of((__popc(l & op.zy_loc) ^ tpar) & 1u);
                const double2 u = sl[l], w = sp[l];
                v0 += sg * (u.x * w.x + u.y * w.y);
                v1 += sg * (u.x * w.y - u.y * w.x);
                const double2 f = make_double2(c.x + yinv.x * sg, c.y + yinv.y * sg);
                sp[l] = cmul(w, f);
                sl[l] = cmul(u, f);
            }
        } else {
            const uint32_t hbit = 31u - __clz(op.x_loc);
            for (uint32_t q = threadIdx.x; q < T / 2; q += blockDim.x) {
                const uint32_t l0 = insert_zero32(q, hbit), l1 = l0 ^ op.x_loc;
                const double2 a = sp[l0], b = sp[l1], la = sl[l0], lb = sl[l1];
                const double s0 = sign_of((__popc(l1 & op.zy_loc) ^ tpar) & 1u);
                const double s1 = sign_of((__popc(l0 & op.zy_loc) ^ tpar) & 1u);
                v0 += s0 * (la.x * b.x + la.y * b.y);
                v1 += s0 * (la.x * b.y - la.y * b.x);
                v0 += s1 * (lb.x * a.x + lb.y * a.y);
                v1 += s1 * (lb.x * a.y - lb.y * a.x);
                sp[l0] = cmad(cscale(yinv, s0), b, cmul(c, a));
                sp[l1] = cmad(cscale(yinv, s1), a, cmul(c, b));
                sl[l0] = cmad(cscale(yinv, s0), lb, cmul(c, la));
                sl[l1] = cmad(cscale(yinv, s1), la, cmul(c, lb));
            }
        }
        // times i^{n_y}, imaginary part
        double im;
        switch (op.n_y & 3u) {
            case 0: im = v1; break;
            case 1: im = v0; break;
            case 2: im = -v1; break;
            default: im = -v0; break;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) im += __shfl_xor_sync(0xffffffffu, im, o);
        if (lane == 0) red[k & 1u][warp] = im;
        __syncthreads();   // also orders this rotation's writes before the next one's reads
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += red[k & 1u][w];
            partials[(static_cast<uint64_t>(k) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
        }
    }
    for (uint32_t j = 0; j < rows; ++j) {
        const uint64_t g = off_t | offj[j];
        gp[g] = sp[threadIdx.x + j * blockDim.x];
        gl[g] = sl[threadIdx.x + j * blockDim.x];
    }
}

// grad[state * np + param_k] = sum over tiles of partials[(k * nb + state) * n_tiles + t]
__global__ void __launch_bounds__(kRotThreads) k_rot_grad(const double* __restrict__ partials,
                                                          uint32_t n_tiles,
                                                          const RotTileOp* __restrict__ ops,
                                                          double* __restrict__ grad, uint64_t np) {
    const uint32_t k = blockIdx.x, b = blockIdx.y;
    const double* row = partials + (static_cast<uint64_t>(k) * gridDim.y + b) * n_tiles;
    double v = 0.0;
    for (uint32_t t = threadIdx.x; t < n_tiles; t += blockDim.x) v += row[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __shared__ double sh[kRotThreads / 32];
    if ((threadIdx.x & 31u) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += sh[w];
        grad[static_cast<uint64_t>(b) * np + ops[k].param] = t;
    }
}

void check_pass(const RotTilePass& p, uint32_t n) {
    if (p.m > n || p.m < 1 || p.m > kRotMaxBits || p.L > p.m || p.h != p.m - p.L ||
        p.h > kRotMaxHigh || p.n_ops == 0 || p.n_ops > kRotMaxOps)
        throw std::logic_error("rotation tile pass: unsupported shape");
}

}  // namespace

size_t rot_tile_smem(uint32_t m, bool backward) {
    return sizeof(double2) * (size_t{1} << m) * (backward ? 2 : 1);
}

void launch_rot_tile_fwd(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t nb,
                         const RotTilePass& p, const RotTileOp* d_ops, const double2* d_cs,
                         uint32_t R) {
    check_pass(p, n);
    const size_t smem = rot_tile_smem(p.m, false);
    cuda_check_launch_attr(cudaFuncSetAttribute(k_rot_tile_fwd,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(smem)));
    const uint32_t threads = std::min<uint32_t>(kRotThreads, std::max<uint32_t>(32, 1u << p.m));
    k_rot_tile_fwd<<<dim3(1u << (n - p.m), nb), threads, smem, ctx.stream>>>(
        st, uint64_t{1} << n, p, d_ops, d_cs, R);
    check_launch("rotation tile pass");
}

void launch_rot_tile_bwd(const LaunchCtx& ctx, double2* psi, double2* lam, uint32_t n,
                         uint32_t nb, const RotTilePass& p, const RotTileOp* d_ops,
                         const double2* d_cs, uint32_t R, double* d_partials, double* d_grad,
                         uint64_t np) {
    check_pass(p, n);
    const size_t smem = rot_tile_smem(p.m, true);
    cuda_check_launch_attr(cudaFuncSetAttribute(k_rot_tile_bwd,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(smem)));
    const uint32_t threads = std::min<uint32_t>(kRotThreads, std::max<uint32_t>(32, 1u << p.m));
    const uint32_t n_tiles = 1u << (n - p.m);
    k_rot_tile_bwd<<<dim3(n_tiles, nb), threads, smem, ctx.stream>>>(
        psi, lam, uint64_t{1} << n, p, d_ops, d_cs, R, d_partials);
    check_launch("rotation tile pass (backward)");
    k_rot_grad<<<dim3(p.n_ops, nb), kRotThreads, 0, ctx.stream>>>(d_partials, n_tiles, d_ops,
                                                                  d_grad, np);
    check_launch("rotation gradients");
}

}  // namespace lqcs_b200
