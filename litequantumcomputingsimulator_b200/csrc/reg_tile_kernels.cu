// reg_tile_kernels.cu — multi-gate passes with the tile held in registers.
//
// Same passes as tile_kernels.cu (one HBM read and write of the state applies a whole list
// of operations), with a different home for the tile: each thread keeps 16 amplitudes in
// registers and shared memory only serves the remaps that change which 4 tile bits are
// register bits (see RegLayout).  Per amplitude and operation the shared-memory kernel
// moves 32 bytes through shared memory; here a dense operation on register bits moves
// none, so the pass runs at the FP64 rate instead of the shared-memory rate.
//
// Operation semantics follow the reference kernels (src/backend/kernels/gate_kernels.cpp):
// a dense operation is a 2^k x 2^k matrix on its targets applied where every control is 1;
// a diagonal operation multiplies by the entry its target bits select; a phase operation
// multiplies the amplitudes whose phase bits are all 1.
#include <algorithm>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "kernels.cuh"
#include "tile.cuh"

namespace lqcs_b200 {

namespace {

constexpr int kE = 1 << kRegBits;   // amplitudes per thread
constexpr uint32_t kRegSlotLayouts = 16;   // layouts whose per-thread slots are tabulated

void check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA launch failed in ") + what + ": " +
                                 cudaGetErrorString(e));
    }
    count_launch();
}

__host__ __device__ constexpr int popc4(int m) {
    return (m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) + ((m >> 3) & 1);
}

// Member l of a group: the bits of l spread over the set bits of mask, lowest first.
__host__ __device__ constexpr int deposit4(int l, int mask) {
    int out = 0, j = 0;
    for (int b = 0; b < kRegBits; ++b) {
        if ((mask >> b) & 1) {
            if ((l >> j) & 1) out |= 1 << b;
            ++j;
        }
    }
    return out;
}

// Shared-memory load the compiler may not hoist or merge: matrix entries are re-read per
// group so they never occupy registers alongside the 16 amplitudes.
__device__ __forceinline__ double2 lds2(uint32_t saddr) {
    double2 r;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "r"(saddr));
    return r;
}

// Matrix entries of an operation, entry i at 16 * i bytes of shared memory (the helpers
// below take any functor of this shape).
struct SharedMat {
    uint32_t base;   // shared-memory address
    __device__ __forceinline__ double2 operator()(uint32_t i) const { return lds2(base + 16u * i); }
};

// Group base of the g-th group of a target mask: g spread over the bits outside TM.
__host__ __device__ constexpr int group_base(int g, int tm) { return deposit4(g, (kE - 1) & ~tm); }

// Dense operation without register controls: one basic block, so the compiler interleaves
// the groups.  Two-target operations take two groups per matrix read (each entry is loaded
// twice per operation instead of four times).
template <int TM, class MS>
__device__ __forceinline__ void reg_dense_free(double2 (&v)[kE], const MS& mat) {
    constexpr int K = popc4(TM);
    constexpr int D = 1 << K;
    constexpr int G = kE / D;   // groups
    if constexpr (K == 1) {
        const double2 m0 = mat(0), m1 = mat(1), m2 = mat(2), m3 = mat(3);
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int b = group_base(g, TM);
            const double2 a0 = v[b], a1 = v[b | TM];
            v[b] = cmad(m1, a1, cmul(m0, a0));
            v[b | TM] = cmad(m3, a1, cmul(m2, a0));
        }
    } else if constexpr (K == 2) {
#pragma unroll
        for (int g = 0; g < G; g += 2) {
            const int b0 = group_base(g, TM), b1 = group_base(g + 1, TM);
            double2 y0[D], y1[D];
#pragma unroll
            for (int r = 0; r < D; ++r) {
                const double2 mr = mat(r * D);
                y0[r] = cmul(mr, v[b0]);
                y1[r] = cmul(mr, v[b1]);
            }
#pragma unroll
            for (int c = 1; c < D; ++c) {
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    const double2 mr = mat(r * D + c);
                    y0[r] = cmad(mr, v[b0 | deposit4(c, TM)], y0[r]);
                    y1[r] = cmad(mr, v[b1 | deposit4(c, TM)], y1[r]);
                }
            }
#pragma unroll
            for (int r = 0; r < D; ++r) {
                v[b0 | deposit4(r, TM)] = y0[r];
                v[b1 | deposit4(r, TM)] = y1[r];
            }
        }
    } else {
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int b = group_base(g, TM);
            double2 y[D];
#pragma unroll
            for (int r = 0; r < D; ++r) {
                double2 acc = cmul(mat(r * D), v[b]);
#pragma unroll
                for (int c = 1; c < D; ++c)
                    acc = cmad(mat(r * D + c), v[b | deposit4(c, TM)], acc);
                y[r] = acc;
            }
#pragma unroll
            for (int r = 0; r < D; ++r) v[b | deposit4(r, TM)] = y[r];
        }
    }
}

// Dense operation with register controls: groups whose control bits are not all 1 skip.
template <int TM, class MS>
__device__ __forceinline__ void reg_dense(double2 (&v)[kE], const MS& mat, uint32_t rcmask) {
    constexpr int K = popc4(TM);
    constexpr int D = 1 << K;
    if constexpr (K == 1) {
        const double2 m0 = mat(0), m1 = mat(1), m2 = mat(2), m3 = mat(3);
#pragma unroll
        for (int b = 0; b < kE; ++b) {
            if (b & TM) continue;
            if ((b & rcmask) != rcmask) continue;
            const double2 a0 = v[b], a1 = v[b | TM];
            v[b] = cmad(m1, a1, cmul(m0, a0));
            v[b | TM] = cmad(m3, a1, cmul(m2, a0));
        }
    } else {
#pragma unroll
        for (int b = 0; b < kE; ++b) {
            if (b & TM) continue;
            if ((b & rcmask) != rcmask) continue;
            double2 y[D];
#pragma unroll
            for (int r = 0; r < D; ++r) {
                double2 acc = cmul(mat(r * D), v[b | deposit4(0, TM)]);
#pragma unroll
                for (int c = 1; c < D; ++c)
                    acc = cmad(mat(r * D + c), v[b | deposit4(c, TM)], acc);
                y[r] = acc;
            }
#pragma unroll
            for (int r = 0; r < D; ++r) v[b | deposit4(r, TM)] = y[r];
        }
    }
}

template <int I>
__device__ __forceinline__ void reg_swapx(double2 (&v)[kE], uint32_t rcmask) {
#pragma unroll
    for (int b = 0; b < kE; ++b) {
        if ((b >> I) & 1) continue;
        if ((b & rcmask) != rcmask) continue;
        const double2 a = v[b];
        v[b] = v[b | (1 << I)];
        v[b | (1 << I)] = a;
    }
}

template <class MS>
__device__ __forceinline__ void dispatch_dense(double2 (&v)[kE], uint32_t code, const MS& mat,
                                               uint32_t rcmask) {
    if (rcmask == 0) {
        switch (code) {
            case 1: reg_dense_free<1>(v, mat); break;
            case 2: reg_dense_free<2>(v, mat); break;
            case 3: reg_dense_free<3>(v, mat); break;
            case 4: reg_dense_free<4>(v, mat); break;
            case 5: reg_dense_free<5>(v, mat); break;
            case 6: reg_dense_free<6>(v, mat); break;
            case 7: reg_dense_free<7>(v, mat); break;
            case 8: reg_dense_free<8>(v, mat); break;
            case 9: reg_dense_free<9>(v, mat); break;
            case 10: reg_dense_free<10>(v, mat); break;
            case 11: reg_dense_free<11>(v, mat); break;
            case 12: reg_dense_free<12>(v, mat); break;
            case 13: reg_dense_free<13>(v, mat); break;
            case 14: reg_dense_free<14>(v, mat); break;
            default: break;
        }
        return;
    }
    switch (code) {
        case 1: reg_dense<1>(v, mat, rcmask); break;
        case 2: reg_dense<2>(v, mat, rcmask); break;
        case 3: reg_dense<3>(v, mat, rcmask); break;
        case 4: reg_dense<4>(v, mat, rcmask); break;
        case 5: reg_dense<5>(v, mat, rcmask); break;
        case 6: reg_dense<6>(v, mat, rcmask); break;
        case 7: reg_dense<7>(v, mat, rcmask); break;
        case 8: reg_dense<8>(v, mat, rcmask); break;
        case 9: reg_dense<9>(v, mat, rcmask); break;
        case 10: reg_dense<10>(v, mat, rcmask); break;
        case 11: reg_dense<11>(v, mat, rcmask); break;
        case 12: reg_dense<12>(v, mat, rcmask); break;
        case 13: reg_dense<13>(v, mat, rcmask); break;
        case 14: reg_dense<14>(v, mat, rcmask); break;
        default: break;   // 4-target operations never reach a register pass
    }
}

__device__ __forceinline__ void dispatch_swapx(double2 (&v)[kE], uint32_t code, uint32_t rcmask) {
    switch (code) {
        case 1: reg_swapx<0>(v, rcmask); break;
        case 2: reg_swapx<1>(v, rcmask); break;
        case 4: reg_swapx<2>(v, rcmask); break;
        default: reg_swapx<3>(v, rcmask); break;
    }
}

// Diagonal whose entry bits sit on register-index bits R (and on thread bits, fixed per
// thread in tpart): amplitude u takes entry tpart | e(u & R), so a thread loads each of its
// 2^|R| distinct entries once and multiplies the 16 / 2^|R| amplitudes that share it.
template <int R, class MS>
__device__ __forceinline__ void reg_diag_r(double2 (&v)[kE], const MS& mat, uint32_t rcmask,
                                           uint32_t tpart, uint32_t rb0, uint32_t rb1,
                                           uint32_t rb2, uint32_t rb3) {
#pragma unroll
    for (int pt = 0; pt < kE; ++pt) {
        if ((pt & R) != pt) continue;
        const uint32_t e = tpart | ((pt & 1) ? rb0 : 0u) | ((pt & 2) ? rb1 : 0u) |
                           ((pt & 4) ? rb2 : 0u) | ((pt & 8) ? rb3 : 0u);
        const double2 f = mat(e);
#pragma unroll
        for (int u = 0; u < kE; ++u)
            if ((u & R) == pt && (u & rcmask) == rcmask) v[u] = cmul(f, v[u]);
    }
}

// Entry (tpart | bits picked from u) of a diagonal for every amplitude u.
template <class MS>
__device__ __forceinline__ void reg_diag(double2 (&v)[kE], const RegOp& op, const MS& mat,
                                         uint32_t rcmask) {
    uint32_t tpart = 0, rb0 = 0, rb1 = 0, rb2 = 0, rb3 = 0;   // entry bit of register bit i
    const uint32_t k = op.k;
    for (uint32_t j = 0; j < k; ++j) {
        const uint32_t loc = op.loc[j], bit = 1u << j;
        if (loc & 0x80u) {
            tpart |= ((threadIdx.x >> (loc & 0x7fu)) & 1u) << j;
        } else {
            rb0 |= loc == 0 ? bit : 0u;
            rb1 |= loc == 1 ? bit : 0u;
            rb2 |= loc == 2 ? bit : 0u;
            rb3 |= loc == 3 ? bit : 0u;
        }
    }
    const uint32_t R = (rb0 ? 1u : 0u) | (rb1 ? 2u : 0u) | (rb2 ? 4u : 0u) | (rb3 ? 8u : 0u);
    switch (R) {
#define LQCS_DIAG_CASE(r) \
    case r: reg_diag_r<r>(v, mat, rcmask, tpart, rb0, rb1, rb2, rb3); break;
        LQCS_DIAG_CASE(0) LQCS_DIAG_CASE(1) LQCS_DIAG_CASE(2) LQCS_DIAG_CASE(3)
        LQCS_DIAG_CASE(4) LQCS_DIAG_CASE(5) LQCS_DIAG_CASE(6) LQCS_DIAG_CASE(7)
        LQCS_DIAG_CASE(8) LQCS_DIAG_CASE(9) LQCS_DIAG_CASE(10) LQCS_DIAG_CASE(11)
        LQCS_DIAG_CASE(12) LQCS_DIAG_CASE(13) LQCS_DIAG_CASE(14)
        default: reg_diag_r<15>(v, mat, rcmask, tpart, rb0, rb1, rb2, rb3); break;
#undef LQCS_DIAG_CASE
    }
}

// d += a * b on the FP64 tensor path, one m8n8k4 step: lane l holds a = A[l / 4][l % 4],
// b = B[l % 4][l / 4] and d = D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void mma_f64(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Two-qubit block on the lane pair (kRegMma), every register index whose control bits are
// all 1.  For register u the warp's 32 amplitudes form A (8 groups on lanes 2..4 x 4 members
// on lanes 0..1), split into real and imaginary parts; the 4 x 4 complex matrix M enters as
// B with column n = 2 j + c holding output member j, part c: B_re[k][n] = c ? Im M[j][k] :
// Re M[j][k], B_im[k][n] = c ? Re M[j][k] : -Im M[j][k].  D = A_re B_re + A_im B_im then
// leaves (Re, Im) of the lane's own new amplitude in its two accumulators.  The whole warp
// runs it (the caller keeps it converged); lane l loads one matrix entry.
__device__ __forceinline__ void reg_mma(double2 (&v)[kE], uint32_t mat, uint32_t rcmask) {
    const uint32_t lane = threadIdx.x & 31u;
    const double2 e = lds2(mat + 16u * (((lane >> 3) << 2) | (lane & 3u)));
    const bool im_col = ((lane >> 2) & 1u) != 0;
    const double b_re = im_col ? e.y : e.x, b_im = im_col ? e.x : -e.y;
    if (rcmask == 0) {
#pragma unroll
        for (int u = 0; u < kE; ++u) {
            double d0 = 0.0, d1 = 0.0;
            mma_f64(d0, d1, v[u].x, b_re);
            mma_f64(d0, d1, v[u].y, b_im);
            v[u] = make_double2(d0, d1);
        }
        return;
    }
#pragma unroll
    for (int u = 0; u < kE; ++u) {
        if ((u & rcmask) != rcmask) continue;   // uniform over the warp
        double d0 = 0.0, d1 = 0.0;
        mma_f64(d0, d1, v[u].x, b_re);
        mma_f64(d0, d1, v[u].y, b_im);
        v[u] = make_double2(d0, d1);
    }
}

// Pauli rotation whose flip is the single register bit XR (kRegPauli after the reduction in
// reg_pauli): amplitude u becomes c a_u + y s_u a_(u ^ XR), s_u = (-1)^parity(u & zr), y
// already carrying the sign of the thread's and the tile's Z-type bits; the partner's sign
// is s_u times (-1)^parity(XR & zr).
template <int XR>
__device__ __forceinline__ void reg_pauli_x(double2 (&v)[kE], double c, double2 y, uint32_t zr) {
    const double sx = (zr & XR) ? -1.0 : 1.0;
#pragma unroll
    for (int u = 0; u < kE; ++u) {
        if (u & XR) continue;
        const double2 a = v[u], b = v[u ^ XR];
        const double su = (__popc(static_cast<uint32_t>(u) & zr) & 1u) ? -1.0 : 1.0;
        const double2 yu = cscale(y, su);
        v[u] = cmad(yu, b, cscale(a, c));
        v[u ^ XR] = cmad(cscale(yu, sx), a, cscale(b, c));
    }
}

// The same with flips on lanes too (lane mask xl): the partner of (u, lane) is (u ^ XR,
// lane ^ xl), fetched by shuffle; XR = 0: flips on lanes only.  Every lane of the warp runs it.
template <int XR>
__device__ __forceinline__ void reg_pauli_xl(double2 (&v)[kE], double c, double2 y, uint32_t zr,
                                             uint32_t xl) {
    const int m = static_cast<int>(xl);
    if constexpr (XR == 0) {
#pragma unroll
        for (int u = 0; u < kE; ++u) {
            const double2 b = shfl_xor_d2(v[u], m);
            const double su = (__popc(static_cast<uint32_t>(u) & zr) & 1u) ? -1.0 : 1.0;
            v[u] = cmad(cscale(y, su), b, cscale(v[u], c));
        }
    } else {
#pragma unroll
        for (int u = 0; u < kE; ++u) {
            if (u & XR) continue;
            const double2 pu = shfl_xor_d2(v[u ^ XR], m), pw = shfl_xor_d2(v[u], m);
            const double su = (__popc(static_cast<uint32_t>(u) & zr) & 1u) ? -1.0 : 1.0;
            const double sw = (__popc(static_cast<uint32_t>(u ^ XR) & zr) & 1u) ? -1.0 : 1.0;
            v[u] = cmad(cscale(y, su), pu, cscale(v[u], c));
            v[u ^ XR] = cmad(cscale(y, sw), pw, cscale(v[u ^ XR], c));
        }
    }
}

// kRegPauli record: matrices (cos, 0), y, out-of-tile Z-type mask (two exact halves).  A flip
// set of several register bits reduces to its lowest bit b: with the register permutation
// U = prod_j CX(b -> b_j) over the other flip bits, U P U has flip bits {b} and Z-type bits
// zr with b toggled once per b_j among them, so the kernel permutes, rotates on one bit and
// permutes back (4 + 4 code paths instead of one per flip set, which at 15 unrolled paths
// made the allocator spill over a kilobyte per thread).
__device__ __forceinline__ void reg_pauli(double2 (&v)[kE], uint32_t mat, uint32_t xr, uint32_t zr,
                                          uint32_t zt, uint32_t xl, uint64_t base) {
    const double c = lds2(mat).x;
    double2 y = lds2(mat + 16u);
    const double2 zd = lds2(mat + 32u);
    const uint64_t zg = static_cast<uint64_t>(zd.x) | (static_cast<uint64_t>(zd.y) << 32);
    if ((__popcll(base & zg) + __popc(threadIdx.x & zt)) & 1) y = make_double2(-y.x, -y.y);
    if (xl != 0 && xr == 0) {   // flips on lanes only
        reg_pauli_xl<0>(v, c, y, zr, xl);
        return;
    }
    if (xr == 0) {   // a Z-type string: the diagonal c + y s_u
        const double2 fp = make_double2(c + y.x, y.y), fm = make_double2(c - y.x, -y.y);
#pragma unroll
        for (int u = 0; u < kE; ++u)
            v[u] = cmul(v[u], (__popc(static_cast<uint32_t>(u) & zr) & 1u) ? fm : fp);
        return;
    }
    const uint32_t b = xr & (0u - xr), rest = xr & ~b;
    for (uint32_t r = rest; r; r &= r - 1) dispatch_swapx(v, r & (0u - r), b);
    const uint32_t zr1 = (__popc(zr & rest) & 1u) ? zr ^ b : zr;
    if (xl != 0) {
        switch (b) {
            case 1: reg_pauli_xl<1>(v, c, y, zr1, xl); break;
            case 2: reg_pauli_xl<2>(v, c, y, zr1, xl); break;
            case 4: reg_pauli_xl<4>(v, c, y, zr1, xl); break;
            default: reg_pauli_xl<8>(v, c, y, zr1, xl); break;
        }
    } else {
        switch (b) {
            case 1: reg_pauli_x<1>(v, c, y, zr1); break;
            case 2: reg_pauli_x<2>(v, c, y, zr1); break;
            case 4: reg_pauli_x<4>(v, c, y, zr1); break;
            default: reg_pauli_x<8>(v, c, y, zr1); break;
        }
    }
    for (uint32_t r = rest; r; r &= r - 1) dispatch_swapx(v, r & (0u - r), b);
}

__device__ __forceinline__ uint32_t thread_slot(const RegLayout& ly, uint32_t tbits) {
    uint32_t s = 0;
    for (uint32_t i = 0; i < tbits; ++i)
        if ((threadIdx.x >> i) & 1u) s ^= ly.tsw[i];
    return s;
}

__device__ __forceinline__ uint64_t thread_goff(const RegLayout& ly, uint32_t tbits,
                                                const uint64_t* gbit) {
    uint64_t g = 0;
    for (uint32_t i = 0; i < tbits; ++i)
        if ((threadIdx.x >> i) & 1u) g |= gbit[ly.tpos[i]];
    return g;
}

// MINB resident CTAs per SM: registers per thread <= 65536 / (MINB * threads).  FMAD: the
// pass has dense records on register bits (FP64 FMAs); MMA: it has tensor-path records.  A
// kernel carries only the paths its pass uses: with both, the register allocation spills
// (364 bytes at 128 registers against 64 for the FMA path alone and 8 for the tensor path
// alone), so each pass runs the variant of its own records.  PAULI: it has Pauli rotations.
template <int M, int MINB, bool FMAD, bool MMA, bool PAULI>
__global__ void __launch_bounds__(1 << (M - kRegBits), MINB)
k_regtile(double2* __restrict__ st, RegPass p, const RegOp* __restrict__ ops,
          const RegLayout* __restrict__ layouts, const double2* __restrict__ mats) {
    constexpr uint32_t kT = 1u << (M - kRegBits);
    constexpr uint32_t kTB = M - kRegBits;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* __restrict__ tile = reinterpret_cast<double2*>(smem);
    double2* smat = tile + (1u << M);
    RegOp* sops = reinterpret_cast<RegOp*>(smat + p.n_mat);
    RegLayout* slay = reinterpret_cast<RegLayout*>(sops + p.n_ops);
    // per-tile diagonal tables, two sets (tile parity) on a 16-byte boundary
    double2* sdyn = reinterpret_cast<double2*>(
        (reinterpret_cast<uintptr_t>(slay + p.n_layouts) + 15u) & ~uintptr_t{15});
    __shared__ uint64_t gbit[kRegMaxBits];    // global offset of each tile bit at the load
    __shared__ uint64_t sgbit[kRegMaxBits];   // and at the store (relabelled by SWAPs)
    __shared__ uint32_t shbits[kTileMaxHigh];
    __shared__ uint32_t sdynrec[kRegMaxDyn];
    // per-thread constants of every tile, computed once: the global offsets of the thread
    // bits at the load (layout 0) and at the store (the last layout), and each layout's
    // shared-memory slot of the thread (the first kRegSlotLayouts layouts); the register
    // bits' offsets are the same for every thread
    __shared__ uint64_t s_ldg[kT], s_stg[kT];
    __shared__ uint64_t s_ldr[kRegBits], s_str[kRegBits];
    __shared__ uint16_t s_tslot[kRegSlotLayouts * kT];
    if (threadIdx.x == 0) {
#pragma unroll
        for (uint32_t i = 0; i < kTileMaxHigh; ++i) shbits[i] = p.hbits[i];   // static indices
#pragma unroll
        for (uint32_t i = 0; i < kRegMaxDyn; ++i) sdynrec[i] = p.dyn_rec[i];
        for (uint32_t b = 0; b < M; ++b)
            gbit[b] = uint64_t{1} << (b < p.L ? b : shbits[b - p.L]);
        if (p.relabel) {
#pragma unroll
            for (uint32_t b = 0; b < kRegMaxBits; ++b)
                if (b < M) sgbit[b] = uint64_t{1} << p.store_qubit[b];
        }
    }
    const uint64_t* __restrict__ stbit = p.relabel ? sgbit : gbit;   // uniform
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(
            mats + static_cast<uint64_t>(blockIdx.y) * p.mat_stride);   // this state's matrices
        uint32_t* dst = reinterpret_cast<uint32_t*>(smat);
        for (uint32_t w = threadIdx.x; w < p.n_mat * 4u; w += kT) dst[w] = src[w];
        src = reinterpret_cast<const uint32_t*>(ops);
        dst = reinterpret_cast<uint32_t*>(sops);
        for (uint32_t w = threadIdx.x; w < p.n_ops * (sizeof(RegOp) / 4); w += kT) dst[w] = src[w];
        src = reinterpret_cast<const uint32_t*>(layouts);
        dst = reinterpret_cast<uint32_t*>(slay);
        for (uint32_t w = threadIdx.x; w < p.n_layouts * (sizeof(RegLayout) / 4); w += kT)
            dst[w] = src[w];
    }
    __syncthreads();
    {
        uint32_t last = 0;   // remaps are never skipped: the store layout is the last one's
        for (uint32_t o = 0; o < p.n_ops; ++o)
            if (sops[o].kind == kRegRemap) last = sops[o].code;
        s_ldg[threadIdx.x] = thread_goff(slay[0], kTB, gbit);
        s_stg[threadIdx.x] = thread_goff(slay[last], kTB, stbit);
        for (uint32_t l = 0; l < p.n_layouts && l < kRegSlotLayouts; ++l)
            s_tslot[l * kT + threadIdx.x] = static_cast<uint16_t>(thread_slot(slay[l], kTB));
        if (threadIdx.x < kRegBits) {
            s_ldr[threadIdx.x] = gbit[slay[0].rpos[threadIdx.x]];
            s_str[threadIdx.x] = stbit[slay[last].rpos[threadIdx.x]];
        }
    }
    __syncthreads();
    const bool slot_table = p.n_layouts <= kRegSlotLayouts;   // uniform
    const uint32_t smat_addr = static_cast<uint32_t>(__cvta_generic_to_shared(smat));
    const uint32_t sdyn_addr = static_cast<uint32_t>(__cvta_generic_to_shared(sdyn));
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    uint32_t parity = 0;
    for (uint64_t tid = blockIdx.x; tid < p.n_tiles; tid += gridDim.x, parity ^= 1u) {
        // a warp's shared-memory slots differ between layouts with different warp bits:
        // the previous tile's last remap must be done before this tile's first
        if (p.sync_tiles) __syncthreads();
        uint64_t base = tid << p.L;
        for (uint32_t i = 0; i < p.h; ++i) base = insert_zero_bit(base, shbits[i]);
        double2 v[kE];
        {
            const uint64_t g = base | s_ldg[threadIdx.x];
            const uint64_t g0 = s_ldr[0], g1 = s_ldr[1], g2 = s_ldr[2], g3 = s_ldr[3];
#pragma unroll
            for (int u = 0; u < kE; ++u)
                v[u] = __ldcs(s + (g | ((u & 1) ? g0 : 0) | ((u & 2) ? g1 : 0) | ((u & 4) ? g2 : 0) |
                                   ((u & 8) ? g3 : 0)));
        }
        // relabelled stores go to places other warps load: all loads before any store
        if (p.load_barrier) __syncthreads();
        // Start the HBM reads of this CTA's next tile into L2 while this one computes, so
        // its loads above hit L2 on the next iteration.  Thread r < 2^h takes the row of
        // high-bit pattern r: 2^L contiguous amplitudes, 16 B * 2^L from a 16 B boundary.
        if (threadIdx.x < (1u << p.h) && tid + gridDim.x < p.n_tiles) {
            uint64_t nb = (tid + gridDim.x) << p.L;
            for (uint32_t i = 0; i < p.h; ++i) {
                nb = insert_zero_bit(nb, shbits[i]);
                if ((threadIdx.x >> i) & 1u) nb |= uint64_t{1} << shbits[i];
            }
            const double2* row = s + nb;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(row), "r"(16u << p.L)
                         : "memory");
        }
        // Per-tile diagonals: entry e of table d is its base entry times every gated term
        // whose out-of-tile qubits are all 1 in this tile and whose entry bits e contains.
        // The barrier after the build also ends the use of the other parity's tables (every
        // warp has finished the previous tile), so the next tile may overwrite them.
        const uint32_t dyn_base = parity * p.dyn_entries;
        if (p.n_dyn) {
            for (uint32_t w = threadIdx.x; w < p.n_dyn * 64u; w += kT) {
                const RegOp& op = sops[sdynrec[w >> 6]];
                const uint32_t e = w & 63u;
                if (e >= (1u << op.k)) continue;
                const double2* src = smat + op.mat_off;
                double2 acc = src[e];
                const double2* term = src + (1u << op.k);
                for (uint32_t t = 0; t < op.nterm; ++t) {
                    const double2 meta = term[2 * t + 1];
                    const uint64_t hi = static_cast<uint64_t>(meta.y);
                    const uint64_t gc = static_cast<uint64_t>(meta.x) | ((hi >> 6) << 32);
                    const uint32_t em = static_cast<uint32_t>(hi & 63u);
                    if ((base & gc) == gc && (e & em) == em) acc = cmul(term[2 * t], acc);
                }
                sdyn[dyn_base + op.dyn_off + e] = acc;
            }
            __syncthreads();
        }
        uint32_t cur = 0;
        for (uint32_t o = 0; o < p.n_ops; ++o) {
            const RegOp& op = sops[o];
            if ((base & op.gcmask) != op.gcmask) continue;   // uniform across the CTA
            const uint32_t kind = op.kind;
            if (kind == kRegRemap) {
                {
                    const RegLayout& ly = slay[cur];
                    const uint32_t ts = slot_table ? s_tslot[cur * kT + threadIdx.x]
                                                   : thread_slot(ly, kTB);
                    const uint32_t r0 = ly.rsw[0], r1 = ly.rsw[1], r2 = ly.rsw[2], r3 = ly.rsw[3];
#pragma unroll
                    for (int u = 0; u < kE; ++u)
                        tile[ts ^ ((u & 1) ? r0 : 0) ^ ((u & 2) ? r1 : 0) ^ ((u & 4) ? r2 : 0) ^
                             ((u & 8) ? r3 : 0)] = v[u];
                }
                cur = op.code;
                const bool local = op.k != 0;   // uniform: warp bits unchanged
                if (local) __syncwarp();
                else __syncthreads();
                {
                    const RegLayout& ly = slay[cur];
                    const uint32_t ts = slot_table ? s_tslot[cur * kT + threadIdx.x]
                                                   : thread_slot(ly, kTB);
                    const uint32_t r0 = ly.rsw[0], r1 = ly.rsw[1], r2 = ly.rsw[2], r3 = ly.rsw[3];
#pragma unroll
                    for (int u = 0; u < kE; ++u)
                        v[u] = tile[ts ^ ((u & 1) ? r0 : 0) ^ ((u & 2) ? r1 : 0) ^
                                    ((u & 4) ? r2 : 0) ^ ((u & 8) ? r3 : 0)];
                }
                if (local) __syncwarp();
                else __syncthreads();
                continue;
            }
            const uint32_t tc = op.tcmask;
            uint32_t moff = op.mat_off;
            if (const uint32_t nsel = op.nsel) {   // matrix picked by the tile's selector bits
                uint32_t sel = 0;
                for (uint32_t i = 0; i < nsel; ++i)
                    sel |= static_cast<uint32_t>((base >> op.selq[i]) & 1u) << i;
                const uint32_t k2 = kind == kRegDense || kind == kRegMma ? 2u * op.k : op.k;
                moff += sel << k2;
            }
            if (kind == kRegMma) {
                if constexpr (MMA) {
                    // controls on warp bits only: the condition is the same on every lane
                    if ((threadIdx.x & tc & ~31u) != (tc & ~31u)) continue;
                    __syncwarp();
                    reg_mma(v, smat_addr + 16u * moff, op.rcmask);
                }
                continue;
            }
            if (kind == kRegPauli) {   // rcmask / tcmask: its Z-type bits, not controls
                if constexpr (PAULI)
                    reg_pauli(v, smat_addr + 16u * moff, op.code, op.rcmask, tc, op.loc[0], base);
                continue;
            }
            if ((threadIdx.x & tc) != tc) continue;
            const uint32_t rc = op.rcmask;
            const uint32_t mat = kind == kRegDiagDyn ? sdyn_addr + 16u * (dyn_base + op.dyn_off)
                                                     : smat_addr + 16u * moff;
            if (kind == kRegDense) {
                if constexpr (FMAD) dispatch_dense(v, op.code, SharedMat{mat}, rc);
            } else if (kind == kRegPhase) {
                const double2 f = lds2(mat);
#pragma unroll
                for (int u = 0; u < kE; ++u)
                    if ((u & rc) == rc) v[u] = cmul(f, v[u]);
            } else if (kind == kRegSwapX) {
                dispatch_swapx(v, op.code, rc);
            } else {
                reg_diag(v, op, SharedMat{mat}, rc);
            }
        }
        {
            const uint64_t g = base | s_stg[threadIdx.x];
            const uint64_t g0 = s_str[0], g1 = s_str[1], g2 = s_str[2], g3 = s_str[3];
#pragma unroll
            for (int u = 0; u < kE; ++u)
                __stcs(s + (g | ((u & 1) ? g0 : 0) | ((u & 2) ? g1 : 0) | ((u & 4) ? g2 : 0) |
                            ((u & 8) ? g3 : 0)),
                       v[u]);
        }
    }
}

// ------------------------------------------------------------------ double-buffered passes
//
// The same pass with the next tile's HBM read overlapped with this tile's compute: each
// thread issues cp.async copies of 16 of the next tile's amplitudes into the second of two
// shared tile buffers while the CTA works on the first, and waits for them only when it
// reaches that tile.  The tile arrives in shared memory in linear order (position q of the
// tile at index q; thread t copies positions j * T + t, so a warp's copy is one coalesced
// 512-byte row), is read into registers through layout 0, and the same buffer then serves
// the remaps (swizzled slots).  One barrier per tile makes the copies visible, ends every
// warp's use of the previous tile's buffer (which the next copies overwrite) and publishes
// the per-tile diagonal tables.

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <int M, int MINB>
__global__ void __launch_bounds__(1 << (M - kRegBits), MINB)
k_regtile_pipe(double2* __restrict__ st, RegPass p, const RegOp* __restrict__ ops,
               const RegLayout* __restrict__ layouts, const double2* __restrict__ mats) {
    constexpr uint32_t kT = 1u << (M - kRegBits);
    constexpr uint32_t kTB = M - kRegBits;
    constexpr uint32_t kN = 1u << M;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* bufs = reinterpret_cast<double2*>(smem);   // two tiles
    double2* smat = bufs + 2 * kN;
    RegOp* sops = reinterpret_cast<RegOp*>(smat + p.n_mat);
    RegLayout* slay = reinterpret_cast<RegLayout*>(sops + p.n_ops);
    double2* sdyn = reinterpret_cast<double2*>(
        (reinterpret_cast<uintptr_t>(slay + p.n_layouts) + 15u) & ~uintptr_t{15});
    __shared__ uint64_t gbit[kRegMaxBits];
    __shared__ uint64_t sgbit[kRegMaxBits];
    __shared__ uint32_t shbits[kTileMaxHigh];
    __shared__ uint32_t sdynrec[kRegMaxDyn];
    // per-thread constants of every tile, computed once: the global offsets of the thread
    // bits at the load (layout 0) and at the store (the last layout), and each layout's
    // shared-memory slot of the thread (the first kRegSlotLayouts layouts); the register
    // bits' offsets are the same for every thread
    __shared__ uint64_t s_ldg[kT], s_stg[kT];
    __shared__ uint64_t s_ldr[kRegBits], s_str[kRegBits];
    __shared__ uint16_t s_tslot[kRegSlotLayouts * kT];
    if (threadIdx.x == 0) {
#pragma unroll
        for (uint32_t i = 0; i < kTileMaxHigh; ++i) shbits[i] = p.hbits[i];
#pragma unroll
        for (uint32_t i = 0; i < kRegMaxDyn; ++i) sdynrec[i] = p.dyn_rec[i];
        for (uint32_t b = 0; b < M; ++b)
            gbit[b] = uint64_t{1} << (b < p.L ? b : shbits[b - p.L]);
        if (p.relabel) {
#pragma unroll
            for (uint32_t b = 0; b < kRegMaxBits; ++b)
                if (b < M) sgbit[b] = uint64_t{1} << p.store_qubit[b];
        }
    }
    const uint64_t* __restrict__ stbit = p.relabel ? sgbit : gbit;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(
            mats + static_cast<uint64_t>(blockIdx.y) * p.mat_stride);
        uint32_t* dst = reinterpret_cast<uint32_t*>(smat);
        for (uint32_t w = threadIdx.x; w < p.n_mat * 4u; w += kT) dst[w] = src[w];
        src = reinterpret_cast<const uint32_t*>(ops);
        dst = reinterpret_cast<uint32_t*>(sops);
        for (uint32_t w = threadIdx.x; w < p.n_ops * (sizeof(RegOp) / 4); w += kT) dst[w] = src[w];
        src = reinterpret_cast<const uint32_t*>(layouts);
        dst = reinterpret_cast<uint32_t*>(slay);
        for (uint32_t w = threadIdx.x; w < p.n_layouts * (sizeof(RegLayout) / 4); w += kT)
            dst[w] = src[w];
    }
    __syncthreads();
    {
        uint32_t last = 0;   // remaps are never skipped: the store layout is the last one's
        for (uint32_t o = 0; o < p.n_ops; ++o)
            if (sops[o].kind == kRegRemap) last = sops[o].code;
        s_ldg[threadIdx.x] = thread_goff(slay[0], kTB, gbit);
        s_stg[threadIdx.x] = thread_goff(slay[last], kTB, stbit);
        for (uint32_t l = 0; l < p.n_layouts && l < kRegSlotLayouts; ++l)
            s_tslot[l * kT + threadIdx.x] = static_cast<uint16_t>(thread_slot(slay[l], kTB));
        if (threadIdx.x < kRegBits) {
            s_ldr[threadIdx.x] = gbit[slay[0].rpos[threadIdx.x]];
            s_str[threadIdx.x] = stbit[slay[last].rpos[threadIdx.x]];
        }
    }
    __syncthreads();
    const bool slot_table = p.n_layouts <= kRegSlotLayouts;   // uniform
    const uint32_t smat_addr = static_cast<uint32_t>(__cvta_generic_to_shared(smat));
    const uint32_t sdyn_addr = static_cast<uint32_t>(__cvta_generic_to_shared(sdyn));
    const uint32_t bufs_addr = static_cast<uint32_t>(__cvta_generic_to_shared(bufs));
    double2* __restrict__ s = st + static_cast<uint64_t>(blockIdx.y) * p.batch_stride;
    // copy positions q = j * kT + t: tile bits 0..kTB-1 from t, the 4 above from j
    uint64_t toff = 0;
    for (uint32_t b = 0; b < kTB; ++b)
        if ((threadIdx.x >> b) & 1u) toff |= gbit[b];
    const uint64_t jb0 = gbit[kTB], jb1 = gbit[kTB + 1], jb2 = gbit[kTB + 2], jb3 = gbit[kTB + 3];
    auto tile_base = [&](uint64_t tile) {
        uint64_t b = tile << p.L;
        for (uint32_t i = 0; i < p.h; ++i) b = insert_zero_bit(b, shbits[i]);
        return b;
    };
    auto issue = [&](uint64_t tile, uint32_t which) {
        const uint64_t g = tile_base(tile) | toff;
        const uint32_t dst = bufs_addr + 16u * (which * kN + threadIdx.x);
#pragma unroll
        for (int j = 0; j < kE; ++j)
            cp_async16(dst + 16u * kT * j, s + (g | ((j & 1) ? jb0 : 0) | ((j & 2) ? jb1 : 0) |
                                               ((j & 4) ? jb2 : 0) | ((j & 8) ? jb3 : 0)));
        cp_async_commit();
    };
    if (blockIdx.x < p.n_tiles) issue(blockIdx.x, 0);
    uint32_t parity = 0;
    for (uint64_t tid = blockIdx.x; tid < p.n_tiles; tid += gridDim.x, parity ^= 1u) {
        const uint64_t base = tile_base(tid);
        // this tile's diagonal tables: their parity's previous user (two tiles back) is done,
        // since every warp passed the previous tile's barrier
        const uint32_t dyn_base = parity * p.dyn_entries;
        if (p.n_dyn) {
            for (uint32_t w = threadIdx.x; w < p.n_dyn * 64u; w += kT) {
                const RegOp& op = sops[sdynrec[w >> 6]];
                const uint32_t e = w & 63u;
                if (e >= (1u << op.k)) continue;
                const double2* src = smat + op.mat_off;
                double2 acc = src[e];
                const double2* term = src + (1u << op.k);
                for (uint32_t t = 0; t < op.nterm; ++t) {
                    const double2 meta = term[2 * t + 1];
                    const uint64_t hi = static_cast<uint64_t>(meta.y);
                    const uint64_t gc = static_cast<uint64_t>(meta.x) | ((hi >> 6) << 32);
                    const uint32_t em = static_cast<uint32_t>(hi & 63u);
                    if ((base & gc) == gc && (e & em) == em) acc = cmul(term[2 * t], acc);
                }
                sdyn[dyn_base + op.dyn_off + e] = acc;
            }
        }
        cp_async_wait_all();
        __syncthreads();
        if (tid + gridDim.x < p.n_tiles) issue(tid + gridDim.x, parity ^ 1u);
        double2* __restrict__ tile = bufs + parity * kN;
        double2 v[kE];
        {
            const RegLayout& ly = slay[0];
            uint32_t tp = 0;
            for (uint32_t i = 0; i < kTB; ++i)
                if ((threadIdx.x >> i) & 1u) tp |= 1u << ly.tpos[i];
            const uint32_t p0 = 1u << ly.rpos[0], p1 = 1u << ly.rpos[1], p2 = 1u << ly.rpos[2],
                           p3 = 1u << ly.rpos[3];
#pragma unroll
            for (int u = 0; u < kE; ++u)
                v[u] = tile[tp | ((u & 1) ? p0 : 0) | ((u & 2) ? p1 : 0) | ((u & 4) ? p2 : 0) |
                            ((u & 8) ? p3 : 0)];
        }
        __syncwarp();   // every lane's linear read before any lane's first remap write
        uint32_t cur = 0;
        for (uint32_t o = 0; o < p.n_ops; ++o) {
            const RegOp& op = sops[o];
            if ((base & op.gcmask) != op.gcmask) continue;
            const uint32_t kind = op.kind;
            if (kind == kRegRemap) {
                {
                    const RegLayout& ly = slay[cur];
                    const uint32_t ts = slot_table ? s_tslot[cur * kT + threadIdx.x]
                                                   : thread_slot(ly, kTB);
                    const uint32_t r0 = ly.rsw[0], r1 = ly.rsw[1], r2 = ly.rsw[2], r3 = ly.rsw[3];
#pragma unroll
                    for (int u = 0; u < kE; ++u)
                        tile[ts ^ ((u & 1) ? r0 : 0) ^ ((u & 2) ? r1 : 0) ^ ((u & 4) ? r2 : 0) ^
                             ((u & 8) ? r3 : 0)] = v[u];
                }
                cur = op.code;
                const bool local = op.k != 0;
                if (local) __syncwarp();
                else __syncthreads();
                {
                    const RegLayout& ly = slay[cur];
                    const uint32_t ts = slot_table ? s_tslot[cur * kT + threadIdx.x]
                                                   : thread_slot(ly, kTB);
                    const uint32_t r0 = ly.rsw[0], r1 = ly.rsw[1], r2 = ly.rsw[2], r3 = ly.rsw[3];
#pragma unroll
                    for (int u = 0; u < kE; ++u)
                        v[u] = tile[ts ^ ((u & 1) ? r0 : 0) ^ ((u & 2) ? r1 : 0) ^
                                    ((u & 4) ? r2 : 0) ^ ((u & 8) ? r3 : 0)];
                }
                if (local) __syncwarp();
                else __syncthreads();
                continue;
            }
            const uint32_t tc = op.tcmask;
            uint32_t moff = op.mat_off;
            if (const uint32_t nsel = op.nsel) {
                uint32_t sel = 0;
                for (uint32_t i = 0; i < nsel; ++i)
                    sel |= static_cast<uint32_t>((base >> op.selq[i]) & 1u) << i;
                const uint32_t k2 = kind == kRegDense || kind == kRegMma ? 2u * op.k : op.k;
                moff += sel << k2;
            }
            if (kind == kRegMma) {
                if ((threadIdx.x & tc & ~31u) != (tc & ~31u)) continue;   // uniform per warp
                __syncwarp();
                reg_mma(v, smat_addr + 16u * moff, op.rcmask);
                continue;
            }
            if (kind == kRegPauli) {
                reg_pauli(v, smat_addr + 16u * moff, op.code, op.rcmask, tc, op.loc[0], base);
                continue;
            }
            if ((threadIdx.x & tc) != tc) continue;
            const uint32_t rc = op.rcmask;
            const uint32_t mat = kind == kRegDiagDyn ? sdyn_addr + 16u * (dyn_base + op.dyn_off)
                                                     : smat_addr + 16u * moff;
            if (kind == kRegDense) {
                dispatch_dense(v, op.code, SharedMat{mat}, rc);
            } else if (kind == kRegPhase) {
                const double2 f = lds2(mat);
#pragma unroll
                for (int u = 0; u < kE; ++u)
                    if ((u & rc) == rc) v[u] = cmul(f, v[u]);
            } else if (kind == kRegSwapX) {
                dispatch_swapx(v, op.code, rc);
            } else {
                reg_diag(v, op, SharedMat{mat}, rc);
            }
        }
        {
            const uint64_t g = base | s_stg[threadIdx.x];
            const uint64_t g0 = s_str[0], g1 = s_str[1], g2 = s_str[2], g3 = s_str[3];
#pragma unroll
            for (int u = 0; u < kE; ++u)
                __stcs(s + (g | ((u & 1) ? g0 : 0) | ((u & 2) ? g1 : 0) | ((u & 4) ? g2 : 0) |
                            ((u & 8) ? g3 : 0)),
                       v[u]);
        }
    }
    cp_async_wait_all();
}

template <int M, int MINB>
void launch_pipe(const LaunchCtx& ctx, double2* st, uint32_t batch, const RegPass& p, size_t smem,
                 const RegOp* d_ops, const RegLayout* d_layouts, const double2* d_mats) {
    constexpr uint32_t kT = 1u << (M - kRegBits);
    auto kern = k_regtile_pipe<M, MINB>;
    cuda_check_launch_attr(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(kRegPipeMaxSmem)));
    const uint32_t by_smem = static_cast<uint32_t>(std::max<size_t>(1, (227 * 1024) / (smem + 1024)));
    const uint64_t want = static_cast<uint64_t>(ctx.num_sms) * std::min<uint32_t>(MINB, by_smem);
    const uint32_t grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(want, p.n_tiles)));
    kern<<<dim3(grid, batch), kT, smem, ctx.stream>>>(st, p, d_ops, d_layouts, d_mats);
    check_launch("register tile pass (double-buffered)");
}

template <int M, int MINB, bool FMAD, bool MMA, bool PAULI>
void launch_mbf(const LaunchCtx& ctx, double2* st, uint32_t batch, const RegPass& p, size_t smem,
                const RegOp* d_ops, const RegLayout* d_layouts, const double2* d_mats) {
    constexpr uint32_t kT = 1u << (M - kRegBits);
    auto kern = k_regtile<M, MINB, FMAD, MMA, PAULI>;
    cuda_check_launch_attr(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(kTileMaxSmem)));
    static const size_t static_smem = [&] {
        cudaFuncAttributes a{};
        cuda_check_launch_attr(cudaFuncGetAttributes(&a, kern));
        return a.sharedSizeBytes;
    }();
    const uint32_t by_smem = static_cast<uint32_t>(
        std::max<size_t>(1, (227 * 1024) / (smem + static_smem + 1024)));
    const uint64_t want = static_cast<uint64_t>(ctx.num_sms) * std::min<uint32_t>(MINB, by_smem);
    const uint32_t grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(want, p.n_tiles)));
    kern<<<dim3(grid, batch), kT, smem, ctx.stream>>>(st, p, d_ops, d_layouts, d_mats);
    check_launch("register tile pass");
}

template <int M, int MINB>
void launch_mb(const LaunchCtx& ctx, double2* st, uint32_t batch, const RegPass& p, size_t smem,
               const RegOp* d_ops, const RegLayout* d_layouts, const double2* d_mats) {
    // four variants: FMA, FMA + Pauli, tensor path, all
    if (!p.mma_ops) {
        if (p.pauli_ops) launch_mbf<M, MINB, true, false, true>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
        else launch_mbf<M, MINB, true, false, false>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
    } else if (!p.fma_dense && !p.pauli_ops) {
        launch_mbf<M, MINB, false, true, false>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
    } else {
        launch_mbf<M, MINB, true, true, true>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
    }
}

// Residency per tile size: about 160 registers per thread keep the dense paths free of
// spills, so M <= 11 run 168-register CTAs (12 warps per SM).  M = 12 runs two CTAs of 128
// registers (a few spilled values; measured faster than one 160-register CTA, which
// LQCS_TILE_OCC=1 selects); M = 13 (512 threads) is capped at 128.
template <int M>
void launch_m(const LaunchCtx& ctx, double2* st, uint32_t batch, const RegPass& p, size_t smem,
              const RegOp* d_ops, const RegLayout* d_layouts, const double2* d_mats) {
    if constexpr (M == 12) {
        static const int occ = [] {
            const char* e = std::getenv("LQCS_TILE_OCC");
            return e ? std::atoi(e) : 2;
        }();
        if (occ >= 2) {
            launch_mb<12, 2>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
            return;
        }
        launch_mb<12, 1>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
    } else if constexpr (M == 13) {
        launch_mb<13, 1>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
    } else if constexpr (M == 11) {
        // three 168-register CTAs per SM by default; LQCS_TILE_OCC=4: four of 128 registers
        static const int occ = [] {
            const char* e = std::getenv("LQCS_TILE_OCC");
            return e ? std::atoi(e) : 3;
        }();
        if (occ >= 4) {
            launch_mb<11, 4>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
            return;
        }
        launch_mb<11, 3>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
    } else {
        constexpr int kMinB = 65536 / ((1 << (M - kRegBits)) * 168);
        launch_mb<M, kMinB>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats);
    }
}

}  // namespace

size_t reg_smem_bytes(const RegPass& pass, uint32_t tiles) {
    const size_t records = sizeof(double2) * ((size_t{tiles} << pass.m) + pass.n_mat) +
                           sizeof(RegOp) * pass.n_ops + sizeof(RegLayout) * pass.n_layouts;
    return pass.n_dyn ? ((records + 15) & ~size_t{15}) + sizeof(double2) * 2 * pass.dyn_entries
                      : records;
}

bool reg_pipe_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("LQCS_REG_PIPE");
        return e != nullptr && std::atoi(e) != 0;
    }();
    return on;
}

void launch_reg_pass(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                     const RegPass& pass, const RegOp* d_ops, const RegLayout* d_layouts,
                     const double2* d_mats) {
    RegPass p = pass;
    p.batch_stride = uint64_t{1} << n;
    p.n_tiles = (uint64_t{1} << n) >> p.m;
    if (reg_pipe_enabled() && (p.m == 11 || p.m == 12)) {
        const size_t smem2 = reg_smem_bytes(p, 2);
        if (smem2 <= kRegPipeMaxSmem && p.n_ops <= kRegMaxRecords && p.n_mat <= kRegMaxMatrix &&
            p.n_dyn <= kRegMaxDyn && p.dyn_entries <= kRegMaxDynEntries && p.n_layouts >= 1 &&
            p.h <= kTileMaxHigh) {
            if (p.m == 12) launch_pipe<12, 1>(ctx, st, batch, p, smem2, d_ops, d_layouts, d_mats);
            else launch_pipe<11, 3>(ctx, st, batch, p, smem2, d_ops, d_layouts, d_mats);
            return;
        }
    }
    const size_t smem = reg_smem_bytes(p);
    if (smem > kTileMaxSmem || p.m < kRegMinBits || p.m > kRegMaxBits || p.h > kTileMaxHigh ||
        p.n_layouts < 1 || p.n_ops > kRegMaxRecords || p.n_mat > kRegMaxMatrix ||
        p.n_dyn > kRegMaxDyn || p.dyn_entries > kRegMaxDynEntries)
        throw std::logic_error("register tile pass: unsupported shape");
    switch (p.m) {
        case 9: launch_m<9>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats); break;
        case 10: launch_m<10>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats); break;
        case 11: launch_m<11>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats); break;
        case 12: launch_m<12>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats); break;
        default: launch_m<13>(ctx, st, batch, p, smem, d_ops, d_layouts, d_mats); break;
    }
}

}  // namespace lqcs_b200
