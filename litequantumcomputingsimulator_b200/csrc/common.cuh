// common.cuh — device helpers shared by the statevector kernels.
//
// Amplitudes are complex128 stored as double2 (x = re, y = im), qubit 0 = least
// significant bit of the basis index (the layout of lqcs::Statevector,
// include/lqcs/backend/statevector.hpp:12-37).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lqcs_b200 {

constexpr int kMaxQubits = 40;     // index arithmetic bound (device memory caps far lower)
constexpr int kMaxDense = 6;       // widest dense block (2^6 x 2^6)
constexpr int kWarp = 32;

__host__ __device__ __forceinline__ uint64_t insert_zero_bit(uint64_t v, unsigned pos) {
    const uint64_t low = (uint64_t{1} << pos) - 1;
    return ((v & ~low) << 1) | (v & low);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc + a*b
__device__ __forceinline__ double2 cmad(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) {
    return make_double2(a.x * s, a.y * s);
}
// |a|^2 rounded as re*re + im*im with two separately rounded products (no FMA), the
// evaluation libstdc++'s std::norm gives on x86-64; keeps prefix sums close to the
// reference's for shot sampling.
__device__ __forceinline__ double norm_rn(double2 a) {
    return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
}

__device__ __forceinline__ double2 shfl_xor_d2(double2 v, int mask) {
    v.x = __shfl_xor_sync(0xffffffffu, v.x, mask);
    v.y = __shfl_xor_sync(0xffffffffu, v.y, mask);
    return v;
}
__device__ __forceinline__ double2 shfl_d2(double2 v, int src) {
    v.x = __shfl_sync(0xffffffffu, v.x, src);
    v.y = __shfl_sync(0xffffffffu, v.y, src);
    return v;
}

// Read-only streaming load of one amplitude (16 B, one 128-bit transaction).
__device__ __forceinline__ double2 ld_amp(const double2* p) { return __ldg(p); }

// Sorted list of bit positions that an enumeration inserts as zeros.
struct BitList {
    uint32_t n;
    uint32_t pos[kMaxQubits];
};

__device__ __forceinline__ uint64_t expand_bits(uint64_t g, const BitList& bl) {
#pragma unroll 1
    for (uint32_t i = 0; i < bl.n; ++i) g = insert_zero_bit(g, bl.pos[i]);
    return g;
}

}  // namespace lqcs_b200
