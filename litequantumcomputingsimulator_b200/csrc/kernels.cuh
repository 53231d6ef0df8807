// kernels.cuh — parameter blocks and host launchers of the sm_100a statevector kernels.
//
// Every launcher enqueues on ctx.stream and never synchronises.  A state "batch" is
// `batch` states of 2^n amplitudes laid out back to back; a launcher applies the same
// operation to each (gridDim.y walks the batch).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace lqcs_b200 {

struct LaunchCtx {
    cudaStream_t stream = nullptr;
    int num_sms = 148;
};

// Counts kernels launched through these launchers (all devices).
uint64_t launch_count();
void count_launch(uint64_t n = 1);

// ---------------------------------------------------------------- gate application

// One-qubit 2x2 (dense or diagonal) on target t, restricted to the subspace where every
// control bit is 1.  Requires n >= 5.
struct Apply1QOp {
    double2 m[4];      // row-major
    uint32_t t;
    uint64_t cmask;    // all control bits
    int diag;          // m[1] == m[2] == 0: multiply by m[0] / m[3]
};
void launch_apply_1q(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                     const Apply1QOp& op);

// Multiply every amplitude whose bits in `mask` are all 1 by `ph` (T, S, Z, P, CZ, CP,
// MCP, ...).  Requires n >= 5.
void launch_phase(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                  uint64_t mask, double2 ph);

// Dense 2^k x 2^k matrix (row-major, device memory, local bit j <-> targets[j]) on
// the subspace where every control bit is 1.  1 <= k <= kMaxDense, any n >= k + nc.
void launch_dense(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                  const uint32_t* targets, uint32_t k, uint64_t cmask,
                  const double2* d_mat);
// The same on the FP64 tensor path (mma.sync.m8n8k4.f64, dense_mma_kernels.cu), k = 4..6;
// launch_dense routes there where dense_mma_enabled(k) (LQCS_DENSE_MMA overrides).
bool dense_mma_enabled(uint32_t k);
void launch_dense_mma(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                      const uint32_t* targets, uint32_t k, uint64_t cmask, const double2* d_mat);

// Diagonal k-qubit operator: amp *= diag[local index] (local bit j <-> targets[j]),
// on the subspace where every control bit is 1.  Device memory diag of 2^k entries.
void launch_diag(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                 const uint32_t* targets, uint32_t k, uint64_t cmask,
                 const double2* d_diag);

// Controlled permutation |l> -> |perm[l]> as cycles.  cycles: flattened local indices,
// cycle_len: lengths (each >= 2).  Device memory.
void launch_perm(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                 const uint32_t* targets, uint32_t k, uint64_t cmask,
                 const uint32_t* d_cycles, const uint32_t* d_cycle_len,
                 uint32_t n_cycles, uint32_t total_len);

// exp(-i theta/2 P) for a Pauli string given by global masks (x = X/Y bits, zy = Z/Y bits,
// n_y = number of Y).  cos_h = cos(theta/2), sin_h = sin(theta/2).  Requires n >= 5.
void launch_pauli_rotation(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                           uint64_t x, uint64_t zy, uint32_t n_y, double cos_h, double sin_h);

// Batched Pauli rotation with one angle per state: cos_sin[b] = (cos, sin) of theta_b/2.
void launch_pauli_rotation_batched(const LaunchCtx& ctx, double2* st, uint32_t n,
                                   uint32_t batch, uint64_t x, uint64_t zy, uint32_t n_y,
                                   const double2* d_cos_sin);

// ---------------------------------------------------------------- state utilities

void launch_set_basis(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                      uint64_t index);
void launch_scale(const LaunchCtx& ctx, double2* st, uint64_t count, double s);
// out[i] = a[i] + alpha * b[i]
void launch_axpy(const LaunchCtx& ctx, double2* out, const double2* b, double2 alpha,
                 uint64_t count);

// ---------------------------------------------------------------- reductions
// All reductions are deterministic: fixed grid, fixed per-thread order, fixed tree.
// `partials` is device scratch of (kMaxReduceBlocks + 1) doubles per output value.

uint32_t reduce_grid(const LaunchCtx& ctx, uint64_t work_items);
constexpr uint32_t kReduceThreads = 256;
constexpr uint32_t kMaxReduceBlocks = 2048;

// sum |amp|^2 over the whole state -> d_out[0]
void launch_norm2(const LaunchCtx& ctx, const double2* st, uint32_t n, double* d_partials,
                  double* d_out);
// sum |amp|^2 over amplitudes with bit q == 1 -> d_out[0]
void launch_bitprob(const LaunchCtx& ctx, const double2* st, uint32_t n, uint32_t q,
                    double* d_partials, double* d_out);
// 2x2 reduced density matrix of qubit q: d_out = {rho00, rho11, re rho01, im rho01}
void launch_rdm1(const LaunchCtx& ctx, const double2* st, uint32_t n, uint32_t q,
                 double* d_partials, double* d_out);
// sum_pairs ||K (a0, a1)||^2 -> d_out[0]
void launch_kraus_prob(const LaunchCtx& ctx, const double2* st, uint32_t n, uint32_t q,
                       const double2 k[4], double* d_partials, double* d_out);
// Pauli expectation: d_out[t] = Re(i^{n_y[t]} sum_i sign_t(i) a_i conj(a_{i^x})) for
// n_terms terms that share the x mask (zy, n_y: host arrays of n_terms entries).
// n_terms <= kMaxTermsPerPass; d_partials holds (kMaxReduceBlocks + 1) * 16 doubles.
constexpr uint32_t kMaxTermsPerPass = 8;
void launch_expect_xgroup(const LaunchCtx& ctx, const double2* st, uint32_t n, uint64_t x,
                          const uint64_t* zy, const uint32_t* n_y, uint32_t n_terms,
                          double* d_partials, double* d_out);
// probabilities p[i] = |a_i|^2 (rounded like std::norm)
void launch_probabilities(const LaunchCtx& ctx, const double2* st, uint32_t n, double* d_p);

// Sampling by inclusive prefix sum of |a_i|^2 and upper_bound per shot.  The scan stores
// per-chunk prefixes in d_tpref (scan_thread_count(n) doubles) and per-segment prefixes in
// d_block (scan_block_count(n) doubles); the search evaluates prefix values from them and the
// state, so the 2^n-entry prefix array is never materialised.
uint64_t scan_block_count(uint32_t n);
uint64_t scan_thread_count(uint32_t n);
void launch_prob_scan(const LaunchCtx& ctx, const double2* st, uint32_t n, double* d_tpref,
                      double* d_block);
// upper_bound(cum, u_s * cum[N-1]) per shot; d_margin[s] = distance to the nearest edge / total
void launch_sample_search(const LaunchCtx& ctx, const double2* st, uint32_t n,
                          const double* d_tpref, const double* d_block, const double* d_u,
                          uint64_t shots, uint64_t* d_idx, double* d_margin);
// The same over the diagonal rho_ii of an n-qubit density matrix held as a 2n-qubit vector
// (element (col << n) | row), and the diagonal itself (2^n doubles).
void launch_dm_diag_scan(const LaunchCtx& ctx, const double2* rho, uint32_t n, double* d_tpref,
                         double* d_block);
void launch_dm_sample_search(const LaunchCtx& ctx, const double2* rho, uint32_t n,
                             const double* d_tpref, const double* d_block, const double* d_u,
                             uint64_t shots, uint64_t* d_idx, double* d_margin);
void launch_dm_diagonal(const LaunchCtx& ctx, const double2* rho, uint32_t n, double* d_p);

// collapse: amplitudes with bit q == outcome scaled by `scale`, the others zeroed
void launch_project(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t q, int outcome,
                    double scale);
// reset tail: move the bit q == 1 half into bit q == 0, zero the bit q == 1 half
void launch_move_to_zero(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t q);

// ---------------------------------------------------------------- Hamiltonian
// out = sum_t c_t P_t in (per state of a batch); terms in device memory.
struct PauliTermDev {
    uint64_t x;
    uint64_t zy;
    double2 coeff;   // c_t * i^{n_y}
};
// Tile bits of the Hamiltonian apply.  Its terms come grouped by x >> ham_tile_bits(n) (the
// groups in any order, terms of a group contiguous); d_groups = {G, G group keys, G + 1 term
// offsets}.  HamiltonianDev builds both.
uint32_t ham_tile_bits(uint32_t n);
void launch_apply_hamiltonian(const LaunchCtx& ctx, const double2* in, double2* out,
                              uint32_t n, uint32_t batch, const PauliTermDev* d_terms,
                              const uint32_t* d_groups);
// ---------------------------------------------------------------- rotation tile passes
// A run of Pauli rotations applied to tiles of 2^m amplitudes in shared memory: local bit
// j < L is qubit j, local bit L + i is qubit hbits[i] (ascending).  Every rotation's X mask
// lies in the tile; its Z / Y bits outside the tile give a sign that is uniform per tile.
constexpr uint32_t kRotThreads = 256;
constexpr uint32_t kRotMaxBits = 12;
constexpr uint32_t kRotMaxHigh = 16;
constexpr uint32_t kRotMaxOps = 64;   // rotations per pass (staged in shared memory)
constexpr uint32_t kRotMaxRows = (1u << kRotMaxBits) / kRotThreads;
struct RotTileOp {
    uint64_t zy_out;   // Z / Y bits outside the tile
    uint32_t x_loc;    // X / Y bits, tile-local (0: diagonal rotation)
    uint32_t zy_loc;   // Z / Y bits, tile-local
    uint32_t param;    // row of the (cos, sin) of theta/2 table ([param][state])
    uint32_t n_y;
    uint32_t pad[2];
};
struct RotTilePass {
    uint32_t m, L, h, n_ops;
    uint32_t hbits[kRotMaxHigh];
};
size_t rot_tile_smem(uint32_t m, bool backward);
void launch_rot_tile_fwd(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t nb,
                         const RotTilePass& p, const RotTileOp* d_ops, const double2* d_cs,
                         uint32_t R);
// Backward pass: per rotation (in the order given) d_grad[state * np + param] =
// Im<lambda|P|psi> before the rotation is undone on psi and lambda.  d_partials holds
// n_ops * nb * 2^(n - m) doubles.
void launch_rot_tile_bwd(const LaunchCtx& ctx, double2* psi, double2* lam, uint32_t n,
                         uint32_t nb, const RotTilePass& p, const RotTileOp* d_ops,
                         const double2* d_cs, uint32_t R, double* d_partials, double* d_grad,
                         uint64_t np);
void cuda_check_launch_attr(cudaError_t e);

// Per-state Re<a|b> -> d_out[b] for a batch of states.  d_partials holds at least
// batch * 64 doubles.
void launch_batched_inner_re_p(const LaunchCtx& ctx, const double2* a, const double2* b,
                               uint32_t n, uint32_t batch, double* d_partials, double* d_out);
// Per-state Im<a|P|b> for a Pauli generator (x, zy, n_y) -> d_out[b * out_stride].
void launch_batched_pauli_im_p(const LaunchCtx& ctx, const double2* a, const double2* b,
                               uint32_t n, uint32_t batch, uint64_t x, uint64_t zy,
                               uint32_t n_y, double* d_partials, double* d_out,
                               uint64_t out_stride);

}  // namespace lqcs_b200
