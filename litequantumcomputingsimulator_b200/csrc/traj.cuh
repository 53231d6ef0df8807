// traj.cuh — batched trajectory kernels (traj_kernels.cu).
#pragma once

#include <cstdint>

#include "kernels.cuh"

namespace lqcs_b200 {

constexpr uint32_t kTrajMaxBlocks = 64;   // reduction blocks per state

struct TrajDecide {
    int mode;                 // 0 Kraus branch, 1 Born-rule outcome (measure / reset)
    int is_measure;           // mode 1: record the outcome in the classical register
    uint32_t clbit;
    uint32_t uniform_index;   // index of this event's uniform within a shot
    uint32_t n_ops;           // mode 0: Kraus operators (2x2 each, device memory)
    const double2* ops;
    const int* forced;        // mode 0, optional (device, per state): branch >= 0 known in
                              // advance -> the state is left alone here (no reduction, nothing
                              // applied); the caller applies that branch elsewhere
};

// Device scratch for a resident batch of R trajectories.
struct TrajScratch {
    double* partials;   // R * 4 * kTrajMaxBlocks
    double2* mats;      // R * 4
    int* flag;          // R
    double* scale;      // R
    uint64_t* regs;     // R classical registers
};

// rdm of qubit q per state -> branch per state (uniform u[(first+b)*per_shot+j]) ->
// K/sqrt(p) applied per state.  States need not be normalised: probabilities are taken
// relative to the state's norm and the chosen branch leaves the state normalised.
void launch_traj_kraus(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch, uint32_t q,
                       const TrajDecide& d, const double* d_uniforms, uint64_t first,
                       uint64_t per_shot, TrajScratch& s);
// Born-rule collapse (reset = 0) or reset to |0> (reset = 1) per state.
void launch_traj_measure(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch,
                         uint32_t q, const TrajDecide& d, const double* d_uniforms,
                         uint64_t first, uint64_t per_shot, int reset, TrajScratch& s);
// Terminal measurement of qubit q without collapsing: state b's amplitudes consistent with
// its earlier terminal outcomes (bits `fixed` equal to vals[b]) give p1 relative to their
// total; the outcome is recorded in vals[b] (bit q) and in the classical register.
void launch_traj_tail_measure(const LaunchCtx& ctx, const double2* st, uint32_t n,
                              uint32_t batch, uint32_t q, const BitList& fixed, uint64_t* vals,
                              uint32_t clbit, uint32_t uniform_index, const double* d_uniforms,
                              uint64_t first, uint64_t per_shot, TrajScratch& s);
// Joint distribution of measured qubits mq[0..m-1] of one state: table[t] = sum of |a|^2
// over the amplitudes whose bit mq[j] equals bit j of t, summed in a fixed order (chunks of
// the free indices, then the chunks in order).  `partial` holds 2^m * chunks doubles, where
// chunks = marginal_chunks(n, m).
uint64_t marginal_chunks(uint32_t n, uint32_t m);
void launch_marginal_table(const LaunchCtx& ctx, const double2* st, uint32_t n,
                           const uint32_t* mq, uint32_t m, double* partial, double* table);
// Per-state choice into a table of normalised 2x2 operators (choice < 0: no-op).
void launch_traj_table(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch, uint32_t q,
                       const double2* d_mats, const int* d_choice);

}  // namespace lqcs_b200
