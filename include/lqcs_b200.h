/*
 * lqcs_b200.h — C ABI of the B200 statevector engine for LiteQuantumComputingSimulator.
 *
 * Every entry point takes plain pointers and sizes, returns an int status (LQCS_OK == 0)
 * and leaves a message for lqcs_last_error() on failure.  The status codes stand in for
 * the C++ exception types the reference throws on the same inputs, so a C++ wrapper can
 * rethrow the same type with the same message:
 *
 *   LQCS_ERR_INVALID_ARGUMENT  -> std::invalid_argument
 *   LQCS_ERR_OUT_OF_RANGE      -> std::out_of_range
 *   LQCS_ERR_LOGIC             -> std::logic_error
 *
 * Amplitude layout (host and device): 2^n complex128 values, interleaved (re, im),
 * qubit 0 is the least significant bit of the basis index — the layout of
 * lqcs::Statevector (include/lqcs/backend/statevector.hpp:12-37).
 *
 * Threading: calls are synchronous with respect to the host unless stated otherwise;
 * one state handle must not be used by two host threads at once.
 */
#ifndef LQCS_B200_H
#define LQCS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
enum lqcs_status {
    LQCS_OK = 0,
    LQCS_ERR_INVALID_ARGUMENT = 1,
    LQCS_ERR_OUT_OF_RANGE = 2,
    LQCS_ERR_LOGIC = 3,
    LQCS_ERR_CUDA = 4,
    LQCS_ERR_OUT_OF_MEMORY = 5,
    LQCS_ERR_TIMEOUT = 6,   /* reserved: no entry point waits on a flag another rank or
                               device sets, so none returns it */
    LQCS_ERR_INTERNAL = 7
};

/* ------------------------------------------------------------------ gate types
 * Same names and the same order as lqcs::GateType
 * (include/lqcs/circuit/gate.hpp:14-28), so a caller can cast the enum value.
 * LQCS_GATE_KRAUS is an engine extension: an explicit one-qubit noise channel placed
 * in the instruction stream (it has no counterpart in lqcs::GateType). */
enum lqcs_gate_type {
    LQCS_GATE_I = 0, LQCS_GATE_X, LQCS_GATE_Y, LQCS_GATE_Z, LQCS_GATE_H,
    LQCS_GATE_S, LQCS_GATE_SDG, LQCS_GATE_T, LQCS_GATE_TDG, LQCS_GATE_SX,
    LQCS_GATE_RX, LQCS_GATE_RY, LQCS_GATE_RZ, LQCS_GATE_P, LQCS_GATE_U,
    LQCS_GATE_SWAP, LQCS_GATE_ISWAP, LQCS_GATE_RXX, LQCS_GATE_RYY, LQCS_GATE_RZZ,
    LQCS_GATE_PAULI_ROTATION,
    LQCS_GATE_UNITARY, LQCS_GATE_PERMUTATION,
    LQCS_GATE_MEASURE, LQCS_GATE_RESET, LQCS_GATE_BARRIER,
    LQCS_GATE_KRAUS = 64
};

/* One circuit instruction: the flattened form of lqcs::Instruction
 * (include/lqcs/circuit/instruction.hpp:9-13) and lqcs::Gate
 * (include/lqcs/circuit/gate.hpp:30-68).
 *   qubits  : n_qubits entries, controls first, then targets (instruction.hpp:11).
 *   matrix  : UNITARY — dim*dim complex, row-major, interleaved (2*dim*dim doubles);
 *             KRAUS   — n_kraus 2x2 complex operators (8 doubles each).
 *   perm    : PERMUTATION — dim entries, |l> -> |perm[l]>.
 *   pauli   : PAULI_ROTATION — n_targets characters from {I,X,Y,Z}; the rightmost
 *             character acts on the first target (gate.hpp:36-37).
 *   params  : rotation angles (RX..U, RXX..RZZ, PAULI_ROTATION use params[0..2]).
 *   clbit   : MEASURE only. */
typedef struct lqcs_instruction {
    int32_t gate_type;
    uint32_t n_controls;
    uint32_t n_qubits;
    uint32_t n_params;
    double params[3];
    uint32_t clbit;
    uint32_t n_kraus;
    const uint32_t* qubits;
    const double* matrix;
    const uint64_t* perm;
    const char* pauli;
} lqcs_instruction;

/* A one-qubit Kraus channel: n_ops operators of 2x2 complex, row-major, interleaved
 * (8 doubles each).  Mirrors lqcs::KrausChannel (include/lqcs/backend/noise.hpp:11-26). */
typedef struct lqcs_kraus_channel {
    uint64_t n_ops;
    const double* ops;
} lqcs_kraus_channel;

/* Mirrors lqcs::StatevectorSimulator::Options
 * (include/lqcs/backend/statevector_simulator.hpp:19-26):
 *   seed / has_seed : std::optional<uint64_t> seed (no seed -> std::random_device)
 *   fuse_gates      : bool fuse_gates = true
 *   num_threads     : accepted and ignored (no GPU meaning)
 *   channels        : NoiseModel::channels(), applied after every unitary instruction on
 *                     every qubit it touches (statevector_simulator.cpp:146-153).
 * Engine knobs (no counterpart in Options; zero means "engine default"):
 *   max_fusion_width : widest dense block the fusion pass may emit (1..6)
 *   fusion_mode      : 0 = default planner, 1 = greedy, 2 = learned cost model,
 *                      3 = gate-by-gate (no fusion even if fuse_gates), 4 = tile passes,
 *                      5 = autotuned (lqcs_autotune's measured choice)
 *   max_resident     : most noise trajectories held on the device at once.
 *   shot_offset      : the call's shots are shots shot_offset.. of a longer run with the same
 *                      seed: the uniforms of the shots before them are skipped, so runs of
 *                      consecutive shot ranges (one per rank) concatenate to the one run. */
typedef struct lqcs_sim_options {
    uint64_t seed;
    int32_t has_seed;
    int32_t fuse_gates;
    int32_t num_threads;
    int32_t max_fusion_width;
    int32_t fusion_mode;
    int32_t max_resident;
    uint64_t n_channels;
    const lqcs_kraus_channel* channels;
    uint64_t shot_offset;
} lqcs_sim_options;

typedef struct lqcs_state lqcs_state; /* opaque device-resident statevector */

/* ------------------------------------------------------------------ errors */

/* Message of the last failed call on this host thread ("" if none).  Replaces the
 * what() text of the exception the reference would have thrown. */
const char* lqcs_last_error(void);

/* Library version string, e.g. "lqcs_b200 0.1.0 sm_100a". */
const char* lqcs_version(void);

/* ------------------------------------------------------------------ states */

/* Allocate a 2^n_qubits complex128 state on the current CUDA device in |0...0>.
 * Replaces lqcs::Statevector::Statevector(n) (src/backend/statevector.cpp:11-25).
 * n_qubits == 0 -> LQCS_ERR_INVALID_ARGUMENT.  The reference's 30-qubit cap is lifted:
 * the cap is what fits in device memory (33 qubits on a 180 GB B200), and larger
 * requests fail with the reference's message style.  stream may be NULL (default
 * stream) or a cudaStream_t all work on this state is ordered on. */
int lqcs_state_create(uint32_t n_qubits, void* stream, lqcs_state** out);

/* Allocate `batch` independent states of n_qubits each, contiguous on the device
 * (state b starts at amplitude b * 2^n_qubits).  Used by batched trajectories and
 * batched gradients; single-state entry points act on state 0. */
int lqcs_state_create_batch(uint32_t n_qubits, uint32_t batch, void* stream,
                            lqcs_state** out);

int lqcs_state_destroy(lqcs_state* st);

int lqcs_state_num_qubits(const lqcs_state* st, uint32_t* out);

/* Device pointer of the amplitudes (interleaved complex128) for zero-copy interop. */
int lqcs_state_device_ptr(const lqcs_state* st, void** out);

/* Reset every state in the handle to |0...0>. */
int lqcs_state_set_zero(lqcs_state* st);

/* Copy n_amps complex128 amplitudes host -> device (n_amps must be 2^n_qubits). */
int lqcs_state_load(lqcs_state* st, const double* host_amps, uint64_t n_amps);

/* Copy n_amps complex128 amplitudes device -> host. */
int lqcs_state_store(const lqcs_state* st, double* host_amps, uint64_t n_amps);

/* ------------------------------------------------------------------ evolution */

/* Apply the unitary instructions of a circuit to the state, skipping Measure and
 * Barrier, failing on Reset — the loop of `evolve`
 * (src/backend/statevector_simulator.cpp:197-207) with the dispatch of
 * `apply_instruction` (src/backend/statevector_simulator.cpp:22-85).
 * fuse_gates != 0 runs the engine's fusion pass first (the place of
 * SingleQubitGateFusion, src/transpiler/gate_fusion.cpp:32-67); max_fusion_width and
 * fusion_mode as in lqcs_sim_options. */
int lqcs_state_apply(lqcs_state* st, const lqcs_instruction* insts, uint64_t n_insts,
                     int32_t fuse_gates, int32_t max_fusion_width, int32_t fusion_mode);

/* A compiled circuit: the unitary instructions fused (or not) and lowered to device
 * operations with their matrices resident on the device, so repeated application costs
 * only kernel launches.  Engine extension: the reference re-dispatches each instruction on
 * every run (src/backend/statevector_simulator.cpp:197-207). */
typedef struct lqcs_program lqcs_program;

int lqcs_program_create(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                        int32_t fuse_gates, int32_t max_fusion_width, int32_t fusion_mode,
                        lqcs_program** out);
int lqcs_program_destroy(lqcs_program* prog);
/* n_ops: device operations; n_gates: source unitary gates. */
int lqcs_program_info(const lqcs_program* prog, uint64_t* n_ops, uint64_t* n_gates);
/* Apply the program to every state of the handle (same n_qubits); waits for completion. */
int lqcs_program_apply(lqcs_state* st, const lqcs_program* prog);

/* Per-operation device timing of one application, measured with CUDA events on the
 * state's stream. */
typedef struct lqcs_op_profile {
    uint32_t kind;          /* 0 one-qubit, 1 phase, 2 dense block, 3 diagonal block,
                               4 permutation, 5 Pauli rotation, 6 shared-memory tile pass,
                               7 register tile pass */
    uint32_t n_targets;     /* block width */
    uint32_t n_gates;       /* source gates merged into the operation */
    uint32_t min_target;
    uint32_t max_target;
    uint32_t n_controls;
    double device_ms;
    double alg_bytes;       /* 32 * 2^n * f: amplitudes the operation can change, read+written */
    double alg_flops;       /* FP64 flops executed: 8 per complex multiply-add (dense blocks),
                               6 per complex multiply (diagonals, phases), 0 for permutations */
} lqcs_op_profile;

int lqcs_program_apply_profiled(lqcs_state* st, const lqcs_program* prog, uint64_t cap,
                                lqcs_op_profile* out, uint64_t* n_out);

/* StatevectorSimulator::run_statevector (src/backend/statevector_simulator.cpp:222-230):
 * a new |0...0> state of n_qubits evolved by the circuit.  Fails if opts has noise
 * channels (same message as the reference). */
int lqcs_run_statevector(uint32_t n_qubits, const lqcs_instruction* insts,
                         uint64_t n_insts, const lqcs_sim_options* opts,
                         void* stream, lqcs_state** out);

/* StatevectorSimulator::run (src/backend/statevector_simulator.cpp:232-265).
 * Writes, for every shot s, the classical register as a bit mask into
 * shot_registers[s] (clbit c -> bit c; the reference's key string is this mask printed
 * with clbit n_clbits-1 leftmost).  Same path selection as the reference: end-of-circuit
 * sampling, or per-shot evolution when the circuit has noise, Reset, or a unitary after
 * a Measure.  n_clbits must be <= 64. */
int lqcs_run(uint32_t n_qubits, uint32_t n_clbits, const lqcs_instruction* insts,
             uint64_t n_insts, uint64_t shots, const lqcs_sim_options* opts,
             uint64_t* shot_registers);

/* ------------------------------------------------------------------ density matrices
 * DensityMatrixSimulator (src/backend/density_matrix_simulator.cpp) on the device.  rho of
 * n qubits lives in a state handle of 2n qubits: element rho_{rc} at index (c << n) | r
 * (DensityMatrix::element, src/backend/density_matrix.cpp).  Each unitary is applied as U on
 * the ket bits and conj(U) on the bra bits, each channel of opts->channels follows every
 * unitary on each qubit it touches, explicit Kraus instructions apply where they stand;
 * Measure and Barrier are skipped, Reset is rejected (as the reference). */
int lqcs_dm_create(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                   const lqcs_sim_options* opts, lqcs_state** out);   /* run_density_matrix */
/* Diagonal rho_ii of a density-matrix handle (2^n doubles): DensityMatrix::probabilities. */
int lqcs_dm_probabilities(const lqcs_state* rho, double* probs);
/* DensityMatrixSimulator::run: terminal measurements only; one register per shot as
 * lqcs_run, drawn from the diagonal with the same uniforms and upper_bound rule. */
int lqcs_dm_run(uint32_t n_qubits, uint32_t n_clbits, const lqcs_instruction* insts,
                uint64_t n_insts, uint64_t shots, const lqcs_sim_options* opts,
                uint64_t* shot_registers);

/* Read `count` amplitudes starting at basis index `first` (of state 0) into host memory
 * (2*count doubles).  Serves Statevector::operator[] (include/lqcs/backend/statevector.hpp:21-22). */
int lqcs_state_read_range(const lqcs_state* st, uint64_t first, uint64_t count, double* host);

/* Host-side matrix of one gate: Gate::base_matrix (src/circuit/gate.cpp:94-201) when
 * with_controls == 0, Gate::matrix (src/circuit/gate.cpp:203-226, controls in the low
 * local bits) otherwise.  Writes dim*dim interleaved complex values (row-major) into out
 * (capacity cap_doubles) and dim into *dim_out.  No device work. */
int lqcs_gate_matrix(const lqcs_instruction* inst, int32_t with_controls, double* out,
                     uint64_t cap_doubles, uint64_t* dim_out);

/* ------------------------------------------------------------------ readout */

/* |amp|^2 of every basis state, written to host (2^n doubles).
 * Replaces Statevector::probabilities (src/backend/statevector.cpp:33-37). */
int lqcs_state_probabilities(const lqcs_state* st, double* host_out);

/* sqrt(sum |amp|^2).  Replaces Statevector::norm (src/backend/statevector.cpp:27-31). */
int lqcs_state_norm(const lqcs_state* st, double* out);

/* Shot sampling: for each uniform u_s in [0,1) returns the basis index of
 * upper_bound(cumulative, u_s * total) over the inclusive prefix sum of |amp|^2 —
 * the loop of run_sampling (src/backend/statevector_simulator.cpp:98-109).  The
 * uniforms are the caller's (the reference draws them from lqcs::Rng).
 * min_margin (may be NULL) receives the smallest distance, relative to the total, of a
 * scaled uniform from the bin edges it fell between: counts equal the reference's
 * whenever that distance exceeds the rounding difference of the two prefix sums. */
int lqcs_state_sample(const lqcs_state* st, const double* uniforms, uint64_t shots,
                      uint64_t* idx_out, double* min_margin);

/* <psi|P|psi> for one Pauli string of length n_qubits (leftmost character = highest
 * qubit).  Replaces Statevector::expectation_value (src/backend/statevector.cpp:39-78). */
int lqcs_state_expectation_pauli(const lqcs_state* st, const char* pauli, double* out);

/* sum_t coeffs[t] * <psi|P_t|psi> over n_terms Pauli strings; per_term (may be NULL)
 * receives each <psi|P_t|psi>.  Replaces algorithms::expectation
 * (src/algorithms/vqe.cpp:11-17). */
int lqcs_state_expectation_terms(const lqcs_state* st, const char* const* paulis,
                                 const double* coeffs, uint64_t n_terms,
                                 double* per_term, double* total);

/* <psi|P_t|psi> for up to LQCS_NOALLOC_MAX_TERMS Pauli strings, for callers that cannot
 * allocate device memory (an arena or pool that owns the device, an embedding that forbids
 * cudaMalloc after start-up).  Allocates nothing: the caller passes the amplitudes
 * (2^n_qubits complex128 in device memory, laid out as above) and a host array of n_terms
 * doubles; the partial sums live in one static device array of 131,200 bytes inside the
 * library, held by every GPU that loads it until exit.  More than LQCS_NOALLOC_MAX_TERMS
 * terms -> LQCS_ERR_INVALID_ARGUMENT.  An ordinary host call: it launches kernels and waits
 * for `stream` (NULL = default stream), so it must not run inside stream capture or in a
 * CUDA host function (cudaLaunchHostFunc, graph host nodes), where CUDA calls are not
 * allowed.  The first call on a device looks up the array's device address (with that
 * device current) and keeps it; after a cudaDeviceReset call lqcs_release_caches, which
 * forgets it.  All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  No counterpart in the reference. */
enum { LQCS_NOALLOC_MAX_TERMS = 16 };
int lqcs_expectation_terms_noalloc(const void* d_amps, uint32_t n_qubits,
                                   const char* const* paulis, uint64_t n_terms,
                                   double* host_values, void* stream);

/* ------------------------------------------------------------------ per-shot kernels */

/* Born-rule collapse of qubit q with the caller's uniform (outcome 1 iff u < p1),
 * projection and renormalisation.  Replaces kernels::collapse_qubit
 * (src/backend/kernels/gate_kernels.cpp:227-247). */
int lqcs_state_collapse(lqcs_state* st, uint32_t qubit, double uniform, int32_t* outcome);

/* Collapse, then move a |1> outcome back to |0>.  Replaces kernels::reset_qubit
 * (src/backend/kernels/gate_kernels.cpp:249-260). */
int lqcs_state_reset_qubit(lqcs_state* st, uint32_t qubit, double uniform);

/* ||K psi||^2 for a 2x2 complex K (8 doubles) on qubit q.  Replaces
 * kernels::kraus_probability (src/backend/kernels/gate_kernels.cpp:262-277). */
int lqcs_state_kraus_probability(const lqcs_state* st, uint32_t qubit, const double* k,
                                 double* out);

/* ------------------------------------------------------------------ gradients */

/* Parametric circuit: the template instructions plus, for parameter p, the index of the
 * instruction whose params[0] it sets — lqcs::ParametricCircuit's template_ and
 * param_inst_ (include/lqcs/circuit/parametric_circuit.hpp:20-63).  Parameterised
 * instructions are RX, RY, RZ or PAULI_ROTATION (generator eigenvalues +-1). */
typedef struct lqcs_parametric_circuit {
    uint32_t n_qubits;
    uint64_t n_insts;
    const lqcs_instruction* insts;
    uint64_t n_params;
    const uint64_t* param_inst;
} lqcs_parametric_circuit;

/* Hamiltonian: real combination of Pauli strings (lqcs::algorithms::Hamiltonian,
 * include/lqcs/algorithms/vqe.hpp:13-18). */
typedef struct lqcs_hamiltonian {
    uint64_t n_terms;
    const double* coeffs;
    const char* const* paulis;
} lqcs_hamiltonian;

/* dE/dtheta by the parameter-shift rule on the GPU, one energy per shifted circuit —
 * the algorithm of algorithms::parameter_shift_gradient
 * (src/algorithms/vqe.cpp:68-94), kept as the plain per-circuit GPU path. */
int lqcs_parameter_shift_gradient(const lqcs_parametric_circuit* pc,
                                  const lqcs_hamiltonian* h, const double* params,
                                  double* grad_out);

/* Adjoint-state gradients for `batch` parameter sets (params is batch x n_params,
 * row-major).  energy_out[b] = <psi(theta_b)|H|psi(theta_b)>, grad_out is
 * batch x n_params.  Exact analytic gradient (no shift, no finite difference); equal to
 * parameter_shift_gradient within rounding.  max_resident bounds how many sets are on
 * the device at once (0 = engine default).  Engine extension: the reference has no
 * adjoint method; it replaces calling parameter_shift_gradient once per set. */
int lqcs_adjoint_gradient(const lqcs_parametric_circuit* pc, const lqcs_hamiltonian* h,
                          const double* params, uint64_t batch, uint32_t max_resident,
                          double* energy_out, double* grad_out);

/* Adjoint gradients of several problems of different qubit counts in one call: problem p
 * has its own ansatz pcs[p], Hamiltonian hs[p] and batches[p] parameter sets params[p]
 * (batches[p] x n_params_p); results go to energy_out[p] / grad_out[p] (either array may be
 * NULL, or hold NULL entries).  Each problem keeps a resident batch and all problems run as
 * one captured CUDA graph whose branches execute concurrently, replayed on later calls with
 * the same problems (new parameter values allowed).  Problems below 5 qubits, or more than
 * half the free device memory in total, run one after another instead.  Engine extension:
 * no counterpart in the reference. */
int lqcs_adjoint_gradient_multi(uint64_t n_problems, const lqcs_parametric_circuit* const* pcs,
                                const lqcs_hamiltonian* const* hs, const double* const* params,
                                const uint64_t* batches, double* const* energy_out,
                                double* const* grad_out);

/* Frees what repeated calls keep on the device between calls — the resident state batches
 * and captured graphs of the last adjoint plans, the compiled programs of the last 16
 * circuits run (run / run_statevector reuse them for the same circuit and options) — and
 * the autotuner's choices.  Engine extension: no counterpart in the reference. */
int lqcs_release_caches(void);

/* Energies only, batched: the forward pass and <psi|H|psi> of lqcs_adjoint_gradient
 * without its backward sweep (about half the time of the gradient call). */
int lqcs_batched_energy(const lqcs_parametric_circuit* pc, const lqcs_hamiltonian* h,
                        const double* params, uint64_t batch, uint32_t max_resident,
                        double* energy_out);

/* ------------------------------------------------------------------ fusion planning */

/* Run the fusion planner on a circuit of n_qubits and report, per emitted block,
 * its width and number of source gates (arrays of capacity `cap`; *n_blocks receives
 * the count).  Used by tests and the cost model; no device work. */
int lqcs_fusion_plan(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                     int32_t max_fusion_width, int32_t fusion_mode, uint64_t cap,
                     uint32_t* block_width, uint32_t* block_gates, uint64_t* n_blocks);

/* ------------------------------------------------------------------ autotuner
 * Engine extension (no counterpart in the reference, whose fusion pass has no knobs):
 * times every candidate fusion plan of the circuit — register tile passes of tile sizes
 * 2^11..2^13 and inner widths 2..3, shared-memory tile passes, greedy dense blocks of width
 * 4..6 — once each (after one untimed application) on a scratch n-qubit state allocated for
 * the call, and remembers the fastest for this circuit; fusion_mode 5 then compiles with it
 * (tuning on first use).  Needs 16 * 2^n bytes free for the scratch state; without them
 * *n_out is 0 and fusion_mode 5 uses the default plan. */
typedef struct lqcs_tune_entry {
    int32_t planner;        /* 0 register tile passes, 1 shared-memory tile passes, 2 greedy */
    uint32_t tile_bits;     /* tile passes: 2^tile_bits amplitudes per tile */
    uint32_t tile_low;      /* tile passes: qubits 0..tile_low-1 always in the tile */
    uint32_t inner;         /* tile passes: widest block fused inside a pass */
    uint32_t width;         /* greedy: widest block */
    uint32_t chosen;        /* 1 for the fastest candidate */
    uint64_t n_ops;         /* device operations (launches) of one application */
    double device_ms;       /* one application, CUDA events */
} lqcs_tune_entry;

int lqcs_autotune(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                  uint64_t cap, lqcs_tune_entry* out, uint64_t* n_out);

/* ------------------------------------------------------------------ cost model
 * A 3-layer, 64-wide FP32 MLP predicting the device time of one device operation from
 * LQCS_COST_FEATURES features (op kind, width, lowest / highest qubit touched, source gate
 * count, register size, FP64 flops per amplitude; see lqcs_costmodel_features), trained by
 * the engine's own FP32
 * forward / backward / Adam kernels on timings the engine measures
 * (lqcs_program_apply_profiled).  fusion_mode 2 uses it to choose among candidate fusion
 * plans; without trained weights it falls back to the greedy plan.  Engine extension: no
 * counterpart in the reference.  Targets are log(milliseconds per 2^24 amplitudes). */
enum { LQCS_COST_FEATURES = 7, LQCS_COST_HIDDEN = 64 };

/* Feature row of one operation (kind as in lqcs_op_profile; flops_per_amp = its alg_flops
 * divided by the amplitudes of one state). */
int lqcs_costmodel_features(uint32_t kind, uint32_t width, uint32_t min_target,
                            uint32_t max_target, uint32_t n_gates, uint32_t n_qubits,
                            double flops_per_amp, float* out);

/* Train from scratch on n rows (features n x LQCS_COST_FEATURES, targets n); the weights
 * stay in the library.  loss_out (may be NULL) receives the final mean squared error. */
int lqcs_costmodel_train(const float* features, const float* targets, uint64_t n,
                         uint32_t epochs, float learning_rate, uint64_t seed, float* loss_out);

/* Predictions for n rows with the current weights. */
int lqcs_costmodel_predict(const float* features, uint64_t n, float* out);

/* Loss and the flattened gradient of every parameter (W1, b1, W2, b2, W3, b3) on a batch,
 * without updating; *n_params_out receives the parameter count. */
int lqcs_costmodel_grad(const float* features, const float* targets, uint64_t n,
                        float* loss_out, float* grad_out, uint64_t grad_cap,
                        uint64_t* n_params_out);

/* Get / set / drop the flattened weights. */
int lqcs_costmodel_get_weights(float* out, uint64_t cap, uint64_t* n_out);
int lqcs_costmodel_set_weights(const float* w, uint64_t n);
int lqcs_costmodel_clear(void);

/* Predicted device time (ms) of the plan a fusion mode would build for a circuit. */
int lqcs_costmodel_plan_ms(uint32_t n_qubits, const lqcs_instruction* insts, uint64_t n_insts,
                           int32_t max_fusion_width, int32_t fusion_mode, double* ms_out);

/* ------------------------------------------------------------------ random numbers */

/* `count` draws of lqcs::Rng(seed).uniform() (include/lqcs/core/random.hpp:10-23):
 * std::uniform_real_distribution<double>(0, 1) over std::mt19937_64 seeded with `seed`.
 * The run paths draw their shot and branch uniforms the same way. */
int lqcs_rng_uniforms(uint64_t seed, uint64_t count, double* out);

/* Raw 64-bit draws `skip` .. `skip + count - 1` of std::mt19937_64 seeded with `seed` (the
 * engine behind lqcs::Rng, include/lqcs/core/random.hpp): what algorithms::shor
 * (src/algorithms/shor.cpp:72-102) draws its bases and simulator seeds from. */
int lqcs_rng_u64(uint64_t seed, uint64_t skip, uint64_t count, uint64_t* out);

/* ------------------------------------------------------------------ diagnostics */

/* Number of kernels this library has launched since load (all devices). */
uint64_t lqcs_kernel_launch_count(void);

/* Host emulation of the register tile kernel, for tests (no device work; engine extension
 * with no counterpart in the reference).  Plans the circuit into register tile passes as
 * lqcs_program_create does with the tile-pass planner (the LQCS_TILE_* overrides apply)
 * and runs every pass thread by thread on the host: with `state` (2^n_qubits complex128,
 * interleaved, in/out) it computes the amplitudes, out of place, fails if a pass stores an
 * amplitude other than exactly once or one its tile did not load, and checks that no store
 * can overtake another thread's load of the same amplitude (in place, a relabelling pass
 * stores to places other warps load); in any case it checks every shared-memory access of
 * the kernel against the barrier model (warps independent between CTA barriers, threads of
 * a warp independent between warp barriers) for a grid of `grid` CTAs (with state == NULL
 * only the first `race_ctas` CTAs are walked).  sync_tiles: 2 = as the kernel runs (a
 * barrier between a CTA's tiles where the last layout's warp bits differ from the first
 * layout's), 1 = a barrier between
 * all tiles, 0 = none, 3 = the double-buffered kernel (LQCS_REG_PIPE=1; 2^11- and
 * 2^12-amplitude tiles); + 8 leaves out the barrier a relabelling pass puts between its
 * loads and stores.  *n_races counts racing accesses; `report` (capacity report_cap)
 * receives the first.  Fails if a gate does not run inside a register pass. */
int lqcs_debug_emulate_register_passes(uint32_t n_qubits, const lqcs_instruction* insts,
                                       uint64_t n_insts, uint64_t grid, int32_t sync_tiles,
                                       double* state, uint64_t race_ctas, uint64_t* n_passes,
                                       uint64_t* n_races, char* report, uint64_t report_cap);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* LQCS_B200_H */
