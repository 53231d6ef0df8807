// engine.hpp — device runtime of the engine: state handles, compiled op programs, and
// the run paths of StatevectorSimulator (end-of-circuit sampling, per-shot evolution,
// trajectory noise) plus expectations and gradients.
#pragma once

#include <cstdint>
#include <memory>
#include <random>
#include <vector>

#include "gates.hpp"
#include "kernels.cuh"
#include "tile_plan.hpp"

namespace lqcs_b200 {

void cuda_check(cudaError_t e, const char* what);

// Owning device allocation.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            bytes = o.bytes;
            o.ptr = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void release();
    void ensure(size_t b);
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

int device_sm_count();
LaunchCtx make_ctx(cudaStream_t s);

// A compiled sequence of device ops with its constant data resident on the device.
struct Program {
    std::vector<DevOp> ops;
    std::vector<uint64_t> mat_off;   // per op: offset (double2) of its matrix / diagonal
    std::vector<uint64_t> cyc_off;   // per op: offset (uint32) of its cycles
    std::vector<uint64_t> len_off;   // per op: offset (uint32) of its cycle lengths
    DeviceBuffer d_mats, d_u32;
    uint64_t source_gates = 0;
    // shared-memory tile passes (ops of kind TILE index into these)
    std::vector<TilePass> passes;
    std::vector<uint64_t> pass_op_off;   // first TileOp of each pass
    std::vector<TileOp> tile_ops;
    std::vector<cd> tile_mats;
    DeviceBuffer d_tile_ops, d_tile_mats;
    // register tile passes (ops of kind TILE with reg_tile set index into these)
    std::vector<RegPass> reg_passes;
    std::vector<uint64_t> reg_op_off, reg_lay_off, reg_mat_off;   // per pass
    std::vector<RegOp> reg_ops;
    std::vector<RegLayout> reg_layouts;
    std::vector<cd> reg_mats;
    DeviceBuffer d_reg_ops, d_reg_layouts, d_reg_mats;

    void build(std::vector<DevOp> ops_in, cudaStream_t stream);
    void launch(const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch) const;
    void launch_op(size_t i, const LaunchCtx& ctx, double2* st, uint32_t n, uint32_t batch) const;
};

// Fusion knobs.
struct FusionConfig {
    bool fuse = true;
    uint32_t max_width = 0;   // 0 = engine default
    int mode = 0;             // 0 default, 1 greedy dense blocks, 2 learned, 3 none, 4 tile passes
};
enum FusionMode {
    kFuseDefault = 0, kFuseGreedy = 1, kFuseLearned = 2, kFuseNone = 3, kFuseTile = 4,
    kFuseAutotune = 5
};

// One fusion plan the autotuner times: register or shared-memory tile passes of a shape, or
// greedy dense blocks of a width.
struct TuneCandidate {
    int planner = 0;          // 0 register tile passes, 1 shared-memory tile passes, 2 greedy
    TileConfig cfg;
    uint32_t width = 0;
};
struct TuneTiming {
    TuneCandidate cand;
    uint64_t n_ops = 0;
    double ms = 0.0;
};
// Times every candidate plan of `gates` once (after one untimed application) on a scratch
// n-qubit state and remembers the fastest for this circuit; fusion_mode 5 compiles with it.
// Empty when no scratch state fits in device memory (mode 5 then uses the default plan).
std::vector<TuneTiming> autotune(const std::vector<GateDesc>& gates, uint32_t n, size_t* best);
void clear_autotune_cache();
uint32_t default_fusion_width();
// Drop the compiled programs kept for repeated circuits (apply_circuit).
void clear_program_cache();
// Free the amplitude buffers kept for new states of the same size.
void clear_state_pool();
// Called by ~lqcs_state: keeps a small amplitude buffer for the next state of its size.
void pool_return(lqcs_state& st);

// Compile a list of unitary gates to a Program (fused or gate by gate).
Program compile(const std::vector<GateDesc>& gates, uint32_t n, const FusionConfig& fc,
                cudaStream_t stream);

// Tile-pass program for a batch whose noise slots (GateDesc::slot) take per-state matrices
// (slots[b][slot_id] for state b).  False when some pass does not fit the register kernel
// or a slot would run outside a pass; `out` is then unusable.
bool compile_slots(const std::vector<GateDesc>& gates, uint32_t n,
                   const std::vector<std::vector<std::array<cd, 4>>>& slots, cudaStream_t stream,
                   Program& out);
std::vector<FusedBlock> plan(const std::vector<GateDesc>& gates, uint32_t n,
                             const FusionConfig& fc);

}  // namespace lqcs_b200

// The opaque handle of the C ABI.
struct lqcs_state {
    int device = 0;
    uint32_t n = 0;
    uint32_t batch = 1;
    cudaStream_t stream = nullptr;
    lqcs_b200::DeviceBuffer amps;
    lqcs_b200::DeviceBuffer scratch;   // reductions (device)
    // sampling: chunk and segment prefixes, uniforms, indices, margins — kept with the state
    // (the largest request so far: 0.5 B per amplitude plus 24 B per shot), so repeated
    // sampling allocates nothing
    lqcs_b200::DeviceBuffer sample_scratch;
    lqcs_b200::LaunchCtx ctx;

    double2* d() const { return amps.as<double2>(); }
    uint64_t len() const { return uint64_t{1} << n; }
    double* partials(size_t values);   // scratch for `values` reduced outputs
    void sync() const;
    ~lqcs_state();   // hands a small amplitude buffer to the state pool
};

// A compiled circuit handle of the C ABI.
struct lqcs_program {
    uint32_t n = 0;
    lqcs_b200::Program prog;
};

namespace lqcs_b200 {

std::unique_ptr<lqcs_program> program_create(uint32_t n, const std::vector<GateDesc>& gates,
                                             const FusionConfig& fc);
void program_profile(lqcs_state& st, const lqcs_program& p, uint64_t cap, lqcs_op_profile* out,
                     uint64_t* n_out);

using Rng = std::mt19937_64;
// One draw of lqcs::Rng::uniform (include/lqcs/core/random.hpp:10-23):
// std::uniform_real_distribution<double>(0, 1) over std::mt19937_64.
double rng_uniform(Rng& r);
Rng make_rng(const lqcs_sim_options* opts);
// NoiseModel channels of the options (each a list of 2x2 Kraus operators).
std::vector<std::vector<std::array<cd, 4>>> decode_channels(const lqcs_sim_options* opts);

// Density-matrix backend (dm.cpp): rho of n qubits as a 2n-qubit device state, element
// rho_{rc} at (c << n) | r.
std::unique_ptr<lqcs_state> dm_evolve(uint32_t n, const std::vector<GateDesc>& gates,
                                      const lqcs_sim_options* opts);
void dm_probabilities(lqcs_state& rho, uint32_t n, double* host);
void dm_run_shots(uint32_t n, uint32_t n_clbits, const std::vector<GateDesc>& gates,
                  uint64_t shots, const lqcs_sim_options* opts, uint64_t* regs);

std::unique_ptr<lqcs_state> new_state(uint32_t n, uint32_t batch, cudaStream_t stream);
uint32_t max_qubits_on_device(uint32_t batch);

// Apply unitary instructions (skip Measure/Barrier, reject Reset).
void apply_circuit(lqcs_state& st, const std::vector<GateDesc>& gates, const FusionConfig& fc);

// Reductions on state 0 of a handle.
double state_norm2(lqcs_state& st);
std::vector<double> expectation_terms(lqcs_state& st, const std::vector<PauliMasks>& terms);
int collapse(lqcs_state& st, uint32_t q, double u);
void reset_qubit(lqcs_state& st, uint32_t q, double u);
double kraus_probability(lqcs_state& st, uint32_t q, const std::array<cd, 4>& k);
void sample(lqcs_state& st, const double* u, uint64_t shots, uint64_t* idx, double* min_margin);

// Expectation values with the scratch in a static device array (static_expect.cu).
// Host emulation of the register tile kernel (reg_emulate.cpp).  sync_tiles: 1 barrier
// between tiles, 0 none, 2 where a remap changes the warp bits (RegPass::cta_remaps).
// pipe: the double-buffered kernel's access pattern (tile sizes 2^11 and 2^12).
void emulate_register_program(uint32_t n, const lqcs_instruction* insts, uint64_t n_insts,
                              uint64_t grid, int sync_tiles, bool pipe, bool drop_load_barrier,
                              cd* state, uint64_t race_ctas, uint64_t* n_passes,
                              uint64_t* n_races, std::string* report);

uint32_t static_expectation_max_terms();
void forget_static_scratch_addresses();   // after a device reset (lqcs_release_caches)
void expectation_terms_static(const void* d_amps, uint32_t n_qubits, const char* const* paulis,
                              uint64_t n_terms, double* host_values, cudaStream_t stream);

// Per-shot evolution (mid-circuit measurement, reset, noise) with many shots resident on
// the device (trajectory.cpp).  `regs` receives the classical register of every shot.
void run_per_shot_batched(uint32_t n, const std::vector<GateDesc>& gates, uint64_t shots,
                          const std::vector<std::vector<std::array<cd, 4>>>& channels,
                          const FusionConfig& fc, Rng& rng, uint32_t max_resident,
                          uint64_t* regs, uint64_t shot_offset = 0);

// StatevectorSimulator::run.
void run_shots(uint32_t n, uint32_t n_clbits, const std::vector<GateDesc>& gates,
               uint64_t shots, const lqcs_sim_options* opts, uint64_t* regs);

// Gradients.
struct Hamiltonian {
    std::vector<double> coeffs;
    std::vector<PauliMasks> terms;
};
Hamiltonian decode_hamiltonian(const lqcs_hamiltonian* h, uint32_t n);
// A Hamiltonian on the device in the grouped form launch_apply_hamiltonian reads.
struct HamiltonianDev {
    DeviceBuffer terms, groups;
    uint32_t n_terms = 0;
    void upload(const Hamiltonian& h, uint32_t n);
};
double energy(lqcs_state& st, const Hamiltonian& h);
// Decode a parametric circuit; parameterised gates must be RX, RY, RZ or rp without controls.
void check_pc(const lqcs_parametric_circuit* pc, std::vector<GateDesc>& tmpl,
              std::vector<uint64_t>& pinst);
// ParametricCircuit::bind (src/circuit/parametric_circuit.cpp:73-96).
std::vector<GateDesc> bind_params(const std::vector<GateDesc>& tmpl,
                                  const std::vector<uint64_t>& param_inst, const double* values);
void parameter_shift(const lqcs_parametric_circuit* pc, const Hamiltonian& h,
                     const double* params, double* grad);
void adjoint_batched(const lqcs_parametric_circuit* pc, const Hamiltonian& h,
                     const double* params, uint64_t batch, uint32_t max_resident,
                     double* energy_out, double* grad_out);
// Frees the cached adjoint plans (their resident state batches and graphs).
void release_adjoint_plans();
void adjoint_batched_multi(uint64_t n_problems, const lqcs_parametric_circuit* const* pcs,
                           const lqcs_hamiltonian* const* hs, const double* const* params,
                           const uint64_t* batches, double* const* energy_out,
                           double* const* grad_out);

}  // namespace lqcs_b200
