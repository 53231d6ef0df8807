// static_expect.cu — Pauli expectation values without any device allocation.
//
// For callers that hold their amplitudes in device memory they manage themselves and may
// not allocate more: code running inside a memory pool or arena that owns the whole
// device, or an embedding that forbids cudaMalloc after start-up.  The regular expectation
// path (lqcs_state_expectation_terms) needs a state handle and scratch it allocates; this
// path uses a fixed scratch array that is part of the library image instead.  It is an
// ordinary host call: it launches kernels, copies the results to the host and waits for
// its stream, so it must not be made inside stream capture or from a CUDA host function
// (cudaLaunchHostFunc or a graph host node, where CUDA calls are not allowed).
//
// The scratch is one file-scope __device__ array of kStaticScratchDoubles doubles
// (131,200 bytes).  Every GPU that loads the library holds its own copy until the process
// exits.  Host code cannot use the array's name as a device address: on first use on a
// device (with that device current) the address is fetched once with
// cudaGetSymbolAddress, checked, cached per device, and passed to the kernels.  A device
// reset (cudaDeviceReset) invalidates that address: lqcs_release_caches forgets the
// cached addresses, so call it after a reset, as for the library's other device caches.
//
// Every call shares the same array and leaves its last contents behind.  The partial
// kernel overwrites every slot the final kernel reads, so nothing has to start at zero.
// Calls whose work overlaps on the GPU (different streams, or different host threads
// without ordering) race on the array and give wrong results; serialise them.
//
// The partial kernel reads, per amplitude, the partner a_{i ^ x_t} of every term: up to
// 16 extra reads per amplitude, mostly from L1/L2 when the X masks are small.  The
// regular path groups terms by X mask instead; with at most 16 terms and a fixed scratch
// this simpler form is kept.
#include <mutex>
#include <stdexcept>
#include <string>

#include "engine.hpp"

namespace lqcs_b200 {

namespace {

constexpr uint32_t kStaticMaxTerms = 16;
constexpr uint32_t kStaticBlocks = 512;
constexpr uint32_t kStaticThreads = 256;
// per term: (re, im) partial per block, then one result per term
constexpr size_t kStaticScratchDoubles =
    size_t{kStaticMaxTerms} * 2 * kStaticBlocks + kStaticMaxTerms;

static __device__ __align__(256) double g_static_scratch[kStaticScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

}  // namespace

void forget_static_scratch_addresses() {
    std::lock_guard<std::mutex> lk(g_mu);
    for (double*& a : g_addr) a = nullptr;
}

namespace {

double* scratch_address() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) invalid("expectation_terms_noalloc: device index too large");
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_addr[dev] == nullptr) {
        void* p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_static_scratch), "cudaGetSymbolAddress");
        g_addr[dev] = static_cast<double*>(p);
    }
    return g_addr[dev];
}

struct StaticTerms {
    uint64_t x[kStaticMaxTerms];
    uint64_t zy[kStaticMaxTerms];
    uint32_t n_y[kStaticMaxTerms];
    uint32_t n_terms;
    uint64_t len;
};

__device__ __forceinline__ double sign_of(uint64_t v) { return (__popcll(v) & 1) ? -1.0 : 1.0; }

// One read of a_i per amplitude for all terms; term t's partner a_{i ^ x_t}.
__global__ void __launch_bounds__(kStaticThreads) k_static_partial(const double2* __restrict__ s,
                                                                   StaticTerms p,
                                                                   double* __restrict__ scratch) {
    double acc[2 * kStaticMaxTerms];
#pragma unroll
    for (int k = 0; k < static_cast<int>(2 * kStaticMaxTerms); ++k) acc[k] = 0.0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < p.len;
         i += stride) {
        const double2 a = __ldg(s + i);
#pragma unroll
        for (int t = 0; t < static_cast<int>(kStaticMaxTerms); ++t) {
            if (t < static_cast<int>(p.n_terms)) {
                const double2 b = __ldg(s + (i ^ p.x[t]));
                const double sg = sign_of(i & p.zy[t]);
                acc[2 * t] += sg * (a.x * b.x + a.y * b.y);
                acc[2 * t + 1] += sg * (a.y * b.x - a.x * b.y);
            }
        }
    }
    __shared__ double sh[2 * kStaticMaxTerms][kStaticThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < static_cast<int>(2 * kStaticMaxTerms); ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) sh[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 2 * p.n_terms) {
        double v = 0.0;
        for (int w = 0; w < static_cast<int>(kStaticThreads / 32); ++w) v += sh[threadIdx.x][w];
        scratch[static_cast<size_t>(threadIdx.x) * kStaticBlocks + blockIdx.x] = v;
    }
}

// One block per term: fixed-order sum of the partials, times i^{n_y}, real part.
__global__ void __launch_bounds__(kStaticThreads) k_static_final(StaticTerms p, uint32_t nb,
                                                                 double* __restrict__ scratch) {
    const uint32_t t = blockIdx.x;
    double re = 0.0, im = 0.0;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
        re += scratch[static_cast<size_t>(2 * t) * kStaticBlocks + b];
        im += scratch[static_cast<size_t>(2 * t + 1) * kStaticBlocks + b];
    }
    __shared__ double sre[kStaticThreads / 32], sim[kStaticThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sre[threadIdx.x >> 5] = re;
        sim[threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0, i = 0.0;
        for (int w = 0; w < static_cast<int>(kStaticThreads / 32); ++w) {
            r += sre[w];
            i += sim[w];
        }
        double v;
        switch (p.n_y[t] & 3u) {
            case 0: v = r; break;
            case 1: v = -i; break;
            case 2: v = -r; break;
            default: v = i; break;
        }
        scratch[size_t{kStaticMaxTerms} * 2 * kStaticBlocks + t] = v;
    }
}

}  // namespace

uint32_t static_expectation_max_terms() { return kStaticMaxTerms; }

void expectation_terms_static(const void* d_amps, uint32_t n_qubits, const char* const* paulis,
                              uint64_t n_terms, double* host_values, cudaStream_t stream) {
    if (d_amps == nullptr) invalid("expectation_terms_noalloc: amplitudes pointer is null");
    if (n_qubits == 0 || n_qubits > 40) invalid("expectation_terms_noalloc: n_qubits must be in [1, 40]");
    if (n_terms > kStaticMaxTerms) {
        invalid("expectation_terms_noalloc: at most " + std::to_string(kStaticMaxTerms) +
                " Pauli terms per call (got " + std::to_string(n_terms) + ")");
    }
    if (n_terms == 0) return;
    if (paulis == nullptr || host_values == nullptr)
        invalid("expectation_terms_noalloc: null argument");
    StaticTerms p{};
    p.n_terms = static_cast<uint32_t>(n_terms);
    p.len = uint64_t{1} << n_qubits;
    for (uint64_t t = 0; t < n_terms; ++t) {
        const PauliMasks m = pauli_global_masks(paulis[t], n_qubits, "expectation_value");
        p.x[t] = m.x;
        p.zy[t] = m.zy;
        p.n_y[t] = m.n_y;
    }
    double* scratch = scratch_address();
    const uint64_t want = (p.len + kStaticThreads - 1) / kStaticThreads;
    const uint32_t nb = static_cast<uint32_t>(want < kStaticBlocks ? want : kStaticBlocks);
    k_static_partial<<<nb, kStaticThreads, 0, stream>>>(static_cast<const double2*>(d_amps), p,
                                                        scratch);
    cuda_check(cudaGetLastError(), "k_static_partial launch");
    count_launch();
    k_static_final<<<p.n_terms, kStaticThreads, 0, stream>>>(p, nb, scratch);
    cuda_check(cudaGetLastError(), "k_static_final launch");
    count_launch();
    cuda_check(cudaMemcpyAsync(host_values, scratch + size_t{kStaticMaxTerms} * 2 * kStaticBlocks,
                               sizeof(double) * n_terms, cudaMemcpyDeviceToHost, stream),
               "D2H expectation values");
    cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
}

}  // namespace lqcs_b200
