// kt_internal.cuh — internal declarations shared by the engine's translation units.
//
// Layout in HBM: a statevector of n qubits is 2^n amplitudes, contiguous,
// little-endian (bit q of the index is qubit q), stored as interleaved
// (re, im) pairs: double2 for complex128, float2 for complex64.  A density
// matrix of n qubits is the same thing over 2n index bits (row bits 0..n-1,
// column bits n..2n-1), i.e. Eigen's column-major element order.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "kettle_b200.h"
#include "kt_complex.cuh"

namespace kt
{

// ---------------------------------------------------------------------------
// errors
void set_error(int32_t code, const std::string& msg);
int32_t cuda_fail(cudaError_t e, const char* where);
const char* last_error_cstr();
// replace this thread's error text with an already formatted message (one
// captured on another thread)
void set_error_text(const std::string& text);

#define KT_CUDA(call)                                   \
    do {                                                \
        cudaError_t kt_e_ = (call);                     \
        if (kt_e_ != cudaSuccess) {                     \
            return ::kt::cuda_fail(kt_e_, #call);       \
        }                                               \
    } while (0)

#define KT_CHECK_LAUNCH(where)                          \
    do {                                                \
        cudaError_t kt_e_ = cudaGetLastError();         \
        if (kt_e_ != cudaSuccess) {                     \
            return ::kt::cuda_fail(kt_e_, where);       \
        }                                               \
    } while (0)

// ---------------------------------------------------------------------------
// device state
struct DevBuf
{
    void* ptr {nullptr};
    size_t bytes {0};
    // grow-only scratch; contents are not preserved across growth
    int32_t reserve(size_t need);
    void release();
};

struct State
{
    int n_bits {0};          // index bits (n for a statevector, 2n for a density matrix)
    int dtype {KT_C128};
    void* amps {nullptr};
    bool owned {false};
    cudaStream_t stream {nullptr};
    DevBuf scratch;          // reductions, CDF, plans
    DevBuf scratch2;
    bool force_jit {false};      // fused applies run compiled blocks whatever fused_jit's size rule says
    int64_t last_launches {0};   // kernels launched by the last apply
    double last_alg_bytes {0.0};  // algorithmic bytes of the last apply
    uint64_t n_amps() const { return uint64_t {1} << n_bits; }
    size_t amp_bytes() const { return dtype == KT_C128 ? 16 : 8; }
};

// ---------------------------------------------------------------------------
// lowered gates: what the kernels consume.  Angles are resolved, matrices
// built once on the host (the reference recomputes cos/sin for every pair,
// simulation/operations.cpp:116-117).
enum GateKind : int32_t
{
    KIND_GEN = 0,   // general 2x2
    KIND_DIAG = 1,  // diag(m00, m11)
    KIND_ANTI = 2,  // [[0, m01], [m10, 0]]
};

struct LGate
{
    int32_t kind;
    int32_t target;
    int32_t control;   // -1 = none
    int32_t flags;     // bit0: m00 == 1 exactly (DIAG gates that leave |0> alone)
    double m[8];       // row-major interleaved complex: m00, m01, m10, m11
};

// Build the matrix of one gate record (the reference's matrices,
// gates/common_u_gates.cpp) and classify it.  Returns KT_OK or an error.
int32_t lower_gate(const kt_gate& g, const double* params, int64_t n_params, int n_qubits, LGate* out);
int32_t lower_gates(const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params,
                    int n_qubits, std::vector<LGate>& out);

// conj(U) on (t + shift, c + shift): the column half of U rho U^dagger.
LGate conj_shifted(const LGate& g, int shift);

// Analytic dU/dtheta (row-major interleaved, like LGate::m) of the rotation
// gates RX/RY/RZ/P and their controlled forms at angle th; false (d = 0) for
// every other op.
bool gate_derivative(int op, double th, double* d);

// GEN_* (kt_complex.cuh) of a gate op, or -1 when it has no angle
int gate_generator(int op);

// ---------------------------------------------------------------------------
// kernels (launchers return KT_OK or a CUDA error status)
int32_t launch_set_basis(State& s, uint64_t index);
int32_t launch_convert_to_state(State& s, const double* dev_c128, uint64_t n);     // c128 staging -> state
int32_t launch_convert_from_state(const State& s, double* dev_c128, uint64_t n);   // state -> c128 staging
int32_t launch_gate_sweep(State& s, const LGate& g);
double sweep_alg_bytes(const State& s, const LGate& g);
int32_t launch_pairs(uint32_t n, uint32_t c, uint32_t t, int kind, uint64_t k0, uint64_t count, uint64_t* dev_out,
                     cudaStream_t stream);

// fused blocks
struct FusedPlan;
int32_t apply_fused(State& s, const std::vector<LGate>& gates);
// adjoint sweep gates, in backward order: U^dagger, the generator of a
// parameterised rotation (gate_generator) and the gradient row (-1: none)
struct AdjGate
{
    LGate adj;
    int32_t gen;
    int32_t row;
};
// un-apply `gates` to psi and lambda with fused blocks; dev_grad[row] = 2 Re <lambda|D psi>
int32_t adjoint_sweep_fused(State& psi, State& lam, const std::vector<AdjGate>& gates, double* dev_grad, DevBuf& work);
// run-time compiled block kernels (kt_jit.cpp): compile each source (which may
// include "kt_fused_dev.cuh") for sm_100a and return its kernels `names[i]`
bool jit_available(std::string* why);
// host threads a run-time compile uses
int jit_threads();
// (load = false: compile only, no device needed)
// (owned: the loaded programs go there for the caller to unload, instead of
// the process-wide list jit_unload_all empties)
int32_t jit_compile(const std::vector<std::string>& sources, const std::vector<std::vector<std::string>>& names,
                    std::vector<std::vector<const void*>>& kernels, bool load = true,
                    std::vector<cudaLibrary_t>* owned = nullptr);
// A plan of the batch engine handed to the generator as raw records of the
// fused planner's types (FBlock, FPhase, and FOp<T> or FOpA<T>), which both
// translation units define alike; rec_bytes guards against a mismatch.
struct BatchPlanView
{
    const void* blocks {nullptr};
    int64_t n_blocks {0};
    const void* phases {nullptr};
    int64_t n_phases {0};
    const void* ops {nullptr};
    int64_t n_ops {0};
    int64_t rec_bytes[3] {0, 0, 0};  // sizeof FBlock, FPhase, op record
};
// Batched compiled block kernels of the batch engine: for every forward plan
// one kernel per block, (void* const* states, const unsigned char* const*
// op_records, unsigned long long n_tiles), blockIdx.y the item; for every
// adjoint plan one per block, (void* const* psi, void* const* lambda, const
// unsigned char* const* op_records, const long long* partial_base, double*
// partial, unsigned long long n_tiles, int n_rows).  Identical kernels are
// compiled once; fwd_smem / bwd_smem get each kernel's dynamic shared memory
// (set as its limit on the current device); the programs go to `libs`.
int32_t jit_batch_compile(int32_t dtype, const std::vector<BatchPlanView>& fwd, const std::vector<BatchPlanView>& bwd,
                          std::vector<std::vector<const void*>>& fk, std::vector<std::vector<const void*>>& bk,
                          std::vector<int32_t>& fwd_smem, std::vector<std::vector<int32_t>>& bwd_smem,
                          std::vector<cudaLibrary_t>& libs);
// host-only: plan an apply and compile its block kernels without loading them
int32_t jit_compile_only(int n, int32_t dtype, const std::vector<LGate>& gates, int64_t* n_kernels);
// host-only: plan the fused adjoint sweep `gates` and compile its block kernels
int32_t jit_adjoint_compile_only(int n, int32_t dtype, const std::vector<AdjGate>& gates, int64_t* n_kernels);
// a tensor map (written to `out`, 128 bytes) over `rows` rows of `row_floats`
// float32 each, boxes of box_rows x box_floats with the 128-byte swizzle;
// false when the driver entry point is missing or rejects the geometry
bool tma_encode_rows_f32(void* base, uint64_t row_floats, uint64_t rows, uint32_t box_floats, uint32_t box_rows,
                         void* out);
// the device's error word set by kernels whose bounded waits ran out (and its
// pinned host copy, which jit_async_error reads); nullptr on failure
unsigned int* async_error_word(int dev, unsigned int** host);
// KT_ERR_TIMEOUT (once) if a TMA block kernel's bounded wait ran out in an
// apply whose error word has reached the host since the last call; KT_OK otherwise
int32_t jit_async_error();
// unload every program jit_compile loaded (their kernels become invalid)
void jit_unload_all();
// compile the fused block kernels of `gates` on this state now (kt_sv_prepare)
int32_t jit_prepare(State& s, const std::vector<LGate>& gates);
// kernels compiled so far, block launches through them, and whether compiling failed
void jit_stats(int64_t* compiled, int64_t* launches, int32_t* failed);
// NVRTC compiles run in this process, and cubins taken from KT_JIT_CACHE_DIR instead
void jit_cache_stats(int64_t* nvrtc_compiles, int64_t* disk_hits);
// host-only: what the fused planner makes of a gate stream; *order (if given)
// receives the planned gates in the order they take effect
int32_t plan_blocks(int n, const std::vector<LGate>& gates, std::vector<double>& out);
int32_t plan_stats(int n, int32_t dtype, const std::vector<LGate>& gates, int64_t* blocks, int64_t* phases,
                   int64_t* ops, int64_t* transposes, std::vector<int32_t>* order = nullptr);

// reductions
int32_t expect_paulis(State& s, const kt_pauli* strings, int64_t n_strings, const double* coeffs,
                      double* out_terms, double* out_total);
int32_t dm_expect_paulis(State& s, int n_qubits, const kt_pauli* strings, int64_t n_strings, const double* coeffs,
                         double* out_terms, double* out_total);
int32_t norm_sq(State& s, double* out);
int32_t inner_product(State& bra, State& ket, double* out);
int32_t measure_probs(State& s, uint32_t q, double* p0, double* p1);
int32_t collapse(State& s, uint32_t q, int32_t outcome, double scale);
int32_t probabilities(State& s, const double* noise, double* host_out);
int32_t sample(State& s, const double* noise, const double* canonicals, int64_t n_shots, uint64_t* out, int32_t mode,
               int32_t* n_rescanned);
int32_t dm_trace(State& s, int n_qubits, double* out);
int32_t dm_diagonal(State& s, int n_qubits, double* host_out);
// density-matrix operations (kt_dm_ops.cu); `traced` in trace order, distinct
int32_t dm_partial_trace(const State& src, int n_qubits, const int32_t* traced, int n_traced, State& dst);
int32_t dm_tensor_product(const State& left, int n_left, const State& right, int n_right, State& dst);
int32_t dm_trace_of_square(State& s, int n_qubits, double* out);

// pin-memory staging helper for host <-> device copies
int32_t copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t st);
int32_t copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t st);

constexpr int SM_COUNT_B200 = 148;
int sm_count();

// Launch-shape knobs chosen by the autotuner (kettle_b200/autotune.py) and
// set through kt_tuning_set, or from KT_TUNING="name=value,..." at first use.
struct Tuning
{
    int fused_ctas_per_sm {2};   // register budget of the fused kernel: 2 (<=128 regs) or 1
    int fused_tile_bits {12};    // K for complex128 (complex64 uses K + 1), clamped to the kernel's range
    int fused_max_ops {256};     // gates per fused block
    int adjoint_fused {1};       // 1: fused backward blocks, 0: one kernel per gate
    int fold_permutations {1};   // 1: X / CX inside a tile become part of a transpose, 0: ops
    int c64_renormalize {1};     // 1: complex64 applies keep the state's norm (per-block rescaling)
    int fused_reg_bits {4};      // complex128 amplitudes per thread in fused blocks: 2^4, or 2^3 (more warps)
    int plan_schedule {3};       // 1: a block's gates run in the dependency order that saves transposes; 2: and each
                                 // new register set is the one that takes the most gates; 3: and the first set
                                 // avoids the 128-byte run bits when it takes gates; 0: the given order
    int plan_deep_qubits {28};   // states of at least this many index bits plan three blocks deep
    int plan_lookahead {1};      // 1: a block's tile may be pinned to the qubits the next gates need most
    int fused_jit {2};           // complex128 blocks as run-time compiled kernels: 0 never, 1 always,
                                 // 2 from a plan's second apply on >= jit_min_qubits qubits
    int jit_min_qubits {26};
    int jit_after {0};           // fused_jit = 2 compiles at this apply of a plan (0: estimated, >= 2)
    int jit_prefetch {1};        // 1: run-time compiled blocks prefetch their CTA's next tile into L2
    int jit_ctas_per_sm {2};     // CTAs per SM of run-time compiled blocks: 2..4
    int jit_merge_diag {1};      // 1: a phase's diagonal ops on thread / tile-external bits as one factor
    int jit_skip_io {2};         // 1: no transpose into a block's load layout or out of its store layout;
                                 // 2: only where that layout still moves whole 128-byte runs
    int jit_async_load {0};      // 1: run-time compiled blocks load the next tile with cp.async into a second buffer
    int jit_fence {0};           // k > 0: run-time compiled blocks fence the amplitudes every k ops
    int jit_scale_ops {1};       // complex128 blocks: uncontrolled real / RX-like ops divided by m00 (one FMA per component)
    int jit_remat {1};           // 1: thread-index terms recomputed every tile, not held across the tile loop
    long long batch_spin_limit {1LL << 25};  // polls of the batch queue before a CTA gives up (~10 s)
    int batch_small_max_qubits {13};         // batch items of at most this many qubits run in shared memory
                                             // (capped at 12 for complex128, 13 for complex64: what fits)
    int batch_jit_min_qubits {13};           // batch HBM items of at least this many qubits run compiled
                                             // block kernels shared by every item of one plan structure (0: never)
    int adjoint_jit {2};         // fused adjoint blocks as run-time compiled kernels: 0 never, 1 always,
                                 // 2 from the second backward sweep of a circuit structure
    int jit_lean_sync {1};       // 1: compiled blocks drop a transpose's second barrier where the phase stores where it loaded
    int jit_tma {0};             // 1: complex128 compiled blocks move tiles with TMA tensor copies, pipelined
    int jit_tma_stages {3};      // TMA blocks: shared-memory tile buffers per CTA (2..4)
    int jit_tma_ctas {1};        // TMA blocks: CTAs per SM (1 or 2: each within half the shared memory)
};
Tuning& tuning();
bool tuning_set(const char* name, long long value);
bool tuning_get(const char* name, long long* value);

}  // namespace kt

// the opaque handles of the C-ABI
struct kt_sv_s
{
    kt::State st;
};

struct kt_dm_s
{
    kt::State st;  // 2n index bits
    int n {0};
};
