/*
 * kettle_b200.h — C-ABI of the B200 circuit-propagation engine.
 *
 * Plain C, no torch or CUDA types in any signature: states are opaque handles,
 * gates and Pauli strings are flat records, all sizes are explicit.  Every
 * function returns an int32 status (KT_OK = 0, negative on error); the message
 * of the most recent error on the calling thread is returned by kt_last_error().
 * Device code never traps: failures surface as status codes.
 *
 * The entry points replace these reference interfaces (paths relative to the
 * kettle project root):
 *   kt_sv_apply          ket::simulate(const QuantumCircuit&, Statevector&, std::optional<int>)
 *                        include/kettle/simulation/simulate.hpp:41, loop at
 *                        source/kettle_internal/simulation/simulate.cpp:265-521
 *   kt_dm_apply          ket::simulate(const QuantumCircuit&, DensityMatrix&, std::optional<int>)
 *                        include/kettle/simulation/simulate_density_matrix.hpp:46
 *   kt_sv_expect         ket::expectation_value(const PauliOperator&, const Statevector&)
 *                        include/kettle/operator/pauli/pauli_operator.hpp:82-84,
 *                        source/kettle_internal/operator/pauli/pauli_operator.cpp:76-103
 *   kt_sv_probabilities  ket::calculate_probabilities_raw(const Statevector&, const QuantumNoise*)
 *                        include/kettle/calculations/probabilities.hpp:43
 *   kt_sv_sample         the sampler behind ket::perform_measurements_as_counts / _as_memory
 *                        include/kettle/calculations/measurements.hpp:41-97,
 *                        source/kettle_internal/calculations/measurements.cpp:235-311
 *   kt_sv_measure_probs / kt_sv_collapse
 *                        the M gate, source/kettle_internal/simulation/measure.hpp:34-55,
 *                        source/kettle_internal/simulation/measure.cpp:22-68
 *   kt_pairs_single / kt_pairs_double
 *                        ket::internal::SingleQubitGatePairGenerator / DoubleQubitGatePairGenerator
 *                        source/kettle_internal/simulation/gate_pair_generator.hpp:25-160
 *   kt_sv_inner          ket::inner_product, source/kettle_internal/state/state.cpp:159-172
 *   kt_sv_tensor_product ket::tensor_product(Statevector, Statevector), state/state.cpp:144-157
 *   kt_sv_diagonal_expectation  ket::diagonal_expectation_value, state/state.cpp:174-188
 *   kt_sample_probabilities     perform_measurements_as_* on a probability vector, measurements.cpp:58-159
 *   kt_dm_measure_probs / kt_dm_collapse  M on a DensityMatrix, measure_density_matrix.cpp:22-105
 *   kt_adjoint_*         no reference counterpart (new capability; the consumer is the
 *                        VQE cost function of example/algorithms/vqe_basic.cpp:61-96)
 *   kt_batch_*           no reference counterpart (new capability)
 */
#ifndef KETTLE_B200_H
#define KETTLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define KT_OK 0
#define KT_ERR_INVALID (-1)      /* bad argument (qubit out of range, null pointer, ...) */
#define KT_ERR_CUDA (-2)         /* a CUDA runtime call failed                          */
#define KT_ERR_NOMEM (-3)        /* device allocation failed                            */
#define KT_ERR_QUBITS (-4)       /* circuit / state qubit-count mismatch                */
#define KT_ERR_TIMEOUT (-5)      /* a bounded device wait ran out                       */
#define KT_ERR_UNSUPPORTED (-6)  /* valid request this build does not implement         */

/* ---- amplitude storage types ----------------------------------------- */
#define KT_C128 0 /* complex<double>: interleaved (re, im) doubles */
#define KT_C64 1  /* complex<float>:  interleaved (re, im) floats; reductions stay FP64 */

/* ---- gate record -------------------------------------------------------
 * `op` is the numeric value of ket::Gate (include/kettle/gates/primitive_gate.hpp:19-52):
 *   H=0 X=1 Y=2 Z=3 S=4 SDAG=5 T=6 TDAG=7 SX=8 SXDAG=9 RX=10 RY=11 RZ=12 P=13
 *   CH=14 CX=15 CY=16 CZ=17 CS=18 CSDAG=19 CT=20 CTDAG=21 CSX=22 CSXDAG=23
 *   CRX=24 CRY=25 CRZ=26 CP=27 U=28 CU=29 M=30
 * It carries what ket::GateInfo carries (primitive_gate.hpp:71-79): target
 * (GateInfo::arg0 for one-target gates, arg1 for controlled gates), control,
 * angle (arg2), and the 2x2 unitary for U/CU (row-major, interleaved re/im:
 * u = {m00.re, m00.im, m01.re, m01.im, m10.re, m10.im, m11.re, m11.im}).
 * For M, `control` holds the classical bit index.
 * `param` >= 0 takes the angle from params[param] instead of `angle`; that is
 * how a circuit's ParameterID-bound gates are evaluated once per call
 * (source/kettle_internal/parameter/parameter_expression.cpp:84-99). */
#define KT_OP_H 0
#define KT_OP_X 1
#define KT_OP_Y 2
#define KT_OP_Z 3
#define KT_OP_S 4
#define KT_OP_SDAG 5
#define KT_OP_T 6
#define KT_OP_TDAG 7
#define KT_OP_SX 8
#define KT_OP_SXDAG 9
#define KT_OP_RX 10
#define KT_OP_RY 11
#define KT_OP_RZ 12
#define KT_OP_P 13
#define KT_OP_CH 14
#define KT_OP_CX 15
#define KT_OP_CY 16
#define KT_OP_CZ 17
#define KT_OP_CS 18
#define KT_OP_CSDAG 19
#define KT_OP_CT 20
#define KT_OP_CTDAG 21
#define KT_OP_CSX 22
#define KT_OP_CSXDAG 23
#define KT_OP_CRX 24
#define KT_OP_CRY 25
#define KT_OP_CRZ 26
#define KT_OP_CP 27
#define KT_OP_U 28
#define KT_OP_CU 29
#define KT_OP_M 30

typedef struct kt_gate {
    uint8_t op;
    uint8_t reserved0;
    uint16_t reserved1;
    uint32_t target;
    uint32_t control;
    int32_t param;
    double angle;
    double u[8];
} kt_gate; /* 88 bytes */

/* ---- Pauli string record -----------------------------------------------
 * ket::SparsePauliString (include/kettle/operator/pauli/sparse_pauli_string.hpp:42-125)
 * as bit masks: bit q of x_mask is set where the term is X or Y, bit q of
 * z_mask where it is Z or Y.  `phase` is ket::PauliPhase (PLUS_ONE=0,
 * PLUS_EYE=1, MINUS_ONE=2, MINUS_EYE=3; PAULI_PHASE_MAP at :32-37).
 * Applied to a basis state: P|i> = i^{#Y} (-1)^{popcount(i & z_mask)} |i ^ x_mask>,
 * with Y = [[0,-i],[i,0]] as in apply_y_gate (simulation/operations.cpp:32-44). */
typedef struct kt_pauli {
    uint64_t x_mask;
    uint64_t z_mask;
    int32_t phase;
    int32_t reserved;
} kt_pauli;

/* ---- errors / device ---------------------------------------------------- */
const char* kt_last_error(void);
int32_t kt_version(void);
int32_t kt_device_synchronize(void);

/* Draw n canonical uniforms with std::mt19937(seed) and
 * std::generate_canonical<double, 53> — exactly the draws the reference's
 * ProbabilitySampler_ makes (measurements.cpp:288-311, prng.cpp:9-19) before
 * scaling them by its distribution bound.  Host-only helper. */
int32_t kt_canonicals_mt19937(uint32_t seed, int64_t n, double* out);

/* Launch-shape knobs of the engine (no reference counterpart), set by the
 * autotuner (kettle_b200/autotune.py) or from KT_TUNING="name=value,...":
 *   fused_ctas_per_sm  1 or 2   (2) register budget of the fused block kernel
 *   fused_tile_bits    9..13    (12) tile qubits per fused block (complex128; complex64
 *                               one more); 13 runs 512-thread CTAs, one per SM
 *   fused_max_ops      1..256   (256) gates per fused block (also the batch engine's fusion depth)
 *   adjoint_fused      0 or 1   (1) fused adjoint blocks (1) or one kernel per gate (0)
 *   fold_permutations  0 or 1   (1) X / CX with every qubit in a tile folded into a
 *                               shared-memory transpose (1) or run as ops (0)
 *   c64_renormalize    0 or 1   (1) complex64 applies rescale every fused block to the
 *                               norm the state had when the apply began (1)
 *   plan_lookahead     0, 1, 2  (1) each fused block's tile qubits chosen among the
 *                               greedy tile and tiles pinned to the qubits the next
 *                               gates need most, by the gates it and the next block
 *                               (2, or states of >= plan_deep_qubits index bits: the
 *                               next two blocks) take
 *   plan_deep_qubits   1..64    (28) see plan_lookahead
 *   plan_schedule      0..3     (3) inside a fused block, a gate whose qubits are
 *                               free of unplaced earlier gates runs as soon as its
 *                               target is a register bit of the current layout
 *                               phase, so a shared-memory transpose comes only when
 *                               no such gate is left (1..3; 0: the gates' given
 *                               order); at a transpose the next register set holds
 *                               the bits used soonest (1) or is built bit by bit to
 *                               take the most gates before the next one (2, 3); with
 *                               3 a block's first set is built from the bits above
 *                               the 128-byte runs when that takes any gate, so the
 *                               tile loads without a transpose
 *   fused_jit          0, 1, 2  (2) fused blocks as kernels compiled at run
 *                               time (NVRTC, cached per block structure: gate bodies
 *                               as straight-line code, every slot and mask a
 *                               constant): 0 never, 1 always, 2 (default) once a
 *                               circuit structure has been applied often enough to
 *                               repay the compile (jit_after) on states of
 *                               >= jit_min_qubits qubits, or after kt_sv_prepare /
 *                               kt_dm_prepare (a prepared structure runs compiled
 *                               at any size);
 *                               without NVRTC, or if a compile fails, the
 *                               precompiled kernels run (kt_jit_stats)
 *   jit_after          0..1e6   (0) the apply at which fused_jit = 2 compiles; 0 estimates
 *                               it from the state size and the host's threads (>= 2)
 *   jit_min_qubits     1..64    (26) the state size from which fused_jit = 2 compiles
 *   jit_ctas_per_sm    2..4     (2) CTAs per SM of compiled 256- or 128-thread blocks
 *   jit_prefetch       0 or 1   (1) each CTA prefetches its next tile into L2
 *   jit_merge_diag     0 or 1   (1) a phase's diagonal gates on thread / tile-external
 *                               qubits applied as one per-thread factor
 *   jit_skip_io        0, 1, 2  (2) load / store in the first / last compute layout
 *                               instead of through a transpose: 1 always, 2 only
 *                               where that layout keeps the lowest tile qubits on
 *                               the lowest thread bits (whole 128-byte runs per
 *                               group of lanes), 0 never
 *   jit_async_load     0 or 1   (0) next tile copied with cp.async into a second
 *                               shared-memory buffer (where two tiles fit a CTA)
 *   jit_fence          0..64    (0) every k gates, an empty asm pins the amplitudes
 *   jit_remat          0 or 1   (1) the thread index passes through an empty asm at
 *                               the top of every tile, so the terms derived from it
 *                               are recomputed per tile rather than held in
 *                               registers across the tile loop (fewer spills)
 *   jit_scale_ops      0 or 1   (1) complex128 compiled blocks run uncontrolled
 *                               gates divided by m00 != 0: real ones with
 *                               m11 = +-m00 (H, RY) and RX-like ones at one FMA per
 *                               component, general ones at 12 FP64 operations per
 *                               pair instead of 16, two-sided diagonals (RZ) as
 *                               one-sided; the block's product of those m00 scales
 *                               one unscaled uncontrolled gate of the block (or
 *                               every amplitude before the store); below 1e-150 the
 *                               apply runs on the precompiled kernels
 *   jit_lean_sync      0 or 1   (1) a compiled block's transpose into a phase that
 *                               stores where it loads (no permutation folded into
 *                               it) skips its second barrier: each thread's next
 *                               writes go to the slots it read itself
 *   adjoint_jit        0, 1, 2  (2) fused adjoint blocks as kernels compiled at run
 *                               time (NVRTC: gradient terms and U^dagger bodies as
 *                               straight-line code): 0 never, 1 always, 2 from the
 *                               second backward sweep of a circuit structure;
 *                               adjoint plans are cached by structure
 *   jit_tma            0 or 1   (0) complex128 compiled blocks (no renormalisation) as
 *                               persistent kernels of one CTA per SM: a producer
 *                               warp moves every tile between HBM and shared
 *                               memory with tensor copies (cp.async.bulk.tensor,
 *                               128-byte swizzle, mbarrier completion, bulk-group
 *                               stores) and jit_tma_stages tile buffers in flight,
 *                               while one thread group computes a tile; a bounded
 *                               wait that runs out makes the next C call return
 *                               KT_ERR_TIMEOUT
 *   jit_tma_stages     2..4     (3) tile buffers per CTA (the kernel must fit 227 KB
 *                               of shared memory)
 *   jit_tma_ctas       1 or 2   (1) TMA-pipelined CTAs per SM; with 2 each must fit
 *                               113 KB (e.g. 11-qubit tiles, 3 stages)
 *   batch_spin_limit   1..1e12  (33554432) polls of an empty job queue after which a
 *                               CTA of a batch's persistent kernel gives up (about
 *                               10 s): the evaluation then stops and
 *                               kt_batch_evaluate returns KT_ERR_TIMEOUT; the value
 *                               is taken when the batch is created (its graph)
 *   batch_small_max_qubits 0..13 (13) batch items of at most this many qubits
 *                               run whole in shared memory, one CTA each (within
 *                               11..12 for complex128 and 12..13 for complex64: what
 *                               fits, and an HBM item needs a whole forward tile);
 *                               taken when the batch is created
 *   batch_jit_min_qubits 0..64 (13) batch items in HBM with at least this many
 *                               qubits run run-time compiled block kernels (one
 *                               launch per block for all items of one plan
 *                               structure) instead of the persistent kernel's
 *                               interpreted blocks; 0: never.  Taken when the batch
 *                               is created; needs NVRTC and one memory wave
 *   fused_reg_bits     3 or 4   (4) complex128 amplitudes per thread in fused blocks
 *                               (2^4; or 2^3 with twice the warps: 12-qubit tiles of
 *                               512 threads, 2 CTAs per SM, or 11-qubit tiles of 256
 *                               threads, 3 CTAs per SM, by fused_tile_bits)
 * Unknown names return KT_ERR_INVALID. */
int32_t kt_tuning_set(const char* name, int64_t value);
int32_t kt_tuning_get(const char* name, int64_t* value);
/* Host-only, complex128: per fused block of an apply of n_qubits, four doubles
 * {ops, layout phases, transposes, FP64 instructions per amplitude of the
 * compiled block (a model of its gate bodies)}; up to `capacity` blocks are
 * written, n_blocks gets the count.  Instrumentation (new): it gives each
 * block's compute bounds beside its HBM bound. */
int32_t kt_plan_blocks(int32_t n_qubits, const kt_gate* gates, int64_t n_gates, const double* params,
                       int64_t n_params, double* out, int64_t capacity, int64_t* n_blocks);
/* Run-time compiled block kernels so far, fused-block launches through them,
 * and 1 if run-time compilation was unavailable or failed (new). */
int32_t kt_jit_stats(int64_t* kernels_compiled, int64_t* block_launches, int32_t* failed);
/* Host-only: programs this process has compiled with NVRTC, and programs it
 * took as cubins from the on-disk cache instead (new).  The cache is on when
 * the environment variable KT_JIT_CACHE_DIR names a directory: every compiled
 * cubin is kept there under a hash of its source, the embedded device
 * headers, the compile options and NVRTC's version, and a later process that
 * generates the same source loads it (a file whose second hash or content
 * hash does not match is compiled again and replaced). */
int32_t kt_jit_cache_stats(int64_t* nvrtc_compiles, int64_t* disk_hits);
/* Host-only: plan an apply of n_qubits in `dtype` and compile its block kernels
 * with NVRTC without loading them (no GPU needed); n_kernels = blocks compiled.
 * With adjoint_jit = 1 it compiles instead the fused adjoint blocks of the
 * circuit's backward sweep (gates reversed, every parameterised rotation a
 * gradient row). */
int32_t kt_jit_compile_only(int32_t n_qubits, int32_t dtype, const kt_gate* gates, int64_t n_gates,
                            const double* params, int64_t n_params, int64_t* n_kernels);

/* ---- statevector handle --------------------------------------------------
 * A statevector of n qubits lives on the current CUDA device as 2^n amplitudes,
 * little-endian (bit q of the index = qubit q), contiguous.  kt_sv_create
 * allocates it and sets |0...0> (Statevector(n), state.cpp:21-28). */
typedef struct kt_sv_s* kt_sv;

int32_t kt_sv_create(int32_t n_qubits, int32_t dtype, kt_sv* out);
/* Non-owning handle over caller memory (e.g. a torch tensor's data pointer). */
int32_t kt_sv_wrap(void* device_amps, int32_t n_qubits, int32_t dtype, kt_sv* out);
int32_t kt_sv_destroy(kt_sv sv);
/* All work of this handle is ordered on `stream` (a cudaStream_t; NULL = legacy default). */
int32_t kt_sv_set_stream(kt_sv sv, void* stream);
int32_t kt_sv_info(kt_sv sv, int32_t* n_qubits, int32_t* dtype, void** device_amps);
/* Set |index> (Statevector(std::string), state.cpp:55-66). */
int32_t kt_sv_set_basis(kt_sv sv, uint64_t index);
/* Host amplitudes are always complex128, interleaved; converted on the device for KT_C64. */
int32_t kt_sv_upload(kt_sv sv, const double* host_amps, uint64_t n_amps);
int32_t kt_sv_download(kt_sv sv, double* host_amps, uint64_t n_amps);
int32_t kt_sv_copy(kt_sv dst, kt_sv src);

/* Apply a gate stream.  mode: 0 = fused (default), 1 = one sweep per gate.
 * M gates are rejected here (they need a host coin; use kt_sv_measure_probs
 * and kt_sv_collapse).  Returns KT_ERR_INVALID for a qubit outside [0, n). */
#define KT_APPLY_FUSED 0
#define KT_APPLY_PER_GATE 1
int32_t kt_sv_apply(kt_sv sv, const kt_gate* gates, int64_t n_gates,
                    const double* params, int64_t n_params, int32_t mode);
/* Compile the fused block kernels of this circuit for `sv` now (new), so that
 * every later kt_sv_apply of a circuit with the same structure (any parameter
 * values) on a state of this size and dtype runs them from its first apply;
 * without it they are compiled once a circuit has been applied often enough to
 * repay the compile (fused_jit = 2).  Returns KT_ERR_CUDA when run-time
 * compilation is unavailable (applies then use the precompiled kernels). */
int32_t kt_sv_prepare(kt_sv sv, const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params);

/* Host-only dry run of the fused planner (no device work, no reference
 * counterpart): the fused blocks, layout phases, gates placed in blocks (X /
 * CX folded into transposes included) and shared-memory transposes
 * kt_sv_apply would use for this gate stream on n_qubits. */
int32_t kt_plan_stats(int32_t n_qubits, int32_t dtype, const kt_gate* gates, int64_t n_gates,
                      const double* params, int64_t n_params, int64_t* blocks, int64_t* phases,
                      int64_t* ops, int64_t* transposes);

/* Host-only, like kt_plan_stats: the fused planner's gates in the order they
 * take effect (blocks in order; in a block, each layout phase's gates, then
 * the X / CX folded into its transpose).  Entries index `gates` (M is not
 * accepted, as in kt_plan_stats).  *count receives the length; KT_ERR_INVALID
 * if it exceeds capacity.  Empty when the state is too small for fused
 * blocks.  No reference counterpart. */
int32_t kt_plan_order(int32_t n_qubits, int32_t dtype, const kt_gate* gates, int64_t n_gates,
                      const double* params, int64_t n_params, int64_t* order, int64_t capacity,
                      int64_t* count);

/* What the most recent kt_sv_apply / kt_dm_apply on this handle launched:
 * kernel launches and the algorithmic HBM bytes they move (read + write of
 * the amplitudes each launch must touch).  Instrumentation; no reference
 * counterpart. */
int32_t kt_sv_apply_stats(kt_sv sv, int64_t* launches, double* alg_bytes);

/* <psi| sum_k c_k P_k |psi>; coeffs interleaved complex128 (nullable = all 1).
 * out_terms (nullable): per-string phase*<P_k> (complex, interleaved);
 * out_total: sum_k c_k phase_k <P_k>, complex, as the reference returns. */
int32_t kt_sv_expect(kt_sv sv, const kt_pauli* strings, int64_t n_strings,
                     const double* coeffs, double* out_terms, double* out_total);

/* Allocation-free variant of kt_sv_expect (no counterpart in the reference).
 * For callers that cannot let the library call cudaMalloc: a host that keeps
 * all device memory in its own pool or arena, or a loop that must not
 * allocate once running.  It takes the amplitudes as a raw device pointer
 * (2^n_qubits elements of `dtype`, on the current device), computes the
 * per-string values and weighted total of kt_sv_expect (bit for bit on GPUs
 * of up to 148 SMs, such as a B200, where both add the same 4-per-SM block
 * partials in the same order; within FP64 rounding on larger ones), and keeps
 * its scratch in one fixed device array inside the library (about 2.5 MB,
 * held by every GPU that loads the library until the process exits), so it
 * calls no cudaMalloc or cudaFree.  At most KT_NOALLOC_MAX_STRINGS strings per call;
 * more is rejected with KT_ERR_INVALID.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  All calls share the one
 * array, so calls that overlap on the GPU (other streams, other host threads)
 * race; order them on one stream.  Returns after the results are on the host. */
#define KT_NOALLOC_MAX_STRINGS 512
int32_t kt_sv_expect_noalloc(const void* device_amps, int32_t n_qubits, int32_t dtype,
                             const kt_pauli* strings, int64_t n_strings, const double* coeffs,
                             double* out_terms, double* out_total, void* stream);

/* |a_i|^2 with the reference's rounding (no FMA), then optional per-qubit
 * readout noise applied qubit by qubit (probabilities.cpp:49-71,110-124).
 * noise: n doubles in [0,1] or NULL.  host_out: 2^n doubles. */
int32_t kt_sv_probabilities(kt_sv sv, const double* noise, double* host_out);

/* Inverse-CDF sampling.  canonicals[s] in [0,1) are scaled by the reference's
 * bound (cdf_last - offset, measurements.cpp:235-256,288-295) and searched
 * with lower_bound semantics.  The result equals the reference's sequential
 * std::partial_sum CDF bit for bit: the device certifies each draw against a
 * rigorous rounding bound and recomputes with an exact sequential scan when
 * a draw cannot be certified (mode 0); mode 1 always uses the sequential scan.
 * n_rescanned (nullable) reports whether the sequential scan ran (0/1). */
int32_t kt_sv_sample(kt_sv sv, const double* noise, const double* canonicals,
                     int64_t n_shots, uint64_t* out_indices, int32_t mode,
                     int32_t* n_rescanned);

/* M gate, split at the host coin: P(0), P(1) of `qubit`; then keep `outcome`
 * and scale by `scale` (the reference uses sqrt(1/P(outcome))). */
int32_t kt_sv_measure_probs(kt_sv sv, uint32_t qubit, double* p0, double* p1);
int32_t kt_sv_collapse(kt_sv sv, uint32_t qubit, int32_t outcome, double scale);

int32_t kt_sv_norm_sq(kt_sv sv, double* out);
int32_t kt_sv_inner(kt_sv bra, kt_sv ket, double* out_re_im);
/* |left> (x) |right> into `out` (n_left + n_right qubits, the same dtype): the
 * left state's qubits are the low ones, out[i_l + i_r 2^n_left] =
 * left[i_l] right[i_r].  Replaces ket::tensor_product(const Statevector&,
 * const Statevector&) (state/statevector.hpp:115, state/state.cpp:144-157). */
int32_t kt_sv_tensor_product(kt_sv left, kt_sv right, kt_sv out);
/* sum_i conj(psi_i) lambda_i psi_i in FP64 for a diagonal operator given by its
 * 2^n complex eigenvalues (interleaved doubles, host).  Replaces
 * ket::diagonal_expectation_value (state/statevector.hpp:119,
 * state/state.cpp:174-188); the sum is taken in another order, so the result
 * agrees within FP64 rounding. */
int32_t kt_sv_diagonal_expectation(kt_sv sv, const double* eigenvalues, double* out_re_im);
/* A dense unitary U on qubits 0..4 of a complex64 state of 12 to 34 qubits,
 * psi <- (I (x) U) psi, as a GEMM on the tensor cores (tcgen05): u is U as
 * 32 x 32 complex entries, row-major, interleaved doubles, U[b][a] mapping
 * basis state a to b.  passes = 3 splits both operands into TF32 parts
 * (hi rounded to nearest, lo the remainder) and sums three TF32 products in
 * FP32, passes = 4 adds the fourth (lo lo): about FP32 accuracy; passes = 1
 * is one plain TF32 product (10-bit mantissas, about 1e-3 relative error).  New: it
 * measures where a dense block on the tensor cores pays against the gate
 * bodies of the fused blocks; the fused planner does not call it. */
int32_t kt_sv_apply_dense5(kt_sv sv, const double* u, int32_t passes);
/* Shots from a caller's probability vector (n doubles, host): the sampler of
 * kt_sv_sample on those values, bit-exact to the reference's sequential CDF
 * and lower_bound (calculations/measurements.cpp:58-159, the
 * perform_measurements_as_* overloads taking std::vector<double>).  `stream`
 * may be NULL; device scratch is allocated for the call and freed after it. */
int32_t kt_sample_probabilities(const double* probabilities, uint64_t n, const double* canonicals,
                                int64_t n_shots, uint64_t* out_indices, int32_t mode, void* stream);

/* ---- pair enumeration (reference order, bit-exact) --------------------------
 * Pairs k0 .. k0+count-1 of SingleQubitGatePairGenerator(t, n).next() and of
 * DoubleQubitGatePairGenerator(c, t, n).next() (`quad` = 0, 2 indices per pair)
 * or .next_unset_and_set() (`quad` = 1, 4 indices), computed on the device
 * by bit arithmetic; host_out receives 2 (or 4) uint64 per pair. */
int32_t kt_pairs_single(uint32_t n_qubits, uint32_t target, uint64_t k0,
                        uint64_t count, uint64_t* host_out);
int32_t kt_pairs_double(uint32_t n_qubits, uint32_t control, uint32_t target,
                        int32_t quad, uint64_t k0, uint64_t count,
                        uint64_t* host_out);

/* ---- density matrix handle ------------------------------------------------
 * rho is N x N (N = 2^n) complex, column-major (element (r, c) at r + c*N) as
 * ket::DensityMatrix's Eigen::MatrixXcd (density_matrix.hpp:109).  It is kept
 * as a 2n-qubit vector: U on qubit q acts on index bit q and conj(U) on bit
 * q + n, which is U rho U^dagger (simulate_density_matrix.cpp:42-548). */
typedef struct kt_dm_s* kt_dm;

int32_t kt_dm_create(int32_t n_qubits, int32_t dtype, kt_dm* out);
int32_t kt_dm_destroy(kt_dm dm);
int32_t kt_dm_set_stream(kt_dm dm, void* stream);
/* rho = |index><index| (DensityMatrix(std::string), density_matrix.cpp:139-148). */
int32_t kt_dm_set_basis(kt_dm dm, uint64_t index);
int32_t kt_dm_upload(kt_dm dm, const double* host_colmajor, uint64_t n_elems);
int32_t kt_dm_download(kt_dm dm, double* host_colmajor, uint64_t n_elems);
int32_t kt_dm_apply(kt_dm dm, const kt_gate* gates, int64_t n_gates,
                    const double* params, int64_t n_params, int32_t mode);
/* kt_sv_prepare for a density matrix (new): plan the 2n-bit gate stream that
 * kt_dm_apply of these gates runs and compile its fused block kernels now, so
 * every apply of the same circuit structure runs them from the first. */
int32_t kt_dm_prepare(kt_dm dm, const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params);
/* Tr(P_k rho) per string and sum_k c_k phase_k Tr(P_k rho) (new: the reference
 * has no density-matrix expectation value). */
int32_t kt_dm_expect(kt_dm dm, const kt_pauli* strings, int64_t n_strings,
                     const double* coeffs, double* out_terms, double* out_total);
int32_t kt_dm_trace(kt_dm dm, double* out_re_im);
/* diagonal of rho as probabilities (for sampling a density matrix) */
int32_t kt_dm_probabilities(kt_dm dm, double* host_out);
/* Partial trace over `n_traced` distinct qubits of `src` into `dst`, which
 * has n - n_traced qubits and src's dtype (n_traced == n leaves the trace in
 * a 0-qubit, 1 x 1 matrix).  `qubits` lists the traced qubits in the order
 * they are traced out; sums are grouped like tracing them one at a time in
 * that order.  Replaces ket::partial_trace (state/density_matrix.hpp:127,
 * state/density_matrix.cpp:231-278), whose front end traces the highest index
 * first. */
int32_t kt_dm_partial_trace(kt_dm src, const int32_t* qubits, int32_t n_traced, kt_dm dst);
/* rho_left (low qubits) (x) rho_right (high qubits) into dst of
 * n_left + n_right qubits: ket::tensor_product (state/density_matrix.cpp:187-214). */
int32_t kt_dm_tensor_product(kt_dm left, kt_dm right, kt_dm dst);
/* Tr(rho^2), FP64: ket::DensityMatrix::trace_of_square (state/density_matrix.hpp:98-104). */
int32_t kt_dm_trace_of_square(kt_dm dm, double* out_re_im);
/* kt_sv_apply_stats for a density matrix's most recent kt_dm_apply (instrumentation). */
int32_t kt_dm_apply_stats(kt_dm dm, int64_t* launches, double* alg_bytes);
/* M gate on a density matrix, split at the host coin like the statevector's:
 * P(b) = sum |rho(r, c)|^2 over the rows r and columns c whose bit `qubit` is
 * b (the reference's definition); then keep outcome o: the (o, o) block
 * scaled by `scale` (the reference uses sqrt(1 / P(o))), the other three
 * blocks cleared.  Replaces simulation/measure_density_matrix.cpp:22-105. */
int32_t kt_dm_measure_probs(kt_dm dm, uint32_t qubit, double* p0, double* p1);
int32_t kt_dm_collapse(kt_dm dm, uint32_t qubit, int32_t outcome, double scale);

/* ---- adjoint differentiation (new) -------------------------------------------
 * E(theta) = <psi(theta)| H |psi(theta)>, psi = U_G ... U_1 |psi0>.
 * kt_adjoint_forward runs the circuit on `sv` and returns Re E (FP64);
 * kt_adjoint_backward then returns dE/dparams[j] for every parameter slot
 * (gates bound through kt_gate.param; literal gates contribute nothing),
 * sweeping the gates backwards with one FP64 inner product per
 * parameterised gate.  `work` needs room for two more statevectors of the
 * same size (lambda and a scratch); checkpoint_every > 0 stores a copy of
 * the forward state every that many gates when memory allows and restores
 * psi from it on the way back instead of relying on un-applying alone. */
typedef struct kt_adjoint_s* kt_adjoint;
int32_t kt_adjoint_create(kt_sv sv, int32_t checkpoint_every, kt_adjoint* out);
int32_t kt_adjoint_destroy(kt_adjoint adj);
int32_t kt_adjoint_forward(kt_adjoint adj, const kt_gate* gates, int64_t n_gates,
                           const double* params, int64_t n_params,
                           const kt_pauli* strings, int64_t n_strings,
                           const double* coeffs, double* energy);
int32_t kt_adjoint_backward(kt_adjoint adj, double* grad, int64_t n_params);

/* ---- batches (new) -------------------------------------------------------------
 * Many independent circuits, each with its own qubit count (1..30), gate
 * list, parameter slots and Hamiltonian, every one starting from |0...0>:
 * E_b = Re <psi_b| sum_k c_k P_k |psi_b> and, with gradients, dE/dparams.
 * Item b's gates bind parameter slot s (kt_gate.param) to
 * params[param_offset + s].  grads[p] is the sum of dE_b/dparams[p] over all
 * items whose gates bind p: with disjoint parameter ranges that is each
 * item's own gradient.  Gradients assume real coefficients (Hermitian H).
 * M gates are rejected.  No reference counterpart.
 *
 * kt_batch_create plans every item once (angles stay symbolic), allocates all
 * device memory, and captures one evaluation as a CUDA graph: parameter
 * upload, a kernel that writes the gate matrices from the parameters, one
 * persistent launch for items whose two states fit in shared memory
 * (q <= 12 complex128, q <= 13 complex64), one persistent launch per memory
 * wave for the others, FP64 finalisation and the download.
 * kt_batch_evaluate replays it on the batch's stream and returns when the
 * results are on the host; KT_ERR_TIMEOUT if a bounded device wait ran out.
 * kt_batch_run = create + evaluate + destroy. */
typedef struct kt_batch_item {
    int32_t n_qubits;
    int32_t reserved;
    int64_t gate_offset;   /* into the gates array   */
    int64_t n_gates;
    int64_t param_offset;  /* into params / grads    */
    int64_t n_params;
    int64_t string_offset; /* into strings / coeffs  */
    int64_t n_strings;
} kt_batch_item;

typedef struct kt_batch_s* kt_batch;
int32_t kt_batch_create(const kt_batch_item* items, int64_t n_items,
                        const kt_gate* gates, int64_t n_gates_total,
                        int64_t n_params_total, const kt_pauli* strings,
                        const double* coeffs, int64_t n_strings_total,
                        int32_t dtype, int32_t with_grad, kt_batch* out);
int32_t kt_batch_set_stream(kt_batch b, void* stream);
/* params: n_params_total values; energies: n_items; grads (nullable; needs
 * with_grad): n_params_total. */
int32_t kt_batch_evaluate(kt_batch b, const double* params, double* energies,
                          double* grads);
/* What the batch was planned into (instrumentation): shared-memory and HBM
 * items, memory waves, jobs (fused blocks and Hamiltonian passes), work
 * units, kernel launches per evaluation, algorithmic HBM bytes per
 * evaluation, device bytes held. */
int32_t kt_batch_stats(kt_batch b, int64_t* small_items, int64_t* large_items,
                       int64_t* waves, int64_t* jobs, int64_t* units,
                       int64_t* launches, double* alg_bytes, double* device_bytes);
/* HBM items that run run-time compiled block kernels (batch_jit_min_qubits):
 * the plan-structure classes they form (one launch per block per class) and
 * how many items those hold (instrumentation). */
int32_t kt_batch_compiled(kt_batch b, int64_t* classes, int64_t* items);
int32_t kt_batch_destroy(kt_batch b);

int32_t kt_batch_run(const kt_batch_item* items, int64_t n_items,
                     const kt_gate* gates, int64_t n_gates_total,
                     const double* params, int64_t n_params_total,
                     const kt_pauli* strings, const double* coeffs,
                     int64_t n_strings_total, int32_t dtype,
                     double* energies, double* grads, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* KETTLE_B200_H */
