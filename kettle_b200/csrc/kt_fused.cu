// kt_fused.cu — fused gate blocks: many gates per HBM pass.
//
// The reference sweeps the whole state once per gate (simulation/simulate.cpp:40-262).
// Here a host planner cuts the gate stream into blocks.  A block fixes a set
// Q of K "tile" qubits (always including the lowest L qubits, so a tile is
// made of 2^L-amplitude contiguous runs: 128 B); every tile (all 2^K
// amplitudes sharing the bits outside Q) is loaded once, all the block's gates
// are applied on chip, and the tile is stored once.
//
//  * A gate needs its target in Q only when it mixes amplitudes (non-diagonal).
//    Diagonal gates (Z, S, T, RZ, P, CZ, CP, CRZ, ...) and controls may sit on
//    any qubit: outside Q their bit is constant over a tile.
//  * Gates may move ahead of earlier gates they share no qubit with, so a block
//    takes every gate it can reach before a conflicting one.
//  * Inside a tile each thread holds R = 2^RB amplitudes in registers.  A
//    layout maps the K tile bits onto RB register bits and K-RB thread bits.
//    A non-diagonal gate is applied in registers when its target is a register
//    bit; the planner groups the block's gates into phases with a fixed
//    register set (chosen by next use) and a shared-memory transpose between
//    phases.  Shared memory is XOR-swizzled (a linear map, so addresses are
//    XORs of per-bit terms) and the lane bits are chosen so the transposes are
//    free of bank conflicts.
//  * Everything that depends only on the layout is resolved on the host: for
//    each gate the register slot of its target, a bit mask of the registers
//    whose control bit is set, the thread-index bits of a control or a diagonal
//    target that is a thread bit.  The kernel does no per-amplitude index math.
//  * Loads and stores use a layout whose lane bits are the L lowest qubits:
//    each warp instruction touches whole 128-byte lines.
#include <algorithm>
#include <cstddef>
#include <complex>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <thread>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>

#include <cuda.h>

#include "kt_fused.cuh"

namespace kt
{

namespace
{

// SHAPE: 2 = 256 threads, 2 CTAs per SM (<= 128 registers); 1 = 256 threads,
// 1 CTA per SM (the compiler's natural allocation); 0 = 512 threads, 1 CTA
// per SM (<= 128 registers: the tiles of 13 complex128 / 14 complex64 qubits).
// Complex128 with 8 amplitudes per thread (fused_reg_bits = 3): 3 = 512
// threads, 2 CTAs per SM (12-qubit tiles, <= 64 registers); 4 = 256 threads,
// 3 CTAs per SM (11-qubit tiles, <= 80 registers).
#define KT_FUSED_BOUNDS(SHAPE)                                                                 \
    __launch_bounds__(((SHAPE) == 0 || (SHAPE) == 3) ? 512 : 256,                               \
                      (SHAPE) == 0 ? 1 : ((SHAPE) == 3 ? 2 : ((SHAPE) == 4 ? 3 : (SHAPE))))

// register bits (amplitudes per thread = 2^RB) of a launch shape
template <typename T, int SHAPE>
struct ShapeCfg
{
    using type = Cfg<T>;
};
template <typename T>
struct ShapeCfg<T, 3>
{
    using type = Cfg3;
};
template <typename T>
struct ShapeCfg<T, 4>
{
    using type = Cfg3;
};

inline int fused_ctas(int shape)
{
    return shape == 2 ? 2 : (shape == 3 ? 2 : (shape == 4 ? 3 : 1));
}

// dynamic shared memory a launch shape may use: the tile plus MAX_OPS_PER_BLOCK op records
inline int fused_smem_limit(int shape)
{
    return shape == 0 ? 160 * 1024 : (shape == 4 ? 72 * 1024 : 96 * 1024);
}

template <typename T, int MINB>
__global__ void KT_FUSED_BOUNDS(MINB) k_fused(typename CxT<T>::type* __restrict__ a, const FBlock* __restrict__ blk,
                                                  const FPhase* __restrict__ phases, const FOp<T>* __restrict__ ops,
                                                  uint64_t n_tiles)
{
    using C = typename CxT<T>::type;
    constexpr int RB = ShapeCfg<T, MINB>::type::RB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ FBlock bk;
    __shared__ FPhase sph[MAX_PHASES_PER_BLOCK];
    const uint32_t t = threadIdx.x;
    if (t == 0) {
        bk = *blk;
    }
    __syncthreads();
    C* sm = reinterpret_cast<C*>(smem_raw);
    FOp<T>* sops = reinterpret_cast<FOp<T>*>(smem_raw + (sizeof(C) << bk.K));
    stage_block(bk, phases, ops, sph, sops, t);
    __syncthreads();
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        fwd_tile<T, RB, false>(a, bk, sph, sops, tile, sm, t, false);
    }
}

// Renormalisation of a complex64 apply: the norm must not drift with the
// FP32 rounding of thousands of gates, so every block rescales what it loads
// to the norm the state had when the apply began (the target: FP64 sums of
// |a|^2 that the first block takes over what it loads).  Each launch leaves,
// per CTA, the FP64 sum of |a|^2 over what it stored; the next launch scales
// its loads by sqrt(target / that), and a last short pass scales the result.
template <typename T, int MINB>
__global__ void KT_FUSED_BOUNDS(MINB) k_fused_norm(typename CxT<T>::type* __restrict__ a,
                                                       const FBlock* __restrict__ blk,
                                                       const FPhase* __restrict__ phases, const FOp<T>* __restrict__ ops,
                                                       uint64_t n_tiles, NormArgs na)
{
    using C = typename CxT<T>::type;
    constexpr int RB = Cfg<T>::RB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ FBlock bk;
    __shared__ FPhase sph[MAX_PHASES_PER_BLOCK];
    __shared__ double w_in[16], w_out[16];
    __shared__ float scale_sh;
    const uint32_t t = threadIdx.x;
    if (t == 0) {
        bk = *blk;
        scale_sh = (na.prev != nullptr) ? static_cast<float>(norm_scale(na.target, na.prev, na.n_parts)) : 1.0f;
    }
    if (t < 16) {
        w_in[t] = 0.0;
        w_out[t] = 0.0;
    }
    __syncthreads();
    C* sm = reinterpret_cast<C*>(smem_raw);
    FOp<T>* sops = reinterpret_cast<FOp<T>*>(smem_raw + (sizeof(C) << bk.K));
    stage_block(bk, phases, ops, sph, sops, t);
    __syncthreads();
    const NormCtx nc {na.in_parts != nullptr ? w_in : nullptr, w_out, scale_sh};
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        fwd_tile<T, RB, false, true>(a, bk, sph, sops, tile, sm, t, false, &nc);
    }
    __syncthreads();
    if (t == 0) {
        double so = 0.0, si = 0.0;
        for (int w = 0; w < 16; ++w) {
            so += w_out[w];
            si += w_in[w];
        }
        na.out_parts[blockIdx.x] = so;
        if (na.in_parts != nullptr) {
            na.in_parts[blockIdx.x] = si;
        }
    }
}

// the last step of a renormalising apply: a *= sqrt(target / last)
template <typename C>
__global__ void k_norm_final(C* __restrict__ a, uint64_t n, const double* __restrict__ target,
                             const double* __restrict__ last, int n_parts)
{
    __shared__ float sc;
    if (threadIdx.x == 0) {
        sc = static_cast<float>(norm_scale(target, last, n_parts));
    }
    __syncthreads();
    const float f = sc;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        C v = a[i];
        v.x *= f;
        v.y *= f;
        a[i] = v;
    }
}

// the renormalising launch sequence of a complex64 apply (see k_fused_norm)
template <typename T>
int32_t run_fused_norm(State& s, const Plan<T>& plan, const FBlock* d_blk, const FPhase* d_ph, const FOp<T>* d_ops,
                       int K, int threads, int shape)
{
    using C = typename CxT<T>::type;
    static bool attr_set[3] = {false, false, false};
    if (!attr_set[shape]) {
        const int bytes = fused_smem_limit(shape);
        switch (shape) {
            case 0: KT_CUDA(cudaFuncSetAttribute(k_fused_norm<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)); break;
            case 1: KT_CUDA(cudaFuncSetAttribute(k_fused_norm<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)); break;
            default: KT_CUDA(cudaFuncSetAttribute(k_fused_norm<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)); break;
        }
        attr_set[shape] = true;
    }
    const int n = s.n_bits;
    const uint64_t n_tiles = uint64_t {1} << (n - K);
    const int grid = static_cast<int>(std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sm_count()) * fused_ctas(shape)));
    // per-CTA sums: target | out (even blocks) | out (odd blocks)
    if (const int32_t rc = s.scratch2.reserve(3 * static_cast<size_t>(grid) * sizeof(double)); rc != KT_OK) {
        return rc;
    }
    double* parts = static_cast<double*>(s.scratch2.ptr);
    double* target = parts;
    double* out[2] = {parts + grid, parts + 2 * grid};
    const double pass_bytes = 2.0 * static_cast<double>(sizeof(C)) * static_cast<double>(s.n_amps());
    for (size_t b = 0; b < plan.blocks.size(); ++b) {
        const auto& fb = plan.blocks[b];
        const size_t smem = (size_t {1} << K) * sizeof(C) + static_cast<size_t>(fb.op_end - fb.op_begin) * sizeof(FOp<T>);
        NormArgs na {};
        na.n_parts = grid;
        na.target = (b == 0) ? nullptr : target;
        na.prev = (b == 0) ? nullptr : out[(b - 1) & 1];
        na.in_parts = (b == 0) ? target : nullptr;
        na.out_parts = out[b & 1];
        C* a = static_cast<C*>(s.amps);
        switch (shape) {
            case 0: k_fused_norm<T, 0><<<grid, threads, smem, s.stream>>>(a, d_blk + b, d_ph, d_ops, n_tiles, na); break;
            case 1: k_fused_norm<T, 1><<<grid, threads, smem, s.stream>>>(a, d_blk + b, d_ph, d_ops, n_tiles, na); break;
            default: k_fused_norm<T, 2><<<grid, threads, smem, s.stream>>>(a, d_blk + b, d_ph, d_ops, n_tiles, na); break;
        }
        KT_CHECK_LAUNCH("k_fused_norm");
        s.last_launches += 1;
        s.last_alg_bytes += pass_bytes;
    }
    if (!plan.blocks.empty()) {
        const unsigned fin_grid = static_cast<unsigned>(std::min<uint64_t>((s.n_amps() + 255) / 256,
                                                                           static_cast<uint64_t>(sm_count()) * 8));
        k_norm_final<C><<<fin_grid, 256, 0, s.stream>>>(static_cast<C*>(s.amps), s.n_amps(), target,
                                                        out[(plan.blocks.size() - 1) & 1], grid);
        KT_CHECK_LAUNCH("k_norm_final");
        s.last_launches += 1;
        s.last_alg_bytes += pass_bytes;
    }
    return KT_OK;
}

// Block formation and planning of a forward apply (n >= Cfg<T>::RB + 5):
// tile size from fused_tile_bits, 8 amplitudes per thread for complex128
// when fused_reg_bits is 3 (12- or 11-qubit tiles).  A block whose phases
// overflow the kernel's table is re-formed with half the ops per block.
template <typename T>
int32_t fused_plan(int n, const std::vector<LGate>& gates, Plan<T>& plan, int* K_out, bool* rb3_out)
{
    constexpr int RB = Cfg<T>::RB;
    constexpr int L = Cfg<T>::L;
    const bool rb3 = std::is_same<T, double>::value && tuning().fused_reg_bits == 3 && n >= 12;
    int K = 0;
    if (rb3) {
        K = std::max(11, std::min(12, tuning().fused_tile_bits));
    } else {
        K = std::min(n, std::min(RB + TBMAX, tuning().fused_tile_bits + (RB - 4)));
    }
    size_t max_ops = static_cast<size_t>(std::min(MAX_OPS_PER_BLOCK, tuning().fused_max_ops));
    for (;;) {
        plan = Plan<T> {};
        const auto blocks = form_blocks(gates, n, K, L, max_ops);
        for (const auto& b : blocks) {
            if (rb3) {
                plan_block<T, Cfg3>(b, gates, n, plan);
            } else {
                plan_block<T>(b, gates, n, plan);
            }
        }
        bool fits = true;
        for (const auto& fb : plan.blocks) {
            if (fb.phase_end - fb.phase_begin > MAX_PHASES_PER_BLOCK) {
                fits = false;
            }
        }
        if (fits) {
            break;
        }
        if (max_ops <= 8) {
            set_error(KT_ERR_INVALID, "fused block planner produced too many phases");
            return KT_ERR_INVALID;
        }
        max_ops /= 2;
    }
    *K_out = K;
    *rb3_out = rb3;
    return KT_OK;
}

// ---------------------------------------------------------------------------
// Plan cache.  Planning depends on the gates' kinds, qubits and a few value
// classes (real, RX-like, pure X, diag(1, .)), not on the angles, so a
// circuit applied again with new parameters reuses its plan: the op records
// take the new matrices and nothing else changes.  Entries are keyed by that
// structure (and the planning knobs), checked in full on a hit.

uint32_t gate_class(const LGate& x)
{
    const double* m = x.m;
    const bool real = m[1] == 0.0 && m[3] == 0.0 && m[5] == 0.0 && m[7] == 0.0;
    const bool rxl = m[1] == 0.0 && m[7] == 0.0 && m[0] == m[6] && m[2] == 0.0 && m[4] == 0.0 && m[3] == m[5];
    // m00 != 0 and m11 = +-m00: the run-time compiled blocks may divide the
    // gate by m00 (jit_scaled), so these are part of the structure
    return static_cast<uint32_t>(x.kind) | (static_cast<uint32_t>(x.flags & 1) << 4) | (real ? 1u << 5 : 0u) |
           (rxl ? 1u << 6 : 0u) | (is_pure_x(x) ? 1u << 7 : 0u) | (m[0] != 0.0 ? 1u << 8 : 0u) |
           (m[6] == m[0] ? 1u << 9 : 0u) | (m[6] == -m[0] ? 1u << 10 : 0u);
}

template <typename T>
struct PlanEntry
{
    std::vector<uint64_t> signature;
    Plan<T> plan;
    int K {0};
    bool rb3 {false};
};

template <typename T>
struct PlanCache
{
    std::mutex m;
    std::unordered_map<uint64_t, PlanEntry<T>> entries;
};

template <typename T>
PlanCache<T>& plan_cache()
{
    static PlanCache<T> c;
    return c;
}

constexpr size_t PLAN_CACHE_MAX = 64;

// fused_plan through the cache; *key identifies the plan's structure
template <typename T>
int32_t fused_plan_cached(int n, const std::vector<LGate>& gates, Plan<T>& plan, int* K_out, bool* rb3_out,
                          uint64_t* key)
{
    const Tuning& tu = tuning();
    std::vector<uint64_t> sig;
    sig.reserve(gates.size() + 2);
    sig.push_back(static_cast<uint64_t>(n) | (static_cast<uint64_t>(sizeof(T)) << 8) |
                  (static_cast<uint64_t>(tu.fused_tile_bits) << 16) | (static_cast<uint64_t>(tu.fold_permutations) << 24) |
                  (static_cast<uint64_t>(tu.fused_reg_bits) << 28) | (static_cast<uint64_t>(tu.plan_lookahead) << 32) |
                  (static_cast<uint64_t>(tu.plan_deep_qubits) << 34) | (static_cast<uint64_t>(tu.plan_schedule) << 42) |
                  (static_cast<uint64_t>(tu.fused_max_ops) << 48));
    for (const LGate& x : gates) {
        sig.push_back(static_cast<uint64_t>(gate_class(x)) | (static_cast<uint64_t>(x.target & 0xFFFF) << 8) |
                      (static_cast<uint64_t>(x.control & 0xFFFF) << 24));
    }
    uint64_t h = 0xcbf29ce484222325ULL;
    for (const uint64_t v : sig) {
        h = (h ^ v) * 0x100000001b3ULL;
        h ^= h >> 29;
    }
    *key = h;
    PlanCache<T>& pc = plan_cache<T>();
    {
        std::lock_guard<std::mutex> lock(pc.m);
        auto it = pc.entries.find(h);
        if (it != pc.entries.end() && it->second.signature == sig) {
            plan = it->second.plan;
            *K_out = it->second.K;
            *rb3_out = it->second.rb3;
            for (size_t i = 0; i < plan.ops.size(); ++i) {
                const LGate& x = gates[static_cast<size_t>(plan.op_gate[i])];
                for (int e = 0; e < 8; ++e) {
                    plan.ops[i].m[e] = static_cast<T>(x.m[e]);
                }
            }
            return KT_OK;
        }
    }
    if (const int32_t rc = fused_plan<T>(n, gates, plan, K_out, rb3_out); rc != KT_OK) {
        return rc;
    }
    std::lock_guard<std::mutex> lock(pc.m);
    if (pc.entries.size() >= PLAN_CACHE_MAX) {
        pc.entries.clear();
    }
    PlanEntry<T>& e = pc.entries[h];
    e.signature = std::move(sig);
    e.plan = plan;
    e.K = *K_out;
    e.rb3 = *rb3_out;
    return KT_OK;
}

// ---------------------------------------------------------------------------
// Run-time compiled block kernels (fused_jit = 1, complex128).  A block's
// kernel is the k_fused tile loop with the block's gate bodies written out as
// straight-line code: the target and control register slots, the thread and
// tile masks are literals, so there is no op dispatch, the control predicates
// fold away (a controlled gate computes only its active pairs) and the
// register allocator sees the whole block.  Matrices are still read from the
// op records, so one compiled kernel serves every angle.  Kernels are cached
// by their source text for the life of the process.

std::string jit_hex(uint64_t v)
{
    char b[40];
    std::snprintf(b, sizeof(b), "0x%llxULL", static_cast<unsigned long long>(v));
    return b;
}

// asynchronous tile loads need a second tile buffer; only where both fit a CTA
inline bool jit_async(int K, size_t elem_bytes)
{
    return tuning().jit_async_load != 0 && 2 * (size_t {1} << K) * elem_bytes <= 227 * 1024;
}

// Batched block kernels (the batch engine's HBM items of one circuit
// structure): one launch runs a block on many states, blockIdx.y selecting
// the item.  Every item has its own state and its own op records (the batch
// writes their matrices from the parameters on the device), so the
// generated code reads an op's matrix from the item's record at a literal
// byte offset instead of a kernel parameter; scaled forms, which need the
// matrices on the host, are off.  Set for the duration of a generation.
struct JitBatch
{
    size_t op_bytes {0};  // bytes of one op record
    size_t m_off {0};     // byte offset of the matrix in a record
};
thread_local const JitBatch* tl_batch = nullptr;

struct JitBatchScope
{
    explicit JitBatchScope(const JitBatch* b) { tl_batch = b; }
    ~JitBatchScope() { tl_batch = nullptr; }
    JitBatchScope(const JitBatchScope&) = delete;
    JitBatchScope& operator=(const JitBatchScope&) = delete;
};

// the text of matrix entry e of op j of the block being generated
template <typename T>
std::string jit_mref(int j, int e)
{
    if (tl_batch != nullptr) {
        const size_t off = static_cast<size_t>(j) * tl_batch->op_bytes + tl_batch->m_off + static_cast<size_t>(e) * sizeof(T);
        return "kt_ldm<$T>(ob, " + std::to_string(off) + "u)";
    }
    return "M.m[" + std::to_string(8 * j + e) + "]";
}

// Scaled forms of the run-time compiled blocks (complex128, jit_scale_ops).
// An uncontrolled op may run divided by its m00 != 0:
//   1 / 2  real with m11 = +m00 / -m00:  [[1, p], [q, +-1]]
//   3      RX-like [[c, i s], [i s, c]]: [[1, i t], [i t, 1]]
//   4      general complex:              [[1, p], [q, r]]
//   5      diagonal [d0, d1]:            [1, d1 / d0]
// The block's product of the m00 they drop multiplies one uncontrolled op
// that is not scaled and scales every amplitude it touches by the same
// factor (the sink: a general, anti-diagonal or diagonal op; a real one
// only when every factor is real), or, with no such op, every amplitude
// before the store (an extra matrix slot).
template <typename T>
int jit_scaled(const FOp<T>& op)
{
    if constexpr (!std::is_same<T, double>::value) {
        return 0;
    } else {
        if (tuning().jit_scale_ops == 0 || tl_batch != nullptr || op.cslot != NO_SLOT || op.cthr != 0 ||
            op.cglob != 0) {
            return 0;
        }
        const bool nz = op.m[0] != 0.0 || op.m[1] != 0.0;
        switch (op.kind) {
            case OP_GENR:
                return op.m[0] == 0.0 ? 0 : (op.m[6] == op.m[0] ? 1 : (op.m[6] == -op.m[0] ? 2 : 0));
            case OP_RXL:
                return op.m[0] != 0.0 ? 3 : 0;
            case OP_GEN:
                return nz ? 4 : 0;
            case OP_DIAG:
                return nz ? 5 : 0;
            default:
                return 0;
        }
    }
}

struct JitScale
{
    int sink {-1};         // op index within the block taking the factor (-1: none)
    bool any {false};      // some op of the block is scaled
    bool own_slot {false}; // the factor has its own matrix slot, applied before the store
};

template <typename T>
JitScale jit_scale_plan(const Plan<T>& plan, size_t b)
{
    const FBlock& fb = plan.blocks[b];
    const int nops = fb.op_end - fb.op_begin;
    auto op_at = [&](int j) -> const FOp<T>& { return plan.ops[static_cast<size_t>(fb.op_begin + j)]; };
    auto unctl = [](const FOp<T>& op) { return op.cslot == NO_SLOT && op.cthr == 0 && op.cglob == 0; };
    JitScale js;
    if constexpr (!std::is_same<T, double>::value) {
        return js;
    }
    if (tuning().jit_scale_ops == 0 || tl_batch != nullptr) {
        return js;
    }
    for (int j = 0; j < nops && js.sink < 0; ++j) {
        const FOp<T>& op = op_at(j);
        if (unctl(op) && (op.kind == OP_GEN || op.kind == OP_ANTI || op.kind == OP_DIAG)) {
            js.sink = j;
        }
    }
    bool cplx = false;
    for (int j = 0; j < nops; ++j) {
        const int sc = (j == js.sink) ? 0 : jit_scaled(op_at(j));
        js.any = js.any || sc != 0;
        cplx = cplx || sc >= 4;
    }
    for (int j = 0; j < nops && js.sink < 0 && !cplx; ++j) {
        const FOp<T>& op = op_at(j);
        if (unctl(op) && (op.kind == OP_GENR || op.kind == OP_RXL) && jit_scaled(op) == 0) {
            js.sink = j;
        }
    }
    js.own_slot = js.any && js.sink < 0;
    return js;
}

// the scaled form op j of block b runs in (0: none)
template <typename T>
int jit_scale_code(const Plan<T>& plan, size_t b, int j, const JitScale& js)
{
    return j == js.sink ? 0 : jit_scaled(plan.ops[static_cast<size_t>(plan.blocks[b].op_begin + j)]);
}

template <typename T>
void jit_emit_op(std::string& s, const FOp<T>& op, int j, int sc)
{
    const int cs = (op.cslot == NO_SLOT) ? -1 : op.cslot;
    auto run = [&](int ts) {
        return std::string("f.crt = ") + std::to_string(cs) + "; f.template run<" + std::to_string(ts) + ", " +
               (cs < 0 ? "-1" : "CS_RT") + ">();";
    };
    // the op's matrix entries: the kernel's constant-bank parameter (batched: the item's op record)
    auto m = [&](int e) { return jit_mref<T>(j, e); };
    auto cx = [&](int e) { return "make_cx<$T>(" + m(e) + ", " + m(e + 1) + ")"; };
    std::string guard;
    if (op.cglob != 0) {
        guard += "if ((base & " + jit_hex(op.cglob) + ") == " + jit_hex(op.cglob) + ") ";
    }
    if (op.cthr != 0) {
        guard += "if ((t & " + std::to_string(op.cthr) + "u) == " + std::to_string(op.cthr) + "u) ";
    }
    s += "        " + guard + "{\n            ";
    switch (op.kind) {
        case OP_GEN:
            if (sc == 4) {
                s += "GenSF<$T, RB> f {v, " + cx(2) + ", " + cx(4) + ", " + cx(6) + "}; " + run(op.tslot);
            } else {
                s += "GenF<$T, RB> f {v, " + cx(0) + ", " + cx(2) + ", " + cx(4) + ", " + cx(6) + "}; " + run(op.tslot);
            }
            break;
        case OP_GENR:
            if (sc == 1 || sc == 2) {
                s += std::string("GenRSF<$T, RB, ") + (sc == 2 ? "true" : "false") + "> f {v, " + m(2) + ", " + m(4) +
                     "}; " + run(op.tslot);
            } else {
                s += "GenRF<$T, RB> f {v, " + m(0) + ", " + m(2) + ", " + m(4) + ", " + m(6) + "}; " + run(op.tslot);
            }
            break;
        case OP_RXL:
            if (sc == 3) {
                s += "RxSF<$T, RB> f {v, " + m(3) + "}; " + run(op.tslot);
            } else {
                s += "RxF<$T, RB> f {v, " + m(0) + ", " + m(3) + "}; " + run(op.tslot);
            }
            break;
        case OP_ANTI:
            s += "AntiF<$T, RB, false> f {v, " + cx(2) + ", " + cx(4) + "}; " + run(op.tslot);
            break;
        case OP_SWAP:
            s += "AntiF<$T, RB, true> f {v, make_cx<$T>(1, 0), make_cx<$T>(1, 0)}; " + run(op.tslot);
            break;
        default: {
            const bool one = (op.kind == OP_DIAG1) || sc == 5;
            if (op.tslot != NO_SLOT) {
                s += std::string("DiagRegF<$T, RB, ") + (one ? "true" : "false") + "> f {v, " + cx(0) + ", " + cx(6) +
                     "}; " + run(op.tslot);
            } else {
                std::string b = "false";
                if (op.tthr != 0 && op.tglob != 0) {
                    b = "((t & " + std::to_string(op.tthr) + "u) != 0u) || ((base & " + jit_hex(op.tglob) + ") != 0ULL)";
                } else if (op.tthr != 0) {
                    b = "(t & " + std::to_string(op.tthr) + "u) != 0u";
                } else if (op.tglob != 0) {
                    b = "(base & " + jit_hex(op.tglob) + ") != 0ULL";
                }
                s += "const bool b = " + b + "; ";
                s += one ? "if (b) " : "";
                s += "{ DiagAllF<$T, RB> f {v, b ? " + cx(6) + " : " + cx(0) + "}; " + run(0) + " }";
            }
            break;
        }
    }
    s += "\n        }\n";
}

// sum over the bits j of `var` of bit_j * strides[j], strides powers of two:
// shift-and-mask runs of consecutive target bits
std::string jit_deposit(const std::string& var, const uint64_t* strides, int nbits)
{
    std::string e;
    int j = 0;
    while (j < nbits) {
        if (strides[j] == 0) {
            ++j;
            continue;
        }
        const int q = __builtin_ctzll(strides[j]);
        int len = 1;
        while (j + len < nbits && strides[j + len] == (uint64_t {1} << (q + len))) {
            ++len;
        }
        const uint64_t mask = (len >= 64) ? ~uint64_t {0} : ((uint64_t {1} << len) - 1);
        if (!e.empty()) {
            e += " | ";
        }
        e += "(((static_cast<uint64_t>(" + var + ") >> " + std::to_string(j) + ") & " + jit_hex(mask) + ") << " +
             std::to_string(q) + ")";
        j += len;
    }
    return e.empty() ? std::string("0ULL") : "(" + e + ")";
}

// XOR over the bits j of t of terms[j] (32-bit shared-memory address terms)
std::string jit_xor_terms(const uint32_t* terms, int nbits, uint32_t start)
{
    std::string e = std::to_string(start) + "u";
    for (int j = 0; j < nbits; ++j) {
        if (terms[j] != 0) {
            e += " ^ ((0u - ((t >> " + std::to_string(j) + ") & 1u)) & " + std::to_string(terms[j]) + "u)";
        }
    }
    return "(" + e + ")";
}

// ---------------------------------------------------------------------------
// TMA-pipelined block kernels (jit_tma, complex128).  The state is seen as a
// tensor of float64 whose dimensions follow the runs of consecutive qubits of a
// block's tile: dimension 0 is (re, im) x qubits 0..2 (one 128-byte row), each
// further dimension starts at the first qubit of a run and reaches the next
// run (the last one the top of the state), so one box of the tensor map is
// the tile, or, when the tile has more than four runs above qubit 2, the part
// of it with the highest runs' bits fixed (those copies differ only in the
// last dimension's coordinate).  Boxes land in shared memory with the 128-byte
// swizzle: amplitude l of the tile (bit j of l = the tile's j-th qubit) sits
// at slot l ^ ((l >> 3) & 7).
struct TmaGeom
{
    bool ok {false};
    int rank {0};
    uint64_t dim[5] {};        // extents (float64 elements for dimension 0)
    uint64_t stride[5] {};     // byte strides of dimensions 1..rank-1
    uint32_t box[5] {};        // box extents
    int start[5] {};           // first qubit of each dimension (0 for dimension 0)
    int copies {1};
    std::vector<uint32_t> copy_add;  // per copy: added to the last dimension's coordinate
    uint32_t box_bytes {0};
};

TmaGeom tma_geom(const FBlock& fb, int n)
{
    TmaGeom g;
    const int K = fb.K;
    if (K < 4 || fb.qubit[0] != 0 || fb.qubit[1] != 1 || fb.qubit[2] != 2) {
        return g;
    }
    std::vector<std::pair<int, int>> runs;  // (first qubit, length <= 8: a box extent <= 256)
    for (int j = 3; j < K;) {
        int len = 1;
        while (j + len < K && fb.qubit[j + len] == fb.qubit[j] + len && len < 8) {
            ++len;
        }
        runs.emplace_back(fb.qubit[j], len);
        j += len;
    }
    const int D = std::min<int>(4, static_cast<int>(runs.size()));
    g.rank = 1 + D;
    for (int r = 1; r <= D; ++r) {
        g.start[r] = runs[static_cast<size_t>(r - 1)].first;
    }
    auto end_of = [&](int r) { return r < D ? g.start[r + 1] : n; };
    g.dim[0] = uint64_t {2} << g.start[1];
    g.box[0] = 16;
    for (int r = 1; r <= D; ++r) {
        g.dim[r] = uint64_t {1} << (end_of(r) - g.start[r]);
        g.stride[r] = uint64_t {16} << g.start[r];
        g.box[r] = 1u << runs[static_cast<size_t>(r - 1)].second;
    }
    std::vector<int> extra;  // qubits of the runs above the fourth, ascending
    for (size_t r = static_cast<size_t>(D); r < runs.size(); ++r) {
        for (int k = 0; k < runs[r].second; ++k) {
            extra.push_back(runs[r].first + k);
        }
    }
    g.copies = 1 << extra.size();
    g.copy_add.assign(static_cast<size_t>(g.copies), 0u);
    for (int c = 0; c < g.copies; ++c) {
        for (size_t k = 0; k < extra.size(); ++k) {
            if ((c >> k) & 1) {
                g.copy_add[static_cast<size_t>(c)] |= 1u << (extra[k] - g.start[D]);
            }
        }
    }
    g.box_bytes = 128u << (K - 3 - static_cast<int>(extra.size()));
    g.ok = true;
    return g;
}

// slot of tile amplitude l in a stage buffer (the 128-byte swizzle, 16-byte amplitudes)
inline uint32_t tma_swz(uint32_t l)
{
    return l ^ ((l >> 3) & 7u);
}

// groups: thread groups computing a tile each per CTA.  Only 1 is used: a
// 544-thread form with two groups over three 12-qubit stage buffers failed
// with an unspecified launch failure on the 30-qubit benchmark (its cause was
// not found by reading the code), so it is not offered.
struct TmaCfg
{
    int groups {1};
    int stages {3};
    TmaGeom geom;
};

// The tile's coordinates in the tensor map: c[0] = 2 (base mod 2^start[1]),
// c[r] = the base's bits from start[r] up to the next dimension.
std::string tma_coord_code(const TmaGeom& g, const std::string& base, const std::string& out)
{
    std::string e;
    for (int r = 0; r < g.rank; ++r) {
        const int lo = g.start[r];
        const int hi = (r == 0) ? g.start[1] : lo + __builtin_ctzll(g.dim[r]);
        const uint64_t mask = (hi - lo >= 64) ? ~uint64_t {0} : ((uint64_t {1} << (hi - lo)) - 1);
        e += out + "[" + std::to_string(r) + "] = static_cast<int32_t>(((" + base + " >> " + std::to_string(lo) + ") & " +
             jit_hex(mask) + ")" + (r == 0 ? " << 1" : "") + ");\n";
    }
    return e;
}

// The body of block b's kernel (everything after its name): the tile loop
// with the layout of every phase written out as constants (tile base, thread
// and register offsets, swizzled shared-memory terms) and the gate bodies as
// straight-line code; matrices arrive in the constant-bank parameter M.
template <typename T>
std::string jit_block_body(const Plan<T>& plan, size_t b, int RB, bool norm, const TmaCfg* tma = nullptr)
{
    const FBlock& fb = plan.blocks[b];
    const int TB = fb.K - RB;
    const int R = 1 << RB;
    const int np = fb.phase_end - fb.phase_begin;
    const int nops = std::max(1, fb.op_end - fb.op_begin);
    const JitScale js = jit_scale_plan(plan, b);
    const bool scale_slot = js.own_slot;
    const FPhase* ph = plan.phases.data() + fb.phase_begin;
    std::vector<uint64_t> free_strides(static_cast<size_t>(std::max(1, fb.nfree)));
    for (int k = 0; k < fb.nfree; ++k) {
        free_strides[static_cast<size_t>(k)] = uint64_t {1} << fb.freebit[k];
    }
    auto reg_off = [&](const FPhase& f, int i) {
        uint64_t o = 0;
        for (int sl = 0; sl < RB; ++sl) {
            if (i & (1 << sl)) {
                o += f.rstride[sl];
            }
        }
        return o;
    };
    auto reg_xor = [&](const uint32_t* terms, int i) {
        uint32_t x = 0;
        for (int sl = 0; sl < RB; ++sl) {
            if (i & (1 << sl)) {
                x ^= terms[sl];
            }
        }
        return x;
    };
    std::string s;
    s.reserve(32768);
    // TMA variant: tile index bit of a phase's register slot / thread bit, and
    // its term in a stage buffer's (128-byte swizzled) slot index
    auto tile_bit = [&](uint64_t stride) {
        for (int k = 0; k < fb.K; ++k) {
            if (bit(fb.qubit[k]) == stride) {
                return k;
            }
        }
        return 0;
    };
    auto tma_reg_term = [&](const FPhase& f, int i) {
        uint32_t x = 0;
        for (int sl = 0; sl < RB; ++sl) {
            if (i & (1 << sl)) {
                x ^= tma_swz(1u << tile_bit(f.rstride[sl]));
            }
        }
        return x;
    };
    auto tma_thr_terms = [&](const FPhase& f) {
        std::vector<uint32_t> tt(static_cast<size_t>(std::max(1, TB)), 0u);
        for (int j = 0; j < TB; ++j) {
            tt[static_cast<size_t>(j)] = tma_swz(1u << tile_bit(f.tstride[j]));
        }
        return tt;
    };
    const int NG = tma ? tma->groups : 1;
    const int NS = tma ? tma->stages : 1;
    const int GT = 1 << TB;  // threads of one tile
    const size_t tile_bytes = (size_t {1} << fb.K) * sizeof(typename CxT<T>::type);
    if (tma) {
        s += "(const __grid_constant__ kt::KtTmap tm, void* a_, unsigned long long n_tiles, unsigned int* err_, "
             "const __grid_constant__ $M<" + std::to_string(8 * (nops + (scale_slot ? 1 : 0))) + "> M)\n{\n";
    } else if (tl_batch != nullptr) {
        s += "(void* const* a_list, const unsigned char* const* o_list, unsigned long long n_tiles)\n{\n";
    } else {
        s += std::string("(void* a_, unsigned long long n_tiles, ") + (norm ? "kt::NormArgs na, " : "") +
             "const __grid_constant__ $M<" + std::to_string(8 * (nops + (scale_slot ? 1 : 0))) + "> M)\n{\n";
    }
    s += "    using namespace kt;\n    using C = $C;\n";
    s += "    constexpr int RB = " + std::to_string(RB) + ";\n";
    if (tma) {
        const TmaGeom& g = tma->geom;
        const std::string NSs = std::to_string(NS) + "ull";
        const std::string TBYTES = std::to_string(tile_bytes) + "u";
        // stage buffers (1024-byte aligned for the swizzle), then the mbarriers:
        // full[s] (the tile's copies landed) and done[s] (its group finished it)
        s += "    (void)a_;\n";
        s += "    extern __shared__ __align__(1024) unsigned char smem_raw[];\n";
        s += "    unsigned char* stage0 = reinterpret_cast<unsigned char*>((reinterpret_cast<unsigned long long>(smem_raw) + "
             "1023ull) & ~1023ull);\n";
        s += "    uint64_t* full = reinterpret_cast<uint64_t*>(stage0 + " + std::to_string(NS * tile_bytes) + "u);\n";
        s += "    uint64_t* done = full + " + std::to_string(NS) + ";\n";
        s += "    if (threadIdx.x == 0) {\n        for (int k = 0; k < " + std::to_string(NS) +
             "; ++k) {\n            kt_mbar_init(full + k, 1);\n            kt_mbar_init(done + k, " + std::to_string(GT) +
             ");\n        }\n        kt_fence_mbar_init();\n    }\n    __syncthreads();\n";
        // the producer: one thread of the last warp issues every copy
        auto copies = [&](const std::string& tile_expr, const std::string& buf, bool load) {
            std::string e = "            {\n                const uint64_t pb = " +
                            jit_deposit(tile_expr, free_strides.data(), fb.nfree) + ";\n                int32_t c[" +
                            std::to_string(g.rank) + "];\n";
            std::string cc = tma_coord_code(g, "pb", "c");
            for (size_t at = 0; at < cc.size();) {
                const size_t nl = cc.find('\n', at);
                e += "                " + cc.substr(at, nl - at + 1);
                at = nl + 1;
            }
            const std::string last = "c[" + std::to_string(g.rank - 1) + "]";
            e += "                const int32_t c_last = " + last + ";\n";
            for (int k = 0; k < g.copies; ++k) {
                e += "                " + last + " = c_last + " + std::to_string(g.copy_add[static_cast<size_t>(k)]) + ";\n";
                const std::string dst = buf + " + " + std::to_string(static_cast<size_t>(k) * g.box_bytes) + "u";
                if (load) {
                    e += "                KtTma<" + std::to_string(g.rank) + ">::load(&tm, " + dst + ", full + st, c);\n";
                } else {
                    e += "                KtTma<" + std::to_string(g.rank) + ">::store(&tm, " + dst + ", c);\n";
                }
            }
            e += "            }\n";
            return e;
        };
        s += "    if (threadIdx.x >= " + std::to_string(NG * GT) + "u) {\n";
        s += "        if (threadIdx.x == " + std::to_string(NG * GT) + "u) {\n";
        s += "            unsigned long long i = 0;\n";
        s += "            for (;; ++i) {\n";
        s += "            const unsigned long long tile = blockIdx.x + i * gridDim.x;\n";
        s += "            if (tile >= n_tiles) {\n                break;\n            }\n";
        s += "            const uint32_t st = static_cast<uint32_t>(i % " + NSs + ");\n";
        s += "            unsigned char* buf = stage0 + st * " + TBYTES + ";\n";
        s += "            if (i >= " + NSs + ") {\n";
        s += "            // the buffer's previous tile: finished by its group, stored, read out of shared memory\n";
        s += "            kt_mbar_wait(done + st, static_cast<uint32_t>(((i / " + NSs + ") - 1ull) & 1ull), err_);\n";
        s += copies("(tile - " + NSs + " * gridDim.x)", "buf", false);
        s += "            kt_bulk_commit();\n            kt_bulk_wait_read0();\n            }\n";
        s += "            kt_mbar_arrive_expect_tx(full + st, " + TBYTES + ");\n";
        s += copies("tile", "buf", true);
        s += "            }\n";
        // the last tiles of each buffer: stored once finished; every load has landed
        s += "            for (unsigned long long j = (i > " + NSs + " ? i - " + NSs + " : 0ull); j < i; ++j) {\n";
        s += "            const uint32_t st = static_cast<uint32_t>(j % " + NSs + ");\n";
        s += "            unsigned char* buf = stage0 + st * " + TBYTES + ";\n";
        s += "            kt_mbar_wait(full + st, static_cast<uint32_t>((j / " + NSs + ") & 1ull), err_);\n";
        s += "            kt_mbar_wait(done + st, static_cast<uint32_t>((j / " + NSs + ") & 1ull), err_);\n";
        s += copies("(blockIdx.x + j * gridDim.x)", "buf", false);
        s += "            kt_bulk_commit();\n            }\n";
        s += "            kt_bulk_wait0();\n";
        s += "        }\n        return;\n    }\n";
        s += "    const uint32_t grp = threadIdx.x >> " + std::to_string(TB) + ";\n";
        s += "    const uint32_t t = threadIdx.x & " + std::to_string(GT - 1) + "u;\n";
        s += "    C* sm = nullptr;\n";
    } else {
        if (tl_batch != nullptr) {
            s += "    C* __restrict__ a = static_cast<C*>(a_list[blockIdx.y]);\n";
            s += "    const unsigned char* __restrict__ ob = o_list[blockIdx.y];\n";
        } else {
            s += "    C* __restrict__ a = static_cast<C*>(a_);\n";
        }
        s += "    extern __shared__ __align__(16) unsigned char smem_raw[];\n";
        s += "    C* sm = reinterpret_cast<C*>(smem_raw);\n";
        s += "    const uint32_t t = threadIdx.x;\n";
    }
    if (norm) {
        // renormalisation (complex64): per-warp FP64 sums of |a|^2 over the
        // loads (first block: the target) and the stores, loads scaled by
        // sqrt(target / what the previous block stored)
        s += "    __shared__ double w_in[16], w_out[16];\n    __shared__ float scale_sh;\n";
        s += "    if (t == 0) {\n        scale_sh = (na.prev != nullptr) ? static_cast<float>(norm_scale(na.target, na.prev, "
             "na.n_parts)) : 1.0f;\n    }\n";
        s += "    if (t < 16) {\n        w_in[t] = 0.0;\n        w_out[t] = 0.0;\n    }\n    __syncthreads();\n";
        s += "    const float sc = scale_sh;\n";
    }
    // A block's first phase may only set up the coalesced load layout (no ops,
    // no permutation to apply) and its last one only the store layout; then
    // the tile is loaded straight into the second phase's layout, or stored
    // from the one before last, and that transpose goes away (the accesses
    // of a warp still cover whole 128-byte lines across its instructions).
    auto identity_store = [&](const FPhase& f) {
        if (f.xor_out != 0) {
            return false;
        }
        for (int sl = 0; sl < RB; ++sl) {
            if (f.rsw_out[sl] != f.rsw[sl]) {
                return false;
            }
        }
        for (int j = 0; j < TB; ++j) {
            if (f.tsw_out[j] != f.tsw[j]) {
                return false;
            }
        }
        return true;
    };
    // jit_skip_io: 1 always loads (stores) the tile straight in the layout of
    // the first (last) compute phase; 2 only where that layout keeps the
    // lowest tile qubits on the lowest thread bits, so each group of lanes
    // still moves whole 128-byte runs (otherwise the io transpose stays)
    const int skip_mode = tuning().jit_skip_io;
    const bool skip_io = skip_mode != 0;
    const int L_run = (sizeof(typename CxT<T>::type) == 16) ? 3 : 4;
    auto coalesced = [&](const FPhase& f) {
        if (tma) {
            // read from / written to a stage buffer: free of bank conflicts when
            // the three lowest thread bits land on independent 16-byte slots
            // of a 128-byte row under the swizzle
            uint32_t g3[3] = {0, 0, 0};
            for (int j = 0; j < 3 && j < TB; ++j) {
                g3[j] = tma_swz(1u << tile_bit(f.tstride[j])) & 7u;
            }
            return g3[0] != 0 && g3[1] != 0 && g3[2] != 0 && g3[0] != g3[1] && g3[0] != g3[2] && g3[1] != g3[2] &&
                   (g3[0] ^ g3[1]) != g3[2];
        }
        if (skip_mode != 2) {
            return true;
        }
        for (int j = 0; j < L_run && j < TB; ++j) {
            if (f.tstride[j] != bit(fb.qubit[j])) {
                return false;
            }
        }
        return true;
    };
    // jit_fence = k: every k ops the amplitudes pass through an empty asm, so
    // the scheduler cannot interleave more than k ops (bounds the live registers)
    const int fence_every = tuning().jit_fence;
    const int first = ((skip_io || tma) && np > 1 && ph[0].op_begin == ph[0].op_end && identity_store(ph[0]) &&
                       coalesced(ph[1]))
                          ? 1
                          : 0;
    const int last = ((skip_io || tma) && np - 1 > first && ph[np - 1].op_begin == ph[np - 1].op_end &&
                      identity_store(ph[np - 2]) && coalesced(ph[np - 2]))
                         ? np - 2
                         : np - 1;
    // jit_async_load: each thread copies its next tile's amplitudes (in the
    // first layout) into its own slots of a second shared-memory buffer with
    // cp.async while the current tile computes; no other thread touches those
    // slots, so a wait_group is the only synchronisation.
    const bool async_load = !tma && jit_async(fb.K, sizeof(typename CxT<T>::type));
    const int n_thr = 1 << TB;
    auto issue_async = [&](const std::string& tile_expr, const std::string& indent) {
        std::string e;
        e += indent + "{\n" + indent + "    const C* src = a + " + jit_deposit(tile_expr, free_strides.data(), fb.nfree) +
             " + " + jit_deposit("t", ph[first].tstride, TB) + ";\n";
        e += indent + "    const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(sb + t));\n";
        // one amplitude per copy: 16 bytes (.cg, L2 only) for complex128, 8 bytes
        // (.ca, the only form for sizes below 16) for complex64; both addresses
        // are aligned to the amplitude size
        const size_t amp = sizeof(typename CxT<T>::type);
        const std::string op = (amp == 16) ? "cp.async.cg.shared.global [%0], [%1], 16;"
                                           : "cp.async.ca.shared.global [%0], [%1], 8;";
        for (int i = 0; i < R; ++i) {
            e += indent + "    asm volatile(\"" + op + "\" :: \"r\"(dst + " +
                 std::to_string(amp * static_cast<size_t>(i) * static_cast<size_t>(n_thr)) + "u), \"l\"(src + " +
                 std::to_string(reg_off(ph[first], i)) + "ULL) : \"memory\");\n";
        }
        e += indent + "}\n";
        return e;
    };
    if (async_load) {
        s += "    C* sb = sm + " + std::to_string(1 << fb.K) + ";\n";
        s += "    if (static_cast<unsigned long long>(blockIdx.x) < n_tiles) {\n";
        s += issue_async("static_cast<unsigned long long>(blockIdx.x)", "        ");
        s += "    }\n    asm volatile(\"cp.async.commit_group;\" ::: \"memory\");\n";
    }
    // jit_remat: the thread index passes through an empty asm at the top of
    // every tile, so the terms derived from it (swizzled shared-memory
    // offsets, thread masks, thread-bit deposits) are recomputed per tile
    // instead of being hoisted out of the loop and held in registers (which
    // made ptxas spill)
    const bool remat = tuning().jit_remat != 0;
    if (remat) {
        s += "    const uint32_t t_outer = t;\n";
    }
    if (tma) {
        // group grp takes the CTA's tiles grp, grp + NG, ...; tile it sits in stage it % NS
        s += "    for (unsigned long long it = grp;; it += " + std::to_string(NG) + "ull) {\n";
        s += "        const unsigned long long tile = blockIdx.x + it * gridDim.x;\n";
        s += "        if (tile >= n_tiles) {\n            break;\n        }\n";
        s += "        const uint32_t st = static_cast<uint32_t>(it % " + std::to_string(NS) + "ull);\n";
    } else {
        s += "    for (unsigned long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {\n";
    }
    if (remat) {
        s += "        uint32_t t_l;\n        asm volatile(\"mov.u32 %0, %1;\" : \"=r\"(t_l) : \"r\"(t_outer));\n";
        s += "        const uint32_t t = t_l;\n";
    }
    s += "        C v[1 << RB];\n";
    s += "        const uint64_t base = " + jit_deposit("tile", free_strides.data(), fb.nfree) + ";\n";
    if (tma) {
        // the tile's copies landed in stage st: read it in the first layout, then
        // the group's barrier before any thread writes the buffer again
        s += "        kt_mbar_wait(full + st, static_cast<uint32_t>((it / " + std::to_string(NS) + "ull) & 1ull), err_);\n";
        s += "        sm = reinterpret_cast<C*>(stage0 + st * " + std::to_string(tile_bytes) + "u);\n";
        const std::vector<uint32_t> tt = tma_thr_terms(ph[first]);
        s += "        {\n            const uint32_t lt = " + jit_xor_terms(tt.data(), TB, 0) + ";\n";
        for (int i = 0; i < R; ++i) {
            s += "            v[" + std::to_string(i) + "] = sm[lt ^ " + std::to_string(tma_reg_term(ph[first], i)) + "u];\n";
        }
        s += "        }\n";
        s += "        kt_bar_sync(1u + grp, " + std::to_string(GT) + "u);\n";
    } else if (async_load) {
        s += "        asm volatile(\"cp.async.wait_group 0;\" ::: \"memory\");\n";
        for (int i = 0; i < R; ++i) {
            s += "        v[" + std::to_string(i) + "] = sb[" + std::to_string(i * n_thr) + "u + t];\n";
        }
    } else {
        s += "        {\n            const C* src = a + base + " + jit_deposit("t", ph[first].tstride, TB) + ";\n";
        for (int i = 0; i < R; ++i) {
            s += "            v[" + std::to_string(i) + "] = src[" + std::to_string(reg_off(ph[first], i)) + "ULL];\n";
        }
        s += "        }\n";
    }
    if (norm) {
        s += "        if (na.in_parts != nullptr) {\n            warp_norm_add<float>(v, w_in, t);\n        }\n";
        s += "#pragma unroll\n        for (int i = 0; i < (1 << RB); ++i) {\n            v[i].x *= sc;\n            v[i].y *= sc;\n        }\n";
    }
    if (tuning().jit_prefetch != 0 && !async_load && !tma) {
        // the next tile of this CTA into L2 while this one computes: one
        // prefetch per 128-byte line when the lowest qubits are the low lanes
        const bool lines_on_lanes = TB >= 3 && ph[first].tstride[0] == 1 && ph[first].tstride[1] == 2 &&
                                    ph[first].tstride[2] == 4;
        s += std::string("        if (") + (lines_on_lanes ? "(t & 7u) == 0u && " : "") + "tile + gridDim.x < n_tiles) {\n";
        s += "            const C* nxt = a + " + jit_deposit("(tile + gridDim.x)", free_strides.data(), fb.nfree) + " + " +
             jit_deposit("t", ph[first].tstride, TB) + ";\n";
        for (int i = 0; i < R; ++i) {
            s += "            asm volatile(\"prefetch.global.L2 [%0];\" :: \"l\"(nxt + " + std::to_string(reg_off(ph[first], i)) +
                 "ULL));\n";
        }
        s += "        }\n";
    }
    // the barrier of a transpose: the whole CTA, or (TMA) the tile's own thread group
    const std::string tbar = tma ? "            kt_bar_sync(1u + grp, " + std::to_string(GT) + "u);\n"
                                 : "            __syncthreads();\n";
    for (int p = first; p <= last; ++p) {
        const FPhase& cur = ph[p];
        if (p > first) {
            const FPhase& prev = ph[p - 1];
            s += "        {\n            const uint32_t so = " + jit_xor_terms(prev.tsw_out, TB, prev.xor_out) + ";\n";
            for (int i = 0; i < R; ++i) {
                s += "            sm[so ^ " + std::to_string(reg_xor(prev.rsw_out, i)) + "u] = v[" + std::to_string(i) + "];\n";
            }
            s += tbar;
            s += "            const uint32_t lo = " + jit_xor_terms(cur.tsw, TB, 0) + ";\n";
            for (int i = 0; i < R; ++i) {
                s += "            v[" + std::to_string(i) + "] = sm[lo ^ " + std::to_string(reg_xor(cur.rsw, i)) + "u];\n";
            }
            // The barrier after the reads keeps the next transpose's writes from
            // overwriting slots other threads have not read yet.  When this
            // phase stores where it loaded (no permutation folded into its
            // store side), each thread's next writes go to exactly the slots
            // it read itself, so no other thread can still need them and the
            // barrier is dropped (jit_lean_sync) -- except after the tile's last
            // transpose, whose slots the next tile's first writes may reuse.
            const bool lean = tuning().jit_lean_sync != 0 && p < last && identity_store(cur);
            s += (lean ? std::string() : tbar) + "        }\n";
        }
        // Diagonal ops whose target (and controls, if any) are thread or
        // tile-external bits scale all of a thread's amplitudes by one factor;
        // they commute with every other op of the phase (those target register
        // bits), so a phase's several such ops become one product of factors
        // applied once, at the phase's end.
        std::vector<int> scal;
        for (int o = cur.op_begin; o < cur.op_end; ++o) {
            const FOp<T>& op = plan.ops[static_cast<size_t>(o)];
            if ((op.kind == OP_DIAG || op.kind == OP_DIAG1) && op.tslot == NO_SLOT && op.cslot == NO_SLOT) {
                scal.push_back(o);
            }
        }
        const bool merge = tuning().jit_merge_diag != 0 && scal.size() >= 2;
        int emitted = 0;
        for (int o = cur.op_begin; o < cur.op_end; ++o) {
            if (merge && std::find(scal.begin(), scal.end(), o) != scal.end()) {
                continue;
            }
            if (fence_every > 0 && emitted > 0 && emitted % fence_every == 0) {
                s += "        kt_jit_fence(v);\n";
            }
            jit_emit_op(s, plan.ops[static_cast<size_t>(o)], o - fb.op_begin, jit_scale_code(plan, b, o - fb.op_begin, js));
            ++emitted;
        }
        if (merge) {
            s += "        {\n            C fac = make_cx<$T>(1, 0);\n";
            for (const int o : scal) {
                const FOp<T>& op = plan.ops[static_cast<size_t>(o)];
                const int j = o - fb.op_begin;
                const bool one_sided = op.kind == OP_DIAG1 || jit_scale_code(plan, b, j, js) == 5;
                auto cx = [&](int e) { return "make_cx<$T>(" + jit_mref<T>(j, e) + ", " + jit_mref<T>(j, e + 1) + ")"; };
                std::string cond;
                if (op.cglob != 0) {
                    cond += "((base & " + jit_hex(op.cglob) + ") == " + jit_hex(op.cglob) + ")";
                }
                if (op.cthr != 0) {
                    cond += std::string(cond.empty() ? "" : " && ") + "((t & " + std::to_string(op.cthr) + "u) == " +
                            std::to_string(op.cthr) + "u)";
                }
                std::string b = "false";
                if (op.tthr != 0 && op.tglob != 0) {
                    b = "(((t & " + std::to_string(op.tthr) + "u) != 0u) || ((base & " + jit_hex(op.tglob) + ") != 0ULL))";
                } else if (op.tthr != 0) {
                    b = "((t & " + std::to_string(op.tthr) + "u) != 0u)";
                } else if (op.tglob != 0) {
                    b = "((base & " + jit_hex(op.tglob) + ") != 0ULL)";
                }
                s += "            ";
                if (!cond.empty()) {
                    s += "if (" + cond + ") ";
                }
                s += "{ const bool b = " + b + "; ";
                if (one_sided) {
                    s += "if (b) { fac = cmul(fac, " + cx(6) + "); } }\n";
                } else {
                    s += "fac = cmul(fac, b ? " + cx(6) + " : " + cx(0) + "); }\n";
                }
            }
            s += "            DiagAllF<$T, RB> f {v, fac}; f.template run<0, -1>();\n        }\n";
        }
        if (async_load && p == first) {
            // this thread's slots were read at the top of the tile; refill them
            s += "        if (tile + gridDim.x < n_tiles) {\n";
            s += issue_async("(tile + gridDim.x)", "            ");
            s += "        }\n        asm volatile(\"cp.async.commit_group;\" ::: \"memory\");\n";
        }
    }
    if (scale_slot) {
        // the factor the scaled ops dropped, with no other op to take it
        s += "        {\n            const C sc = make_cx<$T>(M.m[" + std::to_string(8 * nops) + "], M.m[" +
             std::to_string(8 * nops + 1) + "]);\n";
        for (int i = 0; i < R; ++i) {
            s += "            v[" + std::to_string(i) + "] = cmul(sc, v[" + std::to_string(i) + "]);\n";
        }
        s += "        }\n";
    }
    if (tma) {
        // the tile into its stage buffer in the tensor map's order, visible to
        // the TMA store the producer issues once the whole group has arrived
        const std::vector<uint32_t> tt = tma_thr_terms(ph[last]);
        s += "        {\n            const uint32_t lt = " + jit_xor_terms(tt.data(), TB, 0) + ";\n";
        for (int i = 0; i < R; ++i) {
            s += "            sm[lt ^ " + std::to_string(tma_reg_term(ph[last], i)) + "u] = v[" + std::to_string(i) + "];\n";
        }
        s += "        }\n        kt_fence_proxy_async_smem();\n        kt_mbar_arrive(done + st);\n";
    } else {
        s += "        {\n            C* dst = a + base + " + jit_deposit("t", ph[last].tstride, TB) + ";\n";
        for (int i = 0; i < R; ++i) {
            s += "            dst[" + std::to_string(reg_off(ph[last], i)) + "ULL] = v[" + std::to_string(i) + "];\n";
        }
        s += "        }\n";
    }
    if (norm) {
        s += "        warp_norm_add<float>(v, w_out, t);\n";
    }
    s += "    }\n";
    if (norm) {
        s += "    __syncthreads();\n    if (t == 0) {\n        double so = 0.0, si = 0.0;\n";
        s += "        for (int w = 0; w < 16; ++w) {\n            so += w_out[w];\n            si += w_in[w];\n        }\n";
        s += "        na.out_parts[blockIdx.x] = so;\n        if (na.in_parts != nullptr) {\n            na.in_parts[blockIdx.x] = si;\n        }\n    }\n";
    }
    s += "}\n";
    // the precision's type names
    const bool f32 = std::is_same<T, float>::value;
    auto subst = [&](const std::string& from, const std::string& to) {
        for (size_t at = s.find(from); at != std::string::npos; at = s.find(from, at + to.size())) {
            s.replace(at, from.size(), to);
        }
    };
    subst("$T", f32 ? "float" : "double");
    subst("$C", f32 ? "float2" : "double2");
    subst("$M", f32 ? "KtMatsF" : "KtMats");
    return s;
}

// the matrices of block b's ops, in the layout of its kernel's parameter M
// Block b's matrix parameter.  Scaled ops carry their entries divided by
// m00 (p = m01 / m00, ...); the product of those m00 multiplies the sink's
// entries or fills the extra slot.  *ok is false when its magnitude is below
// 1e-150 (amplitudes inside the block would grow past 1e150): the block
// kernels then do not run this apply.
template <typename T>
std::vector<T> jit_block_mats(const Plan<T>& plan, size_t b, bool* ok)
{
    using Z = std::complex<double>;
    const FBlock& fb = plan.blocks[b];
    const int nops = std::max(1, fb.op_end - fb.op_begin);
    const JitScale js = jit_scale_plan(plan, b);
    std::vector<T> m(static_cast<size_t>(8 * (nops + (js.own_slot ? 1 : 0))), T(0));
    auto put = [&](int j, int e, Z z) {
        m[static_cast<size_t>(8 * j + e)] = static_cast<T>(z.real());
        m[static_cast<size_t>(8 * j + e + 1)] = static_cast<T>(z.imag());
    };
    Z factor(1.0, 0.0);
    for (int j = 0; j < fb.op_end - fb.op_begin; ++j) {
        const FOp<T>& op = plan.ops[static_cast<size_t>(fb.op_begin + j)];
        for (int e = 0; e < 8; ++e) {
            m[static_cast<size_t>(8 * j + e)] = op.m[e];
        }
        auto at = [&](int e) { return Z(static_cast<double>(op.m[e]), static_cast<double>(op.m[e + 1])); };
        const Z m00 = at(0);
        switch (jit_scale_code(plan, b, j, js)) {
            case 1:
            case 2:
                m[static_cast<size_t>(8 * j + 2)] = static_cast<T>(static_cast<double>(op.m[2]) / m00.real());
                m[static_cast<size_t>(8 * j + 4)] = static_cast<T>(static_cast<double>(op.m[4]) / m00.real());
                factor *= m00.real();
                break;
            case 3:
                m[static_cast<size_t>(8 * j + 3)] = static_cast<T>(static_cast<double>(op.m[3]) / m00.real());
                factor *= m00.real();
                break;
            case 4:
                put(j, 2, at(2) / m00);
                put(j, 4, at(4) / m00);
                put(j, 6, at(6) / m00);
                factor *= m00;
                break;
            case 5:
                put(j, 6, at(6) / m00);
                factor *= m00;
                break;
            default:
                break;
        }
    }
    *ok = !js.any || std::abs(factor) >= 1e-150;
    if (js.any) {
        if (js.own_slot) {
            put(nops, 0, factor);
        } else {
            const FOp<T>& op = plan.ops[static_cast<size_t>(fb.op_begin + js.sink)];
            if (op.kind == OP_GENR || op.kind == OP_RXL) {
                // a real sink takes only real factors
                for (int e = 0; e < 8; ++e) {
                    m[static_cast<size_t>(8 * js.sink + e)] *= static_cast<T>(factor.real());
                }
            } else {
                for (int e = 0; e < 8; e += 2) {
                    const Z z(static_cast<double>(m[static_cast<size_t>(8 * js.sink + e)]),
                              static_cast<double>(m[static_cast<size_t>(8 * js.sink + e + 1)]));
                    put(js.sink, e, z * factor);
                }
            }
        }
    }
    return m;
}

constexpr const char* JIT_PRELUDE =
    "#include \"kt_fused_dev.cuh\"\n#include \"kt_tma_dev.cuh\"\n\n"
    "template <int N>\nstruct KtMats\n{\n    double m[N];\n};\n\n"
    "template <int N>\nstruct KtMatsF\n{\n    float m[N];\n};\n\n"
    "template <int N>\n__device__ __forceinline__ void kt_jit_fence(double2 (&v)[N])\n{\n"
    "#pragma unroll\n"
    "    for (int i = 0; i < N; ++i) {\n"
    "        asm volatile(\"\" : \"+d\"(v[i].x), \"+d\"(v[i].y));\n"
    "    }\n"
    "}\n\n"
    "template <int N>\n__device__ __forceinline__ void kt_jit_fence(float2 (&v)[N])\n{\n"
    "#pragma unroll\n"
    "    for (int i = 0; i < N; ++i) {\n"
    "        asm volatile(\"\" : \"+f\"(v[i].x), \"+f\"(v[i].y));\n"
    "    }\n"
    "}\n\n"
    "// a matrix entry of an item's op record (batched block kernels)\n"
    "template <typename T>\n__device__ __forceinline__ T kt_ldm(const unsigned char* p, unsigned off)\n{\n"
    "    return __ldg(reinterpret_cast<const T*>(p + off));\n"
    "}\n\n";

constexpr size_t JIT_MAX_KERNELS = 4096;
constexpr size_t JIT_MAX_SEEN = 65536;

struct JitCache
{
    std::mutex m;
    std::unordered_map<std::string, const void*> kernels;  // launch-bounds prefix + body -> kernel
    std::unordered_set<size_t> seen;                       // plans applied once with the precompiled kernels
    struct PlanState
    {
        int64_t applies {0};
        bool prepared {false};
        int64_t generation {-1};
        int device {-1};
        std::string config;                 // launch bounds, shared memory, renormalisation
        std::vector<const void*> kernels;   // one per block, once compiled
    };
    std::unordered_map<uint64_t, PlanState> plans;        // by plan structure (fused_plan_cached)
    int64_t generation {0};                                // bumped when every program is unloaded
    std::map<std::pair<const void*, int>, int> smem_set;   // (kernel, device) -> shared-memory limit set
    int64_t compiled {0};
    int64_t launches {0};
    bool failed {false};
};

JitCache& jit_cache()
{
    static JitCache c;
    return c;
}

// The kernels of every block of `plan` (compiling the ones not cached yet);
// false when the precompiled kernels should run instead: run-time compilation
// is unavailable or failed, or (`on_repeat`) the plan is new to this process,
// so compiling waits for its second apply.
template <typename T>
bool jit_kernels(const Plan<T>& plan, int RB, int threads, int minb, int smem_bytes, bool on_repeat, bool norm,
                 std::vector<const void*>& out, const std::vector<TmaCfg>* tma = nullptr)
{
    JitCache& jc = jit_cache();
    std::lock_guard<std::mutex> lock(jc.m);
    if (jc.failed) {
        return false;
    }
    const std::string bounds =
        "__launch_bounds__(" + std::to_string(threads) + ", " + std::to_string(minb) + ")";
    const size_t nb = plan.blocks.size();
    std::vector<std::string> keys(nb);
    std::vector<size_t> missing;
    std::unordered_map<std::string, size_t> first_of;
    for (size_t b = 0; b < nb; ++b) {
        keys[b] = bounds + jit_block_body<T>(plan, b, RB, norm, tma ? &(*tma)[b] : nullptr);
        if (jc.kernels.count(keys[b]) == 0 && first_of.count(keys[b]) == 0) {
            first_of[keys[b]] = b;
            missing.push_back(b);
        }
    }
    // bounded memory: past JIT_MAX_KERNELS cached kernels (or JIT_MAX_SEEN plans
    // remembered), start over; the launches of this stream that used the old
    // kernels are ordered before the unload, which waits for the device
    if (jc.kernels.size() + missing.size() > JIT_MAX_KERNELS) {
        cudaDeviceSynchronize();
        jit_unload_all();
        jc.kernels.clear();
        jc.smem_set.clear();
        ++jc.generation;
        missing.clear();
        first_of.clear();
        for (size_t b = 0; b < nb; ++b) {
            if (first_of.count(keys[b]) == 0) {
                first_of[keys[b]] = b;
                missing.push_back(b);
            }
        }
    }
    if (jc.seen.size() > JIT_MAX_SEEN) {
        jc.seen.clear();
    }
    if (jc.plans.size() > JIT_MAX_SEEN) {
        jc.plans.clear();
    }
    if (!missing.empty() && on_repeat) {
        std::string all;
        for (const auto& k : keys) {
            all += k;
        }
        if (jc.seen.insert(std::hash<std::string> {}(all)).second) {
            return false;
        }
    }
    if (!missing.empty()) {
        // a handful of programs, compiled on parallel host threads
        const size_t workers = std::max<size_t>(1, std::min<size_t>(missing.size(), 32));
        std::vector<std::string> sources(workers, JIT_PRELUDE);
        std::vector<std::vector<std::string>> names(workers);
        std::vector<std::vector<size_t>> owner(workers);
        for (size_t i = 0; i < missing.size(); ++i) {
            const size_t w = i % workers;
            const std::string name = "kt_jb" + std::to_string(jc.compiled + static_cast<int64_t>(i));
            sources[w] += "extern \"C\" __global__ void " + bounds + " " + name + keys[missing[i]].substr(bounds.size()) + "\n";
            names[w].push_back(name);
            owner[w].push_back(missing[i]);
        }
        std::vector<std::vector<const void*>> got;
        if (jit_compile(sources, names, got, true) != KT_OK) {
            jc.failed = true;
            cudaGetLastError();  // the precompiled kernels' launch check must not see this failure
            return false;
        }
        for (size_t w = 0; w < workers; ++w) {
            for (size_t k = 0; k < names[w].size(); ++k) {
                jc.kernels[keys[owner[w][k]]] = got[w][k];
            }
        }
        jc.compiled += static_cast<int64_t>(missing.size());
    }
    // the libraries load for every device, but a kernel's shared-memory limit is
    // per device: set it on the current one the first time a kernel runs there
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        dev = 0;
    }
    out.resize(nb);
    for (size_t b = 0; b < nb; ++b) {
        const void* fn = jc.kernels[keys[b]];
        const auto key = std::make_pair(fn, dev);
        auto it = jc.smem_set.find(key);
        if (it == jc.smem_set.end() || it->second < smem_bytes) {
            if (cudaKernelSetAttributeForDevice(reinterpret_cast<cudaKernel_t>(const_cast<void*>(fn)),
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes,
                                                dev) != cudaSuccess) {
                // this configuration does not fit: the precompiled kernels run it
                // (and the runtime's last-error slot is cleared for their launch check)
                cudaGetLastError();
                return false;
            }
            jc.smem_set[key] = smem_bytes;
        }
        out[b] = fn;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Host side of the TMA block kernels: the tensor map of a block over the
// state (cuTensorMapEncodeTiled, reached through the runtime so the library
// keeps no link-time dependency on the driver library), and the error word
// their bounded waits set.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q {};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<EncodeTiledFn>(nullptr);
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

bool tma_encode(const TmaGeom& g, void* amps, CUtensorMap* out)
{
    EncodeTiledFn fn = encode_tiled();
    if (fn == nullptr || !g.ok) {
        return false;
    }
    cuuint64_t dims[5];
    cuuint64_t strides[4];
    cuuint32_t box[5];
    cuuint32_t estr[5];
    for (int r = 0; r < g.rank; ++r) {
        dims[r] = g.dim[r];
        box[r] = g.box[r];
        estr[r] = 1;
        if (r > 0) {
            strides[r - 1] = g.stride[r];
        }
    }
    return fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, static_cast<cuuint32_t>(g.rank), amps, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// One error word per device (set by a TMA block kernel whose bounded wait ran
// out) and a pinned host copy of it, refreshed after every apply that ran
// such kernels; the C entry points report it once the copy has landed.
struct TmaErr
{
    std::mutex m;
    std::map<int, unsigned int*> dev;
    unsigned int* host {nullptr};  // pinned, one word per device ordinal (up to 64)
};

TmaErr& tma_err()
{
    static TmaErr e;
    return e;
}

unsigned int* tma_err_word(int dev, unsigned int** host)
{
    TmaErr& e = tma_err();
    std::lock_guard<std::mutex> lock(e.m);
    if (e.host == nullptr) {
        void* h = nullptr;
        if (cudaMallocHost(&h, 64 * sizeof(unsigned int)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        std::memset(h, 0, 64 * sizeof(unsigned int));
        e.host = static_cast<unsigned int*>(h);
    }
    if (dev < 0 || dev >= 64) {
        return nullptr;
    }
    auto it = e.dev.find(dev);
    if (it == e.dev.end()) {
        void* d = nullptr;
        if (cudaMalloc(&d, 256) != cudaSuccess || cudaMemset(d, 0, 256) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        it = e.dev.emplace(dev, static_cast<unsigned int*>(d)).first;
    }
    *host = e.host + dev;
    return it->second;
}

// The apply of a plan from which its compiled kernels pay for themselves:
// compiling takes about 0.6 s per block kernel on one host thread (the
// blocks compile in parallel), and a compiled pass saves about half of a
// precompiled one, ~2^n * 2 * amplitude bytes at 1.5 TB/s; jit_after
// (>= 1) fixes the count instead.  At least the second apply.
int64_t jit_after_applies(int n, size_t amp_bytes)
{
    if (tuning().jit_after > 0) {
        return tuning().jit_after;
    }
    const double pass = std::ldexp(1.0, n) * 2.0 * static_cast<double>(amp_bytes) / 1.5e12;
    const double threads = jit_threads();
    const double k = std::ceil(0.6 / threads / (0.5 * pass));
    return static_cast<int64_t>(std::max(2.0, std::min(k, 1.0e9)));
}

// The launch of a plan's blocks as run-time compiled kernels, or false when
// the caller should run the precompiled ones: fused_jit = 1 always; 2 on
// states of at least jit_min_qubits index bits once the plan has been applied
// jit_after_applies times, or after kt_sv_prepare (`compile_only`: compile,
// launch nothing).  With `parts` (complex64
// renormalisation: target | out even | out odd, n_parts per-CTA sums each)
// every block gets its NormArgs and the caller finishes with k_norm_final.
template <typename T>
bool jit_launch(State& s, const Plan<T>& plan, uint64_t plan_key, int K, bool rb3, int threads, int shape, double* parts,
                int32_t* rc, int* n_parts_out, bool compile_only = false)
{
    using C = typename CxT<T>::type;
    *rc = KT_OK;
    const int n = s.n_bits;
    const int mode = tuning().fused_jit;
    bool want = compile_only || mode == 1 || (mode == 2 && (n >= tuning().jit_min_qubits || s.force_jit));
    if (!want && mode == 2) {
        // a plan compiled ahead (kt_sv_prepare / kt_dm_prepare) runs compiled at any size
        JitCache& jc = jit_cache();
        std::lock_guard<std::mutex> lock(jc.m);
        const auto it = jc.plans.find(plan_key);
        want = it != jc.plans.end() && it->second.prepared;
    }
    if (!want) {
        return false;
    }
    // the generated kernels keep only the tile in shared memory, so they may
    // run jit_ctas_per_sm CTAs per SM (register budget 65536 / (threads * CTAs))
    int minb = 1;
    if (shape == 2) {
        minb = std::max(2, std::min(4, tuning().jit_ctas_per_sm));
    } else if (shape == 3 || shape == 4) {
        minb = fused_ctas(shape);
    }
    const uint64_t n_tiles = uint64_t {1} << (n - K);
    uint64_t grid = std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sm_count()) * minb);
    size_t smem = (size_t {1} << K) * sizeof(C) * (jit_async(K, sizeof(C)) ? 2 : 1);
    int smem_attr = std::max(fused_smem_limit(shape), static_cast<int>(smem));
    const int RB = rb3 ? Cfg3::RB : Cfg<T>::RB;
    const bool norm = parts != nullptr;
    if (norm && grid > static_cast<uint64_t>(*n_parts_out)) {
        return false;  // the caller reserved per-CTA sums for fewer CTAs
    }
    // TMA-pipelined kernels (complex128, no renormalisation): one persistent
    // CTA per SM of one tile-sized thread group and a producer warp,
    // jit_tma_stages tile buffers; every block's tile must have the three
    // lowest qubits (one 128-byte row per box line)
    std::vector<TmaCfg> tma_cfg;
    if (tuning().jit_tma != 0 && std::is_same<T, double>::value && !norm && encode_tiled() != nullptr) {
        const int groups = 1;
        const int stages = std::max(tuning().jit_tma_stages, 2);
        const size_t tile_bytes = (size_t {1} << K) * sizeof(C);
        const size_t need = static_cast<size_t>(stages) * tile_bytes + 1024 + 16 * static_cast<size_t>(stages);
        const int tthreads = groups * threads + 32;
        // jit_tma_ctas = 2: two such CTAs per SM, each within half of the SM's shared memory
        const int ctas = tuning().jit_tma_ctas;
        const size_t cap = ctas == 2 ? size_t {113} * 1024 : size_t {227} * 1024;
        bool ok = need <= cap && tthreads <= 1024 && (groups * threads) % 32 == 0;
        for (size_t b = 0; ok && b < plan.blocks.size(); ++b) {
            TmaCfg c;
            c.groups = groups;
            c.stages = stages;
            c.geom = tma_geom(plan.blocks[b], n);
            ok = c.geom.ok;
            tma_cfg.push_back(std::move(c));
        }
        if (ok) {
            threads = tthreads;
            minb = ctas;
            grid = std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sm_count()) * static_cast<uint64_t>(ctas));
            smem = need;
            smem_attr = static_cast<int>(need);
        } else {
            tma_cfg.clear();
        }
    }
    const bool use_tma = !tma_cfg.empty();
    // this plan's kernels: resolved once, compiled once the plan has been
    // applied often enough to repay the compile (jit_after_applies)
    std::vector<const void*> jk;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        dev = 0;
    }
    const std::string config = std::to_string(RB) + "/" + std::to_string(threads) + "/" + std::to_string(minb) + "/" +
                               std::to_string(smem_attr) + "/" + (norm ? "n" : "-") + "/" +
                               std::to_string(jit_async(K, sizeof(C)) ? 1 : 0) + "/" +
                               std::to_string(tuning().jit_prefetch) + std::to_string(tuning().jit_merge_diag) +
                               std::to_string(tuning().jit_skip_io) + std::to_string(tuning().jit_fence) +
                               std::to_string(tuning().jit_scale_ops) + std::to_string(tuning().jit_remat) +
                               std::to_string(tuning().jit_lean_sync) +
                               (use_tma ? "/tma" + std::to_string(tma_cfg[0].groups) + "x" +
                                              std::to_string(tma_cfg[0].stages)
                                        : std::string());
    bool ready = false;
    bool compile = compile_only || mode == 1;
    {
        JitCache& jc = jit_cache();
        std::lock_guard<std::mutex> lock(jc.m);
        if (jc.failed) {
            return false;
        }
        JitCache::PlanState& st = jc.plans[plan_key];
        st.applies += compile_only ? 0 : 1;
        st.prepared = st.prepared || compile_only;
        ready = st.generation == jc.generation && st.device == dev && st.config == config &&
                st.kernels.size() == plan.blocks.size();
        if (ready) {
            jk = st.kernels;
        }
        compile = compile || st.prepared || s.force_jit || st.applies >= jit_after_applies(n, sizeof(C));
    }
    if (!ready) {
        if (!compile ||
            !jit_kernels<T>(plan, RB, threads, minb, smem_attr, false, norm, jk, use_tma ? &tma_cfg : nullptr)) {
            return false;
        }
        JitCache& jc = jit_cache();
        std::lock_guard<std::mutex> lock(jc.m);
        JitCache::PlanState& st = jc.plans[plan_key];
        st.generation = jc.generation;
        st.device = dev;
        st.config = config;
        st.kernels = jk;
    }
    if (compile_only) {
        return true;
    }
    void* a = s.amps;
    unsigned long long nt = n_tiles;
    const int np = static_cast<int>(grid);
    double* target = parts;
    double* out[2] = {norm ? parts + np : nullptr, norm ? parts + 2 * np : nullptr};
    const double pass_bytes = 2.0 * static_cast<double>(sizeof(C)) * static_cast<double>(s.n_amps());
    std::vector<std::vector<T>> all_mats(plan.blocks.size());
    for (size_t b = 0; b < plan.blocks.size(); ++b) {
        bool ok = true;
        all_mats[b] = jit_block_mats<T>(plan, b, &ok);
        if (!ok) {
            return false;  // scale factors out of range: the precompiled kernels run this apply
        }
    }
    unsigned int* err_host = nullptr;
    unsigned int* err_dev = use_tma ? tma_err_word(dev, &err_host) : nullptr;
    if (use_tma && err_dev == nullptr) {
        return false;
    }
    for (size_t b = 0; b < plan.blocks.size(); ++b) {
        std::vector<T>& mats = all_mats[b];
        cudaError_t e = cudaSuccess;
        if (use_tma) {
            CUtensorMap tm;
            if (!tma_encode(tma_cfg[b].geom, a, &tm)) {
                *rc = KT_ERR_CUDA;
                set_error(KT_ERR_CUDA, "cuTensorMapEncodeTiled failed for a block's tile");
                return true;
            }
            void* args[] = {&tm, &a, &nt, &err_dev, mats.data()};
            e = cudaLaunchKernel(jk[b], dim3(static_cast<unsigned>(grid)), dim3(static_cast<unsigned>(threads)), args,
                                 smem, s.stream);
        } else if (norm) {
            NormArgs na {};
            na.n_parts = np;
            na.target = (b == 0) ? nullptr : target;
            na.prev = (b == 0) ? nullptr : out[(b - 1) & 1];
            na.in_parts = (b == 0) ? target : nullptr;
            na.out_parts = out[b & 1];
            void* args[] = {&a, &nt, &na, mats.data()};
            e = cudaLaunchKernel(jk[b], dim3(static_cast<unsigned>(grid)), dim3(static_cast<unsigned>(threads)), args,
                                 smem, s.stream);
        } else {
            void* args[] = {&a, &nt, mats.data()};
            e = cudaLaunchKernel(jk[b], dim3(static_cast<unsigned>(grid)), dim3(static_cast<unsigned>(threads)), args,
                                 smem, s.stream);
        }
        if (e != cudaSuccess) {
            *rc = cuda_fail(e, "cudaLaunchKernel(run-time compiled block)");
            return true;
        }
        s.last_launches += 1;
        s.last_alg_bytes += pass_bytes;
    }
    if (use_tma) {
        // the error word to the host once these blocks are done (read by the C entry points)
        const cudaError_t e = cudaMemcpyAsync(err_host, err_dev, sizeof(unsigned int), cudaMemcpyDeviceToHost, s.stream);
        if (e != cudaSuccess) {
            *rc = cuda_fail(e, "cudaMemcpyAsync(block kernel error word)");
            return true;
        }
    }
    *n_parts_out = np;
    jit_cache().launches += static_cast<int64_t>(plan.blocks.size());
    return true;
}

template <typename T>
int32_t run_fused(State& s, const std::vector<LGate>& gates)
{
    using C = typename CxT<T>::type;
    const int n = s.n_bits;
    Plan<T> plan;
    int K = 0;
    bool rb3 = false;
    uint64_t plan_key = 0;
    if (n < Cfg<T>::RB + 5 || gates.empty()) {
        for (const auto& g : gates) {
            if (const int32_t rc = launch_gate_sweep(s, g); rc != KT_OK) {
                return rc;
            }
        }
        return KT_OK;
    }
    if (const int32_t rc = fused_plan_cached<T>(n, gates, plan, &K, &rb3, &plan_key); rc != KT_OK) {
        return rc;
    }
    // upload the plan: blocks | phases | ops
    auto al = [](size_t v) { return (v + 255) & ~size_t {255}; };
    const size_t nb = plan.blocks.size() * sizeof(FBlock);
    const size_t np = plan.phases.size() * sizeof(FPhase);
    const size_t no = std::max<size_t>(1, plan.ops.size()) * sizeof(FOp<T>);
    const size_t off_p = al(nb);
    const size_t off_o = al(off_p + np);
    const size_t need = al(off_o + no);
    if (const int32_t rc = s.scratch.reserve(need); rc != KT_OK) {
        return rc;
    }
    std::vector<unsigned char> host(need, 0);
    std::memcpy(host.data(), plan.blocks.data(), nb);
    std::memcpy(host.data() + off_p, plan.phases.data(), np);
    if (!plan.ops.empty()) {
        std::memcpy(host.data() + off_o, plan.ops.data(), plan.ops.size() * sizeof(FOp<T>));
    }
    char* dev = static_cast<char*>(s.scratch.ptr);
    // pageable source: staged by the time the call returns, so `host` may go away
    KT_CUDA(cudaMemcpyAsync(dev, host.data(), need, cudaMemcpyHostToDevice, s.stream));
    const auto* d_blk = reinterpret_cast<const FBlock*>(dev);
    const auto* d_ph = reinterpret_cast<const FPhase*>(dev + off_p);
    const auto* d_ops = reinterpret_cast<const FOp<T>*>(dev + off_o);
    const int threads = 1 << (K - (rb3 ? Cfg3::RB : Cfg<T>::RB));
    // 512-thread tiles run one CTA per SM; 256-thread tiles follow the register-budget knob
    int shape = threads > 256 ? 0 : (tuning().fused_ctas_per_sm == 1 ? 1 : 2);
    if (rb3) {
        shape = threads > 256 ? 3 : 4;
    }
    if constexpr (std::is_same<T, float>::value) {
        if (tuning().c64_renormalize != 0) {
            // compiled blocks keep the renormalisation: per-CTA sums for up to
            // 4 CTAs per SM, then the closing rescale
            const int max_parts = sm_count() * 4;
            if (const int32_t rc = s.scratch2.reserve(3 * static_cast<size_t>(max_parts) * sizeof(double)); rc != KT_OK) {
                return rc;
            }
            double* parts = static_cast<double*>(s.scratch2.ptr);
            int32_t rc = KT_OK;
            int n_parts = max_parts;
            if (jit_launch<T>(s, plan, plan_key, K, rb3, threads, shape, parts, &rc, &n_parts)) {
                if (rc != KT_OK || plan.blocks.empty()) {
                    return rc;
                }
                const unsigned fin_grid = static_cast<unsigned>(
                    std::min<uint64_t>((s.n_amps() + 255) / 256, static_cast<uint64_t>(sm_count()) * 8));
                k_norm_final<C><<<fin_grid, 256, 0, s.stream>>>(static_cast<C*>(s.amps), s.n_amps(), parts,
                                                                parts + n_parts * (1 + ((plan.blocks.size() - 1) & 1)),
                                                                n_parts);
                KT_CHECK_LAUNCH("k_norm_final");
                s.last_launches += 1;
                s.last_alg_bytes += 2.0 * static_cast<double>(sizeof(C)) * static_cast<double>(s.n_amps());
                return KT_OK;
            }
            return run_fused_norm<T>(s, plan, d_blk, d_ph, d_ops, K, threads, shape);
        }
    }
    static bool attr_set[5] = {false, false, false, false, false};
    if (!attr_set[shape]) {
        const int bytes = fused_smem_limit(shape);
        switch (shape) {
            case 0: KT_CUDA(cudaFuncSetAttribute(k_fused<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)); break;
            case 1: KT_CUDA(cudaFuncSetAttribute(k_fused<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)); break;
            case 3:
            case 4:
                if constexpr (std::is_same<T, double>::value) {
                    if (shape == 3) {
                        KT_CUDA(cudaFuncSetAttribute(k_fused<T, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
                    } else {
                        KT_CUDA(cudaFuncSetAttribute(k_fused<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
                    }
                }
                break;
            default: KT_CUDA(cudaFuncSetAttribute(k_fused<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)); break;
        }
        attr_set[shape] = true;
    }
    const uint64_t n_tiles = uint64_t {1} << (n - K);
    const uint64_t grid = std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sm_count()) * fused_ctas(shape));
    const double pass_bytes = 2.0 * static_cast<double>(sizeof(C)) * static_cast<double>(s.n_amps());
    {
        int32_t rc = KT_OK;
        int n_parts = 0;
        if (jit_launch<T>(s, plan, plan_key, K, rb3, threads, shape, nullptr, &rc, &n_parts)) {
            return rc;
        }
    }
    for (size_t b = 0; b < plan.blocks.size(); ++b) {
        const auto& fb = plan.blocks[b];
        const size_t smem = (size_t {1} << K) * sizeof(C) + static_cast<size_t>(fb.op_end - fb.op_begin) * sizeof(FOp<T>);
        C* a = static_cast<C*>(s.amps);
        const unsigned g = static_cast<unsigned>(grid);
        switch (shape) {
            case 0: k_fused<T, 0><<<g, threads, smem, s.stream>>>(a, d_blk + b, d_ph, d_ops, n_tiles); break;
            case 1: k_fused<T, 1><<<g, threads, smem, s.stream>>>(a, d_blk + b, d_ph, d_ops, n_tiles); break;
            case 3:
            case 4:
                if constexpr (std::is_same<T, double>::value) {
                    if (shape == 3) {
                        k_fused<T, 3><<<g, threads, smem, s.stream>>>(a, d_blk + b, d_ph, d_ops, n_tiles);
                    } else {
                        k_fused<T, 4><<<g, threads, smem, s.stream>>>(a, d_blk + b, d_ph, d_ops, n_tiles);
                    }
                }
                break;
            default: k_fused<T, 2><<<g, threads, smem, s.stream>>>(a, d_blk + b, d_ph, d_ops, n_tiles); break;
        }
        KT_CHECK_LAUNCH("k_fused");
        s.last_launches += 1;
        s.last_alg_bytes += pass_bytes;
    }
    return KT_OK;
}

// ===========================================================================
// Fused adjoint sweep.  The gates arrive in backward order as U^dagger with
// their derivative dU/dtheta; a block un-applies all its gates to psi and
// lambda tile by tile and reduces, for each parameterised gate,
// Re <lambda| D psi> (psi already un-applied through that gate, lambda not
// yet) into per-warp shared-memory slots; each CTA writes one partial per
// gradient row, finalised in a fixed order.  Moving a gate past gates on
// other qubits leaves every term unchanged (U_B commutes with D_A), so the
// forward planner's reordering is valid here too.

template <typename T>
__global__ void __launch_bounds__(256, 2) k_fused_adj(typename CxT<T>::type* __restrict__ psi,
                                                      typename CxT<T>::type* __restrict__ lam,
                                                      const FBlock* __restrict__ blk, const FPhase* __restrict__ phases,
                                                      const FOpA<T>* __restrict__ ops, int n_rows,
                                                      double* __restrict__ partial, uint64_t n_tiles)
{
    using C = typename CxT<T>::type;
    constexpr int RB = CfgA<T>::RB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ FBlock bk;
    __shared__ FPhase sph[MAX_PHASES_PER_BLOCK];
    const uint32_t t = threadIdx.x;
    if (t == 0) {
        bk = *blk;
    }
    __syncthreads();
    const int no = bk.op_end - bk.op_begin;
    const size_t tile_bytes = sizeof(C) << bk.K;
    C* smp = reinterpret_cast<C*>(smem_raw);
    C* sml = reinterpret_cast<C*>(smem_raw + tile_bytes);
    FOpA<T>* sops = reinterpret_cast<FOpA<T>*>(smem_raw + 2 * tile_bytes);
    double* acc = reinterpret_cast<double*>(smem_raw + 2 * tile_bytes + static_cast<size_t>(no) * sizeof(FOpA<T>));
    stage_block(bk, phases, ops, sph, sops, t);
    for (int w = t; w < n_rows * ADJ_WARPS; w += blockDim.x) {
        acc[w] = 0.0;
    }
    __syncthreads();
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        adj_tile<T, RB, false>(psi, lam, bk, sph, sops, tile, smp, sml, acc, t);
    }
    __syncthreads();
    for (int r = t; r < n_rows; r += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < ADJ_WARPS; ++w) {
            s += acc[r * ADJ_WARPS + w];
        }
        partial[static_cast<size_t>(r) * gridDim.x + blockIdx.x] = s;
    }
}

// grad[rows[r]] = 2 * sum_b partial[r][b] in fixed order
__global__ void k_adj_rows(const double* __restrict__ partial, int n_blocks, const int32_t* __restrict__ rows, int n_rows,
                           double* __restrict__ grad)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) {
        return;
    }
    double s = 0.0;
    for (int b = 0; b < n_blocks; ++b) {
        s += partial[static_cast<size_t>(r) * n_blocks + b];
    }
    grad[rows[r]] = 2.0 * s;
}

// ---------------------------------------------------------------------------
// Run-time compiled adjoint blocks (adjoint_jit).  The k_fused_adj tile loop
// for one block with its ops written out: every gradient term a literal
// generator form on literal register / thread slots, every U^dagger a
// straight-line body on psi and then on lambda, control predicates folded;
// the matrices arrive in the constant-bank parameter M (8 entries per op).
template <typename T>
std::string jit_adj_body(const Plan<T, FOpA<T>>& plan, size_t b, int RB)
{
    const FBlock& fb = plan.blocks[b];
    const int TB = fb.K - RB;
    const int R = 1 << RB;
    const int np = fb.phase_end - fb.phase_begin;
    const int nops = std::max(1, fb.op_end - fb.op_begin);
    const FPhase* ph = plan.phases.data() + fb.phase_begin;
    std::vector<uint64_t> free_strides(static_cast<size_t>(std::max(1, fb.nfree)));
    for (int k = 0; k < fb.nfree; ++k) {
        free_strides[static_cast<size_t>(k)] = uint64_t {1} << fb.freebit[k];
    }
    auto reg_off = [&](const FPhase& f, int i) {
        uint64_t o = 0;
        for (int sl = 0; sl < RB; ++sl) {
            if (i & (1 << sl)) {
                o += f.rstride[sl];
            }
        }
        return o;
    };
    auto reg_xor = [&](const uint32_t* terms, int i) {
        uint32_t x = 0;
        for (int sl = 0; sl < RB; ++sl) {
            if (i & (1 << sl)) {
                x ^= terms[sl];
            }
        }
        return x;
    };
    auto replace_all = [](std::string str, const std::string& from, const std::string& to) {
        for (size_t at = str.find(from); at != std::string::npos; at = str.find(from, at + to.size())) {
            str.replace(at, from.size(), to);
        }
        return str;
    };
    std::string s;
    s.reserve(32768);
    if (tl_batch != nullptr) {
        s += "(void* const* p_list, void* const* l_list, const unsigned char* const* o_list, const long long* pbase, "
             "double* partial, unsigned long long n_tiles, int n_rows)\n{\n";
    } else {
        s += "(void* psi_, void* lam_, unsigned long long n_tiles, double* partial, int n_rows, const __grid_constant__ $M<" +
             std::to_string(8 * nops) + "> M)\n{\n";
    }
    s += "    using namespace kt;\n    using C = $C;\n";
    s += "    constexpr int RB = " + std::to_string(RB) + ";\n";
    if (tl_batch != nullptr) {
        s += "    C* __restrict__ psi = static_cast<C*>(p_list[blockIdx.y]);\n"
             "    C* __restrict__ lam = static_cast<C*>(l_list[blockIdx.y]);\n"
             "    const unsigned char* __restrict__ ob = o_list[blockIdx.y];\n"
             "    partial += pbase[blockIdx.y];\n";
    } else {
        s += "    C* __restrict__ psi = static_cast<C*>(psi_);\n    C* __restrict__ lam = static_cast<C*>(lam_);\n";
    }
    s += "    extern __shared__ __align__(16) unsigned char smem_raw[];\n";
    s += "    C* smp = reinterpret_cast<C*>(smem_raw);\n";
    s += "    C* sml = smp + " + std::to_string(1 << fb.K) + ";\n";
    s += "    double* acc = reinterpret_cast<double*>(sml + " + std::to_string(1 << fb.K) + ");\n";
    s += "    const uint32_t t_outer = threadIdx.x;\n";
    s += "    for (int w = threadIdx.x; w < n_rows * " + std::to_string(ADJ_WARPS) + "; w += blockDim.x) {\n"
         "        acc[w] = 0.0;\n    }\n    __syncthreads();\n";
    s += "    for (unsigned long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {\n";
    s += "        uint32_t t_l;\n        asm volatile(\"mov.u32 %0, %1;\" : \"=r\"(t_l) : \"r\"(t_outer));\n";
    s += "        const uint32_t t = t_l;\n        const int lane = static_cast<int>(t & 31u);\n"
         "        const int warp = static_cast<int>(t >> 5);\n";
    s += "        C vp[1 << RB];\n        C vl[1 << RB];\n";
    s += "        const uint64_t base = " + jit_deposit("tile", free_strides.data(), fb.nfree) + ";\n";
    s += "        {\n            const uint64_t off = base + " + jit_deposit("t", ph[0].tstride, TB) + ";\n";
    for (int i = 0; i < R; ++i) {
        s += "            vp[" + std::to_string(i) + "] = psi[off + " + std::to_string(reg_off(ph[0], i)) + "ULL];\n";
        s += "            vl[" + std::to_string(i) + "] = lam[off + " + std::to_string(reg_off(ph[0], i)) + "ULL];\n";
    }
    s += "        }\n";
    for (int p = 0; p < np; ++p) {
        const FPhase& cur = ph[p];
        if (p > 0) {
            const FPhase& prev = ph[p - 1];
            s += "        {\n            const uint32_t so = " + jit_xor_terms(prev.tsw_out, TB, prev.xor_out) + ";\n";
            for (int i = 0; i < R; ++i) {
                const std::string x = std::to_string(reg_xor(prev.rsw_out, i));
                s += "            smp[so ^ " + x + "u] = vp[" + std::to_string(i) + "];\n";
                s += "            sml[so ^ " + x + "u] = vl[" + std::to_string(i) + "];\n";
            }
            s += "            __syncthreads();\n";
            s += "            const uint32_t lo = " + jit_xor_terms(cur.tsw, TB, 0) + ";\n";
            for (int i = 0; i < R; ++i) {
                const std::string x = std::to_string(reg_xor(cur.rsw, i));
                s += "            vp[" + std::to_string(i) + "] = smp[lo ^ " + x + "u];\n";
                s += "            vl[" + std::to_string(i) + "] = sml[lo ^ " + x + "u];\n";
            }
            s += "            __syncthreads();\n        }\n";
        }
        for (int o = cur.op_begin; o < cur.op_end; ++o) {
            const FOpA<T>& op = plan.ops[static_cast<size_t>(o)];
            const int j = o - fb.op_begin;
            const int cs = (op.cslot == NO_SLOT) ? -1 : op.cslot;
            const std::string csf = cs < 0 ? "-1" : "CS_RT";
            s += "        ";
            if (op.cglob != 0) {
                s += "if ((base & " + jit_hex(op.cglob) + ") == " + jit_hex(op.cglob) + ") ";
            }
            s += "{\n";
            const std::string on =
                op.cthr != 0 ? "((t & " + std::to_string(op.cthr) + "u) == " + std::to_string(op.cthr) + "u)" : "true";
            s += "            const bool on = " + on + ";\n";
            if (op.row >= 0) {
                // Re <lambda| dU psi_(g-1)> from psi_g and lambda, before U^dagger touches either
                s += "            double g = 0.0;\n            if (on) {\n                ";
                if (op.tslot != NO_SLOT) {
                    const char* gk = op.gen == GEN_X ? "GEN_X" : op.gen == GEN_Y ? "GEN_Y" : op.gen == GEN_Z ? "GEN_Z" : "GEN_P";
                    s += std::string("GradRegF<$T, RB, ") + gk + "> f {vl, vp, 0.0}; f.crt = " + std::to_string(cs) +
                         "; f.template run<" + std::to_string(op.tslot) + ", " + csf + ">(); g = " +
                         (op.gen == GEN_P ? "" : "0.5 * ") + "f.acc;\n";
                } else {
                    std::string bexpr = "false";
                    if (op.tthr != 0 && op.tglob != 0) {
                        bexpr = "(((t & " + std::to_string(op.tthr) + "u) != 0u) || ((base & " + jit_hex(op.tglob) + ") != 0ULL))";
                    } else if (op.tthr != 0) {
                        bexpr = "((t & " + std::to_string(op.tthr) + "u) != 0u)";
                    } else if (op.tglob != 0) {
                        bexpr = "((base & " + jit_hex(op.tglob) + ") != 0ULL)";
                    }
                    const std::string w = op.gen == GEN_Z ? "(" + bexpr + " ? -0.5 : 0.5)" : "(" + bexpr + " ? -1.0 : 0.0)";
                    s += "GradAllF<$T, RB> f {vl, vp, 0.0}; f.crt = " + std::to_string(cs) + "; f.template run<0, " + csf +
                         ">(); g = " + w + " * f.acc;\n";
                }
                s += "            }\n";
                s += "#pragma unroll\n            for (int s_ = 16; s_ > 0; s_ >>= 1) {\n"
                     "                g += __shfl_down_sync(0xffffffffU, g, s_);\n            }\n";
                s += "            if (lane == 0) {\n                acc[" + std::to_string(op.row) + " * " +
                     std::to_string(ADJ_WARPS) + " + warp] += g;\n            }\n";
            }
            // U^dagger on psi, then on lambda (the forward emitter with its guards folded in here)
            FOp<T> fo {};
            fo.kind = op.kind;
            fo.tslot = op.tslot;
            fo.cslot = op.cslot;
            fo.tthr = op.tthr;
            fo.tglob = op.tglob;
            for (int e = 0; e < 8; ++e) {
                fo.m[e] = op.m[e];
            }
            std::string body;
            jit_emit_op(body, fo, j, 0);
            s += "            if (on) {\n";
            s += replace_all(body, "{v, ", "{vp, ");
            s += replace_all(body, "{v, ", "{vl, ");
            s += "            }\n        }\n";
        }
    }
    {
        const FPhase& last = ph[np - 1];
        s += "        {\n            const uint64_t off = base + " + jit_deposit("t", last.tstride, TB) + ";\n";
        for (int i = 0; i < R; ++i) {
            s += "            psi[off + " + std::to_string(reg_off(last, i)) + "ULL] = vp[" + std::to_string(i) + "];\n";
            s += "            lam[off + " + std::to_string(reg_off(last, i)) + "ULL] = vl[" + std::to_string(i) + "];\n";
        }
        s += "        }\n";
    }
    s += "    }\n    __syncthreads();\n";
    s += "    for (int r = threadIdx.x; r < n_rows; r += blockDim.x) {\n        double sum = 0.0;\n"
         "        for (int w = 0; w < " + std::to_string(ADJ_WARPS) + "; ++w) {\n"
         "            sum += acc[r * " + std::to_string(ADJ_WARPS) + " + w];\n        }\n"
         "        partial[static_cast<size_t>(r) * gridDim.x + blockIdx.x] = sum;\n    }\n}\n";
    const bool f32 = std::is_same<T, float>::value;
    s = replace_all(s, "$T", f32 ? "float" : "double");
    s = replace_all(s, "$C", f32 ? "float2" : "double2");
    s = replace_all(s, "$M", f32 ? "KtMatsF" : "KtMats");
    return s;
}

// The compiled kernels of an adjoint plan's blocks (compiling the ones not
// cached yet); false when run-time compilation is unavailable or failed.
template <typename T>
bool jit_adj_kernels(const Plan<T, FOpA<T>>& plan, int RB, int smem_bytes, std::vector<const void*>& out)
{
    JitCache& jc = jit_cache();
    std::lock_guard<std::mutex> lock(jc.m);
    if (jc.failed) {
        return false;
    }
    const std::string bounds = "__launch_bounds__(256, 2)";
    const size_t nb = plan.blocks.size();
    std::vector<std::string> keys(nb);
    std::vector<size_t> missing;
    std::unordered_map<std::string, size_t> first_of;
    for (size_t b = 0; b < nb; ++b) {
        keys[b] = bounds + jit_adj_body<T>(plan, b, RB);
        if (jc.kernels.count(keys[b]) == 0 && first_of.count(keys[b]) == 0) {
            first_of[keys[b]] = b;
            missing.push_back(b);
        }
    }
    if (jc.kernels.size() + missing.size() > JIT_MAX_KERNELS) {
        return false;
    }
    if (!missing.empty()) {
        const size_t workers = std::max<size_t>(1, std::min<size_t>(missing.size(), 32));
        std::vector<std::string> sources(workers, JIT_PRELUDE);
        std::vector<std::vector<std::string>> names(workers);
        std::vector<std::vector<size_t>> owner(workers);
        for (size_t i = 0; i < missing.size(); ++i) {
            const size_t w = i % workers;
            const std::string name = "kt_ja" + std::to_string(jc.compiled + static_cast<int64_t>(i));
            sources[w] += "extern \"C\" __global__ void " + bounds + " " + name + keys[missing[i]].substr(bounds.size()) + "\n";
            names[w].push_back(name);
            owner[w].push_back(missing[i]);
        }
        std::vector<std::vector<const void*>> got;
        if (jit_compile(sources, names, got, true) != KT_OK) {
            jc.failed = true;
            cudaGetLastError();
            return false;
        }
        for (size_t w = 0; w < workers; ++w) {
            for (size_t k = 0; k < names[w].size(); ++k) {
                jc.kernels[keys[owner[w][k]]] = got[w][k];
            }
        }
        jc.compiled += static_cast<int64_t>(missing.size());
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        dev = 0;
    }
    out.resize(nb);
    for (size_t b = 0; b < nb; ++b) {
        const void* fn = jc.kernels[keys[b]];
        const auto key = std::make_pair(fn, dev);
        auto it = jc.smem_set.find(key);
        if (it == jc.smem_set.end() || it->second < smem_bytes) {
            if (cudaKernelSetAttributeForDevice(reinterpret_cast<cudaKernel_t>(const_cast<void*>(fn)),
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes,
                                                dev) != cudaSuccess) {
                cudaGetLastError();
                return false;
            }
            jc.smem_set[key] = smem_bytes;
        }
        out[b] = fn;
    }
    return true;
}

// Adjoint plans cached by circuit structure (gate kinds, qubits, value
// classes, gradient rows and generators): a repeated gradient with new
// parameters takes the new matrices and reuses the plan (and its kernels).
template <typename T>
struct AdjPlanEntry
{
    std::vector<uint64_t> signature;
    Plan<T, FOpA<T>> plan;
    std::vector<std::vector<int32_t>> rows_of_block;
    int64_t sweeps {0};
    std::vector<const void*> kernels;  // compiled blocks (adjoint_jit), once compiled
    int64_t generation {-1};
    int device {-1};
};

template <typename T>
struct AdjPlanCache
{
    std::mutex m;
    std::unordered_map<uint64_t, AdjPlanEntry<T>> entries;
};

template <typename T>
AdjPlanCache<T>& adj_plan_cache()
{
    static AdjPlanCache<T> c;
    return c;
}

template <typename T>
int32_t run_adjoint_sweep(State& psi, State& lam, const std::vector<AdjGate>& gates, double* dev_grad,
                          DevBuf& work)
{
    using C = typename CxT<T>::type;
    constexpr int RB = CfgA<T>::RB;
    constexpr int L = CfgA<T>::L;
    const int n = psi.n_bits;
    const int K = std::min(n, RB + TB256);
    std::vector<LGate> lg;
    std::vector<AdjExtra> ex;
    lg.reserve(gates.size());
    ex.reserve(gates.size());
    for (const auto& g : gates) {
        lg.push_back(g.adj);
        AdjExtra e {};
        e.row = g.row;
        e.gen = g.gen;
        ex.push_back(e);
    }
    // the plan of this structure: from the cache (new matrices), or planned now
    const size_t max_ops = static_cast<size_t>(std::min(ADJ_MAX_OPS, tuning().fused_max_ops));
    std::vector<uint64_t> sig;
    sig.reserve(2 * lg.size() + 1);
    sig.push_back(static_cast<uint64_t>(n) | (static_cast<uint64_t>(sizeof(T)) << 8) | (static_cast<uint64_t>(K) << 16) |
                  (static_cast<uint64_t>(tuning().fold_permutations) << 24) | (static_cast<uint64_t>(max_ops) << 32));
    for (size_t i = 0; i < lg.size(); ++i) {
        sig.push_back(static_cast<uint64_t>(gate_class(lg[i])) | (static_cast<uint64_t>(lg[i].target & 0xFFFF) << 16) |
                      (static_cast<uint64_t>(lg[i].control & 0xFFFF) << 32) |
                      (static_cast<uint64_t>(ex[i].gen & 0xFF) << 48));
        sig.push_back(static_cast<uint64_t>(static_cast<uint32_t>(ex[i].row)));
    }
    uint64_t key = 0xcbf29ce484222325ULL;
    for (const uint64_t v : sig) {
        key = (key ^ v) * 0x100000001b3ULL;
        key ^= key >> 29;
    }
    Plan<T, FOpA<T>> plan;
    std::vector<std::vector<int32_t>> rows_of_block;
    int64_t sweeps_before = 0;
    bool cached = false;
    {
        AdjPlanCache<T>& pc = adj_plan_cache<T>();
        std::lock_guard<std::mutex> lock(pc.m);
        auto it = pc.entries.find(key);
        if (it != pc.entries.end() && it->second.signature == sig) {
            plan = it->second.plan;
            rows_of_block = it->second.rows_of_block;
            sweeps_before = it->second.sweeps++;
            for (size_t i = 0; i < plan.ops.size(); ++i) {
                const LGate& x = lg[static_cast<size_t>(plan.op_gate[i])];
                for (int e = 0; e < 8; ++e) {
                    plan.ops[i].m[e] = static_cast<T>(x.m[e]);
                }
            }
            cached = true;
        }
    }
    const auto pbs = cached ? std::vector<PlanBlock> {} : form_blocks(lg, n, K, L, max_ops);
    for (const auto& pb : pbs) {
        // local row numbers inside the block
        std::vector<int32_t> rows;
        std::vector<AdjExtra> local(ex.size());
        for (int gi : pb.gates) {
            if (ex[gi].row >= 0) {
                AdjExtra e = ex[gi];
                e.row = static_cast<int32_t>(rows.size());
                rows.push_back(ex[gi].row);
                local[gi] = e;
            } else {
                local[gi] = ex[gi];
            }
        }
        plan_block<T, CfgA<T>, FOpA<T>>(pb, lg, n, plan, local.data());
        rows_of_block.push_back(std::move(rows));
    }
    for (const auto& fb : plan.blocks) {
        if (fb.phase_end - fb.phase_begin > MAX_PHASES_PER_BLOCK) {
            set_error(KT_ERR_INVALID, "fused adjoint planner produced too many phases");
            return KT_ERR_INVALID;
        }
    }
    if (!cached) {
        AdjPlanCache<T>& pc = adj_plan_cache<T>();
        std::lock_guard<std::mutex> lock(pc.m);
        if (pc.entries.size() >= 64) {
            pc.entries.clear();
        }
        AdjPlanEntry<T>& e = pc.entries[key];
        e = AdjPlanEntry<T> {};
        e.signature = sig;
        e.plan = plan;
        e.rows_of_block = rows_of_block;
        e.sweeps = 1;
    }
    const uint64_t n_tiles = uint64_t {1} << (n - K);
    const int grid = static_cast<int>(std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sm_count()) * 2));
    // device layout: blocks | phases | ops | rows | partials
    auto al = [](size_t v) { return (v + 255) & ~size_t {255}; };
    size_t n_rows_total = 0;
    size_t max_rows = 1;
    for (const auto& r : rows_of_block) {
        n_rows_total += r.size();
        max_rows = std::max(max_rows, r.size());
    }
    const size_t nb = plan.blocks.size() * sizeof(FBlock);
    const size_t np = plan.phases.size() * sizeof(FPhase);
    const size_t no = std::max<size_t>(1, plan.ops.size()) * sizeof(FOpA<T>);
    const size_t off_p = al(nb);
    const size_t off_o = al(off_p + np);
    const size_t off_r = al(off_o + no);
    const size_t off_part = al(off_r + std::max<size_t>(1, n_rows_total) * 4);
    const size_t need = al(off_part + max_rows * grid * 8);
    if (const int32_t rc = work.reserve(need); rc != KT_OK) {
        return rc;
    }
    std::vector<unsigned char> host(off_part, 0);
    std::memcpy(host.data(), plan.blocks.data(), nb);
    std::memcpy(host.data() + off_p, plan.phases.data(), np);
    if (!plan.ops.empty()) {
        std::memcpy(host.data() + off_o, plan.ops.data(), plan.ops.size() * sizeof(FOpA<T>));
    }
    {
        size_t w = 0;
        for (const auto& r : rows_of_block) {
            std::memcpy(host.data() + off_r + w * 4, r.data(), r.size() * 4);
            w += r.size();
        }
    }
    char* dev = static_cast<char*>(work.ptr);
    KT_CUDA(cudaMemcpyAsync(dev, host.data(), off_part, cudaMemcpyHostToDevice, psi.stream));
    const auto* d_blk = reinterpret_cast<const FBlock*>(dev);
    const auto* d_ph = reinterpret_cast<const FPhase*>(dev + off_p);
    const auto* d_ops = reinterpret_cast<const FOpA<T>*>(dev + off_o);
    const auto* d_rows = reinterpret_cast<const int32_t*>(dev + off_r);
    auto* d_part = reinterpret_cast<double*>(dev + off_part);
    static bool attr = false;
    if (!attr) {
        const int most = static_cast<int>(2 * (sizeof(C) << (CfgA<T>::RB + TB256)) + ADJ_MAX_OPS * sizeof(FOpA<T>) +
                                          ADJ_MAX_OPS * ADJ_WARPS * sizeof(double));
        KT_CUDA(cudaFuncSetAttribute(k_fused_adj<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
        attr = true;
    }
    const int threads = 1 << (K - RB);
    // compiled blocks: adjoint_jit = 1 always, 2 from a structure's second sweep
    std::vector<const void*> jk;
    const int jmode = tuning().adjoint_jit;
    if (threads >= 32 && threads <= 256 && (jmode == 1 || (jmode == 2 && sweeps_before >= 1))) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            dev = 0;
        }
        bool have = false;
        {
            AdjPlanCache<T>& pc = adj_plan_cache<T>();
            std::lock_guard<std::mutex> lock(pc.m);
            auto it = pc.entries.find(key);
            if (it != pc.entries.end() && it->second.device == dev && it->second.generation == jit_cache().generation &&
                it->second.kernels.size() == plan.blocks.size()) {
                jk = it->second.kernels;
                have = true;
            }
        }
        if (!have) {
            const int most = static_cast<int>(2 * (sizeof(C) << K) + max_rows * ADJ_WARPS * sizeof(double));
            if (jit_adj_kernels<T>(plan, RB, most, jk)) {
                AdjPlanCache<T>& pc = adj_plan_cache<T>();
                std::lock_guard<std::mutex> lock(pc.m);
                auto it = pc.entries.find(key);
                if (it != pc.entries.end()) {
                    it->second.kernels = jk;
                    it->second.device = dev;
                    it->second.generation = jit_cache().generation;
                }
            } else {
                jk.clear();
            }
        }
    }
    size_t row_off = 0;
    for (size_t b = 0; b < plan.blocks.size(); ++b) {
        const auto& fb = plan.blocks[b];
        const int nr = static_cast<int>(rows_of_block[b].size());
        if (!jk.empty()) {
            const size_t smem = 2 * (size_t {1} << K) * sizeof(C) + static_cast<size_t>(nr) * ADJ_WARPS * sizeof(double);
            const int nops = std::max(1, fb.op_end - fb.op_begin);
            std::vector<T> mats(8 * static_cast<size_t>(nops), T(0));
            for (int j = 0; j < fb.op_end - fb.op_begin; ++j) {
                for (int e = 0; e < 8; ++e) {
                    mats[8 * static_cast<size_t>(j) + e] = plan.ops[static_cast<size_t>(fb.op_begin + j)].m[e];
                }
            }
            void* pa = psi.amps;
            void* la = lam.amps;
            unsigned long long nt = n_tiles;
            double* pp = d_part;
            int nrr = nr;
            void* args[] = {&pa, &la, &nt, &pp, &nrr, mats.data()};
            KT_CUDA(cudaLaunchKernel(jk[b], dim3(static_cast<unsigned>(grid)), dim3(static_cast<unsigned>(threads)), args,
                                     smem, psi.stream));
            jit_cache().launches += 1;
        } else {
            const size_t smem = 2 * (size_t {1} << K) * sizeof(C) +
                                static_cast<size_t>(fb.op_end - fb.op_begin) * sizeof(FOpA<T>) +
                                static_cast<size_t>(nr) * ADJ_WARPS * sizeof(double);
            k_fused_adj<T><<<grid, threads, smem, psi.stream>>>(static_cast<C*>(psi.amps), static_cast<C*>(lam.amps),
                                                                d_blk + b, d_ph, d_ops, nr, d_part, n_tiles);
            KT_CHECK_LAUNCH("k_fused_adj");
        }
        if (nr > 0) {
            k_adj_rows<<<(nr + 127) / 128, 128, 0, psi.stream>>>(d_part, grid, d_rows + row_off, nr, dev_grad);
            KT_CHECK_LAUNCH("k_adj_rows");
        }
        row_off += static_cast<size_t>(nr);
        psi.last_launches += 1;
        psi.last_alg_bytes += 4.0 * sizeof(C) * static_cast<double>(psi.n_amps());
    }
    return KT_OK;
}

}  // namespace

int32_t adjoint_sweep_fused(State& psi, State& lam, const std::vector<AdjGate>& gates, double* dev_grad, DevBuf& work)
{
    const int rb = psi.dtype == KT_C128 ? CfgA<double>::RB : CfgA<float>::RB;
    if (psi.n_bits < rb + 5) {
        set_error(KT_ERR_UNSUPPORTED, "fused adjoint sweep needs at least RB + 5 qubits");
        return KT_ERR_UNSUPPORTED;
    }
    return psi.dtype == KT_C128 ? run_adjoint_sweep<double>(psi, lam, gates, dev_grad, work)
                                : run_adjoint_sweep<float>(psi, lam, gates, dev_grad, work);
}

namespace
{

template <typename T>
int32_t jit_compile_only_t(int n, const std::vector<LGate>& gates, int64_t* n_kernels)
{
    *n_kernels = 0;
    if (n < Cfg<T>::RB + 5 || gates.empty()) {
        return KT_OK;
    }
    Plan<T> plan;
    int K = 0;
    bool rb3 = false;
    if (const int32_t rc = fused_plan<T>(n, gates, plan, &K, &rb3); rc != KT_OK) {
        return rc;
    }
    const int RB = rb3 ? Cfg3::RB : Cfg<T>::RB;
    const int threads = 1 << (K - RB);
    // complex64 applies renormalise by default
    const bool norm = std::is_same<T, float>::value && tuning().c64_renormalize != 0;
    const bool tma = tuning().jit_tma != 0 && std::is_same<T, double>::value && !norm;
    std::vector<std::string> sources(1, JIT_PRELUDE);
    std::vector<std::vector<std::string>> names(1);
    for (size_t b = 0; b < plan.blocks.size(); ++b) {
        const std::string name = "kt_jc" + std::to_string(b);
        TmaCfg c;
        c.groups = 1;
        c.stages = std::max(tuning().jit_tma_stages, 2);
        c.geom = tma_geom(plan.blocks[b], n);
        const bool bt = tma && c.geom.ok;
        const int bthreads = bt ? c.groups * threads + 32 : threads;
        sources[0] += "extern \"C\" __global__ void __launch_bounds__(" + std::to_string(bthreads) + ", " +
                      std::to_string(bt ? tuning().jit_tma_ctas : (threads > 256 ? 1 : 2)) + ") " + name +
                      jit_block_body<T>(plan, b, RB, norm, bt ? &c : nullptr) + "\n";
        names[0].push_back(name);
    }
    std::vector<std::vector<const void*>> got;
    if (const int32_t rc = jit_compile(sources, names, got, false); rc != KT_OK) {
        return rc;
    }
    *n_kernels = static_cast<int64_t>(plan.blocks.size());
    return KT_OK;
}

}  // namespace

namespace
{

// a plan of the batch engine rebuilt from its raw records (same types in both units)
template <typename T, typename O>
bool plan_from_view(const BatchPlanView& v, Plan<T, O>& plan)
{
    if (v.rec_bytes[0] != static_cast<int64_t>(sizeof(FBlock)) || v.rec_bytes[1] != static_cast<int64_t>(sizeof(FPhase)) ||
        v.rec_bytes[2] != static_cast<int64_t>(sizeof(O))) {
        return false;
    }
    plan.blocks.resize(static_cast<size_t>(v.n_blocks));
    plan.phases.resize(static_cast<size_t>(v.n_phases));
    plan.ops.resize(static_cast<size_t>(v.n_ops));
    if (v.n_blocks > 0) std::memcpy(plan.blocks.data(), v.blocks, plan.blocks.size() * sizeof(FBlock));
    if (v.n_phases > 0) std::memcpy(plan.phases.data(), v.phases, plan.phases.size() * sizeof(FPhase));
    if (v.n_ops > 0) std::memcpy(static_cast<void*>(plan.ops.data()), v.ops, plan.ops.size() * sizeof(O));
    return true;
}

// Batched kernels stay loaded for the life of the process, in a cache of
// their own (the single-state cache unloads its programs when it fills), so
// a later batch with classes of the same structure skips their compile.  Past
// BATCH_CACHE_MAX kernels a batch compiles, and owns, the ones it misses.
constexpr size_t BATCH_CACHE_MAX = 8192;

struct BatchKernelCache
{
    std::mutex m;
    std::unordered_map<std::string, const void*> kernels;  // launch bounds + body -> kernel
    std::map<std::pair<const void*, int>, int32_t> smem;   // (kernel, device) -> shared-memory limit set
    std::vector<cudaLibrary_t> libs;                        // never unloaded
};

BatchKernelCache& batch_kernel_cache()
{
    static BatchKernelCache* c = new BatchKernelCache();  // outlives every batch, never destroyed
    return *c;
}

template <typename T>
int32_t jit_batch_compile_t(const std::vector<BatchPlanView>& fwd, const std::vector<BatchPlanView>& bwd,
                            std::vector<std::vector<const void*>>& fk, std::vector<std::vector<const void*>>& bk,
                            std::vector<int32_t>& fwd_smem, std::vector<std::vector<int32_t>>& bwd_smem,
                            std::vector<cudaLibrary_t>& libs)
{
    using C = typename CxT<T>::type;
    const std::string bounds = "__launch_bounds__(256, 2)";
    std::vector<std::string> texts;          // unique kernel bodies (launch bounds first)
    std::vector<int32_t> smem;               // dynamic shared memory of each
    std::vector<char> is_adj;
    std::unordered_map<std::string, size_t> index;
    auto intern = [&](std::string text, int32_t bytes, bool adj) {
        auto it = index.find(text);
        if (it != index.end()) {
            smem[it->second] = std::max(smem[it->second], bytes);
            return it->second;
        }
        const size_t i = texts.size();
        index.emplace(text, i);
        texts.push_back(std::move(text));
        smem.push_back(bytes);
        is_adj.push_back(adj ? 1 : 0);
        return i;
    };
    std::vector<std::vector<size_t>> fidx(fwd.size()), bidx(bwd.size());
    fwd_smem.assign(fwd.size(), 0);
    bwd_smem.assign(bwd.size(), {});
    {
        const JitBatch jb {sizeof(FOp<T>), offsetof(FOp<T>, m)};
        JitBatchScope scope(&jb);
        for (size_t c = 0; c < fwd.size(); ++c) {
            Plan<T> plan;
            if (!plan_from_view(fwd[c], plan)) {
                set_error(KT_ERR_INVALID, "batched block kernels: plan record sizes differ");
                return KT_ERR_INVALID;
            }
            for (size_t b = 0; b < plan.blocks.size(); ++b) {
                const int K = plan.blocks[b].K;
                const int32_t bytes = static_cast<int32_t>((size_t {1} << K) * sizeof(C) * (jit_async(K, sizeof(C)) ? 2 : 1));
                fwd_smem[c] = std::max(fwd_smem[c], bytes);
                fidx[c].push_back(intern(bounds + jit_block_body<T>(plan, b, Cfg<T>::RB, false, nullptr), bytes, false));
            }
        }
    }
    {
        const JitBatch jb {sizeof(FOpA<T>), offsetof(FOpA<T>, m)};
        JitBatchScope scope(&jb);
        for (size_t c = 0; c < bwd.size(); ++c) {
            Plan<T, FOpA<T>> plan;
            if (!plan_from_view(bwd[c], plan)) {
                set_error(KT_ERR_INVALID, "batched block kernels: plan record sizes differ");
                return KT_ERR_INVALID;
            }
            for (size_t b = 0; b < plan.blocks.size(); ++b) {
                const FBlock& fb = plan.blocks[b];
                int rows = 0;
                for (int o = fb.op_begin; o < fb.op_end; ++o) {
                    rows = std::max(rows, plan.ops[static_cast<size_t>(o)].row + 1);
                }
                const int32_t bytes = static_cast<int32_t>(2 * (size_t {1} << fb.K) * sizeof(C) +
                                                           static_cast<size_t>(std::max(rows, 1)) * ADJ_WARPS * sizeof(double));
                bwd_smem[c].push_back(bytes);
                bidx[c].push_back(intern(bounds + jit_adj_body<T>(plan, b, CfgA<T>::RB), bytes, true));
            }
        }
    }
    BatchKernelCache& cache = batch_kernel_cache();
    std::lock_guard<std::mutex> lock(cache.m);
    std::vector<const void*> handle(texts.size(), nullptr);
    std::vector<size_t> missing;
    for (size_t i = 0; i < texts.size(); ++i) {
        auto it = cache.kernels.find(texts[i]);
        if (it != cache.kernels.end()) {
            handle[i] = it->second;
        } else {
            missing.push_back(i);
        }
    }
    if (!missing.empty()) {
        // programs of a few kernels each, compiled on parallel host threads;
        // grouped in the order of their texts, so the same kernels always make
        // the same programs (and hit the on-disk cubin cache in a new process)
        std::sort(missing.begin(), missing.end(), [&](size_t x, size_t y) { return texts[x] < texts[y]; });
        const bool keep = cache.kernels.size() + missing.size() <= BATCH_CACHE_MAX;
        const size_t per_prog = 4;
        const size_t n_prog = (missing.size() + per_prog - 1) / per_prog;
        std::vector<std::string> sources(n_prog, JIT_PRELUDE);
        std::vector<std::vector<std::string>> names(n_prog);
        for (size_t m = 0; m < missing.size(); ++m) {
            const size_t i = missing[m];
            const std::string name = std::string(is_adj[i] ? "kt_jab" : "kt_jbb") + std::to_string(m);
            sources[m / per_prog] += "extern \"C\" __global__ void " + bounds + " " + name +
                                     texts[i].substr(bounds.size()) + "\n";
            names[m / per_prog].push_back(name);
        }
        std::vector<std::vector<const void*>> got;
        if (const int32_t rc = jit_compile(sources, names, got, true, keep ? &cache.libs : &libs); rc != KT_OK) {
            return rc;
        }
        for (size_t m = 0; m < missing.size(); ++m) {
            handle[missing[m]] = got[m / per_prog][m % per_prog];
            if (keep) {
                cache.kernels.emplace(texts[missing[m]], handle[missing[m]]);
            }
        }
    }
    int dev = 0;
    KT_CUDA(cudaGetDevice(&dev));
    for (size_t i = 0; i < texts.size(); ++i) {
        // cached kernels remember their limit per device; a batch's own ones are set every time
        const bool cached = cache.kernels.count(texts[i]) != 0;
        int32_t dummy = 0;
        int32_t& set = cached ? cache.smem[std::make_pair(handle[i], dev)] : dummy;
        if (set < smem[i]) {
            KT_CUDA(cudaKernelSetAttributeForDevice(reinterpret_cast<cudaKernel_t>(const_cast<void*>(handle[i])),
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, smem[i], dev));
            set = smem[i];
        }
    }
    fk.assign(fwd.size(), {});
    bk.assign(bwd.size(), {});
    for (size_t c = 0; c < fwd.size(); ++c) {
        for (size_t i : fidx[c]) {
            fk[c].push_back(handle[i]);
        }
    }
    for (size_t c = 0; c < bwd.size(); ++c) {
        for (size_t i : bidx[c]) {
            bk[c].push_back(handle[i]);
        }
    }
    return KT_OK;
}

}  // namespace

int32_t jit_batch_compile(int32_t dtype, const std::vector<BatchPlanView>& fwd, const std::vector<BatchPlanView>& bwd,
                          std::vector<std::vector<const void*>>& fk, std::vector<std::vector<const void*>>& bk,
                          std::vector<int32_t>& fwd_smem, std::vector<std::vector<int32_t>>& bwd_smem,
                          std::vector<cudaLibrary_t>& libs)
{
    return dtype == KT_C128 ? jit_batch_compile_t<double>(fwd, bwd, fk, bk, fwd_smem, bwd_smem, libs)
                            : jit_batch_compile_t<float>(fwd, bwd, fk, bk, fwd_smem, bwd_smem, libs);
}

int32_t jit_adjoint_compile_only(int n, int32_t dtype, const std::vector<AdjGate>& gates, int64_t* n_kernels)
{
    auto run = [&](auto tag) -> int32_t {
        using T = decltype(tag);
        constexpr int RB = CfgA<T>::RB;
        constexpr int L = CfgA<T>::L;
        *n_kernels = 0;
        if (n < RB + 5 || gates.empty()) {
            return KT_OK;
        }
        const int K = std::min(n, RB + TB256);
        std::vector<LGate> lg;
        std::vector<AdjExtra> ex;
        for (const auto& g : gates) {
            lg.push_back(g.adj);
            ex.push_back(AdjExtra {g.row, g.gen});
        }
        const auto pbs = form_blocks(lg, n, K, L, static_cast<size_t>(std::min(ADJ_MAX_OPS, tuning().fused_max_ops)));
        Plan<T, FOpA<T>> plan;
        for (const auto& pb : pbs) {
            std::vector<AdjExtra> local(ex.size());
            int32_t r = 0;
            for (int gi : pb.gates) {
                local[gi] = ex[gi];
                if (ex[gi].row >= 0) {
                    local[gi].row = r++;
                }
            }
            plan_block<T, CfgA<T>, FOpA<T>>(pb, lg, n, plan, local.data());
        }
        std::vector<std::string> sources(1, JIT_PRELUDE);
        std::vector<std::vector<std::string>> names(1);
        for (size_t b = 0; b < plan.blocks.size(); ++b) {
            const std::string name = "kt_jac" + std::to_string(b);
            sources[0] += "extern \"C\" __global__ void __launch_bounds__(256, 2) " + name + jit_adj_body<T>(plan, b, RB) + "\n";
            names[0].push_back(name);
        }
        std::vector<std::vector<const void*>> got;
        if (const int32_t rc = jit_compile(sources, names, got, false); rc != KT_OK) {
            return rc;
        }
        *n_kernels = static_cast<int64_t>(plan.blocks.size());
        return KT_OK;
    };
    return dtype == KT_C64 ? run(float {}) : run(double {});
}

int32_t jit_async_error()
{
    TmaErr& e = tma_err();
    std::lock_guard<std::mutex> lock(e.m);
    if (e.host == nullptr) {
        return KT_OK;
    }
    for (const auto& kv : e.dev) {
        volatile unsigned int* h = e.host + kv.first;
        if (*h != 0u) {
            // clear it on the device (the next launches must start clean) and here
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(kv.first);
            cudaMemset(kv.second, 0, sizeof(unsigned int));
            cudaDeviceSynchronize();
            cudaSetDevice(cur);
            *h = 0u;
            set_error(KT_ERR_TIMEOUT, "a TMA block kernel's bounded wait ran out on device " + std::to_string(kv.first) +
                                          ": the results of the applies since the last check are void");
            return KT_ERR_TIMEOUT;
        }
    }
    return KT_OK;
}

int32_t jit_compile_only(int n, int32_t dtype, const std::vector<LGate>& gates, int64_t* n_kernels)
{
    return dtype == KT_C64 ? jit_compile_only_t<float>(n, gates, n_kernels)
                           : jit_compile_only_t<double>(n, gates, n_kernels);
}

void jit_stats(int64_t* compiled, int64_t* launches, int32_t* failed)
{
    JitCache& jc = jit_cache();
    std::lock_guard<std::mutex> lock(jc.m);
    *compiled = jc.compiled;
    *launches = jc.launches;
    *failed = jc.failed ? 1 : 0;
}

namespace
{

template <typename T>
int32_t jit_prepare_t(State& s, const std::vector<LGate>& gates)
{
    const int n = s.n_bits;
    if (n < Cfg<T>::RB + 5 || gates.empty()) {
        return KT_OK;  // applied one gate at a time: nothing to compile
    }
    Plan<T> plan;
    int K = 0;
    bool rb3 = false;
    uint64_t key = 0;
    if (const int32_t rc = fused_plan_cached<T>(n, gates, plan, &K, &rb3, &key); rc != KT_OK) {
        return rc;
    }
    const int threads = 1 << (K - (rb3 ? Cfg3::RB : Cfg<T>::RB));
    int shape = threads > 256 ? 0 : (tuning().fused_ctas_per_sm == 1 ? 1 : 2);
    if (rb3) {
        shape = threads > 256 ? 3 : 4;
    }
    double* parts = nullptr;
    int n_parts = 0;
    if (std::is_same<T, float>::value && tuning().c64_renormalize != 0) {
        n_parts = sm_count() * 4;
        if (const int32_t rc = s.scratch2.reserve(3 * static_cast<size_t>(n_parts) * sizeof(double)); rc != KT_OK) {
            return rc;
        }
        parts = static_cast<double*>(s.scratch2.ptr);
    }
    int32_t rc = KT_OK;
    if (!jit_launch<T>(s, plan, key, K, rb3, threads, shape, parts, &rc, &n_parts, true)) {
        std::string why;
        if (!jit_available(&why)) {
            set_error(KT_ERR_CUDA, why);
        } else {
            set_error(KT_ERR_CUDA, "the block kernels of this circuit could not be compiled; applies use the "
                                   "precompiled kernels");
        }
        return KT_ERR_CUDA;
    }
    return rc;
}

}  // namespace

int32_t jit_prepare(State& s, const std::vector<LGate>& gates)
{
    return s.dtype == KT_C128 ? jit_prepare_t<double>(s, gates) : jit_prepare_t<float>(s, gates);
}

int32_t apply_fused(State& s, const std::vector<LGate>& gates)
{
    return s.dtype == KT_C128 ? run_fused<double>(s, gates) : run_fused<float>(s, gates);
}

namespace
{

template <typename T>
void plan_only(int n, const std::vector<LGate>& gates, int64_t* blocks, int64_t* phases, int64_t* ops, int64_t* transposes,
               std::vector<int32_t>* order)
{
    *blocks = 0;
    *phases = 0;
    *ops = 0;
    *transposes = 0;
    if (n < Cfg<T>::RB + 5 || gates.empty()) {
        return;
    }
    Plan<T> plan;
    int K = 0;
    bool rb3 = false;
    if (fused_plan<T>(n, gates, plan, &K, &rb3) != KT_OK) {
        return;
    }
    *blocks = static_cast<int64_t>(plan.blocks.size());
    *phases = static_cast<int64_t>(plan.phases.size());
    *ops = static_cast<int64_t>(plan.ops.size()) + plan.folded;  // every gate placed, folded ones included
    *transposes = plan.transposes;
    if (order != nullptr) {
        *order = plan.run_order;
    }
}

}  // namespace

// Per block of a complex128 apply: {ops, layout phases, transposes, FP64
// instructions per amplitude of its compiled form}.  The FP64 count is a
// model of the generated gate bodies: per pair a general gate costs 16 (12
// scaled), a real or RX-like one 8 (4 scaled), an anti-diagonal one 8, a
// swap 0, a diagonal one on a register bit 8 (4 one-sided), a diagonal
// factor on a thread or tile-external bit 8; a control on a register bit or
// outside the tile halves the work, one on a thread bit masks lanes without
// saving issue slots.
int32_t plan_blocks(int n, const std::vector<LGate>& gates, std::vector<double>& out)
{
    out.clear();
    Plan<double> plan;
    int K = 0;
    bool rb3 = false;
    if (const int32_t rc = fused_plan<double>(n, gates, plan, &K, &rb3); rc != KT_OK) {
        return rc;
    }
    for (size_t b = 0; b < plan.blocks.size(); ++b) {
        const FBlock& fb = plan.blocks[b];
        const JitScale js = jit_scale_plan(plan, b);
        double per_pair = 0.0;
        for (int o = fb.op_begin; o < fb.op_end; ++o) {
            const FOp<double>& op = plan.ops[static_cast<size_t>(o)];
            const int sc = jit_scale_code(plan, b, o - fb.op_begin, js);
            double c = 0.0;
            switch (op.kind) {
                case OP_GEN: c = sc == 4 ? 12.0 : 16.0; break;
                case OP_GENR: c = (sc == 1 || sc == 2) ? 4.0 : 8.0; break;
                case OP_RXL: c = sc == 3 ? 4.0 : 8.0; break;
                case OP_ANTI: c = 8.0; break;
                case OP_SWAP: c = 0.0; break;
                default: c = (op.tslot != NO_SLOT && (op.kind == OP_DIAG1 || sc == 5)) ? 4.0 : 8.0; break;
            }
            if (op.cslot != NO_SLOT) {
                c *= 0.5;
            }
            if (op.cglob != 0) {
                c *= 0.5;
            }
            per_pair += c;
        }
        out.push_back(static_cast<double>(fb.op_end - fb.op_begin));
        out.push_back(static_cast<double>(fb.phase_end - fb.phase_begin));
        out.push_back(static_cast<double>(fb.phase_end - fb.phase_begin - 1));
        out.push_back(per_pair / 2.0);
    }
    return KT_OK;
}

int32_t plan_stats(int n, int32_t dtype, const std::vector<LGate>& gates, int64_t* blocks, int64_t* phases,
                   int64_t* ops, int64_t* transposes, std::vector<int32_t>* order)
{
    if (order != nullptr) {
        order->clear();
    }
    if (dtype == KT_C128) {
        plan_only<double>(n, gates, blocks, phases, ops, transposes, order);
    } else {
        plan_only<float>(n, gates, blocks, phases, ops, transposes, order);
    }
    return KT_OK;
}

bool tma_encode_rows_f32(void* base, uint64_t row_floats, uint64_t rows, uint32_t box_floats, uint32_t box_rows,
                         void* out)
{
    EncodeTiledFn fn = encode_tiled();
    if (fn == nullptr) {
        return false;
    }
    const cuuint64_t dims[2] = {row_floats, rows};
    const cuuint64_t strides[1] = {row_floats * sizeof(float)};
    const cuuint32_t box[2] = {box_floats, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(static_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

unsigned int* async_error_word(int dev, unsigned int** host)
{
    return tma_err_word(dev, host);
}

}  // namespace kt
