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
//    phases.  Shared memory is XOR-swizzled so the transposes are free of bank
//    conflicts when the lane bits are chosen with distinct residues.
//  * Loads and stores use a layout whose lane bits are the L lowest qubits:
//    each warp instruction touches whole 128-byte lines.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "kt_complex.cuh"
#include "kt_internal.cuh"

namespace kt
{

namespace
{

constexpr int KMAX = 14;
constexpr int MAX_OPS_PER_BLOCK = 512;

template <typename T>
struct FOp
{
    int32_t kind;        // KIND_GEN / KIND_DIAG / KIND_ANTI
    int32_t tslot;       // GEN/ANTI: register slot of the target; DIAG: tile bit of the target or -1
    uint32_t cmask_loc;  // control as tile bits
    int32_t flags;       // bit0: DIAG with m00 == 1
    uint64_t cmask_glob; // control as global bits (outside the tile)
    uint64_t tglob;      // DIAG target outside the tile: its global bit
    T m[8];
};

struct FPhase
{
    int8_t slot_bit[KMAX];  // slot -> tile bit; slots [0, RB) are register bits, [RB, K) thread bits
    int16_t pad;
    int32_t op_begin;
    int32_t op_end;
};

struct FBlock
{
    int32_t K;
    int32_t nfree;
    int32_t phase_begin;
    int32_t phase_end;
    int32_t qubit[KMAX];    // tile bit -> qubit
    int32_t freebit[64];    // qubits outside the tile, ascending
};

// tile bit configuration per amplitude type
template <typename T>
struct Cfg;
template <>
struct Cfg<double>
{
    static constexpr int RB = 4;     // 16 amplitudes per thread
    static constexpr int TBMAX = 8;  // 256 threads
    static constexpr int L = 3;      // 8 x 16 B = 128 B runs
    static constexpr int LANES = 3;  // lane bits that must differ in residue (16-B smem accesses)
};
template <>
struct Cfg<float>
{
    static constexpr int RB = 5;     // 32 amplitudes per thread
    static constexpr int TBMAX = 8;
    static constexpr int L = 4;      // 16 x 8 B = 128 B runs
    static constexpr int LANES = 4;
};

// XOR swizzle of a tile index for bank-conflict-free transposes: the low G bits
// are XORed with a fold of the higher bits (G = 3 for 16-byte, 4 for 8-byte elements).
template <int G>
__device__ __forceinline__ uint32_t swz(uint32_t l)
{
    uint32_t f = 0;
#pragma unroll
    for (int s = G; s < 32; s += G) {
        f ^= l >> s;
    }
    return l ^ (f & ((1u << G) - 1));
}

template <int RB>
__device__ __forceinline__ uint32_t rloc(int i, const uint32_t (&rbit)[RB])
{
    uint32_t l = 0;
#pragma unroll
    for (int s = 0; s < RB; ++s) {
        if (i & (1 << s)) {
            l |= rbit[s];
        }
    }
    return l;
}

template <typename C, int RB, int S>
__device__ __forceinline__ void gen_pairs(C (&v)[1 << RB], const C m00, const C m01, const C m10, const C m11,
                                          uint32_t tloc, const uint32_t (&rbit)[RB], uint32_t cm)
{
#pragma unroll
    for (int i = 0; i < (1 << RB); ++i) {
        if (i & (1 << S)) {
            continue;
        }
        const int j = i | (1 << S);
        const uint32_t l = tloc | rloc<RB>(i, rbit);
        if ((l & cm) == cm) {
            const C a = v[i];
            const C b = v[j];
            v[i] = cfma(m01, b, cmul(m00, a));
            v[j] = cfma(m11, b, cmul(m10, a));
        }
    }
}

template <typename C, int RB, int S>
__device__ __forceinline__ void anti_pairs(C (&v)[1 << RB], const C m01, const C m10, bool pure_swap, uint32_t tloc,
                                           const uint32_t (&rbit)[RB], uint32_t cm)
{
#pragma unroll
    for (int i = 0; i < (1 << RB); ++i) {
        if (i & (1 << S)) {
            continue;
        }
        const int j = i | (1 << S);
        const uint32_t l = tloc | rloc<RB>(i, rbit);
        if ((l & cm) == cm) {
            const C a = v[i];
            const C b = v[j];
            if (pure_swap) {
                v[i] = b;
                v[j] = a;
            } else {
                v[i] = cmul(m01, b);
                v[j] = cmul(m10, a);
            }
        }
    }
}

template <typename T, int RB>
__device__ __forceinline__ void apply_op(typename CxT<T>::type (&v)[1 << RB], const FOp<T>* __restrict__ opp,
                                         uint32_t tloc, const uint32_t (&rbit)[RB], uint64_t base)
{
    using C = typename CxT<T>::type;
    const int kind = opp->kind;
    const uint64_t cg = opp->cmask_glob;
    if ((base & cg) != cg) {
        return;  // control outside the tile is 0 for this whole tile
    }
    const uint32_t cm = opp->cmask_loc;
    const int ts = opp->tslot;
    if (kind == KIND_DIAG) {
        const C d0 = make_cx<T>(opp->m[0], opp->m[1]);
        const C d1 = make_cx<T>(opp->m[6], opp->m[7]);
        const bool one = opp->flags & 1;
        const uint64_t tg = opp->tglob;
        if (ts < 0) {
            // target outside the tile: one factor for the whole tile
            const bool b = (base & tg) != 0;
            if (!b && one) {
                return;
            }
            const C d = b ? d1 : d0;
#pragma unroll
            for (int i = 0; i < (1 << RB); ++i) {
                const uint32_t l = tloc | rloc<RB>(i, rbit);
                if ((l & cm) == cm) {
                    v[i] = cmul(d, v[i]);
                }
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            const uint32_t l = tloc | rloc<RB>(i, rbit);
            if ((l & cm) == cm) {
                if ((l >> ts) & 1) {
                    v[i] = cmul(d1, v[i]);
                } else if (!one) {
                    v[i] = cmul(d0, v[i]);
                }
            }
        }
        return;
    }
    const C m01 = make_cx<T>(opp->m[2], opp->m[3]);
    const C m10 = make_cx<T>(opp->m[4], opp->m[5]);
    if (kind == KIND_ANTI) {
        const bool pure = opp->flags & 2;
        switch (ts) {
            case 0: anti_pairs<C, RB, 0>(v, m01, m10, pure, tloc, rbit, cm); break;
            case 1: anti_pairs<C, RB, 1>(v, m01, m10, pure, tloc, rbit, cm); break;
            case 2: anti_pairs<C, RB, 2>(v, m01, m10, pure, tloc, rbit, cm); break;
            case 3: anti_pairs<C, RB, 3>(v, m01, m10, pure, tloc, rbit, cm); break;
            default:
                if constexpr (RB > 4) {
                    anti_pairs<C, RB, (RB > 4 ? 4 : 0)>(v, m01, m10, pure, tloc, rbit, cm);
                }
                break;
        }
        return;
    }
    const C m00 = make_cx<T>(opp->m[0], opp->m[1]);
    const C m11 = make_cx<T>(opp->m[6], opp->m[7]);
    switch (ts) {
        case 0: gen_pairs<C, RB, 0>(v, m00, m01, m10, m11, tloc, rbit, cm); break;
        case 1: gen_pairs<C, RB, 1>(v, m00, m01, m10, m11, tloc, rbit, cm); break;
        case 2: gen_pairs<C, RB, 2>(v, m00, m01, m10, m11, tloc, rbit, cm); break;
        case 3: gen_pairs<C, RB, 3>(v, m00, m01, m10, m11, tloc, rbit, cm); break;
        default:
            if constexpr (RB > 4) {
                gen_pairs<C, RB, (RB > 4 ? 4 : 0)>(v, m00, m01, m10, m11, tloc, rbit, cm);
            }
            break;
    }
}

// register-bit strides (global) and the thread offset of a layout
template <int RB>
__device__ __forceinline__ void layout_global(const FPhase& ph, const FBlock& bk, int K, uint32_t t,
                                              uint64_t (&rstride)[RB], uint64_t& toff)
{
#pragma unroll
    for (int s = 0; s < RB; ++s) {
        rstride[s] = uint64_t {1} << bk.qubit[ph.slot_bit[s]];
    }
    toff = 0;
    for (int s = RB; s < K; ++s) {
        if ((t >> (s - RB)) & 1) {
            toff |= uint64_t {1} << bk.qubit[ph.slot_bit[s]];
        }
    }
}

template <int RB>
__device__ __forceinline__ void layout_local(const FPhase& ph, int K, uint32_t t, uint32_t (&rbit)[RB], uint32_t& tloc)
{
#pragma unroll
    for (int s = 0; s < RB; ++s) {
        rbit[s] = 1u << ph.slot_bit[s];
    }
    tloc = 0;
    for (int s = RB; s < K; ++s) {
        if ((t >> (s - RB)) & 1) {
            tloc |= 1u << ph.slot_bit[s];
        }
    }
}

template <int RB>
__device__ __forceinline__ uint64_t roff(int i, const uint64_t (&rstride)[RB])
{
    uint64_t o = 0;
#pragma unroll
    for (int s = 0; s < RB; ++s) {
        if (i & (1 << s)) {
            o |= rstride[s];
        }
    }
    return o;
}

template <typename T>
__global__ void __launch_bounds__(256, 2) k_fused(typename CxT<T>::type* __restrict__ a, const FBlock* __restrict__ blk,
                                                  const FPhase* __restrict__ phases, const FOp<T>* __restrict__ ops,
                                                  uint64_t n_tiles)
{
    using C = typename CxT<T>::type;
    constexpr int RB = Cfg<T>::RB;
    constexpr int R = 1 << RB;
    constexpr int G = (sizeof(C) == 16) ? 3 : 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);

    __shared__ FBlock bk;
    if (threadIdx.x == 0) {
        bk = *blk;
    }
    __syncthreads();
    const int K = bk.K;
    const uint32_t t = threadIdx.x;
    const int pb = bk.phase_begin;
    const int pe = bk.phase_end;

    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        uint64_t base = 0;
        for (int k = 0; k < bk.nfree; ++k) {
            if ((tile >> k) & 1) {
                base |= uint64_t {1} << bk.freebit[k];
            }
        }
        C v[R];
        {
            const FPhase ph = phases[pb];
            uint64_t rs[RB];
            uint64_t toff;
            layout_global<RB>(ph, bk, K, t, rs, toff);
            const C* src = a + base + toff;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                v[i] = src[roff<RB>(i, rs)];
            }
        }
        uint32_t rbit[RB];
        uint32_t tloc;
        for (int p = pb; p < pe; ++p) {
            const FPhase ph = phases[p];
            if (p > pb) {
                // transpose: registers (old layout) -> smem -> registers (new layout)
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    sm[swz<G>(tloc | rloc<RB>(i, rbit))] = v[i];
                }
                __syncthreads();
                layout_local<RB>(ph, K, t, rbit, tloc);
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    v[i] = sm[swz<G>(tloc | rloc<RB>(i, rbit))];
                }
                __syncthreads();
            } else {
                layout_local<RB>(ph, K, t, rbit, tloc);
            }
            for (int o = ph.op_begin; o < ph.op_end; ++o) {
                apply_op<T, RB>(v, ops + o, tloc, rbit, base);
            }
        }
        {
            const FPhase ph = phases[pe - 1];
            uint64_t rs[RB];
            uint64_t toff;
            layout_global<RB>(ph, bk, K, t, rs, toff);
            C* dst = a + base + toff;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                dst[roff<RB>(i, rs)] = v[i];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host planner

struct PlanBlock
{
    int K;
    std::vector<int> qubits;     // tile bit -> qubit (ascending)
    std::vector<int> gates;      // gate indices in execution order
};

uint64_t bit(int q)
{
    return uint64_t {1} << q;
}

// Greedy block formation: in circuit order, take each gate that does not
// share a qubit with a gate skipped before it and whose target (when it must
// be in the tile) fits in the K-qubit set.
std::vector<PlanBlock> form_blocks(const std::vector<LGate>& g, int n, int K, int L)
{
    std::vector<PlanBlock> out;
    std::vector<int> pend(g.size());
    std::iota(pend.begin(), pend.end(), 0);
    const uint64_t all = (n >= 64) ? ~uint64_t {0} : (bit(n) - 1);
    while (!pend.empty()) {
        uint64_t Q = bit(L) - 1;
        uint64_t blocked = 0;
        std::vector<int> take;
        std::vector<int> rest;
        rest.reserve(pend.size());
        for (size_t k = 0; k < pend.size(); ++k) {
            const int idx = pend[k];
            const LGate& x = g[idx];
            const uint64_t touch = bit(x.target) | (x.control >= 0 ? bit(x.control) : 0);
            if ((touch & blocked) != 0 || take.size() >= static_cast<size_t>(MAX_OPS_PER_BLOCK)) {
                blocked |= touch;
                rest.push_back(idx);
            } else {
                const uint64_t need = (x.kind == KIND_DIAG) ? 0 : bit(x.target);
                if (__builtin_popcountll(Q | need) <= K) {
                    Q |= need;
                    take.push_back(idx);
                } else {
                    blocked |= touch;
                    rest.push_back(idx);
                }
            }
            if (blocked == all) {
                rest.insert(rest.end(), pend.begin() + static_cast<long>(k) + 1, pend.end());
                break;
            }
        }
        // fill the tile up to K qubits with the lowest free qubits (longer contiguous runs)
        for (int q = 0; q < n && __builtin_popcountll(Q) < K; ++q) {
            Q |= bit(q);
        }
        PlanBlock b;
        b.K = K;
        for (int q = 0; q < n; ++q) {
            if (Q & bit(q)) {
                b.qubits.push_back(q);
            }
        }
        b.gates = std::move(take);
        out.push_back(std::move(b));
        pend.swap(rest);
    }
    return out;
}

struct Layout
{
    std::vector<int> regs;   // RB tile bits
};

// Thread-slot order: lanes first (distinct residues mod LANES, preferring the
// low tile bits, which are the contiguous qubits), then the remaining bits.
void make_slots(const std::vector<int>& regs, int K, int LANES, int8_t* slot_bit)
{
    std::vector<bool> is_reg(K, false);
    for (int r : regs) {
        is_reg[r] = true;
    }
    int s = 0;
    for (int r : regs) {
        slot_bit[s++] = static_cast<int8_t>(r);
    }
    std::vector<int> lanes;
    std::vector<bool> used(K, false);
    // prefer tile bits 0..LANES-1 when none is a register bit
    bool low_free = true;
    for (int b = 0; b < LANES; ++b) {
        low_free = low_free && !is_reg[b];
    }
    if (low_free) {
        for (int b = 0; b < LANES; ++b) {
            lanes.push_back(b);
        }
    } else {
        std::vector<bool> res_used(LANES, false);
        for (int b = 0; b < K && static_cast<int>(lanes.size()) < LANES; ++b) {
            if (!is_reg[b] && !res_used[b % LANES]) {
                res_used[b % LANES] = true;
                lanes.push_back(b);
            }
        }
        for (int b = 0; b < K && static_cast<int>(lanes.size()) < LANES; ++b) {
            if (!is_reg[b] && std::find(lanes.begin(), lanes.end(), b) == lanes.end()) {
                lanes.push_back(b);
            }
        }
    }
    for (int b : lanes) {
        slot_bit[s++] = static_cast<int8_t>(b);
        used[b] = true;
    }
    for (int b = 0; b < K; ++b) {
        if (!is_reg[b] && !used[b]) {
            slot_bit[s++] = static_cast<int8_t>(b);
        }
    }
}

template <typename T>
struct Plan
{
    std::vector<FBlock> blocks;
    std::vector<FPhase> phases;
    std::vector<FOp<T>> ops;
    int transposes {0};
};

template <typename T>
void plan_block(const PlanBlock& pb, const std::vector<LGate>& g, int n, Plan<T>& plan)
{
    constexpr int RB = Cfg<T>::RB;
    constexpr int L = Cfg<T>::L;
    constexpr int LANES = Cfg<T>::LANES;
    const int K = pb.K;
    std::vector<int> loc(n, -1);
    for (int j = 0; j < K; ++j) {
        loc[pb.qubits[j]] = j;
    }
    FBlock fb {};
    fb.K = K;
    fb.nfree = n - K;
    for (int j = 0; j < K; ++j) {
        fb.qubit[j] = pb.qubits[j];
    }
    int nf = 0;
    for (int q = 0; q < n; ++q) {
        if (loc[q] < 0) {
            fb.freebit[nf++] = q;
        }
    }
    // ops and the register bit each needs (-1 = none)
    const size_t m = pb.gates.size();
    std::vector<int> need(m, -1);
    for (size_t k = 0; k < m; ++k) {
        const LGate& x = g[pb.gates[k]];
        if (x.kind != KIND_DIAG) {
            need[k] = loc[x.target];
        }
    }
    auto next_use = [&](int b, size_t from) -> size_t {
        for (size_t k = from; k < m; ++k) {
            if (need[k] == b) {
                return k;
            }
        }
        return SIZE_MAX;
    };
    // register set for a phase starting at `from`: the RB needed bits used
    // soonest, then (to keep the load/store layout coalesced) bits >= L.
    auto choose = [&](size_t from, const std::vector<int>& keep) -> std::vector<int> {
        std::vector<int> regs;
        for (size_t k = from; k < m && static_cast<int>(regs.size()) < RB; ++k) {
            if (need[k] >= 0 && std::find(regs.begin(), regs.end(), need[k]) == regs.end()) {
                regs.push_back(need[k]);
            }
        }
        for (int b : keep) {
            if (static_cast<int>(regs.size()) >= RB) break;
            if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
        }
        for (int b = K - 1; b >= L && static_cast<int>(regs.size()) < RB; --b) {
            if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
        }
        for (int b = K - 1; b >= 0 && static_cast<int>(regs.size()) < RB; --b) {
            if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
        }
        std::sort(regs.begin(), regs.end());
        return regs;
    };
    auto has_low = [&](const std::vector<int>& regs) {
        for (int r : regs) {
            if (r < L) return true;
        }
        return false;
    };
    auto io_regs = [&]() {
        std::vector<int> regs;
        for (int b = K - 1; b >= L && static_cast<int>(regs.size()) < RB; --b) regs.push_back(b);
        std::sort(regs.begin(), regs.end());
        return regs;
    };
    std::vector<std::pair<std::vector<int>, std::pair<size_t, size_t>>> ph;  // (regs, [begin, end))
    std::vector<int> cur = choose(0, {});
    if (has_low(cur)) {
        ph.push_back({io_regs(), {0, 0}});
    }
    size_t start = 0;
    for (size_t k = 0; k < m; ++k) {
        if (need[k] >= 0 && std::find(cur.begin(), cur.end(), need[k]) == cur.end()) {
            ph.push_back({cur, {start, k}});
            // keep the current bits whose next use is soonest as fillers
            std::vector<int> keep = cur;
            std::sort(keep.begin(), keep.end(), [&](int x, int y) { return next_use(x, k) < next_use(y, k); });
            cur = choose(k, keep);
            start = k;
        }
    }
    ph.push_back({cur, {start, m}});
    if (has_low(cur)) {
        ph.push_back({io_regs(), {m, m}});
    }
    // emit
    fb.phase_begin = static_cast<int32_t>(plan.phases.size());
    for (auto& [regs, range] : ph) {
        FPhase fp {};
        make_slots(regs, K, LANES, fp.slot_bit);
        fp.op_begin = static_cast<int32_t>(plan.ops.size() + range.first);
        fp.op_end = static_cast<int32_t>(plan.ops.size() + range.second);
        plan.phases.push_back(fp);
    }
    fb.phase_end = static_cast<int32_t>(plan.phases.size());
    plan.transposes += static_cast<int>(ph.size()) - 1;
    // ops (in block order, with the register slot of the target in its phase)
    size_t pi = 0;
    for (size_t k = 0; k < m; ++k) {
        while (!(k >= ph[pi].second.first && k < ph[pi].second.second)) {
            ++pi;
        }
        const LGate& x = g[pb.gates[k]];
        FOp<T> op {};
        op.kind = x.kind;
        op.flags = x.flags & 1;
        if (x.kind == KIND_ANTI && x.m[2] == 1.0 && x.m[3] == 0.0 && x.m[4] == 1.0 && x.m[5] == 0.0) {
            op.flags |= 2;  // pure swap (X / CX)
        }
        if (x.control >= 0) {
            if (loc[x.control] >= 0) {
                op.cmask_loc = 1u << loc[x.control];
            } else {
                op.cmask_glob = bit(x.control);
            }
        }
        if (x.kind == KIND_DIAG) {
            if (loc[x.target] >= 0) {
                op.tslot = loc[x.target];
            } else {
                op.tslot = -1;
                op.tglob = bit(x.target);
            }
        } else {
            const auto& regs = ph[pi].first;
            const auto it = std::find(regs.begin(), regs.end(), loc[x.target]);
            op.tslot = static_cast<int32_t>(it - regs.begin());  // regs are slots 0..RB-1 in order
        }
        for (int e = 0; e < 8; ++e) {
            op.m[e] = static_cast<T>(x.m[e]);
        }
        plan.ops.push_back(op);
    }
    plan.blocks.push_back(fb);
}

template <typename T>
int32_t run_fused(State& s, const std::vector<LGate>& gates)
{
    using C = typename CxT<T>::type;
    constexpr int RB = Cfg<T>::RB;
    constexpr int L = Cfg<T>::L;
    const int n = s.n_bits;
    const int K = std::min(n, RB + Cfg<T>::TBMAX);
    if (n < RB + 5 || gates.empty()) {
        for (const auto& g : gates) {
            if (const int32_t rc = launch_gate_sweep(s, g); rc != KT_OK) {
                return rc;
            }
        }
        return KT_OK;
    }
    const auto blocks = form_blocks(gates, n, K, L);
    Plan<T> plan;
    for (const auto& b : blocks) {
        plan_block<T>(b, gates, n, plan);
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
    KT_CUDA(cudaMemcpyAsync(dev, host.data(), need, cudaMemcpyHostToDevice, s.stream));
    const auto* d_blk = reinterpret_cast<const FBlock*>(dev);
    const auto* d_ph = reinterpret_cast<const FPhase*>(dev + off_p);
    const auto* d_ops = reinterpret_cast<const FOp<T>*>(dev + off_o);
    const int threads = 1 << (K - RB);
    const size_t smem = (size_t {1} << K) * sizeof(C);
    static bool attr_set = false;
    if (!attr_set) {
        KT_CUDA(cudaFuncSetAttribute(k_fused<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        attr_set = true;
    }
    const uint64_t n_tiles = uint64_t {1} << (n - K);
    const uint64_t grid = std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sm_count()) * 2);
    const double pass_bytes = 2.0 * static_cast<double>(sizeof(C)) * static_cast<double>(s.n_amps());
    for (size_t b = 0; b < plan.blocks.size(); ++b) {
        k_fused<T><<<static_cast<unsigned>(grid), threads, smem, s.stream>>>(static_cast<C*>(s.amps), d_blk + b, d_ph,
                                                                            d_ops, n_tiles);
        KT_CHECK_LAUNCH("k_fused");
        s.last_launches += 1;
        s.last_alg_bytes += pass_bytes;
    }
    // (the pageable host copy is staged by the time cudaMemcpyAsync returns,
    // so `host` may go out of scope while the kernels run)
    return KT_OK;
}

}  // namespace

int32_t apply_fused(State& s, const std::vector<LGate>& gates)
{
    return s.dtype == KT_C128 ? run_fused<double>(s, gates) : run_fused<float>(s, gates);
}

}  // namespace kt
