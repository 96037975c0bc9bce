// kt_fused.cuh — fused gate blocks: the host planner over the device side in
// kt_fused_dev.cuh (op records, layouts, register-level gate bodies, the
// per-tile bodies of the forward and adjoint kernels).  Shared by the single-state kernels (kt_fused.cu) and the
// batch engine (kt_batch.cu); everything here has internal linkage.
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
#pragma once

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "kt_fused_dev.cuh"
#include "kt_internal.cuh"

namespace kt
{

namespace
{

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
// One block from the pending gates: every gate that can move ahead of the
// gates not taken (no shared qubit with them) and whose non-diagonal target
// fits the tile.  `fixed` (0: grow the tile as gates arrive) pins the tile's
// qubit set up front.  Gates with mark[idx] == skip are treated as gone (taken
// by a block planned before this one); the scan stops once every qubit is
// blocked.  Returns the number of gates taken; `take` (if not null) gets them.
size_t scan_block(const std::vector<LGate>& g, const std::vector<int>& pend, const std::vector<uint32_t>& mark,
                  uint32_t skip, int n, int K, int L, size_t max_ops, uint64_t fixed, uint64_t* Q_out,
                  std::vector<int>* take, const std::vector<uint32_t>* mark2 = nullptr, uint32_t skip2 = 0)
{
    const uint64_t all = (n >= 64) ? ~uint64_t {0} : (bit(n) - 1);
    uint64_t Q = fixed != 0 ? fixed : (bit(L) - 1);
    uint64_t blocked = 0;
    size_t taken = 0;
    if (take != nullptr) {
        take->clear();
    }
    for (const int idx : pend) {
        if (skip != 0 && mark[static_cast<size_t>(idx)] == skip) {
            continue;
        }
        if (mark2 != nullptr && skip2 != 0 && (*mark2)[static_cast<size_t>(idx)] == skip2) {
            continue;
        }
        const LGate& x = g[idx];
        const uint64_t touch = bit(x.target) | (x.control >= 0 ? bit(x.control) : 0);
        if ((touch & blocked) != 0 || taken >= max_ops) {
            blocked |= touch;
        } else {
            const uint64_t need = (x.kind == KIND_DIAG) ? 0 : bit(x.target);
            const bool fits = fixed != 0 ? ((need & ~Q) == 0) : (__builtin_popcountll(Q | need) <= K);
            if (fits) {
                Q |= need;
                ++taken;
                if (take != nullptr) {
                    take->push_back(idx);
                }
            } else {
                blocked |= touch;
            }
        }
        if (blocked == all) {
            break;
        }
    }
    if (Q_out != nullptr) {
        *Q_out = Q;
    }
    return taken;
}

// The tile qubits a lookahead prefers: the L lowest, then the qubits that the
// first `window` pending non-diagonal gates (not marked `skip`) target most
// often (earliest first among equals).
uint64_t lookahead_tile(const std::vector<LGate>& g, const std::vector<int>& pend, const std::vector<uint32_t>& mark,
                        uint32_t skip, int n, int K, int L, size_t window, const std::vector<uint32_t>* mark2 = nullptr,
                        uint32_t skip2 = 0)
{
    int count[64] = {};
    size_t first[64];
    for (int q = 0; q < 64; ++q) {
        first[q] = SIZE_MAX;
    }
    size_t seen = 0;
    for (const int idx : pend) {
        if (seen >= window) {
            break;
        }
        if (skip != 0 && mark[static_cast<size_t>(idx)] == skip) {
            continue;
        }
        if (mark2 != nullptr && skip2 != 0 && (*mark2)[static_cast<size_t>(idx)] == skip2) {
            continue;
        }
        const LGate& x = g[idx];
        if (x.kind != KIND_DIAG) {
            ++count[x.target];
            first[x.target] = std::min(first[x.target], seen);
        }
        ++seen;
    }
    int order[64];
    int no = 0;
    for (int q = L; q < n; ++q) {
        order[no++] = q;
    }
    std::stable_sort(order, order + no, [&](int a, int b) {
        if (count[a] != count[b]) {
            return count[a] > count[b];
        }
        return first[a] < first[b];
    });
    uint64_t Q = bit(L) - 1;
    for (int i = 0; i < no && __builtin_popcountll(Q) < K; ++i) {
        Q |= bit(order[i]);
    }
    return Q;
}

// Candidate tiles for a block: 0 (the tile grows as gates arrive) and the
// lookahead tiles of several windows.
void tile_candidates(const std::vector<LGate>& g, const std::vector<int>& pend, const std::vector<uint32_t>& mark,
                     uint32_t skip, int n, int K, int L, std::vector<uint64_t>& c,
                     const std::vector<uint32_t>* mark2 = nullptr, uint32_t skip2 = 0)
{
    c.assign(1, 0);
    for (int w : {1, 2, 3, 4, 6, 8, 12, 16, 32, 64}) {
        const uint64_t q = lookahead_tile(g, pend, mark, skip, n, K, L, static_cast<size_t>(w) * static_cast<size_t>(K),
                                          mark2, skip2);
        if (std::find(c.begin(), c.end(), q) == c.end()) {
            c.push_back(q);
        }
    }
}

std::vector<PlanBlock> form_blocks(const std::vector<LGate>& g, int n, int K, int L, size_t max_ops)
{
    std::vector<PlanBlock> out;
    std::vector<int> pend(g.size());
    std::iota(pend.begin(), pend.end(), 0);
    const bool look = tuning().plan_lookahead != 0 && K < n && n <= 64;
    std::vector<uint32_t> mark(g.size(), 0);
    std::vector<uint32_t> mark2(g.size(), 0);
    uint32_t stamp = 0;
    uint32_t stamp2 = 0;
    // three blocks deep on large states (a pass there costs milliseconds, a
    // deeper plan ~0.1 s once, the plan cache keeps it), two otherwise
    const int depth = (tuning().plan_lookahead >= 2 || n >= tuning().plan_deep_qubits) ? 3 : 2;
    std::vector<int> take, take2, best_take;
    std::vector<uint64_t> cand1, cand2, cand3;
    while (!pend.empty()) {
        uint64_t Q = 0;
        uint64_t bestQ = 0;
        scan_block(g, pend, mark, 0, n, K, L, max_ops, 0, &bestQ, &best_take);
        if (look) {
            // plan_lookahead: of the candidate tiles, the one whose block and the
            // best next block together take the most gates (ties: the greedy one)
            size_t best_score = 0;
            bool first = true;
            tile_candidates(g, pend, mark, 0, n, K, L, cand1);
            for (const uint64_t c1 : cand1) {
                scan_block(g, pend, mark, 0, n, K, L, max_ops, c1, &Q, &take);
                ++stamp;
                for (const int idx : take) {
                    mark[static_cast<size_t>(idx)] = stamp;
                }
                size_t next = 0;
                if (take.size() < pend.size()) {
                    tile_candidates(g, pend, mark, stamp, n, K, L, cand2);
                    for (const uint64_t c2 : cand2) {
                        if (depth < 3) {
                            next = std::max(next, scan_block(g, pend, mark, stamp, n, K, L, max_ops, c2, nullptr, nullptr));
                            continue;
                        }
                        // three blocks deep: this second block, then the best third
                        const size_t t2 = scan_block(g, pend, mark, stamp, n, K, L, max_ops, c2, nullptr, &take2);
                        ++stamp2;
                        for (const int idx : take2) {
                            mark2[static_cast<size_t>(idx)] = stamp2;
                        }
                        size_t third = 0;
                        tile_candidates(g, pend, mark, stamp, n, K, L, cand3, &mark2, stamp2);
                        for (const uint64_t c3 : cand3) {
                            third = std::max(third, scan_block(g, pend, mark, stamp, n, K, L, max_ops, c3, nullptr,
                                                               nullptr, &mark2, stamp2));
                        }
                        next = std::max(next, t2 + third);
                    }
                }
                const size_t score = take.size() + next;
                if (first || score > best_score) {
                    first = false;
                    best_score = score;
                    best_take.swap(take);
                    bestQ = Q;
                }
            }
        }
        // the chosen block's gates leave the pending list
        ++stamp;
        for (const int idx : best_take) {
            mark[static_cast<size_t>(idx)] = stamp;
        }
        std::vector<int> rest;
        rest.reserve(pend.size() - best_take.size());
        for (const int idx : pend) {
            if (mark[static_cast<size_t>(idx)] != stamp) {
                rest.push_back(idx);
            }
        }
        // fill the tile up to K qubits with the lowest free qubits (longer contiguous runs)
        for (int q = 0; q < n && __builtin_popcountll(bestQ) < K; ++q) {
            bestQ |= bit(q);
        }
        PlanBlock b;
        b.K = K;
        for (int q = 0; q < n; ++q) {
            if (bestQ & bit(q)) {
                b.qubits.push_back(q);
            }
        }
        b.gates = best_take;
        out.push_back(std::move(b));
        pend.swap(rest);
    }
    return out;
}

// Slot order of a layout: register bits, then the lane bits (distinct
// residues mod G so a quarter/half warp hits distinct shared-memory banks;
// the L lowest tile bits when none of them is a register bit, which also
// makes global accesses coalesced), then the remaining thread bits.
void make_slots(const std::vector<int>& regs, int K, int G, int8_t* slot_bit)
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
    bool low_free = true;
    for (int b = 0; b < G; ++b) {
        low_free = low_free && !is_reg[b];
    }
    if (low_free) {
        for (int b = 0; b < G; ++b) {
            lanes.push_back(b);
        }
    } else {
        std::vector<bool> res_used(G, false);
        for (int b = 0; b < K && static_cast<int>(lanes.size()) < G; ++b) {
            if (!is_reg[b] && !res_used[b % G]) {
                res_used[b % G] = true;
                lanes.push_back(b);
            }
        }
        for (int b = 0; b < K && static_cast<int>(lanes.size()) < G; ++b) {
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

template <typename T, typename OPT = FOp<T>>
struct Plan
{
    std::vector<FBlock> blocks;
    std::vector<FPhase> phases;
    std::vector<OPT> ops;
    std::vector<int32_t> op_gate;  // the gate (index into the planned gate list) each op runs
    std::vector<int32_t> run_order;  // every planned gate in the order it takes effect (folded ones included)
    int transposes {0};
    int folded {0};   // X / CX gates folded into transposes
};

// per-gate extras of the adjoint sweep: the gradient row (-1: none) and the generator
struct AdjExtra
{
    int32_t row;
    int32_t gen;
};

// Is this lowered gate X or CX (the matrix [[0, 1], [1, 0]] exactly)?
inline bool is_pure_x(const LGate& x)
{
    return x.kind == KIND_ANTI && x.m[2] == 1.0 && x.m[3] == 0.0 && x.m[4] == 1.0 && x.m[5] == 0.0;
}

template <typename T, typename CFG = Cfg<T>, typename OPT = FOp<T>>
void plan_block(const PlanBlock& pb, const std::vector<LGate>& g, int n, Plan<T, OPT>& plan,
                const AdjExtra* extra = nullptr)
{
    constexpr int RB = CFG::RB;
    constexpr int L = CFG::L;
    constexpr int G = CFG::G;
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
    // X and CX with every qubit in the tile are index permutations; with
    // folding on they become part of the next transpose instead of ops.
    // The tile bit every other non-diagonal gate needs as a register bit.
    const size_t m = pb.gates.size();
    const bool folding = tuning().fold_permutations != 0;
    std::vector<char> fold(m, 0);
    std::vector<int> need(m, -1);
    for (size_t k = 0; k < m; ++k) {
        const LGate& x = g[pb.gates[k]];
        if (folding && is_pure_x(x) && loc[x.target] >= 0 && (x.control < 0 || loc[x.control] >= 0)) {
            fold[k] = 1;
        } else if (x.kind != KIND_DIAG) {
            need[k] = loc[x.target];
        }
    }
    // gates already placed in a phase (list scheduling may run them out of order)
    std::vector<char> done(m, 0);
    // every qubit of each gate (dependencies) and its tile bits (pending permutations)
    std::vector<uint64_t> qmask(m), tmask(m);
    for (size_t k = 0; k < m; ++k) {
        const LGate& x = g[pb.gates[k]];
        qmask[k] = bit(x.target) | (x.control >= 0 ? bit(x.control) : 0);
        tmask[k] = (loc[x.target] >= 0 ? bit(loc[x.target]) : 0) |
                   (x.control >= 0 && loc[x.control] >= 0 ? bit(loc[x.control]) : 0);
    }
    auto next_use = [&](int b, size_t from) -> size_t {
        for (size_t k = from; k < m; ++k) {
            if (!done[k] && need[k] == b) {
                return k;
            }
        }
        return SIZE_MAX;
    };
    // register set for a phase starting at `from`: the RB needed bits used
    // soonest, then current bits by next use, then bits >= L (keeps the
    // load/store layout coalesced)
    auto choose = [&](size_t from, const std::vector<int>& keep) -> std::vector<int> {
        std::vector<int> regs;
        for (size_t k = from; k < m && static_cast<int>(regs.size()) < RB; ++k) {
            if (!done[k] && need[k] >= 0 && std::find(regs.begin(), regs.end(), need[k]) == regs.end()) {
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
    // The gates a phase with register set R would take from the unplaced ones
    // under list scheduling, in one pass: a gate is taken when no earlier
    // untaken gate shares a qubit with it and it fits (a later gate never
    // makes an earlier one ready, and pending permutations only grow).
    auto phase_gain = [&](const std::vector<int>& R) -> int {
        uint64_t blocked = 0;
        uint64_t pend = 0;
        int taken = 0;
        for (size_t i = 0; i < m; ++i) {
            if (done[i]) {
                continue;
            }
            bool ok = (blocked & qmask[i]) == 0;
            if (ok && fold[i]) {
                pend |= tmask[i];
            } else if (ok) {
                ok = (need[i] < 0 || std::find(R.begin(), R.end(), need[i]) != R.end()) && (tmask[i] & pend) == 0;
            }
            if (ok) {
                ++taken;
            } else {
                blocked |= qmask[i];
            }
        }
        return taken;
    };
    // register set for a phase that starts with gate k: need[k], then one bit
    // at a time the one that lets the phase take the most gates (ties: the
    // order choose() would use)
    auto choose_gain = [&](size_t k, const std::vector<int>& keep) -> std::vector<int> {
        std::vector<int> pref;
        for (size_t i = 0; i < m; ++i) {
            if (!done[i] && need[i] >= 0 && std::find(pref.begin(), pref.end(), need[i]) == pref.end()) {
                pref.push_back(need[i]);
            }
        }
        for (int b : keep) {
            if (std::find(pref.begin(), pref.end(), b) == pref.end()) pref.push_back(b);
        }
        for (int b = K - 1; b >= 0; --b) {
            if (std::find(pref.begin(), pref.end(), b) == pref.end()) pref.push_back(b);
        }
        std::vector<int> R;
        if (need[k] >= 0) {
            R.push_back(need[k]);
        }
        while (static_cast<int>(R.size()) < RB) {
            int best = -1;
            int best_gain = -1;
            for (int b : pref) {
                if (std::find(R.begin(), R.end(), b) != R.end()) {
                    continue;
                }
                R.push_back(b);
                const int gn = phase_gain(R);
                R.pop_back();
                if (gn > best_gain) {
                    best_gain = gn;
                    best = b;
                }
            }
            R.push_back(best);
        }
        std::sort(R.begin(), R.end());
        return R;
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
    struct PhaseSpec
    {
        std::vector<int> regs;
        std::vector<size_t> ops;    // gate positions run as ops in this phase
        std::vector<size_t> folds;  // X / CX applied when this phase is stored
    };
    std::vector<PhaseSpec> ph;
    std::vector<int> cur = choose(0, {});
    if (tuning().plan_schedule >= 3 && has_low(cur)) {
        // a first register set of bits >= L only (built bit by bit by the
        // gates it takes): the tile loads straight into it, with no transpose
        std::vector<int> hi;
        while (static_cast<int>(hi.size()) < RB) {
            int best = -1;
            int best_gain = -1;
            for (int b = K - 1; b >= L; --b) {
                if (std::find(hi.begin(), hi.end(), b) != hi.end()) {
                    continue;
                }
                hi.push_back(b);
                const int gn = phase_gain(hi);
                hi.pop_back();
                if (gn > best_gain) {
                    best_gain = gn;
                    best = b;
                }
            }
            if (best < 0) {
                break;
            }
            hi.push_back(best);
        }
        std::sort(hi.begin(), hi.end());
        if (static_cast<int>(hi.size()) == RB && phase_gain(hi) > 0) {
            cur = hi;
        }
    }
    if (has_low(cur)) {
        ph.push_back({io_regs(), {}, {}});
    }
    PhaseSpec open {cur, {}, {}};
    uint64_t pending = 0;  // tile bits of the folded gates waiting in `open`
    // Pending permutations wait for the next transpose.  A gate that touches
    // their qubits before then runs them as ordinary ops first when their
    // targets are register bits (they were only moved past gates on other
    // qubits, which commute with them); otherwise that gate starts a new
    // phase, as a gate on a missing register bit does.  So folding never adds
    // a transpose.
    auto targets_in_regs = [&](const PhaseSpec& sp) {
        for (size_t f : sp.folds) {
            if (std::find(cur.begin(), cur.end(), loc[g[pb.gates[f]].target]) == cur.end()) {
                return false;
            }
        }
        return true;
    };
    // place gate k in the open phase, or start a new phase for it
    auto place = [&](size_t k) {
        const uint64_t qm = tmask[k];
        done[k] = 1;
        if (fold[k]) {
            open.folds.push_back(k);
            pending |= qm;
            return;
        }
        const bool miss = need[k] >= 0 && std::find(cur.begin(), cur.end(), need[k]) == cur.end();
        if (!miss && (qm & pending) != 0 && targets_in_regs(open)) {
            open.ops.insert(open.ops.end(), open.folds.begin(), open.folds.end());
            open.folds.clear();
            pending = 0;
        }
        if (miss || (qm & pending) != 0) {
            // a transpose: it applies the pending permutations; the next
            // register set is chosen by next use
            ph.push_back(open);
            std::vector<int> keep = cur;
            done[k] = 0;
            std::sort(keep.begin(), keep.end(), [&](int a, int b2) { return next_use(a, 0) < next_use(b2, 0); });
            cur = tuning().plan_schedule >= 2 ? choose_gain(k, keep) : choose(0, keep);
            done[k] = 1;
            open = PhaseSpec {cur, {}, {}};
            pending = 0;
        }
        open.ops.push_back(k);
    };
    if (tuning().plan_schedule == 0) {
        for (size_t k = 0; k < m; ++k) {
            place(k);
        }
    } else {
        // List scheduling: a gate is ready once every earlier gate sharing a
        // qubit with it is placed (gates on disjoint qubits commute, so any
        // such order gives the same state).  The earliest ready gate that fits
        // the open phase goes next: a folded permutation always fits (the
        // store composes them in order); another gate fits when its target is
        // a register bit (or it is diagonal) and no pending permutation is on
        // its qubits.  Only when no ready gate fits does the earliest ready
        // one go, through place(), which may start a phase.  That gate is the
        // earliest unplaced one, so the next register set serves it first.
        size_t placed = 0;
        while (placed < m) {
            size_t pick = SIZE_MAX;
            size_t first_ready = SIZE_MAX;
            uint64_t blocked = 0;  // qubits of unplaced gates seen so far (in gate order)
            for (size_t k = 0; k < m; ++k) {
                if (done[k]) {
                    continue;
                }
                const bool rdy = (blocked & qmask[k]) == 0;
                blocked |= qmask[k];
                if (!rdy) {
                    continue;
                }
                if (first_ready == SIZE_MAX) {
                    first_ready = k;
                }
                const uint64_t qm = tmask[k];
                const bool fits = fold[k] || ((need[k] < 0 || std::find(cur.begin(), cur.end(), need[k]) != cur.end()) &&
                                              (qm & pending) == 0);
                if (fits) {
                    pick = k;
                    break;
                }
            }
            place(pick != SIZE_MAX ? pick : first_ready);
            ++placed;
        }
    }
    if (!open.folds.empty() && !has_low(cur) && targets_in_regs(open)) {
        open.ops.insert(open.ops.end(), open.folds.begin(), open.folds.end());
        open.folds.clear();
    }
    ph.push_back(open);
    if (!open.folds.empty() || has_low(cur)) {
        // one more transpose: it applies the last permutations and leaves a
        // coalesced layout for the store
        ph.push_back({io_regs(), {}, {}});
    }
    // phases
    const int TB = K - RB;
    const size_t op_base = plan.ops.size();
    fb.phase_begin = static_cast<int32_t>(plan.phases.size());
    std::vector<std::vector<int8_t>> slots;
    size_t emitted = 0;
    for (auto& spec : ph) {
        int8_t sb[KMAX] = {};
        make_slots(spec.regs, K, G, sb);
        slots.emplace_back(sb, sb + K);
        FPhase fp {};
        // store side: the folded permutation M (columns M e_k) and offset c
        uint32_t col[KMAX];
        for (int k = 0; k < K; ++k) {
            col[k] = 1u << k;
        }
        uint32_t xc = 0;
        for (size_t f : spec.folds) {
            const LGate& x = g[pb.gates[f]];
            const int lt = loc[x.target];
            if (x.control >= 0) {
                const int lc = loc[x.control];
                for (int k = 0; k < K; ++k) {
                    col[k] ^= ((col[k] >> lc) & 1u) << lt;
                }
                xc ^= ((xc >> lc) & 1u) << lt;
            } else {
                xc ^= 1u << lt;
            }
        }
        for (int s2 = 0; s2 < RB; ++s2) {
            fp.rstride[s2] = bit(pb.qubits[sb[s2]]);
            fp.rsw[s2] = swz(1u << sb[s2], G);
            fp.rsw_out[s2] = swz(col[sb[s2]], G);
        }
        for (int j = 0; j < TB; ++j) {
            fp.tstride[j] = bit(pb.qubits[sb[RB + j]]);
            fp.tsw[j] = swz(1u << sb[RB + j], G);
            fp.tsw_out[j] = swz(col[sb[RB + j]], G);
        }
        fp.xor_out = swz(xc, G);
        fp.op_begin = static_cast<int32_t>(op_base + emitted);
        emitted += spec.ops.size();
        fp.op_end = static_cast<int32_t>(op_base + emitted);
        plan.phases.push_back(fp);
        plan.folded += static_cast<int>(spec.folds.size());
    }
    fb.phase_end = static_cast<int32_t>(plan.phases.size());
    plan.transposes += static_cast<int>(ph.size()) - 1;
    // a phase's ops run first, its folded permutations at its store
    for (const auto& spec : ph) {
        for (size_t k : spec.ops) {
            plan.run_order.push_back(pb.gates[k]);
        }
        for (size_t f : spec.folds) {
            plan.run_order.push_back(pb.gates[f]);
        }
    }
    // ops, resolved against the layout of their phase
    for (size_t pi = 0; pi < ph.size(); ++pi) {
        const auto& sb = slots[pi];
        auto reg_slot = [&](int tilebit) -> int {
            for (int s2 = 0; s2 < RB; ++s2) {
                if (sb[s2] == tilebit) return s2;
            }
            return -1;
        };
        auto thread_bit = [&](int tilebit) -> int {
            for (int j = 0; j < TB; ++j) {
                if (sb[RB + j] == tilebit) return j;
            }
            return -1;
        };
        for (size_t k : ph[pi].ops) {
            const LGate& x = g[pb.gates[k]];
            OPT op {};
            op.tslot = NO_SLOT;
            op.cslot = NO_SLOT;
            if (x.control >= 0) {
                const int lc = loc[x.control];
                if (lc < 0) {
                    op.cglob = bit(x.control);
                } else if (const int s2 = reg_slot(lc); s2 >= 0) {
                    op.cslot = static_cast<uint8_t>(s2);
                } else {
                    op.cthr = 1u << thread_bit(lc);
                }
            }
            const bool real = x.m[1] == 0.0 && x.m[3] == 0.0 && x.m[5] == 0.0 && x.m[7] == 0.0;
            if (x.kind == KIND_DIAG) {
                op.kind = (x.flags & 1) ? OP_DIAG1 : OP_DIAG;
                const int lt = loc[x.target];
                if (lt < 0) {
                    op.tglob = bit(x.target);
                } else if (const int s2 = reg_slot(lt); s2 >= 0) {
                    op.tslot = static_cast<uint8_t>(s2);
                } else {
                    op.tthr = 1u << thread_bit(lt);
                }
            } else {
                op.tslot = static_cast<uint8_t>(reg_slot(loc[x.target]));
                if (x.kind == KIND_ANTI) {
                    op.kind = is_pure_x(x) ? OP_SWAP : OP_ANTI;
                } else if (real) {
                    op.kind = OP_GENR;
                } else if (x.m[1] == 0.0 && x.m[7] == 0.0 && x.m[0] == x.m[6] && x.m[2] == 0.0 && x.m[4] == 0.0 &&
                           x.m[3] == x.m[5]) {
                    op.kind = OP_RXL;
                } else {
                    op.kind = OP_GEN;
                }
            }
            for (int e = 0; e < 8; ++e) {
                op.m[e] = static_cast<T>(x.m[e]);
            }
            if constexpr (OPT::HAS_D) {
                const AdjExtra& ex = extra[pb.gates[k]];
                op.row = ex.row;
                op.gen = static_cast<uint8_t>(ex.gen < 0 ? 0 : ex.gen);
            }
            plan.ops.push_back(op);
            plan.op_gate.push_back(pb.gates[k]);
        }
    }
    fb.op_begin = static_cast<int32_t>(op_base);
    fb.op_end = static_cast<int32_t>(plan.ops.size());
    plan.blocks.push_back(fb);
}

}  // namespace

}  // namespace kt
