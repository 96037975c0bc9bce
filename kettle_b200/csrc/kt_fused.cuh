// kt_fused.cuh — fused gate blocks: op records, layouts, register-level gate
// bodies, the per-tile bodies of the forward and adjoint kernels, and the
// host planner.  Shared by the single-state kernels (kt_fused.cu) and the
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

#include "kt_complex.cuh"
#include "kt_internal.cuh"

namespace kt
{

namespace
{

constexpr int KMAX = 14;
constexpr int RBMAX = 5;
constexpr int TBMAX = 9;   // thread bits of a tile: up to 512 threads (the largest forward tiles)
constexpr int TB256 = 8;   // thread bits of the 256-thread kernels (adjoint, batch)
constexpr int MAX_OPS_PER_BLOCK = 256;
constexpr int MAX_PHASES_PER_BLOCK = 64;

enum OpKind : uint8_t
{
    OP_GEN = 0,    // general complex 2x2
    OP_GENR = 1,   // real 2x2 (H, RY, real U)
    OP_ANTI = 2,   // [[0, m01], [m10, 0]]
    OP_SWAP = 3,   // X / CX
    OP_DIAG = 4,   // diag(m00, m11)
    OP_DIAG1 = 5,  // diag(1, m11)
    OP_RXL = 6,    // [[c, i s], [i s, c]] with c, s real (RX, CRX): m[0] = c, m[3] = s
};

constexpr uint8_t NO_SLOT = 0xFF;

template <typename T>
struct FOp
{
    uint8_t kind;
    uint8_t tslot;    // register slot of the target (NO_SLOT: the target is not a register bit)
    uint8_t cslot;    // register slot of the control (NO_SLOT: none, or not a register bit)
    uint8_t pad0;
    uint32_t pad2;
    uint32_t pad3;
    uint32_t cthr;    // control as thread-index bits (0: none)
    uint32_t tthr;    // diagonal target as thread-index bits (0: none)
    uint32_t pad1;
    uint64_t cglob;   // control outside the tile (0: none)
    uint64_t tglob;   // diagonal target outside the tile (0: none)
    T m[8];
    static constexpr bool HAS_D = false;
};

// an op of the adjoint sweep: m = U^dagger; row = gradient row (-1: none);
// gen = the generator of a parameterised rotation (GEN_X/Y/Z/P)
template <typename T>
struct FOpA
{
    uint8_t kind;
    uint8_t tslot;
    uint8_t cslot;
    uint8_t gen;
    int32_t row;
    uint32_t pad3;
    uint32_t cthr;
    uint32_t tthr;
    uint32_t pad1;
    uint64_t cglob;
    uint64_t tglob;
    T m[8];
    static constexpr bool HAS_D = true;
};

// A layout phase.  rsw/tsw address a register or thread bit's amplitude when
// the phase is loaded from shared memory; rsw_out/tsw_out/xor_out when it is
// stored at the next transpose.  They differ when X / CX gates were folded
// into that transpose: an index permutation b -> M b + c over GF(2), stored
// as the swizzled images M e_k (every term) and c (xor_out).
struct FPhase
{
    uint64_t rstride[RBMAX];   // global stride of each register slot
    uint64_t tstride[TBMAX];   // global stride of each thread-index bit
    uint32_t rsw[RBMAX];       // swizzled shared-memory term of each register slot
    uint32_t tsw[TBMAX];       // swizzled shared-memory term of each thread-index bit
    uint32_t rsw_out[RBMAX];
    uint32_t tsw_out[TBMAX];
    uint32_t xor_out;
    int32_t op_begin;
    int32_t op_end;
};

struct FBlock
{
    int32_t K;
    int32_t nfree;
    int32_t phase_begin;
    int32_t phase_end;
    int32_t op_begin;
    int32_t op_end;
    int32_t qubit[KMAX];    // tile bit -> qubit
    int32_t freebit[64];    // qubits outside the tile, ascending
};

// tile configuration per amplitude type
template <typename T>
struct Cfg;
template <>
struct Cfg<double>
{
    static constexpr int RB = 4;     // 16 amplitudes per thread
    static constexpr int L = 3;      // 8 x 16 B = 128 B runs
    static constexpr int G = 3;      // swizzle group (16-byte elements: 8 per 128-byte bank row)
};
template <>
struct Cfg<float>
{
    static constexpr int RB = 5;     // 32 amplitudes per thread
    static constexpr int L = 4;      // 16 x 8 B = 128 B runs
    static constexpr int G = 4;      // 8-byte elements: 16 per bank row
};

// XOR swizzle: the low G bits are XORed with a fold of the higher bits.  It is
// linear over GF(2), so swz(a ^ b) = swz(a) ^ swz(b).
__host__ __device__ inline uint32_t swz(uint32_t l, int G)
{
    uint32_t f = 0;
    for (int s = G; s < 32; s += G) {
        f ^= l >> s;
    }
    return l ^ (f & ((1u << G) - 1));
}

template <int RB, typename U>
__device__ __forceinline__ U xor_terms(int i, const U (&terms)[RBMAX])
{
    U a = 0;
#pragma unroll
    for (int s = 0; s < RB; ++s) {
        if (i & (1 << s)) {
            a ^= terms[s];
        }
    }
    return a;
}

// --- register-level gate bodies -------------------------------------------------
// S: register slot of the target (a template argument, so the register pairs
// are fixed at compile time); CS: -1 without a register control, CS_RT with a
// control on register slot `crt`, read at run time (one predicated body per
// target slot instead of one per target and control slot: the bodies are the
// kernel's code size and register pressure).
constexpr int CS_RT = -2;

template <int S, int CS>
__device__ __forceinline__ bool lower_of_pair(int i, int crt)
{
    if (i & (1 << S)) {
        return false;
    }
    if constexpr (CS == -1) {
        return true;
    } else {
        return ((i >> crt) & 1) != 0;
    }
}

template <int CS>
__device__ __forceinline__ bool ctrl_on(int i, int crt)
{
    if constexpr (CS == -1) {
        return true;
    } else {
        return ((i >> crt) & 1) != 0;
    }
}

template <typename T, int RB>
struct GenF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    C m00, m01, m10, m11;
    int crt = -1;
    template <int S, int CS>
    __device__ __forceinline__ void run()
    {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (lower_of_pair<S, CS>(i, crt)) {
                const int j = i | (1 << S);
                const C a = v[i];
                const C b = v[j];
                v[i] = cfma(m01, b, cmul(m00, a));
                v[j] = cfma(m11, b, cmul(m10, a));
            }
        }
    }
};

template <typename T, int RB>
struct GenRF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    T m00, m01, m10, m11;
    int crt = -1;
    template <int S, int CS>
    __device__ __forceinline__ void run()
    {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (lower_of_pair<S, CS>(i, crt)) {
                const int j = i | (1 << S);
                const C a = v[i];
                const C b = v[j];
                C x, y;
                x.x = fma(m01, b.x, m00 * a.x);
                x.y = fma(m01, b.y, m00 * a.y);
                y.x = fma(m11, b.x, m10 * a.x);
                y.y = fma(m11, b.y, m10 * a.y);
                v[i] = x;
                v[j] = y;
            }
        }
    }
};

// [[c, i s], [i s, c]]: 8 FP64 operations per pair instead of the general 16
template <typename T, int RB>
struct RxF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    T c, s;
    int crt = -1;
    template <int S, int CS>
    __device__ __forceinline__ void run()
    {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (lower_of_pair<S, CS>(i, crt)) {
                const int j = i | (1 << S);
                const C a = v[i];
                const C b = v[j];
                C x, y;
                x.x = fma(-s, b.y, c * a.x);
                x.y = fma(s, b.x, c * a.y);
                y.x = fma(-s, a.y, c * b.x);
                y.y = fma(s, a.x, c * b.y);
                v[i] = x;
                v[j] = y;
            }
        }
    }
};

template <typename T, int RB, bool PURE>
struct AntiF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    C m01, m10;
    int crt = -1;
    template <int S, int CS>
    __device__ __forceinline__ void run()
    {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (lower_of_pair<S, CS>(i, crt)) {
                const int j = i | (1 << S);
                const C a = v[i];
                const C b = v[j];
                if (PURE) {
                    v[i] = b;
                    v[j] = a;
                } else {
                    v[i] = cmul(m01, b);
                    v[j] = cmul(m10, a);
                }
            }
        }
    }
};

// diagonal gate whose target is register slot S
template <typename T, int RB, bool ONE>
struct DiagRegF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    C d0, d1;
    int crt = -1;
    template <int S, int CS>
    __device__ __forceinline__ void run()
    {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (ctrl_on<CS>(i, crt)) {
                if (i & (1 << S)) {
                    v[i] = cmul(d1, v[i]);
                } else if (!ONE) {
                    v[i] = cmul(d0, v[i]);
                }
            }
        }
    }
};

// one factor for every register of this thread (target is a thread bit or outside the tile)
template <typename T, int RB>
struct DiagAllF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    C d;
    int crt = -1;
    template <int S, int CS>
    __device__ __forceinline__ void run()
    {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (ctrl_on<CS>(i, crt)) {
                v[i] = cmul(d, v[i]);
            }
        }
    }
};

template <int RB, int S, typename F>
__device__ __forceinline__ void dispatch_c(int cs, F& f)
{
    if (cs < 0) {
        f.template run<S, -1>();
    } else {
        f.crt = cs;
        f.template run<S, CS_RT>();
    }
}

template <int RB, typename F>
__device__ __forceinline__ void dispatch_sc(int s, int cs, F& f)
{
    switch (s) {
        case 0: dispatch_c<RB, 0>(cs, f); break;
        case 1: dispatch_c<RB, 1>(cs, f); break;
        case 2: dispatch_c<RB, 2>(cs, f); break;
        case 3: dispatch_c<RB, 3>(cs, f); break;
        default: if constexpr (RB > 4) { dispatch_c<RB, (RB > 4 ? 4 : 0)>(cs, f); } break;
    }
}

template <typename T, int RB>
__device__ __forceinline__ void apply_op(typename CxT<T>::type (&v)[1 << RB], const FOp<T>& op, uint32_t t,
                                         uint64_t base)
{
    using C = typename CxT<T>::type;
    if ((base & op.cglob) != op.cglob) {
        return;  // control outside the tile is 0 for the whole tile
    }
    if ((t & op.cthr) != op.cthr) {
        return;  // control on a thread bit is 0 for this thread
    }
    const int kind = op.kind;
    const int ts = op.tslot;
    const int cs = (op.cslot == NO_SLOT) ? -1 : op.cslot;
    switch (kind) {
        case OP_GEN: {
            GenF<T, RB> f {v, make_cx<T>(op.m[0], op.m[1]), make_cx<T>(op.m[2], op.m[3]),
                           make_cx<T>(op.m[4], op.m[5]), make_cx<T>(op.m[6], op.m[7])};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        case OP_GENR: {
            GenRF<T, RB> f {v, op.m[0], op.m[2], op.m[4], op.m[6]};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        case OP_RXL: {
            RxF<T, RB> f {v, op.m[0], op.m[3]};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        case OP_ANTI: {
            AntiF<T, RB, false> f {v, make_cx<T>(op.m[2], op.m[3]), make_cx<T>(op.m[4], op.m[5])};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        case OP_SWAP: {
            // through the multiply path: a register-move body needs temporaries that spill
            AntiF<T, RB, false> f {v, make_cx<T>(1, 0), make_cx<T>(1, 0)};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        default:
            break;
    }
    // diagonal
    const C d1 = make_cx<T>(op.m[6], op.m[7]);
    const C d0 = make_cx<T>(op.m[0], op.m[1]);
    if (ts != NO_SLOT) {
        if (kind == OP_DIAG1) {
            DiagRegF<T, RB, true> f {v, d0, d1};
            dispatch_sc<RB>(ts, cs, f);
        } else {
            DiagRegF<T, RB, false> f {v, d0, d1};
            dispatch_sc<RB>(ts, cs, f);
        }
        return;
    }
    const bool b = ((t & op.tthr) != 0) || ((base & op.tglob) != 0);
    if (!b && kind == OP_DIAG1) {
        return;
    }
    DiagAllF<T, RB> f {v, b ? d1 : d0};
    dispatch_c<RB, 99>(cs, f);
}

template <typename T>
struct CfgA;
template <>
struct CfgA<double>
{
    static constexpr int RB = 3;  // 8 amplitudes of psi and 8 of lambda per thread
    static constexpr int L = 3;
    static constexpr int G = 3;
};
template <>
struct CfgA<float>
{
    static constexpr int RB = 4;
    static constexpr int L = 4;
    static constexpr int G = 4;
};

constexpr int ADJ_WARPS = 8;          // 256 threads
// ops (and so gradient rows) per adjoint block: two 2^11-amplitude tiles, 128
// op records and 128 x 8 row slots stay under 96 KB of shared memory, so two
// CTAs fit on an SM
constexpr int ADJ_MAX_OPS = 128;

// Gradient terms.  A parameterised gate is U = exp(-i theta G / 2) with G a
// Pauli (RX, RY, RZ and their controlled forms: G = X, Y, Z on the target,
// times the control projector) or P(theta) = diag(1, e^(i theta)).  With
// psi_g = U psi_(g-1) (the state before U^dagger is un-applied):
//   dU/dtheta psi_(g-1) = -(i/2) G psi_g   =>  Re <lambda| dU psi_(g-1)> = Im <lambda| G psi_g> / 2
//   dP/dtheta psi_(g-1) = i Pi_1 psi_g     =>  Re <lambda| dP psi_(g-1)> = -Im <lambda| Pi_1 psi_g>
// so the term is a sign pattern over conj(lambda) * psi, no matrix products
// (the rows are doubled when they are finalised).
__device__ __forceinline__ double im_cj(double2 a, double2 b)
{
    return a.x * b.y - a.y * b.x;  // Im(conj(a) b)
}

__device__ __forceinline__ double re_cj(double2 a, double2 b)
{
    return a.x * b.x + a.y * b.y;  // Re(conj(a) b)
}

// generator on register slot S (control register slot CS)
template <typename T, int RB, int GENK>
struct GradRegF
{
    using C = typename CxT<T>::type;
    const C (&l)[1 << RB];
    const C (&p)[1 << RB];
    double acc;
    int crt = -1;
    template <int S, int CS>
    __device__ __forceinline__ void run()
    {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (lower_of_pair<S, CS>(i, crt)) {
                const int j = i | (1 << S);
                const double2 l0 = to_d2(l[i]), l1 = to_d2(l[j]);
                const double2 p0 = to_d2(p[i]), p1 = to_d2(p[j]);
                if constexpr (GENK == GEN_X) {
                    acc += im_cj(l0, p1) + im_cj(l1, p0);
                } else if constexpr (GENK == GEN_Y) {
                    acc += re_cj(l1, p0) - re_cj(l0, p1);
                } else if constexpr (GENK == GEN_Z) {
                    acc += im_cj(l0, p0) - im_cj(l1, p1);
                } else {
                    acc -= im_cj(l1, p1);
                }
            }
        }
    }
};

// sum of Im(conj(lambda) psi) over this thread's registers with the control on
// (a diagonal generator whose target bit is fixed for the thread)
template <typename T, int RB>
struct GradAllF
{
    using C = typename CxT<T>::type;
    const C (&l)[1 << RB];
    const C (&p)[1 << RB];
    double acc;
    int crt = -1;
    template <int S, int CS>
    __device__ __forceinline__ void run()
    {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (ctrl_on<CS>(i, crt)) {
                acc += im_cj(to_d2(l[i]), to_d2(p[i]));
            }
        }
    }
};

// apply the op's U^dagger to one register array (the forward gate bodies)
template <typename T, int RB, typename OPT>
__device__ __forceinline__ void apply_u(typename CxT<T>::type (&v)[1 << RB], const OPT& op, uint32_t t, uint64_t base)
{
    using C = typename CxT<T>::type;
    const int kind = op.kind;
    const int ts = op.tslot;
    const int cs = (op.cslot == NO_SLOT) ? -1 : op.cslot;
    switch (kind) {
        case OP_GEN: {
            GenF<T, RB> f {v, make_cx<T>(op.m[0], op.m[1]), make_cx<T>(op.m[2], op.m[3]), make_cx<T>(op.m[4], op.m[5]),
                           make_cx<T>(op.m[6], op.m[7])};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        case OP_GENR: {
            GenRF<T, RB> f {v, op.m[0], op.m[2], op.m[4], op.m[6]};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        case OP_RXL: {
            RxF<T, RB> f {v, op.m[0], op.m[3]};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        case OP_ANTI: {
            AntiF<T, RB, false> f {v, make_cx<T>(op.m[2], op.m[3]), make_cx<T>(op.m[4], op.m[5])};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        case OP_SWAP: {
            // through the multiply path: a register-move body needs temporaries that spill
            AntiF<T, RB, false> f {v, make_cx<T>(1, 0), make_cx<T>(1, 0)};
            dispatch_sc<RB>(ts, cs, f);
            return;
        }
        default:
            break;
    }
    const C d1 = make_cx<T>(op.m[6], op.m[7]);
    const C d0 = make_cx<T>(op.m[0], op.m[1]);
    if (ts != NO_SLOT) {
        if (kind == OP_DIAG1) {
            DiagRegF<T, RB, true> f {v, d0, d1};
            dispatch_sc<RB>(ts, cs, f);
        } else {
            DiagRegF<T, RB, false> f {v, d0, d1};
            dispatch_sc<RB>(ts, cs, f);
        }
        return;
    }
    const bool b = ((t & op.tthr) != 0) || ((base & op.tglob) != 0);
    if (!b && kind == OP_DIAG1) {
        return;
    }
    DiagAllF<T, RB> f {v, b ? d1 : d0};
    dispatch_c<RB, 99>(cs, f);
}

// Re <lambda| dU/dtheta psi_(g-1)> over this thread's registers, from psi_g
template <typename T, int RB, typename OPT>
__device__ __forceinline__ double grad_term(const typename CxT<T>::type (&l)[1 << RB],
                                            const typename CxT<T>::type (&p)[1 << RB], const OPT& op, uint32_t t,
                                            uint64_t base)
{
    const int ts = op.tslot;
    const int cs = (op.cslot == NO_SLOT) ? -1 : op.cslot;
    if (ts != NO_SLOT) {
        switch (op.gen) {
            case GEN_X: {
                GradRegF<T, RB, GEN_X> f {l, p, 0.0};
                dispatch_sc<RB>(ts, cs, f);
                return 0.5 * f.acc;
            }
            case GEN_Y: {
                GradRegF<T, RB, GEN_Y> f {l, p, 0.0};
                dispatch_sc<RB>(ts, cs, f);
                return 0.5 * f.acc;
            }
            case GEN_Z: {
                GradRegF<T, RB, GEN_Z> f {l, p, 0.0};
                dispatch_sc<RB>(ts, cs, f);
                return 0.5 * f.acc;
            }
            default: {
                GradRegF<T, RB, GEN_P> f {l, p, 0.0};
                dispatch_sc<RB>(ts, cs, f);
                return f.acc;
            }
        }
    }
    // Z or P whose target is a thread bit or outside the tile
    const bool b = ((t & op.tthr) != 0) || ((base & op.tglob) != 0);
    const double w = (op.gen == GEN_Z) ? (b ? -0.5 : 0.5) : (b ? -1.0 : 0.0);
    if (w == 0.0) {
        return 0.0;
    }
    GradAllF<T, RB> f {l, p, 0.0};
    dispatch_c<RB, 99>(cs, f);
    return w * f.acc;
}

// --- per-tile bodies ------------------------------------------------------------
// The amplitude base index of a tile: the tile number's bits spread over the
// qubits outside the tile.
__device__ __forceinline__ uint64_t tile_base(const FBlock& bk, uint64_t tile)
{
    uint64_t base = 0;
    for (int k = 0; k < bk.nfree; ++k) {
        if ((tile >> k) & 1) {
            base |= uint64_t {1} << bk.freebit[k];
        }
    }
    return base;
}

template <int RB>
__device__ __forceinline__ uint64_t reg_offset(const FPhase& ph, int i)
{
    uint64_t o = 0;
#pragma unroll
    for (int s = 0; s < RB; ++s) {
        if (i & (1 << s)) {
            o += ph.rstride[s];
        }
    }
    return o;
}

__device__ __forceinline__ uint64_t thread_offset(const FPhase& ph, uint32_t t, int TB)
{
    uint64_t toff = 0;
    for (int j = 0; j < TB; ++j) {
        if ((t >> j) & 1) {
            toff += ph.tstride[j];
        }
    }
    return toff;
}

// Copy a block's phase table and op records into shared memory (bk must be
// loaded and visible first); word copies by all threads of the CTA.
template <typename OPT>
__device__ __forceinline__ void stage_block(const FBlock& bk, const FPhase* __restrict__ phases,
                                            const OPT* __restrict__ ops, FPhase* sph, OPT* sops, uint32_t t)
{
    const int np = bk.phase_end - bk.phase_begin;
    const int no = bk.op_end - bk.op_begin;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(phases + bk.phase_begin);
    uint32_t* dst = reinterpret_cast<uint32_t*>(sph);
    for (int w = t; w < np * static_cast<int>(sizeof(FPhase) / 4); w += blockDim.x) {
        dst[w] = src[w];
    }
    const uint32_t* so = reinterpret_cast<const uint32_t*>(ops + bk.op_begin);
    uint32_t* dop = reinterpret_cast<uint32_t*>(sops);
    for (int w = t; w < no * static_cast<int>(sizeof(OPT) / 4); w += blockDim.x) {
        dop[w] = so[w];
    }
}

// this thread's part of a phase's store-side shared-memory address
__device__ __forceinline__ uint32_t store_thread_term(const FPhase& ph, uint32_t t, int TB)
{
    uint32_t a = ph.xor_out;
    for (int j = 0; j < TB; ++j) {
        if ((t >> j) & 1) {
            a ^= ph.tsw_out[j];
        }
    }
    return a;
}

template <bool LDCG, typename C>
__device__ __forceinline__ C load_amp(const C* p)
{
    if constexpr (LDCG) {
        return __ldcg(p);  // L2 only: the tile may have been written by another CTA of this launch
    } else {
        return *p;
    }
}

// One tile of a forward block: load it (or, with `init`, start from
// |0...0>), run the block's phases with a shared-memory transpose between
// them, store it.  The block, its phases and ops are already in shared memory.
// Norm bookkeeping of a renormalising apply (complex64): per-warp FP64 sums
// of |a|^2 in shared memory, and the scale applied to every loaded amplitude.
struct NormCtx
{
    double* warp_in;   // sums over the loaded amplitudes (nullptr: not wanted)
    double* warp_out;  // sums over the stored amplitudes
    float scale;
};

// sum of |v_i|^2 over this thread's registers (a pairwise tree in T), then
// over the warp in FP64, added to slot[warp] by lane 0
template <typename T, int R, typename C>
__device__ __forceinline__ void warp_norm_add(const C (&v)[R], double* slot, uint32_t t)
{
    T q[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
        q[i] = v[i].x * v[i].x + v[i].y * v[i].y;
    }
#pragma unroll
    for (int w = 1; w < R; w <<= 1) {
#pragma unroll
        for (int i = 0; i < R; i += 2 * w) {
            q[i] += q[i + w];
        }
    }
    double d = static_cast<double>(q[0]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        d += __shfl_down_sync(0xffffffffU, d, o);
    }
    if ((t & 31) == 0) {
        slot[t >> 5] += d;
    }
}

template <typename T, int RB, bool LDCG, bool NORM = false>
__device__ __forceinline__ void fwd_tile(typename CxT<T>::type* __restrict__ a, const FBlock& bk,
                                         const FPhase* sph, const FOp<T>* sops, uint64_t tile,
                                         typename CxT<T>::type* sm, uint32_t t, bool init,
                                         const NormCtx* nc = nullptr)
{
    using C = typename CxT<T>::type;
    constexpr int R = 1 << RB;
    const int TB = bk.K - RB;
    const int np = bk.phase_end - bk.phase_begin;
    const int op0 = bk.op_begin;
    const uint64_t base = tile_base(bk, tile);
    C v[R];
    {
        const FPhase& ph = sph[0];
        const uint64_t toff = thread_offset(ph, t, TB);
        const C* src = a + base + toff;
        if (init) {
#pragma unroll
            for (int i = 0; i < R; ++i) {
                v[i] = make_cx<T>((base + toff + reg_offset<RB>(ph, i)) == 0 ? T(1) : T(0), T(0));
            }
        } else {
#pragma unroll
            for (int i = 0; i < R; ++i) {
                v[i] = load_amp<LDCG>(src + reg_offset<RB>(ph, i));
            }
        }
        if constexpr (NORM) {
            if (nc->warp_in != nullptr) {
                warp_norm_add<T>(v, nc->warp_in, t);
            }
            const T sc = static_cast<T>(nc->scale);
#pragma unroll
            for (int i = 0; i < R; ++i) {
                v[i].x *= sc;
                v[i].y *= sc;
            }
        }
    }
    for (int p = 0; p < np; ++p) {
        const FPhase& ph = sph[p];
        uint32_t tsw = 0;
        for (int j = 0; j < TB; ++j) {
            if ((t >> j) & 1) {
                tsw ^= ph.tsw[j];
            }
        }
        if (p > 0) {
            // transpose: registers (previous layout, through its folded
            // permutation) -> smem -> registers (this layout)
            const FPhase& pp = sph[p - 1];
            const uint32_t tso = store_thread_term(pp, t, TB);
#pragma unroll
            for (int i = 0; i < R; ++i) {
                sm[tso ^ xor_terms<RB>(i, pp.rsw_out)] = v[i];
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < R; ++i) {
                v[i] = sm[tsw ^ xor_terms<RB>(i, ph.rsw)];
            }
            __syncthreads();
        }
        for (int o = ph.op_begin; o < ph.op_end; ++o) {
            apply_op<T, RB>(v, sops[o - op0], t, base);
        }
    }
    {
        const FPhase& ph = sph[np - 1];
        C* dst = a + base + thread_offset(ph, t, TB);
#pragma unroll
        for (int i = 0; i < R; ++i) {
            dst[reg_offset<RB>(ph, i)] = v[i];
        }
    }
    if constexpr (NORM) {
        warp_norm_add<T>(v, nc->warp_out, t);
    }
}

// One tile of an adjoint block: psi and lambda go through the block's ops
// (U^dagger on both); each parameterised op first adds this tile's share of
// Re <lambda| dU/dtheta psi_(g-1)> into acc[row * ADJ_WARPS + warp].
template <typename T, int RB, bool LDCG>
__device__ __forceinline__ void adj_tile(typename CxT<T>::type* __restrict__ psi, typename CxT<T>::type* __restrict__ lam,
                                         const FBlock& bk, const FPhase* sph, const FOpA<T>* sops, uint64_t tile,
                                         typename CxT<T>::type* smp, typename CxT<T>::type* sml, double* acc,
                                         uint32_t t)
{
    using C = typename CxT<T>::type;
    constexpr int R = 1 << RB;
    const int TB = bk.K - RB;
    const int np = bk.phase_end - bk.phase_begin;
    const int op0 = bk.op_begin;
    const int lane = t & 31;
    const int warp = t >> 5;
    const uint64_t base = tile_base(bk, tile);
    C vp[R];
    C vl[R];
    {
        const FPhase& ph = sph[0];
        const uint64_t off = base + thread_offset(ph, t, TB);
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const uint64_t o = off + reg_offset<RB>(ph, i);
            vp[i] = load_amp<LDCG>(psi + o);
            vl[i] = load_amp<LDCG>(lam + o);
        }
    }
    for (int p = 0; p < np; ++p) {
        const FPhase& ph = sph[p];
        uint32_t tsw = 0;
        for (int j = 0; j < TB; ++j) {
            if ((t >> j) & 1) {
                tsw ^= ph.tsw[j];
            }
        }
        if (p > 0) {
            const FPhase& pp = sph[p - 1];
            const uint32_t tso = store_thread_term(pp, t, TB);
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const uint32_t x = tso ^ xor_terms<RB>(i, pp.rsw_out);
                smp[x] = vp[i];
                sml[x] = vl[i];
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const uint32_t x = tsw ^ xor_terms<RB>(i, ph.rsw);
                vp[i] = smp[x];
                vl[i] = sml[x];
            }
            __syncthreads();
        }
        for (int o = ph.op_begin; o < ph.op_end; ++o) {
            const FOpA<T>& op = sops[o - op0];
            if ((base & op.cglob) != op.cglob) {
                continue;  // control outside the tile is 0: nothing changes, the derivative term is 0
            }
            const bool on = (t & op.cthr) == op.cthr;
            if (op.row >= 0) {
                // the gradient term reads psi_g and lambda before U^dagger is applied to either
                double g = on ? grad_term<T, RB>(vl, vp, op, t, base) : 0.0;
#pragma unroll
                for (int s = 16; s > 0; s >>= 1) {
                    g += __shfl_down_sync(0xffffffffU, g, s);
                }
                if (lane == 0) {
                    acc[op.row * ADJ_WARPS + warp] += g;
                }
            }
            if (on) {
                apply_u<T, RB>(vp, op, t, base);
                apply_u<T, RB>(vl, op, t, base);
            }
        }
    }
    {
        const FPhase& ph = sph[np - 1];
        const uint64_t off = base + thread_offset(ph, t, TB);
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const uint64_t o = off + reg_offset<RB>(ph, i);
            psi[o] = vp[i];
            lam[o] = vl[i];
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
std::vector<PlanBlock> form_blocks(const std::vector<LGate>& g, int n, int K, int L, size_t max_ops)
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
            if ((touch & blocked) != 0 || take.size() >= max_ops) {
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
    auto next_use = [&](int b, size_t from) -> size_t {
        for (size_t k = from; k < m; ++k) {
            if (need[k] == b) {
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
    auto tile_mask = [&](const LGate& x) -> uint64_t {
        uint64_t mk = 0;
        if (loc[x.target] >= 0) mk |= bit(loc[x.target]);
        if (x.control >= 0 && loc[x.control] >= 0) mk |= bit(loc[x.control]);
        return mk;
    };
    struct PhaseSpec
    {
        std::vector<int> regs;
        std::vector<size_t> ops;    // gate positions run as ops in this phase
        std::vector<size_t> folds;  // X / CX applied when this phase is stored
    };
    std::vector<PhaseSpec> ph;
    std::vector<int> cur = choose(0, {});
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
    for (size_t k = 0; k < m; ++k) {
        const LGate& x = g[pb.gates[k]];
        const uint64_t qm = tile_mask(x);
        if (fold[k]) {
            open.folds.push_back(k);
            pending |= qm;
            continue;
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
            std::sort(keep.begin(), keep.end(), [&](int a, int b2) { return next_use(a, k) < next_use(b2, k); });
            cur = choose(k, keep);
            open = PhaseSpec {cur, {}, {}};
            pending = 0;
        }
        open.ops.push_back(k);
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
