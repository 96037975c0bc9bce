// kt_fused_dev.cuh — the device side of fused gate blocks: op records,
// layouts, register-level gate bodies and the per-tile bodies of the forward
// and adjoint kernels.  Included by kt_fused.cuh (with the host planner) and,
// through the run-time compiler, by the generated block kernels (kt_jit.cpp),
// so it depends on nothing but kt_complex.cuh.
#pragma once

#include "kt_complex.cuh"

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
// 8 complex128 amplitudes per thread (the forward kernel's fused_reg_bits = 3 shapes)
struct Cfg3
{
    static constexpr int RB = 3;
    static constexpr int L = 3;
    static constexpr int G = 3;
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

// A real gate with m11 = +-m00 != 0 divided by m00, [[1, p], [q, +-1]]; its
// factor m00 is applied once per block elsewhere (run-time compiled blocks):
// one FMA per component instead of a multiply and an FMA.
template <typename T, int RB, bool NEG>
struct GenRSF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    T p, q;
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
                x.x = fma(p, b.x, a.x);
                x.y = fma(p, b.y, a.y);
                y.x = fma(q, a.x, NEG ? -b.x : b.x);
                y.y = fma(q, a.y, NEG ? -b.y : b.y);
                v[i] = x;
                v[j] = y;
            }
        }
    }
};

// A general gate divided by m00 != 0, [[1, p], [q, r]]: 12 FP64 operations
// per pair instead of 16, the factor m00 applied once per block elsewhere
template <typename T, int RB>
struct GenSF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    C p, q, r;
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
                v[i] = cfma(p, b, a);
                v[j] = cfma(r, b, cmul(q, a));
            }
        }
    }
};

// [[1, i t], [i t, 1]]: an RX-like gate [[c, i s], [i s, c]] divided by c != 0
// (t = s / c), its factor c applied once per block elsewhere
template <typename T, int RB>
struct RxSF
{
    using C = typename CxT<T>::type;
    C (&v)[1 << RB];
    T t;
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
                x.x = fma(-t, b.y, a.x);
                x.y = fma(t, b.x, a.y);
                y.x = fma(-t, a.y, b.x);
                y.y = fma(t, a.x, b.y);
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

// complex64 states: a thread's terms of one op are formed and summed in FP32
// (the amplitudes carry FP32 precision; at most 2^RB terms), and only that
// sum joins the FP64 accumulator
__device__ __forceinline__ float im_cj(float2 a, float2 b)
{
    return a.x * b.y - a.y * b.x;
}

__device__ __forceinline__ float re_cj(float2 a, float2 b)
{
    return a.x * b.x + a.y * b.y;
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
        using R = T;  // the terms' precision: FP64 for complex128, FP32 for complex64
        R sum = 0;
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (lower_of_pair<S, CS>(i, crt)) {
                const int j = i | (1 << S);
                const C l0 = l[i], l1 = l[j];
                const C p0 = p[i], p1 = p[j];
                if constexpr (GENK == GEN_X) {
                    sum += im_cj(l0, p1) + im_cj(l1, p0);
                } else if constexpr (GENK == GEN_Y) {
                    sum += re_cj(l1, p0) - re_cj(l0, p1);
                } else if constexpr (GENK == GEN_Z) {
                    sum += im_cj(l0, p0) - im_cj(l1, p1);
                } else {
                    sum -= im_cj(l1, p1);
                }
            }
        }
        acc += static_cast<double>(sum);
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
        T sum = 0;
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            if (ctrl_on<CS>(i, crt)) {
                sum += im_cj(l[i], p[i]);
            }
        }
        acc += static_cast<double>(sum);
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
struct NormArgs
{
    const double* target;  // per-CTA target sums (nullptr in the first block)
    const double* prev;    // per-CTA sums left by the previous block (nullptr in the first block)
    int n_parts;
    double* in_parts;      // first block: per-CTA sums over the loads (the target)
    double* out_parts;     // per-CTA sums over the stores
};

__device__ __forceinline__ double norm_scale(const double* target, const double* prev, int n)
{
    double num = 0.0, den = 0.0;
    for (int i = 0; i < n; ++i) {
        num += target[i];
        den += prev[i];
    }
    return (num > 0.0 && den > 0.0) ? sqrt(num / den) : 1.0;
}

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

// The pieces of a forward tile: the load in phase 0's layout, the transpose
// between two phases (registers -> shared memory through the previous
// phase's folded permutation -> registers in this phase's layout), the store
// in the last phase's layout.
template <typename T, int RB, bool LDCG>
__device__ __forceinline__ void tile_load(typename CxT<T>::type (&v)[1 << RB], const typename CxT<T>::type* __restrict__ a,
                                          const FPhase& ph, uint64_t base, uint32_t t, int TB, bool init)
{
    const uint64_t toff = thread_offset(ph, t, TB);
    const typename CxT<T>::type* src = a + base + toff;
    if (init) {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            v[i] = make_cx<T>((base + toff + reg_offset<RB>(ph, i)) == 0 ? T(1) : T(0), T(0));
        }
    } else {
#pragma unroll
        for (int i = 0; i < (1 << RB); ++i) {
            v[i] = load_amp<LDCG>(src + reg_offset<RB>(ph, i));
        }
    }
}

template <typename T, int RB>
__device__ __forceinline__ void tile_transpose(typename CxT<T>::type (&v)[1 << RB], typename CxT<T>::type* sm,
                                               const FPhase& prev, const FPhase& ph, uint32_t t, int TB)
{
    uint32_t tsw = 0;
    for (int j = 0; j < TB; ++j) {
        if ((t >> j) & 1) {
            tsw ^= ph.tsw[j];
        }
    }
    const uint32_t tso = store_thread_term(prev, t, TB);
#pragma unroll
    for (int i = 0; i < (1 << RB); ++i) {
        sm[tso ^ xor_terms<RB>(i, prev.rsw_out)] = v[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < (1 << RB); ++i) {
        v[i] = sm[tsw ^ xor_terms<RB>(i, ph.rsw)];
    }
    __syncthreads();
}

template <typename T, int RB>
__device__ __forceinline__ void tile_store(const typename CxT<T>::type (&v)[1 << RB], typename CxT<T>::type* __restrict__ a,
                                           const FPhase& ph, uint64_t base, uint32_t t, int TB)
{
    typename CxT<T>::type* dst = a + base + thread_offset(ph, t, TB);
#pragma unroll
    for (int i = 0; i < (1 << RB); ++i) {
        dst[reg_offset<RB>(ph, i)] = v[i];
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
    tile_load<T, RB, LDCG>(v, a, sph[0], base, t, TB, init);
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
    for (int p = 0; p < np; ++p) {
        const FPhase& ph = sph[p];
        if (p > 0) {
            tile_transpose<T, RB>(v, sm, sph[p - 1], ph, t, TB);
        }
        for (int o = ph.op_begin; o < ph.op_end; ++o) {
            apply_op<T, RB>(v, sops[o - op0], t, base);
        }
    }
    tile_store<T, RB>(v, a, sph[np - 1], base, t, TB);
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

}  // namespace

}  // namespace kt
