// kt_sweep.cu — one HBM sweep per gate, and the pair-index enumeration.
//
// The reference walks the 2^(n-1) (or 2^(n-2)) amplitude pairs of a gate with
// SingleQubitGatePairGenerator / DoubleQubitGatePairGenerator
// (simulation/gate_pair_generator.hpp:25-160), whose order makes the high
// index bits move fastest.  Every pair is independent, so here pair k is
// mapped to its amplitudes by inserting a zero bit at the target (and at the
// control, then setting it): consecutive k give consecutive addresses, so a
// warp's loads are coalesced.  kt_pairs_* reproduce the reference's order
// itself, bit for bit, for verification.
#include "kt_complex.cuh"
#include "kt_internal.cuh"

namespace kt
{

namespace
{

constexpr int SWEEP_THREADS = 256;
constexpr int SWEEP_UNROLL = 4;

template <typename T>
struct Mat2
{
    T v[8];
};

template <typename T, int KIND, bool CTRL>
__global__ void __launch_bounds__(SWEEP_THREADS) k_sweep(typename CxT<T>::type* __restrict__ a, uint64_t n_pairs,
                                                         int t, int c, int lo, int hi, Mat2<T> m, int m00_is_one)
{
    using C = typename CxT<T>::type;
    const uint64_t base = (uint64_t)blockIdx.x * (SWEEP_THREADS * SWEEP_UNROLL) + threadIdx.x;
    const uint64_t tb = uint64_t {1} << t;
    uint64_t s0[SWEEP_UNROLL];
    C x0[SWEEP_UNROLL], x1[SWEEP_UNROLL];
    bool ok[SWEEP_UNROLL];
#pragma unroll
    for (int j = 0; j < SWEEP_UNROLL; ++j) {
        const uint64_t k = base + (uint64_t)j * SWEEP_THREADS;
        ok[j] = k < n_pairs;
        uint64_t i;
        if (CTRL) {
            i = insert_zero_bit(insert_zero_bit(k, lo), hi) | (uint64_t {1} << c);
        } else {
            i = insert_zero_bit(k, t);
        }
        s0[j] = i;
        if (ok[j]) {
            if (!(KIND == KIND_DIAG && m00_is_one)) {
                x0[j] = a[i];
            }
            x1[j] = a[i | tb];
        }
    }
#pragma unroll
    for (int j = 0; j < SWEEP_UNROLL; ++j) {
        if (!ok[j]) {
            continue;
        }
        const C m00 = make_cx<T>(m.v[0], m.v[1]);
        const C m01 = make_cx<T>(m.v[2], m.v[3]);
        const C m10 = make_cx<T>(m.v[4], m.v[5]);
        const C m11 = make_cx<T>(m.v[6], m.v[7]);
        if (KIND == KIND_GEN) {
            const C n0 = cfma(m01, x1[j], cmul(m00, x0[j]));
            const C n1 = cfma(m11, x1[j], cmul(m10, x0[j]));
            a[s0[j]] = n0;
            a[s0[j] | tb] = n1;
        } else if (KIND == KIND_ANTI) {
            a[s0[j]] = cmul(m01, x1[j]);
            a[s0[j] | tb] = cmul(m10, x0[j]);
        } else {
            if (!m00_is_one) {
                a[s0[j]] = cmul(m00, x0[j]);
            }
            a[s0[j] | tb] = cmul(m11, x1[j]);
        }
    }
}

template <typename T>
int32_t sweep_typed(State& s, const LGate& g)
{
    using C = typename CxT<T>::type;
    const int n = s.n_bits;
    const bool ctrl = g.control >= 0;
    if (ctrl && n < 2) {
        return KT_OK;
    }
    const uint64_t n_pairs = ctrl ? (uint64_t {1} << (n - 2)) : (uint64_t {1} << (n - 1));
    const uint64_t per_block = SWEEP_THREADS * SWEEP_UNROLL;
    const uint64_t blocks = (n_pairs + per_block - 1) / per_block;
    Mat2<T> m;
    for (int k = 0; k < 8; ++k) {
        m.v[k] = static_cast<T>(g.m[k]);
    }
    const int t = g.target;
    const int c = ctrl ? g.control : 0;
    const int lo = ctrl ? (c < t ? c : t) : t;
    const int hi = ctrl ? (c < t ? t : c) : t;
    C* a = static_cast<C*>(s.amps);
    const int one = (g.flags & 1) ? 1 : 0;
    const dim3 grid(static_cast<unsigned>(blocks));
#define KT_SWEEP_LAUNCH(KIND)                                                                                   \
    if (ctrl) {                                                                                                 \
        k_sweep<T, KIND, true><<<grid, SWEEP_THREADS, 0, s.stream>>>(a, n_pairs, t, c, lo, hi, m, one);         \
    } else {                                                                                                    \
        k_sweep<T, KIND, false><<<grid, SWEEP_THREADS, 0, s.stream>>>(a, n_pairs, t, c, lo, hi, m, one);        \
    }
    switch (g.kind) {
        case KIND_GEN: KT_SWEEP_LAUNCH(KIND_GEN); break;
        case KIND_ANTI: KT_SWEEP_LAUNCH(KIND_ANTI); break;
        default: KT_SWEEP_LAUNCH(KIND_DIAG); break;
    }
#undef KT_SWEEP_LAUNCH
    KT_CHECK_LAUNCH("k_sweep");
    return KT_OK;
}

// --- reference pair order ---------------------------------------------------
// kind 0: single-target next(); 1: double next(); 2: double next_unset_and_set()
__global__ void k_pairs(uint32_t n, uint32_t c, uint32_t t, int kind, uint64_t k0, uint64_t count,
                        uint64_t* __restrict__ out)
{
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) {
        return;
    }
    const uint64_t k = k0 + j;
    if (kind == 0) {
        // (i0, i1) = (k / 2^(n-t-1), k % 2^(n-t-1)); s0 = i0 + i1 * 2^(t+1)
        const uint32_t hb = n - t - 1;
        const uint64_t i0 = k >> hb;
        const uint64_t i1 = k & ((uint64_t {1} << hb) - 1);
        const uint64_t s0 = i0 + (i1 << (t + 1));
        out[2 * j] = s0;
        out[2 * j + 1] = s0 + (uint64_t {1} << t);
        return;
    }
    const uint32_t lo = c < t ? c : t;
    const uint32_t hi = c < t ? t : c;
    const uint32_t b2 = n - hi - 1;          // bits of i2
    const uint32_t b1 = hi - lo - 1;         // bits of i1
    const uint64_t i0 = k >> (b1 + b2);
    const uint64_t i1 = (k >> b2) & ((uint64_t {1} << b1) - 1);
    const uint64_t i2 = k & ((uint64_t {1} << b2) - 1);
    const uint64_t base = i0 + (i1 << (lo + 1)) + (i2 << (hi + 1));
    const uint64_t cs = uint64_t {1} << c;
    const uint64_t ts = uint64_t {1} << t;
    if (kind == 1) {
        out[2 * j] = base + cs;
        out[2 * j + 1] = base + cs + ts;
    } else {
        out[4 * j] = base;
        out[4 * j + 1] = base + ts;
        out[4 * j + 2] = base + cs;
        out[4 * j + 3] = base + cs + ts;
    }
}

template <typename C>
__global__ void k_set_basis(C* __restrict__ a, uint64_t n, uint64_t index)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        C v;
        v.x = (i == index) ? 1 : 0;
        v.y = 0;
        a[i] = v;
    }
}

__global__ void k_c128_to_c64(const double2* __restrict__ src, float2* __restrict__ dst, uint64_t n)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double2 v = src[i];
        dst[i] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    }
}

__global__ void k_c64_to_c128(const float2* __restrict__ src, double2* __restrict__ dst, uint64_t n)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float2 v = src[i];
        dst[i] = make_double2(v.x, v.y);
    }
}

unsigned grid_for(uint64_t n, int threads)
{
    const uint64_t want = (n + threads - 1) / threads;
    const uint64_t cap = static_cast<uint64_t>(sm_count()) * 16;
    return static_cast<unsigned>(want < cap ? (want == 0 ? 1 : want) : cap);
}

}  // namespace

double sweep_alg_bytes(const State& s, const LGate& g)
{
    // read + write of every amplitude the sweep touches
    const double all = 2.0 * static_cast<double>(s.amp_bytes()) * static_cast<double>(s.n_amps());
    double frac = (g.control >= 0) ? 0.5 : 1.0;
    if (g.kind == KIND_DIAG && (g.flags & 1)) {
        frac *= 0.5;
    }
    return all * frac;
}

int32_t launch_gate_sweep(State& s, const LGate& g)
{
    s.last_launches += 1;
    s.last_alg_bytes += sweep_alg_bytes(s, g);
    return s.dtype == KT_C128 ? sweep_typed<double>(s, g) : sweep_typed<float>(s, g);
}

int32_t launch_pairs(uint32_t n, uint32_t c, uint32_t t, int kind, uint64_t k0, uint64_t count, uint64_t* dev_out,
                     cudaStream_t stream)
{
    if (count == 0) {
        return KT_OK;
    }
    const int threads = 256;
    const uint64_t blocks = (count + threads - 1) / threads;
    k_pairs<<<static_cast<unsigned>(blocks), threads, 0, stream>>>(n, c, t, kind, k0, count, dev_out);
    KT_CHECK_LAUNCH("k_pairs");
    return KT_OK;
}

int32_t launch_set_basis(State& s, uint64_t index)
{
    const uint64_t n = s.n_amps();
    if (s.dtype == KT_C128) {
        k_set_basis<double2><<<grid_for(n, 256), 256, 0, s.stream>>>(static_cast<double2*>(s.amps), n, index);
    } else {
        k_set_basis<float2><<<grid_for(n, 256), 256, 0, s.stream>>>(static_cast<float2*>(s.amps), n, index);
    }
    KT_CHECK_LAUNCH("k_set_basis");
    return KT_OK;
}

int32_t launch_convert_to_state(State& s, const double* dev_c128, uint64_t n)
{
    k_c128_to_c64<<<grid_for(n, 256), 256, 0, s.stream>>>(reinterpret_cast<const double2*>(dev_c128),
                                                           static_cast<float2*>(s.amps), n);
    KT_CHECK_LAUNCH("k_c128_to_c64");
    return KT_OK;
}

int32_t launch_convert_from_state(const State& s, double* dev_c128, uint64_t n)
{
    k_c64_to_c128<<<grid_for(n, 256), 256, 0, s.stream>>>(static_cast<const float2*>(s.amps),
                                                           reinterpret_cast<double2*>(dev_c128), n);
    KT_CHECK_LAUNCH("k_c64_to_c128");
    return KT_OK;
}

}  // namespace kt
