// kt_reduce.cu — FP64 reductions over a state: Pauli expectation values,
// norms, inner products, M-gate probabilities and collapse, probabilities,
// and density-matrix trace / Pauli expectation.
//
// Pauli expectation.  The reference copies the state, applies X / Y / Z one
// sweep per site and takes an inner product (operator/pauli/pauli_operator.cpp:76-103).
// With x = the X/Y mask and z = the Z/Y mask of a string,
//   P|i> = i^{#Y} (-1)^{popcount(i & z)} |i ^ x>,
// so <psi|P|psi> = i^{#Y} sum_i conj(psi[i ^ x]) psi[i] (-1)^{popcount(i & z)}.
// Pairing i with j = i ^ x (h = top bit of x clear in i): v = conj(psi[j]) psi[i]
// contributes s_i v + s_j conj(v), and s_j = s_i (-1)^{popcount(x & z)} is
// constant per string, so each string needs one real FP64 accumulator:
// 2 s_i Re(v) when popcount(x & z) is even, 2 s_i Im(v) (times i) when odd.
// Strings with the same x share one read of the state.
#include <algorithm>
#include <map>

#include "kt_complex.cuh"
#include "kt_internal.cuh"

namespace kt
{

namespace
{

constexpr int RED_THREADS = 256;
constexpr int PAULI_MAXG = 16;  // strings per pass slot

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_down_sync(0xffffffffU, v, o);
    }
    return v;
}

// Block-reduce `cnt` accumulators (cnt <= PAULI_MAXG); thread 0 of the block
// writes them to out[j * out_stride] (j < cnt).
template <int MAXG>
__device__ void block_reduce_store(double (&acc)[MAXG], int cnt, double* out, uint64_t out_stride)
{
    __shared__ double sh[RED_THREADS / 32][MAXG];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < MAXG; ++j) {
        if (j < cnt) {
            const double w = warp_sum(acc[j]);
            if (lane == 0) {
                sh[warp][j] = w;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < cnt) {
        double s = 0.0;
        for (int w = 0; w < RED_THREADS / 32; ++w) {
            s += sh[w][threadIdx.x];
        }
        out[threadIdx.x * out_stride] = s;
    }
}

struct PauliSlot
{
    uint64_t x;       // X/Y mask shared by the slot's strings
    int32_t h;        // top bit of x, -1 when x == 0
    int32_t first;    // index of the first string of this slot in the z / out arrays
    int32_t count;    // <= PAULI_MAXG
    int32_t pad;
};

// The slot's work with MAXG >= count accumulators and U grid-stride steps
// (their loads) in flight per thread.  Each thread still adds its terms in the order
// of the plain grid-stride loop (k, k + stride, ...), so the partials do not
// depend on MAXG or U.
template <typename C, int MAXG, int U>
__device__ __forceinline__ void pauli_slot(const C* __restrict__ a, int n, const PauliSlot& sl,
                                           const uint64_t* __restrict__ zmask, double* __restrict__ partial)
{
    uint64_t zs[MAXG];
    double acc[MAXG];
    int par[MAXG];
#pragma unroll
    for (int j = 0; j < MAXG; ++j) {
        zs[j] = (j < sl.count) ? zmask[sl.first + j] : 0;
        par[j] = __popcll(sl.x & zs[j]) & 1;
        acc[j] = 0.0;
    }
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (sl.h < 0) {
        const uint64_t N = uint64_t {1} << n;
        auto add = [&](uint64_t i, double2 v) {
            const double p = v.x * v.x + v.y * v.y;
#pragma unroll
            for (int j = 0; j < MAXG; ++j) {
                if (j < sl.count) {
                    acc[j] += (__popcll(i & zs[j]) & 1) ? -p : p;
                }
            }
        };
        for (; k + (U - 1) * stride < N; k += U * stride) {
            double2 v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                v[u] = to_d2(a[k + u * stride]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                add(k + u * stride, v[u]);
            }
        }
        for (; k < N; k += stride) {
            add(k, to_d2(a[k]));
        }
    } else {
        const uint64_t half = uint64_t {1} << (n - 1);
        auto add = [&](uint64_t i, double2 ai, double2 aj) {
            // v = conj(a_j) * a_i
            const double vr = aj.x * ai.x + aj.y * ai.y;
            const double vi = aj.x * ai.y - aj.y * ai.x;
#pragma unroll
            for (int j = 0; j < MAXG; ++j) {
                if (j < sl.count) {
                    const double t = par[j] ? vi : vr;
                    acc[j] += (__popcll(i & zs[j]) & 1) ? -t : t;
                }
            }
        };
        for (; k + (U - 1) * stride < half; k += U * stride) {
            double2 ai[U], aj[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint64_t i = insert_zero_bit(k + u * stride, sl.h);
                ai[u] = to_d2(a[i]);
                aj[u] = to_d2(a[i ^ sl.x]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                add(insert_zero_bit(k + u * stride, sl.h), ai[u], aj[u]);
            }
        }
        for (; k < half; k += stride) {
            const uint64_t i = insert_zero_bit(k, sl.h);
            add(i, to_d2(a[i]), to_d2(a[i ^ sl.x]));
        }
    }
    block_reduce_store<MAXG>(acc, sl.count, partial + (uint64_t)sl.first * gridDim.x + blockIdx.x, gridDim.x);
}

// grid: (blocks, n_slots).  partial[(first + j) * gridDim.x + blockIdx.x].
// A slot of one string (the usual case: distinct X/Y masks) runs without the
// other accumulators' predicated code and keeps 4 pair loads in flight.
template <typename C>
__global__ void __launch_bounds__(RED_THREADS) k_pauli(const C* __restrict__ a, int n, const PauliSlot* __restrict__ slots,
                                                       const uint64_t* __restrict__ zmask, double* __restrict__ partial)
{
    const PauliSlot sl = slots[blockIdx.y];
    if (sl.count == 1) {
        pauli_slot<C, 1, 4>(a, n, sl, zmask, partial);
    } else if (sl.count <= 4) {
        pauli_slot<C, 4, 4>(a, n, sl, zmask, partial);
    } else {
        pauli_slot<C, PAULI_MAXG, 2>(a, n, sl, zmask, partial);
    }
}

// One thread per string: fixed-order sum of the per-block partials, then the
// string's complex value  phase * i^{#Y} * (odd ? 2i R : 2R)  (R: the real sum;
// the diagonal case uses R directly).
__global__ void k_pauli_finalize(const double* __restrict__ partial, int n_blocks, const uint64_t* __restrict__ xm,
                                 const uint64_t* __restrict__ zm, const int32_t* __restrict__ phase, int64_t n_strings,
                                 double* __restrict__ terms)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_strings) {
        return;
    }
    double r = 0.0;
    for (int b = 0; b < n_blocks; ++b) {
        r += partial[(uint64_t)s * n_blocks + b];
    }
    const uint64_t x = xm[s];
    const uint64_t z = zm[s];
    double re = 0.0, im = 0.0;
    if (x == 0) {
        re = r;
    } else if (__popcll(x & z) & 1) {
        im = 2.0 * r;
    } else {
        re = 2.0 * r;
    }
    // multiply by i^k, k = #Y + phase
    const int k = (__popcll(x & z) + phase[s]) & 3;
    double ore = re, oim = im;
    if (k == 1) { ore = -im; oim = re; }
    else if (k == 2) { ore = -re; oim = -im; }
    else if (k == 3) { ore = im; oim = -re; }
    terms[2 * s] = ore;
    terms[2 * s + 1] = oim;
}

// total = sum_k coeff_k * term_k in string order (one thread, FP64).
__global__ void k_weighted_total(const double* __restrict__ terms, const double* __restrict__ coeffs, int64_t n,
                                 double* __restrict__ total)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    double re = 0.0, im = 0.0;
    for (int64_t k = 0; k < n; ++k) {
        const double cr = coeffs ? coeffs[2 * k] : 1.0;
        const double ci = coeffs ? coeffs[2 * k + 1] : 0.0;
        const double tr = terms[2 * k], ti = terms[2 * k + 1];
        re += cr * tr - ci * ti;
        im += cr * ti + ci * tr;
    }
    total[0] = re;
    total[1] = im;
}

// generic FP64 sums ----------------------------------------------------------
// mode 0: sum |a|^2 -> out[0];  mode 1: P(bit q = 0), P(bit q = 1) -> out[0], out[1]
// mode 2: <b|a> (complex) -> out[0], out[1]
template <typename C>
__global__ void __launch_bounds__(RED_THREADS) k_sums(const C* __restrict__ a, const C* __restrict__ b, uint64_t N,
                                                      int mode, int q, double* __restrict__ partial)
{
    double acc[2] = {0.0, 0.0};
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        const double2 v = to_d2(a[i]);
        if (mode == 2) {
            const double2 w = to_d2(b[i]);
            acc[0] += w.x * v.x + w.y * v.y;
            acc[1] += w.x * v.y - w.y * v.x;
        } else {
            const double p = v.x * v.x + v.y * v.y;
            if (mode == 1 && ((i >> q) & 1)) {
                acc[1] += p;
            } else {
                acc[0] += p;
            }
        }
    }
    double acc2[PAULI_MAXG];
#pragma unroll
    for (int j = 0; j < PAULI_MAXG; ++j) {
        acc2[j] = (j < 2) ? acc[j] : 0.0;
    }
    block_reduce_store<PAULI_MAXG>(acc2, 2, partial + blockIdx.x, gridDim.x);
}

__global__ void k_sums_finalize(const double* __restrict__ partial, int n_blocks, double* __restrict__ out)
{
    if (threadIdx.x < 2 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < n_blocks; ++b) {
            s += partial[(uint64_t)threadIdx.x * n_blocks + b];
        }
        out[threadIdx.x] = s;
    }
}

template <typename C>
__global__ void k_collapse(C* __restrict__ a, uint64_t N, int q, int outcome, double scale)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        C v = a[i];
        if (static_cast<int>((i >> q) & 1) == outcome) {
            v.x = v.x * scale;
            v.y = v.y * scale;
        } else {
            v.x = 0;
            v.y = 0;
        }
        a[i] = v;
    }
}

// |a_i|^2 with round-to-nearest products and sum, no contraction: the value
// std::norm gives on the host (calculations/probabilities.cpp:58).
template <typename C>
__global__ void k_probs(const C* __restrict__ a, uint64_t N, double* __restrict__ p)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        const double2 v = to_d2(a[i]);
        p[i] = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
    }
}

// readout noise on qubit q (probabilities.cpp:110-124), no contraction
__global__ void k_noise(double* __restrict__ p, uint64_t half, int q, double e)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const double one_m = __dsub_rn(1.0, e);
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < half; k += stride) {
        const uint64_t i0 = insert_zero_bit(k, q);
        const uint64_t i1 = i0 | (uint64_t {1} << q);
        const double p0 = p[i0], p1 = p[i1];
        p[i0] = __dadd_rn(__dmul_rn(one_m, p0), __dmul_rn(e, p1));
        p[i1] = __dadd_rn(__dmul_rn(one_m, p1), __dmul_rn(e, p0));
    }
}

// density matrix ----------------------------------------------------------------
// Tr(P rho) = sum_j <j^x|P|j> rho[j, j^x];  one block per string.
template <typename C>
__global__ void __launch_bounds__(RED_THREADS) k_dm_pauli(const C* __restrict__ rho, int n, const uint64_t* __restrict__ xm,
                                                          const uint64_t* __restrict__ zm, double* __restrict__ partial)
{
    const int s = blockIdx.x;
    const uint64_t N = uint64_t {1} << n;
    const uint64_t x = xm[s], z = zm[s];
    double acc[PAULI_MAXG];
#pragma unroll
    for (int j = 0; j < PAULI_MAXG; ++j) {
        acc[j] = 0.0;
    }
    for (uint64_t j = threadIdx.x; j < N; j += blockDim.x) {
        const double2 v = to_d2(rho[j + ((j ^ x) << n)]);
        const bool neg = __popcll(j & z) & 1;
        acc[0] += neg ? -v.x : v.x;
        acc[1] += neg ? -v.y : v.y;
    }
    block_reduce_store<PAULI_MAXG>(acc, 2, partial + 2 * (uint64_t)s, 1);
}

__global__ void k_dm_pauli_finalize(const double* __restrict__ partial, const uint64_t* __restrict__ xm,
                                    const uint64_t* __restrict__ zm, const int32_t* __restrict__ phase, int64_t n_strings,
                                    double* __restrict__ terms)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_strings) {
        return;
    }
    const double re = partial[2 * s], im = partial[2 * s + 1];
    const int k = (__popcll(xm[s] & zm[s]) + phase[s]) & 3;
    double ore = re, oim = im;
    if (k == 1) { ore = -im; oim = re; }
    else if (k == 2) { ore = -re; oim = -im; }
    else if (k == 3) { ore = im; oim = -re; }
    terms[2 * s] = ore;
    terms[2 * s + 1] = oim;
}

template <typename C>
__global__ void k_dm_diag(const C* __restrict__ rho, int n, double* __restrict__ out, int as_complex)
{
    const uint64_t N = uint64_t {1} << n;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < N; j += (uint64_t)gridDim.x * blockDim.x) {
        const double2 v = to_d2(rho[j + (j << n)]);
        if (as_complex) {
            out[2 * j] = v.x;
            out[2 * j + 1] = v.y;
        } else {
            out[j] = v.x;
        }
    }
}

int reduce_blocks(uint64_t work)
{
    const uint64_t want = (work + RED_THREADS - 1) / RED_THREADS;
    const uint64_t cap = static_cast<uint64_t>(sm_count()) * 4;
    return static_cast<int>(std::max<uint64_t>(1, std::min(want, cap)));
}

template <typename F>
int32_t with_dtype(const State& s, F&& f)
{
    if (s.dtype == KT_C128) {
        return f(static_cast<const double2*>(s.amps));
    }
    return f(static_cast<const float2*>(s.amps));
}

int32_t run_sums(State& s, const State* other, int mode, int q, double* host_out2)
{
    const uint64_t N = s.n_amps();
    const int blocks = reduce_blocks(N);
    const size_t need = (2 * static_cast<size_t>(blocks) + 2) * sizeof(double);
    if (const int32_t rc = s.scratch.reserve(need); rc != KT_OK) {
        return rc;
    }
    double* partial = static_cast<double*>(s.scratch.ptr);
    double* out = partial + 2 * blocks;
    const int32_t rc = with_dtype(s, [&](auto* a) -> int32_t {
        using C = std::remove_cv_t<std::remove_pointer_t<decltype(a)>>;
        const C* b = other ? static_cast<const C*>(other->amps) : nullptr;
        k_sums<C><<<blocks, RED_THREADS, 0, s.stream>>>(a, b, N, mode, q, partial);
        KT_CHECK_LAUNCH("k_sums");
        return KT_OK;
    });
    if (rc != KT_OK) {
        return rc;
    }
    k_sums_finalize<<<1, 32, 0, s.stream>>>(partial, blocks, out);
    KT_CHECK_LAUNCH("k_sums_finalize");
    return copy_d2h(host_out2, out, 2 * sizeof(double), s.stream);
}

}  // namespace

int32_t expect_paulis(State& s, const kt_pauli* strings, int64_t n_strings, const double* coeffs, double* out_terms,
                      double* out_total)
{
    if (n_strings <= 0) {
        if (out_total) {
            out_total[0] = 0.0;
            out_total[1] = 0.0;
        }
        return KT_OK;
    }
    const int n = s.n_bits;
    const uint64_t valid = (n >= 64) ? ~uint64_t {0} : ((uint64_t {1} << n) - 1);
    // group strings by X/Y mask, keeping input order inside each group; the
    // kernel writes results in the slot order, mapped back by `order`.
    std::map<uint64_t, std::vector<int64_t>> groups;
    for (int64_t k = 0; k < n_strings; ++k) {
        if ((strings[k].x_mask & ~valid) != 0 || (strings[k].z_mask & ~valid) != 0) {
            set_error(KT_ERR_INVALID, "Pauli string acts on a qubit beyond the state");
            return KT_ERR_INVALID;
        }
        groups[strings[k].x_mask].push_back(k);
    }
    std::vector<PauliSlot> slots;
    std::vector<int64_t> order;  // slot position -> input string index
    order.reserve(static_cast<size_t>(n_strings));
    for (auto& [x, idx] : groups) {
        for (size_t o = 0; o < idx.size(); o += PAULI_MAXG) {
            PauliSlot sl {};
            sl.x = x;
            sl.h = (x == 0) ? -1 : 63 - __builtin_clzll(x);
            sl.first = static_cast<int32_t>(order.size());
            sl.count = static_cast<int32_t>(std::min<size_t>(PAULI_MAXG, idx.size() - o));
            for (int j = 0; j < sl.count; ++j) {
                order.push_back(idx[o + j]);
            }
            slots.push_back(sl);
        }
    }
    std::vector<uint64_t> hx(static_cast<size_t>(n_strings)), hz(static_cast<size_t>(n_strings));
    std::vector<int32_t> hp(static_cast<size_t>(n_strings));
    for (size_t p = 0; p < order.size(); ++p) {
        hx[p] = strings[order[p]].x_mask;
        hz[p] = strings[order[p]].z_mask;
        hp[p] = strings[order[p]].phase & 3;
    }
    const int blocks = reduce_blocks(s.n_amps() / 2 + 1);
    // scratch layout (bytes, 256-aligned pieces)
    auto al = [](size_t v) { return (v + 255) & ~size_t {255}; };
    const size_t ns = static_cast<size_t>(n_strings);
    const size_t off_slots = 0;
    const size_t off_x = al(off_slots + slots.size() * sizeof(PauliSlot));
    const size_t off_z = al(off_x + ns * 8);
    const size_t off_p = al(off_z + ns * 8);
    const size_t off_part = al(off_p + ns * 4);
    const size_t off_terms = al(off_part + ns * static_cast<size_t>(blocks) * 8);
    const size_t off_coef = al(off_terms + ns * 16);
    const size_t off_tot = al(off_coef + ns * 16);
    const size_t need = off_tot + 16;
    if (const int32_t rc = s.scratch.reserve(need); rc != KT_OK) {
        return rc;
    }
    char* base = static_cast<char*>(s.scratch.ptr);
    auto* d_slots = reinterpret_cast<PauliSlot*>(base + off_slots);
    auto* d_x = reinterpret_cast<uint64_t*>(base + off_x);
    auto* d_z = reinterpret_cast<uint64_t*>(base + off_z);
    auto* d_p = reinterpret_cast<int32_t*>(base + off_p);
    auto* d_part = reinterpret_cast<double*>(base + off_part);
    auto* d_terms = reinterpret_cast<double*>(base + off_terms);
    auto* d_coef = reinterpret_cast<double*>(base + off_coef);
    auto* d_tot = reinterpret_cast<double*>(base + off_tot);
    if (int32_t rc = copy_h2d(d_slots, slots.data(), slots.size() * sizeof(PauliSlot), s.stream); rc != KT_OK) return rc;
    if (int32_t rc = copy_h2d(d_x, hx.data(), ns * 8, s.stream); rc != KT_OK) return rc;
    if (int32_t rc = copy_h2d(d_z, hz.data(), ns * 8, s.stream); rc != KT_OK) return rc;
    if (int32_t rc = copy_h2d(d_p, hp.data(), ns * 4, s.stream); rc != KT_OK) return rc;
    const int32_t rc = with_dtype(s, [&](auto* a) -> int32_t {
        using C = std::remove_cv_t<std::remove_pointer_t<decltype(a)>>;
        // grid.y is limited to 65535: launch the slots in chunks
        for (size_t s0 = 0; s0 < slots.size(); s0 += 65535) {
            const unsigned ny = static_cast<unsigned>(std::min<size_t>(65535, slots.size() - s0));
            k_pauli<C><<<dim3(blocks, ny), RED_THREADS, 0, s.stream>>>(a, n, d_slots + s0, d_z, d_part);
            KT_CHECK_LAUNCH("k_pauli");
        }
        return KT_OK;
    });
    if (rc != KT_OK) {
        return rc;
    }
    k_pauli_finalize<<<static_cast<unsigned>((n_strings + 127) / 128), 128, 0, s.stream>>>(d_part, blocks, d_x, d_z, d_p,
                                                                                           n_strings, d_terms);
    KT_CHECK_LAUNCH("k_pauli_finalize");
    std::vector<double> terms_sorted(2 * ns);
    if (int32_t r2 = copy_d2h(terms_sorted.data(), d_terms, ns * 16, s.stream); r2 != KT_OK) return r2;
    std::vector<double> terms(2 * ns);
    for (size_t p = 0; p < order.size(); ++p) {
        terms[2 * order[p]] = terms_sorted[2 * p];
        terms[2 * order[p] + 1] = terms_sorted[2 * p + 1];
    }
    if (out_terms) {
        std::copy(terms.begin(), terms.end(), out_terms);
    }
    if (out_total) {
        // weighted sum in input order, on the device in FP64
        if (int32_t r3 = copy_h2d(d_terms, terms.data(), ns * 16, s.stream); r3 != KT_OK) return r3;
        const double* dc = nullptr;
        if (coeffs) {
            if (int32_t r4 = copy_h2d(d_coef, coeffs, ns * 16, s.stream); r4 != KT_OK) return r4;
            dc = d_coef;
        }
        k_weighted_total<<<1, 32, 0, s.stream>>>(d_terms, dc, n_strings, d_tot);
        KT_CHECK_LAUNCH("k_weighted_total");
        if (int32_t r5 = copy_d2h(out_total, d_tot, 16, s.stream); r5 != KT_OK) return r5;
    }
    return KT_OK;
}

// The Pauli-expectation kernels on caller-provided device tables (used by the
// allocation-free entry point): k_pauli over `n_slots` slots, then the
// per-string finalisation into `terms` (slot order).
int32_t pauli_terms_launch(const void* amps, int n, int32_t dtype, const void* slots, int n_slots,
                           const uint64_t* xm, const uint64_t* zm, const int32_t* phase, int64_t n_strings,
                           double* partial, int blocks, double* terms, cudaStream_t stream)
{
    const auto* sl = static_cast<const PauliSlot*>(slots);
    for (int s0 = 0; s0 < n_slots; s0 += 65535) {
        const unsigned ny = static_cast<unsigned>(std::min(65535, n_slots - s0));
        if (dtype == KT_C128) {
            k_pauli<double2><<<dim3(blocks, ny), RED_THREADS, 0, stream>>>(static_cast<const double2*>(amps), n, sl + s0,
                                                                          zm, partial);
        } else {
            k_pauli<float2><<<dim3(blocks, ny), RED_THREADS, 0, stream>>>(static_cast<const float2*>(amps), n, sl + s0,
                                                                         zm, partial);
        }
        KT_CHECK_LAUNCH("k_pauli");
    }
    k_pauli_finalize<<<static_cast<unsigned>((n_strings + 127) / 128), 128, 0, stream>>>(partial, blocks, xm, zm, phase,
                                                                                         n_strings, terms);
    KT_CHECK_LAUNCH("k_pauli_finalize");
    return KT_OK;
}

int32_t weighted_total_launch(const double* terms, const double* coeffs, int64_t n, double* total, cudaStream_t stream)
{
    k_weighted_total<<<1, 32, 0, stream>>>(terms, coeffs, n, total);
    KT_CHECK_LAUNCH("k_weighted_total");
    return KT_OK;
}

int pauli_slot_bytes()
{
    return static_cast<int>(sizeof(PauliSlot));
}

int pauli_slot_width()
{
    return PAULI_MAXG;
}

// reduction blocks per string of kt_sv_expect on a state of n_bits index bits
int pauli_blocks(int n_bits)
{
    return reduce_blocks((uint64_t {1} << n_bits) / 2 + 1);
}

int32_t norm_sq(State& s, double* out)
{
    double r[2];
    const int32_t rc = run_sums(s, nullptr, 0, 0, r);
    if (rc == KT_OK) {
        *out = r[0];
    }
    return rc;
}

int32_t inner_product(State& bra, State& ket, double* out)
{
    // <bra|ket> = sum conj(bra_i) ket_i: k_sums mode 2 computes sum conj(b) a with a = ket
    return run_sums(ket, &bra, 2, 0, out);
}

int32_t measure_probs(State& s, uint32_t q, double* p0, double* p1)
{
    double r[2];
    const int32_t rc = run_sums(s, nullptr, 1, static_cast<int>(q), r);
    if (rc == KT_OK) {
        *p0 = r[0];
        *p1 = r[1];
    }
    return rc;
}

int32_t collapse(State& s, uint32_t q, int32_t outcome, double scale)
{
    const uint64_t N = s.n_amps();
    const int blocks = reduce_blocks(N) * 4;
    if (s.dtype == KT_C128) {
        k_collapse<double2><<<blocks, RED_THREADS, 0, s.stream>>>(static_cast<double2*>(s.amps), N, static_cast<int>(q),
                                                                  outcome, scale);
    } else {
        k_collapse<float2><<<blocks, RED_THREADS, 0, s.stream>>>(static_cast<float2*>(s.amps), N, static_cast<int>(q),
                                                                 outcome, scale);
    }
    KT_CHECK_LAUNCH("k_collapse");
    return KT_OK;
}

// device probabilities into `dev_p` (N doubles), with optional noise (host array of n)
int32_t device_probabilities(State& s, const double* noise, double* dev_p)
{
    const uint64_t N = s.n_amps();
    const int blocks = reduce_blocks(N) * 4;
    if (s.dtype == KT_C128) {
        k_probs<double2><<<blocks, RED_THREADS, 0, s.stream>>>(static_cast<const double2*>(s.amps), N, dev_p);
    } else {
        k_probs<float2><<<blocks, RED_THREADS, 0, s.stream>>>(static_cast<const float2*>(s.amps), N, dev_p);
    }
    KT_CHECK_LAUNCH("k_probs");
    if (noise != nullptr) {
        for (int q = 0; q < s.n_bits; ++q) {
            if (!(noise[q] >= 0.0 && noise[q] <= 1.0)) {
                set_error(KT_ERR_INVALID, "ERROR: Cannot set probability in QuantumNoise object outside of [0, 1].");
                return KT_ERR_INVALID;
            }
            k_noise<<<blocks, RED_THREADS, 0, s.stream>>>(dev_p, N / 2, q, noise[q]);
            KT_CHECK_LAUNCH("k_noise");
        }
    }
    return KT_OK;
}

int32_t probabilities(State& s, const double* noise, double* host_out)
{
    const uint64_t N = s.n_amps();
    if (const int32_t rc = s.scratch2.reserve(N * sizeof(double)); rc != KT_OK) {
        return rc;
    }
    double* dp = static_cast<double*>(s.scratch2.ptr);
    if (const int32_t rc = device_probabilities(s, noise, dp); rc != KT_OK) {
        return rc;
    }
    return copy_d2h(host_out, dp, N * sizeof(double), s.stream);
}

int32_t dm_expect_paulis(State& s, int n, const kt_pauli* strings, int64_t n_strings, const double* coeffs,
                         double* out_terms, double* out_total)
{
    if (n_strings <= 0) {
        if (out_total) {
            out_total[0] = 0.0;
            out_total[1] = 0.0;
        }
        return KT_OK;
    }
    const size_t ns = static_cast<size_t>(n_strings);
    const uint64_t valid = (uint64_t {1} << n) - 1;
    std::vector<uint64_t> hx(ns), hz(ns);
    std::vector<int32_t> hp(ns);
    for (size_t k = 0; k < ns; ++k) {
        if ((strings[k].x_mask & ~valid) != 0 || (strings[k].z_mask & ~valid) != 0) {
            set_error(KT_ERR_INVALID, "Pauli string acts on a qubit beyond the density matrix");
            return KT_ERR_INVALID;
        }
        hx[k] = strings[k].x_mask;
        hz[k] = strings[k].z_mask;
        hp[k] = strings[k].phase & 3;
    }
    auto al = [](size_t v) { return (v + 255) & ~size_t {255}; };
    const size_t off_x = 0;
    const size_t off_z = al(ns * 8);
    const size_t off_p = al(off_z + ns * 8);
    const size_t off_part = al(off_p + ns * 4);
    const size_t off_terms = al(off_part + ns * 16);
    const size_t off_coef = al(off_terms + ns * 16);
    const size_t off_tot = al(off_coef + ns * 16);
    if (const int32_t rc = s.scratch.reserve(off_tot + 16); rc != KT_OK) {
        return rc;
    }
    char* base = static_cast<char*>(s.scratch.ptr);
    auto* d_x = reinterpret_cast<uint64_t*>(base + off_x);
    auto* d_z = reinterpret_cast<uint64_t*>(base + off_z);
    auto* d_p = reinterpret_cast<int32_t*>(base + off_p);
    auto* d_part = reinterpret_cast<double*>(base + off_part);
    auto* d_terms = reinterpret_cast<double*>(base + off_terms);
    auto* d_coef = reinterpret_cast<double*>(base + off_coef);
    auto* d_tot = reinterpret_cast<double*>(base + off_tot);
    if (int32_t rc = copy_h2d(d_x, hx.data(), ns * 8, s.stream); rc != KT_OK) return rc;
    if (int32_t rc = copy_h2d(d_z, hz.data(), ns * 8, s.stream); rc != KT_OK) return rc;
    if (int32_t rc = copy_h2d(d_p, hp.data(), ns * 4, s.stream); rc != KT_OK) return rc;
    const int32_t rc = with_dtype(s, [&](auto* a) -> int32_t {
        using C = std::remove_cv_t<std::remove_pointer_t<decltype(a)>>;
        for (size_t s0 = 0; s0 < ns; s0 += 65535) {
            const unsigned nb = static_cast<unsigned>(std::min<size_t>(65535, ns - s0));
            k_dm_pauli<C><<<nb, RED_THREADS, 0, s.stream>>>(a, n, d_x + s0, d_z + s0, d_part + 2 * s0);
            KT_CHECK_LAUNCH("k_dm_pauli");
        }
        return KT_OK;
    });
    if (rc != KT_OK) {
        return rc;
    }
    k_dm_pauli_finalize<<<static_cast<unsigned>((ns + 127) / 128), 128, 0, s.stream>>>(d_part, d_x, d_z, d_p, n_strings,
                                                                                       d_terms);
    KT_CHECK_LAUNCH("k_dm_pauli_finalize");
    if (out_terms) {
        if (int32_t r2 = copy_d2h(out_terms, d_terms, ns * 16, s.stream); r2 != KT_OK) return r2;
    }
    if (out_total) {
        const double* dc = nullptr;
        if (coeffs) {
            if (int32_t r4 = copy_h2d(d_coef, coeffs, ns * 16, s.stream); r4 != KT_OK) return r4;
            dc = d_coef;
        }
        k_weighted_total<<<1, 32, 0, s.stream>>>(d_terms, dc, n_strings, d_tot);
        KT_CHECK_LAUNCH("k_weighted_total");
        if (int32_t r5 = copy_d2h(out_total, d_tot, 16, s.stream); r5 != KT_OK) return r5;
    }
    return KT_OK;
}

int32_t dm_trace(State& s, int n, double* out)
{
    const uint64_t N = uint64_t {1} << n;
    if (const int32_t rc = s.scratch.reserve(N * 16); rc != KT_OK) {
        return rc;
    }
    double* d = static_cast<double*>(s.scratch.ptr);
    const int32_t rc = with_dtype(s, [&](auto* a) -> int32_t {
        using C = std::remove_cv_t<std::remove_pointer_t<decltype(a)>>;
        k_dm_diag<C><<<reduce_blocks(N), RED_THREADS, 0, s.stream>>>(a, n, d, 1);
        KT_CHECK_LAUNCH("k_dm_diag");
        return KT_OK;
    });
    if (rc != KT_OK) {
        return rc;
    }
    std::vector<double> h(2 * N);
    if (int32_t r2 = copy_d2h(h.data(), d, N * 16, s.stream); r2 != KT_OK) return r2;
    double re = 0.0, im = 0.0;
    for (uint64_t j = 0; j < N; ++j) {
        re += h[2 * j];
        im += h[2 * j + 1];
    }
    out[0] = re;
    out[1] = im;
    return KT_OK;
}

int32_t dm_diagonal(State& s, int n, double* host_out)
{
    const uint64_t N = uint64_t {1} << n;
    if (const int32_t rc = s.scratch.reserve(N * 8); rc != KT_OK) {
        return rc;
    }
    double* d = static_cast<double*>(s.scratch.ptr);
    const int32_t rc = with_dtype(s, [&](auto* a) -> int32_t {
        using C = std::remove_cv_t<std::remove_pointer_t<decltype(a)>>;
        k_dm_diag<C><<<reduce_blocks(N), RED_THREADS, 0, s.stream>>>(a, n, d, 0);
        KT_CHECK_LAUNCH("k_dm_diag");
        return KT_OK;
    });
    if (rc != KT_OK) {
        return rc;
    }
    return copy_d2h(host_out, d, N * 8, s.stream);
}

}  // namespace kt
