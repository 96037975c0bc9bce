// kt_adjoint.cu — adjoint differentiation of E(theta) = <psi|H|psi>.
//
// No reference counterpart: kettle has no gradient of any kind (its VQE loop,
// example/algorithms/vqe_basic.cpp:61-96, drives a derivative-free optimiser).
//
// forward:  psi = U_G ... U_1 psi0 (fused sweeps), E = Re <psi|H|psi> (FP64).
// backward: lambda = H psi, then for g = G .. 1
//              psi    <- U_g^dagger psi              (psi is now psi_{g-1})
//              dE/dtheta_g = 2 Re <lambda| dU_g/dtheta psi_{g-1}>   (FP64)
//              lambda <- U_g^dagger lambda
//           one kernel per gate reads and writes both states once and
//           reduces the inner product per block; the per-gate sums are
//           finalised in a fixed order (deterministic).
// Checkpoints: with checkpoint_every = k > 0 the forward pass keeps a copy of
// psi after every k gates while device memory allows; the backward pass
// restores psi from them instead of relying on un-applying alone.  When no
// copy fits (large qubit counts), the sweep runs on psi and lambda only.
#include <algorithm>
#include <complex>
#include <cmath>
#include <map>
#include <vector>

#include "kt_complex.cuh"
#include "kt_internal.cuh"

namespace kt
{
int32_t expect_paulis(State& s, const kt_pauli* strings, int64_t n_strings, const double* coeffs, double* out_terms,
                      double* out_total);
}

namespace
{

using kt::KIND_ANTI;
using kt::KIND_DIAG;
using kt::KIND_GEN;

constexpr int ADJ_THREADS = 256;

struct HGroup
{
    uint64_t x;
    int32_t first;
    int32_t count;
};

struct HTerm
{
    uint64_t z;
    double wr, wi;  // c * phase * i^{#Y} * (-1)^{popcount(x & z)}
};

// lambda[j] = sum_groups sum_s w_s (-1)^{popcount(j & z_s)} psi[j ^ x], and
// each block's FP64 partial of Re <psi|lambda> (the energy) in
// epart[blockIdx.x].  A thread takes 4 consecutive outputs j0 .. j0 + 3
// (j0 a multiple of 4) at a time: one gather of the 4 partners per group, and
// per term one popcount of j0 & z (the low two bits of j0 are zero, so the
// 4 signs differ only by the parity of k & z for k < 4).  Groups and terms are
// staged in shared memory when they fit (`staged`).  lambda is formed in
// FP64 and stored in the state's precision; the energy uses the FP64 values.
template <typename C>
__global__ void __launch_bounds__(ADJ_THREADS) k_hsum(const C* __restrict__ psi, C* __restrict__ lam, uint64_t N,
                                                      const HGroup* __restrict__ groups, int n_groups,
                                                      const HTerm* __restrict__ terms, int n_terms, int staged,
                                                      double* __restrict__ epart)
{
    extern __shared__ __align__(16) unsigned char hs_raw[];
    __shared__ double red[ADJ_THREADS / 32];
    const HGroup* gp = groups;
    const HTerm* tp = terms;
    if (staged) {
        auto* sg = reinterpret_cast<HGroup*>(hs_raw);
        auto* st = reinterpret_cast<HTerm*>(hs_raw + ((static_cast<size_t>(n_groups) * sizeof(HGroup) + 15) & ~size_t {15}));
        for (int i = threadIdx.x; i < n_groups; i += blockDim.x) {
            sg[i] = groups[i];
        }
        for (int i = threadIdx.x; i < n_terms; i += blockDim.x) {
            st[i] = terms[i];
        }
        __syncthreads();
        gp = sg;
        tp = st;
    }
    double e = 0.0;
    const int kmax = N < 4 ? static_cast<int>(N) : 4;  // states of 1 or 2 amplitudes
    const uint64_t stride = 4ULL * gridDim.x * blockDim.x;
    for (uint64_t j0 = 4ULL * (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x); j0 < N; j0 += stride) {
        double ar[4] = {0.0, 0.0, 0.0, 0.0}, ai[4] = {0.0, 0.0, 0.0, 0.0};
        for (int g = 0; g < n_groups; ++g) {
            const HGroup gr = gp[g];
            double2 pv[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                pv[k] = k < kmax ? kt::to_d2(psi[(j0 + k) ^ gr.x]) : make_double2(0.0, 0.0);
            }
            double fr[4] = {0.0, 0.0, 0.0, 0.0}, fi[4] = {0.0, 0.0, 0.0, 0.0};
            for (int s = gr.first; s < gr.first + gr.count; ++s) {
                const HTerm t = tp[s];
                const int par = __popcll(j0 & t.z) & 1;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const bool neg = (par ^ (__popc(static_cast<unsigned>(k) & static_cast<unsigned>(t.z)) & 1)) != 0;
                    fr[k] += neg ? -t.wr : t.wr;
                    fi[k] += neg ? -t.wi : t.wi;
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                ar[k] += fr[k] * pv[k].x - fi[k] * pv[k].y;
                ai[k] += fr[k] * pv[k].y + fi[k] * pv[k].x;
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < kmax) {
                const double2 pj = kt::to_d2(psi[j0 + k]);
                e += pj.x * ar[k] + pj.y * ai[k];
                C o;
                o.x = ar[k];
                o.y = ai[k];
                lam[j0 + k] = o;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_down_sync(0xffffffffU, e, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = e;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < ADJ_THREADS / 32; ++w) {
            b += red[w];
        }
        epart[blockIdx.x] = b;
    }
}

// a *= (re + i im)
template <typename C>
__global__ void k_scale_state(C* __restrict__ a, uint64_t N, double re, double im)
{
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double2 v = kt::to_d2(a[i]);
        C o;
        o.x = v.x * re - v.y * im;
        o.y = v.x * im + v.y * re;
        a[i] = o;
    }
}

template <typename T>
struct M2
{
    T u[8];  // U^dagger, row-major interleaved
    T d[8];  // dU/dtheta, row-major interleaved (used when has_grad)
};

// One backward gate: psi, lambda <- U^dagger psi, U^dagger lambda; optional
// sum over pairs of conj(lambda_old) . (D psi_new), per block.
template <typename T, int KIND, bool CTRL, bool GRAD>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_gate(typename kt::CxT<T>::type* __restrict__ psi,
                                                          typename kt::CxT<T>::type* __restrict__ lam, uint64_t n_pairs,
                                                          int t, int c, int lo, int hi, M2<T> m, double* __restrict__ partial)
{
    using C = typename kt::CxT<T>::type;
    const uint64_t tb = uint64_t {1} << t;
    const C u00 = kt::make_cx<T>(m.u[0], m.u[1]), u01 = kt::make_cx<T>(m.u[2], m.u[3]);
    const C u10 = kt::make_cx<T>(m.u[4], m.u[5]), u11 = kt::make_cx<T>(m.u[6], m.u[7]);
    const C d00 = kt::make_cx<T>(m.d[0], m.d[1]), d01 = kt::make_cx<T>(m.d[2], m.d[3]);
    const C d10 = kt::make_cx<T>(m.d[4], m.d[5]), d11 = kt::make_cx<T>(m.d[6], m.d[7]);
    double acc = 0.0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_pairs; k += stride) {
        uint64_t i0;
        if (CTRL) {
            i0 = kt::insert_zero_bit(kt::insert_zero_bit(k, lo), hi) | (uint64_t {1} << c);
        } else {
            i0 = kt::insert_zero_bit(k, t);
        }
        const uint64_t i1 = i0 | tb;
        const C p0 = psi[i0], p1 = psi[i1];
        const C l0 = lam[i0], l1 = lam[i1];
        C q0, q1, m0, m1;
        if (KIND == KIND_GEN) {
            q0 = kt::cfma(u01, p1, kt::cmul(u00, p0));
            q1 = kt::cfma(u11, p1, kt::cmul(u10, p0));
            m0 = kt::cfma(u01, l1, kt::cmul(u00, l0));
            m1 = kt::cfma(u11, l1, kt::cmul(u10, l0));
        } else if (KIND == KIND_ANTI) {
            q0 = kt::cmul(u01, p1);
            q1 = kt::cmul(u10, p0);
            m0 = kt::cmul(u01, l1);
            m1 = kt::cmul(u10, l0);
        } else {
            q0 = kt::cmul(u00, p0);
            q1 = kt::cmul(u11, p1);
            m0 = kt::cmul(u00, l0);
            m1 = kt::cmul(u11, l1);
        }
        if (GRAD) {
            // D psi_new; D has the same sparsity class as U for every rotation
            C e0, e1;
            if (KIND == KIND_DIAG) {
                e0 = kt::cmul(d00, q0);
                e1 = kt::cmul(d11, q1);
            } else {
                e0 = kt::cfma(d01, q1, kt::cmul(d00, q0));
                e1 = kt::cfma(d11, q1, kt::cmul(d10, q0));
            }
            const double2 a0 = kt::to_d2(l0), a1 = kt::to_d2(l1);
            const double2 b0 = kt::to_d2(e0), b1 = kt::to_d2(e1);
            acc += a0.x * b0.x + a0.y * b0.y + a1.x * b1.x + a1.y * b1.y;  // Re conj(l) e
        }
        psi[i0] = q0;
        psi[i1] = q1;
        lam[i0] = m0;
        lam[i1] = m1;
    }
    if (GRAD) {
        __shared__ double sh[ADJ_THREADS / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffU, acc, o);
        }
        if ((threadIdx.x & 31) == 0) {
            sh[threadIdx.x >> 5] = acc;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < ADJ_THREADS / 32; ++w) {
                s += sh[w];
            }
            partial[blockIdx.x] = s;
        }
    }
}

__global__ void k_grad_finalize(const double* __restrict__ partial, int n_blocks, int n_rows, double* __restrict__ out)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) {
        return;
    }
    double s = 0.0;
    for (int b = 0; b < n_blocks; ++b) {
        s += partial[(size_t)r * n_blocks + b];
    }
    out[r] = 2.0 * s;
}

struct BGate
{
    kt::LGate adj;   // U^dagger (kind preserved)
    double d[8];     // dU/dtheta (the one-kernel-per-gate sweep)
    int32_t slot;    // parameter slot, -1 = no gradient
    int32_t gen;     // generator of the rotation (the fused sweep)
};

}  // namespace

struct kt_adjoint_s
{
    kt_sv sv {nullptr};
    kt::State* psi {nullptr};
    kt::State lam;
    int32_t checkpoint_every {0};
    std::vector<void*> checkpoints;
    std::vector<BGate> gates;
    int64_t n_params {0};
    std::vector<HGroup> hgroups;
    std::vector<HTerm> hterms;
    kt::DevBuf dev;     // partials and gradients of the backward sweep
    kt::DevBuf hdev;    // the Hamiltonian's groups and terms, the energy partials (forward)
    kt::DevBuf fused_work;  // plans and partials of the fused sweep
    bool forward_done {false};
    uint64_t last_structure {0};  // gate kinds, qubits and parameter slots of the previous forward
    int64_t repeats {0};          // consecutive forwards of that structure
};

namespace
{

int32_t invalid(const char* msg)
{
    kt::set_error(KT_ERR_INVALID, msg);
    return KT_ERR_INVALID;
}

void free_checkpoints(kt_adjoint_s* a)
{
    for (void* p : a->checkpoints) {
        cudaFree(p);
    }
    a->checkpoints.clear();
}

template <typename T>
int32_t launch_adj(kt::State& psi, kt::State& lam, const BGate& bg, double* partial, int blocks)
{
    using C = typename kt::CxT<T>::type;
    const kt::LGate& g = bg.adj;
    const int n = psi.n_bits;
    const bool ctrl = g.control >= 0;
    const uint64_t n_pairs = ctrl ? (uint64_t {1} << (n - 2)) : (uint64_t {1} << (n - 1));
    M2<T> m;
    for (int k = 0; k < 8; ++k) {
        m.u[k] = static_cast<T>(g.m[k]);
        m.d[k] = static_cast<T>(bg.d[k]);
    }
    const int t = g.target;
    const int c = ctrl ? g.control : 0;
    const int lo = ctrl ? std::min(c, t) : t;
    const int hi = ctrl ? std::max(c, t) : t;
    C* p = static_cast<C*>(psi.amps);
    C* l = static_cast<C*>(lam.amps);
    const bool grad = bg.slot >= 0;
#define KT_ADJ(KIND, CT, GR) \
    k_adj_gate<T, KIND, CT, GR><<<blocks, ADJ_THREADS, 0, psi.stream>>>(p, l, n_pairs, t, c, lo, hi, m, partial)
#define KT_ADJ_K(KIND)                                   \
    if (ctrl) {                                          \
        if (grad) KT_ADJ(KIND, true, true);              \
        else KT_ADJ(KIND, true, false);                  \
    } else {                                             \
        if (grad) KT_ADJ(KIND, false, true);             \
        else KT_ADJ(KIND, false, false);                 \
    }
    switch (g.kind) {
        case KIND_GEN: KT_ADJ_K(KIND_GEN); break;
        case KIND_ANTI: KT_ADJ_K(KIND_ANTI); break;
        default: KT_ADJ_K(KIND_DIAG); break;
    }
#undef KT_ADJ_K
#undef KT_ADJ
    KT_CHECK_LAUNCH("k_adj_gate");
    return KT_OK;
}

}  // namespace

extern "C" {

int32_t kt_adjoint_create(kt_sv sv, int32_t checkpoint_every, kt_adjoint* out)
{
    if (out == nullptr || sv == nullptr) {
        return invalid("null pointer");
    }
    *out = nullptr;
    auto* a = new kt_adjoint_s {};
    a->sv = sv;
    a->psi = &sv->st;
    a->checkpoint_every = std::max(0, checkpoint_every);
    a->lam.n_bits = a->psi->n_bits;
    a->lam.dtype = a->psi->dtype;
    a->lam.stream = a->psi->stream;
    const size_t bytes = a->psi->n_amps() * a->psi->amp_bytes();
    const cudaError_t e = cudaMalloc(&a->lam.amps, bytes);
    if (e != cudaSuccess) {
        delete a;
        return kt::cuda_fail(e, "cudaMalloc(lambda)");
    }
    a->lam.owned = true;
    *out = a;
    return KT_OK;
}

int32_t kt_adjoint_destroy(kt_adjoint a)
{
    if (a != nullptr) {
        free_checkpoints(a);
        if (a->lam.amps) {
            cudaFree(a->lam.amps);
        }
        a->lam.scratch.release();
        a->lam.scratch2.release();
        a->dev.release();
        a->hdev.release();
        a->fused_work.release();
        delete a;
    }
    return KT_OK;
}

int32_t kt_adjoint_forward(kt_adjoint a, const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params,
                           const kt_pauli* strings, int64_t n_strings, const double* coeffs, double* energy)
{
    try {
        if (a == nullptr || energy == nullptr) {
            return invalid("null pointer");
        }
        if (n_gates < 0 || (n_gates > 0 && gates == nullptr) || n_strings <= 0 || strings == nullptr) {
            return invalid("bad gate or Pauli arrays");
        }
        kt::State& psi = *a->psi;
        a->lam.stream = psi.stream;
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, psi.n_bits, lg); rc != KT_OK) {
            return rc;
        }
        // a forward of the structure this handle just ran (a training or VQE
        // loop) runs its fused blocks compiled, like the backward sweep
        // (adjoint_jit = 2 from the second call; 1 always), whatever the
        // state's size
        uint64_t sig = 0xcbf29ce484222325ULL ^ static_cast<uint64_t>(n_gates);
        for (int64_t i = 0; i < n_gates; ++i) {
            const uint64_t v = static_cast<uint64_t>(gates[i].op) | (static_cast<uint64_t>(gates[i].target) << 8) |
                               (static_cast<uint64_t>(gates[i].control) << 28) |
                               (static_cast<uint64_t>(gates[i].param >= 0 ? 1 : 0) << 48);
            sig = (sig ^ v) * 0x100000001b3ULL;
            sig ^= sig >> 29;
        }
        a->repeats = (sig == a->last_structure) ? a->repeats + 1 : 0;
        a->last_structure = sig;
        const int jmode = kt::tuning().adjoint_jit;
        psi.force_jit = jmode == 1 || (jmode == 2 && a->repeats >= 1);
        struct Reset
        {
            kt::State& s;
            ~Reset() { s.force_jit = false; }
        } reset_force {psi};
        // backward records: U^dagger and dU/dtheta
        a->gates.clear();
        a->gates.reserve(lg.size());
        for (int64_t i = 0; i < n_gates; ++i) {
            BGate b {};
            b.adj = lg[i];
            // U^dagger = conj transpose (kind is preserved)
            const double* m = lg[i].m;
            double* u = b.adj.m;
            u[0] = m[0]; u[1] = -m[1];
            u[2] = m[4]; u[3] = -m[5];
            u[4] = m[2]; u[5] = -m[3];
            u[6] = m[6]; u[7] = -m[7];
            b.adj.flags = (b.adj.kind == KIND_DIAG && u[0] == 1.0 && u[1] == 0.0) ? 1 : 0;
            b.slot = -1;
            const kt_gate& g = gates[i];
            if (g.param >= 0) {
                const double th = params[g.param];
                if (kt::gate_derivative(g.op, th, b.d)) {
                    b.slot = g.param;
                    b.gen = kt::gate_generator(g.op);
                }
            }
            a->gates.push_back(b);
        }
        a->n_params = n_params;
        // forward with optional checkpoints
        free_checkpoints(a);
        const int64_t k = a->checkpoint_every;
        if (k > 0 && n_gates > k) {
            const size_t bytes = psi.n_amps() * psi.amp_bytes();
            for (int64_t g0 = 0; g0 < n_gates; g0 += k) {
                const int64_t g1 = std::min<int64_t>(n_gates, g0 + k);
                std::vector<kt::LGate> seg(lg.begin() + g0, lg.begin() + g1);
                psi.last_launches = 0;
                psi.last_alg_bytes = 0.0;
                if (const int32_t rc = kt::apply_fused(psi, seg); rc != KT_OK) {
                    return rc;
                }
                if (g1 < n_gates) {
                    void* cp = nullptr;
                    if (cudaMalloc(&cp, bytes) != cudaSuccess) {
                        cudaGetLastError();  // no room: continue without further checkpoints
                        a->checkpoint_every = -1;
                    } else {
                        KT_CUDA(cudaMemcpyAsync(cp, psi.amps, bytes, cudaMemcpyDeviceToDevice, psi.stream));
                        a->checkpoints.push_back(cp);
                    }
                }
                if (a->checkpoint_every < 0) {
                    std::vector<kt::LGate> tail(lg.begin() + g1, lg.end());
                    if (const int32_t rc = kt::apply_fused(psi, tail); rc != KT_OK) {
                        return rc;
                    }
                    a->checkpoint_every = static_cast<int32_t>(k);
                    break;
                }
            }
        } else {
            psi.last_launches = 0;
            psi.last_alg_bytes = 0.0;
            if (const int32_t rc = kt::apply_fused(psi, lg); rc != KT_OK) {
                return rc;
            }
        }
        // H as X/Y-mask groups for lambda = H psi
        std::map<uint64_t, std::vector<int64_t>> groups;
        const uint64_t valid = (uint64_t {1} << psi.n_bits) - 1;
        for (int64_t s = 0; s < n_strings; ++s) {
            if ((strings[s].x_mask & ~valid) || (strings[s].z_mask & ~valid)) {
                return invalid("Pauli string acts on a qubit beyond the state");
            }
            groups[strings[s].x_mask].push_back(s);
        }
        a->hgroups.clear();
        a->hterms.clear();
        for (auto& [x, idx] : groups) {
            HGroup gr {x, static_cast<int32_t>(a->hterms.size()), static_cast<int32_t>(idx.size())};
            for (int64_t s : idx) {
                const uint64_t z = strings[s].z_mask;
                const int k4 = (__builtin_popcountll(x & z) + strings[s].phase) & 3;  // i^{#Y} * phase
                const double cr = coeffs ? coeffs[2 * s] : 1.0, ci = coeffs ? coeffs[2 * s + 1] : 0.0;
                double wr = cr, wi = ci;
                for (int r = 0; r < k4; ++r) {  // multiply by i
                    const double tr = -wi;
                    wi = wr;
                    wr = tr;
                }
                if (__builtin_popcountll(x & z) & 1) {
                    wr = -wr;
                    wi = -wi;
                }
                a->hterms.push_back({z, wr, wi});
            }
            a->hgroups.push_back(gr);
        }
        // lambda = H psi now (the backward starts from it) and the energy
        // Re <psi|lambda> from its FP64 values: one pass per X/Y-mask group
        kt::State& lam = a->lam;
        const uint64_t N = psi.n_amps();
        auto al = [](size_t v) { return (v + 255) & ~size_t {255}; };
        const size_t gbytes = a->hgroups.size() * sizeof(HGroup);
        const size_t tbytes = a->hterms.size() * sizeof(HTerm);
        const int hblocks = static_cast<int>(std::min<uint64_t>(std::max<uint64_t>(1, (N / 4 + ADJ_THREADS - 1) / ADJ_THREADS),
                                                                static_cast<uint64_t>(kt::sm_count()) * 8));
        const size_t off_t = al(gbytes);
        const size_t off_e = al(off_t + tbytes);
        if (const int32_t rc = a->hdev.reserve(al(off_e + static_cast<size_t>(hblocks) * sizeof(double))); rc != KT_OK) {
            return rc;
        }
        char* hb = static_cast<char*>(a->hdev.ptr);
        auto* d_groups = reinterpret_cast<HGroup*>(hb);
        auto* d_terms = reinterpret_cast<HTerm*>(hb + off_t);
        auto* d_epart = reinterpret_cast<double*>(hb + off_e);
        KT_CUDA(cudaMemcpyAsync(d_groups, a->hgroups.data(), gbytes, cudaMemcpyHostToDevice, psi.stream));
        KT_CUDA(cudaMemcpyAsync(d_terms, a->hterms.data(), tbytes, cudaMemcpyHostToDevice, psi.stream));
        const size_t staged_bytes = al(gbytes) + tbytes;
        const int staged = staged_bytes <= 48 * 1024 ? 1 : 0;
        const size_t hsmem = staged ? staged_bytes : 0;
        const int ng = static_cast<int>(a->hgroups.size());
        const int nt = static_cast<int>(a->hterms.size());
        if (psi.dtype == KT_C128) {
            k_hsum<double2><<<hblocks, ADJ_THREADS, hsmem, psi.stream>>>(static_cast<const double2*>(psi.amps),
                                                                         static_cast<double2*>(lam.amps), N, d_groups,
                                                                         ng, d_terms, nt, staged, d_epart);
        } else {
            k_hsum<float2><<<hblocks, ADJ_THREADS, hsmem, psi.stream>>>(static_cast<const float2*>(psi.amps),
                                                                        static_cast<float2*>(lam.amps), N, d_groups,
                                                                        ng, d_terms, nt, staged, d_epart);
        }
        KT_CHECK_LAUNCH("k_hsum");
        std::vector<double> ep(static_cast<size_t>(hblocks));
        if (const int32_t rc = kt::copy_d2h(ep.data(), d_epart, ep.size() * sizeof(double), psi.stream); rc != KT_OK) {
            return rc;
        }
        double total = 0.0;
        for (const double v : ep) {
            total += v;  // block order: the same bits on every call
        }
        *energy = total;
        a->forward_done = true;
        return KT_OK;
    } catch (const std::exception& e) {
        kt::set_error(KT_ERR_INVALID, e.what());
        return KT_ERR_INVALID;
    }
}

int32_t kt_adjoint_backward(kt_adjoint a, double* grad, int64_t n_params)
{
    try {
        if (a == nullptr || (n_params > 0 && grad == nullptr)) {
            return invalid("null pointer");
        }
        if (!a->forward_done) {
            return invalid("kt_adjoint_backward needs a kt_adjoint_forward first");
        }
        if (n_params < a->n_params) {
            return invalid("gradient buffer smaller than the parameter count of the forward pass");
        }
        kt::State& psi = *a->psi;
        kt::State& lam = a->lam;
        lam.stream = psi.stream;
        const uint64_t N = psi.n_amps();
        const int blocks = static_cast<int>(std::min<uint64_t>(
            std::max<uint64_t>(1, (N / 2 + ADJ_THREADS - 1) / ADJ_THREADS), static_cast<uint64_t>(kt::sm_count()) * 4));
        int n_grad = 0;
        for (const auto& b : a->gates) {
            n_grad += b.slot >= 0 ? 1 : 0;
        }
        auto al = [](size_t v) { return (v + 255) & ~size_t {255}; };
        const size_t off_part = 0;
        const size_t off_out = al(off_part + static_cast<size_t>(std::max(1, n_grad)) * blocks * sizeof(double));
        const size_t need = al(off_out + static_cast<size_t>(std::max(1, n_grad)) * sizeof(double));
        if (const int32_t rc = a->dev.reserve(need); rc != KT_OK) {
            return rc;
        }
        char* base = static_cast<char*>(a->dev.ptr);
        auto* d_part = reinterpret_cast<double*>(base + off_part);
        auto* d_out = reinterpret_cast<double*>(base + off_out);
        // lambda = H psi was formed by the forward pass
        // backward sweep
        const int64_t G = static_cast<int64_t>(a->gates.size());
        const int64_t k = a->checkpoint_every;
        const size_t bytes = N * psi.amp_bytes();
        std::vector<int32_t> row_slot;
        row_slot.reserve(n_grad);
        int row = n_grad;
        const int rb_fused = (psi.dtype == KT_C128) ? 3 : 4;
        if (kt::tuning().adjoint_fused != 0 && psi.n_bits >= rb_fused + 5) {
            // fused blocks per checkpoint segment, last segment first; rows in forward order
            std::vector<int32_t> row_of(static_cast<size_t>(G), -1);
            for (int64_t g = 0, r = 0; g < G; ++g) {
                if (a->gates[g].slot >= 0) {
                    row_of[g] = static_cast<int32_t>(r++);
                }
            }
            const int64_t seg = (k > 0) ? k : std::max<int64_t>(G, 1);
            const int64_t n_seg = (G + seg - 1) / seg;
            // Without checkpoints, an uncontrolled diagonal U^dagger with
            // |m00| = 1 (RZ, literal phases) runs one-sided, diag(1, m11 / m00),
            // on psi and lambda: every gradient term is bilinear in conj(lambda)
            // and psi, so the common unit factor m00 they both drop leaves it
            // unchanged, and half the amplitudes are touched.  psi gets the
            // product of the dropped factors back at the end.  (A checkpoint
            // restores psi alone, so with checkpoints every op keeps its form.)
            const bool one_sided = a->checkpoints.empty();
            std::complex<double> dropped(1.0, 0.0);
            for (int64_t j = n_seg - 1; j >= 0; --j) {
                const int64_t g0 = j * seg;
                const int64_t g1 = std::min<int64_t>(G, g0 + seg);
                if (j < n_seg - 1 && k > 0 && static_cast<size_t>(j) < a->checkpoints.size()) {
                    // psi is exactly the forward state after gates [0, g1)
                    KT_CUDA(cudaMemcpyAsync(psi.amps, a->checkpoints[j], bytes, cudaMemcpyDeviceToDevice, psi.stream));
                }
                std::vector<kt::AdjGate> sweep;
                sweep.reserve(static_cast<size_t>(g1 - g0));
                for (int64_t g = g1 - 1; g >= g0; --g) {
                    kt::AdjGate ag {};
                    ag.adj = a->gates[g].adj;
                    ag.gen = a->gates[g].gen;
                    ag.row = row_of[g];
                    if (one_sided && ag.adj.kind == KIND_DIAG && ag.adj.control < 0 && (ag.adj.flags & 1) == 0) {
                        const std::complex<double> m00(ag.adj.m[0], ag.adj.m[1]), m11(ag.adj.m[6], ag.adj.m[7]);
                        if (std::abs(std::norm(m00) - 1.0) < 1e-12) {
                            const std::complex<double> r = m11 * std::conj(m00);
                            ag.adj.m[0] = 1.0;
                            ag.adj.m[1] = 0.0;
                            ag.adj.m[6] = r.real();
                            ag.adj.m[7] = r.imag();
                            ag.adj.flags |= 1;
                            dropped *= m00;
                        }
                    }
                    sweep.push_back(ag);
                }
                if (const int32_t rc = kt::adjoint_sweep_fused(psi, lam, sweep, d_out, a->fused_work); rc != KT_OK) {
                    return rc;
                }
            }
            if (dropped != std::complex<double>(1.0, 0.0)) {
                const unsigned sb = static_cast<unsigned>(std::min<uint64_t>((N + ADJ_THREADS - 1) / ADJ_THREADS,
                                                                             static_cast<uint64_t>(kt::sm_count()) * 8));
                if (psi.dtype == KT_C128) {
                    k_scale_state<double2><<<sb, ADJ_THREADS, 0, psi.stream>>>(static_cast<double2*>(psi.amps), N,
                                                                             dropped.real(), dropped.imag());
                } else {
                    k_scale_state<float2><<<sb, ADJ_THREADS, 0, psi.stream>>>(static_cast<float2*>(psi.amps), N,
                                                                            dropped.real(), dropped.imag());
                }
                KT_CHECK_LAUNCH("k_scale_state");
            }
            std::vector<double> rows_f(static_cast<size_t>(std::max(1, n_grad)));
            if (n_grad > 0) {
                if (const int32_t rc = kt::copy_d2h(rows_f.data(), d_out, n_grad * sizeof(double), psi.stream);
                    rc != KT_OK) {
                    return rc;
                }
            } else {
                KT_CUDA(cudaStreamSynchronize(psi.stream));
            }
            std::fill(grad, grad + n_params, 0.0);
            int rr = 0;
            for (const auto& bg : a->gates) {
                if (bg.slot >= 0) {
                    grad[bg.slot] += rows_f[rr++];
                }
            }
            a->forward_done = false;
            return KT_OK;
        }
        for (int64_t g = G - 1; g >= 0; --g) {
            const BGate& bg = a->gates[g];
            double* part = nullptr;
            if (bg.slot >= 0) {
                --row;
                part = d_part + static_cast<size_t>(row) * blocks;
            }
            const int32_t rc = (psi.dtype == KT_C128) ? launch_adj<double>(psi, lam, bg, part, blocks)
                                                      : launch_adj<float>(psi, lam, bg, part, blocks);
            if (rc != KT_OK) {
                return rc;
            }
            // psi now holds the state after gates [0, g); restore it exactly from a checkpoint
            if (k > 0 && g > 0 && g % k == 0) {
                const size_t ci = static_cast<size_t>(g / k - 1);
                if (ci < a->checkpoints.size()) {
                    KT_CUDA(cudaMemcpyAsync(psi.amps, a->checkpoints[ci], bytes, cudaMemcpyDeviceToDevice, psi.stream));
                }
            }
        }
        std::vector<double> rows(static_cast<size_t>(std::max(1, n_grad)));
        if (n_grad > 0) {
            k_grad_finalize<<<(n_grad + 127) / 128, 128, 0, psi.stream>>>(d_part, blocks, n_grad, d_out);
            KT_CHECK_LAUNCH("k_grad_finalize");
            if (const int32_t rc = kt::copy_d2h(rows.data(), d_out, n_grad * sizeof(double), psi.stream); rc != KT_OK) {
                return rc;
            }
        } else {
            KT_CUDA(cudaStreamSynchronize(psi.stream));
        }
        std::fill(grad, grad + n_params, 0.0);
        int r = 0;
        for (const auto& bg : a->gates) {
            if (bg.slot >= 0) {
                grad[bg.slot] += rows[r++];
            }
        }
        a->forward_done = false;  // psi has been un-applied back to the initial state
        return KT_OK;
    } catch (const std::exception& e) {
        kt::set_error(KT_ERR_INVALID, e.what());
        return KT_ERR_INVALID;
    }
}

}  // extern "C"
