// kt_state_ops.cu — statevector and density-matrix operations of kettle's
// public API beside propagation:
//
//  * kt_sv_tensor_product: |left> (x) |right>, the left state's qubits the low
//    ones: out[i_l + i_r 2^n_l] = left[i_l] right[i_r] (state/state.cpp:144-157);
//  * kt_sv_diagonal_expectation: sum_i conj(psi_i) lambda_i psi_i for a
//    diagonal operator given by its 2^n eigenvalues (state/state.cpp:174-188),
//    FP64 block partials added on the host in block order;
//  * kt_sample_probabilities: shots from a caller's probability vector
//    through the same certified / exact CDF sampler as kt_sv_sample
//    (calculations/measurements.cpp:58-159);
//  * kt_dm_measure_probs / kt_dm_collapse: an M gate on a density matrix
//    (simulation/measure_density_matrix.cpp:22-105).  The reference's
//    probabilities are P(b) = sum |rho(r, c)|^2 over the rows and columns
//    whose measured bit is b; the outcome o keeps the (o, o) block scaled by
//    the caller's factor (the reference passes sqrt(1 / P(o))) and clears the
//    other three blocks.
#include <algorithm>
#include <vector>

#include "kt_complex.cuh"
#include "kt_internal.cuh"

namespace kt
{
int32_t sample_from_probabilities(State& s, const double* host_probs, uint64_t n, const double* canonicals,
                                  int64_t n_shots, uint64_t* out, int32_t mode, int32_t* n_rescanned);
}  // namespace kt

namespace
{

using kt::to_d2;

constexpr int SO_THREADS = 256;

template <typename C>
__device__ __forceinline__ C from_d2(double2 v);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 v)
{
    return v;
}
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 v)
{
    return make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
}

template <typename C>
__global__ void k_sv_tensor_product(const C* __restrict__ left, int nl, const C* __restrict__ right,
                                    C* __restrict__ out, uint64_t N)
{
    const uint64_t lmask = (uint64_t {1} << nl) - 1;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < N;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double2 a = to_d2(left[i & lmask]);
        const double2 b = to_d2(right[i >> nl]);
        out[i] = from_d2<C>(make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x));
    }
}

// per block: sum_i conj(psi_i) lambda_i psi_i (FP64), two doubles per block
template <typename C>
__global__ void __launch_bounds__(SO_THREADS) k_sv_diag_expect(const C* __restrict__ psi,
                                                               const double2* __restrict__ lam, uint64_t N,
                                                               double* __restrict__ partial)
{
    double re = 0.0;
    double im = 0.0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < N;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double2 p = to_d2(psi[i]);
        const double2 l = lam[i];
        // (conj(p) * l) * p, in the reference's order
        const double tr = p.x * l.x + p.y * l.y;
        const double ti = p.x * l.y - p.y * l.x;
        re += tr * p.x - ti * p.y;
        im += tr * p.y + ti * p.x;
    }
    __shared__ double sh[2][SO_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffU, re, o);
        im += __shfl_down_sync(0xffffffffU, im, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = re;
        sh[1][threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < SO_THREADS / 32; ++w) {
            a += sh[0][w];
            b += sh[1][w];
        }
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
    }
}

// per block: sum |rho(r, c)|^2 over bit q of r = bit q of c = 0, and = 1
template <typename C>
__global__ void __launch_bounds__(SO_THREADS) k_dm_block_norms(const C* __restrict__ rho, int n, int q, double* __restrict__ partial)
{
    const uint64_t N2 = uint64_t {1} << (2 * n);
    double p0 = 0.0;
    double p1 = 0.0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < N2;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t br = (i >> q) & 1U;
        const uint64_t bc = (i >> (q + n)) & 1U;
        if (br != bc) {
            continue;
        }
        const double2 v = to_d2(rho[i]);
        const double nrm = __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));  // std::norm, no contraction
        if (br == 0) {
            p0 += nrm;
        } else {
            p1 += nrm;
        }
    }
    __shared__ double sh[2][SO_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p0 += __shfl_down_sync(0xffffffffU, p0, o);
        p1 += __shfl_down_sync(0xffffffffU, p1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = p0;
        sh[1][threadIdx.x >> 5] = p1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < SO_THREADS / 32; ++w) {
            a += sh[0][w];
            b += sh[1][w];
        }
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
    }
}

template <typename C>
__global__ void k_dm_collapse(C* __restrict__ rho, int n, int q, int outcome, double scale)
{
    const uint64_t N2 = uint64_t {1} << (2 * n);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < N2;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int br = static_cast<int>((i >> q) & 1U);
        const int bc = static_cast<int>((i >> (q + n)) & 1U);
        if (br == bc && br == outcome) {
            const double2 v = to_d2(rho[i]);
            rho[i] = from_d2<C>(make_double2(v.x * scale, v.y * scale));
        } else {
            rho[i] = from_d2<C>(make_double2(0.0, 0.0));
        }
    }
}

unsigned grid_for(uint64_t n)
{
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((n + SO_THREADS - 1) / SO_THREADS,
                                                                           static_cast<uint64_t>(kt::sm_count()) * 8)));
}

int32_t fail(int32_t code, const char* msg)
{
    kt::set_error(code, msg);
    return code;
}

template <typename F>
int32_t guarded(F&& f)
{
    try {
        const int32_t rc = f();
        return rc == KT_OK ? kt::jit_async_error() : rc;
    } catch (const std::bad_alloc&) {
        return fail(KT_ERR_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        kt::set_error(KT_ERR_INVALID, e.what());
        return KT_ERR_INVALID;
    } catch (...) {
        return fail(KT_ERR_INVALID, "unknown exception");
    }
}

// FP64 block partials (two per block) summed on the host in block order
int32_t reduce_pairs(kt::State& s, unsigned blocks, double* out)
{
    std::vector<double> h(2 * static_cast<size_t>(blocks));
    KT_CUDA(cudaMemcpyAsync(h.data(), s.scratch.ptr, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    KT_CUDA(cudaStreamSynchronize(s.stream));
    double a = 0.0, b = 0.0;
    for (unsigned k = 0; k < blocks; ++k) {
        a += h[2 * k];
        b += h[2 * k + 1];
    }
    out[0] = a;
    out[1] = b;
    return KT_OK;
}

}  // namespace

extern "C" {

int32_t kt_sv_tensor_product(kt_sv left, kt_sv right, kt_sv out)
{
    return guarded([&]() -> int32_t {
        if (left == nullptr || right == nullptr || out == nullptr) {
            return fail(KT_ERR_INVALID, "null handle");
        }
        const kt::State& L = left->st;
        const kt::State& R = right->st;
        kt::State& O = out->st;
        if (L.dtype != R.dtype || L.dtype != O.dtype) {
            return fail(KT_ERR_INVALID, "kt_sv_tensor_product: the three states must have the same dtype");
        }
        if (O.n_bits != L.n_bits + R.n_bits) {
            return fail(KT_ERR_QUBITS, "kt_sv_tensor_product: the output must have the qubits of both inputs");
        }
        // the inputs' pending work is ordered before the product on the output's stream
        cudaEvent_t ev[2] = {nullptr, nullptr};
        for (int k = 0; k < 2; ++k) {
            KT_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
            KT_CUDA(cudaEventRecord(ev[k], k == 0 ? L.stream : R.stream));
            KT_CUDA(cudaStreamWaitEvent(O.stream, ev[k], 0));
            KT_CUDA(cudaEventDestroy(ev[k]));
        }
        const uint64_t N = O.n_amps();
        if (O.dtype == KT_C128) {
            k_sv_tensor_product<double2><<<grid_for(N), SO_THREADS, 0, O.stream>>>(
                static_cast<const double2*>(L.amps), L.n_bits, static_cast<const double2*>(R.amps),
                static_cast<double2*>(O.amps), N);
        } else {
            k_sv_tensor_product<float2><<<grid_for(N), SO_THREADS, 0, O.stream>>>(
                static_cast<const float2*>(L.amps), L.n_bits, static_cast<const float2*>(R.amps),
                static_cast<float2*>(O.amps), N);
        }
        KT_CHECK_LAUNCH("k_sv_tensor_product");
        return KT_OK;
    });
}

int32_t kt_sv_diagonal_expectation(kt_sv sv, const double* eigenvalues, double* out_re_im)
{
    return guarded([&]() -> int32_t {
        if (sv == nullptr || eigenvalues == nullptr || out_re_im == nullptr) {
            return fail(KT_ERR_INVALID, "null pointer");
        }
        kt::State& s = sv->st;
        const uint64_t N = s.n_amps();
        const unsigned blocks = grid_for(N);
        if (const int32_t rc = s.scratch.reserve(2 * static_cast<size_t>(blocks) * sizeof(double)); rc != KT_OK) {
            return rc;
        }
        if (const int32_t rc = s.scratch2.reserve(N * sizeof(double2)); rc != KT_OK) {
            return rc;
        }
        KT_CUDA(cudaMemcpyAsync(s.scratch2.ptr, eigenvalues, N * sizeof(double2), cudaMemcpyHostToDevice, s.stream));
        auto* part = static_cast<double*>(s.scratch.ptr);
        const auto* lam = static_cast<const double2*>(s.scratch2.ptr);
        if (s.dtype == KT_C128) {
            k_sv_diag_expect<double2><<<blocks, SO_THREADS, 0, s.stream>>>(static_cast<const double2*>(s.amps), lam, N, part);
        } else {
            k_sv_diag_expect<float2><<<blocks, SO_THREADS, 0, s.stream>>>(static_cast<const float2*>(s.amps), lam, N, part);
        }
        KT_CHECK_LAUNCH("k_sv_diag_expect");
        return reduce_pairs(s, blocks, out_re_im);
    });
}

int32_t kt_sample_probabilities(const double* probabilities, uint64_t n, const double* canonicals, int64_t n_shots,
                                uint64_t* out_indices, int32_t mode, void* stream)
{
    return guarded([&]() -> int32_t {
        if (n == 0 || probabilities == nullptr) {
            return fail(KT_ERR_INVALID, "kt_sample_probabilities: empty probability vector");
        }
        if (n_shots < 0 || (n_shots > 0 && (canonicals == nullptr || out_indices == nullptr))) {
            return fail(KT_ERR_INVALID, "bad shot buffers");
        }
        kt::State s;
        s.stream = static_cast<cudaStream_t>(stream);
        const int32_t rc = kt::sample_from_probabilities(s, probabilities, n, canonicals, n_shots, out_indices, mode,
                                                         nullptr);
        s.scratch.release();
        s.scratch2.release();
        return rc;
    });
}

int32_t kt_dm_measure_probs(kt_dm dm, uint32_t qubit, double* p0, double* p1)
{
    return guarded([&]() -> int32_t {
        if (dm == nullptr || p0 == nullptr || p1 == nullptr) {
            return fail(KT_ERR_INVALID, "null pointer");
        }
        if (qubit >= static_cast<uint32_t>(dm->n)) {
            return fail(KT_ERR_INVALID, "measured qubit out of range");
        }
        kt::State& s = dm->st;
        const unsigned blocks = grid_for(s.n_amps());
        if (const int32_t rc = s.scratch.reserve(2 * static_cast<size_t>(blocks) * sizeof(double)); rc != KT_OK) {
            return rc;
        }
        auto* part = static_cast<double*>(s.scratch.ptr);
        if (s.dtype == KT_C128) {
            k_dm_block_norms<double2><<<blocks, SO_THREADS, 0, s.stream>>>(static_cast<const double2*>(s.amps), dm->n,
                                                                          static_cast<int>(qubit), part);
        } else {
            k_dm_block_norms<float2><<<blocks, SO_THREADS, 0, s.stream>>>(static_cast<const float2*>(s.amps), dm->n,
                                                                         static_cast<int>(qubit), part);
        }
        KT_CHECK_LAUNCH("k_dm_block_norms");
        double r[2];
        if (const int32_t rc = reduce_pairs(s, blocks, r); rc != KT_OK) {
            return rc;
        }
        *p0 = r[0];
        *p1 = r[1];
        return KT_OK;
    });
}

int32_t kt_dm_collapse(kt_dm dm, uint32_t qubit, int32_t outcome, double scale)
{
    return guarded([&]() -> int32_t {
        if (dm == nullptr) {
            return fail(KT_ERR_INVALID, "null handle");
        }
        if (qubit >= static_cast<uint32_t>(dm->n) || (outcome != 0 && outcome != 1)) {
            return fail(KT_ERR_INVALID, "kt_dm_collapse: qubit out of range or outcome not 0 / 1");
        }
        kt::State& s = dm->st;
        const unsigned blocks = grid_for(s.n_amps());
        if (s.dtype == KT_C128) {
            k_dm_collapse<double2><<<blocks, SO_THREADS, 0, s.stream>>>(static_cast<double2*>(s.amps), dm->n,
                                                                       static_cast<int>(qubit), outcome, scale);
        } else {
            k_dm_collapse<float2><<<blocks, SO_THREADS, 0, s.stream>>>(static_cast<float2*>(s.amps), dm->n,
                                                                      static_cast<int>(qubit), outcome, scale);
        }
        KT_CHECK_LAUNCH("k_dm_collapse");
        return KT_OK;
    });
}

}  // extern "C"
