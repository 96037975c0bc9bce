// kt_sample.cu — inverse-CDF shot sampling, bit-exact to the reference.
//
// The reference (calculations/measurements.cpp:235-311) builds the CDF with a
// sequential std::partial_sum, draws u = c * (last - offset) + 0.0 from a
// canonical c, and takes lower_bound(cdf, u).  A parallel prefix sum rounds
// differently, so the device works in two tiers:
//
//  fast: chunk sums (FP64, any order) -> chunk offsets E_b (one block, made
//        exactly monotone with a max fix-up) -> per shot, a binary search over
//        E and a sequential scan inside the chunk from E_b.  Every value v used
//        differs from the sequential CDF by at most
//            delta = (N + 1024) * 2^-53 * total * 1.01
//        (error bound of any summation order of non-negative terms), so a shot
//        whose u lies further than 2*delta + (slack for the bound on u) from
//        both neighbouring values has provably the same lower_bound index as
//        the reference.  The bound (last - offset) is certified the same way.
//  exact: if any shot (or the bound) is not certified, one thread recomputes
//        the sequential CDF exactly as std::partial_sum does, and every shot is
//        re-searched with the reference's own arithmetic.
//
// Probabilities use __dmul_rn / __dadd_rn: no FMA, as std::norm compiles
// without contraction.
#include <algorithm>
#include <cmath>

#include "kt_complex.cuh"
#include "kt_internal.cuh"

namespace kt
{

int32_t device_probabilities(State& s, const double* noise, double* dev_p);

namespace
{

constexpr int CHUNK = 1024;  // elements per chunk (power of two)

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_down_sync(0xffffffffU, v, o);
    }
    return v;
}

// one warp per chunk
__global__ void k_chunk_sums(const double* __restrict__ p, uint64_t N, uint64_t n_chunks, double* __restrict__ sums,
                             unsigned long long* __restrict__ last_nz)
{
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n_chunks) {
        return;
    }
    const uint64_t beg = warp * CHUNK;
    const uint64_t end = beg + CHUNK < N ? beg + CHUNK : N;
    double acc = 0.0;
    unsigned long long nz = 0;
    bool any = false;
    for (uint64_t i = beg + lane; i < end; i += 32) {
        const double v = p[i];
        acc += v;
        if (v > 0.0) {
            nz = i;
            any = true;
        }
    }
    acc = warp_sum_d(acc);
    if (lane == 0) {
        sums[warp] = acc;
    }
    if (any) {
        atomicMax(last_nz, nz + 1);  // store index + 1 (0 = none)
    }
}

// Exclusive offsets E[0..n_chunks] of the chunk sums, single block.  Each
// thread scans a contiguous run sequentially; runs are joined by a block scan
// and finally made exactly non-decreasing with a prefix max.
__global__ void k_chunk_offsets(const double* __restrict__ sums, uint64_t n_chunks, double* __restrict__ E)
{
    __shared__ double sh_tot[1024];
    __shared__ double sh_last[1024];
    const int t = threadIdx.x;
    const int T = blockDim.x;
    const uint64_t per = (n_chunks + T - 1) / T;
    const uint64_t beg = (uint64_t)t * per;
    const uint64_t end = beg + per < n_chunks ? beg + per : n_chunks;
    double tot = 0.0;
    for (uint64_t b = beg; b < end; ++b) {
        tot += sums[b];
    }
    sh_tot[t] = tot;
    __syncthreads();
    if (t == 0) {
        double run = 0.0;
        for (int k = 0; k < T; ++k) {
            const double v = sh_tot[k];
            sh_tot[k] = run;
            run += v;
        }
    }
    __syncthreads();
    double run = sh_tot[t];
    for (uint64_t b = beg; b < end; ++b) {
        E[b] = run;
        run += sums[b];
    }
    sh_last[t] = run;
    __syncthreads();
    if (t == 0) {
        double m = 0.0;
        for (int k = 0; k < T; ++k) {
            const double v = sh_last[k];
            sh_last[k] = m;  // max of everything before run k
            m = v > m ? v : m;
        }
        E[n_chunks] = m;
    }
    __syncthreads();
    const double before = sh_last[t];
    double m = before;
    for (uint64_t b = beg; b < end; ++b) {
        m = E[b] > m ? E[b] : m;
        E[b] = m;
    }
    __syncthreads();
    if (t == 0) {
        // the total must not sit below the last offset
        const double lastE = n_chunks > 0 ? E[n_chunks - 1] : 0.0;
        if (E[n_chunks] < lastE) {
            E[n_chunks] = lastE;
        }
    }
}

// approximate CDF value at index i (sequential from its chunk offset)
__device__ double approx_cdf(const double* __restrict__ p, const double* __restrict__ E, uint64_t i)
{
    const uint64_t b = i / CHUNK;
    double c = E[b];
    for (uint64_t j = b * CHUNK; j <= i; ++j) {
        c = c + p[j];
    }
    return c;
}

struct SampleInfo
{
    double total;     // E[n_chunks]
    double bound;     // last - offset (approximate)
    double margin;    // certification margin on u and on cdf values
    int32_t bound_ok; // bound certified
    int32_t pad;
};

__global__ void k_sample_bound(const double* __restrict__ p, const double* __restrict__ E, uint64_t N, uint64_t n_chunks,
                               const unsigned long long* __restrict__ last_nz, SampleInfo* __restrict__ info)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    const double total = E[n_chunks];
    const double delta = (static_cast<double>(N) + 1024.0) * 1.1102230246251565e-16 * total * 1.01;
    const unsigned long long jnz = *last_nz;  // index + 1 of the last p > 0
    double second = 0.0;
    int ok = 1;
    if (jnz >= 2) {
        const uint64_t js = jnz - 1;
        // the last element strictly below `last` in the sequential CDF is
        // cdf[js - 1] provided p[js] is not swallowed by rounding there
        if (!(p[js] > 8.0 * delta)) {
            ok = 0;
        }
        second = approx_cdf(p, E, js - 1);
    } else {
        second = 0.0;  // a single non-zero entry (or none): nothing strictly below in [0, js)
        if (jnz == 0) {
            ok = 0;
        }
    }
    const double last = total;
    const double offset = (last - second) * 1.0e-4;
    const double bound = last - offset;
    info->total = total;
    info->bound = bound;
    // |bound - bound_seq| <= delta (last) + 1e-4 * 2 delta (offset) + rounding
    info->margin = 2.0 * delta + 1.0e-4 * 2.0 * delta + 4.0 * 2.220446049250313e-16 * total;
    info->bound_ok = ok;
}

__global__ void k_sample_fast(const double* __restrict__ p, const double* __restrict__ E, uint64_t N, uint64_t n_chunks,
                              const SampleInfo* __restrict__ info, const double* __restrict__ canon, int64_t n_shots,
                              uint64_t* __restrict__ out, int* __restrict__ uncertified)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) {
        return;
    }
    const SampleInfo inf = *info;
    const double u = __dadd_rn(__dmul_rn(canon[s], __dsub_rn(inf.bound, 0.0)), 0.0);
    const double m = inf.margin;
    // chunk b with E[b] < u <= E[b+1]
    uint64_t lo = 0, len = n_chunks;
    while (len > 0) {
        const uint64_t half = len / 2;
        if (E[lo + half + 1] < u) {
            lo = lo + half + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    const uint64_t b = lo < n_chunks ? lo : n_chunks - 1;
    double prev = E[b];
    double c = prev;
    uint64_t idx = N;
    const uint64_t end = (b + 1) * CHUNK < N ? (b + 1) * CHUNK : N;
    for (uint64_t j = b * CHUNK; j < end; ++j) {
        c = c + p[j];
        if (c >= u) {
            idx = j;
            break;
        }
        prev = c;
    }
    bool ok = inf.bound_ok != 0 && idx < N;
    if (ok) {
        // value at idx comfortably >= u, value before idx comfortably < u
        ok = (c - m > u + m) && (idx == 0 || prev + m < u - m);
        if (idx == b * CHUNK && idx != 0) {
            // previous value is the end of the previous chunk: E[b] approximates it
            ok = ok && (E[b] + m < u - m);
        }
    }
    out[s] = idx < N ? idx : N - 1;
    if (!ok) {
        atomicAdd(uncertified, 1);
    }
}

// exact tier -------------------------------------------------------------------
// std::partial_sum: cdf[0] = p[0]; cdf[i] = cdf[i-1] + p[i] (one thread).
__global__ void k_seq_cdf(const double* __restrict__ p, uint64_t N, double* __restrict__ cdf)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    double acc = p[0];
    cdf[0] = acc;
    for (uint64_t i = 1; i < N; ++i) {
        acc = __dadd_rn(acc, p[i]);
        cdf[i] = acc;
    }
}

// cumulative_end_offset_ (measurements.cpp:235-256) and the distribution bound
__global__ void k_seq_bound(const double* __restrict__ cdf, uint64_t N, double* __restrict__ bound)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    const double last = cdf[N - 1];
    double second = 0.0;
    for (uint64_t i = N - 1; i > 0; --i) {
        if (cdf[i - 1] < last) {
            second = cdf[i - 1];
            break;
        }
    }
    const double offset = __dmul_rn(__dsub_rn(last, second), 1.0e-4);
    *bound = __dsub_rn(last, offset);
}

__global__ void k_seq_search(const double* __restrict__ cdf, uint64_t N, const double* __restrict__ bound,
                             const double* __restrict__ canon, int64_t n_shots, uint64_t* __restrict__ out)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) {
        return;
    }
    const double u = __dadd_rn(__dmul_rn(canon[s], __dsub_rn(*bound, 0.0)), 0.0);
    uint64_t lo = 0, len = N;
    while (len > 0) {
        const uint64_t half = len / 2;
        if (cdf[lo + half] < u) {
            lo = lo + half + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    out[s] = lo < N ? lo : N - 1;
}

}  // namespace

int32_t sample(State& s, const double* noise, const double* canonicals, int64_t n_shots, uint64_t* out, int32_t mode,
               int32_t* n_rescanned)
{
    if (n_rescanned) {
        *n_rescanned = 0;
    }
    if (n_shots <= 0) {
        return KT_OK;
    }
    const uint64_t N = s.n_amps();
    const uint64_t n_chunks = (N + CHUNK - 1) / CHUNK;
    auto al = [](size_t v) { return (v + 255) & ~size_t {255}; };
    const size_t ns = static_cast<size_t>(n_shots);
    // scratch2: probabilities (N) ; scratch: everything else
    if (const int32_t rc = s.scratch2.reserve(al(N * 8) + al(N * 8)); rc != KT_OK) {
        return rc;
    }
    const size_t off_sums = 0;
    const size_t off_E = al(off_sums + n_chunks * 8);
    const size_t off_nz = al(off_E + (n_chunks + 1) * 8);
    const size_t off_info = al(off_nz + 8);
    const size_t off_canon = al(off_info + sizeof(SampleInfo));
    const size_t off_out = al(off_canon + ns * 8);
    const size_t off_unc = al(off_out + ns * 8);
    const size_t off_bound = al(off_unc + 8);
    if (const int32_t rc = s.scratch.reserve(off_bound + 8); rc != KT_OK) {
        return rc;
    }
    double* dp = static_cast<double*>(s.scratch2.ptr);
    double* dcdf = reinterpret_cast<double*>(static_cast<char*>(s.scratch2.ptr) + al(N * 8));
    char* base = static_cast<char*>(s.scratch.ptr);
    auto* d_sums = reinterpret_cast<double*>(base + off_sums);
    auto* d_E = reinterpret_cast<double*>(base + off_E);
    auto* d_nz = reinterpret_cast<unsigned long long*>(base + off_nz);
    auto* d_info = reinterpret_cast<SampleInfo*>(base + off_info);
    auto* d_canon = reinterpret_cast<double*>(base + off_canon);
    auto* d_out = reinterpret_cast<uint64_t*>(base + off_out);
    auto* d_unc = reinterpret_cast<int*>(base + off_unc);
    auto* d_bound = reinterpret_cast<double*>(base + off_bound);

    if (const int32_t rc = device_probabilities(s, noise, dp); rc != KT_OK) {
        return rc;
    }
    if (const int32_t rc = copy_h2d(d_canon, canonicals, ns * 8, s.stream); rc != KT_OK) {
        return rc;
    }
    int unc = 0;
    if (mode == 0) {
        KT_CUDA(cudaMemsetAsync(d_nz, 0, 8, s.stream));
        KT_CUDA(cudaMemsetAsync(d_unc, 0, 4, s.stream));
        const uint64_t threads = n_chunks * 32;
        k_chunk_sums<<<static_cast<unsigned>((threads + 255) / 256), 256, 0, s.stream>>>(dp, N, n_chunks, d_sums, d_nz);
        KT_CHECK_LAUNCH("k_chunk_sums");
        k_chunk_offsets<<<1, 1024, 0, s.stream>>>(d_sums, n_chunks, d_E);
        KT_CHECK_LAUNCH("k_chunk_offsets");
        k_sample_bound<<<1, 32, 0, s.stream>>>(dp, d_E, N, n_chunks, d_nz, d_info);
        KT_CHECK_LAUNCH("k_sample_bound");
        k_sample_fast<<<static_cast<unsigned>((ns + 127) / 128), 128, 0, s.stream>>>(dp, d_E, N, n_chunks, d_info,
                                                                                       d_canon, n_shots, d_out, d_unc);
        KT_CHECK_LAUNCH("k_sample_fast");
        if (const int32_t rc = copy_d2h(&unc, d_unc, 4, s.stream); rc != KT_OK) {
            return rc;
        }
    }
    if (mode != 0 || unc != 0) {
        k_seq_cdf<<<1, 32, 0, s.stream>>>(dp, N, dcdf);
        KT_CHECK_LAUNCH("k_seq_cdf");
        k_seq_bound<<<1, 32, 0, s.stream>>>(dcdf, N, d_bound);
        KT_CHECK_LAUNCH("k_seq_bound");
        k_seq_search<<<static_cast<unsigned>((ns + 127) / 128), 128, 0, s.stream>>>(dcdf, N, d_bound, d_canon, n_shots,
                                                                                     d_out);
        KT_CHECK_LAUNCH("k_seq_search");
        if (n_rescanned) {
            *n_rescanned = 1;
        }
    }
    return copy_d2h(out, d_out, ns * 8, s.stream);
}

}  // namespace kt
