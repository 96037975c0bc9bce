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
// The sequential sum s_i = fl(s_{i-1} + p_i) of std::partial_sum, computed
// exactly by one block.  While s stays in one binade [2^E, 2^(E+1)) every
// representable value is a multiple of u = 2^(E-52), so (no tie, no binade
// exit) fl(s + p) = s + rint(p / u) * u exactly: a run of additions is an
// integer prefix sum, which the block computes in parallel (uint64 units).
// An element whose p/u is an exact tie (.5), is large (>= 2^50 units), or
// whose running sum leaves the binade is added with one IEEE add instead,
// after which the block continues from the new (exact) s.  Each 8192-element
// tile costs one block scan, plus one round per such element.
constexpr int XS_THREADS = 1024;
constexpr int XS_EPT = 16;
constexpr int XS_TILE = XS_THREADS * XS_EPT;

__device__ __forceinline__ unsigned long long block_excl_scan_u64(unsigned long long v, unsigned long long* sh,
                                                                  unsigned long long& total)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffU, x, o);
        if (lane >= o) {
            x += y;
        }
    }
    if (lane == 31) {
        sh[warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = (lane < XS_THREADS / 32) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffU, w, o);
            if (lane >= o) {
                w += y;
            }
        }
        sh[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    total = sh[XS_THREADS / 32 - 1];
    const unsigned long long before = (warp > 0) ? sh[warp - 1] : 0ULL;
    const unsigned long long r = before + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(XS_THREADS) k_exact_cdf(const double* __restrict__ p, uint64_t N, double* __restrict__ cdf)
{
    __shared__ unsigned long long sh[32];
    __shared__ double s_sh;
    __shared__ unsigned long long i_sh;
    __shared__ unsigned int viol_sh;
    const int t = threadIdx.x;
    if (t == 0) {
        s_sh = p[0];
        cdf[0] = p[0];
        i_sh = 1;
    }
    __syncthreads();
    constexpr unsigned long long TWO53 = 1ULL << 53;
    while (true) {
        const uint64_t i = i_sh;
        const double s = s_sh;
        if (i >= N) {
            break;
        }
        if (s < 0x1p-900) {
            // zero or tiny running value (subnormal spacing, huge 1/ulp): plain IEEE steps
            if (t == 0) {
                const double nv = __dadd_rn(s, p[i]);
                s_sh = nv;
                cdf[i] = nv;
                i_sh = i + 1;
            }
            __syncthreads();
            continue;
        }
        int E;
        frexp(s, &E);                       // s in [2^(E-1), 2^E)
        const double inv_u = ldexp(1.0, 53 - E);  // 1 / ulp(s)
        const double u = ldexp(1.0, E - 53);
        const unsigned long long m = static_cast<unsigned long long>(s * inv_u);  // exact, in [2^52, 2^53)
        // this thread's elements: i + t*EPT + k
        unsigned long long r[XS_EPT];
        unsigned int bad = XS_TILE;  // first flagged local index
        unsigned long long run = 0;
        const uint64_t b0 = i + static_cast<uint64_t>(t) * XS_EPT;
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            const uint64_t g = b0 + k;
            double q = 0.0;
            if (g < N) {
                q = p[g] * inv_u;
            }
            const double f = floor(q);
            const bool tie = (q - f) == 0.5;
            const bool big = !(q < 1125899906842624.0);  // 2^50 (also catches inf)
            if ((tie || big) && g < N && bad == XS_TILE) {
                bad = t * XS_EPT + k;
            }
            r[k] = big ? 0ULL : static_cast<unsigned long long>(rint(q));
            run += r[k];
        }
        unsigned long long total;
        const unsigned long long excl = block_excl_scan_u64(run, sh, total);
        // binade exit: first element whose running sum reaches 2^53 units
        unsigned long long acc = m + excl;
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            acc += r[k];
            const unsigned int li = t * XS_EPT + k;
            if (acc >= TWO53 && li < bad) {
                bad = li;
            }
        }
        if (t == 0) {
            viol_sh = XS_TILE;
        }
        __syncthreads();
        atomicMin(&viol_sh, bad);
        __syncthreads();
        const uint64_t tile_len = (N - i) < XS_TILE ? (N - i) : XS_TILE;
        const unsigned int v = viol_sh < tile_len ? viol_sh : static_cast<unsigned int>(tile_len);
        // commit the elements before v
        acc = m + excl;
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            acc += r[k];
            const unsigned int li = t * XS_EPT + k;
            if (li < v) {
                cdf[i + li] = static_cast<double>(acc) * u;
            }
        }
        // the value before element v, for thread 0's IEEE step
        if (v < tile_len) {
            // running value just before v: the thread owning v - 1 knows it
            const unsigned int last = v;  // element index to add with an IEEE add
            if (last == 0) {
                if (t == 0) {
                    const double nv = __dadd_rn(s, p[i]);
                    cdf[i] = nv;
                    s_sh = nv;
                    i_sh = i + 1;
                }
            } else {
                const unsigned int owner = (last - 1) / XS_EPT;
                if (static_cast<unsigned int>(t) == owner) {
                    unsigned long long a2 = m + excl;
                    for (int k = 0; k < XS_EPT; ++k) {
                        if (t * XS_EPT + k < last) {
                            a2 += r[k];
                        }
                    }
                    const double before = static_cast<double>(a2) * u;
                    const double nv = __dadd_rn(before, p[i + last]);
                    cdf[i + last] = nv;
                    s_sh = nv;
                    i_sh = i + last + 1;
                }
            }
        } else {
            if (t == 0) {
                s_sh = static_cast<double>(m + total) * u;
                i_sh = i + tile_len;
            }
        }
        __syncthreads();
    }
}

// cumulative_end_offset_ (measurements.cpp:235-256): the last value strictly
// below `last`, found as the largest index holding one.
__global__ void k_last_below(const double* __restrict__ cdf, uint64_t N, unsigned long long* __restrict__ idx1)
{
    const double last = cdf[N - 1];
    unsigned long long best = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i + 1 < N; i += (uint64_t)gridDim.x * blockDim.x) {
        if (cdf[i] < last) {
            best = static_cast<unsigned long long>(i) + 1;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_down_sync(0xffffffffU, best, o);
        best = y > best ? y : best;
    }
    if ((threadIdx.x & 31) == 0 && best != 0) {
        atomicMax(idx1, best);
    }
}

// the distribution bound last - (last - second) * 1e-4 (measurements.cpp:288-295)
__global__ void k_seq_bound(const double* __restrict__ cdf, uint64_t N, const unsigned long long* __restrict__ idx1,
                            double* __restrict__ bound)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    const double last = cdf[N - 1];
    const unsigned long long j = *idx1;
    const double second = (j == 0) ? 0.0 : cdf[j - 1];
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
    // The certified tier pays off while the worst-case rounding bound of a
    // sequential sum, ~N * 2^-53, stays far below a typical probability ~1/N.
    const bool try_fast = (mode == 0) && N <= (uint64_t {1} << 22);
    if (!try_fast) {
        unc = 1;
    }
    if (try_fast) {
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
    if (unc != 0) {
        k_exact_cdf<<<1, XS_THREADS, 0, s.stream>>>(dp, N, dcdf);
        KT_CHECK_LAUNCH("k_exact_cdf");
        KT_CUDA(cudaMemsetAsync(d_nz, 0, 8, s.stream));
        const unsigned lb_blocks = static_cast<unsigned>(std::min<uint64_t>((N + 255) / 256, sm_count() * 8ULL));
        k_last_below<<<lb_blocks, 256, 0, s.stream>>>(dcdf, N, d_nz);
        KT_CHECK_LAUNCH("k_last_below");
        k_seq_bound<<<1, 32, 0, s.stream>>>(dcdf, N, d_nz, d_bound);
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
