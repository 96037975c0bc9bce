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
// exactly.  While s stays in one binade [2^(E-1), 2^E) every representable
// value is a multiple of u = 2^(E-53), so (no binade exit)
// fl(s + p) = s + rint(p / u) * u exactly away from ties, and an exact tie
// (p / u = n + 1/2) rounds s / u + n to even: a run of additions is an
// integer prefix sum, or a composition of run maps (RunMap below) where it
// holds ties.  The array is cut into tiles of XS_TILE elements:
//  1. tile sums (FP64, any order) and their exclusive scan give each tile an
//     approximate start value, hence a guess of its binade (or "all zero");
//  2. every tile with a guess sums rint(p / u) in uint64, flagging huge terms
//     (>= 2^50 units) and listing the tiles with exact ties, whose run maps
//     are composed in element order (k_tile_runs);
//  3. one block walks the tiles in order with the exact running value s: a
//     tile whose guess is s's binade, has no huge term and does not reach
//     2^53 units is passed over in O(1) (its start value is recorded); any
//     other tile is computed element by element from the exact s (the same
//     run-map scan, with one IEEE add for each huge term or binade exit);
//  4. every recorded tile writes its CDF from its exact start value: all of
//     them for a caller's probability vector; for the state's own
//     probabilities only the tiles that the bound and the shots land in,
//     found from the exact tile start values (k_shot_tiles below).
// A wrong guess only sends a tile down the element-by-element path: the
// result never depends on the approximate sums.
constexpr int XS_THREADS = 1024;
constexpr int XS_EPT = 16;
constexpr int XS_TILE = XS_THREADS * XS_EPT;
constexpr int XS_STAGE = XS_TILE + XS_TILE / 16;  // a staged tile, one pad double per 16 elements
constexpr int TILE_ZERO = -100000;    // every p in the tile is +0: s passes unchanged
constexpr int TILE_DIRTY = -200000;   // no binade guess, or a flagged term
constexpr double TINY = 0x1p-900;     // below this the running value is summed with IEEE adds

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

// Where the exact tier reads probability i: a vector (a caller's, or the
// state's with readout noise, written by the probability pass), or the
// state's own |a_i|^2 formed on the spot exactly as the probability pass
// forms them (round-to-nearest products and sum, no contraction), so the
// noiseless state path never writes the 8 B per amplitude vector.
struct ProbVec
{
    const double* __restrict__ p;
    __device__ __forceinline__ double operator[](uint64_t i) const { return p[i]; }
};

template <typename C>
struct ProbAmps
{
    const C* __restrict__ a;
    __device__ __forceinline__ double operator[](uint64_t i) const
    {
        const double2 v = to_d2(a[i]);
        return __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
    }
};

// Tile integer sums for these binades are formed during the probability pass
// (candidate k: the binade [2^(-k-1), 2^-k), units 2^(-k-53)): a normalised
// state's running sum starts most tiles in [1/16, 1), so only the other
// tiles are read a second time by k_tile_ints.  Four candidates for
// complex128 amplitudes, whose pass is bound by DRAM with the arithmetic
// hidden; two for complex64, whose 8-byte amplitudes leave less time per
// element (tiles in [1/4, 1): the second read covers about a fifth of them).
// N_CAND is the layout stride of the candidate sums.
constexpr int N_CAND = 4;

template <typename C>
constexpr int cand_count()
{
    return sizeof(C) == 16 ? 4 : 2;
}

// A run of additions inside one binade, as a function of the running value v
// in that binade's units: v -> v + S, or, once the run holds an exact tie,
// v -> v + S + ((v + c) & 1).  A tie element p = (n + 1/2) u gives
// fl(v u + p) = (v + n + ((v + n) & 1)) u (round half to even), so after it
// the parity of the running value no longer depends on v, and runs compose
// in order in the same form.  c: bit 0 the parity offset, bit 1 "has a tie".
struct RunMap
{
    unsigned long long S;
    int c;
};

__device__ __forceinline__ unsigned long long run_apply(const RunMap& a, unsigned long long v)
{
    return v + a.S + ((a.c & 2) ? ((v + static_cast<unsigned long long>(a.c)) & 1ULL) : 0ULL);
}

// run a, then run b
__device__ __forceinline__ RunMap run_then(const RunMap& a, const RunMap& b)
{
    if (a.c & 2) {
        const unsigned long long pa = (a.S + static_cast<unsigned long long>(a.c)) & 1ULL;  // parity after a
        const unsigned long long inc = b.S + ((b.c & 2) ? ((pa + static_cast<unsigned long long>(b.c)) & 1ULL) : 0ULL);
        return RunMap {a.S + inc, a.c};
    }
    if (b.c & 2) {
        return RunMap {a.S + b.S, static_cast<int>((a.S + static_cast<unsigned long long>(b.c)) & 1ULL) | 2};
    }
    return RunMap {a.S + b.S, 0};
}

// one element's run, q = p / u (the caller has excluded huge terms)
__device__ __forceinline__ RunMap run_of(double q)
{
    const double f = floor(q);
    if ((q - f) == 0.5) {
        const unsigned long long n = static_cast<unsigned long long>(f);
        return RunMap {n, static_cast<int>(n & 1ULL) | 2};
    }
    return RunMap {static_cast<unsigned long long>(rint(q)), 0};
}

__device__ __forceinline__ RunMap shfl_up_run(const RunMap& a, int o)
{
    return RunMap {__shfl_up_sync(0xffffffffU, a.S, o), __shfl_up_sync(0xffffffffU, a.c, o)};
}

// inclusive scan of the lanes' runs in lane order
__device__ __forceinline__ RunMap warp_scan_runs(RunMap x)
{
    const int lane = static_cast<int>(threadIdx.x & 31);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const RunMap y = shfl_up_run(x, o);
        if (lane >= o) {
            x = run_then(y, x);
        }
    }
    return x;
}

// exclusive scan of the threads' runs in thread order (XS_THREADS threads);
// sh holds 32 runs
__device__ __forceinline__ RunMap block_excl_scan_runs(const RunMap v, RunMap* sh)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const RunMap x = warp_scan_runs(v);
    if (lane == 31) {
        sh[warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        const RunMap w = warp_scan_runs(sh[lane]);
        __syncwarp();
        sh[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    RunMap in_warp = shfl_up_run(x, 1);
    if (lane == 0) {
        in_warp = RunMap {0, 0};
    }
    const RunMap r = (warp > 0) ? run_then(sh[warp - 1], in_warp) : in_warp;
    __syncthreads();
    return r;
}

// shared state of the element-by-element path
struct XState
{
    unsigned long long sh[32];
    RunMap shr[32];
    double s;
    unsigned long long i;
    unsigned int viol;
};

// cdf[beg, end) (at most XS_TILE elements) as the sequential sum continued
// from the exact value s_in, by the whole block (XS_THREADS threads); returns
// the value after element end-1.  The probabilities are staged once in st
// (XS_STAGE doubles of shared memory, element j at j + j / 16: a thread's
// XS_EPT consecutive elements then fall on distinct bank pairs), so a window
// that restarts after a binade exit re-reads shared memory, not DRAM; each
// committed CDF value replaces its probability there (no later window reads
// it), and the tile's CDF is stored with coalesced writes at the end.
template <typename P>
__device__ double exact_range(const P src, uint64_t beg, uint64_t end, double s_in, double* __restrict__ cdf, XState& X,
                              double* __restrict__ st)
{
    const int t = threadIdx.x;
    const uint64_t len = end - beg;
    auto slot = [&](uint64_t g) -> double& {
        const uint64_t j = g - beg;
        return st[j + (j >> 4)];
    };
    __syncthreads();
    {
        // all XS_EPT loads of a thread in flight before the first store
        double v[XS_EPT];
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            const uint64_t j = static_cast<uint64_t>(t) + static_cast<uint64_t>(k) * XS_THREADS;
            v[k] = j < len ? src[beg + j] : 0.0;
        }
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            const uint64_t j = static_cast<uint64_t>(t) + static_cast<uint64_t>(k) * XS_THREADS;
            if (j < len) {
                st[j + (j >> 4)] = v[k];
            }
        }
    }
    if (t == 0) {
        X.s = s_in;
        X.i = beg;
    }
    __syncthreads();
    constexpr unsigned long long TWO53 = 1ULL << 53;
    while (true) {
        const uint64_t i = X.i;
        const double s = X.s;
        __syncthreads();  // every thread has read (i, s) before anyone moves them on
        if (i >= end) {
            break;
        }
        if (s < TINY) {
            // zero or tiny running value (subnormal spacing, huge 1/ulp): plain IEEE steps
            if (t == 0) {
                const double nv = __dadd_rn(s, slot(i));
                X.s = nv;
                slot(i) = nv;
                X.i = i + 1;
            }
            __syncthreads();
            continue;
        }
        int E;
        frexp(s, &E);                             // s in [2^(E-1), 2^E)
        const double inv_u = ldexp(1.0, 53 - E);  // 1 / ulp(s)
        const double u = ldexp(1.0, E - 53);
        const unsigned long long m = static_cast<unsigned long long>(s * inv_u);  // exact, in [2^52, 2^53)
        const uint64_t b0 = i + static_cast<uint64_t>(t) * XS_EPT;
        // this thread's element k as a run (ties included); a huge term ends
        // the integer path and counts as nothing here.  Only a window that
        // holds a tie takes this form: its probabilities are read again at
        // each use rather than held (64 registers per thread)
        auto elem = [&](int k, bool& big) -> RunMap {
            const uint64_t g = b0 + static_cast<uint64_t>(k);
            big = false;
            if (g >= end) {
                return RunMap {0ULL, 0};
            }
            const double q = slot(g) * inv_u;
            if (!(q < 1125899906842624.0)) {  // 2^50 (also catches inf)
                big = true;
                return RunMap {0ULL, 0};
            }
            return run_of(q);
        };
        unsigned long long r[XS_EPT];
        unsigned int bad = XS_TILE;  // first huge term or binade exit (local index)
        unsigned long long run = 0;
        int has_tie = 0;
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            const uint64_t g = b0 + k;
            double q = 0.0;
            if (g < end) {
                q = slot(g) * inv_u;
            }
            const double f = floor(q);
            const bool big = !(q < 1125899906842624.0);  // 2^50 (also catches inf)
            if (big && g < end && bad == XS_TILE) {
                bad = t * XS_EPT + k;
            }
            if ((q - f) == 0.5 && g < end) {
                has_tie = 1;
            }
            r[k] = big ? 0ULL : static_cast<unsigned long long>(rint(q));
            run += r[k];
        }
        const bool ties = __syncthreads_or(has_tie) != 0;
        // the exact value before this thread's first element, in units
        unsigned long long start;
        if (!ties) {
            unsigned long long total;
            start = m + block_excl_scan_u64(run, X.sh, total);
        } else {
            RunMap tm {0ULL, 0};
            for (int k = 0; k < XS_EPT; ++k) {
                bool big;
                tm = run_then(tm, elem(k, big));
            }
            start = run_apply(block_excl_scan_runs(tm, X.shr), m);
        }
        // the value after element k, from the value before it
        auto step = [&](int k, unsigned long long a) -> unsigned long long {
            if (!ties) {
                return a + r[k];
            }
            bool big;
            return run_apply(elem(k, big), a);
        };
        // binade exit: first element whose running value reaches 2^53 units
        unsigned long long acc = start;
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            acc = step(k, acc);
            const unsigned int li = t * XS_EPT + k;
            if (acc >= TWO53 && li < bad) {
                bad = li;
            }
        }
        if (t == 0) {
            X.viol = XS_TILE;
        }
        __syncthreads();
        // one shared atomic per warp, not per thread: same-address atomics serialise
        bad = __reduce_min_sync(0xffffffffU, bad);
        if ((t & 31) == 0) {
            atomicMin(&X.viol, bad);
        }
        __syncthreads();
        const uint64_t tile_len = (end - i) < XS_TILE ? (end - i) : XS_TILE;
        const unsigned int v = X.viol < tile_len ? X.viol : static_cast<unsigned int>(tile_len);
        // commit the elements before v (each thread reads and then replaces
        // only its own elements; before_v is the value just before element v)
        acc = start;
        unsigned long long before_v = start;
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            acc = step(k, acc);
            const unsigned int li = t * XS_EPT + k;
            if (li + 1 == v) {
                before_v = acc;
            }
            if (li < v) {
                slot(i + li) = static_cast<double>(acc) * u;
                if (v == tile_len && li + 1 == tile_len) {
                    X.s = static_cast<double>(acc) * u;  // every element of the window went in
                    X.i = i + tile_len;
                }
            }
        }
        if (v < tile_len) {
            // element v gets one IEEE add onto the value just before it
            if (v == 0) {
                if (t == 0) {
                    const double nv = __dadd_rn(s, slot(i));
                    slot(i) = nv;
                    X.s = nv;
                    X.i = i + 1;
                }
            } else {
                const unsigned int owner = (v - 1) / XS_EPT;
                if (static_cast<unsigned int>(t) == owner) {
                    const double before = static_cast<double>(before_v) * u;
                    const double nv = __dadd_rn(before, slot(i + v));
                    slot(i + v) = nv;
                    X.s = nv;
                    X.i = i + v + 1;
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < XS_EPT; ++k) {
        const uint64_t j = static_cast<uint64_t>(t) + static_cast<uint64_t>(k) * XS_THREADS;
        if (j < len) {
            cdf[beg + j] = st[j + (j >> 4)];
        }
    }
    return X.s;
}

// 1. FP64 sum of each tile (any order)
__global__ void __launch_bounds__(256) k_tile_sums(const double* __restrict__ p, uint64_t N, double* __restrict__ tsum)
{
    __shared__ double sh[8];
    const uint64_t beg = static_cast<uint64_t>(blockIdx.x) * XS_TILE;
    const uint64_t end = beg + XS_TILE < N ? beg + XS_TILE : N;
    double acc = 0.0;
    for (uint64_t i = beg + threadIdx.x; i < end; i += 256) {
        acc += p[i];
    }
    acc = warp_sum_d(acc);
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) {
            s += sh[w];
        }
        tsum[blockIdx.x] = s;
    }
}

// 0 + 1 + 2 fused, for the state's own probabilities without readout noise:
// each tile's FP64 sum of |a_i|^2 (any order, as above) and its integer sums
// in the cand_count<C>() candidate binades with their flags, as k_tile_ints forms them
// (cflag bit k: a tie in candidate k, bit 8 + k: a huge term); the
// probabilities are not stored
template <typename C>
__global__ void __launch_bounds__(256) k_probs_tiles(const C* __restrict__ a, uint64_t N, double* __restrict__ tsum,
                                                     unsigned long long* __restrict__ cints, int* __restrict__ cflag)
{
    constexpr int NC = cand_count<C>();
    __shared__ double sh[8];
    __shared__ unsigned long long shi[NC][8];
    __shared__ int flag_sh;
    if (threadIdx.x == 0) {
        flag_sh = 0;
    }
    const ProbAmps<C> p {a};
    const uint64_t beg = static_cast<uint64_t>(blockIdx.x) * XS_TILE;
    const uint64_t end = beg + XS_TILE < N ? beg + XS_TILE : N;
    double acc = 0.0;
    // x_k = q 2^(53+k) = 2^k x_0: with x_0 = fl + F (fl an integer, F in [0, 1)),
    // rint(x_k) = 2^k fl + floor(2^k F + 1/2) away from ties, and with the top
    // four bits of F as T = floor(16 F) (exact: 16 F is a scaling) that is
    // (T + 2^(3-k)) >> (4-k); x_k is a tie when 2^(k+1) F is an odd integer,
    // i.e. 16 F is an integer with T's low 4-k bits equal to 2^(3-k).
    unsigned long long sfl = 0;  // sum of fl
    unsigned int small[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        small[k] = 0;
    }
    int fl = 0;
    for (uint64_t i = beg + threadIdx.x; i < end; i += 256) {
        const double q = p[i];
        acc += q;
        const double x0 = q * 0x1p53;  // exact: a power of two
        if (!(x0 < 0x1p47)) {
            // 2^50 units and more in some candidate binade (or inf / NaN)
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                if (!(x0 < static_cast<double>(1ULL << (50 - k)))) {
                    fl |= 1 << (8 + k);
                }
            }
        }
        const double f0 = floor(x0);
        const double y = (x0 - f0) * 16.0;  // exact
        const double ty = floor(y);
        const unsigned int T = static_cast<unsigned int>(ty);
        const bool whole = (y == ty);
        sfl += static_cast<unsigned long long>(f0);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            small[k] += (T + (8u >> k)) >> (4 - k);
            if (whole && (T & ((16u >> k) - 1u)) == (8u >> k)) {
                fl |= 1 << k;
            }
        }
    }
    unsigned long long ci[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        // can wrap only when candidate k has a term of 2^50 units or more, and
        // such a candidate's sum is never used
        ci[k] = (sfl << k) + small[k];
    }
    acc = warp_sum_d(acc);
#pragma unroll
    for (int k = 0; k < NC; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ci[k] += __shfl_down_sync(0xffffffffU, ci[k], o);
        }
    }
    __syncthreads();  // flag_sh is cleared
    if (fl != 0) {
        atomicOr(&flag_sh, fl);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5] = acc;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            shi[k][threadIdx.x >> 5] = ci[k];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) {
            t += sh[w];
        }
        tsum[blockIdx.x] = t;
        for (int k = 0; k < NC; ++k) {
            unsigned long long v = 0;
            for (int w = 0; w < 8; ++w) {
                v += shi[k][w];
            }
            cints[static_cast<uint64_t>(blockIdx.x) * N_CAND + k] = v;
        }
        cflag[blockIdx.x] = flag_sh;
    }
}

// 1b. one block: approximate start value of every tile, and its binade guess
// (with cints: a tile guessed in a candidate binade takes that binade's
// integer sum; a huge term there makes it dirty, a tie lists it in tie_list
// for k_tile_runs).
// The tile sums pass through shared memory GUESS_PER x XS_THREADS at a time:
// loaded coalesced, each thread then scans GUESS_PER consecutive ones.
constexpr int GUESS_PER = 4;
constexpr int GUESS_CHUNK = GUESS_PER * XS_THREADS;

__global__ void __launch_bounds__(XS_THREADS) k_tile_guess(const double* __restrict__ tsum, uint64_t n_tiles,
                                                           int* __restrict__ code,
                                                           const unsigned long long* __restrict__ cints,
                                                           const int* __restrict__ cflag,
                                                           unsigned long long* __restrict__ ints,
                                                           int* __restrict__ tie, unsigned long long* __restrict__ tie_list,
                                                           unsigned int* __restrict__ tie_count, int n_cand)
{
    __shared__ double st[GUESS_CHUNK];
    __shared__ double sh[32];
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    double carry = 0.0;  // approximate sum of the chunks before this one (the same in every thread)
    for (uint64_t c0 = 0; c0 < n_tiles; c0 += GUESS_CHUNK) {
        for (int j = t; j < GUESS_CHUNK; j += XS_THREADS) {
            const uint64_t k = c0 + static_cast<uint64_t>(j);
            st[j] = k < n_tiles ? tsum[k] : 0.0;
        }
        __syncthreads();
        double loc[GUESS_PER];
        double local = 0.0;
#pragma unroll
        for (int i = 0; i < GUESS_PER; ++i) {
            loc[i] = st[t * GUESS_PER + i];
            local += loc[i];
        }
        // exclusive block scan of the thread sums (FP64, approximate)
        double x = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffU, x, o);
            if (lane >= o) {
                x += y;
            }
        }
        if (lane == 31) {
            sh[warp] = x;
        }
        __syncthreads();
        if (warp == 0) {
            double w = sh[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double y = __shfl_up_sync(0xffffffffU, w, o);
                if (lane >= o) {
                    w += y;
                }
            }
            sh[lane] = w;
        }
        __syncthreads();
        double a0 = carry + ((warp > 0) ? sh[warp - 1] : 0.0) + (x - local);
#pragma unroll
        for (int i = 0; i < GUESS_PER; ++i) {
            const uint64_t k = c0 + static_cast<uint64_t>(t * GUESS_PER + i);
            const double ts = loc[i];
            const double a1 = a0 + ts;
            if (k < n_tiles) {
                int c = TILE_DIRTY;
                if (ts == 0.0) {
                    c = TILE_ZERO;
                } else if (a0 >= 2.0 * TINY) {
                    int e0, e1;
                    frexp(a0 * (1.0 - 0x1p-20), &e0);
                    frexp(a1 * (1.0 + 0x1p-20), &e1);
                    if (e0 == e1) {
                        c = e0;
                    }
                }
                int has_tie = 0;
                if (cints != nullptr && c <= 0 && c > -n_cand) {
                    const int j = -c;
                    const int f = cflag[k];
                    if ((f >> (8 + j)) & 1) {
                        c = TILE_DIRTY;
                    } else if ((f >> j) & 1) {
                        has_tie = 1;
                        tie_list[atomicAdd(tie_count, 1U)] = k;
                    } else {
                        ints[k] = cints[k * N_CAND + static_cast<uint64_t>(j)];
                    }
                }
                code[k] = c;
                tie[k] = has_tie;
            }
            a0 = a1;
        }
        carry += sh[31];
        __syncthreads();  // st and sh are reused by the next chunk
    }
}

// 2. integer sum of a tile in the units of its guessed binade; a huge term
// makes it dirty, an exact tie lists it for k_tile_runs (tiles guessed in one
// of the n_cand candidate binades have theirs already)
template <typename P>
__global__ void __launch_bounds__(256) k_tile_ints(const P p, uint64_t N, int* __restrict__ code,
                                                   unsigned long long* __restrict__ ints, int n_cand,
                                                   int* __restrict__ tie, unsigned long long* __restrict__ tie_list,
                                                   unsigned int* __restrict__ tie_count)
{
    __shared__ unsigned long long sh[8];
    __shared__ int flag_sh;
    const int c = code[blockIdx.x];
    if (c == TILE_ZERO || c == TILE_DIRTY || (c <= 0 && c > -n_cand)) {
        return;
    }
    if (threadIdx.x == 0) {
        flag_sh = 0;
    }
    __syncthreads();
    const double inv_u = ldexp(1.0, 53 - c);
    const uint64_t beg = static_cast<uint64_t>(blockIdx.x) * XS_TILE;
    const uint64_t end = beg + XS_TILE < N ? beg + XS_TILE : N;
    unsigned long long acc = 0;
    int fl = 0;  // bit 0: an exact tie, bit 1: a huge term (2^50 units and more, or inf / NaN)
    for (uint64_t i = beg + threadIdx.x; i < end; i += 256) {
        const double q = p[i] * inv_u;
        const double f = floor(q);
        if ((q - f) == 0.5) {
            fl |= 1;
        }
        if (!(q < 1125899906842624.0)) {
            fl |= 2;
        }
        acc += (fl & 2) ? 0ULL : static_cast<unsigned long long>(rint(q));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_down_sync(0xffffffffU, acc, o);
    }
    if (fl != 0) {
        atomicOr(&flag_sh, fl);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (int w = 0; w < 8; ++w) {
            s += sh[w];
        }
        ints[blockIdx.x] = s;
        if (flag_sh & 2) {
            code[blockIdx.x] = TILE_DIRTY;
        } else if (flag_sh & 1) {
            tie[blockIdx.x] = 1;
            tie_list[atomicAdd(tie_count, 1U)] = blockIdx.x;
        }
    }
}

// 2b. the run map (RunMap) of every listed tile with a tie, in the units of
// its guessed binade: each thread composes XS_EPT consecutive elements in
// order, then the block composes the threads' runs in order
template <typename P>
__global__ void __launch_bounds__(XS_THREADS) k_tile_runs(const P p, uint64_t N, int* __restrict__ code,
                                                          const unsigned long long* __restrict__ tie_list,
                                                          const unsigned int* __restrict__ tie_count,
                                                          unsigned long long* __restrict__ run_s,
                                                          int* __restrict__ run_c)
{
    __shared__ RunMap sh[32];
    __shared__ int big_sh;
    const int t = threadIdx.x;
    const unsigned int count = *tie_count;
    for (unsigned int li = blockIdx.x; li < count; li += gridDim.x) {
        const uint64_t tile = tie_list[li];
        const int c = code[tile];
        if (t == 0) {
            big_sh = 0;
        }
        __syncthreads();
        const double inv_u = ldexp(1.0, 53 - c);
        const uint64_t beg = tile * XS_TILE;
        const uint64_t end = beg + XS_TILE < N ? beg + XS_TILE : N;
        RunMap r {0, 0};
        bool big = false;
        const uint64_t b0 = beg + static_cast<uint64_t>(t) * XS_EPT;
#pragma unroll
        for (int k = 0; k < XS_EPT; ++k) {
            const uint64_t g = b0 + k;
            if (g < end) {
                const double q = p[g] * inv_u;
                big = big || !(q < 1125899906842624.0);
                r = run_then(r, run_of(big ? 0.0 : q));
            }
        }
        if (big) {
            big_sh = 1;
        }
        // the block's composition in thread order: an exclusive scan, then
        // the last thread's run appended
        const RunMap before = block_excl_scan_runs(r, sh);
        if (t == XS_THREADS - 1) {
            const RunMap all = run_then(before, r);
            run_s[tile] = all.S;
            run_c[tile] = all.c;
            if (big_sh) {
                code[tile] = TILE_DIRTY;  // not reached: the tile was flagged for its ties only
            }
        }
        __syncthreads();
    }
}

// 3. one block: the exact running value through all tiles.  carry[t] gets the
// exact value before tile t, or -1 when the tile's CDF was written here;
// tstart[t] the exact value before tile t in every case, and tstart[n_tiles]
// the last CDF value (so tstart[t + 1] is tile t's last CDF value).
template <typename P>
__global__ void __launch_bounds__(XS_THREADS) k_exact_chain(const P p, uint64_t N, uint64_t n_tiles,
                                                            const int* __restrict__ code,
                                                            const unsigned long long* __restrict__ ints,
                                                            const int* __restrict__ tie,
                                                            const unsigned long long* __restrict__ run_s,
                                                            const int* __restrict__ run_c,
                                                            double* __restrict__ carry, double* __restrict__ tstart,
                                                            double* __restrict__ cdf)
{
    extern __shared__ double stage[];  // XS_STAGE doubles: the tile exact_range works on
    __shared__ XState X;
    __shared__ unsigned long long t_sh;
    __shared__ double s_sh;
    __shared__ unsigned int first_sh;
    __shared__ unsigned long long m_sh;
    const int t = threadIdx.x;
    if (t == 0) {
        t_sh = 0;
        s_sh = 0.0;  // the value before element 0: cdf[0] = 0 + p[0] = p[0]
    }
    __syncthreads();
    constexpr unsigned long long TWO53 = 1ULL << 53;
    while (true) {
        const uint64_t t0 = t_sh;
        const double s = s_sh;
        if (t == 0) {
            first_sh = XS_THREADS;
        }
        __syncthreads();
        if (t0 >= n_tiles) {
            break;
        }
        // fast step over tiles t0 .. t0 + XS_THREADS - 1
        const bool normal = s >= TINY;
        int E = 0;
        unsigned long long m = 0;
        double u = 0.0;
        if (normal) {
            frexp(s, &E);
            m = static_cast<unsigned long long>(s * ldexp(1.0, 53 - E));
            u = ldexp(1.0, E - 53);
        }
        const uint64_t tile = t0 + static_cast<uint64_t>(t);
        const int c = tile < n_tiles ? code[tile] : TILE_DIRTY;
        // the tile's additions as a run: its integer sum, or its run map when
        // it holds a tie (the plain integer scan when no tile of the step does)
        const bool live = tile < n_tiles && c != TILE_ZERO && c != TILE_DIRTY;
        const bool tile_tie = live && tie[tile] != 0;
        unsigned long long mt, me;  // the exact value before and after the tile, in units
        if (__syncthreads_or(tile_tie) == 0) {
            const unsigned long long I = live ? ints[tile] : 0ULL;
            unsigned long long total;
            mt = m + block_excl_scan_u64(I, X.sh, total);
            me = mt + I;
        } else {
            const RunMap R = tile_tie ? RunMap {run_s[tile], run_c[tile]} : RunMap {live ? ints[tile] : 0ULL, 0};
            mt = run_apply(block_excl_scan_runs(R, X.shr), m);
            me = run_apply(R, mt);
        }
        bool ok = tile < n_tiles && (c == TILE_ZERO || (normal && c == E));
        if (ok && normal && me >= TWO53) {
            ok = false;
        }
        const unsigned int wmin = __reduce_min_sync(0xffffffffU, ok ? 0xffffffffU : static_cast<unsigned int>(t));
        if ((t & 31) == 0 && wmin != 0xffffffffU) {
            atomicMin(&first_sh, wmin);
        }
        __syncthreads();
        const unsigned int first = first_sh;
        if (static_cast<unsigned int>(t) < first) {
            const double c0 = normal ? static_cast<double>(mt) * u : s;
            carry[tile] = c0;
            tstart[tile] = c0;
            if (static_cast<unsigned int>(t) + 1 == first) {
                m_sh = me;
            }
        }
        __syncthreads();
        if (t == 0) {
            if (first > 0) {
                s_sh = normal ? static_cast<double>(m_sh) * u : s;
            }
            t_sh = t0 + first;
        }
        __syncthreads();
        if (first == XS_THREADS) {
            continue;
        }
        const uint64_t bad = t_sh;
        if (bad >= n_tiles) {
            break;
        }
        // tile `bad`, element by element from the exact value
        const uint64_t beg = bad * XS_TILE;
        const uint64_t end = beg + XS_TILE < N ? beg + XS_TILE : N;
        if (t == 0) {
            tstart[bad] = s_sh;
        }
        const double s_out = exact_range(p, beg, end, s_sh, cdf, X, stage);
        __syncthreads();
        if (t == 0) {
            carry[bad] = -1.0;
            s_sh = s_out;
            t_sh = bad + 1;
        }
        __syncthreads();
    }
    if (t == 0) {
        tstart[n_tiles] = s_sh;
    }
}

// 4. the CDF of every tile passed over in step 3 (list == nullptr: block b
// writes tile b), or of the *count tiles in `list`, from its exact start value
template <typename P>
__global__ void __launch_bounds__(XS_THREADS) k_tile_write(const P p, uint64_t N,
                                                           const int* __restrict__ code,
                                                           const double* __restrict__ carry, double* __restrict__ cdf,
                                                           const unsigned long long* __restrict__ list,
                                                           const unsigned int* __restrict__ count,
                                                           const int* __restrict__ tie)
{
    // warp w holds the tile's elements [w * 32 * XS_EPT, (w + 1) * 32 * XS_EPT)
    // as XS_EPT rows of 32 consecutive elements, one per lane, so every load
    // and store of a row is one coalesced 256-byte access; the integer prefix
    // runs row by row (a warp scan per row, the warp's earlier rows carried)
    // after a block scan of the warp totals, in element order
    __shared__ unsigned long long sh[32];
    __shared__ RunMap shr[32];
    uint64_t tile = blockIdx.x;
    if (list != nullptr) {
        if (blockIdx.x >= *count) {
            return;
        }
        tile = list[blockIdx.x];
    }
    const double c0 = carry[tile];
    if (c0 < 0.0) {
        return;
    }
    const uint64_t beg = tile * XS_TILE;
    const uint64_t end = beg + XS_TILE < N ? beg + XS_TILE : N;
    const int lane = static_cast<int>(threadIdx.x & 31);
    const uint64_t wb = beg + static_cast<uint64_t>(threadIdx.x >> 5) * (32 * XS_EPT) + lane;
    const int c = code[tile];
    if (c == TILE_ZERO) {
        for (int k = 0; k < XS_EPT; ++k) {
            const uint64_t g = wb + static_cast<uint64_t>(k) * 32;
            if (g < end) {
                cdf[g] = c0;
            }
        }
        return;
    }
    const double inv_u = ldexp(1.0, 53 - c);
    const double u = ldexp(1.0, c - 53);
    const unsigned long long m = static_cast<unsigned long long>(c0 * inv_u);
    if (tie[tile]) {
        // the same rows, composed as run maps (a tie's rounding depends on the
        // parity of the value before it): each warp's run over its rows, a block
        // scan of those in warp order, then every row's lane scan from the
        // exact value before it
        // (the probabilities are read twice rather than held: this path is
        // rare, and 1024 threads have 64 registers each)
        const int warp = static_cast<int>(threadIdx.x >> 5);
        RunMap w {0ULL, 0};
        for (int k = 0; k < XS_EPT; ++k) {
            const uint64_t g = wb + static_cast<uint64_t>(k) * 32;
            const RunMap row = warp_scan_runs((g < end) ? run_of(p[g] * inv_u) : RunMap {0ULL, 0});
            w = run_then(w, RunMap {__shfl_sync(0xffffffffU, row.S, 31), __shfl_sync(0xffffffffU, row.c, 31)});
        }
        if (lane == 0) {
            shr[warp] = w;
        }
        __syncthreads();
        if (warp == 0) {
            const RunMap x = warp_scan_runs(shr[lane]);
            __syncwarp();
            shr[lane] = x;  // inclusive over warps
        }
        __syncthreads();
        unsigned long long acc = (warp > 0) ? run_apply(shr[warp - 1], m) : m;
        for (int k = 0; k < XS_EPT; ++k) {
            const uint64_t g = wb + static_cast<uint64_t>(k) * 32;
            const RunMap x = warp_scan_runs((g < end) ? run_of(p[g] * inv_u) : RunMap {0ULL, 0});
            if (g < end) {
                cdf[g] = static_cast<double>(run_apply(x, acc)) * u;
            }
            acc = run_apply(RunMap {__shfl_sync(0xffffffffU, x.S, 31), __shfl_sync(0xffffffffU, x.c, 31)}, acc);
        }
        return;
    }
    unsigned long long r[XS_EPT];
    unsigned long long run = 0;
#pragma unroll
    for (int k = 0; k < XS_EPT; ++k) {
        const uint64_t g = wb + static_cast<uint64_t>(k) * 32;
        r[k] = (g < end) ? static_cast<unsigned long long>(rint(p[g] * inv_u)) : 0ULL;
        run += r[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        run += __shfl_xor_sync(0xffffffffU, run, o);  // the warp's total, in every lane
    }
    unsigned long long total;
    const unsigned long long before = block_excl_scan_u64(lane == 0 ? run : 0ULL, sh, total);
    unsigned long long acc = m + __shfl_sync(0xffffffffU, before, 0);
#pragma unroll
    for (int k = 0; k < XS_EPT; ++k) {
        unsigned long long x = r[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffU, x, o);
            if (lane >= o) {
                x += y;
            }
        }
        const uint64_t g = wb + static_cast<uint64_t>(k) * 32;
        if (g < end) {
            cdf[g] = static_cast<double>(acc + x) * u;
        }
        acc += __shfl_sync(0xffffffffU, x, 31);
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

// The searches above on a CDF written only where they look.  For a
// non-decreasing CDF (the state's own probabilities are never negative)
// lower_bound(cdf, v) lies in the first tile whose last value, tstart[t + 1],
// is not below v: every element of the tiles before it is at most their last
// value, which is below v.  So the distribution bound and every shot first
// pick their tile from the n_tiles + 1 exact tile start values, the tiles
// picked (at most one per shot, plus the bound's) get their CDF written, and
// each search finishes inside its tile: the same indices as the searches over
// the whole CDF, without writing the 8 B per amplitude of the other tiles.

// the first t in [0, n_tiles) with tstart[t + 1] >= v, or n_tiles
__device__ __forceinline__ uint64_t tile_of(const double* __restrict__ tstart, uint64_t n_tiles, double v)
{
    uint64_t lo = 0, len = n_tiles;
    while (len > 0) {
        const uint64_t half = len / 2;
        if (tstart[lo + half + 1] < v) {
            lo = lo + half + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    return lo;
}

// lower_bound(cdf + beg, cdf + end, v) - cdf
__device__ __forceinline__ uint64_t lower_bound_in(const double* __restrict__ cdf, uint64_t beg, uint64_t end, double v)
{
    uint64_t lo = beg, len = end - beg;
    while (len > 0) {
        const uint64_t half = len / 2;
        if (cdf[lo + half] < v) {
            lo = lo + half + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    return lo;
}

// the tile holding lower_bound(cdf, last), listed alone for k_tile_write
__global__ void k_bound_tile(const double* __restrict__ tstart, uint64_t n_tiles, unsigned long long* __restrict__ list,
                             unsigned int* __restrict__ count)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    const uint64_t t = tile_of(tstart, n_tiles, tstart[n_tiles]);
    list[0] = t < n_tiles ? t : n_tiles - 1;
    *count = 1;
}

// cumulative_end_offset_ and the distribution bound (measurements.cpp:235-256,
// 288-295) from the bound tile's CDF: j = lower_bound(cdf, last), second =
// cdf[j - 1] (the previous tile's last value, tstart[t], when j starts tile t)
__global__ void k_sparse_bound(const double* __restrict__ cdf, uint64_t N, const double* __restrict__ tstart,
                               uint64_t n_tiles, const unsigned long long* __restrict__ list, double* __restrict__ bound)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    const double last = tstart[n_tiles];
    const uint64_t t = list[0];
    const uint64_t beg = t * XS_TILE;
    const uint64_t end = beg + XS_TILE < N ? beg + XS_TILE : N;
    const uint64_t j = lower_bound_in(cdf, beg, end, last);
    const double second = (j == 0) ? 0.0 : (j == beg ? tstart[t] : cdf[j - 1]);
    const double offset = __dmul_rn(__dsub_rn(last, second), 1.0e-4);
    *bound = __dsub_rn(last, offset);
}

// each shot's tile; every tile some shot picks is listed once
__global__ void k_shot_tiles(const double* __restrict__ tstart, uint64_t n_tiles, const double* __restrict__ bound,
                             const double* __restrict__ canon, int64_t n_shots,
                             unsigned long long* __restrict__ shot_tile, int* __restrict__ hit,
                             unsigned long long* __restrict__ list, unsigned int* __restrict__ count)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) {
        return;
    }
    const double u = __dadd_rn(__dmul_rn(canon[s], __dsub_rn(*bound, 0.0)), 0.0);
    const uint64_t t = tile_of(tstart, n_tiles, u);
    shot_tile[s] = t;
    if (t < n_tiles && atomicExch(&hit[t], 1) == 0) {
        list[atomicAdd(count, 1U)] = t;
    }
}

__global__ void k_shot_search(const double* __restrict__ cdf, uint64_t N, uint64_t n_tiles,
                              const double* __restrict__ bound, const double* __restrict__ canon, int64_t n_shots,
                              const unsigned long long* __restrict__ shot_tile, uint64_t* __restrict__ out)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) {
        return;
    }
    const uint64_t t = shot_tile[s];
    if (t >= n_tiles) {
        out[s] = N - 1;  // u above every CDF value: lower_bound gives N, clamped as k_seq_search does
        return;
    }
    const double u = __dadd_rn(__dmul_rn(canon[s], __dsub_rn(*bound, 0.0)), 0.0);
    const uint64_t beg = t * XS_TILE;
    const uint64_t end = beg + XS_TILE < N ? beg + XS_TILE : N;
    const uint64_t lo = lower_bound_in(cdf, beg, end, u);
    out[s] = lo < N ? lo : N - 1;
}

}  // namespace

namespace
{

// device buffers of the exact tier
struct ExactBufs
{
    uint64_t N, n_tiles;
    int64_t n_shots;
    int* code;
    unsigned long long* ints;
    double* carry;
    double* tstart;
    double* cdf;
    int* hit;
    unsigned long long* list;
    unsigned int* count;
    unsigned long long* stile;
    int* tie;
    unsigned long long* run_s;
    int* run_c;
    unsigned long long* tie_list;
    unsigned int* tie_count;
    unsigned long long* nz;
    double* bound;
    const double* canon;
    uint64_t* out;
};

// steps 2-4 of the exact tier and the searches, reading probabilities from p.
// sorted: every probability is >= 0 (the state's own), so the CDF never
// decreases and only the tiles the searches land in are written.
template <typename P>
int32_t exact_tail(cudaStream_t st, const P p, const ExactBufs& b, int n_cand, bool sorted)
{
    const uint64_t N = b.N, n_tiles = b.n_tiles;
    k_tile_ints<P><<<static_cast<unsigned>(n_tiles), 256, 0, st>>>(p, N, b.code, b.ints, n_cand, b.tie,
                                                                     b.tie_list, b.tie_count);
    KT_CHECK_LAUNCH("k_tile_ints");
    k_tile_runs<P><<<static_cast<unsigned>(sm_count()), XS_THREADS, 0, st>>>(p, N, b.code, b.tie_list, b.tie_count,
                                                                             b.run_s, b.run_c);
    KT_CHECK_LAUNCH("k_tile_runs");
    constexpr int stage_bytes = XS_STAGE * static_cast<int>(sizeof(double));
    KT_CUDA(cudaFuncSetAttribute(k_exact_chain<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, stage_bytes));
    k_exact_chain<P><<<1, XS_THREADS, stage_bytes, st>>>(p, N, n_tiles, b.code, b.ints, b.tie, b.run_s, b.run_c,
                                                         b.carry, b.tstart, b.cdf);
    KT_CHECK_LAUNCH("k_exact_chain");
    const unsigned shot_blocks = static_cast<unsigned>((b.n_shots + 127) / 128);
    if (sorted) {
        k_bound_tile<<<1, 32, 0, st>>>(b.tstart, n_tiles, b.list, b.count);
        KT_CHECK_LAUNCH("k_bound_tile");
        k_tile_write<P><<<1, XS_THREADS, 0, st>>>(p, N, b.code, b.carry, b.cdf, b.list, b.count, b.tie);
        KT_CHECK_LAUNCH("k_tile_write");
        k_sparse_bound<<<1, 32, 0, st>>>(b.cdf, N, b.tstart, n_tiles, b.list, b.bound);
        KT_CHECK_LAUNCH("k_sparse_bound");
        KT_CUDA(cudaMemsetAsync(b.hit, 0, n_tiles * 4, st));
        KT_CUDA(cudaMemsetAsync(b.count, 0, 4, st));
        k_shot_tiles<<<shot_blocks, 128, 0, st>>>(b.tstart, n_tiles, b.bound, b.canon, b.n_shots, b.stile, b.hit, b.list,
                                                  b.count);
        KT_CHECK_LAUNCH("k_shot_tiles");
        const unsigned n_write = static_cast<unsigned>(std::min<uint64_t>(static_cast<uint64_t>(b.n_shots), n_tiles));
        k_tile_write<P><<<n_write, XS_THREADS, 0, st>>>(p, N, b.code, b.carry, b.cdf, b.list, b.count, b.tie);
        KT_CHECK_LAUNCH("k_tile_write");
        k_shot_search<<<shot_blocks, 128, 0, st>>>(b.cdf, N, n_tiles, b.bound, b.canon, b.n_shots, b.stile, b.out);
        KT_CHECK_LAUNCH("k_shot_search");
        return KT_OK;
    }
    // a caller's vector may hold negative entries: the whole CDF, and the
    // reference's scan for the end offset
    k_tile_write<P><<<static_cast<unsigned>(n_tiles), XS_THREADS, 0, st>>>(p, N, b.code, b.carry, b.cdf, nullptr,
                                                                           nullptr, b.tie);
    KT_CHECK_LAUNCH("k_tile_write");
    KT_CUDA(cudaMemsetAsync(b.nz, 0, 8, st));
    const unsigned lb_blocks = static_cast<unsigned>(std::min<uint64_t>((N + 255) / 256, sm_count() * 8ULL));
    k_last_below<<<lb_blocks, 256, 0, st>>>(b.cdf, N, b.nz);
    KT_CHECK_LAUNCH("k_last_below");
    k_seq_bound<<<1, 32, 0, st>>>(b.cdf, N, b.nz, b.bound);
    KT_CHECK_LAUNCH("k_seq_bound");
    k_seq_search<<<shot_blocks, 128, 0, st>>>(b.cdf, N, b.bound, b.canon, b.n_shots, b.out);
    KT_CHECK_LAUNCH("k_seq_search");
    return KT_OK;
}

// The sampler over N probabilities: the state's own (|a_i|^2 with its noise)
// or, with host_probs, a caller's vector uploaded as it is.
int32_t sample_core(State& s, uint64_t N, const double* host_probs, const double* noise, const double* canonicals,
                    int64_t n_shots, uint64_t* out, int32_t mode, int32_t* n_rescanned)
{
    if (n_rescanned) {
        *n_rescanned = 0;
    }
    if (n_shots <= 0) {
        return KT_OK;
    }
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
    const uint64_t n_xt = (N + XS_TILE - 1) / XS_TILE;
    const size_t off_tsum = al(off_bound + 8);
    const size_t off_code = al(off_tsum + n_xt * 8);
    const size_t off_ints = al(off_code + n_xt * 4);
    const size_t off_carry = al(off_ints + n_xt * 8);
    const size_t off_tstart = al(off_carry + n_xt * 8);
    const size_t off_hit = al(off_tstart + (n_xt + 1) * 8);
    const size_t off_list = al(off_hit + n_xt * 4);
    const size_t off_count = al(off_list + n_xt * 8);
    const size_t off_stile = al(off_count + 8);
    const size_t off_cints = al(off_stile + ns * 8);
    const size_t off_cflag = al(off_cints + n_xt * N_CAND * 8);
    const size_t off_tie = al(off_cflag + n_xt * 4);
    const size_t off_runs = al(off_tie + n_xt * 4);
    const size_t off_runc = al(off_runs + n_xt * 8);
    const size_t off_tlist = al(off_runc + n_xt * 4);
    const size_t off_tcount = al(off_tlist + n_xt * 8);
    if (const int32_t rc = s.scratch.reserve(off_tcount + 8); rc != KT_OK) {
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
    auto* d_tsum = reinterpret_cast<double*>(base + off_tsum);
    auto* d_code = reinterpret_cast<int*>(base + off_code);
    auto* d_ints = reinterpret_cast<unsigned long long*>(base + off_ints);
    auto* d_carry = reinterpret_cast<double*>(base + off_carry);
    auto* d_tstart = reinterpret_cast<double*>(base + off_tstart);
    auto* d_hit = reinterpret_cast<int*>(base + off_hit);
    auto* d_list = reinterpret_cast<unsigned long long*>(base + off_list);
    auto* d_count = reinterpret_cast<unsigned int*>(base + off_count);
    auto* d_stile = reinterpret_cast<unsigned long long*>(base + off_stile);
    auto* d_cints = reinterpret_cast<unsigned long long*>(base + off_cints);
    auto* d_cflag = reinterpret_cast<int*>(base + off_cflag);
    auto* d_tie = reinterpret_cast<int*>(base + off_tie);
    auto* d_runs = reinterpret_cast<unsigned long long*>(base + off_runs);
    auto* d_runc = reinterpret_cast<int*>(base + off_runc);
    auto* d_tlist = reinterpret_cast<unsigned long long*>(base + off_tlist);
    auto* d_tcount = reinterpret_cast<unsigned int*>(base + off_tcount);

    // the exact tier straight away (above the fast tier's size) on the state's
    // own noiseless probabilities: their pass forms the tile sums and the
    // candidate integer sums, and stores no probabilities
    const bool fused_tiles = host_probs == nullptr && noise == nullptr && !(mode == 0 && N <= (uint64_t {1} << 22));
    if (host_probs != nullptr) {
        if (const int32_t rc = copy_h2d(dp, host_probs, N * 8, s.stream); rc != KT_OK) {
            return rc;
        }
    } else if (fused_tiles) {
        const unsigned nt = static_cast<unsigned>((N + XS_TILE - 1) / XS_TILE);
        if (s.dtype == KT_C128) {
            k_probs_tiles<double2><<<nt, 256, 0, s.stream>>>(static_cast<const double2*>(s.amps), N, d_tsum, d_cints,
                                                             d_cflag);
        } else {
            k_probs_tiles<float2><<<nt, 256, 0, s.stream>>>(static_cast<const float2*>(s.amps), N, d_tsum, d_cints,
                                                            d_cflag);
        }
        KT_CHECK_LAUNCH("k_probs_tiles");
    } else if (const int32_t rc = device_probabilities(s, noise, dp); rc != KT_OK) {
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
        const uint64_t n_tiles = (N + XS_TILE - 1) / XS_TILE;
        if (!fused_tiles) {
            k_tile_sums<<<static_cast<unsigned>(n_tiles), 256, 0, s.stream>>>(dp, N, d_tsum);
            KT_CHECK_LAUNCH("k_tile_sums");
        }
        KT_CUDA(cudaMemsetAsync(d_tcount, 0, 4, s.stream));
        const int n_cand = !fused_tiles ? 0 : (s.dtype == KT_C128 ? cand_count<double2>() : cand_count<float2>());
        k_tile_guess<<<1, XS_THREADS, 0, s.stream>>>(d_tsum, n_tiles, d_code, fused_tiles ? d_cints : nullptr, d_cflag,
                                                     d_ints, d_tie, d_tlist, d_tcount, n_cand);
        KT_CHECK_LAUNCH("k_tile_guess");
        const ExactBufs xb {N,      n_tiles, n_shots, d_code,  d_ints,  d_carry, d_tstart, dcdf,   d_hit,
                            d_list, d_count, d_stile, d_tie,   d_runs,  d_runc,  d_tlist,  d_tcount, d_nz,
                            d_bound, d_canon, d_out};
        int32_t rc = KT_OK;
        if (!fused_tiles) {
            rc = exact_tail(s.stream, ProbVec {dp}, xb, 0, host_probs == nullptr);
        } else if (s.dtype == KT_C128) {
            rc = exact_tail(s.stream, ProbAmps<double2> {static_cast<const double2*>(s.amps)}, xb, n_cand, true);
        } else {
            rc = exact_tail(s.stream, ProbAmps<float2> {static_cast<const float2*>(s.amps)}, xb, n_cand, true);
        }
        if (rc != KT_OK) {
            return rc;
        }
        if (n_rescanned) {
            *n_rescanned = 1;
        }
    }
    return copy_d2h(out, d_out, ns * 8, s.stream);
}

}  // namespace

int32_t sample(State& s, const double* noise, const double* canonicals, int64_t n_shots, uint64_t* out, int32_t mode,
               int32_t* n_rescanned)
{
    return sample_core(s, s.n_amps(), nullptr, noise, canonicals, n_shots, out, mode, n_rescanned);
}

int32_t sample_from_probabilities(State& s, const double* host_probs, uint64_t n, const double* canonicals,
                                  int64_t n_shots, uint64_t* out, int32_t mode, int32_t* n_rescanned)
{
    return sample_core(s, n, host_probs, nullptr, canonicals, n_shots, out, mode, n_rescanned);
}

}  // namespace kt
