// kt_dm_ops.cu — density-matrix operations after propagation: partial trace,
// tensor product, and the trace of rho^2 (purity).
//
// Layout: a density matrix of n qubits is 2^(2n) amplitudes in the element
// order r + c * 2^n (row bits 0..n-1, column bits n..2n-1), complex128 or
// complex64 (FP64 arithmetic in both).
//
// Partial trace.  The reference traces one qubit at a time, the highest index
// first (state/density_matrix.cpp:231-278):
//     reduced(r', c') = current(r, c) + current(r + 2^q, c + 2^q),
// r, c = r', c' with a 0 inserted at bit q.  Over k traced qubits the result
// is a sum of 2^k diagonal blocks, grouped as that sequence of pairwise sums:
// the innermost pairs differ in the first qubit traced, the outermost in the
// last.  Each output element's 2^k leaves are added in that same tree order
// (pairwise stacks over aligned subtrees, then the subtrees pairwise), so the
// sums round like the reference's sequence of reduced matrices.  When few
// outputs remain, up to 32 warps share one warp of outputs, one subtree each.  Each leaf is one
// gathered element; rows and columns share the traced bits, so a launch reads
// 4^m 2^k elements and writes 4^m (m = n - k).
//
// Tensor product (state/density_matrix.cpp:187-214): the left factor's qubits
// are the low ones, out(r, c) = L(r mod A, c mod A) * R(r / A, c / A).
//
// Trace of rho^2 (state/density_matrix.cpp, trace_of_square: (rho * rho).trace()
// with Eigen): sum_ij rho(i, j) rho(j, i).  The product is symmetric in (i, j),
// so 32x32 tiles on and above the tile diagonal are read once each, the
// off-diagonal ones counted twice, and the transposed partner is read through
// shared memory so every global read is coalesced.
#include <algorithm>
#include <vector>

#include "kt_complex.cuh"
#include "kt_internal.cuh"

namespace kt
{

namespace
{

constexpr int DM_THREADS = 256;
constexpr int DM_PT_MAX_THREADS = 1024;
constexpr int DM_MAX_QUBITS = 17;

// bit positions handed to the partial-trace kernel
struct TraceMap
{
    int8_t keep[DM_MAX_QUBITS];    // kept qubits, ascending: bit j of r' goes to keep[j]
    int8_t traced[DM_MAX_QUBITS];  // traced qubits, in trace order: bit j of the leaf counter
    int32_t m;                     // kept qubits
    int32_t k;                     // traced qubits
};

// 256-entry lookup: the 8 bits of x placed at pos[base .. base + 7]
__device__ __forceinline__ uint32_t spread8(uint32_t x, const int8_t* pos, int base, int count)
{
    uint32_t v = 0;
    for (int b = 0; b < 8; ++b) {
        const int j = base + b;
        if (j < count && ((x >> b) & 1U) != 0U) {
            v |= 1U << pos[j];
        }
    }
    return v;
}

// Sum of the leaves lo .. lo + count - 1 (count a power of 2, lo a multiple
// of it): one subtree of the reference's grouping, by a pairwise stack.
template <typename C>
__device__ __forceinline__ double2 trace_subtree(const C* __restrict__ rho, int n, uint64_t base, uint32_t lo,
                                                 uint32_t count, int levels, const uint32_t (*tr_tab)[256])
{
    double2 stack[DM_MAX_QUBITS + 1];
    double2 acc = make_double2(0.0, 0.0);
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t t = lo + i;
        const uint64_t off = tr_tab[0][t & 255U] | tr_tab[1][(t >> 8) & 255U] | tr_tab[2][t >> 16];
        double2 v = to_d2(rho[base + off + (off << n)]);
        int j = 0;
        while (((i >> j) & 1U) != 0U) {
            v.x = stack[j].x + v.x;
            v.y = stack[j].y + v.y;
            ++j;
        }
        if (j < levels) {
            stack[j] = v;
        } else {
            acc = v;
        }
    }
    return acc;
}

// Thread layout: lanes = 32 consecutive output elements; a block holds
// `out_warps` such warps of outputs times G = 2^g leaf groups (warp w: group
// w % G, output warp w / G).  Group j sums the leaves j 2^(k-g) .. (j+1) 2^(k-g) - 1
// (the subtrees under the top g tree levels), and the G partials are then
// added pairwise in tree order, so the grouping stays the reference's.
template <typename C>
__global__ void __launch_bounds__(DM_PT_MAX_THREADS)
    k_partial_trace(const C* __restrict__ rho, int n, TraceMap map, int g, C* __restrict__ out)
{
    __shared__ uint32_t keep_tab[2][256];
    __shared__ uint32_t tr_tab[3][256];
    __shared__ double2 part[DM_PT_MAX_THREADS];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        keep_tab[0][i] = spread8(static_cast<uint32_t>(i), map.keep, 0, map.m);
        keep_tab[1][i] = spread8(static_cast<uint32_t>(i), map.keep, 8, map.m);
        tr_tab[0][i] = spread8(static_cast<uint32_t>(i), map.traced, 0, map.k);
        tr_tab[1][i] = spread8(static_cast<uint32_t>(i), map.traced, 8, map.k);
        tr_tab[2][i] = spread8(static_cast<uint32_t>(i), map.traced, 16, map.k);
    }
    __syncthreads();

    const int m = map.m;
    const int k = map.k;
    const int G = 1 << g;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int group = warp & (G - 1);
    const int out_warp = warp >> g;
    const int out_warps = (blockDim.x >> 5) >> g;
    const uint64_t n_out = uint64_t {1} << (2 * m);
    const uint64_t M = uint64_t {1} << m;
    const uint32_t per_group = 1U << (k - g);
    const uint64_t chunk = 32ULL * out_warps;
    for (uint64_t o0 = (uint64_t)blockIdx.x * chunk; o0 < n_out; o0 += (uint64_t)gridDim.x * chunk) {
        const uint64_t o = o0 + (uint64_t)out_warp * 32 + lane;
        double2 v = make_double2(0.0, 0.0);
        if (o < n_out) {
            const uint32_t rr = static_cast<uint32_t>(o & (M - 1));
            const uint32_t cc = static_cast<uint32_t>(o >> m);
            const uint64_t row = keep_tab[0][rr & 255U] | keep_tab[1][rr >> 8];
            const uint64_t col = keep_tab[0][cc & 255U] | keep_tab[1][cc >> 8];
            v = trace_subtree(rho, n, row + (col << n), static_cast<uint32_t>(group) * per_group, per_group, k - g,
                              tr_tab);
        }
        if (G == 1) {
            if (o < n_out) {
                out[o] = from_d2<C>(v);
            }
            continue;
        }
        part[threadIdx.x] = v;
        __syncthreads();
        if (group == 0 && o < n_out) {
            // partial of group j sits at warp (out_warp * G + j)
            double2 vals[32];
            for (int j = 0; j < G; ++j) {
                vals[j] = part[((out_warp << g) + j) * 32 + lane];
            }
            for (int step = 1; step < G; step <<= 1) {
                for (int j = 0; j < G; j += 2 * step) {
                    vals[j].x = vals[j].x + vals[j + step].x;
                    vals[j].y = vals[j].y + vals[j + step].y;
                }
            }
            out[o] = from_d2<C>(vals[0]);
        }
        __syncthreads();
    }
}

template <typename C>
__global__ void __launch_bounds__(DM_THREADS)
    k_tensor_product(const C* __restrict__ left, int nl, const C* __restrict__ right, int nr, C* __restrict__ out)
{
    const int n = nl + nr;
    const uint64_t n_out = uint64_t {1} << (2 * n);
    const uint64_t D = uint64_t {1} << n;
    const uint64_t A = uint64_t {1} << nl;
    const uint64_t B = uint64_t {1} << nr;
    for (uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; o < n_out; o += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = o & (D - 1);
        const uint64_t c = o >> n;
        const double2 a = to_d2(left[(r & (A - 1)) + ((c & (A - 1)) << nl)]);
        const double2 b = to_d2(right[(r >> nl) + ((c >> nl) * B)]);
        out[o] = from_d2<C>(make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x));
    }
}

constexpr int TS = 32;  // trace-of-square tile side

// One tile pair (bi <= bj) per block step; partial sums per block.
template <typename C>
__global__ void __launch_bounds__(DM_THREADS)
    k_trace_square(const C* __restrict__ rho, int n, double* __restrict__ partial)
{
    __shared__ double2 tile[TS][TS + 1];
    __shared__ double red[2][DM_THREADS / 32];
    const uint64_t N = uint64_t {1} << n;
    const uint64_t T = (N + TS - 1) / TS;  // tiles per side
    const int tx = threadIdx.x & (TS - 1);
    const int ty = threadIdx.x / TS;       // 0..7
    double sre = 0.0, sim = 0.0;
    for (uint64_t p = blockIdx.x; p < T * T; p += gridDim.x) {
        // p -> (bi, bj); the pairs below the tile diagonal are counted by their mirror
        const uint64_t bi = p / T;
        const uint64_t bj = p % T;
        if (bi > bj) {
            continue;
        }
        const double w = (bi == bj) ? 1.0 : 2.0;
        __syncthreads();
        // tile (bj, bi): rows bj*TS.., columns bi*TS..; element (r, c) at r + c N
        for (int yy = ty; yy < TS; yy += DM_THREADS / TS) {
            const uint64_t r = bj * TS + tx;
            const uint64_t c = bi * TS + yy;
            tile[yy][tx] = (r < N && c < N) ? to_d2(rho[r + c * N]) : make_double2(0.0, 0.0);
        }
        __syncthreads();
        // rho(i, j) for i in tile row bi, j in tile column bj, times rho(j, i) = tile[i][j]
        for (int yy = ty; yy < TS; yy += DM_THREADS / TS) {
            const uint64_t i = bi * TS + tx;
            const uint64_t j = bj * TS + yy;
            if (i < N && j < N) {
                const double2 a = to_d2(rho[i + j * N]);
                const double2 b = tile[tx][yy];
                sre += w * (a.x * b.x - a.y * b.y);
                sim += w * (a.x * b.y + a.y * b.x);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sre += __shfl_down_sync(0xffffffffU, sre, o);
        sim += __shfl_down_sync(0xffffffffU, sim, o);
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = sre;
        red[1][warp] = sim;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < DM_THREADS / 32; ++q) {
            a += red[0][q];
            b += red[1][q];
        }
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
    }
}

int dm_blocks(uint64_t work)
{
    const uint64_t want = (work + DM_THREADS - 1) / DM_THREADS;
    const uint64_t cap = static_cast<uint64_t>(sm_count()) * 8;
    return static_cast<int>(std::max<uint64_t>(1, std::min(want, cap)));
}

}  // namespace

int32_t dm_partial_trace(const State& src, int n, const int32_t* traced, int k, State& dst)
{
    TraceMap map {};
    map.m = n - k;
    map.k = k;
    uint32_t mask = 0;
    for (int j = 0; j < k; ++j) {
        map.traced[j] = static_cast<int8_t>(traced[j]);
        mask |= 1U << traced[j];
    }
    int jm = 0;
    for (int q = 0; q < n; ++q) {
        if (((mask >> q) & 1U) == 0U) {
            map.keep[jm++] = static_cast<int8_t>(q);
        }
    }
    // leaf groups per output: enough threads to fill the GPU when few outputs
    // remain (G = 2^g <= 32, at most 2^k), 256-thread blocks up to G = 8
    const uint64_t n_out = uint64_t {1} << (2 * map.m);
    const uint64_t want_threads = static_cast<uint64_t>(sm_count()) * 2048;
    int g = 0;
    while (g < 5 && g < k && n_out * (uint64_t {1} << g) < want_threads) {
        ++g;
    }
    const int G = 1 << g;
    const int out_warps = G <= 8 ? 8 / G : 1;
    const int threads = 32 * out_warps * G;
    const uint64_t chunk = 32ULL * out_warps;
    const uint64_t want_blocks = (n_out + chunk - 1) / chunk;
    const int blocks = static_cast<int>(std::max<uint64_t>(
        1, std::min<uint64_t>(want_blocks, static_cast<uint64_t>(sm_count()) * (2048 / threads))));
    if (src.dtype == KT_C128) {
        k_partial_trace<double2><<<blocks, threads, 0, dst.stream>>>(static_cast<const double2*>(src.amps), n, map, g,
                                                                     static_cast<double2*>(dst.amps));
    } else {
        k_partial_trace<float2><<<blocks, threads, 0, dst.stream>>>(static_cast<const float2*>(src.amps), n, map, g,
                                                                    static_cast<float2*>(dst.amps));
    }
    KT_CHECK_LAUNCH("k_partial_trace");
    return KT_OK;
}

int32_t dm_tensor_product(const State& left, int nl, const State& right, int nr, State& dst)
{
    const uint64_t n_out = uint64_t {1} << (2 * (nl + nr));
    const int blocks = dm_blocks(n_out);
    if (dst.dtype == KT_C128) {
        k_tensor_product<double2><<<blocks, DM_THREADS, 0, dst.stream>>>(
            static_cast<const double2*>(left.amps), nl, static_cast<const double2*>(right.amps), nr,
            static_cast<double2*>(dst.amps));
    } else {
        k_tensor_product<float2><<<blocks, DM_THREADS, 0, dst.stream>>>(
            static_cast<const float2*>(left.amps), nl, static_cast<const float2*>(right.amps), nr,
            static_cast<float2*>(dst.amps));
    }
    KT_CHECK_LAUNCH("k_tensor_product");
    return KT_OK;
}

int32_t dm_trace_of_square(State& s, int n, double* out)
{
    const uint64_t N = uint64_t {1} << n;
    const uint64_t T = (N + TS - 1) / TS;
    const int blocks = static_cast<int>(std::min<uint64_t>(T * T, static_cast<uint64_t>(sm_count()) * 8));
    if (const int32_t rc = s.scratch.reserve(static_cast<size_t>(blocks) * 16); rc != KT_OK) {
        return rc;
    }
    double* d = static_cast<double*>(s.scratch.ptr);
    if (s.dtype == KT_C128) {
        k_trace_square<double2><<<blocks, DM_THREADS, 0, s.stream>>>(static_cast<const double2*>(s.amps), n, d);
    } else {
        k_trace_square<float2><<<blocks, DM_THREADS, 0, s.stream>>>(static_cast<const float2*>(s.amps), n, d);
    }
    KT_CHECK_LAUNCH("k_trace_square");
    std::vector<double> h(2 * static_cast<size_t>(blocks));
    if (const int32_t rc = copy_d2h(h.data(), d, h.size() * sizeof(double), s.stream); rc != KT_OK) {
        return rc;
    }
    double re = 0.0, im = 0.0;
    for (int b = 0; b < blocks; ++b) {
        re += h[2 * b];
        im += h[2 * b + 1];
    }
    out[0] = re;
    out[1] = im;
    return KT_OK;
}

}  // namespace kt
