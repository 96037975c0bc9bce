// kt_dense.cu — a dense unitary on the five lowest qubits of a complex64
// state as a GEMM on the fifth-generation tensor cores (tcgen05), with the
// operands split into TF32 parts so the product keeps about FP32 accuracy.
//
// The state, viewed as rows of 32 amplitudes (64 floats, re / im
// interleaved), is X (2^n / 32 rows x 64).  The unitary U (32 x 32 complex)
// acts on every row as the real 64 x 64 matrix M of its interleaved form:
// Y = X M.  One persistent CTA per SM walks tiles of 128 rows:
//   * a producer warp loads a tile as two TMA boxes (128 rows x 128 bytes
//     each, 128-byte swizzle: the K-major layout the MMA reads its A
//     operand in);
//   * 128 split threads rewrite the tile in place as its TF32 part
//     hi = x rounded to 10 mantissa bits (to nearest), and write the exact
//     remainder lo = x - hi beside it;
//   * one thread issues the MMAs D = hi Bhi + hi Blo + lo Bhi (three TF32
//     products accumulated in FP32 in tensor memory; passes = 4 adds
//     lo Blo, passes = 1 keeps only a plain TF32 product of the unsplit
//     tile), where B = M^T is stored K-major and split the same way on the
//     host;
//   * the 128 threads read D back from tensor memory (one row each), write
//     it over the tile in shared memory, and one of them stores the tile
//     with TMA.
// Four tile stages keep up to four tiles' loads in flight; two remainder
// buffers and two accumulators let one tile's split and MMAs overlap the
// previous tile's read-back, and a stage is handed back to the producer once
// its store has read it, one tile later.  Every wait is
// bounded (kt_mbar_wait): one that runs out sets the device error word, the
// kernel runs to its end without data, waits a bounded time for its own
// copies and products still in flight, frees its tensor memory, and the
// entry point reports KT_ERR_TIMEOUT.  Loads and stores use this GPU's own
// memory only; no copy uses cluster multicast.
//
// With hi rounded to nearest, |lo| <= 2^-11 |x| and the TF32 operand keeps
// 11 of its bits, so three products are exact to about 2^-22 of |x| |m|
// (the dropped lo Blo is of that size too) and four to about 2^-22 |x| |m|
// without the dropped term: close to an FP32 GEMM's error, which is what a
// complex64 state carries.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "kt_complex.cuh"
#include "kt_internal.cuh"
#include "kt_tma_dev.cuh"

namespace
{

using kt::KtTmap;

constexpr int DT_STAGES = 4;            // tile buffers (TMA ring; hi in place; the read-back's staging)
constexpr int DT_SLOTS = 2;             // remainder buffers and accumulators
constexpr int DT_THREADS = 192;         // producer warp, MMA warp, 4 split / read-back warps
constexpr int DT_ROWS = 128;            // rows per tile: the MMA's M
constexpr int DT_SUB = DT_ROWS * 128;   // one 128-row x 128-byte K slice of a tile (16 KB)
constexpr int DT_TILE = 2 * DT_SUB;     // a tile: 128 rows x 64 floats (32 KB)
constexpr int DT_BSUB = 64 * 128;       // one 64-row K slice of B (8 KB)
constexpr int DT_B = 2 * DT_BSUB;       // B: 64 x 64 floats (16 KB)
constexpr uint32_t DT_TMEM_COLS = 128;  // two 64-column FP32 accumulators
// shared memory from a 1024-byte aligned base
constexpr int OFF_BHI = 0;
constexpr int OFF_BLO = DT_B;
constexpr int OFF_A = 2 * DT_B;
constexpr int OFF_L = OFF_A + DT_STAGES * DT_TILE;
constexpr int OFF_BAR = OFF_L + DT_SLOTS * DT_TILE;
constexpr int DT_SMEM = OFF_BAR + (2 * DT_STAGES + 2 * DT_SLOTS) * 8 + 16 + 1024;  // barriers, TMEM address, alignment

// instruction descriptor of tcgen05.mma kind::tf32: D in FP32, A and B TF32
// and K-major, N = 64 (bits 17-22: N / 8), M = 128 (bits 24-28: M / 16)
constexpr uint32_t DT_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// Shared-memory matrix descriptor of a K-major operand in 128-byte swizzled
// rows (the layout a SWIZZLE_128B TMA box lands in): start address / 16,
// leading offset unused by this layout (1), 8-row groups 1024 bytes apart,
// descriptor version 1, swizzle mode 2 (128 bytes).  Stepping K by 8 TF32
// inside a 128-byte row adds 32 bytes to the start address.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    uint64_t d = static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
    d |= uint64_t {1} << 16;
    d |= uint64_t {1024 >> 4} << 32;
    d |= uint64_t {1} << 46;
    d |= uint64_t {2} << 61;
    return d;
}

__device__ __forceinline__ void tc_fence_before()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// whole warp: allocate `cols` columns of tensor memory, the address lands in *slot
__device__ __forceinline__ void tc_alloc(uint32_t* slot, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(kt::kt_smem_u32(slot)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// one thread: D (+)= A B^T over K = 8
__device__ __forceinline__ void tc_mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile(
        "{\n"
        "    .reg .pred p;\n"
        "    setp.ne.b32 p, %4, 0;\n"
        "    tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n"
        "}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(DT_IDESC), "r"(accumulate)
        : "memory");
}

// `bar` completes one arrival once every MMA this thread issued so far has completed
__device__ __forceinline__ void tc_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     kt::kt_smem_u32(bar))
                 : "memory");
}

// whole warp: 16 consecutive FP32 columns of the warp's 32 tensor-memory lanes, one lane per thread
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t* v)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tc_wait_ld()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// a bounded wait that ignores the error word: the drain at the end
__device__ __forceinline__ void drain_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t addr = kt::kt_smem_u32(bar);
    const unsigned long long t0 = kt::kt_globaltimer();
#pragma unroll 1
    while (!kt::kt_mbar_try_wait(addr, parity)) {
        if (kt::kt_globaltimer() - t0 > 200000000ull) {
            return;
        }
    }
}

// x rounded to a TF32 value (10 mantissa bits, to nearest, ties away from zero)
__device__ __forceinline__ float tf32_hi(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__global__ void __launch_bounds__(DT_THREADS, 1)
    k_dense5_tc(const __grid_constant__ KtTmap tm, const float* __restrict__ bmat, uint64_t n_tiles, int passes,
                unsigned int* __restrict__ err)
{
    extern __shared__ unsigned char dt_raw[];
    const uint32_t raw = kt::kt_smem_u32(dt_raw);
    unsigned char* sm = dt_raw + ((1024u - (raw & 1023u)) & 1023u);
    auto* full = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
    uint64_t* empty = full + DT_STAGES;
    uint64_t* split = empty + DT_STAGES;
    uint64_t* mmad = split + DT_SLOTS;
    auto* tslot = reinterpret_cast<uint32_t*>(mmad + DT_SLOTS);
    const int warp = static_cast<int>(threadIdx.x >> 5);
    const int lane = static_cast<int>(threadIdx.x & 31);
    // B (hi, then lo; row n holds 64 floats over k) into the swizzled K-major layout
    for (int e = static_cast<int>(threadIdx.x); e < 2 * 64 * 16; e += DT_THREADS) {
        const int mat = e >> 10;
        const int n = (e >> 4) & 63;
        const int c16 = e & 15;
        const float4 v = reinterpret_cast<const float4*>(bmat)[e];
        const int off = mat * DT_B + (c16 >> 3) * DT_BSUB + n * 128 + (((c16 & 7) ^ (n & 7)) << 4);
        *reinterpret_cast<float4*>(sm + off) = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < DT_STAGES; ++s) {
            kt::kt_mbar_init(&full[s], 1);
            kt::kt_mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < DT_SLOTS; ++s) {
            kt::kt_mbar_init(&split[s], 128);
            kt::kt_mbar_init(&mmad[s], 1);
        }
        kt::kt_fence_mbar_init();
    }
    if (warp == 1) {
        tc_alloc(tslot, DT_TMEM_COLS);
    }
    kt::kt_fence_proxy_async_smem();  // B, written by these threads, is read by the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint64_t mine = n_tiles > blockIdx.x ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    if (warp == 0) {
        if (lane == 0) {
            for (uint64_t i = 0; i < mine; ++i) {
                const int s = static_cast<int>(i % DT_STAGES);
                if (i >= DT_STAGES) {
                    kt::kt_mbar_wait(&empty[s], static_cast<uint32_t>((i / DT_STAGES - 1) & 1), err);
                }
                kt::kt_mbar_arrive_expect_tx(&full[s], DT_TILE);
                const int32_t row = static_cast<int32_t>((blockIdx.x + i * gridDim.x) * DT_ROWS);
                const int32_t c0[2] = {0, row};
                const int32_t c1[2] = {32, row};
                kt::KtTma<2>::load(&tm, sm + OFF_A + s * DT_TILE, &full[s], c0);
                kt::KtTma<2>::load(&tm, sm + OFF_A + s * DT_TILE + DT_SUB, &full[s], c1);
            }
            // the copies still in flight (any, only after a wait ran out) land before the CTA ends
            for (uint64_t i = mine > DT_STAGES ? mine - DT_STAGES : 0; i < mine; ++i) {
                drain_wait(&full[i % DT_STAGES], static_cast<uint32_t>((i / DT_STAGES) & 1));
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t a0 = kt::kt_smem_u32(sm + OFF_A);
            const uint32_t l0 = kt::kt_smem_u32(sm + OFF_L);
            const uint32_t bh = kt::kt_smem_u32(sm + OFF_BHI);
            const uint32_t bl = kt::kt_smem_u32(sm + OFF_BLO);
            for (uint64_t i = 0; i < mine; ++i) {
                const int s = static_cast<int>(i % DT_STAGES);
                const int h = static_cast<int>(i % DT_SLOTS);
                kt::kt_mbar_wait(&split[h], static_cast<uint32_t>((i / DT_SLOTS) & 1), err);
                tc_fence_after();
                const uint32_t d = tmem + static_cast<uint32_t>(h * 64);
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    // K = 64 in steps of 8: K slice k / 4, 32 bytes per step inside its 128-byte rows
                    const uint32_t ka = static_cast<uint32_t>((k >> 2) * DT_SUB + (k & 3) * 32);
                    const uint32_t kb = static_cast<uint32_t>((k >> 2) * DT_BSUB + (k & 3) * 32);
                    const uint64_t ahi = sw128_desc(a0 + static_cast<uint32_t>(s * DT_TILE) + ka);
                    const uint64_t bhi = sw128_desc(bh + kb);
                    tc_mma_tf32(d, ahi, bhi, k > 0 ? 1u : 0u);
                    if (passes >= 3) {
                        const uint64_t alo = sw128_desc(l0 + static_cast<uint32_t>(h * DT_TILE) + ka);
                        const uint64_t blo = sw128_desc(bl + kb);
                        tc_mma_tf32(d, ahi, blo, 1u);
                        tc_mma_tf32(d, alo, bhi, 1u);
                        if (passes == 4) {
                            tc_mma_tf32(d, alo, blo, 1u);
                        }
                    }
                }
                tc_commit(&mmad[h]);
            }
            // every product issued has completed before the tensor memory is freed
            if (mine > 0) {
                drain_wait(&mmad[(mine - 1) % DT_SLOTS], static_cast<uint32_t>(((mine - 1) / DT_SLOTS) & 1));
            }
        }
        __syncwarp();
    } else {
        const int et = static_cast<int>(threadIdx.x) - 64;  // 0..127
        const int q = warp & 3;                              // the tensor-memory lane quarter this warp reads
        const int r = q * 32 + lane;                         // the tile row this thread reads back
        const uint32_t lanes = tmem + (static_cast<uint32_t>(q * 32) << 16);
        auto split_tile = [&](uint64_t i) {
            const int s = static_cast<int>(i % DT_STAGES);
            kt::kt_mbar_wait(&full[s], static_cast<uint32_t>((i / DT_STAGES) & 1), err);
            if (passes >= 3) {
                auto* A = reinterpret_cast<float4*>(sm + OFF_A + s * DT_TILE);
                auto* L = reinterpret_cast<float4*>(sm + OFF_L + static_cast<int>(i % DT_SLOTS) * DT_TILE);
#pragma unroll 4
                for (int j = et; j < DT_TILE / 16; j += 128) {
                    const float4 x = A[j];
                    const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
                    A[j] = h;
                    L[j] = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
                }
                kt::kt_fence_proxy_async_smem();
            }
            tc_fence_before();
            kt::kt_mbar_arrive(&split[i % DT_SLOTS]);
        };
        auto read_back = [&](uint64_t i) {
            const int s = static_cast<int>(i % DT_STAGES);
            const uint32_t h = static_cast<uint32_t>(i % DT_SLOTS);
            kt::kt_mbar_wait(&mmad[h], static_cast<uint32_t>((i / DT_SLOTS) & 1), err);
            tc_fence_after();
            uint32_t v[64];
            tc_ld16(lanes + h * 64, v);
            tc_ld16(lanes + h * 64 + 16, v + 16);
            tc_ld16(lanes + h * 64 + 32, v + 32);
            tc_ld16(lanes + h * 64 + 48, v + 48);
            tc_wait_ld();
#pragma unroll
            for (int k = 0; k < 64; ++k) {
                asm volatile("" : "+r"(v[k]));  // no use of v moves above the wait
            }
            unsigned char* out = sm + OFF_A + s * DT_TILE;
#pragma unroll
            for (int c16 = 0; c16 < 16; ++c16) {
                const int off = (c16 >> 3) * DT_SUB + r * 128 + (((c16 & 7) ^ (r & 7)) << 4);
                *reinterpret_cast<uint4*>(out + off) = make_uint4(v[4 * c16], v[4 * c16 + 1], v[4 * c16 + 2], v[4 * c16 + 3]);
            }
            kt::kt_fence_proxy_async_smem();
            tc_fence_before();
            kt::kt_bar_sync(1, 128);
            if (et == 0) {
                const int32_t row = static_cast<int32_t>((blockIdx.x + i * gridDim.x) * DT_ROWS);
                const int32_t c0[2] = {0, row};
                const int32_t c1[2] = {32, row};
                kt::KtTma<2>::store(&tm, out, c0);
                kt::KtTma<2>::store(&tm, out + DT_SUB, c1);
                kt::kt_bulk_commit();
                // the previous tile's store has read its stage: hand that stage back
                asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                if (i > 0) {
                    kt::kt_mbar_arrive(&empty[(i - 1) % DT_STAGES]);
                }
            }
        };
        for (uint64_t i = 0; i < mine; ++i) {
            split_tile(i);
            if (i > 0) {
                read_back(i - 1);
            }
        }
        if (mine > 0) {
            read_back(mine - 1);
        }
        if (et == 0) {
            kt::kt_bulk_wait0();
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) {
        tc_dealloc(tmem, DT_TMEM_COLS);
    }
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
    } catch (...) {
        return fail(KT_ERR_INVALID, "unknown exception");
    }
}

}  // namespace

extern "C" int32_t kt_sv_apply_dense5(kt_sv sv, const double* u, int32_t passes)
{
    return guarded([&]() -> int32_t {
        if (sv == nullptr || u == nullptr) {
            return fail(KT_ERR_INVALID, "null argument");
        }
        kt::State& s = sv->st;
        if (s.dtype != KT_C64) {
            return fail(KT_ERR_INVALID, "kt_sv_apply_dense5: complex64 states only");
        }
        if (s.n_bits < 12 || s.n_bits > 34) {
            return fail(KT_ERR_QUBITS, "kt_sv_apply_dense5: the state must have 12 to 34 qubits");
        }
        if (passes != 1 && passes != 3 && passes != 4) {
            return fail(KT_ERR_INVALID, "kt_sv_apply_dense5: passes must be 1, 3 or 4");
        }
        // B[n][k] = M[k][n] (K-major), M the real form of U on interleaved rows:
        // re y_b = sum_a (Re U_ba re x_a - Im U_ba im x_a), im y_b = sum_a (Im U_ba re x_a + Re U_ba im x_a)
        std::vector<float> b(2 * 64 * 64);
        auto put = [&](int n, int k, double val) {
            const float f = static_cast<float>(val);
            uint32_t w = 0;
            std::memcpy(&w, &f, sizeof(w));
            w = (w + 0x1000u) & 0xFFFFE000u;  // to nearest TF32, ties away from zero (|val| <= 1)
            float hi = 0.0f;
            std::memcpy(&hi, &w, sizeof(hi));
            b[static_cast<size_t>(n * 64 + k)] = hi;
            b[static_cast<size_t>(4096 + n * 64 + k)] = static_cast<float>(val - static_cast<double>(hi));
        };
        for (int o = 0; o < 32; ++o) {
            for (int a = 0; a < 32; ++a) {
                const double ur = u[2 * (32 * o + a)];
                const double ui = u[2 * (32 * o + a) + 1];
                put(2 * o, 2 * a, ur);
                put(2 * o, 2 * a + 1, -ui);
                put(2 * o + 1, 2 * a, ui);
                put(2 * o + 1, 2 * a + 1, ur);
            }
        }
        if (passes == 1) {
            for (size_t k = 0; k < 4096; ++k) {
                b[k] = static_cast<float>(b[k] + b[4096 + k]);  // the plain product uses B as given
            }
        }
        if (const int32_t rc = s.scratch.reserve(b.size() * sizeof(float)); rc != KT_OK) {
            return rc;
        }
        if (const int32_t rc = kt::copy_h2d(s.scratch.ptr, b.data(), b.size() * sizeof(float), s.stream); rc != KT_OK) {
            return rc;
        }
        int dev = 0;
        KT_CUDA(cudaGetDevice(&dev));
        unsigned int* err_host = nullptr;
        unsigned int* err_dev = kt::async_error_word(dev, &err_host);
        if (err_dev == nullptr) {
            return fail(KT_ERR_CUDA, "kt_sv_apply_dense5: no device error word");
        }
        const uint64_t rows = (uint64_t {1} << s.n_bits) / 32;
        KtTmap tm {};
        if (!kt::tma_encode_rows_f32(s.amps, 64, rows, 32, DT_ROWS, &tm)) {
            return fail(KT_ERR_CUDA, "kt_sv_apply_dense5: cuTensorMapEncodeTiled failed");
        }
        static bool attr = false;
        if (!attr) {
            KT_CUDA(cudaFuncSetAttribute(k_dense5_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, DT_SMEM));
            attr = true;
        }
        const uint64_t n_tiles = rows / DT_ROWS;
        const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(n_tiles, static_cast<uint64_t>(kt::sm_count())));
        k_dense5_tc<<<grid, DT_THREADS, DT_SMEM, s.stream>>>(tm, static_cast<const float*>(s.scratch.ptr), n_tiles,
                                                              passes, err_dev);
        KT_CHECK_LAUNCH("k_dense5_tc");
        // the error word to the host once the kernel is done (read by the entry points' guard)
        KT_CUDA(cudaMemcpyAsync(err_host, err_dev, sizeof(unsigned int), cudaMemcpyDeviceToHost, s.stream));
        s.last_launches = 1;
        s.last_alg_bytes = 2.0 * 8.0 * std::ldexp(1.0, s.n_bits);
        return KT_OK;
    });
}
