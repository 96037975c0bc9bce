// kt_batch.cu — batches of independent circuits: energies and adjoint gradients.
//
// No reference counterpart (kettle evaluates one circuit at a time; its VQE
// loop, example/algorithms/vqe_basic.cpp:61-96, calls simulate and
// expectation_value once per cost evaluation).
//
// A batch is planned once.  Every item starts from |0...0>, runs its gates,
// and yields E_b = Re <psi_b| H_b |psi_b> and, with gradients on, the
// adjoint-method derivatives (forward, lambda = H psi, backward with one FP64
// inner product per parameterised gate).  Angles stay symbolic in the plan:
// an evaluation uploads the parameter vector and a kernel writes the matrices
// (and derivatives) of every parameterised op record in place.
//
// Items whose psi and lambda fit in shared memory (2^q amplitudes each;
// q <= 12 for complex128, q <= 13 for complex64) run in one persistent launch,
// one CTA per item at a time, taking items from an atomic queue (largest
// first); all of an item's work happens in shared memory.
//
// Larger items live in HBM (an arena holding psi and lambda of every item of
// a memory wave).  Their work is cut into jobs — the item's fused forward
// blocks, one Hamiltonian job (lambda = H psi and the energy), its fused
// adjoint blocks — and each job into units (ranges of tiles).  One persistent
// launch per wave serves a device queue of ready jobs: it starts with every
// item's first job (costliest chains first); a CTA takes the next unit of the
// oldest queued job that still has one, and the CTA that finishes a job's last
// unit appends the item's next job.  A CTA waits only while no job is ready
// (then every job in flight is being run by some CTA, which will queue its
// successor), so the waits end; they are bounded anyway and set an error
// status on expiry.
//
// The whole evaluation — parameter upload, matrix patching, the two
// persistent launches (on forked streams), FP64 finalisation, download — is
// one CUDA graph, captured when the batch is created and replayed by every
// evaluation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "kt_fused.cuh"

namespace kt
{

namespace
{

constexpr int B_THREADS = 256;
constexpr int BATCH_FWD_MAX_OPS = 256;   // ops per forward block
constexpr int BATCH_BWD_MAX_OPS = ADJ_MAX_OPS;  // ops (and gradient rows) per adjoint block
constexpr int UNITS_PER_JOB = 64;        // a job's tiles are cut into at most this many units
constexpr int HAM_SMEM_STRINGS = 512;    // strings staged in shared memory by a Hamiltonian unit
constexpr int HJ = 8;                    // amplitudes per thread per step of a Hamiltonian unit (B_THREADS * HJ
                                         // divides every chunk: 2^12 or 2^13 amplitudes)

enum : int32_t
{
    JOB_FWD = 0,
    JOB_HAM = 1,
    JOB_BWD = 2,
};

enum : int32_t
{
    TAB_FWD = 0,
    TAB_BWD = 1,
    TAB_SMALL = 2,
};

struct BJob
{
    int32_t kind;
    int32_t inst;            // HBM item (index into BInst)
    int32_t block;           // block index in the forward or adjoint table (-1 for JOB_HAM)
    int32_t n_units;
    int32_t tiles_per_unit;  // tiles (or Hamiltonian chunks) per unit
    int32_t succ;            // the item's next job, queued when this one's last unit is done (-1: none)
    int32_t n_rows;          // JOB_BWD: gradient rows of the block
    int32_t init;            // JOB_FWD: the item's first block starts from |0...0>
    int64_t part;            // JOB_BWD: part[part + r * n_units + u]; JOB_HAM: epart[part + u]
    int64_t n_tiles;         // tiles (chunks) of the item for this job's tile size
};

struct BInst
{
    int64_t psi;     // element offset of psi in the arena
    int64_t lam;     // element offset of lambda
    int32_t q;
    int32_t n_str;
    int64_t str;     // first string in the string table
};

// A Pauli term ready for the kernels: coefficient * i^(#Y + phase), so that
// (c P psi)[j] = (cr + i ci) (-1)^popcount((j ^ x) & z) psi[j ^ x].
struct BStr
{
    uint64_t x;
    uint64_t z;
    double cr;
    double ci;
};

// one op record whose matrix comes from a parameter
struct BPatch
{
    int32_t table;
    int32_t op;      // KT_OP_* of the gate
    int64_t index;   // record index in its table
    int64_t param;   // index into the parameter vector
    int32_t one_sided;  // the record is a one-sided diagonal diag(1, m11 / m00) (see one_sided_diagonals)
    int32_t pad;
};

struct RowSrc
{
    int64_t first;   // row value = 2 * sum of part[first .. first + count)
    int32_t count;
    int32_t pad;
};

struct ESrc
{
    int64_t first;   // energy = sum of epart[first .. first + count)
    int32_t count;
    int32_t pad;
    int64_t out;     // item index
};

// an op of a shared-memory item: U, U^dagger and dU/dtheta
template <typename T>
struct SOp
{
    int16_t kind;     // KIND_GEN / KIND_DIAG / KIND_ANTI
    int16_t target;
    int16_t control;  // -1: none
    int16_t pad;
    int32_t row;      // gradient row (-1: none)
    int32_t pad2;
    T u[8];
    T ua[8];
    T d[8];
};

struct SItem
{
    int32_t q;
    int32_t n_ops;
    int64_t op;       // first op
    int32_t n_str;
    int32_t pad;
    int64_t str;      // first string
    int64_t out;      // item index
};

template <typename T>
struct BArgs
{
    typename CxT<T>::type* arena;
    const BJob* jobs;
    const BInst* insts;
    int* queue;               // ready jobs in the order they became ready (-1: slot not written yet)
    int n_jobs;               // jobs of this wave: every one enters the queue exactly once
    const FBlock* fblk;
    const FPhase* fph;
    const FOp<T>* fops;
    const FBlock* bblk;
    const FPhase* bph;
    const FOpA<T>* bops;
    const BStr* strs;
    double* part;
    double* epart;
    int* done;
    unsigned long long* qhead;  // first queue slot whose job may still have units to hand out
    unsigned long long* qtail;  // queue slots reserved so far
    int* taken;                 // per job: units handed out
    int* status;
    int with_grad;
    long long spin_limit;       // polls of an empty queue before the CTA gives up (batch_spin_limit)
};

// ---------------------------------------------------------------------------
// device helpers

// The block-wide sum of v (256 threads), the same value in every thread.
__device__ __forceinline__ double block_sum(double v, double* sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_down_sync(0xffffffffU, v, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5] = v;
    }
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < B_THREADS / 32; ++w) {
        s += sh[w];
    }
    return s;
}

// U and dU/dtheta of a rotation gate (the matrices of gates/common_u_gates.cpp)
__device__ void rotation(int op, double th, double* u, double* d)
{
    for (int e = 0; e < 8; ++e) {
        u[e] = 0.0;
        d[e] = 0.0;
    }
    double s, c;
    sincos(0.5 * th, &s, &c);
    switch (op) {
        case KT_OP_RX: case KT_OP_CRX:
            u[0] = c; u[3] = -s; u[5] = -s; u[6] = c;
            d[0] = -0.5 * s; d[3] = -0.5 * c; d[5] = -0.5 * c; d[6] = -0.5 * s;
            break;
        case KT_OP_RY: case KT_OP_CRY:
            u[0] = c; u[2] = -s; u[4] = s; u[6] = c;
            d[0] = -0.5 * s; d[2] = -0.5 * c; d[4] = 0.5 * c; d[6] = -0.5 * s;
            break;
        case KT_OP_RZ: case KT_OP_CRZ:
            u[0] = c; u[1] = -s; u[6] = c; u[7] = s;
            d[0] = -0.5 * s; d[1] = -0.5 * c; d[6] = -0.5 * s; d[7] = 0.5 * c;
            break;
        default: {  // KT_OP_P, KT_OP_CP
            double sp, cp;
            sincos(th, &sp, &cp);
            u[0] = 1.0; u[6] = cp; u[7] = sp;
            d[6] = -sp; d[7] = cp;
            break;
        }
    }
}

template <typename T>
__global__ void k_batch_patch(const double* __restrict__ params, const BPatch* __restrict__ patches, int64_t n,
                              FOp<T>* __restrict__ fops, FOpA<T>* __restrict__ bops, SOp<T>* __restrict__ sops)
{
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const BPatch p = patches[i];
    double u[8], d[8];
    rotation(p.op, params[p.param], u, d);
    const double ua[8] = {u[0], -u[1], u[4], -u[5], u[2], -u[3], u[6], -u[7]};
    if (p.one_sided != 0) {
        // diag(u00, u11) as diag(1, u11 / u00); |u00| = 1 (RZ, P): U^dagger the conjugates
        const double r = u[6] * u[0] + u[7] * u[1];
        const double i = u[7] * u[0] - u[6] * u[1];
        T* m = (p.table == TAB_FWD) ? fops[p.index].m : bops[p.index].m;
        const double one[8] = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, r, (p.table == TAB_FWD) ? i : -i};
        for (int e = 0; e < 8; ++e) {
            m[e] = static_cast<T>(one[e]);
        }
    } else if (p.table == TAB_FWD) {
        for (int e = 0; e < 8; ++e) {
            fops[p.index].m[e] = static_cast<T>(u[e]);
        }
    } else if (p.table == TAB_BWD) {
        for (int e = 0; e < 8; ++e) {
            bops[p.index].m[e] = static_cast<T>(ua[e]);
        }
    } else {
        for (int e = 0; e < 8; ++e) {
            sops[p.index].u[e] = static_cast<T>(u[e]);
            sops[p.index].ua[e] = static_cast<T>(ua[e]);
            sops[p.index].d[e] = static_cast<T>(d[e]);
        }
    }
}

template <typename C, typename T>
__device__ __forceinline__ void pair_apply(C& a, C& b, int kind, const T* m)
{
    const C m00 = make_cx<T>(m[0], m[1]), m01 = make_cx<T>(m[2], m[3]);
    const C m10 = make_cx<T>(m[4], m[5]), m11 = make_cx<T>(m[6], m[7]);
    if (kind == KIND_GEN) {
        const C x = cfma(m01, b, cmul(m00, a));
        const C y = cfma(m11, b, cmul(m10, a));
        a = x;
        b = y;
    } else if (kind == KIND_ANTI) {
        const C x = cmul(m01, b);
        const C y = cmul(m10, a);
        a = x;
        b = y;
    } else {
        a = cmul(m00, a);
        b = cmul(m11, b);
    }
}

// lowest index of pair k of a gate on (target, control): the target bit is 0,
// the control bit (if any) is 1
__device__ __forceinline__ int pair_index(int k, int tq, int cq)
{
    if (cq < 0) {
        return static_cast<int>(insert_zero_bit(static_cast<uint64_t>(k), tq));
    }
    const int lo = min(cq, tq), hi = max(cq, tq);
    return static_cast<int>(insert_zero_bit(insert_zero_bit(static_cast<uint64_t>(k), lo), hi)) | (1 << cq);
}

// ---------------------------------------------------------------------------
// items in shared memory: one CTA runs an item's whole evaluation
template <typename T>
__global__ void __launch_bounds__(B_THREADS) k_batch_small(const SItem* __restrict__ items, int n_items,
                                                           const SOp<T>* __restrict__ ops, const BStr* __restrict__ strs,
                                                           double* __restrict__ energies, double* __restrict__ rowval,
                                                           int with_grad, unsigned int* __restrict__ counter)
{
    using C = typename CxT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[B_THREADS / 32];
    __shared__ int item_sh;
    const int t = threadIdx.x;
    while (true) {
        if (t == 0) {
            item_sh = static_cast<int>(atomicAdd(counter, 1u));
        }
        __syncthreads();
        const int it = item_sh;
        __syncthreads();
        if (it >= n_items) {
            break;
        }
        const SItem bi = items[it];
        const int N = 1 << bi.q;
        C* psi = reinterpret_cast<C*>(smem_raw);
        C* lam = psi + N;
        for (int i = t; i < N; i += B_THREADS) {
            psi[i] = make_cx<T>(i == 0 ? T(1) : T(0), T(0));
        }
        __syncthreads();
        const SOp<T>* op = ops + bi.op;
        for (int g = 0; g < bi.n_ops; ++g) {
            const int kind = op[g].kind, tq = op[g].target, cq = op[g].control;
            const int npairs = (cq >= 0) ? (N >> 2) : (N >> 1);
            for (int k = t; k < npairs; k += B_THREADS) {
                const int i0 = pair_index(k, tq, cq);
                C a = psi[i0], b = psi[i0 | (1 << tq)];
                pair_apply<C, T>(a, b, kind, op[g].u);
                psi[i0] = a;
                psi[i0 | (1 << tq)] = b;
            }
            __syncthreads();
        }
        // lambda = H psi and E = Re <psi|lambda>
        const BStr* st = strs + bi.str;
        double e = 0.0;
        for (int j = t; j < N; j += B_THREADS) {
            double lr = 0.0, li = 0.0;
            for (int s = 0; s < bi.n_str; ++s) {
                const BStr bs = st[s];
                const int src = j ^ static_cast<int>(bs.x);
                const double sg = (__popcll(static_cast<uint64_t>(src) & bs.z) & 1) ? -1.0 : 1.0;
                const double2 p = to_d2(psi[src]);
                lr += sg * (bs.cr * p.x - bs.ci * p.y);
                li += sg * (bs.cr * p.y + bs.ci * p.x);
            }
            const double2 pj = to_d2(psi[j]);
            e += pj.x * lr + pj.y * li;
            if (with_grad) {
                lam[j] = make_cx<T>(static_cast<T>(lr), static_cast<T>(li));
            }
        }
        e = block_sum(e, red);
        if (t == 0) {
            energies[bi.out] = e;
        }
        if (with_grad) {
            __syncthreads();
            for (int g = bi.n_ops - 1; g >= 0; --g) {
                const int kind = op[g].kind, tq = op[g].target, cq = op[g].control;
                const int npairs = (cq >= 0) ? (N >> 2) : (N >> 1);
                const int row = op[g].row;
                double acc = 0.0;
                for (int k = t; k < npairs; k += B_THREADS) {
                    const int i0 = pair_index(k, tq, cq);
                    const int i1 = i0 | (1 << tq);
                    C a = psi[i0], b = psi[i1];
                    pair_apply<C, T>(a, b, kind, op[g].ua);
                    C la = lam[i0], lb = lam[i1];
                    if (row >= 0) {
                        C ea = a, eb = b;
                        pair_apply<C, T>(ea, eb, kind, op[g].d);
                        const double2 x0 = to_d2(la), x1 = to_d2(lb);
                        const double2 y0 = to_d2(ea), y1 = to_d2(eb);
                        acc += x0.x * y0.x + x0.y * y0.y + x1.x * y1.x + x1.y * y1.y;
                    }
                    pair_apply<C, T>(la, lb, kind, op[g].ua);
                    psi[i0] = a;
                    psi[i1] = b;
                    lam[i0] = la;
                    lam[i1] = lb;
                }
                if (row >= 0) {
                    const double s = block_sum(acc, red);
                    if (t == 0) {
                        rowval[row] = 2.0 * s;
                    }
                }
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

// lambda = H psi over the amplitudes [j0, j1) of one item and this thread's
// share of Re <psi|lambda> (HJ amplitudes per thread at a time: HJ
// independent gathers per string in flight); j1 - j0 is a multiple of
// B_THREADS * HJ
template <typename T>
__device__ double ham_range(const typename CxT<T>::type* psi, typename CxT<T>::type* lam, const BStr* st, int n_str,
                            uint64_t j0, uint64_t j1, int with_grad)
{
    // lambda in the state's precision (FP32 terms for complex64, whose lambda
    // is stored in FP32 anyway); the energy in FP64
    using C = typename CxT<T>::type;
    double e = 0.0;
    for (uint64_t jb = j0 + threadIdx.x; jb < j1; jb += B_THREADS * HJ) {
        T lr[HJ], li[HJ];
#pragma unroll
        for (int k = 0; k < HJ; ++k) {
            lr[k] = 0;
            li[k] = 0;
        }
        for (int s = 0; s < n_str; ++s) {
            const BStr bs = st[s];
            const T cr = static_cast<T>(bs.cr), ci = static_cast<T>(bs.ci);
            C pv[HJ];
#pragma unroll
            for (int k = 0; k < HJ; ++k) {
                pv[k] = __ldcg(psi + ((jb + static_cast<uint64_t>(k) * B_THREADS) ^ bs.x));
            }
#pragma unroll
            for (int k = 0; k < HJ; ++k) {
                const uint64_t src = (jb + static_cast<uint64_t>(k) * B_THREADS) ^ bs.x;
                const T sg = (__popcll(src & bs.z) & 1) ? T(-1) : T(1);
                lr[k] += sg * (cr * pv[k].x - ci * pv[k].y);
                li[k] += sg * (cr * pv[k].y + ci * pv[k].x);
            }
        }
#pragma unroll
        for (int k = 0; k < HJ; ++k) {
            const uint64_t j = jb + static_cast<uint64_t>(k) * B_THREADS;
            const double2 pj = to_d2(__ldcg(psi + j));
            e += pj.x * static_cast<double>(lr[k]) + pj.y * static_cast<double>(li[k]);
            if (with_grad) {
                lam[j] = make_cx<T>(lr[k], li[k]);
            }
        }
    }
    return e;
}

// ---------------------------------------------------------------------------
// items in HBM that run compiled block kernels: every launch serves the items
// of one plan structure, blockIdx.y the item (see jit_batch_compile)

// |0...0> into every listed state
template <typename C>
__global__ void k_batch_basis(void* const* __restrict__ states, uint64_t n_amps)
{
    C* a = static_cast<C*>(states[blockIdx.y]);
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_amps;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        a[i] = (i == 0) ? C {1, 0} : C {0, 0};
    }
}

// lambda = H psi and the energy partials of the listed items, which have
// n_chunks chunks of 2^K amplitudes each: epart[ebase[item] + chunk].  The
// units (item, chunk) are taken in item-major order by all CTAs at once, so
// the CTAs work on one item at a time and its psi[j ^ x] gathers stay in L2.
template <typename T>
__global__ void __launch_bounds__(B_THREADS) k_batch_ham_items(typename CxT<T>::type* __restrict__ arena,
                                                               const BInst* __restrict__ insts,
                                                               const int64_t* __restrict__ list,
                                                               const int64_t* __restrict__ ebase,
                                                               const BStr* __restrict__ strs, double* __restrict__ epart,
                                                               int K, int with_grad, uint64_t n_items, uint64_t n_chunks)
{
    using C = typename CxT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[B_THREADS / 32];
    BStr* sst = reinterpret_cast<BStr*>(smem_raw);
    const uint64_t chunk = uint64_t {1} << K;
    int64_t staged = -1;
    for (uint64_t u = blockIdx.x; u < n_items * n_chunks; u += gridDim.x) {
        const int64_t item = static_cast<int64_t>(u / n_chunks);
        const uint64_t c = u % n_chunks;
        const BInst inst = insts[list[item]];
        const BStr* st = strs + inst.str;
        if (inst.n_str <= HAM_SMEM_STRINGS) {
            if (item != staged) {
                __syncthreads();  // every thread is done with the previous item's strings
                for (int s = threadIdx.x; s < inst.n_str; s += B_THREADS) {
                    sst[s] = st[s];
                }
                __syncthreads();
                staged = item;
            }
            st = sst;
        }
        const double e = block_sum(ham_range<T>(arena + inst.psi, arena + inst.lam, st, inst.n_str, c * chunk,
                                                (c + 1) * chunk, with_grad),
                                   red);
        if (threadIdx.x == 0) {
            epart[ebase[item] + static_cast<int64_t>(c)] = e;
        }
    }
}

// ---------------------------------------------------------------------------
// items in HBM: the persistent work-queue kernel
template <typename T>
__global__ void __launch_bounds__(B_THREADS, 2) k_batch_persist(BArgs<T> A)
{
    using C = typename CxT<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ FBlock bk;
    __shared__ FPhase sph[MAX_PHASES_PER_BLOCK];
    __shared__ double red[B_THREADS / 32];
    __shared__ int2 wu_sh;
    __shared__ int stop_sh;
    const uint32_t t = threadIdx.x;
    while (true) {
        if (t == 0) {
            // take a unit of the oldest ready job that still has one; wait only
            // while nothing is ready (every job in flight has a running CTA)
            int stop = 0;
            int2 got = make_int2(-1, -1);
            long long spins = 0;
            while (true) {
                if (*reinterpret_cast<volatile int*>(A.status) != 0) {
                    stop = 1;
                    break;
                }
                const unsigned long long h = *reinterpret_cast<volatile unsigned long long*>(A.qhead);
                if (h >= static_cast<unsigned long long>(A.n_jobs)) {
                    stop = 1;  // every job has been handed out
                    break;
                }
                if (h < *reinterpret_cast<volatile unsigned long long*>(A.qtail)) {
                    const int j = *reinterpret_cast<volatile int*>(A.queue + h);
                    if (j >= 0) {
                        const int u = atomicAdd(A.taken + j, 1);
                        if (u < A.jobs[j].n_units) {
                            got = make_int2(j, u);
                            break;
                        }
                        atomicCAS(A.qhead, h, h + 1);  // job exhausted: move the head on
                        continue;
                    }
                }
                if (++spins > A.spin_limit) {
                    atomicExch(A.status, 1);
                    stop = 1;
                    break;
                }
                __nanosleep(128);
            }
            __threadfence();  // the job's inputs were written by its predecessor's units
            wu_sh = got;
            stop_sh = stop;
        }
        __syncthreads();
        if (stop_sh) {
            break;
        }
        const int2 wu = wu_sh;
        const BJob job = A.jobs[wu.x];
        const BInst inst = A.insts[job.inst];
        const uint64_t t0 = static_cast<uint64_t>(wu.y) * static_cast<uint64_t>(job.tiles_per_unit);
        const uint64_t t1 = min(t0 + static_cast<uint64_t>(job.tiles_per_unit), static_cast<uint64_t>(job.n_tiles));
        C* psi = A.arena + inst.psi;
        if (job.kind == JOB_FWD) {
            if (t == 0) {
                bk = A.fblk[job.block];
            }
            __syncthreads();
            C* sm = reinterpret_cast<C*>(smem_raw);
            FOp<T>* sops = reinterpret_cast<FOp<T>*>(smem_raw + (sizeof(C) << bk.K));
            stage_block(bk, A.fph, A.fops, sph, sops, t);
            __syncthreads();
            for (uint64_t tile = t0; tile < t1; ++tile) {
                fwd_tile<T, Cfg<T>::RB, true>(psi, bk, sph, sops, tile, sm, t, job.init != 0);
            }
        } else if (job.kind == JOB_BWD) {
            if (t == 0) {
                bk = A.bblk[job.block];
            }
            __syncthreads();
            const size_t tile_bytes = sizeof(C) << bk.K;
            C* smp = reinterpret_cast<C*>(smem_raw);
            C* sml = reinterpret_cast<C*>(smem_raw + tile_bytes);
            FOpA<T>* sops = reinterpret_cast<FOpA<T>*>(smem_raw + 2 * tile_bytes);
            double* acc = reinterpret_cast<double*>(smem_raw + 2 * tile_bytes +
                                                    static_cast<size_t>(bk.op_end - bk.op_begin) * sizeof(FOpA<T>));
            stage_block(bk, A.bph, A.bops, sph, sops, t);
            for (int w = t; w < job.n_rows * ADJ_WARPS; w += B_THREADS) {
                acc[w] = 0.0;
            }
            __syncthreads();
            C* lam = A.arena + inst.lam;
            for (uint64_t tile = t0; tile < t1; ++tile) {
                adj_tile<T, CfgA<T>::RB, true>(psi, lam, bk, sph, sops, tile, smp, sml, acc, t);
            }
            __syncthreads();
            for (int r = t; r < job.n_rows; r += B_THREADS) {
                double s = 0.0;
                for (int w = 0; w < ADJ_WARPS; ++w) {
                    s += acc[r * ADJ_WARPS + w];
                }
                A.part[job.part + static_cast<int64_t>(r) * job.n_units + wu.y] = s;
            }
        } else {
            // lambda = H psi over this unit's chunks and its share of Re <psi|lambda>
            const int chunk_bits = inst.q - (63 - __clzll(static_cast<long long>(job.n_tiles)));
            const BStr* st = A.strs + inst.str;
            BStr* sst = reinterpret_cast<BStr*>(smem_raw);
            if (inst.n_str <= HAM_SMEM_STRINGS) {
                for (int s = t; s < inst.n_str; s += B_THREADS) {
                    sst[s] = st[s];
                }
                st = sst;
            }
            __syncthreads();
            C* lam = A.arena + inst.lam;
            const double e = block_sum(ham_range<T>(psi, lam, st, inst.n_str, t0 << chunk_bits, t1 << chunk_bits,
                                                    A.with_grad),
                                       red);
            if (t == 0) {
                A.epart[job.part + wu.y] = e;
            }
        }
        __syncthreads();
        if (t == 0) {
            __threadfence();
            const int d = atomicAdd(A.done + wu.x, 1) + 1;
            if (d == job.n_units && job.succ >= 0) {
                // the last unit of the job: its successor is ready
                __threadfence();
                const unsigned long long pos = atomicAdd(A.qtail, 1ULL);
                *reinterpret_cast<volatile int*>(A.queue + pos) = job.succ;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// finalisation (fixed summation order)
__global__ void k_batch_energy(const double* __restrict__ epart, const ESrc* __restrict__ src, int64_t n,
                               double* __restrict__ energies)
{
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const ESrc e = src[i];
    double s = 0.0;
    for (int u = 0; u < e.count; ++u) {
        s += epart[e.first + u];
    }
    energies[e.out] = s;
}

__global__ void k_batch_rows(const double* __restrict__ part, const RowSrc* __restrict__ src, int64_t n,
                             double* __restrict__ rowval)
{
    const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) {
        return;
    }
    const RowSrc rs = src[r];
    double s = 0.0;
    for (int u = 0; u < rs.count; ++u) {
        s += part[rs.first + u];
    }
    rowval[r] = 2.0 * s;
}

// grads[p] = sum of the rows bound to parameter p, in row order
__global__ void k_batch_grads(const double* __restrict__ rowval, const int64_t* __restrict__ first,
                              const int64_t* __restrict__ rows, int64_t n_params, double* __restrict__ grads)
{
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= n_params) {
        return;
    }
    double s = 0.0;
    for (int64_t k = first[p]; k < first[p + 1]; ++k) {
        s += rowval[rows[k]];
    }
    grads[p] = s;
}

// ---------------------------------------------------------------------------
// host planning

bool has_angle(int op)
{
    return (op >= KT_OP_RX && op <= KT_OP_P) || (op >= KT_OP_CRX && op <= KT_OP_CP);
}

int32_t fail(int32_t code, const std::string& msg)
{
    set_error(code, msg);
    return code;
}

// Lower an item's gates with a stand-in angle for every bound parameter (so
// the op kinds are those of a generic angle); `slot` gets the parameter slot
// of each gate (-1: literal).
int32_t lower_symbolic(const kt_gate* gates, int64_t n_gates, int64_t n_params, int q, std::vector<LGate>& lg,
                       std::vector<int32_t>& slot)
{
    lg.resize(static_cast<size_t>(n_gates));
    slot.assign(static_cast<size_t>(n_gates), -1);
    for (int64_t i = 0; i < n_gates; ++i) {
        kt_gate g = gates[i];
        if (g.op == KT_OP_M) {
            return fail(KT_ERR_INVALID, "gate " + std::to_string(i) + ": M gates are not supported in batches");
        }
        if (has_angle(g.op) && g.param >= 0) {
            if (g.param >= n_params) {
                return fail(KT_ERR_INVALID, "gate " + std::to_string(i) + ": parameter slot " + std::to_string(g.param) +
                                                " out of range for the item's " + std::to_string(n_params) + " parameters");
            }
            slot[static_cast<size_t>(i)] = g.param;
            g.param = -1;
            g.angle = 1.0;  // generic stand-in: no entry of U vanishes by accident
        }
        if (const int32_t rc = lower_gate(g, nullptr, 0, q, &lg[static_cast<size_t>(i)]); rc != KT_OK) {
            return rc;
        }
    }
    return KT_OK;
}

LGate dagger(const LGate& l)
{
    LGate a = l;
    const double* m = l.m;
    a.m[0] = m[0]; a.m[1] = -m[1];
    a.m[2] = m[4]; a.m[3] = -m[5];
    a.m[4] = m[2]; a.m[5] = -m[3];
    a.m[6] = m[6]; a.m[7] = -m[7];
    a.flags = (a.kind == KIND_DIAG && a.m[0] == 1.0 && a.m[1] == 0.0) ? 1 : 0;
    return a;
}

// What one HBM item contributes to the global tables (indices local to it).
template <typename T>
struct ItemPlan
{
    Plan<T> fwd;
    Plan<T, FOpA<T>> bwd;
    std::vector<std::vector<int32_t>> rows_of_block;  // adjoint block -> local row ids
    std::vector<int32_t> row_slot;                    // local row -> parameter slot
    std::vector<std::pair<int64_t, int32_t>> fpatch;  // (local forward op, gate index)
    std::vector<std::pair<int64_t, int32_t>> bpatch;  // (local adjoint op, gate index)
    std::vector<int32_t> slot;                        // gate -> slot
    std::vector<uint8_t> opcode;                      // gate -> KT_OP_*
    std::vector<uint8_t> fone, bone;                  // op -> made one-sided (one_sided_diagonals)
    uint64_t key {0};                                 // structure of both plans (plan_structure_key)
    int32_t rc {KT_OK};
    std::string err;
};

// A hash of everything the text of an item's batched block kernels depends
// on: the qubit count, the blocks, phases and op records of both plans (the
// records without their matrices) and the rows of every adjoint block.  The
// planner value-initialises its records, so equal structures hash equal.
template <typename T>
uint64_t plan_structure_key(const ItemPlan<T>& ip, int q)
{
    std::string bytes;
    auto add = [&](const void* p, size_t n) { bytes.append(static_cast<const char*>(p), n); };
    add(&q, sizeof(q));
    auto add_plan = [&](const auto& plan) {
        const uint64_t counts[3] = {plan.blocks.size(), plan.phases.size(), plan.ops.size()};
        add(counts, sizeof(counts));
        add(plan.blocks.data(), plan.blocks.size() * sizeof(FBlock));
        add(plan.phases.data(), plan.phases.size() * sizeof(FPhase));
        for (auto op : plan.ops) {
            std::memset(static_cast<void*>(op.m), 0, sizeof(op.m));
            add(&op, sizeof(op));
        }
    };
    add_plan(ip.fwd);
    add_plan(ip.bwd);
    for (const auto& r : ip.rows_of_block) {
        const uint64_t n = r.size();
        add(&n, sizeof(n));
    }
    return std::hash<std::string> {}(bytes);
}

template <typename P>
bool phases_fit(const P& plan)
{
    for (const auto& fb : plan.blocks) {
        if (fb.phase_end - fb.phase_begin > MAX_PHASES_PER_BLOCK) {
            return false;
        }
    }
    return true;
}

// An item's energy and gradient do not depend on a global phase of psi: the
// energy is <psi|H|psi>, lambda = H psi carries psi's phase, and every
// gradient term is bilinear in conj(lambda) and psi.  So an uncontrolled
// diagonal op with |m00| = 1 (RZ, P, literal phases) may run as the
// one-sided diag(1, m11 / m00) in both sweeps: it drops the same unit factor
// from psi and lambda, and touches half the amplitudes.  Returns, per op,
// whether it was rewritten (its patch then writes the one-sided form).
template <typename P>
std::vector<uint8_t> one_sided_diagonals(P& plan)
{
    std::vector<uint8_t> flag(plan.ops.size(), 0);
    for (size_t o = 0; o < plan.ops.size(); ++o) {
        auto& op = plan.ops[o];
        if (op.kind != OP_DIAG || op.cslot != NO_SLOT || op.cthr != 0 || op.cglob != 0) {
            continue;
        }
        const double m0r = static_cast<double>(op.m[0]), m0i = static_cast<double>(op.m[1]);
        const double m1r = static_cast<double>(op.m[6]), m1i = static_cast<double>(op.m[7]);
        if (std::abs(m0r * m0r + m0i * m0i - 1.0) > 1e-12) {
            continue;
        }
        // m11 conj(m00)
        const double r = m1r * m0r + m1i * m0i;
        const double i = m1i * m0r - m1r * m0i;
        for (int e = 0; e < 8; ++e) {
            op.m[e] = 0;
        }
        op.m[0] = 1;
        using E = std::remove_reference_t<decltype(op.m[0])>;
        op.m[6] = static_cast<E>(r);
        op.m[7] = static_cast<E>(i);
        op.kind = OP_DIAG1;
        flag[o] = 1;
    }
    return flag;
}

template <typename T>
void plan_item(const kt_batch_item& it, const kt_gate* gates, bool with_grad, ItemPlan<T>& ip)
{
    const int q = it.n_qubits;
    std::vector<LGate> lg;
    if ((ip.rc = lower_symbolic(gates + it.gate_offset, it.n_gates, it.n_params, q, lg, ip.slot)) != KT_OK) {
        ip.err = last_error_cstr();
        return;
    }
    ip.opcode.resize(lg.size());
    for (size_t i = 0; i < lg.size(); ++i) {
        ip.opcode[i] = gates[it.gate_offset + static_cast<int64_t>(i)].op;
    }
    // forward blocks (an item without gates still gets one block: it writes |0...0>)
    const int K = Cfg<T>::RB + TB256;
    // fusion depth: the fused_max_ops knob (set by the autotuner), within the kernel's budgets
    const size_t fwd_ops = static_cast<size_t>(std::min(BATCH_FWD_MAX_OPS, tuning().fused_max_ops));
    const size_t bwd_ops = static_cast<size_t>(std::min(BATCH_BWD_MAX_OPS, tuning().fused_max_ops));
    auto pbs = form_blocks(lg, q, K, Cfg<T>::L, fwd_ops);
    if (pbs.empty()) {
        PlanBlock b;
        b.K = K;
        for (int j = 0; j < K; ++j) {
            b.qubits.push_back(j);
        }
        pbs.push_back(b);
    }
    for (const auto& pb : pbs) {
        plan_block<T>(pb, lg, q, ip.fwd);
    }
    for (size_t o = 0; o < ip.fwd.ops.size(); ++o) {
        const int32_t gi = ip.fwd.op_gate[o];
        if (ip.slot[static_cast<size_t>(gi)] >= 0) {
            ip.fpatch.emplace_back(static_cast<int64_t>(o), gi);
        }
    }
    if (with_grad) {
        // adjoint blocks over the reversed gate list (U^dagger; rows in backward order)
        const int KA = CfgA<T>::RB + TB256;
        const size_t G = lg.size();
        std::vector<LGate> rl(G);
        std::vector<AdjExtra> ex(G);
        std::vector<int32_t> gate_of(G);
        int32_t n_rows = 0;
        for (size_t k = 0; k < G; ++k) {
            const size_t gi = G - 1 - k;
            gate_of[k] = static_cast<int32_t>(gi);
            rl[k] = dagger(lg[gi]);
            ex[k].row = -1;
            ex[k].gen = gate_generator(ip.opcode[gi]);
            if (ip.slot[gi] >= 0 && ex[k].gen >= 0) {
                ex[k].row = n_rows++;
                ip.row_slot.push_back(ip.slot[gi]);
            }
        }
        const auto abs = form_blocks(rl, q, KA, CfgA<T>::L, bwd_ops);
        for (const auto& pb : abs) {
            std::vector<int32_t> rows;
            std::vector<AdjExtra> local(ex.size());
            for (int gi : pb.gates) {
                local[gi] = ex[gi];
                if (ex[gi].row >= 0) {
                    local[gi].row = static_cast<int32_t>(rows.size());
                    rows.push_back(ex[gi].row);
                }
            }
            plan_block<T, CfgA<T>, FOpA<T>>(pb, rl, q, ip.bwd, local.data());
            ip.rows_of_block.push_back(std::move(rows));
        }
        for (size_t o = 0; o < ip.bwd.ops.size(); ++o) {
            const int32_t g = gate_of[static_cast<size_t>(ip.bwd.op_gate[o])];
            if (ip.slot[static_cast<size_t>(g)] >= 0) {
                ip.bpatch.emplace_back(static_cast<int64_t>(o), g);
            }
        }
    }
    if (!phases_fit(ip.fwd) || !phases_fit(ip.bwd)) {
        ip.rc = KT_ERR_INVALID;
        set_error(KT_ERR_INVALID, "batch planner produced too many phases");
        ip.err = last_error_cstr();
    }
    ip.fone = one_sided_diagonals(ip.fwd);
    ip.bone = one_sided_diagonals(ip.bwd);
    ip.key = plan_structure_key(ip, q);
}

template <typename P>
void append_plan(P& dst, const P& src)
{
    const int32_t ph0 = static_cast<int32_t>(dst.phases.size());
    const int32_t op0 = static_cast<int32_t>(dst.ops.size());
    for (auto b : src.blocks) {
        b.phase_begin += ph0;
        b.phase_end += ph0;
        b.op_begin += op0;
        b.op_end += op0;
        dst.blocks.push_back(b);
    }
    for (auto p : src.phases) {
        p.op_begin += op0;
        p.op_end += op0;
        dst.phases.push_back(p);
    }
    dst.ops.insert(dst.ops.end(), src.ops.begin(), src.ops.end());
}

template <typename P>
BatchPlanView view_of(const P& plan)
{
    BatchPlanView v;
    v.blocks = plan.blocks.data();
    v.n_blocks = static_cast<int64_t>(plan.blocks.size());
    v.phases = plan.phases.data();
    v.n_phases = static_cast<int64_t>(plan.phases.size());
    v.ops = plan.ops.data();
    v.n_ops = static_cast<int64_t>(plan.ops.size());
    v.rec_bytes[0] = static_cast<int64_t>(sizeof(FBlock));
    v.rec_bytes[1] = static_cast<int64_t>(sizeof(FPhase));
    v.rec_bytes[2] = static_cast<int64_t>(sizeof(typename decltype(plan.ops)::value_type));
    return v;
}

// tile qubits of the batch's forward and adjoint blocks (256-thread tiles)
template <typename T>
constexpr int K_FWD = Cfg<T>::RB + TB256;
template <typename T>
constexpr int K_BWD = CfgA<T>::RB + TB256;

// CTAs per item of a compiled class launch: about four per SM over the class,
// at most one per tile
int32_t ctas_per_item(size_t n_items, int64_t tiles)
{
    const int64_t want = (4 * static_cast<int64_t>(sm_count()) + static_cast<int64_t>(n_items) - 1) /
                         static_cast<int64_t>(n_items);
    return static_cast<int32_t>(std::max<int64_t>(1, std::min<int64_t>(tiles, want)));
}

int64_t units_for(int64_t n_tiles, int32_t* tiles_per_unit)
{
    const int64_t tpu = std::max<int64_t>(1, (n_tiles + UNITS_PER_JOB - 1) / UNITS_PER_JOB);
    *tiles_per_unit = static_cast<int32_t>(tpu);
    return (n_tiles + tpu - 1) / tpu;
}

BStr make_str(const kt_pauli& p, const double* coeffs, int64_t s)
{
    const int k4 = (__builtin_popcountll(p.x_mask & p.z_mask) + p.phase) & 3;
    double cr = coeffs ? coeffs[2 * s] : 1.0;
    double ci = coeffs ? coeffs[2 * s + 1] : 0.0;
    for (int r = 0; r < k4; ++r) {
        const double tr = -ci;
        ci = cr;
        cr = tr;
    }
    return BStr {p.x_mask, p.z_mask, cr, ci};
}

}  // namespace
}  // namespace kt

// ---------------------------------------------------------------------------
// the handle

struct kt_batch_s
{
    int32_t dtype {KT_C128};
    int32_t with_grad {1};
    int64_t n_items {0};
    int64_t n_params {0};
    int64_t n_small {0};
    int64_t n_large {0};
    int64_t n_waves {0};
    int64_t n_jobs {0};
    int64_t n_units {0};
    int64_t launches {0};
    double alg_bytes {0.0};
    size_t device_bytes {0};
    void* meta {nullptr};
    void* arena {nullptr};
    double* h_params {nullptr};   // pinned
    double* h_out {nullptr};      // pinned: energies | grads | status
    size_t out_bytes {0};
    cudaStream_t s0 {nullptr};
    cudaStream_t s1 {nullptr};
    cudaEvent_t ev_fork {nullptr};
    cudaEvent_t ev_join {nullptr};
    cudaGraph_t graph {nullptr};
    cudaGraphExec_t exec {nullptr};
    cudaStream_t user {nullptr};
    // compiled classes: streams their chains run on inside the graph, and the
    // programs holding their kernels (unloaded with the batch)
    static constexpr int N_CLASS_STREAMS = 4;
    cudaStream_t cs[N_CLASS_STREAMS] {};
    cudaEvent_t cev[N_CLASS_STREAMS] {};
    std::vector<cudaLibrary_t> libs;
    int64_t n_classes {0};
    int64_t n_compiled_items {0};
};

namespace kt
{
namespace
{

void release(kt_batch_s* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (int i = 0; i < kt_batch_s::N_CLASS_STREAMS; ++i) {
        if (b->cev[i]) cudaEventDestroy(b->cev[i]);
        if (b->cs[i]) cudaStreamDestroy(b->cs[i]);
    }
    for (cudaLibrary_t lib : b->libs) {
        cudaLibraryUnload(lib);
    }
    b->libs.clear();
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->s0) cudaStreamDestroy(b->s0);
    if (b->s1) cudaStreamDestroy(b->s1);
    if (b->meta) cudaFree(b->meta);
    if (b->arena) cudaFree(b->arena);
    if (b->h_params) cudaFreeHost(b->h_params);
    if (b->h_out) cudaFreeHost(b->h_out);
}

// Byte layout of the device metadata block (256-byte aligned pieces).
struct Layout
{
    size_t size {0};
    size_t add(size_t bytes)
    {
        const size_t at = size;
        size = (size + std::max<size_t>(bytes, 1) + 255) & ~size_t {255};
        return at;
    }
};

template <typename T>
int32_t create(const kt_batch_item* items, int64_t n_items, const kt_gate* gates, int64_t n_params,
               const kt_pauli* strings, const double* coeffs, int32_t with_grad, kt_batch_s* B)
{
    using C = typename CxT<T>::type;
    // shared-memory items: at most what fits (12 / 13 qubits), at least one
    // below a forward tile, since an HBM item needs a whole tile of 2^K_FWD amplitudes
    const int qsmall = std::max(K_FWD<T> - 1, std::min((sizeof(T) == 8) ? 12 : 13, tuning().batch_small_max_qubits));
    std::vector<int64_t> small, large;
    for (int64_t b = 0; b < n_items; ++b) {
        (items[b].n_qubits <= qsmall ? small : large).push_back(b);
    }
    auto cost = [&](int64_t b) {
        return std::ldexp(1.0, items[b].n_qubits) * static_cast<double>(items[b].n_gates + 1);
    };
    std::stable_sort(small.begin(), small.end(), [&](int64_t a, int64_t b) { return cost(a) > cost(b); });
    std::stable_sort(large.begin(), large.end(), [&](int64_t a, int64_t b) { return cost(a) > cost(b); });

    // Pauli terms of every item
    std::vector<BStr> strs;
    std::vector<int64_t> str_first(static_cast<size_t>(n_items));
    for (int64_t b = 0; b < n_items; ++b) {
        str_first[b] = static_cast<int64_t>(strs.size());
        for (int64_t s = 0; s < items[b].n_strings; ++s) {
            strs.push_back(make_str(strings[items[b].string_offset + s], coeffs, items[b].string_offset + s));
        }
    }

    // gradient rows (global ids) and the parameter each one belongs to
    std::vector<int64_t> row_param;
    std::vector<BPatch> patches;

    // --- shared-memory items
    std::vector<SItem> sitems;
    std::vector<SOp<T>> sops;
    for (int64_t b : small) {
        const kt_batch_item& it = items[b];
        std::vector<LGate> lg;
        std::vector<int32_t> slot;
        if (const int32_t rc = lower_symbolic(gates + it.gate_offset, it.n_gates, it.n_params, it.n_qubits, lg, slot);
            rc != KT_OK) {
            return rc;
        }
        SItem si {};
        si.q = it.n_qubits;
        si.n_ops = static_cast<int32_t>(lg.size());
        si.op = static_cast<int64_t>(sops.size());
        si.n_str = static_cast<int32_t>(it.n_strings);
        si.str = str_first[b];
        si.out = b;
        for (size_t g = 0; g < lg.size(); ++g) {
            const LGate& l = lg[g];
            SOp<T> o {};
            o.kind = static_cast<int16_t>(l.kind);
            o.target = static_cast<int16_t>(l.target);
            o.control = static_cast<int16_t>(l.control);
            o.row = -1;
            const LGate a = dagger(l);
            for (int e = 0; e < 8; ++e) {
                o.u[e] = static_cast<T>(l.m[e]);
                o.ua[e] = static_cast<T>(a.m[e]);
            }
            const int op = gates[it.gate_offset + static_cast<int64_t>(g)].op;
            if (slot[g] >= 0) {
                patches.push_back(BPatch {TAB_SMALL, op, static_cast<int64_t>(sops.size()), it.param_offset + slot[g]});
                double scratch[8];
                if (with_grad && gate_derivative(op, 1.0, scratch)) {
                    o.row = static_cast<int32_t>(row_param.size());
                    row_param.push_back(it.param_offset + slot[g]);
                }
            }
            sops.push_back(o);
        }
        sitems.push_back(si);
    }
    const int64_t small_rows_end = static_cast<int64_t>(row_param.size());

    // --- HBM items: planned in parallel, then merged into the global tables
    std::vector<ItemPlan<T>> ips(large.size());
    {
        const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        const size_t nt = std::min<size_t>(hw, std::max<size_t>(1, large.size()));
        std::vector<std::thread> pool;
        for (size_t w = 0; w < nt; ++w) {
            pool.emplace_back([&, w] {
                for (size_t k = w; k < large.size(); k += nt) {
                    try {
                        plan_item<T>(items[large[k]], gates, with_grad != 0, ips[k]);
                    } catch (const std::exception& e) {
                        ips[k].rc = KT_ERR_INVALID;
                        set_error(KT_ERR_INVALID, e.what());
                        ips[k].err = last_error_cstr();
                    }
                }
            });
        }
        for (auto& th : pool) {
            th.join();
        }
    }
    for (const auto& ip : ips) {
        if (ip.rc != KT_OK) {
            set_error_text(ip.err);
            return ip.rc;
        }
    }

    // memory waves: HBM items in cost order, packed while the arena fits
    const size_t per_amp = sizeof(C) * (with_grad ? 2 : 1);
    size_t free_b = 0, total_b = 0;
    KT_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t reserve = std::max<size_t>(size_t {4} << 30, total_b / 16);
    const size_t budget = free_b > reserve ? (free_b - reserve) * 3 / 4 : 0;
    std::vector<int32_t> wave_of(large.size());
    std::vector<int64_t> inst_off(large.size());
    size_t arena_bytes = 0;
    {
        int32_t w = 0;
        size_t used = 0;
        for (size_t k = 0; k < large.size(); ++k) {
            const size_t need = (size_t {1} << items[large[k]].n_qubits) * per_amp;
            if (need > budget) {
                return fail(KT_ERR_NOMEM, "a " + std::to_string(items[large[k]].n_qubits) +
                                              "-qubit item does not fit in device memory");
            }
            if (used + need > budget) {
                ++w;
                used = 0;
            }
            wave_of[k] = w;
            inst_off[k] = static_cast<int64_t>(used / sizeof(C));
            used += need;
            arena_bytes = std::max(arena_bytes, used);
        }
        B->n_waves = large.empty() ? 0 : w + 1;
    }

    // --- compiled classes: HBM items of at least batch_jit_min_qubits qubits
    // whose plans have one structure share batched block kernels, one launch
    // per block for all of them (single memory wave only)
    struct Class
    {
        std::vector<size_t> members;           // large-item indices
        int q {0};
        int32_t cpi_f {1}, cpi_a {1};          // CTAs per item: forward blocks, adjoint blocks
        std::vector<int32_t> rows;             // gradient rows of each adjoint block
        std::vector<const void*> fk, bk;       // kernels
        int32_t fsmem {0};
        std::vector<int32_t> bsmem;
    };
    std::vector<Class> cls;
    std::vector<int32_t> class_of(large.size(), -1);
    const int jit_min = tuning().batch_jit_min_qubits;
    if (jit_min > 0 && B->n_waves == 1 && !large.empty() && jit_available(nullptr)) {
        std::unordered_map<uint64_t, int32_t> by_key;
        for (size_t k = 0; k < large.size(); ++k) {
            if (items[large[k]].n_qubits < jit_min) {
                continue;
            }
            auto it = by_key.find(ips[k].key);
            if (it == by_key.end() || cls[static_cast<size_t>(it->second)].members.size() >= 65535) {
                it = by_key.insert_or_assign(ips[k].key, static_cast<int32_t>(cls.size())).first;
                cls.emplace_back();
            }
            class_of[k] = it->second;
            cls[static_cast<size_t>(it->second)].members.push_back(k);
        }
        std::vector<BatchPlanView> fv, bv;
        for (Class& c : cls) {
            const ItemPlan<T>& rep = ips[c.members.front()];
            c.q = items[large[c.members.front()]].n_qubits;
            c.cpi_f = ctas_per_item(c.members.size(), int64_t {1} << (c.q - K_FWD<T>));
            c.cpi_a = ctas_per_item(c.members.size(), int64_t {1} << (c.q - K_BWD<T>));
            for (const auto& r : rep.rows_of_block) {
                c.rows.push_back(static_cast<int32_t>(r.size()));
            }
            fv.push_back(view_of(rep.fwd));
            bv.push_back(view_of(rep.bwd));
        }
        std::vector<std::vector<const void*>> fk, bk;
        std::vector<int32_t> fsm;
        std::vector<std::vector<int32_t>> bsm;
        if (!cls.empty()) {
            if (jit_batch_compile(sizeof(T) == 8 ? KT_C128 : KT_C64, fv, bv, fk, bk, fsm, bsm, B->libs) == KT_OK) {
                for (size_t c = 0; c < cls.size(); ++c) {
                    cls[c].fk = fk[c];
                    cls[c].bk = bk[c];
                    cls[c].fsmem = fsm[c];
                    cls[c].bsmem = bsm[c];
                }
            } else {
                // run-time compilation failed: every item runs in the persistent kernel
                for (cudaLibrary_t lib : B->libs) {
                    cudaLibraryUnload(lib);
                }
                B->libs.clear();
                cls.clear();
                std::fill(class_of.begin(), class_of.end(), -1);
                cudaGetLastError();
            }
        }
    }
    B->n_classes = static_cast<int64_t>(cls.size());
    // per compiled item: its op records in the merged tables (per block), the
    // Hamiltonian partials' base and each adjoint block's partials' base
    std::vector<std::vector<int64_t>> item_fop(large.size()), item_bop(large.size()), item_pbase(large.size());
    std::vector<int64_t> item_ebase(large.size(), 0);

    Plan<T> gf;
    Plan<T, FOpA<T>> gb;
    std::vector<BInst> insts(large.size());
    std::vector<BJob> jobs;
    std::vector<std::vector<int32_t>> chain(large.size());  // job ids per HBM item in execution order
    std::vector<RowSrc> row_src;                             // rows of HBM items (ids from small_rows_end on)
    std::vector<ESrc> esrc;
    int64_t part_size = 0, epart_size = 0;
    double alg = 0.0;
    const int K = Cfg<T>::RB + TB256;
    const int KA = CfgA<T>::RB + TB256;
    for (size_t k = 0; k < large.size(); ++k) {
        const kt_batch_item& it = items[large[k]];
        ItemPlan<T>& ip = ips[k];
        const int q = it.n_qubits;
        BInst& in = insts[k];
        in.q = q;
        in.psi = inst_off[k];
        in.lam = with_grad ? inst_off[k] + (int64_t {1} << q) : inst_off[k];
        in.n_str = static_cast<int32_t>(it.n_strings);
        in.str = str_first[large[k]];
        const double state_bytes = std::ldexp(static_cast<double>(sizeof(C)), q);
        const int32_t fb0 = static_cast<int32_t>(gf.blocks.size());
        const int64_t fo0 = static_cast<int64_t>(gf.ops.size());
        append_plan(gf, ip.fwd);
        for (const auto& [lop, g] : ip.fpatch) {
            patches.push_back(BPatch {TAB_FWD, ip.opcode[g], fo0 + lop, it.param_offset + ip.slot[g],
                                      ip.fone[static_cast<size_t>(lop)], 0});
        }
        if (class_of[k] >= 0) {
            // a compiled class's item: its blocks run as class launches, no jobs
            const Class& c = cls[static_cast<size_t>(class_of[k])];
            for (const auto& fb : ip.fwd.blocks) {
                item_fop[k].push_back(fo0 + fb.op_begin);
            }
            alg += (1.0 + 2.0 * static_cast<double>(ip.fwd.blocks.size())) * state_bytes;  // |0...0>, then the blocks
            item_ebase[k] = epart_size;
            const int32_t n_chunks = static_cast<int32_t>(int64_t {1} << (c.q - K_FWD<T>));
            esrc.push_back(ESrc {epart_size, n_chunks, 0, large[k]});
            epart_size += n_chunks;
            alg += (with_grad ? 2.0 : 1.0) * state_bytes;
            if (with_grad) {
                const int64_t bo0 = static_cast<int64_t>(gb.ops.size());
                append_plan(gb, ip.bwd);
                for (const auto& [lop, g] : ip.bpatch) {
                    patches.push_back(BPatch {TAB_BWD, ip.opcode[g], bo0 + lop, it.param_offset + ip.slot[g],
                                              ip.bone[static_cast<size_t>(lop)], 0});
                }
                const int64_t row0 = static_cast<int64_t>(row_param.size());
                for (int32_t sl : ip.row_slot) {
                    row_param.push_back(it.param_offset + sl);
                }
                row_src.resize(row_param.size() - static_cast<size_t>(small_rows_end));
                for (size_t b = 0; b < ip.bwd.blocks.size(); ++b) {
                    item_bop[k].push_back(bo0 + ip.bwd.blocks[b].op_begin);
                    item_pbase[k].push_back(part_size);
                    const auto& rows = ip.rows_of_block[b];
                    for (size_t r = 0; r < rows.size(); ++r) {
                        const int64_t grow = row0 + rows[r];
                        row_src[static_cast<size_t>(grow - small_rows_end)] =
                            RowSrc {part_size + static_cast<int64_t>(r) * c.cpi_a, c.cpi_a, 0};
                    }
                    part_size += static_cast<int64_t>(rows.size()) * c.cpi_a;
                    alg += 4.0 * state_bytes;
                }
            }
            ip = ItemPlan<T>();
            continue;
        }
        for (size_t b = 0; b < ip.fwd.blocks.size(); ++b) {
            BJob j {};
            j.kind = JOB_FWD;
            j.inst = static_cast<int32_t>(k);
            j.block = fb0 + static_cast<int32_t>(b);
            j.n_tiles = int64_t {1} << (q - K);
            j.n_units = static_cast<int32_t>(units_for(j.n_tiles, &j.tiles_per_unit));
            j.init = (b == 0) ? 1 : 0;
            j.succ = -1;
            chain[k].push_back(static_cast<int32_t>(jobs.size()));
            jobs.push_back(j);
            alg += (b == 0 ? 1.0 : 2.0) * state_bytes;
        }
        {
            BJob j {};
            j.kind = JOB_HAM;
            j.inst = static_cast<int32_t>(k);
            j.block = -1;
            j.n_tiles = int64_t {1} << (q - K);
            j.n_units = static_cast<int32_t>(units_for(j.n_tiles, &j.tiles_per_unit));
            j.part = epart_size;
            j.succ = -1;
            epart_size += j.n_units;
            esrc.push_back(ESrc {j.part, j.n_units, 0, large[k]});
            chain[k].push_back(static_cast<int32_t>(jobs.size()));
            jobs.push_back(j);
            alg += (with_grad ? 2.0 : 1.0) * state_bytes;
        }
        if (with_grad) {
            const int32_t bb0 = static_cast<int32_t>(gb.blocks.size());
            const int64_t bo0 = static_cast<int64_t>(gb.ops.size());
            append_plan(gb, ip.bwd);
            for (const auto& [lop, g] : ip.bpatch) {
                patches.push_back(BPatch {TAB_BWD, ip.opcode[g], bo0 + lop, it.param_offset + ip.slot[g],
                                          ip.bone[static_cast<size_t>(lop)], 0});
            }
            const int64_t row0 = static_cast<int64_t>(row_param.size());
            for (int32_t s : ip.row_slot) {
                row_param.push_back(it.param_offset + s);
            }
            row_src.resize(row_param.size() - static_cast<size_t>(small_rows_end));
            for (size_t b = 0; b < ip.bwd.blocks.size(); ++b) {
                BJob j {};
                j.kind = JOB_BWD;
                j.inst = static_cast<int32_t>(k);
                j.block = bb0 + static_cast<int32_t>(b);
                j.n_tiles = int64_t {1} << (q - KA);
                j.n_units = static_cast<int32_t>(units_for(j.n_tiles, &j.tiles_per_unit));
                j.n_rows = static_cast<int32_t>(ip.rows_of_block[b].size());
                j.part = part_size;
                j.succ = -1;
                for (int32_t r = 0; r < j.n_rows; ++r) {
                    const int64_t grow = row0 + ip.rows_of_block[b][static_cast<size_t>(r)];
                    row_src[static_cast<size_t>(grow - small_rows_end)] =
                        RowSrc {j.part + static_cast<int64_t>(r) * j.n_units, j.n_units, 0};
                }
                part_size += static_cast<int64_t>(j.n_rows) * j.n_units;
                chain[k].push_back(static_cast<int32_t>(jobs.size()));
                jobs.push_back(j);
                alg += 4.0 * state_bytes;
            }
        }
        for (size_t c = 1; c < chain[k].size(); ++c) {
            jobs[static_cast<size_t>(chain[k][c - 1])].succ = chain[k][c];
        }
        ip = ItemPlan<T>();  // free the item's copy
    }

    // ready queues per wave: each item's first job, the costliest chains first;
    // later jobs are appended on the device as their predecessors finish
    std::vector<std::vector<int32_t>> queue0(static_cast<size_t>(B->n_waves));
    std::vector<int32_t> wave_jobs(static_cast<size_t>(B->n_waves), 0);
    {
        std::vector<std::vector<size_t>> by_wave(static_cast<size_t>(B->n_waves));
        for (size_t k = 0; k < large.size(); ++k) {
            if (!chain[k].empty()) {  // compiled items have no jobs
                by_wave[static_cast<size_t>(wave_of[k])].push_back(k);
            }
        }
        for (size_t w = 0; w < by_wave.size(); ++w) {
            auto chain_cost = [&](size_t k) {
                double c = 0.0;
                for (int32_t jid : chain[k]) {
                    c += static_cast<double>(jobs[static_cast<size_t>(jid)].n_tiles);
                }
                return c;
            };
            std::vector<size_t> order = by_wave[w];
            std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return chain_cost(x) > chain_cost(y); });
            for (size_t k : order) {
                queue0[w].push_back(chain[k].front());
                wave_jobs[w] += static_cast<int32_t>(chain[k].size());
            }
        }
    }
    B->n_jobs = static_cast<int64_t>(jobs.size());
    B->n_units = 0;
    for (const auto& j : jobs) {
        B->n_units += j.n_units;
    }

    // parameter -> rows (CSR, rows in id order)
    std::vector<int64_t> p_first(static_cast<size_t>(n_params) + 1, 0);
    std::vector<int64_t> p_rows(row_param.size());
    for (int64_t p : row_param) {
        ++p_first[static_cast<size_t>(p) + 1];
    }
    for (size_t p = 0; p < static_cast<size_t>(n_params); ++p) {
        p_first[p + 1] += p_first[p];
    }
    {
        std::vector<int64_t> fill(p_first.begin(), p_first.end() - 1);
        for (size_t r = 0; r < row_param.size(); ++r) {
            p_rows[static_cast<size_t>(fill[static_cast<size_t>(row_param[r])]++)] = static_cast<int64_t>(r);
        }
    }

    // --- device metadata
    Layout lay;
    const size_t o_sitems = lay.add(sitems.size() * sizeof(SItem));
    const size_t o_sops = lay.add(sops.size() * sizeof(SOp<T>));
    const size_t o_strs = lay.add(strs.size() * sizeof(BStr));
    const size_t o_insts = lay.add(insts.size() * sizeof(BInst));
    const size_t o_jobs = lay.add(jobs.size() * sizeof(BJob));
    // per wave: the queue's initial contents (static) and its head and tail
    std::vector<size_t> o_q0(queue0.size());
    std::vector<std::vector<int32_t>> q_init(queue0.size());
    std::vector<unsigned long long> ht_init;
    for (size_t w = 0; w < queue0.size(); ++w) {
        q_init[w].assign(static_cast<size_t>(wave_jobs[w]), -1);
        std::copy(queue0[w].begin(), queue0[w].end(), q_init[w].begin());
        o_q0[w] = lay.add(q_init[w].size() * sizeof(int32_t));
        ht_init.push_back(0ULL);
        ht_init.push_back(static_cast<unsigned long long>(queue0[w].size()));
    }
    const size_t o_ht0 = lay.add(ht_init.size() * sizeof(unsigned long long));
    const size_t o_fblk = lay.add(gf.blocks.size() * sizeof(FBlock));
    const size_t o_fph = lay.add(gf.phases.size() * sizeof(FPhase));
    const size_t o_fops = lay.add(gf.ops.size() * sizeof(FOp<T>));
    const size_t o_bblk = lay.add(gb.blocks.size() * sizeof(FBlock));
    const size_t o_bph = lay.add(gb.phases.size() * sizeof(FPhase));
    const size_t o_bops = lay.add(gb.ops.size() * sizeof(FOpA<T>));
    const size_t o_patch = lay.add(patches.size() * sizeof(BPatch));
    const size_t o_rsrc = lay.add(row_src.size() * sizeof(RowSrc));
    const size_t o_esrc = lay.add(esrc.size() * sizeof(ESrc));
    const size_t o_pfirst = lay.add(p_first.size() * sizeof(int64_t));
    const size_t o_prows = lay.add(p_rows.size() * sizeof(int64_t));
    // compiled classes' launch arrays, 8-byte words per class: states, lambdas,
    // item (BInst) indices, energy bases, then per forward block the items' op
    // records, per adjoint block their op records and partials' bases
    struct ClassWords
    {
        size_t a, l, list, ebase;
        std::vector<size_t> fop, bop, pbase;
    };
    std::vector<ClassWords> cw(cls.size());
    size_t n_words = 0;
    for (size_t c = 0; c < cls.size(); ++c) {
        const size_t n = cls[c].members.size();
        const size_t k0 = cls[c].members.front();
        cw[c].a = n_words;
        cw[c].l = n_words + n;
        cw[c].list = n_words + 2 * n;
        cw[c].ebase = n_words + 3 * n;
        n_words += 4 * n;
        for (size_t b = 0; b < item_fop[k0].size(); ++b) {
            cw[c].fop.push_back(n_words);
            n_words += n;
        }
        for (size_t b = 0; b < item_bop[k0].size(); ++b) {
            cw[c].bop.push_back(n_words);
            cw[c].pbase.push_back(n_words + n);
            n_words += 2 * n;
        }
    }
    const size_t o_cls = lay.add(n_words * sizeof(uint64_t));
    const size_t upload_end = lay.size;  // everything above is uploaded once, here
    const size_t o_params = lay.add(static_cast<size_t>(n_params) * sizeof(double));
    const size_t o_part = lay.add(static_cast<size_t>(part_size) * sizeof(double));
    const size_t o_epart = lay.add(static_cast<size_t>(epart_size) * sizeof(double));
    const size_t o_rowval = lay.add(row_param.size() * sizeof(double));
    // queues (rewritten from their initial contents by every evaluation)
    std::vector<size_t> o_q(queue0.size());
    for (size_t w = 0; w < queue0.size(); ++w) {
        o_q[w] = lay.add(q_init[w].size() * sizeof(int32_t));
    }
    const size_t o_ht = lay.add(ht_init.size() * sizeof(unsigned long long));
    // counters (zeroed by every evaluation): small-item queue, status, per job units done and taken
    const size_t count_bytes = sizeof(unsigned int) * 2 + 2 * sizeof(int) * jobs.size();
    const size_t o_count = lay.add(count_bytes);
    B->out_bytes = static_cast<size_t>(n_items + n_params) * sizeof(double) + sizeof(double);
    const size_t o_out = lay.add(B->out_bytes);

    KT_CUDA(cudaMalloc(&B->meta, lay.size));
    if (arena_bytes > 0) {
        KT_CUDA(cudaMalloc(&B->arena, arena_bytes));
    }
    B->device_bytes = lay.size + arena_bytes;
    {
        std::vector<unsigned char> host(upload_end, 0);
        auto put = [&](size_t off, const void* src, size_t bytes) {
            if (bytes > 0) {
                std::memcpy(host.data() + off, src, bytes);
            }
        };
        put(o_sitems, sitems.data(), sitems.size() * sizeof(SItem));
        put(o_sops, sops.data(), sops.size() * sizeof(SOp<T>));
        put(o_strs, strs.data(), strs.size() * sizeof(BStr));
        put(o_insts, insts.data(), insts.size() * sizeof(BInst));
        put(o_jobs, jobs.data(), jobs.size() * sizeof(BJob));
        for (size_t w = 0; w < q_init.size(); ++w) {
            put(o_q0[w], q_init[w].data(), q_init[w].size() * sizeof(int32_t));
        }
        put(o_ht0, ht_init.data(), ht_init.size() * sizeof(unsigned long long));
        put(o_fblk, gf.blocks.data(), gf.blocks.size() * sizeof(FBlock));
        put(o_fph, gf.phases.data(), gf.phases.size() * sizeof(FPhase));
        put(o_fops, gf.ops.data(), gf.ops.size() * sizeof(FOp<T>));
        put(o_bblk, gb.blocks.data(), gb.blocks.size() * sizeof(FBlock));
        put(o_bph, gb.phases.data(), gb.phases.size() * sizeof(FPhase));
        put(o_bops, gb.ops.data(), gb.ops.size() * sizeof(FOpA<T>));
        put(o_patch, patches.data(), patches.size() * sizeof(BPatch));
        put(o_rsrc, row_src.data(), row_src.size() * sizeof(RowSrc));
        put(o_esrc, esrc.data(), esrc.size() * sizeof(ESrc));
        put(o_pfirst, p_first.data(), p_first.size() * sizeof(int64_t));
        put(o_prows, p_rows.data(), p_rows.size() * sizeof(int64_t));
        if (n_words > 0) {
            // device addresses: the arena's states and the merged op tables in this block
            std::vector<uint64_t> words(n_words, 0);
            const uint64_t arena0 = reinterpret_cast<uint64_t>(B->arena);
            const uint64_t fops0 = reinterpret_cast<uint64_t>(B->meta) + o_fops;
            const uint64_t bops0 = reinterpret_cast<uint64_t>(B->meta) + o_bops;
            for (size_t c = 0; c < cls.size(); ++c) {
                const auto& mem = cls[c].members;
                for (size_t i = 0; i < mem.size(); ++i) {
                    const size_t k = mem[i];
                    words[cw[c].a + i] = arena0 + static_cast<uint64_t>(insts[k].psi) * sizeof(C);
                    words[cw[c].l + i] = arena0 + static_cast<uint64_t>(insts[k].lam) * sizeof(C);
                    words[cw[c].list + i] = static_cast<uint64_t>(k);
                    words[cw[c].ebase + i] = static_cast<uint64_t>(item_ebase[k]);
                    for (size_t b = 0; b < cw[c].fop.size(); ++b) {
                        words[cw[c].fop[b] + i] = fops0 + static_cast<uint64_t>(item_fop[k][b]) * sizeof(FOp<T>);
                    }
                    for (size_t b = 0; b < cw[c].bop.size(); ++b) {
                        words[cw[c].bop[b] + i] = bops0 + static_cast<uint64_t>(item_bop[k][b]) * sizeof(FOpA<T>);
                        words[cw[c].pbase[b] + i] = static_cast<uint64_t>(item_pbase[k][b]);
                    }
                }
            }
            put(o_cls, words.data(), n_words * sizeof(uint64_t));
        }
        KT_CUDA(cudaMemcpy(B->meta, host.data(), upload_end, cudaMemcpyHostToDevice));
    }
    KT_CUDA(cudaMallocHost(reinterpret_cast<void**>(&B->h_params),
                           std::max<size_t>(8, static_cast<size_t>(n_params) * sizeof(double))));
    KT_CUDA(cudaMallocHost(reinterpret_cast<void**>(&B->h_out), B->out_bytes));
    KT_CUDA(cudaStreamCreateWithFlags(&B->s0, cudaStreamNonBlocking));
    KT_CUDA(cudaStreamCreateWithFlags(&B->s1, cudaStreamNonBlocking));
    KT_CUDA(cudaEventCreateWithFlags(&B->ev_fork, cudaEventDisableTiming));
    KT_CUDA(cudaEventCreateWithFlags(&B->ev_join, cudaEventDisableTiming));
    const int n_cs = std::min<int>(kt_batch_s::N_CLASS_STREAMS, static_cast<int>(cls.size()));
    for (int i = 0; i < n_cs; ++i) {
        KT_CUDA(cudaStreamCreateWithFlags(&B->cs[i], cudaStreamNonBlocking));
        KT_CUDA(cudaEventCreateWithFlags(&B->cev[i], cudaEventDisableTiming));
    }

    char* M = static_cast<char*>(B->meta);
    auto at = [&](size_t off) { return static_cast<void*>(M + off); };
    double* d_energies = static_cast<double*>(at(o_out));
    double* d_grads = d_energies + n_items;
    int* d_status_out = reinterpret_cast<int*>(d_grads + n_params);
    unsigned int* d_small_counter = static_cast<unsigned int*>(at(o_count));
    int* d_status = reinterpret_cast<int*>(d_small_counter + 1);
    int* d_done = reinterpret_cast<int*>(d_small_counter + 2);
    int* d_taken = d_done + jobs.size();
    unsigned long long* d_ht = static_cast<unsigned long long*>(at(o_ht));

    // launch shapes
    size_t small_smem = 0;
    for (const auto& si : sitems) {
        small_smem = std::max(small_smem, 2 * (size_t {1} << si.q) * sizeof(C));
    }
    int small_grid = 0;
    if (!sitems.empty()) {
        KT_CUDA(cudaFuncSetAttribute(k_batch_small<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(small_smem)));
        int per_sm = 0;
        KT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_small<T>, B_THREADS, small_smem));
        small_grid = static_cast<int>(std::min<int64_t>(static_cast<int64_t>(sitems.size()),
                                                        static_cast<int64_t>(std::max(1, per_sm)) * sm_count()));
    }
    const size_t fwd_smem = (sizeof(C) << K) + BATCH_FWD_MAX_OPS * sizeof(FOp<T>);
    const size_t bwd_smem = 2 * (sizeof(C) << KA) + BATCH_BWD_MAX_OPS * sizeof(FOpA<T>) +
                            BATCH_BWD_MAX_OPS * ADJ_WARPS * sizeof(double);
    const size_t ham_smem = HAM_SMEM_STRINGS * sizeof(BStr);
    const size_t big_smem = std::max({fwd_smem, bwd_smem, ham_smem});
    int big_grid = 0;
    if (!large.empty()) {
        KT_CUDA(cudaFuncSetAttribute(k_batch_persist<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(big_smem)));
        int per_sm = 0;
        KT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persist<T>, B_THREADS, big_smem));
        big_grid = std::max(1, per_sm) * sm_count();
    }

    // --- capture one evaluation
    int64_t launches = 0;
    cudaStream_t s0 = B->s0, s1 = B->s1;
    KT_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    auto chk = [&](cudaError_t e) {
        if (ce == cudaSuccess && e != cudaSuccess) {
            ce = e;
        }
    };
    if (n_params > 0) {
        chk(cudaMemcpyAsync(at(o_params), B->h_params, static_cast<size_t>(n_params) * sizeof(double),
                            cudaMemcpyHostToDevice, s0));
    }
    if (!patches.empty()) {
        const int64_t np = static_cast<int64_t>(patches.size());
        k_batch_patch<T><<<static_cast<unsigned>((np + 255) / 256), 256, 0, s0>>>(
            static_cast<const double*>(at(o_params)), static_cast<const BPatch*>(at(o_patch)), np,
            static_cast<FOp<T>*>(at(o_fops)), static_cast<FOpA<T>*>(at(o_bops)), static_cast<SOp<T>*>(at(o_sops)));
        chk(cudaGetLastError());
        ++launches;
    }
    chk(cudaMemsetAsync(at(o_count), 0, count_bytes, s0));
    for (size_t w = 0; w < q_init.size(); ++w) {
        chk(cudaMemcpyAsync(at(o_q[w]), at(o_q0[w]), q_init[w].size() * sizeof(int32_t), cudaMemcpyDeviceToDevice, s0));
    }
    if (!ht_init.empty()) {
        chk(cudaMemcpyAsync(d_ht, at(o_ht0), ht_init.size() * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                            s0));
    }
    chk(cudaMemsetAsync(d_status_out, 0, sizeof(double), s0));
    chk(cudaEventRecord(B->ev_fork, s0));
    chk(cudaStreamWaitEvent(s1, B->ev_fork, 0));
    if (!sitems.empty()) {
        k_batch_small<T><<<small_grid, B_THREADS, small_smem, s1>>>(
            static_cast<const SItem*>(at(o_sitems)), static_cast<int>(sitems.size()),
            static_cast<const SOp<T>*>(at(o_sops)), static_cast<const BStr*>(at(o_strs)), d_energies,
            static_cast<double*>(at(o_rowval)), with_grad, d_small_counter);
        chk(cudaGetLastError());
        ++launches;
    }
    chk(cudaEventRecord(B->ev_join, s1));
    // compiled classes: one chain per class (|0...0>, forward blocks, lambda = H psi
    // and the energy partials, adjoint blocks), the classes spread over streams
    for (int i = 0; i < n_cs; ++i) {
        chk(cudaStreamWaitEvent(B->cs[i], B->ev_fork, 0));
    }
    {
        uint64_t* words_dev = static_cast<uint64_t*>(at(o_cls));
        C* arena = static_cast<C*>(B->arena);
        for (size_t c = 0; c < cls.size(); ++c) {
            const Class& cl = cls[c];
            cudaStream_t st = B->cs[c % static_cast<size_t>(n_cs)];
            const unsigned n = static_cast<unsigned>(cl.members.size());
            void* a_list = words_dev + cw[c].a;
            void* l_list = words_dev + cw[c].l;
            k_batch_basis<C><<<dim3(static_cast<unsigned>(cl.cpi_f), n), B_THREADS, 0, st>>>(
                static_cast<void* const*>(a_list), uint64_t {1} << cl.q);
            chk(cudaGetLastError());
            ++launches;
            unsigned long long nt_f = 1ULL << (cl.q - K_FWD<T>);
            for (size_t b = 0; b < cl.fk.size(); ++b) {
                void* o_list = words_dev + cw[c].fop[b];
                void* args[] = {&a_list, &o_list, &nt_f};
                chk(cudaLaunchKernel(cl.fk[b], dim3(static_cast<unsigned>(cl.cpi_f), n), dim3(B_THREADS), args,
                                     static_cast<size_t>(cl.fsmem), st));
                ++launches;
            }
            const uint64_t n_chunks = uint64_t {1} << (cl.q - K_FWD<T>);
            const unsigned ham_grid = static_cast<unsigned>(
                std::min<uint64_t>(n_chunks * n, static_cast<uint64_t>(4 * sm_count())));
            k_batch_ham_items<T><<<ham_grid, B_THREADS, ham_smem, st>>>(
                arena, static_cast<const BInst*>(at(o_insts)), reinterpret_cast<const int64_t*>(words_dev + cw[c].list),
                reinterpret_cast<const int64_t*>(words_dev + cw[c].ebase), static_cast<const BStr*>(at(o_strs)),
                static_cast<double*>(at(o_epart)), K_FWD<T>, with_grad, static_cast<uint64_t>(n), n_chunks);
            chk(cudaGetLastError());
            ++launches;
            if (with_grad) {
                unsigned long long nt_a = 1ULL << (cl.q - K_BWD<T>);
                double* part = static_cast<double*>(at(o_part));
                for (size_t b = 0; b < cl.bk.size(); ++b) {
                    void* o_list = words_dev + cw[c].bop[b];
                    void* pbase = words_dev + cw[c].pbase[b];
                    int rows = cl.rows[b];
                    void* args[] = {&a_list, &l_list, &o_list, &pbase, &part, &nt_a, &rows};
                    chk(cudaLaunchKernel(cl.bk[b], dim3(static_cast<unsigned>(cl.cpi_a), n), dim3(B_THREADS), args,
                                         static_cast<size_t>(cl.bsmem[b]), st));
                    ++launches;
                }
            }
        }
    }
    for (int i = 0; i < n_cs; ++i) {
        chk(cudaEventRecord(B->cev[i], B->cs[i]));
    }
    for (size_t w = 0; w < q_init.size(); ++w) {
        if (wave_jobs[w] == 0) {
            continue;  // every item of the wave runs compiled kernels
        }
        BArgs<T> a {};
        a.arena = static_cast<C*>(B->arena);
        a.jobs = static_cast<const BJob*>(at(o_jobs));
        a.insts = static_cast<const BInst*>(at(o_insts));
        a.queue = static_cast<int*>(at(o_q[w]));
        a.n_jobs = wave_jobs[w];
        a.fblk = static_cast<const FBlock*>(at(o_fblk));
        a.fph = static_cast<const FPhase*>(at(o_fph));
        a.fops = static_cast<const FOp<T>*>(at(o_fops));
        a.bblk = static_cast<const FBlock*>(at(o_bblk));
        a.bph = static_cast<const FPhase*>(at(o_bph));
        a.bops = static_cast<const FOpA<T>*>(at(o_bops));
        a.strs = static_cast<const BStr*>(at(o_strs));
        a.part = static_cast<double*>(at(o_part));
        a.epart = static_cast<double*>(at(o_epart));
        a.done = d_done;
        a.taken = d_taken;
        a.qhead = d_ht + 2 * w;
        a.qtail = d_ht + 2 * w + 1;
        a.status = d_status;
        a.with_grad = with_grad;
        a.spin_limit = tuning().batch_spin_limit;
        k_batch_persist<T><<<big_grid, B_THREADS, big_smem, s0>>>(a);
        chk(cudaGetLastError());
        ++launches;
    }
    chk(cudaStreamWaitEvent(s0, B->ev_join, 0));
    for (int i = 0; i < n_cs; ++i) {
        chk(cudaStreamWaitEvent(s0, B->cev[i], 0));
    }
    if (!esrc.empty()) {
        const int64_t n = static_cast<int64_t>(esrc.size());
        k_batch_energy<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s0>>>(
            static_cast<const double*>(at(o_epart)), static_cast<const ESrc*>(at(o_esrc)), n, d_energies);
        chk(cudaGetLastError());
        ++launches;
    }
    if (with_grad && !row_src.empty()) {
        const int64_t n = static_cast<int64_t>(row_src.size());
        k_batch_rows<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s0>>>(
            static_cast<const double*>(at(o_part)), static_cast<const RowSrc*>(at(o_rsrc)), n,
            static_cast<double*>(at(o_rowval)) + small_rows_end);
        chk(cudaGetLastError());
        ++launches;
    }
    if (with_grad && n_params > 0) {
        k_batch_grads<<<static_cast<unsigned>((n_params + 255) / 256), 256, 0, s0>>>(
            static_cast<const double*>(at(o_rowval)), static_cast<const int64_t*>(at(o_pfirst)),
            static_cast<const int64_t*>(at(o_prows)), n_params, d_grads);
        chk(cudaGetLastError());
        ++launches;
    }
    chk(cudaMemcpyAsync(d_status_out, d_status, sizeof(int), cudaMemcpyDeviceToDevice, s0));
    chk(cudaMemcpyAsync(B->h_out, d_energies, B->out_bytes, cudaMemcpyDeviceToHost, s0));
    const cudaError_t end = cudaStreamEndCapture(s0, &B->graph);
    if (ce != cudaSuccess) {
        return cuda_fail(ce, "batch graph capture");
    }
    if (end != cudaSuccess) {
        return cuda_fail(end, "cudaStreamEndCapture(batch)");
    }
    KT_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
    B->launches = launches;
    B->alg_bytes = alg;
    B->n_small = static_cast<int64_t>(small.size());
    B->n_large = static_cast<int64_t>(large.size());
    B->n_compiled_items = 0;
    for (const Class& c : cls) {
        B->n_compiled_items += static_cast<int64_t>(c.members.size());
    }
    return KT_OK;
}

}  // namespace
}  // namespace kt

extern "C" {

int32_t kt_batch_create(const kt_batch_item* items, int64_t n_items, const kt_gate* gates, int64_t n_gates_total,
                        int64_t n_params_total, const kt_pauli* strings, const double* coeffs, int64_t n_strings_total,
                        int32_t dtype, int32_t with_grad, kt_batch* out)
{
    try {
        if (out == nullptr) {
            return kt::fail(KT_ERR_INVALID, "out is NULL");
        }
        *out = nullptr;
        if (n_items < 1 || items == nullptr || n_gates_total < 0 || (n_gates_total > 0 && gates == nullptr) ||
            n_params_total < 0 || n_strings_total < 1 || strings == nullptr) {
            return kt::fail(KT_ERR_INVALID, "bad batch arrays");
        }
        if (dtype != KT_C128 && dtype != KT_C64) {
            return kt::fail(KT_ERR_INVALID, "dtype must be KT_C128 or KT_C64");
        }
        for (int64_t b = 0; b < n_items; ++b) {
            const kt_batch_item& it = items[b];
            if (it.n_qubits < 1 || it.n_qubits > 30 || it.gate_offset < 0 || it.n_gates < 0 ||
                it.gate_offset + it.n_gates > n_gates_total || it.param_offset < 0 || it.n_params < 0 ||
                it.param_offset + it.n_params > n_params_total || it.string_offset < 0 || it.n_strings < 1 ||
                it.string_offset + it.n_strings > n_strings_total) {
                return kt::fail(KT_ERR_INVALID, "batch item " + std::to_string(b) + " out of range");
            }
            const uint64_t mask = (uint64_t {1} << it.n_qubits) - 1;
            for (int64_t s = 0; s < it.n_strings; ++s) {
                const kt_pauli& p = strings[it.string_offset + s];
                if (((p.x_mask | p.z_mask) & ~mask) != 0) {
                    return kt::fail(KT_ERR_INVALID, "batch item " + std::to_string(b) + ": Pauli string " +
                                                        std::to_string(s) + " acts outside its qubits");
                }
            }
        }
        auto* B = new kt_batch_s();
        B->dtype = dtype;
        B->with_grad = with_grad ? 1 : 0;
        B->n_items = n_items;
        B->n_params = n_params_total;
        const int32_t rc = (dtype == KT_C128)
                               ? kt::create<double>(items, n_items, gates, n_params_total, strings, coeffs, B->with_grad, B)
                               : kt::create<float>(items, n_items, gates, n_params_total, strings, coeffs, B->with_grad, B);
        if (rc != KT_OK) {
            kt::release(B);
            delete B;
            return rc;
        }
        *out = B;
        return KT_OK;
    } catch (const std::exception& e) {
        return kt::fail(KT_ERR_INVALID, e.what());
    }
}

int32_t kt_batch_set_stream(kt_batch b, void* stream)
{
    if (b == nullptr) {
        return kt::fail(KT_ERR_INVALID, "batch is NULL");
    }
    b->user = static_cast<cudaStream_t>(stream);
    return KT_OK;
}

int32_t kt_batch_evaluate(kt_batch b, const double* params, double* energies, double* grads)
{
    if (b == nullptr || energies == nullptr || (b->n_params > 0 && params == nullptr)) {
        return kt::fail(KT_ERR_INVALID, "batch, energies or params is NULL");
    }
    if (grads != nullptr && !b->with_grad) {
        return kt::fail(KT_ERR_INVALID, "batch was created without gradients");
    }
    if (b->n_params > 0) {
        std::memcpy(b->h_params, params, static_cast<size_t>(b->n_params) * sizeof(double));
    }
    KT_CUDA(cudaGraphLaunch(b->exec, b->user));
    KT_CUDA(cudaStreamSynchronize(b->user));
    const double* o = b->h_out;
    int status = 0;
    std::memcpy(&status, o + b->n_items + b->n_params, sizeof(int));
    if (status != 0) {
        return kt::fail(KT_ERR_TIMEOUT, "batch: a CTA waited too long for a ready job");
    }
    std::memcpy(energies, o, static_cast<size_t>(b->n_items) * sizeof(double));
    if (grads != nullptr && b->n_params > 0) {
        std::memcpy(grads, o + b->n_items, static_cast<size_t>(b->n_params) * sizeof(double));
    }
    return KT_OK;
}

int32_t kt_batch_stats(kt_batch b, int64_t* small_items, int64_t* large_items, int64_t* waves, int64_t* jobs,
                       int64_t* units, int64_t* launches, double* alg_bytes, double* device_bytes)
{
    if (b == nullptr) {
        return kt::fail(KT_ERR_INVALID, "batch is NULL");
    }
    if (small_items) *small_items = b->n_small;
    if (large_items) *large_items = b->n_large;
    if (waves) *waves = b->n_waves;
    if (jobs) *jobs = b->n_jobs;
    if (units) *units = b->n_units;
    if (launches) *launches = b->launches;
    if (alg_bytes) *alg_bytes = b->alg_bytes;
    if (device_bytes) *device_bytes = static_cast<double>(b->device_bytes);
    return KT_OK;
}

int32_t kt_batch_compiled(kt_batch b, int64_t* classes, int64_t* items)
{
    if (b == nullptr) {
        return kt::fail(KT_ERR_INVALID, "batch is NULL");
    }
    if (classes) *classes = b->n_classes;
    if (items) *items = b->n_compiled_items;
    return KT_OK;
}

int32_t kt_batch_destroy(kt_batch b)
{
    if (b == nullptr) {
        return KT_OK;
    }
    cudaStreamSynchronize(b->user);
    kt::release(b);
    delete b;
    return KT_OK;
}

int32_t kt_batch_run(const kt_batch_item* items, int64_t n_items, const kt_gate* gates, int64_t n_gates_total,
                     const double* params, int64_t n_params_total, const kt_pauli* strings, const double* coeffs,
                     int64_t n_strings_total, int32_t dtype, double* energies, double* grads, void* stream)
{
    kt_batch b = nullptr;
    int32_t rc = kt_batch_create(items, n_items, gates, n_gates_total, n_params_total, strings, coeffs,
                                 n_strings_total, dtype, grads != nullptr ? 1 : 0, &b);
    if (rc != KT_OK) {
        return rc;
    }
    kt_batch_set_stream(b, stream);
    rc = kt_batch_evaluate(b, params, energies, grads);
    kt_batch_destroy(b);
    return rc;
}

}  // extern "C"
