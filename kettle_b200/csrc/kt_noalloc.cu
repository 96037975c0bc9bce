// kt_noalloc.cu — Pauli expectation values without any device allocation.
//
// kt_sv_expect keeps its reduction tables and per-block partial sums in a
// scratch buffer it grows with cudaMalloc.  Some callers cannot allow that:
// a host that owns every byte of device memory through its own pool or
// arena, or a control loop that must not allocate once it is running.  For
// them, kt_sv_expect_noalloc computes the same values with its scratch in one
// file-scope device array of fixed size, so the call allocates nothing on the
// device: it only copies the caller's small host tables into that array and
// launches the same kernels as kt_sv_expect.
//
// The array lives in every GPU that loads the library, from module load until
// the process exits (about 2.5 MB).  Host code never passes the array's name
// to a kernel (in host code that name is only a stand-in for the device
// symbol): the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, on the first call made on
// it, and cached.
#include <algorithm>
#include <array>
#include <mutex>

#include "kt_internal.cuh"

namespace kt
{
int32_t pauli_terms_launch(const void* amps, int n, int32_t dtype, const void* slots, int n_slots, const uint64_t* xm,
                           const uint64_t* zm, const int32_t* phase, int64_t n_strings, double* partial, int blocks,
                           double* terms, cudaStream_t stream);
int32_t weighted_total_launch(const double* terms, const double* coeffs, int64_t n, double* total, cudaStream_t stream);
int pauli_slot_bytes();
int pauli_slot_width();
int pauli_blocks(int n_bits);
}  // namespace kt

namespace
{

constexpr int NA_MAX_STRINGS = KT_NOALLOC_MAX_STRINGS;
constexpr int NA_BLOCKS = 592;            // reduction blocks per string: kt_sv_expect's 4 per SM of a B200
constexpr int NA_SLOT_WIDTH = 16;         // strings per slot, as kt_sv_expect groups them

// layout-identical to the slot record the reduction kernels read
struct NaSlot
{
    uint64_t x;
    int32_t h;
    int32_t first;
    int32_t count;
    int32_t pad;
};

constexpr size_t al256(size_t v)
{
    return (v + 255) & ~size_t {255};
}

constexpr size_t OFF_SLOTS = 0;
constexpr size_t OFF_X = al256(OFF_SLOTS + NA_MAX_STRINGS * sizeof(NaSlot));
constexpr size_t OFF_Z = al256(OFF_X + NA_MAX_STRINGS * 8);
constexpr size_t OFF_P = al256(OFF_Z + NA_MAX_STRINGS * 8);
constexpr size_t OFF_PART = al256(OFF_P + NA_MAX_STRINGS * 4);
constexpr size_t OFF_TERMS = al256(OFF_PART + size_t {NA_MAX_STRINGS} * NA_BLOCKS * 8);
constexpr size_t OFF_COEF = al256(OFF_TERMS + NA_MAX_STRINGS * 16);
constexpr size_t OFF_TOTAL = al256(OFF_COEF + NA_MAX_STRINGS * 16);
constexpr size_t NA_BYTES = al256(OFF_TOTAL + 16);

// The scratch.  Every call overwrites the parts it reads back, so nothing in it
// has to start at zero; each reduction block writes its own partial sum before
// the finalisation reads it.  Calls that overlap on the GPU share it and race.
__device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

std::mutex g_addr_mutex;
std::array<void*, 128> g_addr {};  // device address of g_noalloc_scratch, per device ordinal

int32_t fail(int32_t code, const std::string& msg)
{
    kt::set_error(code, msg);
    return code;
}

// An exception (std::bad_alloc from std::to_string, say) must not cross the C interface.
template <typename F>
int32_t guarded(F&& f)
{
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return fail(KT_ERR_NOMEM, "kt_sv_expect_noalloc: host allocation failed");
    } catch (const std::exception& e) {
        return fail(KT_ERR_INVALID, std::string("kt_sv_expect_noalloc: ") + e.what());
    } catch (...) {
        return fail(KT_ERR_INVALID, "kt_sv_expect_noalloc: unknown exception");
    }
}

// Once per device, with that device current: the device address of the array.
int32_t scratch_address(char** out)
{
    int dev = 0;
    KT_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= static_cast<int>(g_addr.size())) {
        return fail(KT_ERR_UNSUPPORTED, "kt_sv_expect_noalloc: device ordinal out of range");
    }
    std::lock_guard<std::mutex> lock {g_addr_mutex};
    if (g_addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            return kt::cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        }
        g_addr[dev] = p;
    }
    *out = static_cast<char*>(g_addr[dev]);
    return KT_OK;
}

int32_t expect_noalloc(const void* device_amps, int32_t n_qubits, int32_t dtype, const kt_pauli* strings,
                       int64_t n_strings, const double* coeffs, double* out_terms, double* out_total, void* stream)
{
    if (device_amps == nullptr) {
        return fail(KT_ERR_INVALID, "kt_sv_expect_noalloc: null device amplitude pointer");
    }
    if (dtype != KT_C128 && dtype != KT_C64) {
        return fail(KT_ERR_INVALID, "kt_sv_expect_noalloc: dtype must be KT_C128 or KT_C64");
    }
    if (n_qubits < 1 || n_qubits > 34) {
        return fail(KT_ERR_INVALID, "kt_sv_expect_noalloc: qubit count out of range (1..34)");
    }
    if (n_strings < 0 || n_strings > NA_MAX_STRINGS) {
        return fail(KT_ERR_INVALID, "kt_sv_expect_noalloc: at most " + std::to_string(NA_MAX_STRINGS) +
                                        " Pauli strings per call (got " + std::to_string(n_strings) +
                                        "); split the operator or use kt_sv_expect");
    }
    if (n_strings > 0 && strings == nullptr) {
        return fail(KT_ERR_INVALID, "kt_sv_expect_noalloc: null Pauli string array");
    }
    if (kt::pauli_slot_bytes() != static_cast<int>(sizeof(NaSlot)) || kt::pauli_slot_width() != NA_SLOT_WIDTH) {
        return fail(KT_ERR_UNSUPPORTED, "kt_sv_expect_noalloc: slot layout mismatch");
    }
    if (n_strings == 0) {
        if (out_total) {
            out_total[0] = 0.0;
            out_total[1] = 0.0;
        }
        return KT_OK;
    }
    const uint64_t valid = (n_qubits >= 64) ? ~uint64_t {0} : ((uint64_t {1} << n_qubits) - 1);
    for (int64_t k = 0; k < n_strings; ++k) {
        if ((strings[k].x_mask & ~valid) != 0 || (strings[k].z_mask & ~valid) != 0) {
            return fail(KT_ERR_INVALID, "kt_sv_expect_noalloc: Pauli string acts on a qubit beyond the state");
        }
    }
    char* dev = nullptr;
    if (const int32_t rc = scratch_address(&dev); rc != KT_OK) {
        return rc;
    }
    const auto st = static_cast<cudaStream_t>(stream);
    const int ns = static_cast<int>(n_strings);
    // group by X/Y mask (stable), slots of at most NA_SLOT_WIDTH strings; host tables live on the stack
    std::array<int, NA_MAX_STRINGS> order;
    for (int k = 0; k < ns; ++k) {
        order[k] = k;
    }
    std::stable_sort(order.begin(), order.begin() + ns,
                     [&](int a, int b) { return strings[a].x_mask < strings[b].x_mask; });
    std::array<NaSlot, NA_MAX_STRINGS> slots {};
    std::array<uint64_t, NA_MAX_STRINGS> hx {};
    std::array<uint64_t, NA_MAX_STRINGS> hz {};
    std::array<int32_t, NA_MAX_STRINGS> hp {};
    int n_slots = 0;
    for (int p = 0; p < ns;) {
        const uint64_t x = strings[order[p]].x_mask;
        int q = p;
        while (q < ns && strings[order[q]].x_mask == x && q - p < NA_SLOT_WIDTH) {
            ++q;
        }
        NaSlot sl {};
        sl.x = x;
        sl.h = (x == 0) ? -1 : 63 - __builtin_clzll(x);
        sl.first = p;
        sl.count = q - p;
        slots[n_slots++] = sl;
        p = q;
    }
    for (int p = 0; p < ns; ++p) {
        hx[p] = strings[order[p]].x_mask;
        hz[p] = strings[order[p]].z_mask;
        hp[p] = strings[order[p]].phase & 3;
    }
    KT_CUDA(cudaMemcpyAsync(dev + OFF_SLOTS, slots.data(), n_slots * sizeof(NaSlot), cudaMemcpyHostToDevice, st));
    KT_CUDA(cudaMemcpyAsync(dev + OFF_X, hx.data(), ns * 8, cudaMemcpyHostToDevice, st));
    KT_CUDA(cudaMemcpyAsync(dev + OFF_Z, hz.data(), ns * 8, cudaMemcpyHostToDevice, st));
    KT_CUDA(cudaMemcpyAsync(dev + OFF_P, hp.data(), ns * 4, cudaMemcpyHostToDevice, st));
    // kt_sv_expect's block count where it fits the array (every GPU of up to
    // 148 SMs): the partial sums are then added in the same order, bit for bit
    const int blocks = std::min(NA_BLOCKS, kt::pauli_blocks(n_qubits));
    auto* d_terms = reinterpret_cast<double*>(dev + OFF_TERMS);
    if (const int32_t rc = kt::pauli_terms_launch(device_amps, n_qubits, dtype, dev + OFF_SLOTS, n_slots,
                                                  reinterpret_cast<const uint64_t*>(dev + OFF_X),
                                                  reinterpret_cast<const uint64_t*>(dev + OFF_Z),
                                                  reinterpret_cast<const int32_t*>(dev + OFF_P), n_strings,
                                                  reinterpret_cast<double*>(dev + OFF_PART), blocks, d_terms, st);
        rc != KT_OK) {
        return rc;
    }
    // terms come back in slot order; put them in input order
    std::array<double, 2 * NA_MAX_STRINGS> sorted {};
    std::array<double, 2 * NA_MAX_STRINGS> terms {};
    KT_CUDA(cudaMemcpyAsync(sorted.data(), d_terms, ns * 16, cudaMemcpyDeviceToHost, st));
    KT_CUDA(cudaStreamSynchronize(st));
    for (int p = 0; p < ns; ++p) {
        terms[2 * order[p]] = sorted[2 * p];
        terms[2 * order[p] + 1] = sorted[2 * p + 1];
    }
    if (out_terms != nullptr) {
        std::copy(terms.begin(), terms.begin() + 2 * ns, out_terms);
    }
    if (out_total != nullptr) {
        // the weighted sum in input order, in FP64 on the device
        KT_CUDA(cudaMemcpyAsync(d_terms, terms.data(), ns * 16, cudaMemcpyHostToDevice, st));
        const double* d_coef = nullptr;
        if (coeffs != nullptr) {
            KT_CUDA(cudaMemcpyAsync(dev + OFF_COEF, coeffs, ns * 16, cudaMemcpyHostToDevice, st));
            d_coef = reinterpret_cast<const double*>(dev + OFF_COEF);
        }
        auto* d_total = reinterpret_cast<double*>(dev + OFF_TOTAL);
        if (const int32_t rc = kt::weighted_total_launch(d_terms, d_coef, n_strings, d_total, st); rc != KT_OK) {
            return rc;
        }
        KT_CUDA(cudaMemcpyAsync(out_total, d_total, 16, cudaMemcpyDeviceToHost, st));
        KT_CUDA(cudaStreamSynchronize(st));
    }
    return KT_OK;
}

}  // namespace

extern "C" int32_t kt_sv_expect_noalloc(const void* device_amps, int32_t n_qubits, int32_t dtype,
                                        const kt_pauli* strings, int64_t n_strings, const double* coeffs,
                                        double* out_terms, double* out_total, void* stream)
{
    return guarded([&] {
        return expect_noalloc(device_amps, n_qubits, dtype, strings, n_strings, coeffs, out_terms, out_total, stream);
    });
}
