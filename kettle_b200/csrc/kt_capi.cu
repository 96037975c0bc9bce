// kt_capi.cu — the extern "C" entry points of include/kettle_b200.h.
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "kt_internal.cuh"

namespace kt
{
const char* last_error_cstr();
}

namespace
{

template <typename F>
int32_t guard(F&& f)
{
    try {
        const int32_t rc = f();
        return rc == KT_OK ? kt::jit_async_error() : rc;
    } catch (const std::bad_alloc&) {
        kt::set_error(KT_ERR_NOMEM, "host allocation failed");
        return KT_ERR_NOMEM;
    } catch (const std::exception& e) {
        kt::set_error(KT_ERR_INVALID, e.what());
        return KT_ERR_INVALID;
    } catch (...) {
        kt::set_error(KT_ERR_INVALID, "unknown exception");
        return KT_ERR_INVALID;
    }
}

int32_t invalid(const char* msg)
{
    kt::set_error(KT_ERR_INVALID, msg);
    return KT_ERR_INVALID;
}

int32_t check_dtype(int32_t dtype)
{
    return (dtype == KT_C128 || dtype == KT_C64) ? KT_OK : invalid("dtype must be KT_C128 or KT_C64");
}

int32_t alloc_state(kt::State& st, int bits, int32_t dtype)
{
    st.n_bits = bits;
    st.dtype = dtype;
    const size_t bytes = (size_t {1} << bits) * st.amp_bytes();
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        return kt::cuda_fail(e, "cudaMalloc(state)");
    }
    st.amps = p;
    st.owned = true;
    return KT_OK;
}

void free_state(kt::State& st)
{
    if (st.owned && st.amps != nullptr) {
        cudaFree(st.amps);
    }
    st.amps = nullptr;
    st.scratch.release();
    st.scratch2.release();
}

int32_t upload(kt::State& st, const double* host, uint64_t n_amps)
{
    if (host == nullptr) {
        return invalid("null host buffer");
    }
    if (n_amps != st.n_amps()) {
        return invalid("amplitude count does not match the state size");
    }
    if (st.dtype == KT_C128) {
        KT_CUDA(cudaMemcpyAsync(st.amps, host, n_amps * 16, cudaMemcpyHostToDevice, st.stream));
        KT_CUDA(cudaStreamSynchronize(st.stream));
        return KT_OK;
    }
    if (const int32_t rc = st.scratch2.reserve(n_amps * 16); rc != KT_OK) {
        return rc;
    }
    KT_CUDA(cudaMemcpyAsync(st.scratch2.ptr, host, n_amps * 16, cudaMemcpyHostToDevice, st.stream));
    if (const int32_t rc = kt::launch_convert_to_state(st, static_cast<const double*>(st.scratch2.ptr), n_amps);
        rc != KT_OK) {
        return rc;
    }
    KT_CUDA(cudaStreamSynchronize(st.stream));
    return KT_OK;
}

int32_t download(kt::State& st, double* host, uint64_t n_amps)
{
    if (host == nullptr) {
        return invalid("null host buffer");
    }
    if (n_amps != st.n_amps()) {
        return invalid("amplitude count does not match the state size");
    }
    if (st.dtype == KT_C128) {
        return kt::copy_d2h(host, st.amps, n_amps * 16, st.stream);
    }
    if (const int32_t rc = st.scratch2.reserve(n_amps * 16); rc != KT_OK) {
        return rc;
    }
    if (const int32_t rc = kt::launch_convert_from_state(st, static_cast<double*>(st.scratch2.ptr), n_amps);
        rc != KT_OK) {
        return rc;
    }
    return kt::copy_d2h(host, st.scratch2.ptr, n_amps * 16, st.stream);
}

int32_t apply_lowered(kt::State& st, const std::vector<kt::LGate>& lg, int32_t mode)
{
    st.last_launches = 0;
    st.last_alg_bytes = 0.0;
    if (mode == KT_APPLY_PER_GATE) {
        for (const auto& g : lg) {
            if (const int32_t rc = kt::launch_gate_sweep(st, g); rc != KT_OK) {
                return rc;
            }
        }
        return KT_OK;
    }
    if (mode != KT_APPLY_FUSED) {
        return invalid("mode must be KT_APPLY_FUSED or KT_APPLY_PER_GATE");
    }
    return kt::apply_fused(st, lg);
}

}  // namespace

extern "C" {

const char* kt_last_error(void)
{
    return kt::last_error_cstr();
}

int32_t kt_version(void)
{
    return 100;
}

int32_t kt_device_synchronize(void)
{
    KT_CUDA(cudaDeviceSynchronize());
    return KT_OK;
}

int32_t kt_canonicals_mt19937(uint32_t seed, int64_t n, double* out)
{
    return guard([&]() -> int32_t {
        if (n < 0 || (n > 0 && out == nullptr)) {
            return invalid("bad output buffer");
        }
        std::mt19937 prng {seed};
        for (int64_t i = 0; i < n; ++i) {
            out[i] = std::generate_canonical<double, std::numeric_limits<double>::digits>(prng);
        }
        return KT_OK;
    });
}

int32_t kt_tuning_set(const char* name, int64_t value)
{
    return kt::tuning_set(name, value) ? KT_OK : invalid("unknown tuning knob");
}

int32_t kt_tuning_get(const char* name, int64_t* value)
{
    long long v = 0;
    if (value == nullptr || !kt::tuning_get(name, &v)) {
        return invalid("unknown tuning knob");
    }
    *value = v;
    return KT_OK;
}

int32_t kt_jit_compile_only(int32_t n_qubits, int32_t dtype, const kt_gate* gates, int64_t n_gates,
                            const double* params, int64_t n_params, int64_t* n_kernels)
{
    return guard([&]() -> int32_t {
        if (n_kernels == nullptr || n_gates < 0 || (n_gates > 0 && gates == nullptr)) {
            return invalid("bad arguments");
        }
        if (const int32_t rc = check_dtype(dtype); rc != KT_OK) {
            return rc;
        }
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, n_qubits, lg); rc != KT_OK) {
            return rc;
        }
        if (kt::tuning().adjoint_jit == 1) {
            // the backward sweep of the circuit read as an ansatz: the gates in
            // reverse order (their matrices do not change the kernels), every
            // parameterised rotation a gradient row
            std::vector<kt::AdjGate> sweep;
            int32_t rows = 0;
            for (int64_t i = 0; i < n_gates; ++i) {
                if (gates[i].param >= 0 && kt::gate_generator(gates[i].op) >= 0) {
                    ++rows;
                }
            }
            for (int64_t i = n_gates - 1; i >= 0; --i) {
                kt::AdjGate ag {};
                ag.adj = lg[static_cast<size_t>(i)];
                ag.row = -1;
                ag.gen = 0;
                if (gates[i].param >= 0 && kt::gate_generator(gates[i].op) >= 0) {
                    ag.gen = kt::gate_generator(gates[i].op);
                    ag.row = --rows;
                }
                sweep.push_back(ag);
            }
            return kt::jit_adjoint_compile_only(n_qubits, dtype, sweep, n_kernels);
        }
        return kt::jit_compile_only(n_qubits, dtype, lg, n_kernels);
    });
}

int32_t kt_sv_prepare(kt_sv sv, const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params)
{
    return guard([&]() -> int32_t {
        if (sv == nullptr) {
            return invalid("null handle");
        }
        if (n_gates < 0 || (n_gates > 0 && gates == nullptr)) {
            return invalid("bad gate array");
        }
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, sv->st.n_bits, lg); rc != KT_OK) {
            return rc;
        }
        return kt::jit_prepare(sv->st, lg);
    });
}

int32_t kt_jit_stats(int64_t* kernels_compiled, int64_t* block_launches, int32_t* failed)
{
    if (kernels_compiled == nullptr || block_launches == nullptr || failed == nullptr) {
        return invalid("null pointer");
    }
    kt::jit_stats(kernels_compiled, block_launches, failed);
    return KT_OK;
}

int32_t kt_jit_cache_stats(int64_t* nvrtc_compiles, int64_t* disk_hits)
{
    if (nvrtc_compiles == nullptr || disk_hits == nullptr) {
        return invalid("null pointer");
    }
    kt::jit_cache_stats(nvrtc_compiles, disk_hits);
    return KT_OK;
}

// ---- statevector --------------------------------------------------------------

int32_t kt_sv_create(int32_t n_qubits, int32_t dtype, kt_sv* out)
{
    return guard([&]() -> int32_t {
        if (out == nullptr) {
            return invalid("null output handle");
        }
        *out = nullptr;
        if (const int32_t rc = check_dtype(dtype); rc != KT_OK) {
            return rc;
        }
        if (n_qubits < 1 || n_qubits > 34) {
            return invalid("There must be at least 1 qubit in the Statevector (and at most 34 here).");
        }
        auto* h = new kt_sv_s {};
        if (const int32_t rc = alloc_state(h->st, n_qubits, dtype); rc != KT_OK) {
            delete h;
            return rc;
        }
        if (const int32_t rc = kt::launch_set_basis(h->st, 0); rc != KT_OK) {
            free_state(h->st);
            delete h;
            return rc;
        }
        *out = h;
        return KT_OK;
    });
}

int32_t kt_sv_wrap(void* device_amps, int32_t n_qubits, int32_t dtype, kt_sv* out)
{
    return guard([&]() -> int32_t {
        if (out == nullptr || device_amps == nullptr) {
            return invalid("null pointer");
        }
        if (const int32_t rc = check_dtype(dtype); rc != KT_OK) {
            return rc;
        }
        if (n_qubits < 1 || n_qubits > 34) {
            return invalid("qubit count out of range");
        }
        auto* h = new kt_sv_s {};
        h->st.n_bits = n_qubits;
        h->st.dtype = dtype;
        h->st.amps = device_amps;
        h->st.owned = false;
        *out = h;
        return KT_OK;
    });
}

int32_t kt_sv_destroy(kt_sv sv)
{
    if (sv != nullptr) {
        free_state(sv->st);
        delete sv;
    }
    return KT_OK;
}

int32_t kt_sv_set_stream(kt_sv sv, void* stream)
{
    if (sv == nullptr) {
        return invalid("null handle");
    }
    sv->st.stream = static_cast<cudaStream_t>(stream);
    return KT_OK;
}

int32_t kt_sv_info(kt_sv sv, int32_t* n_qubits, int32_t* dtype, void** device_amps)
{
    if (sv == nullptr) {
        return invalid("null handle");
    }
    if (n_qubits) *n_qubits = sv->st.n_bits;
    if (dtype) *dtype = sv->st.dtype;
    if (device_amps) *device_amps = sv->st.amps;
    return KT_OK;
}

int32_t kt_sv_set_basis(kt_sv sv, uint64_t index)
{
    return guard([&]() -> int32_t {
        if (sv == nullptr) {
            return invalid("null handle");
        }
        if (index >= sv->st.n_amps()) {
            return invalid("Out-of-bounds access for the quantum state.");
        }
        return kt::launch_set_basis(sv->st, index);
    });
}

int32_t kt_sv_upload(kt_sv sv, const double* host_amps, uint64_t n_amps)
{
    return guard([&]() -> int32_t { return sv ? upload(sv->st, host_amps, n_amps) : invalid("null handle"); });
}

int32_t kt_sv_download(kt_sv sv, double* host_amps, uint64_t n_amps)
{
    return guard([&]() -> int32_t { return sv ? download(sv->st, host_amps, n_amps) : invalid("null handle"); });
}

int32_t kt_sv_copy(kt_sv dst, kt_sv src)
{
    return guard([&]() -> int32_t {
        if (dst == nullptr || src == nullptr) {
            return invalid("null handle");
        }
        if (dst->st.n_bits != src->st.n_bits || dst->st.dtype != src->st.dtype) {
            return invalid("states differ in size or type");
        }
        KT_CUDA(cudaMemcpyAsync(dst->st.amps, src->st.amps, src->st.n_amps() * src->st.amp_bytes(),
                                cudaMemcpyDeviceToDevice, dst->st.stream));
        return KT_OK;
    });
}

int32_t kt_sv_apply(kt_sv sv, const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params,
                    int32_t mode)
{
    return guard([&]() -> int32_t {
        if (sv == nullptr) {
            return invalid("null handle");
        }
        if (n_gates < 0 || (n_gates > 0 && gates == nullptr)) {
            return invalid("bad gate array");
        }
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, sv->st.n_bits, lg); rc != KT_OK) {
            return rc;
        }
        return apply_lowered(sv->st, lg, mode);
    });
}

int32_t kt_plan_stats(int32_t n_qubits, int32_t dtype, const kt_gate* gates, int64_t n_gates, const double* params,
                      int64_t n_params, int64_t* blocks, int64_t* phases, int64_t* ops, int64_t* transposes)
{
    return guard([&]() -> int32_t {
        if (blocks == nullptr || phases == nullptr || ops == nullptr || transposes == nullptr) {
            return invalid("null output pointer");
        }
        if (const int32_t rc = check_dtype(dtype); rc != KT_OK) {
            return rc;
        }
        if (n_qubits < 1 || n_qubits > 40 || n_gates < 0 || (n_gates > 0 && gates == nullptr)) {
            return invalid("bad qubit count or gate array");
        }
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, n_qubits, lg); rc != KT_OK) {
            return rc;
        }
        return kt::plan_stats(n_qubits, dtype, lg, blocks, phases, ops, transposes);
    });
}

int32_t kt_plan_blocks(int32_t n_qubits, const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params,
                       double* out, int64_t capacity, int64_t* n_blocks)
{
    return guard([&]() -> int32_t {
        if (n_blocks == nullptr || capacity < 0 || (capacity > 0 && out == nullptr)) {
            return invalid("bad output array");
        }
        if (n_qubits < 1 || n_qubits > 40 || n_gates < 0 || (n_gates > 0 && gates == nullptr)) {
            return invalid("bad qubit count or gate array");
        }
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, n_qubits, lg); rc != KT_OK) {
            return rc;
        }
        std::vector<double> v;
        if (const int32_t rc = kt::plan_blocks(n_qubits, lg, v); rc != KT_OK) {
            return rc;
        }
        *n_blocks = static_cast<int64_t>(v.size() / 4);
        std::copy(v.begin(), v.begin() + static_cast<std::ptrdiff_t>(std::min<size_t>(v.size(), 4 * static_cast<size_t>(capacity))), out);
        return KT_OK;
    });
}

int32_t kt_plan_order(int32_t n_qubits, int32_t dtype, const kt_gate* gates, int64_t n_gates, const double* params,
                      int64_t n_params, int64_t* order, int64_t capacity, int64_t* count)
{
    return guard([&]() -> int32_t {
        if (count == nullptr || capacity < 0 || (capacity > 0 && order == nullptr)) {
            return invalid("bad output array");
        }
        if (const int32_t rc = check_dtype(dtype); rc != KT_OK) {
            return rc;
        }
        if (n_qubits < 1 || n_qubits > 40 || n_gates < 0 || (n_gates > 0 && gates == nullptr)) {
            return invalid("bad qubit count or gate array");
        }
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, n_qubits, lg); rc != KT_OK) {
            return rc;
        }
        int64_t blocks = 0, phases = 0, ops = 0, transposes = 0;
        std::vector<int32_t> run;
        if (const int32_t rc = kt::plan_stats(n_qubits, dtype, lg, &blocks, &phases, &ops, &transposes, &run);
            rc != KT_OK) {
            return rc;
        }
        *count = static_cast<int64_t>(run.size());
        if (*count > capacity) {
            return invalid("order array too small");
        }
        for (size_t i = 0; i < run.size(); ++i) {
            order[i] = run[i];
        }
        return KT_OK;
    });
}

int32_t kt_sv_apply_stats(kt_sv sv, int64_t* launches, double* alg_bytes)
{
    if (sv == nullptr) {
        return invalid("null handle");
    }
    if (launches) *launches = sv->st.last_launches;
    if (alg_bytes) *alg_bytes = sv->st.last_alg_bytes;
    return KT_OK;
}

int32_t kt_dm_apply_stats(kt_dm dm, int64_t* launches, double* alg_bytes)
{
    if (dm == nullptr) {
        return invalid("null handle");
    }
    if (launches) *launches = dm->st.last_launches;
    if (alg_bytes) *alg_bytes = dm->st.last_alg_bytes;
    return KT_OK;
}

int32_t kt_sv_expect(kt_sv sv, const kt_pauli* strings, int64_t n_strings, const double* coeffs, double* out_terms,
                     double* out_total)
{
    return guard([&]() -> int32_t {
        if (sv == nullptr) {
            return invalid("null handle");
        }
        if (n_strings < 0 || (n_strings > 0 && strings == nullptr)) {
            return invalid("bad Pauli string array");
        }
        return kt::expect_paulis(sv->st, strings, n_strings, coeffs, out_terms, out_total);
    });
}

int32_t kt_sv_probabilities(kt_sv sv, const double* noise, double* host_out)
{
    return guard([&]() -> int32_t {
        if (sv == nullptr || host_out == nullptr) {
            return invalid("null pointer");
        }
        return kt::probabilities(sv->st, noise, host_out);
    });
}

int32_t kt_sv_sample(kt_sv sv, const double* noise, const double* canonicals, int64_t n_shots, uint64_t* out_indices,
                     int32_t mode, int32_t* n_rescanned)
{
    return guard([&]() -> int32_t {
        if (sv == nullptr) {
            return invalid("null handle");
        }
        if (n_shots < 0 || (n_shots > 0 && (canonicals == nullptr || out_indices == nullptr))) {
            return invalid("bad shot buffers");
        }
        return kt::sample(sv->st, noise, canonicals, n_shots, out_indices, mode, n_rescanned);
    });
}

int32_t kt_sv_measure_probs(kt_sv sv, uint32_t qubit, double* p0, double* p1)
{
    return guard([&]() -> int32_t {
        if (sv == nullptr || p0 == nullptr || p1 == nullptr) {
            return invalid("null pointer");
        }
        if (qubit >= static_cast<uint32_t>(sv->st.n_bits)) {
            return invalid("measured qubit out of range");
        }
        return kt::measure_probs(sv->st, qubit, p0, p1);
    });
}

int32_t kt_sv_collapse(kt_sv sv, uint32_t qubit, int32_t outcome, double scale)
{
    return guard([&]() -> int32_t {
        if (sv == nullptr) {
            return invalid("null handle");
        }
        if (qubit >= static_cast<uint32_t>(sv->st.n_bits) || (outcome != 0 && outcome != 1)) {
            return invalid("bad qubit or outcome");
        }
        return kt::collapse(sv->st, qubit, outcome, scale);
    });
}

int32_t kt_sv_norm_sq(kt_sv sv, double* out)
{
    return guard([&]() -> int32_t { return (sv && out) ? kt::norm_sq(sv->st, out) : invalid("null pointer"); });
}

int32_t kt_sv_inner(kt_sv bra, kt_sv ket, double* out_re_im)
{
    return guard([&]() -> int32_t {
        if (bra == nullptr || ket == nullptr || out_re_im == nullptr) {
            return invalid("null pointer");
        }
        if (bra->st.n_bits != ket->st.n_bits || bra->st.dtype != ket->st.dtype) {
            return invalid("ERROR: cannot calculate inner product between two states of different sizes.");
        }
        return kt::inner_product(bra->st, ket->st, out_re_im);
    });
}

// ---- pairs ----------------------------------------------------------------------

static int32_t run_pairs(uint32_t n, uint32_t c, uint32_t t, int kind, uint64_t k0, uint64_t count, uint64_t* host_out)
{
    const int per = (kind == 2) ? 4 : 2;
    if (count == 0) {
        return KT_OK;
    }
    void* d = nullptr;
    KT_CUDA(cudaMalloc(&d, count * per * sizeof(uint64_t)));
    int32_t rc = kt::launch_pairs(n, c, t, kind, k0, count, static_cast<uint64_t*>(d), nullptr);
    if (rc == KT_OK) {
        rc = kt::copy_d2h(host_out, d, count * per * sizeof(uint64_t), nullptr);
    }
    cudaFree(d);
    return rc;
}

int32_t kt_pairs_single(uint32_t n_qubits, uint32_t target, uint64_t k0, uint64_t count, uint64_t* host_out)
{
    return guard([&]() -> int32_t {
        if (n_qubits < 1 || n_qubits > 40 || target >= n_qubits) {
            return invalid("bad qubit count or target");
        }
        const uint64_t size = uint64_t {1} << (n_qubits - 1);
        if (k0 > size || count > size - k0 || (count > 0 && host_out == nullptr)) {
            return invalid("pair range out of bounds");
        }
        return run_pairs(n_qubits, 0, target, 0, k0, count, host_out);
    });
}

int32_t kt_pairs_double(uint32_t n_qubits, uint32_t control, uint32_t target, int32_t quad, uint64_t k0, uint64_t count,
                        uint64_t* host_out)
{
    return guard([&]() -> int32_t {
        if (n_qubits < 2 || n_qubits > 40 || target >= n_qubits || control >= n_qubits || control == target) {
            return invalid("bad qubit count, control or target");
        }
        const uint64_t size = uint64_t {1} << (n_qubits - 2);
        if (k0 > size || count > size - k0 || (count > 0 && host_out == nullptr)) {
            return invalid("pair range out of bounds");
        }
        return run_pairs(n_qubits, control, target, quad ? 2 : 1, k0, count, host_out);
    });
}

// ---- density matrix ---------------------------------------------------------------

int32_t kt_dm_create(int32_t n_qubits, int32_t dtype, kt_dm* out)
{
    return guard([&]() -> int32_t {
        if (out == nullptr) {
            return invalid("null output handle");
        }
        *out = nullptr;
        if (const int32_t rc = check_dtype(dtype); rc != KT_OK) {
            return rc;
        }
        if (n_qubits < 0 || n_qubits > 17) {
            return invalid("density matrix qubit count out of range (0..17)");
        }
        auto* h = new kt_dm_s {};
        h->n = n_qubits;
        if (const int32_t rc = alloc_state(h->st, 2 * n_qubits, dtype); rc != KT_OK) {
            delete h;
            return rc;
        }
        if (const int32_t rc = kt::launch_set_basis(h->st, 0); rc != KT_OK) {
            free_state(h->st);
            delete h;
            return rc;
        }
        *out = h;
        return KT_OK;
    });
}

int32_t kt_dm_destroy(kt_dm dm)
{
    if (dm != nullptr) {
        free_state(dm->st);
        delete dm;
    }
    return KT_OK;
}

int32_t kt_dm_set_stream(kt_dm dm, void* stream)
{
    if (dm == nullptr) {
        return invalid("null handle");
    }
    dm->st.stream = static_cast<cudaStream_t>(stream);
    return KT_OK;
}

int32_t kt_dm_set_basis(kt_dm dm, uint64_t index)
{
    return guard([&]() -> int32_t {
        if (dm == nullptr) {
            return invalid("null handle");
        }
        const uint64_t N = uint64_t {1} << dm->n;
        if (index >= N) {
            return invalid("basis index out of range");
        }
        return kt::launch_set_basis(dm->st, index + index * N);
    });
}

int32_t kt_dm_upload(kt_dm dm, const double* host_colmajor, uint64_t n_elems)
{
    return guard([&]() -> int32_t { return dm ? upload(dm->st, host_colmajor, n_elems) : invalid("null handle"); });
}

int32_t kt_dm_download(kt_dm dm, double* host_colmajor, uint64_t n_elems)
{
    return guard([&]() -> int32_t { return dm ? download(dm->st, host_colmajor, n_elems) : invalid("null handle"); });
}

int32_t kt_dm_apply(kt_dm dm, const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params,
                    int32_t mode)
{
    return guard([&]() -> int32_t {
        if (dm == nullptr) {
            return invalid("null handle");
        }
        if (n_gates < 0 || (n_gates > 0 && gates == nullptr)) {
            return invalid("bad gate array");
        }
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, dm->n, lg); rc != KT_OK) {
            return rc;
        }
        // U rho U^dagger = U on the row bits, conj(U) on the column bits
        std::vector<kt::LGate> both;
        both.reserve(2 * lg.size());
        for (const auto& g : lg) {
            both.push_back(g);
            both.push_back(kt::conj_shifted(g, dm->n));
        }
        return apply_lowered(dm->st, both, mode);
    });
}

int32_t kt_dm_prepare(kt_dm dm, const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params)
{
    return guard([&]() -> int32_t {
        if (dm == nullptr) {
            return invalid("null handle");
        }
        if (n_gates < 0 || (n_gates > 0 && gates == nullptr)) {
            return invalid("bad gate array");
        }
        std::vector<kt::LGate> lg;
        if (const int32_t rc = kt::lower_gates(gates, n_gates, params, n_params, dm->n, lg); rc != KT_OK) {
            return rc;
        }
        // the same 2n-bit gate stream kt_dm_apply plans
        std::vector<kt::LGate> both;
        both.reserve(2 * lg.size());
        for (const auto& g : lg) {
            both.push_back(g);
            both.push_back(kt::conj_shifted(g, dm->n));
        }
        return kt::jit_prepare(dm->st, both);
    });
}

int32_t kt_dm_expect(kt_dm dm, const kt_pauli* strings, int64_t n_strings, const double* coeffs, double* out_terms,
                     double* out_total)
{
    return guard([&]() -> int32_t {
        if (dm == nullptr) {
            return invalid("null handle");
        }
        if (n_strings < 0 || (n_strings > 0 && strings == nullptr)) {
            return invalid("bad Pauli string array");
        }
        if (dm->n == 0) {
            return invalid("a density matrix of 0 qubits has no Pauli expectation value");
        }
        return kt::dm_expect_paulis(dm->st, dm->n, strings, n_strings, coeffs, out_terms, out_total);
    });
}

int32_t kt_dm_trace(kt_dm dm, double* out_re_im)
{
    return guard([&]() -> int32_t { return (dm && out_re_im) ? kt::dm_trace(dm->st, dm->n, out_re_im) : invalid("null pointer"); });
}

int32_t kt_dm_probabilities(kt_dm dm, double* host_out)
{
    return guard([&]() -> int32_t { return (dm && host_out) ? kt::dm_diagonal(dm->st, dm->n, host_out) : invalid("null pointer"); });
}

int32_t kt_dm_partial_trace(kt_dm src, const int32_t* qubits, int32_t n_traced, kt_dm dst)
{
    return guard([&]() -> int32_t {
        if (src == nullptr || dst == nullptr || src == dst) {
            return invalid("partial trace needs two distinct density matrices");
        }
        if (n_traced < 0 || n_traced > src->n || (n_traced > 0 && qubits == nullptr)) {
            return invalid("bad traced-qubit array");
        }
        uint32_t seen = 0;
        for (int32_t j = 0; j < n_traced; ++j) {
            if (qubits[j] < 0 || qubits[j] >= src->n) {
                return invalid("ERROR: Cannot take partial trace; found qubit index out of bounds\n");
            }
            if (((seen >> qubits[j]) & 1U) != 0U) {
                return invalid("traced qubits must be distinct");
            }
            seen |= 1U << qubits[j];
        }
        if (dst->n != src->n - n_traced || dst->st.dtype != src->st.dtype) {
            return invalid("the output density matrix needs n - n_traced qubits and the input's dtype");
        }
        if (n_traced == 0) {
            KT_CUDA(cudaMemcpyAsync(dst->st.amps, src->st.amps, src->st.n_amps() * src->st.amp_bytes(),
                                    cudaMemcpyDeviceToDevice, dst->st.stream));
            return KT_OK;
        }
        return kt::dm_partial_trace(src->st, src->n, qubits, n_traced, dst->st);
    });
}

int32_t kt_dm_tensor_product(kt_dm left, kt_dm right, kt_dm dst)
{
    return guard([&]() -> int32_t {
        if (left == nullptr || right == nullptr || dst == nullptr || dst == left || dst == right) {
            return invalid("tensor product needs two inputs and a distinct output");
        }
        if (dst->n != left->n + right->n || left->st.dtype != dst->st.dtype || right->st.dtype != dst->st.dtype) {
            return invalid("the output density matrix needs n_left + n_right qubits and the inputs' dtype");
        }
        return kt::dm_tensor_product(left->st, left->n, right->st, right->n, dst->st);
    });
}

int32_t kt_dm_trace_of_square(kt_dm dm, double* out_re_im)
{
    return guard([&]() -> int32_t {
        return (dm && out_re_im) ? kt::dm_trace_of_square(dm->st, dm->n, out_re_im) : invalid("null pointer");
    });
}

}  // extern "C"
