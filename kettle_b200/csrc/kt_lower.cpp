// kt_lower.cpp — host side: error state, scratch buffers and gate lowering.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "kt_internal.cuh"

namespace kt
{

namespace
{
thread_local std::string g_last_error;
}

void set_error(int32_t code, const std::string& msg)
{
    std::ostringstream os;
    os << "kettle_b200 error " << code << ": " << msg;
    g_last_error = os.str();
}

const char* last_error_cstr()
{
    return g_last_error.c_str();
}

void set_error_text(const std::string& text)
{
    g_last_error = text;
}

int32_t cuda_fail(cudaError_t e, const char* where)
{
    std::ostringstream os;
    os << where << ": " << cudaGetErrorName(e) << " (" << cudaGetErrorString(e) << ")";
    const int32_t code = (e == cudaErrorMemoryAllocation) ? KT_ERR_NOMEM : KT_ERR_CUDA;
    set_error(code, os.str());
    return code;
}

int32_t DevBuf::reserve(size_t need)
{
    if (need <= bytes) {
        return KT_OK;
    }
    release();
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
        return cuda_fail(e, "cudaMalloc(scratch)");
    }
    ptr = p;
    bytes = need;
    return KT_OK;
}

void DevBuf::release()
{
    if (ptr != nullptr) {
        cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
}

int sm_count()
{
    static int cached = -1;
    if (cached < 0) {
        int dev = 0;
        int v = SM_COUNT_B200;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess) {
            cached = v;
        } else {
            cached = SM_COUNT_B200;
        }
    }
    return cached;
}

namespace
{

bool set_knob(Tuning& t, const std::string& name, long long v)
{
    if (name == "fused_ctas_per_sm") {
        t.fused_ctas_per_sm = (v == 1) ? 1 : 2;
    } else if (name == "fused_tile_bits") {
        t.fused_tile_bits = static_cast<int>(std::max(9LL, std::min(13LL, v)));
    } else if (name == "adjoint_fused") {
        t.adjoint_fused = (v != 0) ? 1 : 0;
    } else if (name == "fused_max_ops") {
        t.fused_max_ops = static_cast<int>(std::max(1LL, std::min(256LL, v)));
    } else if (name == "fold_permutations") {
        t.fold_permutations = (v != 0) ? 1 : 0;
    } else if (name == "c64_renormalize") {
        t.c64_renormalize = (v != 0) ? 1 : 0;
    } else if (name == "fused_reg_bits") {
        t.fused_reg_bits = (v == 3) ? 3 : 4;
    } else if (name == "jit_remat") {
        t.jit_remat = (v != 0) ? 1 : 0;
    } else if (name == "adjoint_jit") {
        t.adjoint_jit = static_cast<int>(std::max(0LL, std::min(2LL, v)));
    } else if (name == "jit_lean_sync") {
        t.jit_lean_sync = (v != 0) ? 1 : 0;
    } else if (name == "jit_tma") {
        t.jit_tma = (v != 0) ? 1 : 0;
    } else if (name == "jit_tma_ctas") {
        t.jit_tma_ctas = (v >= 2) ? 2 : 1;
    } else if (name == "jit_tma_stages") {
        t.jit_tma_stages = static_cast<int>(std::max(2LL, std::min(4LL, v)));
    } else if (name == "batch_spin_limit") {
        t.batch_spin_limit = std::max(1LL, std::min(1000000000000LL, v));
    } else if (name == "batch_small_max_qubits") {
        t.batch_small_max_qubits = static_cast<int>(std::max(0LL, std::min(13LL, v)));
    } else if (name == "batch_jit_min_qubits") {
        t.batch_jit_min_qubits = static_cast<int>(std::max(0LL, std::min(64LL, v)));
    } else if (name == "jit_scale_ops") {
        t.jit_scale_ops = (v != 0) ? 1 : 0;
    } else if (name == "plan_schedule") {
        t.plan_schedule = static_cast<int>(std::max(0LL, std::min(3LL, v)));
    } else if (name == "plan_deep_qubits") {
        t.plan_deep_qubits = static_cast<int>(std::max(1LL, std::min(64LL, v)));
    } else if (name == "plan_lookahead") {
        t.plan_lookahead = static_cast<int>(std::max(0LL, std::min(2LL, v)));
    } else if (name == "fused_jit") {
        t.fused_jit = static_cast<int>(std::max(0LL, std::min(2LL, v)));
    } else if (name == "jit_ctas_per_sm") {
        t.jit_ctas_per_sm = static_cast<int>(std::max(2LL, std::min(4LL, v)));
    } else if (name == "jit_async_load") {
        t.jit_async_load = (v != 0) ? 1 : 0;
    } else if (name == "jit_fence") {
        t.jit_fence = static_cast<int>(std::max(0LL, std::min(64LL, v)));
    } else if (name == "jit_skip_io") {
        t.jit_skip_io = static_cast<int>(std::max(0LL, std::min(2LL, v)));
    } else if (name == "jit_merge_diag") {
        t.jit_merge_diag = (v != 0) ? 1 : 0;
    } else if (name == "jit_prefetch") {
        t.jit_prefetch = (v != 0) ? 1 : 0;
    } else if (name == "jit_after") {
        t.jit_after = static_cast<int>(std::max(0LL, std::min(1000000LL, v)));
    } else if (name == "jit_min_qubits") {
        t.jit_min_qubits = static_cast<int>(std::max(1LL, std::min(64LL, v)));
    } else {
        return false;
    }
    return true;
}

}  // namespace

Tuning& tuning()
{
    static Tuning t = [] {
        Tuning d;
        if (const char* env = std::getenv("KT_TUNING")) {
            std::string s {env};
            size_t pos = 0;
            while (pos < s.size()) {
                const size_t end = s.find(',', pos);
                const std::string kv = s.substr(pos, end == std::string::npos ? std::string::npos : end - pos);
                const size_t eq = kv.find('=');
                if (eq != std::string::npos) {
                    set_knob(d, kv.substr(0, eq), std::atoll(kv.c_str() + eq + 1));
                }
                if (end == std::string::npos) {
                    break;
                }
                pos = end + 1;
            }
        }
        return d;
    }();
    return t;
}

bool tuning_set(const char* name, long long value)
{
    return name != nullptr && set_knob(tuning(), name, value);
}

bool tuning_get(const char* name, long long* value)
{
    if (name == nullptr || value == nullptr) {
        return false;
    }
    const std::string n {name};
    const Tuning& t = tuning();
    if (n == "fused_ctas_per_sm") {
        *value = t.fused_ctas_per_sm;
    } else if (n == "fused_tile_bits") {
        *value = t.fused_tile_bits;
    } else if (n == "adjoint_fused") {
        *value = t.adjoint_fused;
    } else if (n == "fused_max_ops") {
        *value = t.fused_max_ops;
    } else if (n == "fold_permutations") {
        *value = t.fold_permutations;
    } else if (n == "c64_renormalize") {
        *value = t.c64_renormalize;
    } else if (n == "fused_reg_bits") {
        *value = t.fused_reg_bits;
    } else if (n == "jit_remat") {
        *value = t.jit_remat;
    } else if (n == "adjoint_jit") {
        *value = t.adjoint_jit;
    } else if (n == "jit_lean_sync") {
        *value = t.jit_lean_sync;
    } else if (n == "jit_tma") {
        *value = t.jit_tma;
    } else if (n == "jit_tma_ctas") {
        *value = t.jit_tma_ctas;
    } else if (n == "jit_tma_stages") {
        *value = t.jit_tma_stages;
    } else if (n == "batch_spin_limit") {
        *value = t.batch_spin_limit;
    } else if (n == "batch_small_max_qubits") {
        *value = t.batch_small_max_qubits;
    } else if (n == "batch_jit_min_qubits") {
        *value = t.batch_jit_min_qubits;
    } else if (n == "jit_scale_ops") {
        *value = t.jit_scale_ops;
    } else if (n == "plan_schedule") {
        *value = t.plan_schedule;
    } else if (n == "plan_deep_qubits") {
        *value = t.plan_deep_qubits;
    } else if (n == "plan_lookahead") {
        *value = t.plan_lookahead;
    } else if (n == "fused_jit") {
        *value = t.fused_jit;
    } else if (n == "jit_ctas_per_sm") {
        *value = t.jit_ctas_per_sm;
    } else if (n == "jit_async_load") {
        *value = t.jit_async_load;
    } else if (n == "jit_fence") {
        *value = t.jit_fence;
    } else if (n == "jit_skip_io") {
        *value = t.jit_skip_io;
    } else if (n == "jit_merge_diag") {
        *value = t.jit_merge_diag;
    } else if (n == "jit_prefetch") {
        *value = t.jit_prefetch;
    } else if (n == "jit_after") {
        *value = t.jit_after;
    } else if (n == "jit_min_qubits") {
        *value = t.jit_min_qubits;
    } else {
        return false;
    }
    return true;
}

int32_t copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0) {
        return KT_OK;
    }
    KT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return KT_OK;
}

int32_t copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0) {
        return KT_OK;
    }
    KT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    KT_CUDA(cudaStreamSynchronize(st));
    return KT_OK;
}

// ---------------------------------------------------------------------------
// gate lowering
//
// Matrices follow gates/common_u_gates.cpp of the reference: RX/RY/RZ use
// cos(theta/2), sin(theta/2); P uses cos(theta), sin(theta); U/CU carry the
// caller's matrix.  Controlled variants (CH ... CP, CU) apply the same 2x2 to
// the control = 1 half, as DoubleQubitGatePairGenerator::next() selects
// (simulation/gate_pair_generator.hpp:113-131).

namespace
{

constexpr double SQ12 = 0.70710678118654752440;  // M_SQRT1_2

bool is_controlled(int op)
{
    return (op >= KT_OP_CH && op <= KT_OP_CP) || op == KT_OP_CU;
}

bool has_angle(int op)
{
    return (op >= KT_OP_RX && op <= KT_OP_P) || (op >= KT_OP_CRX && op <= KT_OP_CP);
}

void set_m(LGate& g, double a, double b, double c, double d, double e, double f, double h, double i)
{
    g.m[0] = a; g.m[1] = b; g.m[2] = c; g.m[3] = d;
    g.m[4] = e; g.m[5] = f; g.m[6] = h; g.m[7] = i;
}

}  // namespace

int32_t lower_gate(const kt_gate& g, const double* params, int64_t n_params, int n_qubits, LGate* out)
{
    const int op = g.op;
    if (op == KT_OP_M) {
        set_error(KT_ERR_INVALID, "M gates are applied through kt_sv_measure_probs / kt_sv_collapse");
        return KT_ERR_INVALID;
    }
    if (op > KT_OP_CU) {
        set_error(KT_ERR_INVALID, "unknown gate op " + std::to_string(op));
        return KT_ERR_INVALID;
    }
    if (g.target >= static_cast<uint32_t>(n_qubits)) {
        set_error(KT_ERR_INVALID, "target qubit " + std::to_string(g.target) + " out of range for " +
                                      std::to_string(n_qubits) + " qubits");
        return KT_ERR_INVALID;
    }
    LGate l {};
    l.target = static_cast<int32_t>(g.target);
    l.control = -1;
    if (is_controlled(op)) {
        if (g.control >= static_cast<uint32_t>(n_qubits) || g.control == g.target) {
            set_error(KT_ERR_INVALID, "control qubit " + std::to_string(g.control) + " invalid for target " +
                                          std::to_string(g.target));
            return KT_ERR_INVALID;
        }
        l.control = static_cast<int32_t>(g.control);
    }
    double th = g.angle;
    if (has_angle(op) && g.param >= 0) {
        if (params == nullptr || g.param >= n_params) {
            set_error(KT_ERR_INVALID, "parameter slot " + std::to_string(g.param) + " out of range");
            return KT_ERR_INVALID;
        }
        th = params[g.param];
    }
    switch (op) {
        case KT_OP_H: case KT_OP_CH: l.kind = KIND_GEN; set_m(l, SQ12, 0, SQ12, 0, SQ12, 0, -SQ12, 0); break;
        case KT_OP_X: case KT_OP_CX: l.kind = KIND_ANTI; set_m(l, 0, 0, 1, 0, 1, 0, 0, 0); break;
        case KT_OP_Y: case KT_OP_CY: l.kind = KIND_ANTI; set_m(l, 0, 0, 0, -1, 0, 1, 0, 0); break;
        case KT_OP_Z: case KT_OP_CZ: l.kind = KIND_DIAG; set_m(l, 1, 0, 0, 0, 0, 0, -1, 0); break;
        case KT_OP_S: case KT_OP_CS: l.kind = KIND_DIAG; set_m(l, 1, 0, 0, 0, 0, 0, 0, 1); break;
        case KT_OP_SDAG: case KT_OP_CSDAG: l.kind = KIND_DIAG; set_m(l, 1, 0, 0, 0, 0, 0, 0, -1); break;
        case KT_OP_T: case KT_OP_CT: l.kind = KIND_DIAG; set_m(l, 1, 0, 0, 0, 0, 0, SQ12, SQ12); break;
        case KT_OP_TDAG: case KT_OP_CTDAG: l.kind = KIND_DIAG; set_m(l, 1, 0, 0, 0, 0, 0, SQ12, -SQ12); break;
        case KT_OP_SX: case KT_OP_CSX: l.kind = KIND_GEN; set_m(l, 0.5, 0.5, 0.5, -0.5, 0.5, -0.5, 0.5, 0.5); break;
        case KT_OP_SXDAG: case KT_OP_CSXDAG: l.kind = KIND_GEN; set_m(l, 0.5, -0.5, 0.5, 0.5, 0.5, 0.5, 0.5, -0.5); break;
        case KT_OP_RX: case KT_OP_CRX: {
            const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
            l.kind = KIND_GEN; set_m(l, c, 0, 0, -s, 0, -s, c, 0);
            break;
        }
        case KT_OP_RY: case KT_OP_CRY: {
            const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
            l.kind = KIND_GEN; set_m(l, c, 0, -s, 0, s, 0, c, 0);
            break;
        }
        case KT_OP_RZ: case KT_OP_CRZ: {
            const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
            l.kind = KIND_DIAG; set_m(l, c, -s, 0, 0, 0, 0, c, s);
            break;
        }
        case KT_OP_P: case KT_OP_CP: {
            l.kind = KIND_DIAG; set_m(l, 1, 0, 0, 0, 0, 0, std::cos(th), std::sin(th));
            break;
        }
        case KT_OP_U: case KT_OP_CU: {
            std::memcpy(l.m, g.u, sizeof(l.m));
            const bool off_zero = l.m[2] == 0.0 && l.m[3] == 0.0 && l.m[4] == 0.0 && l.m[5] == 0.0;
            const bool diag_zero = l.m[0] == 0.0 && l.m[1] == 0.0 && l.m[6] == 0.0 && l.m[7] == 0.0;
            l.kind = off_zero ? KIND_DIAG : (diag_zero ? KIND_ANTI : KIND_GEN);
            break;
        }
        default:
            set_error(KT_ERR_INVALID, "unsupported gate op " + std::to_string(op));
            return KT_ERR_INVALID;
    }
    l.flags = (l.kind == KIND_DIAG && l.m[0] == 1.0 && l.m[1] == 0.0) ? 1 : 0;
    *out = l;
    return KT_OK;
}

int32_t lower_gates(const kt_gate* gates, int64_t n_gates, const double* params, int64_t n_params, int n_qubits,
                    std::vector<LGate>& out)
{
    out.clear();
    out.reserve(static_cast<size_t>(n_gates));
    for (int64_t i = 0; i < n_gates; ++i) {
        LGate l {};
        const int32_t rc = lower_gate(gates[i], params, n_params, n_qubits, &l);
        if (rc != KT_OK) {
            return rc;
        }
        out.push_back(l);
    }
    return KT_OK;
}

bool gate_derivative(int op, double th, double* d)
{
    std::fill(d, d + 8, 0.0);
    const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
    switch (op) {
        case KT_OP_RX: case KT_OP_CRX:
            // [[c, -i s], [-i s, c]]' = [[-s/2, -i c/2], [-i c/2, -s/2]]
            d[0] = -0.5 * s; d[3] = -0.5 * c; d[5] = -0.5 * c; d[6] = -0.5 * s;
            return true;
        case KT_OP_RY: case KT_OP_CRY:
            // [[c, -s], [s, c]]' = [[-s/2, -c/2], [c/2, -s/2]]
            d[0] = -0.5 * s; d[2] = -0.5 * c; d[4] = 0.5 * c; d[6] = -0.5 * s;
            return true;
        case KT_OP_RZ: case KT_OP_CRZ:
            // diag(c - i s, c + i s)' = diag(-s/2 - i c/2, -s/2 + i c/2)
            d[0] = -0.5 * s; d[1] = -0.5 * c; d[6] = -0.5 * s; d[7] = 0.5 * c;
            return true;
        case KT_OP_P: case KT_OP_CP:
            // diag(1, cos + i sin)' = diag(0, -sin + i cos)
            d[6] = -std::sin(th); d[7] = std::cos(th);
            return true;
        default:
            return false;
    }
}

int gate_generator(int op)
{
    switch (op) {
        case KT_OP_RX: case KT_OP_CRX: return GEN_X;
        case KT_OP_RY: case KT_OP_CRY: return GEN_Y;
        case KT_OP_RZ: case KT_OP_CRZ: return GEN_Z;
        case KT_OP_P: case KT_OP_CP: return GEN_P;
        default: return -1;
    }
}

LGate conj_shifted(const LGate& g, int shift)
{
    LGate c = g;
    c.target = g.target + shift;
    c.control = (g.control >= 0) ? g.control + shift : -1;
    for (int k = 1; k < 8; k += 2) {
        c.m[k] = -g.m[k];
    }
    c.flags = (c.kind == KIND_DIAG && c.m[0] == 1.0 && c.m[1] == 0.0) ? 1 : 0;
    return c;
}

}  // namespace kt
