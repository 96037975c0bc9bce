// ref_capi.cpp — test infrastructure, NOT product code.
//
// A flat C interface over the reference kettle library, compiled from the
// reference's own sources into oracle/_ref/libkettle_ref.so (see oracle/Makefile).
// The tests use it to pin the C restatement in oracle/kt_oracle.c and to produce
// golden vectors; bench.py's reference arm times it.  Every function drives the
// reference through its public API (ket::QuantumCircuit adders, ket::simulate,
// ket::expectation_value, ket::perform_measurements_as_memory, ...), or, for the
// pair enumerations, through its header-only generators
// (source/kettle_internal/simulation/gate_pair_generator.hpp).
#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <optional>
#include <string>
#include <unordered_map>
#include <vector>

#include "kettle/kettle.hpp"
#include "kettle_internal/simulation/gate_pair_generator.hpp"

#include "kettle_b200.h"

namespace
{

thread_local std::string g_err;

auto seed_opt(int64_t seed) -> std::optional<int>
{
    if (seed < 0) {
        return std::nullopt;
    }
    return static_cast<int>(seed);
}

auto to_matrix(const double* u) -> ket::Matrix2X2
{
    return ket::Matrix2X2 {
        .elem00 = {u[0], u[1]},
        .elem01 = {u[2], u[3]},
        .elem10 = {u[4], u[5]},
        .elem11 = {u[6], u[7]},
    };
}

// Translate one kt_gate record into the reference's adder call.  Parameter
// slots map onto reference ParameterIDs: the first gate that names a slot
// creates the parameter with `parameterized{}`, later ones reuse the id, so
// shared parameters exercise the reference's own bookkeeping.
struct CircuitBuilder
{
    ket::QuantumCircuit circuit;
    const double* params;
    std::unordered_map<int32_t, ket::param::ParameterID> ids;

    CircuitBuilder(std::size_t n, const double* p)
        : circuit {n}
        , params {p}
    {}

    void add(const kt_gate& g)
    {
        using namespace ket;
        const auto t = static_cast<std::size_t>(g.target);
        const auto c = static_cast<std::size_t>(g.control);
        switch (g.op) {
            case KT_OP_H: circuit.add_h_gate(t); return;
            case KT_OP_X: circuit.add_x_gate(t); return;
            case KT_OP_Y: circuit.add_y_gate(t); return;
            case KT_OP_Z: circuit.add_z_gate(t); return;
            case KT_OP_S: circuit.add_s_gate(t); return;
            case KT_OP_SDAG: circuit.add_sdag_gate(t); return;
            case KT_OP_T: circuit.add_t_gate(t); return;
            case KT_OP_TDAG: circuit.add_tdag_gate(t); return;
            case KT_OP_SX: circuit.add_sx_gate(t); return;
            case KT_OP_SXDAG: circuit.add_sxdag_gate(t); return;
            case KT_OP_CH: circuit.add_ch_gate(c, t); return;
            case KT_OP_CX: circuit.add_cx_gate(c, t); return;
            case KT_OP_CY: circuit.add_cy_gate(c, t); return;
            case KT_OP_CZ: circuit.add_cz_gate(c, t); return;
            case KT_OP_CS: circuit.add_cs_gate(c, t); return;
            case KT_OP_CSDAG: circuit.add_csdag_gate(c, t); return;
            case KT_OP_CT: circuit.add_ct_gate(c, t); return;
            case KT_OP_CTDAG: circuit.add_ctdag_gate(c, t); return;
            case KT_OP_CSX: circuit.add_csx_gate(c, t); return;
            case KT_OP_CSXDAG: circuit.add_csxdag_gate(c, t); return;
            case KT_OP_U: circuit.add_u_gate(to_matrix(g.u), t); return;
            case KT_OP_CU: circuit.add_cu_gate(to_matrix(g.u), c, t); return;
            case KT_OP_M: circuit.add_m_gate(t, c); return;
            default: break;
        }
        // angle gates
        if (g.param >= 0) {
            auto it = ids.find(g.param);
            const bool fresh = (it == ids.end());
            const double v = params[g.param];
            ket::param::ParameterID id {};
            switch (g.op) {
                case KT_OP_RX: if (fresh) { id = circuit.add_rx_gate(t, v, ket::param::parameterized {}); } else { circuit.add_rx_gate(t, it->second); } break;
                case KT_OP_RY: if (fresh) { id = circuit.add_ry_gate(t, v, ket::param::parameterized {}); } else { circuit.add_ry_gate(t, it->second); } break;
                case KT_OP_RZ: if (fresh) { id = circuit.add_rz_gate(t, v, ket::param::parameterized {}); } else { circuit.add_rz_gate(t, it->second); } break;
                case KT_OP_P: if (fresh) { id = circuit.add_p_gate(t, v, ket::param::parameterized {}); } else { circuit.add_p_gate(t, it->second); } break;
                case KT_OP_CRX: if (fresh) { id = circuit.add_crx_gate(c, t, v, ket::param::parameterized {}); } else { circuit.add_crx_gate(c, t, it->second); } break;
                case KT_OP_CRY: if (fresh) { id = circuit.add_cry_gate(c, t, v, ket::param::parameterized {}); } else { circuit.add_cry_gate(c, t, it->second); } break;
                case KT_OP_CRZ: if (fresh) { id = circuit.add_crz_gate(c, t, v, ket::param::parameterized {}); } else { circuit.add_crz_gate(c, t, it->second); } break;
                case KT_OP_CP: if (fresh) { id = circuit.add_cp_gate(c, t, v, ket::param::parameterized {}); } else { circuit.add_cp_gate(c, t, it->second); } break;
                default: throw std::runtime_error {"ref_capi: unknown gate op"};
            }
            if (fresh) {
                ids.emplace(g.param, id);
            }
            return;
        }
        switch (g.op) {
            case KT_OP_RX: circuit.add_rx_gate(t, g.angle); return;
            case KT_OP_RY: circuit.add_ry_gate(t, g.angle); return;
            case KT_OP_RZ: circuit.add_rz_gate(t, g.angle); return;
            case KT_OP_P: circuit.add_p_gate(t, g.angle); return;
            case KT_OP_CRX: circuit.add_crx_gate(c, t, g.angle); return;
            case KT_OP_CRY: circuit.add_cry_gate(c, t, g.angle); return;
            case KT_OP_CRZ: circuit.add_crz_gate(c, t, g.angle); return;
            case KT_OP_CP: circuit.add_cp_gate(c, t, g.angle); return;
            default: throw std::runtime_error {"ref_capi: unknown gate op"};
        }
    }
};

auto host_state(int n, const double* amps) -> ket::Statevector
{
    const std::size_t n_states = std::size_t {1} << n;
    std::vector<std::complex<double>> coeffs(n_states);
    std::memcpy(coeffs.data(), amps, n_states * sizeof(std::complex<double>));
    return ket::Statevector {std::move(coeffs), ket::Endian::LITTLE, 1.0e-6};
}

void copy_out(const ket::Statevector& sv, double* amps)
{
    for (std::size_t i = 0; i < sv.n_states(); ++i) {
        amps[2 * i] = sv[i].real();
        amps[2 * i + 1] = sv[i].imag();
    }
}

auto to_string(const kt_pauli& p, std::size_t n) -> ket::SparsePauliString
{
    auto s = ket::SparsePauliString {n, static_cast<ket::PauliPhase>(p.phase)};
    for (std::size_t q = 0; q < n; ++q) {
        const bool x = ((p.x_mask >> q) & 1U) != 0;
        const bool z = ((p.z_mask >> q) & 1U) != 0;
        if (x && z) {
            s.add(q, ket::PauliTerm::Y);
        } else if (x) {
            s.add(q, ket::PauliTerm::X);
        } else if (z) {
            s.add(q, ket::PauliTerm::Z);
        }
    }
    return s;
}

template <typename F>
auto guarded(F&& f) -> int32_t
{
    try {
        f();
        return KT_OK;
    } catch (const std::exception& e) {
        g_err = e.what();
        return KT_ERR_INVALID;
    } catch (...) {
        g_err = "unknown exception";
        return KT_ERR_INVALID;
    }
}

}  // namespace

extern "C" {

const char* ref_last_error(void)
{
    return g_err.c_str();
}

// ket::simulate on a statevector (inout amplitudes, complex128 interleaved).
// cbits (nullable) receives the classical register after the run (-1 = unset).
int32_t ref_simulate_sv(int32_t n, const kt_gate* gates, int64_t n_gates, const double* params,
                        double* amps, int64_t seed, int32_t* cbits)
{
    return guarded([&] {
        CircuitBuilder b {static_cast<std::size_t>(n), params};
        for (int64_t i = 0; i < n_gates; ++i) {
            b.add(gates[i]);
        }
        auto sv = host_state(n, amps);
        auto sim = ket::StatevectorSimulator {};
        sim.run(b.circuit, sv, seed_opt(seed));
        copy_out(sv, amps);
        if (cbits != nullptr) {
            const auto& reg = sim.classical_register();
            for (std::size_t i = 0; i < b.circuit.n_bits(); ++i) {
                cbits[i] = reg.is_measured(i) ? reg.get(i) : -1;
            }
        }
    });
}

// Wall time of ket::simulate alone on a fresh Statevector(n) = |0...0>: the
// reference's CPU path for the CPU-baseline leg of bench.py.  The state is
// built once per call outside the timed region.
int32_t ref_time_sv(int32_t n, const kt_gate* gates, int64_t n_gates, const double* params, double* seconds)
{
    return guarded([&] {
        CircuitBuilder b {static_cast<std::size_t>(n), params};
        for (int64_t i = 0; i < n_gates; ++i) {
            b.add(gates[i]);
        }
        auto sv = ket::Statevector {static_cast<std::size_t>(n)};
        const auto t0 = std::chrono::steady_clock::now();
        ket::simulate(b.circuit, sv);
        const auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();
    });
}

// A reference Statevector(n) kept across calls, so a benchmark can time
// ket::simulate step after step without rebuilding a large state.
void* ref_sv_alloc(int32_t n)
{
    try {
        return new ket::Statevector {static_cast<std::size_t>(n)};
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_sv_free(void* h)
{
    delete static_cast<ket::Statevector*>(h);
}

int32_t ref_sv_time(void* h, const kt_gate* gates, int64_t n_gates, const double* params, double* seconds)
{
    return guarded([&] {
        auto& sv = *static_cast<ket::Statevector*>(h);
        CircuitBuilder b {sv.n_qubits(), params};
        for (int64_t i = 0; i < n_gates; ++i) {
            b.add(gates[i]);
        }
        const auto t0 = std::chrono::steady_clock::now();
        ket::simulate(b.circuit, sv);
        const auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();
    });
}

// ket::simulate on a density matrix (inout, column-major N x N complex128).
int32_t ref_simulate_dm(int32_t n, const kt_gate* gates, int64_t n_gates, const double* params,
                        double* rho, int64_t seed)
{
    return guarded([&] {
        CircuitBuilder b {static_cast<std::size_t>(n), params};
        for (int64_t i = 0; i < n_gates; ++i) {
            b.add(gates[i]);
        }
        const auto N = static_cast<Eigen::Index>(std::size_t {1} << n);
        Eigen::MatrixXcd m(N, N);
        std::memcpy(m.data(), rho, static_cast<std::size_t>(N * N) * sizeof(std::complex<double>));
        auto dm = ket::DensityMatrix {std::move(m), ket::density_matrix_nocheck {}};
        ket::simulate(b.circuit, dm, seed_opt(seed));
        std::memcpy(rho, dm.matrix().data(), static_cast<std::size_t>(N * N) * sizeof(std::complex<double>));
    });
}

// ket::partial_trace (density_matrix.cpp:231-278), column-major in and out.
int32_t ref_dm_partial_trace(int32_t n, const double* rho, const int64_t* qubits, int32_t k, double* out)
{
    return guarded([&] {
        const auto N = static_cast<Eigen::Index>(std::size_t {1} << n);
        Eigen::MatrixXcd m(N, N);
        std::memcpy(m.data(), rho, static_cast<std::size_t>(N * N) * sizeof(std::complex<double>));
        const auto dm = ket::DensityMatrix {std::move(m), ket::density_matrix_nocheck {}};
        std::vector<std::size_t> idx(qubits, qubits + k);
        const auto red = ket::partial_trace(dm, idx);
        const auto M = static_cast<std::size_t>(red.n_states());
        std::memcpy(out, red.matrix().data(), M * M * sizeof(std::complex<double>));
    });
}

// ket::tensor_product (density_matrix.cpp:187-214)
int32_t ref_dm_tensor_product(int32_t nl, const double* left, int32_t nr, const double* right, double* out)
{
    return guarded([&] {
        const auto A = static_cast<Eigen::Index>(std::size_t {1} << nl);
        const auto B = static_cast<Eigen::Index>(std::size_t {1} << nr);
        Eigen::MatrixXcd l(A, A);
        Eigen::MatrixXcd r(B, B);
        std::memcpy(l.data(), left, static_cast<std::size_t>(A * A) * sizeof(std::complex<double>));
        std::memcpy(r.data(), right, static_cast<std::size_t>(B * B) * sizeof(std::complex<double>));
        const auto t = ket::tensor_product(ket::DensityMatrix {std::move(l), ket::density_matrix_nocheck {}},
                                           ket::DensityMatrix {std::move(r), ket::density_matrix_nocheck {}});
        const auto D = static_cast<std::size_t>(t.n_states());
        std::memcpy(out, t.matrix().data(), D * D * sizeof(std::complex<double>));
    });
}

// DensityMatrix::trace_of_square
int32_t ref_dm_trace_of_square(int32_t n, const double* rho, double* out)
{
    return guarded([&] {
        const auto N = static_cast<Eigen::Index>(std::size_t {1} << n);
        Eigen::MatrixXcd m(N, N);
        std::memcpy(m.data(), rho, static_cast<std::size_t>(N * N) * sizeof(std::complex<double>));
        const auto v = ket::DensityMatrix {std::move(m), ket::density_matrix_nocheck {}}.trace_of_square();
        out[0] = v.real();
        out[1] = v.imag();
    });
}

// statevector_to_density_matrix (density_matrix.cpp:170-185), column-major out.
int32_t ref_sv_to_dm(int32_t n, const double* amps, double* rho)
{
    return guarded([&] {
        const auto sv = host_state(n, amps);
        const auto dm = ket::statevector_to_density_matrix(sv);
        const auto N = static_cast<std::size_t>(dm.n_states());
        std::memcpy(rho, dm.matrix().data(), N * N * sizeof(std::complex<double>));
    });
}

// ket::expectation_value for every string (phase * <P>) and for the whole operator.
int32_t ref_expect_sv(int32_t n, const double* amps, const kt_pauli* strings, int64_t n_strings,
                      const double* coeffs, double* out_terms, double* out_total)
{
    return guarded([&] {
        const auto sv = host_state(n, amps);
        std::vector<ket::WeightedPauliString> terms;
        for (int64_t k = 0; k < n_strings; ++k) {
            auto s = to_string(strings[k], static_cast<std::size_t>(n));
            if (out_terms != nullptr) {
                const auto v = ket::expectation_value(s, sv);
                out_terms[2 * k] = v.real();
                out_terms[2 * k + 1] = v.imag();
            }
            const std::complex<double> c = (coeffs != nullptr) ? std::complex<double> {coeffs[2 * k], coeffs[2 * k + 1]}
                                                                : std::complex<double> {1.0, 0.0};
            terms.push_back(ket::WeightedPauliString {c, std::move(s)});
        }
        if (out_total != nullptr && n_strings > 0) {
            const auto op = ket::PauliOperator {std::move(terms)};
            const auto v = ket::expectation_value(op, sv);
            out_total[0] = v.real();
            out_total[1] = v.imag();
        }
    });
}

static auto make_noise(int32_t n, const double* noise) -> std::optional<ket::QuantumNoise>
{
    if (noise == nullptr) {
        return std::nullopt;
    }
    auto qn = ket::QuantumNoise {static_cast<std::size_t>(n)};
    for (int32_t q = 0; q < n; ++q) {
        qn.set(static_cast<std::size_t>(q), noise[q]);
    }
    return qn;
}

int32_t ref_probabilities(int32_t n, const double* amps, const double* noise, double* out)
{
    return guarded([&] {
        const auto sv = host_state(n, amps);
        const auto qn = make_noise(n, noise);
        const auto p = ket::calculate_probabilities_raw(sv, qn ? &qn.value() : nullptr);
        std::memcpy(out, p.data(), p.size() * sizeof(double));
    });
}

// perform_measurements_as_memory with mt19937(seed): the sampled state indices.
int32_t ref_sample_memory(int32_t n, const double* amps, const double* noise, int64_t n_shots,
                          int64_t seed, uint64_t* out)
{
    return guarded([&] {
        const auto sv = host_state(n, amps);
        const auto qn = make_noise(n, noise);
        const auto mem = ket::perform_measurements_as_memory(sv, static_cast<std::size_t>(n_shots),
                                                             qn ? &qn.value() : nullptr, seed_opt(seed));
        for (std::size_t i = 0; i < mem.size(); ++i) {
            out[i] = mem[i];
        }
    });
}

// perform_measurements_as_counts: writes "bitstring count\n" lines into buf.
int32_t ref_sample_counts(int32_t n, const double* amps, int64_t n_shots, int64_t seed, char* buf,
                          int64_t buf_len)
{
    return guarded([&] {
        const auto sv = host_state(n, amps);
        const auto counts = ket::perform_measurements_as_counts(sv, static_cast<std::size_t>(n_shots), nullptr,
                                                                seed_opt(seed));
        std::string s;
        for (const auto& [bits, cnt] : counts) {
            s += bits + " " + std::to_string(cnt) + "\n";
        }
        if (static_cast<int64_t>(s.size()) + 1 > buf_len) {
            throw std::runtime_error {"ref_sample_counts: buffer too small"};
        }
        std::memcpy(buf, s.c_str(), s.size() + 1);
    });
}

int32_t ref_pairs_single(uint32_t n, uint32_t t, uint64_t k0, uint64_t count, uint64_t* out)
{
    return guarded([&] {
        auto gen = ket::internal::SingleQubitGatePairGenerator<std::size_t> {t, n};
        gen.set_state(k0);
        for (uint64_t k = 0; k < count; ++k) {
            const auto [a, b] = gen.next();
            out[2 * k] = a;
            out[2 * k + 1] = b;
        }
    });
}

int32_t ref_pairs_double(uint32_t n, uint32_t c, uint32_t t, int32_t quad, uint64_t k0, uint64_t count,
                         uint64_t* out)
{
    return guarded([&] {
        auto gen = ket::internal::DoubleQubitGatePairGenerator<std::size_t> {c, t, n};
        gen.set_state(k0);
        for (uint64_t k = 0; k < count; ++k) {
            if (quad != 0) {
                const auto [a, b, cc, d] = gen.next_unset_and_set();
                out[4 * k] = a;
                out[4 * k + 1] = b;
                out[4 * k + 2] = cc;
                out[4 * k + 3] = d;
            } else {
                const auto [a, b] = gen.next();
                out[2 * k] = a;
                out[2 * k + 1] = b;
            }
        }
    });
}

// generate_random_unitary2x2(seed) (random_u_gates.cpp:13-43), row-major interleaved.
int32_t ref_random_unitary(int32_t seed, double* u)
{
    return guarded([&] {
        const auto m = ket::generate_random_unitary2x2(seed);
        const std::complex<double> e[4] = {m.elem00, m.elem01, m.elem10, m.elem11};
        for (int i = 0; i < 4; ++i) {
            u[2 * i] = e[i].real();
            u[2 * i + 1] = e[i].imag();
        }
    });
}

// perform_measurements_as_memory(const std::vector<double>&, n_shots, seed)
// (calculations/measurements.cpp:73-94)
int32_t ref_sample_probabilities(const double* probs, int64_t n, int64_t n_shots, int64_t seed, uint64_t* out)
{
    return guarded([&] {
        const auto p = std::vector<double>(probs, probs + n);
        const auto m = ket::perform_measurements_as_memory(p, static_cast<std::size_t>(n_shots), static_cast<int>(seed));
        for (int64_t k = 0; k < n_shots; ++k) {
            out[k] = m[static_cast<std::size_t>(k)];
        }
    });
}

// `count` matrices from one std::mt19937(seed) stream, one
// generate_random_unitary2x2(std::mt19937&) call after another
// (gates/random_u_gates.cpp:13-36); 8 doubles per matrix
int32_t ref_random_unitaries(int32_t seed, int64_t count, double* u)
{
    return guarded([&] {
        auto prng = std::mt19937 {static_cast<std::mt19937::result_type>(seed)};
        for (int64_t k = 0; k < count; ++k) {
            const auto m = ket::generate_random_unitary2x2(prng);
            const std::complex<double> e[4] = {m.elem00, m.elem01, m.elem10, m.elem11};
            for (int i = 0; i < 4; ++i) {
                u[8 * k + 2 * i] = e[i].real();
                u[8 * k + 2 * i + 1] = e[i].imag();
            }
        }
    });
}

}  // extern "C"
