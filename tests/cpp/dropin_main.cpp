// dropin_main.cpp — one program, two builds.
//
// Uses only the kettle API (namespace ket, <kettle/kettle.hpp>).  It is
// compiled against the reference library (oracle/_ref, from the reference's
// own sources) and against this engine's C++ front end; tests/test_gpu_dropin.py
// runs both and compares what they print.
//
//   dropin <n_qubits> <layers> <seed>
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include <unistd.h>

#include <kettle/kettle.hpp>

namespace
{

struct SplitMix
{
    std::uint64_t s;
    auto next() -> std::uint64_t
    {
        std::uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    auto uniform() -> double { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
    auto below(std::uint64_t k) -> std::size_t { return static_cast<std::size_t>(next() % k); }
};

auto unitary(SplitMix& r) -> ket::Matrix2X2
{
    const double a = 6.283185307179586 * r.uniform(), b = 6.283185307179586 * r.uniform();
    const double c = 6.283185307179586 * r.uniform(), psi = std::asin(std::sqrt(r.uniform()));
    const std::complex<double> g {std::cos(a), std::sin(a)}, eb {std::cos(b), std::sin(b)}, ec {std::cos(c), std::sin(c)};
    return ket::Matrix2X2 {.elem00 = g * std::cos(psi) * eb, .elem01 = g * std::sin(psi) * ec,
                           .elem10 = -g * std::sin(psi) / ec, .elem11 = g * std::cos(psi) / eb};
}

void build(ket::QuantumCircuit& c, std::size_t n, int layers, SplitMix& r)
{
    for (int l = 0; l < layers; ++l) {
        for (std::size_t q = 0; q < n; ++q) {
            switch (r.below(6)) {
                case 0: c.add_h_gate(q); break;
                case 1: c.add_rx_gate(q, 6.283185307179586 * r.uniform()); break;
                case 2: c.add_ry_gate(q, 6.283185307179586 * r.uniform()); break;
                case 3: c.add_rz_gate(q, 6.283185307179586 * r.uniform()); break;
                case 4: c.add_u_gate(unitary(r), q); break;
                default: c.add_sx_gate(q); break;
            }
        }
        for (std::size_t q = static_cast<std::size_t>(l % 2); q + 1 < n; q += 2) {
            c.add_cx_gate(q, q + 1);
        }
        for (std::size_t k = 0; k < n / 2; ++k) {
            const std::size_t a = r.below(n);
            std::size_t b = r.below(n - 1);
            if (b >= a) {
                ++b;
            }
            switch (r.below(6)) {
                case 0: c.add_crx_gate(a, b, 6.283185307179586 * r.uniform()); break;
                case 1: c.add_cry_gate(a, b, 6.283185307179586 * r.uniform()); break;
                case 2: c.add_crz_gate(a, b, 6.283185307179586 * r.uniform()); break;
                case 3: c.add_cp_gate(a, b, 6.283185307179586 * r.uniform()); break;
                case 4: c.add_cz_gate(a, b); break;
                default: c.add_cu_gate(unitary(r), a, b); break;
            }
        }
    }
}

auto hamiltonian(std::size_t n, SplitMix& r) -> ket::PauliOperator
{
    std::vector<ket::WeightedPauliString> terms;
    for (int k = 0; k < 40; ++k) {
        auto s = ket::SparsePauliString {n};
        for (std::size_t q = 0; q < n; ++q) {
            const auto t = r.below(4);
            if (t == 1) s.add(q, ket::PauliTerm::X);
            if (t == 2) s.add(q, ket::PauliTerm::Y);
            if (t == 3) s.add(q, ket::PauliTerm::Z);
        }
        terms.push_back(ket::WeightedPauliString {{r.uniform() - 0.5, r.uniform() - 0.5}, s});
    }
    return ket::PauliOperator {terms};
}

auto fnv1a(const std::string& text) -> unsigned long long
{
    unsigned long long h = 0xcbf29ce484222325ULL;
    for (const unsigned char ch : text) {
        h = (h ^ ch) * 0x100000001b3ULL;
    }
    return h;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: dropin n layers seed\n");
        return 2;
    }
    const auto n = static_cast<std::size_t>(std::atoi(argv[1]));
    const int layers = std::atoi(argv[2]);
    const int seed = std::atoi(argv[3]);
    SplitMix r {static_cast<std::uint64_t>(seed)};

    // 1. statevector propagation with shared parameters
    auto circuit = ket::QuantumCircuit {n};
    build(circuit, n, layers, r);
    const auto id = circuit.add_ry_gate(0, 0.25, ket::param::parameterized {});
    circuit.add_rz_gate(n - 1, id);
    circuit.add_crx_gate(n - 1, 0, id);
    circuit.set_parameter_value(id, 0.75);
    auto sv = ket::Statevector {n};
    ket::simulate(circuit, sv);
    for (std::size_t i = 0; i < sv.n_states(); ++i) {
        std::printf("amp %zu %.17g %.17g\n", i, sv[i].real(), sv[i].imag());
    }

    // 2. Pauli expectation value
    const auto op = hamiltonian(n, r);
    const auto e = ket::expectation_value(op, sv);
    std::printf("expect %.17g %.17g\n", e.real(), e.imag());

    // 3. shot sampling (bit-exact given the seed)
    const auto counts = ket::perform_measurements_as_counts(sv, 4096, nullptr, seed);
    for (const auto& [bits, cnt] : counts) {
        std::printf("count %s %zu\n", bits.c_str(), cnt);
    }

    // 4. mid-circuit measurement
    auto mc = ket::QuantumCircuit {n};
    build(mc, n, 2, r);
    mc.add_m_gate(0);
    mc.add_h_gate(0);
    mc.add_m_gate(n - 1);
    auto msv = ket::Statevector {n};
    auto sim = ket::StatevectorSimulator {};
    sim.run(mc, msv, seed);
    std::printf("cbit0 %d cbitN %d\n", sim.classical_register().get(0), sim.classical_register().get(n - 1));
    for (std::size_t i = 0; i < msv.n_states(); ++i) {
        std::printf("mamp %zu %.17g %.17g\n", i, msv[i].real(), msv[i].imag());
    }

    // 5b. classical control flow and circuit loggers
    auto cf = ket::QuantumCircuit {n};
    build(cf, n, 1, r);
    cf.add_m_gate(0);
    cf.add_classical_register_circuit_logger();
    auto sub_x = ket::QuantumCircuit {n};
    sub_x.add_x_gate(1);
    sub_x.add_h_gate(n - 1);
    cf.add_if_statement(0, sub_x);
    cf.add_m_gate(1);
    auto sub_ry = ket::QuantumCircuit {n};
    sub_ry.add_ry_gate(0, 0.3);
    sub_ry.add_cx_gate(0, n - 1);
    auto sub_rz = ket::QuantumCircuit {n};
    sub_rz.add_rz_gate(0, 0.7);
    sub_rz.add_h_gate(1);
    cf.add_if_else_statement(1, sub_ry, sub_rz);
    cf.add_if_not_statement(0, sub_ry);
    cf.add_statevector_circuit_logger();
    cf.add_if_statement(ket::ControlFlowPredicate {{0, 1}, {1, 0}, ket::ControlFlowBooleanKind::IF_NOT}, sub_rz);
    cf.add_if_not_else_statement(1, sub_x, sub_ry);
    cf.add_m_gate(n - 1);
    cf.add_classical_register_circuit_logger();
    auto csv = ket::Statevector {n};
    auto csim = ket::StatevectorSimulator {};
    csim.run(cf, csv, seed + 7);
    std::printf("cfbits %d %d %d\n", csim.classical_register().get(0), csim.classical_register().get(1),
                csim.classical_register().get(n - 1));
    int k = 0;
    for (const auto& logger : csim.circuit_loggers()) {
        if (logger.is_classical_register_circuit_logger()) {
            const auto& creg = logger.get_classical_register_circuit_logger().classical_register();
            for (std::size_t b = 0; b < n; ++b) {
                std::printf("logbit %d %zu %d\n", k, b, creg.is_measured(b) ? creg.get(b) : -1);
            }
        } else if (logger.is_statevector_circuit_logger()) {
            const auto& lsv = logger.get_statevector_circuit_logger().statevector();
            for (std::size_t i = 0; i < lsv.n_states(); ++i) {
                std::printf("logamp %d %zu %.17g %.17g\n", k, i, lsv[i].real(), lsv[i].imag());
            }
        }
        ++k;
    }
    for (std::size_t i = 0; i < csv.n_states(); ++i) {
        std::printf("cfamp %zu %.17g %.17g\n", i, csv[i].real(), csv[i].imag());
    }

    // 5. density matrix propagation
    const std::size_t nd = n < 5 ? n : 5;
    auto dc = ket::QuantumCircuit {nd};
    build(dc, nd, 3, r);
    auto dm = ket::DensityMatrix {std::string(nd, '0')};
    ket::simulate(dc, dm);
    const auto& m = dm.matrix();
    for (long rr = 0; rr < static_cast<long>(dm.n_states()); ++rr) {
        for (long cc = 0; cc < static_cast<long>(dm.n_states()); ++cc) {
            std::printf("rho %ld %ld %.17g %.17g\n", rr, cc, m(rr, cc).real(), m(rr, cc).imag());
        }
    }
    // 6. on-disk formats
    // 6a. the statevector text, bit for bit, on a state both builds hold
    //     exactly: amplitudes made here, with zeros, negative zeros and values
    //     that print as -0.00000000000000
    std::vector<std::complex<double>> coeffs(std::size_t {1} << n);
    double norm2 = 0.0;
    for (std::size_t i = 0; i < coeffs.size(); ++i) {
        double re = r.uniform() - 0.5;
        double im = r.uniform() - 0.5;
        switch (i % 7) {
            case 1: re = 0.0; break;
            case 2: im = -0.0; break;
            case 3: re = -1e-17; break;
            case 4: im = 4e-15; break;
            default: break;
        }
        coeffs[i] = {re, im};
        norm2 += re * re + im * im;
    }
    const double inv_norm = 1.0 / std::sqrt(norm2);
    for (auto& c : coeffs) {
        c *= inv_norm;
    }
    const auto hsv = ket::Statevector {coeffs};
    for (const auto endian : {ket::Endian::LITTLE, ket::Endian::BIG}) {
        std::ostringstream text;
        ket::save_statevector(text, hsv, endian);
        const auto str = text.str();
        std::printf("svtext %d %zu %016llx\n", static_cast<int>(endian == ket::Endian::BIG), str.size(), fnv1a(str));
        std::istringstream in {str};
        const auto back = ket::load_statevector(in);
        double dev = 0.0;
        for (std::size_t i = 0; i < hsv.n_states(); ++i) {
            dev = std::max(dev, std::abs(back[i] - hsv[i]));
        }
        std::printf("svload %d %zu %.3g\n", static_cast<int>(endian == ket::Endian::BIG), back.n_qubits(), dev);
    }

    // 6b. the simulated state through a file, big-endian, and back
    const auto tmp = std::filesystem::temp_directory_path();
    const auto tag = std::to_string(static_cast<long>(getpid()));
    const auto sv_path = tmp / ("kt_dropin_sv_" + tag + ".txt");
    ket::save_statevector(sv_path, sv, ket::Endian::BIG);
    const auto sv_back = ket::load_statevector(sv_path);
    for (std::size_t i = 0; i < sv_back.n_states(); ++i) {
        std::printf("ioamp %zu %.17g %.17g\n", i, sv_back[i].real(), sv_back[i].imag());
    }

    // 6c. numpy's complex text, read as big-endian and, from a file, as little-endian
    std::ostringstream np_text;
    np_text << n << '\n';
    char buf[96];
    for (std::size_t i = 0; i < sv.n_states(); ++i) {
        const auto v = sv[i];
        std::snprintf(buf, sizeof(buf), (i % 3 == 0) ? "(%.17g%+.17gj)\n" : "(%.8e%+.8ej)\n", v.real(), v.imag());
        np_text << buf;
    }
    std::istringstream np_in {np_text.str()};
    const auto np_sv = ket::read_numpy_statevector(np_in, ket::Endian::BIG);
    for (std::size_t i = 0; i < np_sv.n_states(); ++i) {
        std::printf("npamp %zu %.17g %.17g\n", i, np_sv[i].real(), np_sv[i].imag());
    }
    const auto np_path = tmp / ("kt_dropin_np_" + tag + ".txt");
    {
        auto out = std::ofstream {np_path};
        out << np_text.str();
    }
    const auto np_file = ket::read_numpy_statevector(np_path);
    double np_dev = 0.0;
    for (std::size_t i = 0; i < np_file.n_states(); ++i) {
        np_dev = std::max(np_dev, std::abs(np_file[i] - sv[i]));
    }
    std::printf("npfile %.3g\n", np_dev);

    // 6d. a Hamiltonian in the "re im : (q, P) ..." text, then its expectation value
    std::ostringstream ham_text;
    for (int k = 0; k < 30; ++k) {
        std::snprintf(buf, sizeof(buf), "%.17g %.17g :", r.uniform() - 0.5, (k % 4 == 0) ? 0.0 : r.uniform() - 0.5);
        ham_text << buf;
        for (std::size_t q = 0; q < n; ++q) {
            const auto t = r.below(4);
            if (t != 0) {
                ham_text << " (" << q << ", " << "XYZ"[t - 1] << ')';
            }
        }
        ham_text << '\n';
    }
    std::istringstream ham_in {ham_text.str()};
    const auto ham = ket::read_pauli_operator(ham_in, n);
    const auto he = ket::expectation_value(ham, sv);
    std::printf("pauliop %zu %.17g %.17g\n", ham.weighted_pauli_strings().size(), he.real(), he.imag());
    const auto ham_path = tmp / ("kt_dropin_ham_" + tag + ".txt");
    {
        auto out = std::ofstream {ham_path};
        out << ham_text.str();
    }
    const auto he_file = ket::expectation_value(ket::read_pauli_operator(ham_path, n), sv);
    std::printf("pauliopfile %.17g %.17g\n", he_file.real(), he_file.imag());
    std::filesystem::remove(sv_path);
    std::filesystem::remove(np_path);
    std::filesystem::remove(ham_path);

    // 6e. the readers' errors
    const auto missing = tmp / ("kt_dropin_missing_" + tag + ".txt");
    try {
        (void) ket::load_statevector(missing);
    } catch (const std::exception& err) {
        std::printf("ioerr load %d\n", static_cast<int>(std::string {err.what()}.find("unable to open file to load statevector") != std::string::npos));
    }
    try {
        (void) ket::read_numpy_statevector(missing);
    } catch (const std::exception& err) {
        std::printf("ioerr numpy %d\n", static_cast<int>(std::string {err.what()}.find("unable to open file for statevector") != std::string::npos));
    }
    try {
        (void) ket::read_pauli_operator(missing, n);
    } catch (const std::exception& err) {
        std::printf("ioerr pauli %d\n", static_cast<int>(std::string {err.what()}.find("ERROR: unable to open: ") != std::string::npos));
    }
    try {
        std::istringstream bad {"0.5 0.0 : (0, W)\n"};
        (void) ket::read_pauli_operator(bad, n);
        std::printf("ioerr badterm none\n");
    } catch (const std::out_of_range&) {
        std::printf("ioerr badterm out_of_range\n");
    }
    // 7. compound gates (Toffoli family, CCU, SWAP, CSWAP, QFT / inverse QFT)
    if (n >= 4) {
        auto cg = ket::QuantumCircuit {n};
        build(cg, n, 1, r);
        const auto pick3 = [&]() {
            std::size_t a = r.below(n), b = r.below(n), c = r.below(n);
            while (b == a) b = r.below(n);
            while (c == a || c == b) c = r.below(n);
            return std::tuple<std::size_t, std::size_t, std::size_t> {a, b, c};
        };
        const auto [a0, b0, c0] = pick3();
        cg.add_ccx_gate(a0, b0, c0);
        const auto [a1, b1, c1] = pick3();
        cg.add_ccy_gate({{a1, b1, c1}});
        const auto [a2, b2, c2] = pick3();
        cg.add_ccz_gate(a2, b2, c2);
        const auto [a3, b3, c3] = pick3();
        cg.add_ccu_gate(unitary(r), a3, b3, c3);
        const auto [a4, b4, c4] = pick3();
        cg.add_swap_gate(a4, b4);
        cg.add_cswap_gate(c4, a4, b4);
        std::vector<std::size_t> fourier;
        for (std::size_t q = 0; q < n; q += 2) {
            fourier.push_back(q);
        }
        std::vector<std::size_t> all(n);
        for (std::size_t q = 0; q < n; ++q) {
            all[q] = n - 1 - q;
        }
        cg.add_qft_gate(fourier);
        cg.add_iqft_gate(all);
        auto cgs = ket::Statevector {n};
        ket::simulate(cg, cgs);
        std::printf("cgelems %zu\n", cg.n_circuit_elements());
        for (std::size_t i = 0; i < cgs.n_states(); ++i) {
            std::printf("cgamp %zu %.17g %.17g\n", i, cgs[i].real(), cgs[i].imag());
        }
        const auto root = ket::matrix_square_root(unitary(r));
        std::printf("sqrtu %.17g %.17g %.17g %.17g\n", root.elem00.real(), root.elem01.imag(), root.elem10.real(),
                    root.elem11.imag());
    }

    // 8. density-matrix partial traces, tensor products and purity
    {
        const std::size_t nt = n < 6 ? n : 6;
        auto tc = ket::QuantumCircuit {nt};
        build(tc, nt, 2, r);
        auto tdm = ket::DensityMatrix {std::string(nt, '0')};
        ket::simulate(tc, tdm);
        const auto print_dm = [](const char* tag, int id, const ket::DensityMatrix& d) {
            const auto& mm = d.matrix();
            std::printf("%s %d nq %zu\n", tag, id, d.n_qubits());
            for (long rr = 0; rr < static_cast<long>(d.n_states()); ++rr) {
                for (long cc = 0; cc < static_cast<long>(d.n_states()); ++cc) {
                    std::printf("%s %d %ld %ld %.17g %.17g\n", tag, id, rr, cc, mm(rr, cc).real(), mm(rr, cc).imag());
                }
            }
        };
        std::vector<std::vector<std::size_t>> cases {{0}, {nt - 1}};
        if (nt >= 3) {
            cases.push_back({nt - 1, 0, 1});
            cases.push_back({1, 1});
            cases.push_back({2, 0});
        }
        std::vector<std::size_t> every(nt);
        for (std::size_t q = 0; q < nt; ++q) {
            every[q] = q;
        }
        cases.push_back(every);
        for (std::size_t j = 0; j < cases.size(); ++j) {
            print_dm("ptrace", static_cast<int>(j), ket::partial_trace(tdm, cases[j]));
        }
        try {
            (void) ket::partial_trace(tdm, {nt});
        } catch (const std::runtime_error& err) {
            std::printf("pterr %d\n", static_cast<int>(std::string {err.what()}.find("out of bounds") != std::string::npos));
        }
        auto lc = ket::QuantumCircuit {2};
        build(lc, 2, 2, r);
        auto ldm = ket::DensityMatrix {"00"};
        ket::simulate(lc, ldm);
        const auto tp = ket::tensor_product(ldm, tdm);
        print_dm("tensor", 0, ket::partial_trace(tp, {1}));
        const auto tp3 = ket::tensor_product({ldm, ket::DensityMatrix {"1"}, ldm});
        print_dm("tensor", 1, tp3);
        const auto t2 = tdm.trace_of_square();
        const auto mixed = ket::partial_trace(tdm, {0});
        const auto m2 = mixed.trace_of_square();
        std::printf("purity %.17g %.17g %d %.17g %.17g %d\n", t2.real(), t2.imag(), static_cast<int>(tdm.is_pure()),
                    m2.real(), m2.imag(), static_cast<int>(mixed.is_pure()));
    }
    // 9. circuit transforms: U / CU gates lowered to primitive gates, circuits appended
    if (n >= 2) {
        auto uc = ket::QuantumCircuit {n};
        build(uc, n, 1, r);
        uc.add_u_gate(ket::h_gate(), 0);
        uc.add_u_gate(ket::rx_gate(0.3), n - 1);
        uc.add_u_gate(ket::p_gate(-1.1), 1);
        uc.add_u_gate(unitary(r), 0);
        uc.add_cu_gate(unitary(r), 0, n - 1);
        uc.add_cu_gate(ket::sx_gate(), n - 1, 0);
        auto prod = ket::rz_gate(2.0);
        prod *= ket::ry_gate(0.4);
        uc.add_u_gate(prod, 1);
        uc.add_cu_gate(ket::x_gate() * std::complex<double> {0.0, 1.0}, 1, 0);
        const auto tr = ket::transpile_to_primitive(uc);
        int k = 0;
        for (const auto& el : tr) {
            const auto& gi = el.get_gate();
            std::printf("tpgate %d %d %zu %zu %.17g\n", k++, static_cast<int>(gi.gate), gi.arg0, gi.arg1, gi.arg2);
        }
        const auto joined = ket::append_circuits(tr, uc);
        std::printf("tpelems %zu %zu %zu\n", uc.n_circuit_elements(), tr.n_circuit_elements(), joined.n_circuit_elements());
        auto js = ket::Statevector {n};
        ket::simulate(joined, js);
        for (std::size_t i = 0; i < js.n_states(); ++i) {
            std::printf("tpamp %zu %.17g %.17g\n", i, js[i].real(), js[i].imag());
        }
        try {
            (void) ket::append_circuits(tr, ket::QuantumCircuit {n + 1});
        } catch (const std::runtime_error& err) {
            std::printf("tperr %s\n", std::string {err.what()}.find("different numbers of qubits") != std::string::npos ? "qubits" : "other");
        }
    }
    // 10. a Pauli string applied to a state, statevector tensor products, a
    //     diagonal expectation value, sampling from a probability vector, the
    //     circuit-and-state marginal counts, and M gates on a density matrix
    {
        auto pc = ket::QuantumCircuit {n};
        build(pc, n, 2, r);
        auto ps = ket::Statevector {n};
        ket::simulate(pc, ps);
        auto terms = std::vector<std::pair<std::size_t, ket::PauliTerm>> {};
        const ket::PauliTerm kinds[3] = {ket::PauliTerm::X, ket::PauliTerm::Y, ket::PauliTerm::Z};
        for (std::size_t q = 0; q < n; ++q) {
            if (r.below(4) != 0) {
                terms.emplace_back(q, kinds[r.below(3)]);
            }
        }
        ket::simulate(ket::SparsePauliString {terms, n, ket::PauliPhase::MINUS_EYE}, ps);
        for (std::size_t i = 0; i < ps.n_states(); ++i) {
            std::printf("psamp %zu %.17g %.17g\n", i, ps[i].real(), ps[i].imag());
        }
        try {
            ket::simulate(ket::SparsePauliString {n + 1}, ps);
        } catch (const std::runtime_error& err) {
            std::printf("pserr %d\n", static_cast<int>(std::string {err.what()}.find("different number of qubits") != std::string::npos));
        }
        const std::size_t na = (n + 1) / 2;
        auto ca = ket::QuantumCircuit {na};
        build(ca, na, 2, r);
        auto cb = ket::QuantumCircuit {n - na + 1};
        build(cb, n - na + 1, 2, r);
        auto sa = ket::Statevector {na};
        auto sb = ket::Statevector {n - na + 1};
        ket::simulate(ca, sa);
        ket::simulate(cb, sb);
        const auto tp = ket::tensor_product(sa, sb);
        for (std::size_t i = 0; i < tp.n_states(); ++i) {
            std::printf("svtp %zu %.17g %.17g\n", i, tp[i].real(), tp[i].imag());
        }
        auto eig = std::vector<std::complex<double>> {};
        for (std::size_t i = 0; i < ps.n_states(); ++i) {
            eig.emplace_back(2.0 * r.uniform() - 1.0, 2.0 * r.uniform() - 1.0);
        }
        const auto de = ket::diagonal_expectation_value(eig, ps);
        std::printf("diagexp %.17g %.17g\n", de.real(), de.imag());
        const auto probs = ket::calculate_probabilities_raw(ps);
        const auto mem = ket::perform_measurements_as_memory(probs, 64, 17);
        for (std::size_t k = 0; k < mem.size(); ++k) {
            std::printf("pmem %zu %zu\n", k, mem[k]);
        }
        for (const auto& [idx, cnt] : ket::perform_measurements_as_counts_raw(probs, 256, 23)) {
            std::printf("pcraw %zu %zu\n", idx, cnt);
        }
        for (const auto& [bits, cnt] : ket::perform_measurements_as_counts_marginal(probs, 256, {0, n - 1}, 29)) {
            std::printf("pcmarg %s %zu\n", bits.c_str(), cnt);
        }
        auto odd = std::vector<double> {0.25, 0.5, 0.25};
        for (const auto& [idx, cnt] : ket::perform_measurements_as_counts_raw(odd, 64, 31)) {
            std::printf("pcodd %zu %zu\n", idx, cnt);
        }
        try {
            (void) ket::perform_measurements_as_counts_marginal(odd, 8, {}, 31);
        } catch (const std::runtime_error& err) {
            std::printf("pmerr %d\n", static_cast<int>(std::string {err.what()}.find("power of 2") != std::string::npos));
        }
        for (const auto& [bits, cnt] : ket::perform_measurements_as_counts_marginal(pc, ket::Statevector {n}, 6, {1}, nullptr, 37)) {
            std::printf("ccmarg %s %zu\n", bits.c_str(), cnt);
        }
        // M gates on a density matrix (fewer qubits: the reference's density
        // matrix passes are slow)
        const std::size_t nd = std::min<std::size_t>(n, 5);
        auto mc = ket::QuantumCircuit {nd, nd};
        build(mc, nd, 1, r);
        mc.add_m_gate(0, 0);
        build(mc, nd, 1, r);
        mc.add_m_gate(nd - 1, nd - 1);
        mc.add_m_gate(1 % nd, 1 % nd);
        auto mdm = ket::DensityMatrix {std::string(nd, '0')};
        auto dsim = ket::DensityMatrixSimulator {nd};
        dsim.run(mc, mdm, 43);
        std::printf("dmmbits %d %d %d\n", dsim.classical_register().get(0), dsim.classical_register().get(nd - 1),
                    dsim.classical_register().get(1 % nd));
        const auto& dm2 = mdm.matrix();
        for (long rr = 0; rr < dm2.rows(); ++rr) {
            for (long cc = 0; cc < dm2.cols(); ++cc) {
                std::printf("dmmrho %ld %ld %.17g %.17g\n", rr, cc, dm2(rr, cc).real(), dm2(rr, cc).imag());
            }
        }
    }
    return 0;
}
