// dropin_host_main.cpp — the host-side utilities of the kettle API, built once
// against the reference library and once against the ket:: front end; both
// builds must print the same text.
//
//   dropin_host <mode>
//     host    bitstring / state-index / dynamic-bitset conversions, binary
//             fraction expansions, marginal strips, seeded random 2x2
//             unitaries, n-local ansatz circuits, integer ranges, gate
//             matrices by kind, Pauli-string equality, circuit adders and
//             compound gates, transpiled circuits, classical registers and
//             control-flow predicates, 2x2 matrix arithmetic, Pauli strings
//             and operators, readout noise, memory-to-counts, and the errors
//             of each (no GPU is touched)
//     states  seeded random states and projections of them, and the io/
//             text formats (statevector save / load, numpy text, Pauli
//             operator text); the front end keeps states on the GPU
//
// Doubles are printed as hexadecimal floating point, so equal text means
// equal bits.  Uses only the public kettle API.
#include <complex>
#include <cstdint>
#include <cstdio>
#include <exception>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "kettle/kettle.hpp"

namespace
{

void show_error(const char* what, const std::exception& e)
{
    std::string msg = e.what();
    for (auto& c : msg) {
        if (c == '\n') {
            c = '|';
        }
    }
    std::printf("err %s %s\n", what, msg.c_str());
}

std::string bits_text(const std::vector<std::uint8_t>& bits)
{
    std::string out;
    for (auto b : bits) {
        out += std::to_string(static_cast<int>(b));
    }
    return out.empty() ? "-" : out;
}

void show_matrix(const char* tag, int key, const ket::Matrix2X2& m)
{
    const std::complex<double> e[4] = {m.elem00, m.elem01, m.elem10, m.elem11};
    std::printf("%s %d", tag, key);
    for (const auto& z : e) {
        std::printf(" %a %a", z.real(), z.imag());
    }
    std::printf("\n");
}

void nlocal_and_helpers();
void host_objects();

void host_mode()
{
    // every index of 1..5 qubits, both endians, through every conversion
    for (std::size_t n = 1; n <= 5; ++n) {
        for (std::size_t i = 0; i < (std::size_t {1} << n); ++i) {
            const auto le = ket::state_index_to_bitstring_little_endian(i, n);
            const auto be = ket::state_index_to_bitstring_big_endian(i, n);
            const auto dle = ket::state_index_to_dynamic_bitset_little_endian(i, n);
            const auto dbe = ket::state_index_to_dynamic_bitset_big_endian(i, n);
            std::printf("conv %zu %zu %s %s %s %s %zu %zu %zu %zu %s %s\n", n, i, le.c_str(), be.c_str(),
                        bits_text(dle).c_str(), bits_text(dbe).c_str(), ket::bitstring_to_state_index_little_endian(le),
                        ket::bitstring_to_state_index_big_endian(be), ket::dynamic_bitset_to_state_index_little_endian(dle),
                        ket::dynamic_bitset_to_state_index_big_endian(dbe),
                        ket::dynamic_bitset_to_bitstring(dle).c_str(), bits_text(ket::bitstring_to_dynamic_bitset(be)).c_str());
            std::printf("frac %zu %zu %a %a\n", n, i, ket::binary_fraction_expansion(le, ket::Endian::LITTLE),
                        ket::binary_fraction_expansion(le, ket::Endian::BIG));
        }
    }
    // the generic forms, the empty string, non-0/1 bytes in a bitset
    std::printf("generic %zu %zu %s %s\n", ket::bitstring_to_state_index("0110", ket::Endian::LITTLE),
                ket::bitstring_to_state_index("0110", ket::Endian::BIG),
                ket::state_index_to_bitstring(6, 4, ket::Endian::LITTLE).c_str(),
                bits_text(ket::state_index_to_dynamic_bitset(6, 4, ket::Endian::BIG)).c_str());
    std::printf("empty %zu %zu %a %s\n", ket::bitstring_to_state_index("", ket::Endian::LITTLE),
                ket::bitstring_to_state_index("", ket::Endian::BIG), ket::binary_fraction_expansion(""),
                bits_text(ket::bitstring_to_dynamic_bitset("")).c_str());
    std::printf("bytes %s %zu\n", ket::dynamic_bitset_to_bitstring({0, 2, 7, 0, 1}).c_str(),
                ket::dynamic_bitset_to_state_index({0, 3, 0, 1}, ket::Endian::BIG));
    std::printf("long %a %a\n", ket::binary_fraction_expansion("1011011101111011111011111101111111", ket::Endian::LITTLE),
                ket::binary_fraction_expansion("1011011101111011111011111101111111", ket::Endian::BIG));
    // errors
    try {
        (void)ket::bitstring_to_state_index("01x1", ket::Endian::LITTLE);
    } catch (const std::exception& e) {
        show_error("index_of_marginal", e);
    }
    try {
        (void)ket::bitstring_to_dynamic_bitset("0121");
    } catch (const std::exception& e) {
        show_error("bitset_of_bad", e);
    }
    try {
        (void)ket::binary_fraction_expansion("10 1");
    } catch (const std::exception& e) {
        show_error("fraction_of_bad", e);
    }
    try {
        (void)ket::state_index_to_bitstring_little_endian(8, 3);
    } catch (const std::exception& e) {
        show_error("index_too_large", e);
    }
    try {
        (void)ket::state_index_to_dynamic_bitset_big_endian(100, 4);
    } catch (const std::exception& e) {
        show_error("bitset_index_too_large", e);
    }
    // marginal strips, valid and invalid
    const char* marginals[] = {"", "x", "xxx", "01", "01xx", "xx01", "0x1", "x0x", "1xx0", "xx", "0xxx1", "101x"};
    for (const char* m : marginals) {
        try {
            std::printf("rstrip '%s' '%s'\n", m, ket::rstrip_marginal_bits(m).c_str());
        } catch (const std::exception& e) {
            show_error("rstrip", e);
        }
        try {
            std::printf("lstrip '%s' '%s'\n", m, ket::lstrip_marginal_bits(m).c_str());
        } catch (const std::exception& e) {
            show_error("lstrip", e);
        }
    }
    // random 2x2 unitaries: seeded, and a stream from one generator
    for (int seed = 0; seed < 12; ++seed) {
        show_matrix("useed", seed, ket::generate_random_unitary2x2(seed));
    }
    auto prng = std::mt19937 {20240};
    for (int k = 0; k < 8; ++k) {
        show_matrix("ustream", k, ket::generate_random_unitary2x2(prng));
    }
    nlocal_and_helpers();
    host_objects();
}

template <typename Integer>
void show_range(const char* tag, const std::vector<Integer>& v)
{
    std::printf("%s %zu", tag, v.size());
    for (auto x : v) {
        std::printf(" %lld", static_cast<long long>(x));
    }
    std::printf("\n");
}

void show_nlocal(int key, std::size_t n, const std::vector<ket::GeneralGate>& rot, const std::vector<ket::GeneralGate>& ent,
                 ket::NLocalEntangelement kind, std::size_t reps, ket::SkipLastRotationLayerFlag flag)
{
    try {
        auto [circuit, ids] = ket::n_local(n, rot, ent, kind, reps, flag);
        std::printf("nlocal %d n=%zu elements=%zu params=%zu\n", key, circuit.n_qubits(), circuit.n_circuit_elements(),
                    ids.size());
        int k = 0;
        for (const auto& el : circuit) {
            const auto& gi = el.get_gate();
            std::printf("nlgate %d %d %d %zu %zu %a\n", key, k++, static_cast<int>(gi.gate), gi.arg0, gi.arg1, gi.arg2);
        }
        for (std::size_t j = 0; j < ids.size(); ++j) {
            circuit.set_parameter_value(ids[j], 0.125 * static_cast<double>(j + 1));
        }
        for (std::size_t j = 0; j < ids.size(); ++j) {
            const auto& data = circuit.parameter_data_map().at(ids[j]);
            std::printf("nlparam %d %zu %zu %a\n", key, j, data.count, data.value ? *data.value : -1.0);
        }
    } catch (const std::exception& e) {
        show_error("nlocal", e);
    }
}

void nlocal_and_helpers()
{
    using G = ket::Gate;
    using CG = ket::CompoundGate;
    using NE = ket::NLocalEntangelement;
    using SK = ket::SkipLastRotationLayerFlag;
    show_nlocal(0, 2, {G::RZ, G::RY}, {G::CX}, NE::LINEAR, 1, SK::FALSE);
    show_nlocal(1, 4, {G::RY, G::H}, {G::CZ}, NE::FULL, 2, SK::FALSE);
    show_nlocal(2, 5, {G::RX, G::CRY}, {G::CP}, NE::LINEAR, 2, SK::TRUE);
    show_nlocal(3, 4, {CG::CCX, G::RZ}, {CG::CCZ, G::CX}, NE::FULL, 1, SK::FALSE);
    show_nlocal(4, 6, {G::X, G::CH, CG::CCY}, {CG::CCY, G::CSX}, NE::LINEAR, 1, SK::FALSE);
    show_nlocal(5, 3, {G::P, G::SX}, {G::CRZ}, NE::LINEAR, 3, SK::TRUE);
    show_nlocal(6, 4, {G::RY}, {G::CRX}, NE::FULL, 1, SK::FALSE);   // the reference's FULL angle-gate loop
    show_nlocal(7, 1, {G::RY}, {G::CRX}, NE::FULL, 1, SK::FALSE);
    show_nlocal(8, 1, {G::RY}, {CG::CCX}, NE::LINEAR, 1, SK::FALSE);
    show_nlocal(9, 3, {G::U}, {G::CX}, NE::LINEAR, 1, SK::FALSE);
    show_nlocal(10, 3, {G::RY}, {G::H}, NE::LINEAR, 1, SK::FALSE);
    show_nlocal(11, 3, {G::M}, {G::CX}, NE::LINEAR, 1, SK::FALSE);
    show_nlocal(12, 3, {}, {}, NE::LINEAR, 2, SK::FALSE);

    show_range("ar0", ket::arange(std::size_t {6}));
    show_range("ar1", ket::arange(5));
    show_range("ar2", ket::arange(-3));
    show_range("ar3", ket::arange(2, 11, 3));
    show_range("ar4", ket::arange(10, 1, -4));
    show_range("ar5", ket::arange(std::size_t {7}, std::size_t {2}, -2));
    show_range("ar6", ket::arange(4, 4));
    show_range("ar7", ket::arange(1, 5, -1));
    show_range("rv0", ket::revarange(std::size_t {5}));
    show_range("rv1", ket::revarange(-1, 8, 3));
    show_range("rv2", ket::revarange(9, 0, -2));
    try {
        (void)ket::arange(0, 5, 0);
    } catch (const std::exception& e) {
        show_error("arange_step", e);
    }

    show_matrix("mi", 0, ket::i_gate());
    int k = 0;
    for (auto g : {G::H, G::X, G::Y, G::Z, G::S, G::SDAG, G::T, G::TDAG, G::SX, G::SXDAG, G::CH, G::CX, G::CY, G::CZ,
                   G::CS, G::CSDAG, G::CT, G::CTDAG, G::CSX, G::CSXDAG}) {
        show_matrix("mna", k++, ket::non_angle_gate(g));
    }
    k = 0;
    for (auto g : {G::RX, G::RY, G::RZ, G::P, G::CRX, G::CRY, G::CRZ, G::CP}) {
        const double angle = 0.3 + 0.7 * k;
        show_matrix("ma", k++, ket::angle_gate(g, angle));
    }
    try {
        (void)ket::non_angle_gate(G::RX);
    } catch (const std::exception& e) {
        show_error("non_angle", e);
    }
    try {
        (void)ket::angle_gate(G::H, 1.0);
    } catch (const std::exception& e) {
        show_error("angle", e);
    }

    using P = ket::PauliTerm;
    const auto a = ket::SparsePauliString {{{0, P::X}, {2, P::Z}, {3, P::Y}}, 5};
    const auto b = ket::SparsePauliString {{{3, P::Y}, {1, P::I}, {0, P::X}, {2, P::Z}}, 5, ket::PauliPhase::MINUS_ONE};
    const auto c = ket::SparsePauliString {{{0, P::X}, {2, P::Z}, {3, P::Y}}, 6};
    const auto d = ket::SparsePauliString {{{0, P::X}, {2, P::Z}, {3, P::X}}, 5};
    const auto e = ket::SparsePauliString {{P::X, P::I, P::Z, P::Y, P::I}};
    const ket::SparsePauliString* all[] = {&a, &b, &c, &d, &e};
    for (int i = 0; i < 5; ++i) {
        for (int j = 0; j < 5; ++j) {
            std::printf("peq %d %d %d %d\n", i, j, static_cast<int>(all[i]->equal_up_to_phase(*all[j])),
                        static_cast<int>(*all[i] == *all[j]));
        }
    }
}

void show_circuit(const char* tag, int key, const ket::QuantumCircuit& c)
{
    std::printf("%s %d n=%zu bits=%zu elements=%zu\n", tag, key, c.n_qubits(), c.n_bits(), c.n_circuit_elements());
    int k = 0;
    for (const auto& el : c) {
        if (!el.is_gate()) {
            std::printf("%s %d %d nongate\n", tag, key, k++);
            continue;
        }
        const auto& gi = el.get_gate();
        std::printf("%s %d %d %d %zu %zu %a", tag, key, k++, static_cast<int>(gi.gate), gi.arg0, gi.arg1, gi.arg2);
        if (gi.unitary_ptr) {
            const auto& m = *gi.unitary_ptr;
            for (const auto& z : {m.elem00, m.elem01, m.elem10, m.elem11}) {
                std::printf(" %a %a", z.real(), z.imag());
            }
        }
        std::printf("\n");
    }
}

#define KET_TRY(tag, expr)                  \
    try {                                   \
        expr;                               \
        std::printf("noerr %s\n", tag);     \
    } catch (const std::exception& e) {     \
        show_error(tag, e);                 \
    }

void host_objects()
{
    // circuit adders: range errors, pop_back, compound gates' primitive sequences
    auto c = ket::QuantumCircuit {3};
    KET_TRY("x_range", c.add_x_gate(3));
    KET_TRY("cx_target_range", c.add_cx_gate(0, 3));
    KET_TRY("cx_control_range", c.add_cx_gate(4, 0));
    KET_TRY("rx_range", c.add_rx_gate(5, 0.1));
    KET_TRY("crz_range", c.add_crz_gate(1, 9, 0.1));
    KET_TRY("m_bit_range", c.add_m_gate(0, 7));
    KET_TRY("m_qubit_range", c.add_m_gate(3));
    KET_TRY("u_range", c.add_u_gate(ket::h_gate(), 3));
    KET_TRY("ccx_range", c.add_ccx_gate(0, 1, 3));
    KET_TRY("swap_range", c.add_swap_gate(0, 3));
    {
        auto e = ket::QuantumCircuit {2};
        KET_TRY("pop_empty", e.pop_back());
    }
    auto cc = ket::QuantumCircuit {5};
    cc.add_ccx_gate(0, 1, 2);
    cc.add_ccy_gate(4, 2, 0);
    cc.add_ccz_gate(1, 3, 4);
    cc.add_ccu_gate(ket::generate_random_unitary2x2(5), 2, 0, 4);
    cc.add_swap_gate(1, 3);
    cc.add_cswap_gate(0, 2, 4);
    cc.add_qft_gate({0, 1, 2, 3});
    cc.add_iqft_gate({4, 2, 1});
    cc.add_u_gate(ket::generate_random_unitary2x2(6), 1);
    cc.add_cu_gate(ket::generate_random_unitary2x2(7), 3, 2);
    show_circuit("ccirc", 0, cc);
    show_circuit("ctrans", 0, ket::transpile_to_primitive(cc));
    auto joined = ket::append_circuits(cc, cc);
    std::printf("joined %zu\n", joined.n_circuit_elements());
    cc.pop_back();
    std::printf("popped %zu\n", cc.n_circuit_elements());

    // classical register and control-flow predicates
    auto reg = ket::ClassicalRegister {3};
    reg.set(1, 1);
    reg.set(2, 0);
    std::printf("creg %d %d %d %d\n", static_cast<int>(reg.is_measured(0)), static_cast<int>(reg.is_measured(1)),
                reg.get(1), reg.get(2));
    KET_TRY("creg_get_unmeasured", (void)reg.get(0));
    // (no out-of-range register indices: the reference does not check them)
    KET_TRY("creg_set_value", reg.set(0, 2));
    using K = ket::ControlFlowBooleanKind;
    KET_TRY("pred_sizes", ket::ControlFlowPredicate({0, 1}, {1}, K::IF));
    KET_TRY("pred_bits", ket::ControlFlowPredicate({0}, {2}, K::IF));
    KET_TRY("pred_empty", ket::ControlFlowPredicate({}, {}, K::IF));
    {
        const auto p_if = ket::ControlFlowPredicate({1, 2}, {1, 0}, K::IF);
        const auto p_not = ket::ControlFlowPredicate({1, 2}, {1, 0}, K::IF_NOT);
        const auto p_other = ket::ControlFlowPredicate({1}, {0}, K::IF);
        std::printf("pred %d %d %d\n", static_cast<int>(p_if(reg)), static_cast<int>(p_not(reg)),
                    static_cast<int>(p_other(reg)));
        const auto p_unmeasured = ket::ControlFlowPredicate({0}, {1}, K::IF);
        KET_TRY("pred_unmeasured", (void)p_unmeasured(reg));
    }

    // 2x2 matrices
    int key = 0;
    for (int seed : {21, 22, 23}) {
        const auto u = ket::generate_random_unitary2x2(seed);
        const auto v = ket::generate_random_unitary2x2(seed + 100);
        show_matrix("mprod", key, u * v);
        show_matrix("msum", key, u + v);
        show_matrix("mscale", key, u * std::complex<double> {0.5, -1.25});
        show_matrix("mscale2", key, std::complex<double> {-2.0, 0.75} * v);
        show_matrix("mdag", key, ket::conjugate_transpose(u));
        show_matrix("msqrt", key, ket::matrix_square_root(u));
        const auto det = ket::determinant(u);
        const auto tr = ket::trace(u);
        std::printf("mdet %d %a %a %a %a %d %d\n", key, det.real(), det.imag(), tr.real(), tr.imag(),
                    static_cast<int>(ket::almost_eq(u, u)), static_cast<int>(ket::almost_eq(u, v)));
        auto w = u;
        w *= v;
        w += u;
        w *= 2.0;
        show_matrix("minplace", key, w);
        ++key;
    }
    for (const auto& g : {ket::x_gate(), ket::h_gate(), ket::z_gate(), ket::sx_gate(), ket::t_gate()}) {
        show_matrix("msqrt_fixed", key++, ket::matrix_square_root(g));
    }

    // Pauli strings and operators
    using P = ket::PauliTerm;
    auto sp = ket::SparsePauliString {4};
    sp.add(1, P::X);
    sp.add(3, P::Z);
    KET_TRY("pauli_add_twice", sp.add(1, P::Y));
    KET_TRY("pauli_add_range", sp.add(4, P::Y));
    KET_TRY("pauli_at_missing", (void)sp.at(2));
    sp.overwrite(1, P::Y);
    sp.overwrite(0, P::Z);
    sp.remove(3);
    sp.remove(2);
    std::printf("pstr %zu %d %d %d %d\n", sp.size(), static_cast<int>(sp.at(1)), static_cast<int>(sp.at(0)),
                static_cast<int>(sp.contains_index(3)), static_cast<int>(sp.contains_index(0)));
    KET_TRY("pauli_zero_qubits", ket::SparsePauliString {0});
    auto op = ket::PauliOperator {4};
    op.add({{0.5, -0.25}, sp});
    KET_TRY("pauliop_qubits", op.add({{1.0, 0.0}, ket::SparsePauliString {3}}));
    std::printf("pop %zu %zu\n", op.size(), op.n_qubits());

    // readout noise
    auto nz = ket::QuantumNoise {3};
    nz.set(1, 0.25);
    std::printf("noise %a %a\n", nz.get(0), nz.get(1));
    KET_TRY("noise_value", nz.set(1, 1.5));
    KET_TRY("noise_negative", nz.set(1, -0.1));
    KET_TRY("noise_range", nz.set(5, 0.1));
    KET_TRY("noise_get_range", (void)nz.get(7));

    // circuit comparison (loggers skipped, primitive gates against U gates of
    // their matrices, bound angles, M gates, control flow) and predicate order
    {
        auto a = ket::QuantumCircuit {3};
        a.add_x_gate(0);
        a.add_rx_gate(1, 0.75);
        a.add_cp_gate(2, 0, -1.25);
        a.add_m_gate(1);
        auto b = ket::QuantumCircuit {3};
        b.add_classical_register_circuit_logger();
        b.add_u_gate(ket::x_gate(), 0);
        b.add_u_gate(ket::rx_gate(0.75), 1);
        b.add_statevector_circuit_logger();
        b.add_cu_gate(ket::p_gate(-1.25), 2, 0);
        b.add_m_gate(1);
        b.add_classical_register_circuit_logger();
        auto c = ket::QuantumCircuit {3};
        c.add_x_gate(0);
        const auto id = c.add_rx_gate(1, 0.1, ket::param::parameterized {});
        c.add_cp_gate(2, 0, -1.25);
        c.add_m_gate(1);
        auto d = a;
        d.add_h_gate(2);
        auto e = ket::QuantumCircuit {3};
        e.add_rx_gate(1, 0.75);
        e.add_x_gate(0);
        e.add_cp_gate(2, 0, -1.25);
        e.add_m_gate(1);
        auto f = ket::QuantumCircuit {3};
        f.add_x_gate(0);
        f.add_rx_gate(1, 0.75);
        f.add_cp_gate(0, 2, -1.25);
        f.add_m_gate(1, 2);
        auto g = ket::QuantumCircuit {3, 5};
        g.add_x_gate(0);
        KET_TRY("cmp_unset_param", (void)ket::almost_eq(a, c));
        c.set_parameter_value(id, 0.75);
        auto sub0 = ket::QuantumCircuit {3};
        sub0.add_h_gate(1);
        auto sub1 = ket::QuantumCircuit {3};
        sub1.add_u_gate(ket::h_gate(), 1);
        auto cf0 = a;
        cf0.add_if_statement(1, sub0);
        auto cf1 = a;
        cf1.add_if_statement(1, sub1);
        auto cf2 = a;
        cf2.add_if_not_statement(1, sub1);
        auto cf3 = a;
        cf3.add_if_else_statement(1, sub0, sub1);
        auto cf4 = a;
        cf4.add_if_else_statement(1, sub1, sub0);
        const ket::QuantumCircuit* all[] = {&a, &b, &c, &d, &e, &f, &g, &cf0, &cf1, &cf2, &cf3, &cf4};
        constexpr int n_all = 12;
        for (int i = 0; i < n_all; ++i) {
            std::printf("ceq %d", i);
            for (int j = 0; j < n_all; ++j) {
                std::printf(" %d", static_cast<int>(ket::almost_eq(*all[i], *all[j])));
            }
            std::printf("\n");
        }
        auto near = ket::QuantumCircuit {1};
        near.add_rx_gate(0, 0.5 + 1.0e-9);
        auto far = ket::QuantumCircuit {1};
        far.add_rx_gate(0, 0.5 + 1.0e-3);
        auto base = ket::QuantumCircuit {1};
        base.add_rx_gate(0, 0.5);
        std::printf("ctol %d %d %d\n", static_cast<int>(ket::almost_eq(base, near)),
                    static_cast<int>(ket::almost_eq(base, far)), static_cast<int>(ket::almost_eq(base, far, 1.0e-4)));
        using K = ket::ControlFlowBooleanKind;
        const ket::ControlFlowPredicate preds[] = {
            ket::ControlFlowPredicate({0, 1}, {1, 0}, K::IF), ket::ControlFlowPredicate({0, 1}, {1, 0}, K::IF_NOT),
            ket::ControlFlowPredicate({0, 2}, {1, 0}, K::IF), ket::ControlFlowPredicate({0, 1}, {0, 1}, K::IF),
            ket::ControlFlowPredicate({0}, {1}, K::IF)};
        for (int i = 0; i < 5; ++i) {
            for (int j = 0; j < 5; ++j) {
                std::printf("predcmp %d %d %d %d %d\n", i, j, static_cast<int>(preds[i] == preds[j]),
                            static_cast<int>(preds[i] != preds[j]), static_cast<int>(preds[i] < preds[j]));
            }
        }
    }

    // measurement memory to counts and fractions
    const std::vector<std::size_t> memory = {3, 1, 3, 0, 7, 3, 1, 0, 0, 3};
    for (const auto& [k, v] : ket::memory_to_counts(memory)) {
        std::printf("mcount %zu %zu\n", k, v);
    }
    for (const auto& [k, v] : ket::memory_to_fractions(memory)) {
        std::printf("mfrac %zu %a\n", k, v);
    }
}

void show_state(const char* tag, int key, const ket::Statevector& s)
{
    for (std::size_t i = 0; i < s.n_states(); ++i) {
        std::printf("%s %d %zu %a %a\n", tag, key, i, s[i].real(), s[i].imag());
    }
}

void states_mode()
{
    int key = 0;
    for (std::size_t n = 1; n <= 6; ++n) {
        for (int seed : {1, 7, 2024}) {
            show_state("rstate", key++, ket::generate_random_state(n, seed));
        }
    }
    auto prng = std::mt19937 {99};
    const auto a = ket::generate_random_state(3, prng);
    const auto b = ket::generate_random_state(4, prng);  // continues the same stream
    show_state("rstream", 0, a);
    show_state("rstream", 1, b);
    try {
        (void)ket::generate_random_state(0, 3);
    } catch (const std::exception& e) {
        show_error("zero_qubits", e);
    }

    const auto psi = ket::generate_random_state(5, 11);
    struct Case
    {
        std::vector<std::size_t> qubits;
        std::vector<std::uint8_t> values;
    };
    const Case cases[] = {
        {{0}, {0}}, {{0}, {1}}, {{4}, {1}}, {{1, 3}, {1, 0}}, {{3, 1}, {0, 1}}, {{0, 2, 4}, {1, 1, 0}},
        {{4, 3, 2, 1}, {0, 1, 1, 0}}, {{2, 2}, {1, 1}},
    };
    key = 0;
    for (const auto& c : cases) {
        show_state("proj", key++, ket::project_statevector(psi, c.qubits, c.values));
    }
    // errors, each in the reference's order of checks
    const Case bad[] = {
        {{0, 1, 2, 3, 4}, {0, 0, 0, 0, 0}},  // every qubit
        {{5}, {0}},                           // out of range
        {{1}, {2}},                           // not a bit value
        {{1, 2}, {0}},                        // lengths differ
        {{2, 2}, {0, 1}},                     // contradictory: nothing left
    };
    for (const auto& c : bad) {
        try {
            (void)ket::project_statevector(psi, c.qubits, c.values);
            std::printf("noerr %d\n", key);
        } catch (const std::exception& e) {
            show_error("project", e);
        }
        ++key;
    }
    // a state with no weight where the projection looks: the norm check
    auto zero_one = ket::Statevector {"01"};
    try {
        (void)ket::project_statevector(zero_one, {1}, {0});
    } catch (const std::exception& e) {
        show_error("project_norm", e);
    }
    show_state("proj_basis", 0, ket::project_statevector(zero_one, {1}, {1}));

    // the text formats of io/: a random state saved in both endians (the
    // text itself compared), loaded back, read from numpy's complex text;
    // a Hamiltonian read from the "re im : (q, P)" text
    const auto io_state = ket::generate_random_state(4, 31);
    key = 0;
    for (const auto endian : {ket::Endian::LITTLE, ket::Endian::BIG}) {
        std::ostringstream text;
        ket::save_statevector(text, io_state, endian);
        std::istringstream lines {text.str()};
        std::string line;
        int k = 0;
        while (std::getline(lines, line)) {
            std::printf("svline %d %d [%s]\n", key, k++, line.c_str());
        }
        std::istringstream in {text.str()};
        show_state("svload", key, ket::load_statevector(in));
        ++key;
    }
    std::ostringstream np_text;
    np_text << 3 << '\n';
    char buf[96];
    const auto np_src = ket::generate_random_state(3, 32);
    for (std::size_t i = 0; i < np_src.n_states(); ++i) {
        const auto v = np_src[i];
        std::snprintf(buf, sizeof(buf), (i % 2 == 0) ? "(%.17g%+.17gj)\n" : "(%.8e%+.8ej)\n", v.real(), v.imag());
        np_text << buf;
    }
    for (const auto endian : {ket::Endian::LITTLE, ket::Endian::BIG}) {
        std::istringstream np_in {np_text.str()};
        show_state("npload", static_cast<int>(endian == ket::Endian::BIG), ket::read_numpy_statevector(np_in, endian));
    }
    std::istringstream ham_in {
        "0.5 -0.25 : (0, X) (2, Z)\n"
        "-1.125 0 : (1, Y)\n"
        "3.0e-2 1.5e-1 : (0, Z) (1, Z) (2, X)\n"
        "0.75 0.0 :\n"};
    try {
        const auto ham = ket::read_pauli_operator(ham_in, 3);
        int t = 0;
        for (const auto& ws : ham.weighted_pauli_strings()) {
            std::printf("ham %d %a %a %d", t++, ws.coefficient.real(), ws.coefficient.imag(),
                        static_cast<int>(ws.pauli_string.phase()));
            for (const auto& [q, term] : ws.pauli_string.terms()) {
                std::printf(" %zu:%d", q, static_cast<int>(term));
            }
            std::printf("\n");
        }
    } catch (const std::exception& e) {
        show_error("ham", e);
    }
}

}  // namespace

int main(int argc, char** argv)
{
    const std::string mode = argc > 1 ? argv[1] : "host";
    try {
        if (mode == "host") {
            host_mode();
        } else if (mode == "states") {
            states_mode();
        } else {
            std::fprintf(stderr, "usage: dropin_host host|states\n");
            return 2;
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "unexpected: %s\n", e.what());
        return 1;
    }
    return 0;
}
