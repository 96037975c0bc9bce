// ket_b200.cpp — host implementation of the ket:: drop-in API over the C-ABI.
#include "kettle/ket_b200.hpp"

#include <algorithm>
#include <cmath>
#include <iomanip>
#include <numeric>
#include <sstream>

namespace ket
{

namespace
{

void check(int32_t rc)
{
    if (rc != KT_OK) {
        throw std::runtime_error {std::string {kt_last_error()}};
    }
}

auto gate_name(Gate g) -> const char*
{
    static const char* names[] = {"H",   "X",   "Y",     "Z",  "S",     "SDAG", "T",     "TDAG", "SX",  "SXDAG", "RX",
                                  "RY",  "RZ",  "P",     "CH", "CX",    "CY",   "CZ",    "CS",   "CSDAG", "CT",
                                  "CTDAG", "CSX", "CSXDAG", "CRX", "CRY", "CRZ", "CP", "U", "CU", "M"};
    return names[static_cast<int>(g)];
}

bool is_controlled(Gate g)
{
    return (g >= Gate::CH && g <= Gate::CP) || g == Gate::CU;
}

bool is_power_of_2(std::size_t v)
{
    return v > 0 && (v & (v - 1)) == 0;
}

void check_bitstring(const std::string& s)
{
    if (s.empty() || !std::all_of(s.begin(), s.end(), [](char c) { return c == '0' || c == '1'; })) {
        throw std::runtime_error {"Received bitstring with inputs that aren't '0' or '1'\n"};
    }
}

auto to_record(const GateInfo& gi, const param::ParameterDataMap& pmap) -> kt_gate
{
    kt_gate r {};
    r.op = static_cast<uint8_t>(gi.gate);
    r.param = -1;
    if (gi.gate == Gate::M) {
        r.target = static_cast<uint32_t>(gi.arg0);
        r.control = static_cast<uint32_t>(gi.arg1);
        return r;
    }
    if (is_controlled(gi.gate)) {
        r.control = static_cast<uint32_t>(gi.arg0);
        r.target = static_cast<uint32_t>(gi.arg1);
    } else {
        r.target = static_cast<uint32_t>(gi.arg0);
    }
    r.angle = gi.arg2;
    if (gi.parameter) {
        const auto it = pmap.find(*gi.parameter);
        if (it == pmap.end() || !it->second.value) {
            throw std::runtime_error {"ERROR: cannot perform simulation with an uninitialized parameter value.\n"};
        }
        r.angle = *it->second.value;
    }
    if (gi.unitary_ptr) {
        const Matrix2X2& m = *gi.unitary_ptr;
        const std::complex<double> e[4] = {m.elem00, m.elem01, m.elem10, m.elem11};
        for (int i = 0; i < 4; ++i) {
            r.u[2 * i] = e[i].real();
            r.u[2 * i + 1] = e[i].imag();
        }
    }
    return r;
}

auto make_prng(std::optional<int> seed) -> std::mt19937
{
    // ket::internal::get_prng_ (common/prng.cpp:9-19)
    if (seed) {
        return std::mt19937 {static_cast<std::mt19937::result_type>(seed.value())};
    }
    auto device = std::random_device {};
    return std::mt19937 {device()};
}

}  // namespace

// ---- matrices ------------------------------------------------------------------------

auto conjugate_transpose(const Matrix2X2& m) -> Matrix2X2
{
    return {std::conj(m.elem00), std::conj(m.elem10), std::conj(m.elem01), std::conj(m.elem11)};
}

auto operator*(const Matrix2X2& a, const Matrix2X2& b) -> Matrix2X2
{
    return {a.elem00 * b.elem00 + a.elem01 * b.elem10, a.elem00 * b.elem01 + a.elem01 * b.elem11,
            a.elem10 * b.elem00 + a.elem11 * b.elem10, a.elem10 * b.elem01 + a.elem11 * b.elem11};
}

auto operator+(const Matrix2X2& a, const Matrix2X2& b) -> Matrix2X2
{
    return {a.elem00 + b.elem00, a.elem01 + b.elem01, a.elem10 + b.elem10, a.elem11 + b.elem11};
}

auto operator*(const Matrix2X2& a, std::complex<double> k) -> Matrix2X2
{
    return {a.elem00 * k, a.elem01 * k, a.elem10 * k, a.elem11 * k};
}

auto operator*(std::complex<double> k, const Matrix2X2& a) -> Matrix2X2
{
    return a * k;
}

auto determinant(const Matrix2X2& m) -> std::complex<double>
{
    return m.elem00 * m.elem11 - m.elem10 * m.elem01;
}

auto trace(const Matrix2X2& m) -> std::complex<double>
{
    return m.elem00 + m.elem11;
}

auto matrix_square_root(const Matrix2X2& m, double tolerance) -> Matrix2X2
{
    // sqrt(M) = (M + s I) / t with s = sqrt(det M), t = sqrt(tr M + 2 s); the
    // other sign of s where tr M + 2 s vanishes (within the tolerance)
    const auto tr = m.elem00 + m.elem11;
    const auto det = m.elem00 * m.elem11 - m.elem01 * m.elem10;
    auto s = std::sqrt(det);
    std::complex<double> t;
    if (std::norm(tr + 2.0 * s) > tolerance) {
        t = std::sqrt(tr + 2.0 * s);
    } else {
        t = std::sqrt(tr - 2.0 * s);
        s = -s;
    }
    return {(m.elem00 + s) / t, m.elem01 / t, m.elem10 / t, (m.elem11 + s) / t};
}

auto almost_eq(const std::complex<double>& l, const std::complex<double>& r, double tol_sq) noexcept -> bool
{
    const double dr = l.real() - r.real();
    const double di = l.imag() - r.imag();
    return (dr * dr + di * di) < tol_sq;
}

auto almost_eq(const Matrix2X2& l, const Matrix2X2& r, double tol_sq) noexcept -> bool
{
    return almost_eq(l.elem00, r.elem00, tol_sq) && almost_eq(l.elem01, r.elem01, tol_sq) &&
           almost_eq(l.elem10, r.elem10, tol_sq) && almost_eq(l.elem11, r.elem11, tol_sq);
}

namespace
{
constexpr double SQ12 = 0.70710678118654752440;
}

auto i_gate() noexcept -> Matrix2X2 { return {{1, 0}, {0, 0}, {0, 0}, {1, 0}}; }
auto h_gate() noexcept -> Matrix2X2 { return {{SQ12, 0}, {SQ12, 0}, {SQ12, 0}, {-SQ12, 0}}; }
auto x_gate() noexcept -> Matrix2X2 { return {{0, 0}, {1, 0}, {1, 0}, {0, 0}}; }
auto y_gate() noexcept -> Matrix2X2 { return {{0, 0}, {0, -1}, {0, 1}, {0, 0}}; }
auto z_gate() noexcept -> Matrix2X2 { return {{1, 0}, {0, 0}, {0, 0}, {-1, 0}}; }
auto s_gate() noexcept -> Matrix2X2 { return {{1, 0}, {0, 0}, {0, 0}, {0, 1}}; }
auto sdag_gate() noexcept -> Matrix2X2 { return {{1, 0}, {0, 0}, {0, 0}, {0, -1}}; }
auto t_gate() noexcept -> Matrix2X2 { return {{1, 0}, {0, 0}, {0, 0}, {SQ12, SQ12}}; }
auto tdag_gate() noexcept -> Matrix2X2 { return {{1, 0}, {0, 0}, {0, 0}, {SQ12, -SQ12}}; }
auto sx_gate() noexcept -> Matrix2X2 { return {{0.5, 0.5}, {0.5, -0.5}, {0.5, -0.5}, {0.5, 0.5}}; }
auto sxdag_gate() noexcept -> Matrix2X2 { return {{0.5, -0.5}, {0.5, 0.5}, {0.5, 0.5}, {0.5, -0.5}}; }
auto rx_gate(double a) noexcept -> Matrix2X2
{
    const double c = std::cos(a / 2.0), s = std::sin(a / 2.0);
    return {{c, 0}, {0, -s}, {0, -s}, {c, 0}};
}
auto ry_gate(double a) noexcept -> Matrix2X2
{
    const double c = std::cos(a / 2.0), s = std::sin(a / 2.0);
    return {{c, 0}, {-s, 0}, {s, 0}, {c, 0}};
}
auto rz_gate(double a) noexcept -> Matrix2X2
{
    const double c = std::cos(a / 2.0), s = std::sin(a / 2.0);
    return {{c, -s}, {0, 0}, {0, 0}, {c, s}};
}
auto p_gate(double a) noexcept -> Matrix2X2 { return {{1, 0}, {0, 0}, {0, 0}, {std::cos(a), std::sin(a)}}; }

auto non_angle_gate(Gate gate) -> Matrix2X2
{
    // gates/common_u_gates.cpp:172-207: a controlled gate maps to the matrix it controls
    switch (gate) {
    case Gate::H: case Gate::CH: return h_gate();
    case Gate::X: case Gate::CX: return x_gate();
    case Gate::Y: case Gate::CY: return y_gate();
    case Gate::Z: case Gate::CZ: return z_gate();
    case Gate::S: case Gate::CS: return s_gate();
    case Gate::SDAG: case Gate::CSDAG: return sdag_gate();
    case Gate::T: case Gate::CT: return t_gate();
    case Gate::TDAG: case Gate::CTDAG: return tdag_gate();
    case Gate::SX: case Gate::CSX: return sx_gate();
    case Gate::SXDAG: case Gate::CSXDAG: return sxdag_gate();
    default: throw std::runtime_error {"UNREACHABLE: dev error, invalid non-angle gate provided\n"};
    }
}

auto angle_gate(Gate gate, double angle) -> Matrix2X2
{
    // gates/common_u_gates.cpp:209-226
    switch (gate) {
    case Gate::RX: case Gate::CRX: return rx_gate(angle);
    case Gate::RY: case Gate::CRY: return ry_gate(angle);
    case Gate::RZ: case Gate::CRZ: return rz_gate(angle);
    case Gate::P: case Gate::CP: return p_gate(angle);
    default: throw std::runtime_error {"UNREACHABLE: dev error, invalid angle gate provided\n"};
    }
}

auto generate_random_unitary2x2(std::mt19937& prng) -> Matrix2X2
{
    // gates/random_u_gates.cpp:13-36: U = e^{i a} [[cos p e^{i f}, sin p e^{i c}], [-sin p e^{-i c}, cos p e^{-i f}]]
    // with a, f, c uniform in [0, 2 pi) and p = asin(sqrt(u)), u uniform in [0, 1)
    // (Haar measure on U(2)); the products and quotients are formed in the
    // reference's order so the matrices agree bit for bit
    auto unit = std::uniform_real_distribution<double> {0.0, 1.0};
    const double two_pi = 2.0 * M_PI;
    const double a = two_pi * unit(prng);
    const double f = two_pi * unit(prng);
    const double c = two_pi * unit(prng);
    const double p = std::asin(std::sqrt(unit(prng)));
    const std::complex<double> phase {std::cos(a), std::sin(a)};
    const std::complex<double> ef {std::cos(f), std::sin(f)};
    const std::complex<double> ec {std::cos(c), std::sin(c)};
    const double cp = std::cos(p);
    const double sp = std::sin(p);
    Matrix2X2 m;
    m.elem00 = phase * cp * ef;
    m.elem01 = phase * sp * ec;
    m.elem10 = -phase * sp / ec;
    m.elem11 = phase * cp / ef;
    return m;
}

auto generate_random_unitary2x2(int seed) -> Matrix2X2
{
    auto prng = make_prng(seed);
    return generate_random_unitary2x2(prng);
}

auto generate_random_unitary2x2() -> Matrix2X2
{
    auto prng = make_prng(std::nullopt);
    return generate_random_unitary2x2(prng);
}

// ---- parameters ----------------------------------------------------------------------

auto param::ParameterIdHash::operator()(const ParameterID& id) const noexcept -> std::size_t
{
    std::size_t out = 0;
    for (const auto byte : id) {
        out = (out * 31) ^ byte;
    }
    return out;
}

// ---- circuit ---------------------------------------------------------------------------

QuantumCircuit::QuantumCircuit(std::size_t n_qubits, std::size_t n_bits)
    : n_qubits_ {n_qubits}
    , n_bits_ {n_bits}
{}

QuantumCircuit::QuantumCircuit(std::size_t n_qubits)
    : n_qubits_ {n_qubits}
    , n_bits_ {n_qubits}
{}

void QuantumCircuit::pop_back()
{
    if (elements_.empty()) {
        throw std::runtime_error {"ERROR: called `pop_back()` on a `QuantumCircuit` instance with no circuit elements.\n"};
    }
    elements_.pop_back();
}

// ---- control flow and loggers (circuit.cpp:905-1000, control_flow_predicate.cpp:13-69) ------------

ControlFlowPredicate::ControlFlowPredicate(std::vector<std::size_t> bit_indices_to_check, std::vector<int> expected_bits,
                                           ControlFlowBooleanKind control_kind)
    : bit_indices_to_check_ {std::move(bit_indices_to_check)}
    , expected_bits_ {std::move(expected_bits)}
    , control_kind_ {control_kind}
{
    if (bit_indices_to_check_.size() != expected_bits_.size()) {
        std::ostringstream err;
        err << "There is a mismatch in the number of bits to check, and the number of expected bits:\n";
        err << "bit_indices_to_check.size() = " << bit_indices_to_check_.size() << '\n';
        err << "expected_bits.size() = " << expected_bits_.size() << '\n';
        throw std::runtime_error {err.str()};
    }
    if (bit_indices_to_check_.empty()) {
        throw std::runtime_error {"The control flow predicate must depend on at least one bit.\n"};
    }
    for (int b : expected_bits_) {
        if (b != 0 && b != 1) {
            throw std::runtime_error {"The expected bits must all be 0 or 1.\n"};
        }
    }
}

auto ControlFlowPredicate::operator()(const ClassicalRegister& creg) const -> bool
{
    bool all_match = true;
    for (std::size_t i = 0; i < bit_indices_to_check_.size(); ++i) {
        const auto bit_index = bit_indices_to_check_[i];
        if (!creg.is_measured(bit_index)) {
            std::ostringstream err;
            err << "There is no measured bit at classical register " << bit_index << '\n';
            throw std::runtime_error {err.str()};
        }
        if (creg.get(bit_index) != expected_bits_[i]) {
            all_match = false;
            break;
        }
    }
    return (control_kind_ == ControlFlowBooleanKind::IF) ? all_match : !all_match;
}

void ClassicalRegisterCircuitLogger::add_classical_register(ClassicalRegister cregister)
{
    cregister_ = std::make_shared<const ClassicalRegister>(std::move(cregister));
}

auto ClassicalRegisterCircuitLogger::classical_register() const -> const ClassicalRegister&
{
    if (!cregister_) {
        throw std::runtime_error {"ERROR: Cannot access classical register; it is not in the logger\n"};
    }
    return *cregister_;
}

void StatevectorCircuitLogger::add_statevector(Statevector statevector)
{
    statevector_ = std::make_shared<const Statevector>(std::move(statevector));
}

auto StatevectorCircuitLogger::statevector() const -> const Statevector&
{
    if (!statevector_) {
        throw std::runtime_error {"ERROR: Cannot access statevector; it is not in the logger\n"};
    }
    return *statevector_;
}

void DensityMatrixCircuitLogger::add_density_matrix(DensityMatrix density_matrix)
{
    density_matrix_ = std::make_shared<const DensityMatrix>(std::move(density_matrix));
}

auto DensityMatrixCircuitLogger::density_matrix() const -> const DensityMatrix&
{
    if (!density_matrix_) {
        throw std::runtime_error {"ERROR: Cannot access density matrix; it is not in the logger\n"};
    }
    return *density_matrix_;
}

void QuantumCircuit::add_if_statement(ControlFlowPredicate predicate, QuantumCircuit circuit, double tolerance)
{
    for (auto bit_index : predicate.bit_indices_to_check()) {
        check_bit_range_(bit_index);
    }
    merge_subcircuit_parameters_(circuit, tolerance);
    elements_.emplace_back(ClassicalIfStatement {std::move(predicate), std::make_shared<const QuantumCircuit>(std::move(circuit))});
}

void QuantumCircuit::add_if_statement(std::size_t bit_index, QuantumCircuit subcircuit)
{
    add_if_statement(ControlFlowPredicate {{bit_index}, {1}, ControlFlowBooleanKind::IF}, std::move(subcircuit));
}

void QuantumCircuit::add_if_not_statement(std::size_t bit_index, QuantumCircuit subcircuit)
{
    add_if_statement(ControlFlowPredicate {{bit_index}, {0}, ControlFlowBooleanKind::IF}, std::move(subcircuit));
}

void QuantumCircuit::add_if_else_statement(ControlFlowPredicate predicate, QuantumCircuit if_subcircuit,
                                           QuantumCircuit else_subcircuit)
{
    // as in the reference, the branches' parameters are not merged into this circuit's
    for (auto bit_index : predicate.bit_indices_to_check()) {
        check_bit_range_(bit_index);
    }
    elements_.emplace_back(ClassicalIfElseStatement {std::move(predicate),
                                                     std::make_shared<const QuantumCircuit>(std::move(if_subcircuit)),
                                                     std::make_shared<const QuantumCircuit>(std::move(else_subcircuit))});
}

void QuantumCircuit::add_if_else_statement(std::size_t bit_index, QuantumCircuit if_subcircuit, QuantumCircuit else_subcircuit)
{
    add_if_else_statement(ControlFlowPredicate {{bit_index}, {1}, ControlFlowBooleanKind::IF}, std::move(if_subcircuit),
                          std::move(else_subcircuit));
}

void QuantumCircuit::add_if_not_else_statement(std::size_t bit_index, QuantumCircuit if_subcircuit,
                                               QuantumCircuit else_subcircuit)
{
    add_if_else_statement(ControlFlowPredicate {{bit_index}, {0}, ControlFlowBooleanKind::IF}, std::move(if_subcircuit),
                          std::move(else_subcircuit));
}

void QuantumCircuit::add_classical_register_circuit_logger()
{
    elements_.emplace_back(ClassicalRegisterCircuitLogger {});
}

void QuantumCircuit::add_statevector_circuit_logger()
{
    elements_.emplace_back(StatevectorCircuitLogger {});
}

void QuantumCircuit::add_circuit_logger(CircuitLogger circuit_logger)
{
    elements_.emplace_back(std::move(circuit_logger));
}

// circuit.cpp:1158-1197: parameters of an if-statement's sub-circuit join this circuit's
void QuantumCircuit::merge_subcircuit_parameters_(const QuantumCircuit& subcircuit, double tolerance)
{
    for (const auto& [id, sub_data] : subcircuit.parameter_data_) {
        const auto [it, inserted] = parameter_data_.insert({id, sub_data});
        if (inserted) {
            continue;
        }
        auto& cur = it->second;
        cur.count += sub_data.count;
        if (!cur.value && sub_data.value) {
            cur.value = sub_data.value;
            continue;
        }
        if (cur.value && sub_data.value && std::fabs(*cur.value - *sub_data.value) > tolerance) {
            throw std::runtime_error {"ERROR: found two parameter instances with same id but different non-optional values\n"};
        }
    }
}

void QuantumCircuit::set_parameter_value(const param::ParameterID& id, double angle)
{
    if (!parameter_data_.contains(id)) {
        throw std::out_of_range {"ERROR: no parameter found with the provided id.\n"};
    }
    parameter_data_[id].value = angle;
}

void QuantumCircuit::check_qubit_range_(std::size_t index, const char* qubit_name, const char* gate_name_s) const
{
    // circuit/circuit.cpp check_qubit_range_
    if (index >= n_qubits_) {
        std::stringstream err;
        err << "The index for the " << qubit_name << " at which the '" << gate_name_s << "' gate is applied, is out of bounds.\n";
        err << "n_qubits             = " << n_qubits_ << '\n';
        err << "provided qubit index = " << index << '\n';
        throw std::runtime_error {err.str()};
    }
}

void QuantumCircuit::check_bit_range_(std::size_t bit_index) const
{
    if (bit_index >= n_bits_) {
        std::stringstream err;
        err << "The bit index at which the 'M' gate is applied, is out of bounds.\n";
        err << "n_bits             = " << n_bits_ << '\n';
        err << "provided bit index = " << bit_index << '\n';
        throw std::runtime_error {err.str()};
    }
}

auto QuantumCircuit::new_parameter_(std::optional<double> value) -> param::ParameterID
{
    // a fresh random 16-byte id (parameter/parameter.cpp, parameter_internal.hpp)
    auto prng = make_prng(std::nullopt);
    auto dist = std::uniform_int_distribution<int> {0, 255};
    param::ParameterID id {};
    for (auto& b : id) {
        b = static_cast<std::uint8_t>(dist(prng));
    }
    std::stringstream name;
    name << "theta" << parameter_count_++;
    parameter_data_[id] = param::ParameterData {.value = value, .name = name.str(), .count = 1};
    return id;
}

void QuantumCircuit::use_parameter_(const param::ParameterID& id)
{
    auto it = parameter_data_.find(id);
    if (it != parameter_data_.end()) {
        ++it->second.count;
        return;
    }
    std::stringstream name;
    name << "theta" << parameter_count_++;
    parameter_data_[id] = param::ParameterData {.value = std::nullopt, .name = name.str(), .count = 1};
}

void QuantumCircuit::add_one_(Gate g, std::size_t target)
{
    check_qubit_range_(target, "qubit", gate_name(g));
    elements_.push_back(GateInfo {g, target, 0, 0.0, std::nullopt, std::nullopt});
}

void QuantumCircuit::add_one_angle_(Gate g, std::size_t target, double angle)
{
    check_qubit_range_(target, "qubit", gate_name(g));
    elements_.push_back(GateInfo {g, target, 0, angle, std::nullopt, std::nullopt});
}

auto QuantumCircuit::add_one_param_(Gate g, std::size_t target, double angle) -> param::ParameterID
{
    check_qubit_range_(target, "qubit", gate_name(g));
    const auto id = new_parameter_(angle);
    elements_.push_back(GateInfo {g, target, 0, 0.0, std::nullopt, id});
    return id;
}

void QuantumCircuit::add_one_param_id_(Gate g, std::size_t target, const param::ParameterID& id)
{
    check_qubit_range_(target, "qubit", gate_name(g));
    use_parameter_(id);
    elements_.push_back(GateInfo {g, target, 0, 0.0, std::nullopt, id});
}

void QuantumCircuit::add_ctrl_(Gate g, std::size_t control, std::size_t target)
{
    check_qubit_range_(control, "control qubit", gate_name(g));
    check_qubit_range_(target, "target qubit", gate_name(g));
    elements_.push_back(GateInfo {g, control, target, 0.0, std::nullopt, std::nullopt});
}

void QuantumCircuit::add_ctrl_angle_(Gate g, std::size_t control, std::size_t target, double angle)
{
    check_qubit_range_(control, "control qubit", gate_name(g));
    check_qubit_range_(target, "target qubit", gate_name(g));
    elements_.push_back(GateInfo {g, control, target, angle, std::nullopt, std::nullopt});
}

auto QuantumCircuit::add_ctrl_param_(Gate g, std::size_t control, std::size_t target, double angle) -> param::ParameterID
{
    check_qubit_range_(control, "control qubit", gate_name(g));
    check_qubit_range_(target, "target qubit", gate_name(g));
    const auto id = new_parameter_(angle);
    elements_.push_back(GateInfo {g, control, target, 0.0, std::nullopt, id});
    return id;
}

void QuantumCircuit::add_ctrl_param_id_(Gate g, std::size_t control, std::size_t target, const param::ParameterID& id)
{
    check_qubit_range_(control, "control qubit", gate_name(g));
    check_qubit_range_(target, "target qubit", gate_name(g));
    use_parameter_(id);
    elements_.push_back(GateInfo {g, control, target, 0.0, std::nullopt, id});
}

#define KET_DEF_ONE(name, G)                                                    \
    void QuantumCircuit::add_##name##_gate(std::size_t t) { add_one_(Gate::G, t); } \
    void QuantumCircuit::add_##name##_gate(const std::vector<std::size_t>& idx) \
    {                                                                           \
        for (auto t : idx) add_one_(Gate::G, t);                                \
    }
KET_DEF_ONE(h, H)
KET_DEF_ONE(x, X)
KET_DEF_ONE(y, Y)
KET_DEF_ONE(z, Z)
KET_DEF_ONE(s, S)
KET_DEF_ONE(sdag, SDAG)
KET_DEF_ONE(t, T)
KET_DEF_ONE(tdag, TDAG)
KET_DEF_ONE(sx, SX)
KET_DEF_ONE(sxdag, SXDAG)
#undef KET_DEF_ONE

#define KET_DEF_ANGLE(name, G)                                                                              \
    void QuantumCircuit::add_##name##_gate(std::size_t t, double a) { add_one_angle_(Gate::G, t, a); }     \
    auto QuantumCircuit::add_##name##_gate(std::size_t t, double a, param::parameterized) -> param::ParameterID \
    {                                                                                                       \
        return add_one_param_(Gate::G, t, a);                                                               \
    }                                                                                                       \
    void QuantumCircuit::add_##name##_gate(std::size_t t, const param::ParameterID& id)                    \
    {                                                                                                       \
        add_one_param_id_(Gate::G, t, id);                                                                  \
    }                                                                                                       \
    void QuantumCircuit::add_##name##_gate(const std::vector<std::pair<std::size_t, double>>& pairs)       \
    {                                                                                                       \
        for (const auto& [t, a] : pairs) add_one_angle_(Gate::G, t, a);                                     \
    }
KET_DEF_ANGLE(rx, RX)
KET_DEF_ANGLE(ry, RY)
KET_DEF_ANGLE(rz, RZ)
KET_DEF_ANGLE(p, P)
#undef KET_DEF_ANGLE

#define KET_DEF_CTRL(name, G)                                                                          \
    void QuantumCircuit::add_##name##_gate(std::size_t c, std::size_t t) { add_ctrl_(Gate::G, c, t); } \
    void QuantumCircuit::add_##name##_gate(const std::vector<std::pair<std::size_t, std::size_t>>& ps) \
    {                                                                                                  \
        for (const auto& [c, t] : ps) add_ctrl_(Gate::G, c, t);                                        \
    }
KET_DEF_CTRL(ch, CH)
KET_DEF_CTRL(cx, CX)
KET_DEF_CTRL(cy, CY)
KET_DEF_CTRL(cz, CZ)
KET_DEF_CTRL(cs, CS)
KET_DEF_CTRL(csdag, CSDAG)
KET_DEF_CTRL(ct, CT)
KET_DEF_CTRL(ctdag, CTDAG)
KET_DEF_CTRL(csx, CSX)
KET_DEF_CTRL(csxdag, CSXDAG)
#undef KET_DEF_CTRL

#define KET_DEF_CTRL_ANGLE(name, G)                                                                                 \
    void QuantumCircuit::add_##name##_gate(std::size_t c, std::size_t t, double a) { add_ctrl_angle_(Gate::G, c, t, a); } \
    auto QuantumCircuit::add_##name##_gate(std::size_t c, std::size_t t, double a, param::parameterized)            \
        -> param::ParameterID                                                                                       \
    {                                                                                                               \
        return add_ctrl_param_(Gate::G, c, t, a);                                                                   \
    }                                                                                                               \
    void QuantumCircuit::add_##name##_gate(std::size_t c, std::size_t t, const param::ParameterID& id)             \
    {                                                                                                               \
        add_ctrl_param_id_(Gate::G, c, t, id);                                                                      \
    }                                                                                                               \
    void QuantumCircuit::add_##name##_gate(const std::vector<std::tuple<std::size_t, std::size_t, double>>& ts)    \
    {                                                                                                               \
        for (const auto& [c, t, a] : ts) add_ctrl_angle_(Gate::G, c, t, a);                                         \
    }
KET_DEF_CTRL_ANGLE(crx, CRX)
KET_DEF_CTRL_ANGLE(cry, CRY)
KET_DEF_CTRL_ANGLE(crz, CRZ)
KET_DEF_CTRL_ANGLE(cp, CP)
#undef KET_DEF_CTRL_ANGLE

void QuantumCircuit::add_u_gate(const Matrix2X2& gate, std::size_t target)
{
    check_qubit_range_(target, "qubit", "U");
    elements_.push_back(GateInfo {Gate::U, target, 0, 0.0, gate, std::nullopt});
}

void QuantumCircuit::add_u_gate(const Matrix2X2& gate, const std::vector<std::size_t>& indices)
{
    for (auto t : indices) {
        add_u_gate(gate, t);
    }
}

void QuantumCircuit::add_cu_gate(const Matrix2X2& gate, std::size_t control, std::size_t target)
{
    check_qubit_range_(control, "control qubit", "CU");
    check_qubit_range_(target, "target qubit", "CU");
    elements_.push_back(GateInfo {Gate::CU, control, target, 0.0, gate, std::nullopt});
}

void QuantumCircuit::add_cu_gate(const Matrix2X2& gate, const std::vector<std::pair<std::size_t, std::size_t>>& pairs)
{
    for (const auto& [c, t] : pairs) {
        add_cu_gate(gate, c, t);
    }
}

// ---- compound gates (circuit/circuit.cpp:723-900) ------------------------------------------

void QuantumCircuit::add_ccx_gate(std::size_t c0, std::size_t c1, std::size_t target)
{
    // sqrt(X) on the target under c1, c1 XOR c0, and c0: X exactly when both are set
    add_csx_gate(c1, target);
    add_cx_gate(c0, c1);
    add_cx_gate(c1, target);
    add_csx_gate(c1, target);
    add_cx_gate(c0, c1);
    add_csx_gate(c0, target);
}

void QuantumCircuit::add_ccx_gate(const Triplets& triplets)
{
    for (const auto& [c0, c1, t] : triplets) {
        add_ccx_gate(c0, c1, t);
    }
}

void QuantumCircuit::add_ccy_gate(std::size_t c0, std::size_t c1, std::size_t target)
{
    add_sdag_gate(target);
    add_ccx_gate(c0, c1, target);
    add_s_gate(target);
}

void QuantumCircuit::add_ccy_gate(const Triplets& triplets)
{
    for (const auto& [c0, c1, t] : triplets) {
        add_ccy_gate(c0, c1, t);
    }
}

void QuantumCircuit::add_ccz_gate(std::size_t c0, std::size_t c1, std::size_t target)
{
    add_h_gate(target);
    add_ccx_gate(c0, c1, target);
    add_h_gate(target);
}

void QuantumCircuit::add_ccz_gate(const Triplets& triplets)
{
    for (const auto& [c0, c1, t] : triplets) {
        add_ccz_gate(c0, c1, t);
    }
}

void QuantumCircuit::add_ccu_gate(const Matrix2X2& unitary, std::size_t c0, std::size_t c1, std::size_t target)
{
    const auto root = matrix_square_root(unitary);
    const auto root_adj = conjugate_transpose(root);
    add_cu_gate(root, c1, target);
    add_cx_gate(c0, c1);
    add_cu_gate(root_adj, c1, target);
    add_cx_gate(c0, c1);
    add_cu_gate(root, c0, target);
}

void QuantumCircuit::add_ccu_gate(const Matrix2X2& unitary, const Triplets& triplets)
{
    for (const auto& [c0, c1, t] : triplets) {
        add_ccu_gate(unitary, c0, c1, t);
    }
}

void QuantumCircuit::add_swap_gate(std::size_t t0, std::size_t t1)
{
    if (t0 == t1) {
        throw std::runtime_error {"Cannot swap a index with itself"};
    }
    add_cx_gate(t0, t1);
    add_cx_gate(t1, t0);
    add_cx_gate(t0, t1);
}

void QuantumCircuit::add_swap_gate(const std::vector<std::pair<std::size_t, std::size_t>>& target_index_pairs)
{
    for (const auto& [t0, t1] : target_index_pairs) {
        add_swap_gate(t0, t1);
    }
}

void QuantumCircuit::add_cswap_gate(std::size_t control, std::size_t t0, std::size_t t1)
{
    if (t0 == t1) {
        throw std::runtime_error {"Cannot swap a qubit with itself"};
    }
    if (control == t0 || control == t1) {
        throw std::runtime_error {"Cannot use the control qubit as one of the qubits to be swapped"};
    }
    add_cx_gate(t1, t0);
    add_ccx_gate(control, t0, t1);
    add_cx_gate(t1, t0);
}

void QuantumCircuit::add_cswap_gate(const Triplets& triplets)
{
    for (const auto& [c, t0, t1] : triplets) {
        add_cswap_gate(c, t0, t1);
    }
}

namespace
{

// reverse the order of `indices` with swaps, outermost pair first
void fourier_swaps(QuantumCircuit& circuit, const std::vector<std::size_t>& indices)
{
    if (indices.empty()) {
        return;
    }
    std::size_t left = 0;
    std::size_t right = indices.size() - 1;
    while (right > left) {
        circuit.add_swap_gate(indices[left], indices[right]);
        ++left;
        --right;
    }
}

}  // namespace

void QuantumCircuit::add_qft_gate(const std::vector<std::size_t>& indices)
{
    // H on each target, then CP(2 pi / 2^d) from every later index at distance d - 1
    const auto size = indices.size();
    for (std::size_t i = 0; i < size; ++i) {
        add_h_gate(indices[i]);
        std::size_t denom_bits = 2;
        for (std::size_t j = i + 1; j < size; ++j) {
            const double angle = 2.0 * M_PI / static_cast<double>(std::size_t {1} << denom_bits);
            add_cp_gate(indices[j], indices[i], angle);
            ++denom_bits;
        }
    }
    fourier_swaps(*this, indices);
}

void QuantumCircuit::add_iqft_gate(const std::vector<std::size_t>& indices)
{
    // the adjoint: the swaps, then the forward sequence reversed with negated angles
    fourier_swaps(*this, indices);
    const auto size = indices.size();
    for (std::size_t ii = size; ii-- > 0;) {
        std::size_t denom_bits = size - ii;
        for (std::size_t jj = size; jj-- > ii + 1;) {
            const double angle = 2.0 * M_PI / static_cast<double>(std::size_t {1} << denom_bits);
            add_cp_gate(indices[jj], indices[ii], -angle);
            --denom_bits;
        }
        add_h_gate(indices[ii]);
    }
}

void QuantumCircuit::add_m_gate(std::size_t target)
{
    add_m_gate(target, target);
}

void QuantumCircuit::add_m_gate(const std::vector<std::size_t>& indices)
{
    for (auto t : indices) {
        add_m_gate(t, t);
    }
}

void QuantumCircuit::add_m_gate(std::size_t target, std::size_t bit_index)
{
    check_qubit_range_(target, "qubit", "M");
    check_bit_range_(bit_index);
    elements_.push_back(GateInfo {Gate::M, target, bit_index, 0.0, std::nullopt, std::nullopt});
}

// ---- bitstrings -------------------------------------------------------------------------

auto endian_flip(std::size_t value, std::size_t n_relevant_bits) -> std::size_t
{
    std::size_t backward = 0;
    for (std::size_t i = 0; i < n_relevant_bits; ++i) {
        backward = (backward << 1U) | (value & 1U);
        value >>= 1U;
    }
    return backward;
}

auto bitstring_to_state_index(const std::string& bitstring, Endian input_endian) -> std::size_t
{
    // state/qubit_state_conversion.cpp:35-53: any string of '0' / '1', the empty one included
    if (!std::all_of(bitstring.begin(), bitstring.end(), [](char c) { return c == '0' || c == '1'; })) {
        check_bitstring(bitstring);
    }
    std::size_t big = 0;
    for (char c : bitstring) {
        big = (big << 1U) + (c == '1' ? 1U : 0U);
    }
    return input_endian == Endian::BIG ? big : endian_flip(big, bitstring.size());
}

auto state_index_to_bitstring(std::size_t i_state, std::size_t n_qubits, Endian endian) -> std::string
{
    const auto bits = state_index_to_dynamic_bitset(i_state, n_qubits, endian);
    return dynamic_bitset_to_bitstring(bits);
}

auto state_index_to_dynamic_bitset(std::size_t i_state, std::size_t n_qubits, Endian input_endian)
    -> std::vector<std::uint8_t>
{
    // state/qubit_state_conversion.cpp:55-81: qubit q is bit q of the index
    if (n_qubits < 64 && i_state >= (std::size_t {1} << n_qubits)) {
        throw std::runtime_error {"The state index exceeds the number of possible states."};
    }
    std::vector<std::uint8_t> bits(n_qubits, 0);
    for (std::size_t q = 0; q < n_qubits && q < 64; ++q) {
        const auto pos = input_endian == Endian::LITTLE ? q : n_qubits - 1 - q;
        bits[pos] = static_cast<std::uint8_t>((i_state >> q) & 1U);
    }
    return bits;
}

auto dynamic_bitset_to_bitstring(const std::vector<std::uint8_t>& bits) -> std::string
{
    std::string out;
    out.reserve(bits.size());
    for (auto b : bits) {
        out.push_back(b == 0 ? '0' : '1');
    }
    return out;
}

auto dynamic_bitset_to_state_index(const std::vector<std::uint8_t>& dyn_bitset, Endian input_endian) -> std::size_t
{
    return bitstring_to_state_index(dynamic_bitset_to_bitstring(dyn_bitset), input_endian);
}

auto bitstring_to_dynamic_bitset(const std::string& bitstring) -> std::vector<std::uint8_t>
{
    if (!std::all_of(bitstring.begin(), bitstring.end(), [](char c) { return c == '0' || c == '1'; })) {
        check_bitstring(bitstring);
    }
    std::vector<std::uint8_t> bits;
    bits.reserve(bitstring.size());
    for (char c : bitstring) {
        bits.push_back(c == '0' ? 0 : 1);
    }
    return bits;
}

auto bitstring_to_state_index_little_endian(const std::string& bitstring) -> std::size_t
{
    return bitstring_to_state_index(bitstring, Endian::LITTLE);
}

auto bitstring_to_state_index_big_endian(const std::string& bitstring) -> std::size_t
{
    return bitstring_to_state_index(bitstring, Endian::BIG);
}

auto state_index_to_bitstring_little_endian(std::size_t i_state, std::size_t n_qubits) -> std::string
{
    return state_index_to_bitstring(i_state, n_qubits, Endian::LITTLE);
}

auto state_index_to_bitstring_big_endian(std::size_t i_state, std::size_t n_qubits) -> std::string
{
    return state_index_to_bitstring(i_state, n_qubits, Endian::BIG);
}

auto state_index_to_dynamic_bitset_little_endian(std::size_t i_state, std::size_t n_qubits) -> std::vector<std::uint8_t>
{
    return state_index_to_dynamic_bitset(i_state, n_qubits, Endian::LITTLE);
}

auto state_index_to_dynamic_bitset_big_endian(std::size_t i_state, std::size_t n_qubits) -> std::vector<std::uint8_t>
{
    return state_index_to_dynamic_bitset(i_state, n_qubits, Endian::BIG);
}

auto dynamic_bitset_to_state_index_little_endian(const std::vector<std::uint8_t>& dyn_bitset) -> std::size_t
{
    return dynamic_bitset_to_state_index(dyn_bitset, Endian::LITTLE);
}

auto dynamic_bitset_to_state_index_big_endian(const std::vector<std::uint8_t>& dyn_bitset) -> std::size_t
{
    return dynamic_bitset_to_state_index(dyn_bitset, Endian::BIG);
}

auto binary_fraction_expansion(const std::string& bitstring, Endian endian) -> double
{
    // state/qubit_state_conversion.cpp:153-182: the digit read first has weight 1/2,
    // the next 1/4, ...; halving and adding in that order gives the same rounding
    if (!std::all_of(bitstring.begin(), bitstring.end(), [](char c) { return c == '0' || c == '1'; })) {
        check_bitstring(bitstring);
    }
    double value = 0.0;
    double weight = 1.0;
    const auto n = bitstring.size();
    for (std::size_t k = 0; k < n; ++k) {
        const char c = endian == Endian::LITTLE ? bitstring[k] : bitstring[n - 1 - k];
        weight *= 0.5;
        if (c == '1') {
            value += weight;
        }
    }
    return value;
}

namespace
{

// state/marginal.cpp:48-78: true when no '0' / '1' lies beyond the first
// marginal character, reading from the kept end towards the stripped one
bool marginals_only_at_end(const std::string& s, bool right_end)
{
    bool seen_marginal = false;
    const auto n = s.size();
    for (std::size_t k = 0; k < n; ++k) {
        const char c = right_end ? s[k] : s[n - 1 - k];
        if (c == 'x') {
            seen_marginal = true;
        } else if (seen_marginal) {
            return false;
        }
    }
    return true;
}

}  // namespace

auto rstrip_marginal_bits(const std::string& marginal_bitstring) -> std::string
{
    if (!marginals_only_at_end(marginal_bitstring, true)) {
        throw std::runtime_error {"The bitstring '" + marginal_bitstring + "' cannot be rstripped of its marginal bits\n"};
    }
    return marginal_bitstring.substr(0, std::min(marginal_bitstring.find('x'), marginal_bitstring.size()));
}

auto lstrip_marginal_bits(const std::string& marginal_bitstring) -> std::string
{
    if (!marginals_only_at_end(marginal_bitstring, false)) {
        throw std::runtime_error {"The bitstring '" + marginal_bitstring + "' cannot be lstripped of its marginal bits\n"};
    }
    const auto first_kept = marginal_bitstring.find_first_not_of('x');
    return first_kept == std::string::npos ? std::string {} : marginal_bitstring.substr(first_kept);
}

// ---- Statevector ------------------------------------------------------------------------------

Statevector::Statevector(std::size_t n_qubits, DType dtype)
    : n_qubits_ {n_qubits}
    , n_states_ {std::size_t {1} << n_qubits}
    , dtype_ {dtype}
{
    if (n_qubits_ == 0) {
        throw std::runtime_error {"There must be at least 1 qubit in the Statevector.\n"};
    }
    check(kt_sv_create(static_cast<int32_t>(n_qubits_), static_cast<int32_t>(dtype_), &handle_));
}

Statevector::Statevector(std::vector<std::complex<double>> coefficients, Endian input_endian,
                         double normalization_tolerance, DType dtype)
    : dtype_ {dtype}
{
    // state/state.cpp:30-118: size, power of two, normalisation, endianness
    if (coefficients.size() < 2) {
        throw std::runtime_error {"There must be at least 2 coefficients, representing the states for one qubit.\n"};
    }
    if (!is_power_of_2(coefficients.size())) {
        std::stringstream err;
        err << "The provided coefficients must have a size equal to a power of 2.\n";
        err << "Found size = " << coefficients.size();
        throw std::runtime_error {err.str()};
    }
    double sum = 0.0;
    for (const auto& c : coefficients) {
        sum += std::norm(c);
    }
    if (!(std::fabs(sum - 1.0) < normalization_tolerance)) {
        std::stringstream err;
        err << "The provided coefficients are not properly normalized.\n";
        err << "Found sum of squared norms : " << std::fixed << std::setprecision(14) << sum;
        throw std::runtime_error {err.str()};
    }
    n_states_ = coefficients.size();
    n_qubits_ = static_cast<std::size_t>(__builtin_ctzll(n_states_));
    if (input_endian == Endian::BIG) {
        for (std::size_t i = 0; i < n_states_; ++i) {
            const auto j = endian_flip(i, n_qubits_);
            if (i < j) {
                std::swap(coefficients[i], coefficients[j]);
            }
        }
    }
    check(kt_sv_create(static_cast<int32_t>(n_qubits_), static_cast<int32_t>(dtype_), &handle_));
    check(kt_sv_upload(handle_, reinterpret_cast<const double*>(coefficients.data()), n_states_));
    host_ = std::move(coefficients);
    host_valid_ = (dtype_ == DType::C128);
}

Statevector::Statevector(const std::string& computational_state, Endian input_endian, DType dtype)
    : n_qubits_ {computational_state.size()}
    , n_states_ {std::size_t {1} << computational_state.size()}
    , dtype_ {dtype}
{
    check_bitstring(computational_state);
    const auto index = bitstring_to_state_index(computational_state, input_endian);
    check(kt_sv_create(static_cast<int32_t>(n_qubits_), static_cast<int32_t>(dtype_), &handle_));
    check(kt_sv_set_basis(handle_, index));
}

Statevector::Statevector(const Statevector& other)
    : n_qubits_ {other.n_qubits_}
    , n_states_ {other.n_states_}
    , dtype_ {other.dtype_}
{
    check(kt_sv_create(static_cast<int32_t>(n_qubits_), static_cast<int32_t>(dtype_), &handle_));
    check(kt_sv_copy(handle_, other.device()));
    host_ = other.host_;
    host_valid_ = other.host_valid_;
}

Statevector::Statevector(Statevector&& other) noexcept
    : n_qubits_ {other.n_qubits_}
    , n_states_ {other.n_states_}
    , dtype_ {other.dtype_}
    , handle_ {other.handle_}
    , host_ {std::move(other.host_)}
    , host_valid_ {other.host_valid_}
    , host_dirty_ {other.host_dirty_}
{
    other.handle_ = nullptr;
}

auto Statevector::operator=(const Statevector& other) -> Statevector&
{
    if (this != &other) {
        Statevector tmp {other};
        *this = std::move(tmp);
    }
    return *this;
}

auto Statevector::operator=(Statevector&& other) noexcept -> Statevector&
{
    if (this != &other) {
        if (handle_ != nullptr) {
            kt_sv_destroy(handle_);
        }
        n_qubits_ = other.n_qubits_;
        n_states_ = other.n_states_;
        dtype_ = other.dtype_;
        handle_ = other.handle_;
        host_ = std::move(other.host_);
        host_valid_ = other.host_valid_;
        host_dirty_ = other.host_dirty_;
        other.handle_ = nullptr;
    }
    return *this;
}

Statevector::~Statevector()
{
    if (handle_ != nullptr) {
        kt_sv_destroy(handle_);
    }
}

void Statevector::pull_() const
{
    if (host_dirty_ || host_valid_) {
        return;
    }
    host_.resize(n_states_);
    check(kt_sv_download(handle_, reinterpret_cast<double*>(host_.data()), n_states_));
    host_valid_ = true;
}

auto Statevector::device() const -> kt_sv
{
    if (host_dirty_) {
        check(kt_sv_upload(handle_, reinterpret_cast<const double*>(host_.data()), n_states_));
        host_dirty_ = false;
        host_valid_ = (dtype_ == DType::C128);
    }
    return handle_;
}

void Statevector::mark_device_modified() const
{
    host_valid_ = false;
}

void Statevector::check_index_(std::size_t index) const
{
    if (index >= n_states_) {
        throw std::runtime_error {"Out-of-bounds access for the quantum state.\n"};
    }
}

auto Statevector::operator[](std::size_t index) const -> const std::complex<double>&
{
    pull_();
    return host_[index];
}

auto Statevector::operator[](std::size_t index) -> std::complex<double>&
{
    pull_();
    host_dirty_ = true;
    return host_[index];
}

auto Statevector::at(std::size_t index) const -> const std::complex<double>&
{
    check_index_(index);
    return (*this)[index];
}

auto Statevector::at(std::size_t index) -> std::complex<double>&
{
    check_index_(index);
    return (*this)[index];
}

auto Statevector::at(const std::string& bitstring, Endian endian) const -> const std::complex<double>&
{
    const auto i = bitstring_to_state_index(bitstring, endian);
    check_index_(i);
    return (*this)[i];
}

auto Statevector::at(const std::string& bitstring, Endian endian) -> std::complex<double>&
{
    const auto i = bitstring_to_state_index(bitstring, endian);
    check_index_(i);
    return (*this)[i];
}

auto almost_eq(const Statevector& left, const Statevector& right, double tolerance_sq) noexcept -> bool
{
    if (left.n_qubits() != right.n_qubits()) {
        return false;
    }
    for (std::size_t i = 0; i < left.n_states(); ++i) {
        if (!almost_eq(left[i], right[i], tolerance_sq)) {
            return false;
        }
    }
    return true;
}

auto inner_product(const Statevector& bra, const Statevector& ket_state) -> std::complex<double>
{
    if (bra.n_states() != ket_state.n_states()) {
        throw std::runtime_error {"ERROR: cannot calculate inner product between two states of different sizes.\n"};
    }
    double out[2];
    check(kt_sv_inner(bra.device(), ket_state.device(), out));
    return {out[0], out[1]};
}

auto inner_product_norm_squared(const Statevector& left, const Statevector& right) -> double
{
    return std::norm(inner_product(left, right));
}

auto tensor_product(const Statevector& left, const Statevector& right) -> Statevector
{
    // state/state.cpp:144-157: the product is built as a new Statevector from its
    // coefficients, whose constructor checks the normalisation
    if (left.dtype() != right.dtype()) {
        throw std::runtime_error {"ERROR: cannot take the tensor product of states of different precision.\n"};
    }
    Statevector out {left.n_qubits() + right.n_qubits(), left.dtype()};
    check(kt_sv_tensor_product(left.device(), right.device(), out.device()));
    out.mark_device_modified();
    double sum = 0.0;
    check(kt_sv_norm_sq(out.device(), &sum));
    if (!(std::fabs(sum - 1.0) < CONSTRUCTION_NORMALIZATION_TOLERANCE)) {
        std::stringstream err;
        err << "The provided coefficients are not properly normalized.\n";
        err << "Found sum of squared norms : " << std::fixed << std::setprecision(14) << sum;
        throw std::runtime_error {err.str()};
    }
    return out;
}

auto diagonal_expectation_value(const std::vector<std::complex<double>>& eigenvalues, const Statevector& state)
    -> std::complex<double>
{
    if (eigenvalues.size() != state.n_states()) {
        throw std::runtime_error {"ERROR: mismatch in sizes when taking expectation value of diagonal operator.\n"};
    }
    double out[2] = {0.0, 0.0};
    check(kt_sv_diagonal_expectation(state.device(), reinterpret_cast<const double*>(eigenvalues.data()), out));
    return {out[0], out[1]};
}

auto generate_random_state(std::size_t n_qubits, std::mt19937& prng) -> Statevector
{
    // state/random.cpp:19-58: every magnitude first, then one phase per amplitude
    if (n_qubits == 0) {
        throw std::runtime_error {"Cannot generate a quantum state with 0 qubits.\n"};
    }
    const std::size_t n_states = std::size_t {1} << n_qubits;
    auto draw_magnitude = std::uniform_real_distribution<double> {1.0e-3, 1.0e1};
    auto draw_phase = std::uniform_real_distribution<double> {0.0, 2.0 * M_PI};
    std::vector<double> mags(n_states);
    for (auto& m : mags) {
        m = draw_magnitude(prng);
    }
    double sum_sq = 0.0;  // summed in index order
    for (double m : mags) {
        sum_sq = sum_sq + m * m;
    }
    const double scale = 1.0 / std::sqrt(sum_sq);
    std::vector<std::complex<double>> amps(n_states);
    for (std::size_t i = 0; i < n_states; ++i) {
        const double phase = draw_phase(prng);
        const double r = scale * mags[i];
        amps[i] = {r * std::cos(phase), r * std::sin(phase)};
    }
    return Statevector {std::move(amps)};
}

auto generate_random_state(std::size_t n_qubits, int seed) -> Statevector
{
    auto prng = make_prng(seed);
    return generate_random_state(n_qubits, prng);
}

auto generate_random_state(std::size_t n_qubits) -> Statevector
{
    auto prng = make_prng(std::nullopt);
    return generate_random_state(n_qubits, prng);
}

auto project_statevector(const Statevector& statevector, const std::vector<std::size_t>& qubit_indices,
                         const std::vector<std::uint8_t>& expected_measurements, double minimum_norm_tol) -> Statevector
{
    // state/project_state.cpp:19-115, checks in the reference's order
    const auto n = statevector.n_qubits();
    if (qubit_indices.size() == n) {
        throw std::runtime_error {"ERROR: cannot collapse all qubits, remaining state won't exist.\n"};
    }
    if (!qubit_indices.empty() && *std::max_element(qubit_indices.begin(), qubit_indices.end()) >= n) {
        throw std::runtime_error {"ERROR: qubit indices exceed the number of qubits in the statevector.\n"};
    }
    if (!std::all_of(expected_measurements.begin(), expected_measurements.end(),
                     [](std::uint8_t v) { return v == 0 || v == 1; })) {
        throw std::runtime_error {"ERROR: all expected measurements must be 0 or 1.\n"};
    }
    if (qubit_indices.size() != expected_measurements.size()) {
        throw std::runtime_error {"ERROR: mismatch in number of qubit indices and number of expected measurements.\n"};
    }
    // the projected qubits as a mask and the value they must hold
    std::size_t mask = 0;
    std::size_t want = 0;
    bool contradictory = false;
    for (std::size_t k = 0; k < qubit_indices.size(); ++k) {
        const std::size_t bit = std::size_t {1} << qubit_indices[k];
        const std::size_t val = expected_measurements[k] ? bit : 0;
        if ((mask & bit) && (want & bit) != val) {
            contradictory = true;  // one qubit asked for both 0 and 1: nothing matches
        }
        mask |= bit;
        want |= val;
    }
    std::vector<std::complex<double>> kept;
    if (qubit_indices.size() < n) {
        kept.reserve(std::size_t {1} << (n - qubit_indices.size()));
    }
    if (!contradictory) {
        for (std::size_t i = 0; i < statevector.n_states(); ++i) {
            if ((i & mask) == want) {
                kept.push_back(statevector[i]);
            }
        }
    }
    double sum_sq = 0.0;
    for (const auto& a : kept) {
        sum_sq += std::norm(a);
    }
    const double root = std::sqrt(sum_sq);
    if (root < minimum_norm_tol) {
        throw std::runtime_error {"The state cannot be normalized; norm of remaining amplitudes is 0.0\n"};
    }
    const double inv = 1.0 / root;
    for (auto& a : kept) {
        a *= inv;
    }
    return Statevector {std::move(kept)};
}

// ---- DensityMatrix ------------------------------------------------------------------------------

DensityMatrix::DensityMatrix(HostMatrix matrix, const density_matrix_nocheck&, DType dtype)
    : n_states_ {static_cast<std::size_t>(matrix.cols())}
    , dtype_ {dtype}
{
    if (matrix.rows() != matrix.cols() || !is_power_of_2(n_states_) || n_states_ < 1) {
        throw std::runtime_error {"The provided coefficients must have a size equal to a power of 2.\n"};
    }
    n_qubits_ = static_cast<std::size_t>(__builtin_ctzll(n_states_));
    check(kt_dm_create(static_cast<int32_t>(n_qubits_), static_cast<int32_t>(dtype_), &handle_));
    check(kt_dm_upload(handle_, reinterpret_cast<const double*>(matrix.data()), n_states_ * n_states_));
    host_ = std::move(matrix);
    host_valid_ = (dtype_ == DType::C128);
}

DensityMatrix::DensityMatrix(const std::string& bitstring, Endian input_endian, DType dtype)
    : n_qubits_ {bitstring.size()}
    , n_states_ {std::size_t {1} << bitstring.size()}
    , dtype_ {dtype}
{
    const auto index = bitstring_to_state_index(bitstring, input_endian);
    check(kt_dm_create(static_cast<int32_t>(n_qubits_), static_cast<int32_t>(dtype_), &handle_));
    check(kt_dm_set_basis(handle_, index));
}

DensityMatrix::DensityMatrix(const DensityMatrix& other)
    : n_qubits_ {other.n_qubits_}
    , n_states_ {other.n_states_}
    , dtype_ {other.dtype_}
{
    other.pull_();
    check(kt_dm_create(static_cast<int32_t>(n_qubits_), static_cast<int32_t>(dtype_), &handle_));
    check(kt_dm_upload(handle_, reinterpret_cast<const double*>(other.host_.data()), n_states_ * n_states_));
    host_ = other.host_;
    host_valid_ = true;
}

DensityMatrix::DensityMatrix(DensityMatrix&& other) noexcept
    : n_qubits_ {other.n_qubits_}
    , n_states_ {other.n_states_}
    , dtype_ {other.dtype_}
    , handle_ {other.handle_}
    , host_ {std::move(other.host_)}
    , host_valid_ {other.host_valid_}
    , host_dirty_ {other.host_dirty_}
{
    other.handle_ = nullptr;
}

auto DensityMatrix::operator=(const DensityMatrix& other) -> DensityMatrix&
{
    if (this != &other) {
        DensityMatrix tmp {other};
        *this = std::move(tmp);
    }
    return *this;
}

auto DensityMatrix::operator=(DensityMatrix&& other) noexcept -> DensityMatrix&
{
    if (this != &other) {
        if (handle_ != nullptr) {
            kt_dm_destroy(handle_);
        }
        n_qubits_ = other.n_qubits_;
        n_states_ = other.n_states_;
        dtype_ = other.dtype_;
        handle_ = other.handle_;
        host_ = std::move(other.host_);
        host_valid_ = other.host_valid_;
        host_dirty_ = other.host_dirty_;
        other.handle_ = nullptr;
    }
    return *this;
}

DensityMatrix::~DensityMatrix()
{
    if (handle_ != nullptr) {
        kt_dm_destroy(handle_);
    }
}

void DensityMatrix::pull_() const
{
    if (host_dirty_ || host_valid_) {
        return;
    }
    const auto N = static_cast<std::ptrdiff_t>(n_states_);
    if (host_.rows() != N) {
        host_ = HostMatrix {N, N};
    }
    check(kt_dm_download(handle_, reinterpret_cast<double*>(host_.data()), n_states_ * n_states_));
    host_valid_ = true;
}

auto DensityMatrix::matrix() const -> const HostMatrix&
{
    pull_();
    return host_;
}

auto DensityMatrix::matrix() -> HostMatrix&
{
    pull_();
    host_dirty_ = true;
    return host_;
}

auto DensityMatrix::device() const -> kt_dm
{
    if (host_dirty_) {
        check(kt_dm_upload(handle_, reinterpret_cast<const double*>(host_.data()), n_states_ * n_states_));
        host_dirty_ = false;
        host_valid_ = (dtype_ == DType::C128);
    }
    return handle_;
}

void DensityMatrix::mark_device_modified() const
{
    host_valid_ = false;
}

auto DensityMatrix::trace() const -> std::complex<double>
{
    double out[2];
    check(kt_dm_trace(device(), out));
    return {out[0], out[1]};
}

DensityMatrix::DensityMatrix(kt_dm handle, std::size_t n_qubits, DType dtype)
    : n_qubits_ {n_qubits}
    , n_states_ {std::size_t {1} << n_qubits}
    , dtype_ {dtype}
    , handle_ {handle}
{}

auto DensityMatrix::trace_of_square() const -> std::complex<double>
{
    double out[2];
    check(kt_dm_trace_of_square(device(), out));
    return {out[0], out[1]};
}

auto DensityMatrix::is_pure(double tolerance) const -> bool
{
    return std::norm(trace_of_square() - std::complex<double> {1.0, 0.0}) <= tolerance;
}

auto tensor_product(const DensityMatrix& left, const DensityMatrix& right) -> DensityMatrix
{
    const auto n = left.n_qubits() + right.n_qubits();
    const auto dtype = (left.dtype_ == DType::C64 && right.dtype_ == DType::C64) ? DType::C64 : DType::C128;
    if (left.dtype_ != dtype || right.dtype_ != dtype) {
        // mixed storage: the complex64 factor is widened first
        const DensityMatrix wide_left = (left.dtype_ == dtype) ? left : DensityMatrix {left.matrix(), density_matrix_nocheck {}, dtype};
        const DensityMatrix wide_right = (right.dtype_ == dtype) ? right : DensityMatrix {right.matrix(), density_matrix_nocheck {}, dtype};
        return tensor_product(wide_left, wide_right);
    }
    kt_dm out = nullptr;
    check(kt_dm_create(static_cast<int32_t>(n), static_cast<int32_t>(dtype), &out));
    auto result = DensityMatrix {out, n, dtype};
    check(kt_dm_tensor_product(left.device(), right.device(), out));
    return result;
}

auto tensor_product(const std::vector<DensityMatrix>& density_matrices) -> DensityMatrix
{
    if (density_matrices.size() < 2) {
        throw std::runtime_error {"Cannot take tensor product of 0 or 1 matrices.\n"};
    }
    auto output = tensor_product(density_matrices[0], density_matrices[1]);
    for (std::size_t i = 2; i < density_matrices.size(); ++i) {
        output = tensor_product(output, density_matrices[i]);
    }
    return output;
}

auto partial_trace(const DensityMatrix& density_matrix, std::vector<std::size_t> qubit_indices) -> DensityMatrix
{
    // state/density_matrix.cpp:231-278: indices sorted high to low, each one an
    // index into the matrix left by the traces before it
    const auto n = density_matrix.n_qubits();
    const auto out_of_range = [n](std::size_t index) { return index >= n; };
    if (std::any_of(qubit_indices.begin(), qubit_indices.end(), out_of_range) || qubit_indices.size() > n) {
        throw std::runtime_error {"ERROR: Cannot take partial trace; found qubit index out of bounds\n"};
    }
    std::sort(qubit_indices.begin(), qubit_indices.end(), [](auto x, auto y) { return x > y; });
    std::vector<std::size_t> remaining(n);
    for (std::size_t q = 0; q < n; ++q) {
        remaining[q] = q;
    }
    std::vector<int32_t> traced;
    traced.reserve(qubit_indices.size());
    for (const auto position : qubit_indices) {
        if (position >= remaining.size()) {
            throw std::runtime_error {"ERROR: Cannot take partial trace; found qubit index out of bounds\n"};
        }
        traced.push_back(static_cast<int32_t>(remaining[position]));
        remaining.erase(remaining.begin() + static_cast<std::ptrdiff_t>(position));
    }
    const auto m = remaining.size();
    kt_dm out = nullptr;
    check(kt_dm_create(static_cast<int32_t>(m), static_cast<int32_t>(density_matrix.dtype_), &out));
    auto result = DensityMatrix {out, m, density_matrix.dtype_};
    check(kt_dm_partial_trace(density_matrix.device(), traced.data(), static_cast<int32_t>(traced.size()), out));
    return result;
}

auto statevector_to_density_matrix(const Statevector& sv) -> DensityMatrix
{
    // density_matrix.cpp:170-185: rho(i0, i1) = psi[i0] conj(psi[i1])
    const auto N = static_cast<std::ptrdiff_t>(sv.n_states());
    HostMatrix m {N, N};
    for (std::ptrdiff_t i0 = 0; i0 < N; ++i0) {
        for (std::ptrdiff_t i1 = 0; i1 < N; ++i1) {
            m(i0, i1) = sv[static_cast<std::size_t>(i0)] * std::conj(sv[static_cast<std::size_t>(i1)]);
        }
    }
    return DensityMatrix {std::move(m), density_matrix_nocheck {}, sv.dtype()};
}

// ---- simulation -------------------------------------------------------------------------------

namespace
{

void check_valid_number_of_qubits(std::size_t circuit_n, std::size_t state_n)
{
    // simulation/simulate.cpp:523-532
    if (circuit_n != state_n) {
        throw std::runtime_error {"Invalid simulation; circuit and state have different number of qubits."};
    }
    if (circuit_n == 0) {
        throw std::runtime_error {"Cannot simulate a circuit or state with zero qubits."};
    }
}

// The circuit as the reference's simulate loop walks it (simulate.cpp:418-507):
// a stack of element lists with instruction pointers, if / if-else statements
// evaluated against the classical register on the host, loggers taking
// snapshots.  Consecutive gates (across statement boundaries) are collected
// and handed to the engine as one fused apply; anything that needs the state
// (M, a logger) or the classical register (a predicate) flushes them first.
// Gate parameters come from the top circuit's parameter map, as in the reference.
template <typename ApplyFn, typename MeasureFn, typename LogFn>
void run_elements(const QuantumCircuit& circuit, const ClassicalRegister& creg, ApplyFn&& apply, MeasureFn&& measure,
                  LogFn&& log)
{
    const auto& pmap = circuit.parameter_data_map();
    std::vector<kt_gate> seg;
    auto flush = [&]() {
        if (!seg.empty()) {
            apply(seg);
            seg.clear();
        }
    };
    std::vector<const std::vector<CircuitElement>*> stack {&circuit.circuit_elements()};
    std::vector<std::size_t> ip {0};
    while (!stack.empty()) {
        const auto& elems = *stack.back();
        const std::size_t i = ip.back()++;
        if (i >= elems.size()) {
            stack.pop_back();
            ip.pop_back();
            continue;
        }
        const auto& el = elems[i];
        if (el.is_gate()) {
            const auto& gi = el.get_gate();
            if (gi.gate == Gate::M) {
                flush();
                measure(gi.arg0, gi.arg1);
            } else {
                seg.push_back(to_record(gi, pmap));
            }
        } else if (el.is_control_flow()) {
            flush();
            const auto& cf = el.get_control_flow();
            const QuantumCircuit* sub = nullptr;
            if (cf.is_if_statement()) {
                const auto& st = cf.get_if_statement();
                if (st(creg)) {
                    sub = st.circuit().get();
                }
            } else {
                const auto& st = cf.get_if_else_statement();
                sub = st(creg) ? st.if_circuit().get() : st.else_circuit().get();
            }
            if (sub != nullptr) {
                stack.push_back(&sub->circuit_elements());
                ip.push_back(0);
            }
        } else {
            flush();
            log(el.get_circuit_logger());
        }
    }
    flush();
}

}  // namespace

void StatevectorSimulator::run(const QuantumCircuit& circuit, Statevector& state, std::optional<int> prng_seed)
{
    check_valid_number_of_qubits(circuit.n_qubits(), state.n_qubits());
    cregister_.emplace(circuit.n_bits());
    circuit_loggers_.clear();
    kt_sv h = state.device();
    run_elements(
        circuit, *cregister_,
        [&](const std::vector<kt_gate>& seg) {
            check(kt_sv_apply(h, seg.data(), static_cast<int64_t>(seg.size()), nullptr, 0, KT_APPLY_FUSED));
        },
        [&](std::size_t qubit, std::size_t bit) {
            // measure.hpp:34-55: P(0), P(1); a fresh prng per M gate; discrete draw; collapse
            double p0 = 0.0, p1 = 0.0;
            check(kt_sv_measure_probs(h, static_cast<uint32_t>(qubit), &p0, &p1));
            auto prng = make_prng(prng_seed);
            auto coin = std::discrete_distribution<int> {{p0, p1}};
            const int outcome = coin(prng);
            const double norm = std::sqrt(1.0 / (outcome == 0 ? p0 : p1));
            check(kt_sv_collapse(h, static_cast<uint32_t>(qubit), outcome, norm));
            cregister_->set(bit, outcome);
        },
        [&](const CircuitLogger& logger) {
            if (logger.is_classical_register_circuit_logger()) {
                auto l = logger.get_classical_register_circuit_logger();
                l.add_classical_register(*cregister_);
                circuit_loggers_.emplace_back(std::move(l));
            } else if (logger.is_statevector_circuit_logger()) {
                state.mark_device_modified();
                auto l = logger.get_statevector_circuit_logger();
                l.add_statevector(state);
                circuit_loggers_.emplace_back(std::move(l));
            } else {
                throw std::runtime_error {"DEV ERROR: unimplemented circuit logger in `simulate_loop_body_iterative_()`\n"};
            }
        });
    state.mark_device_modified();
    has_been_run_ = true;
}

auto StatevectorSimulator::classical_register() const -> const ClassicalRegister&
{
    if (!cregister_) {
        throw std::runtime_error {"ERROR: Cannot access classical register; no simulation has been run\n"};
    }
    return *cregister_;
}

auto StatevectorSimulator::classical_register() -> ClassicalRegister&
{
    if (!cregister_) {
        throw std::runtime_error {"ERROR: Cannot access classical register; no simulation has been run\n"};
    }
    return *cregister_;
}

void DensityMatrixSimulator::run(const QuantumCircuit& circuit, DensityMatrix& state, std::optional<int> prng_seed)
{
    check_valid_number_of_qubits(circuit.n_qubits(), state.n_qubits());
    if (circuit.n_qubits() != n_qubits_) {
        throw std::runtime_error {"Invalid simulation; circuit and state have different number of qubits."};
    }
    cregister_.emplace(circuit.n_bits());
    kt_dm h = state.device();
    run_elements(
        circuit, *cregister_,
        [&](const std::vector<kt_gate>& seg) {
            check(kt_dm_apply(h, seg.data(), static_cast<int64_t>(seg.size()), nullptr, 0, KT_APPLY_FUSED));
        },
        [&](std::size_t qubit, std::size_t bit) {
            // simulation/measure_density_matrix.hpp:33-56: P(0), P(1); a fresh prng per
            // M gate; discrete draw; the surviving block scaled by sqrt(1 / P)
            double p0 = 0.0, p1 = 0.0;
            check(kt_dm_measure_probs(h, static_cast<uint32_t>(qubit), &p0, &p1));
            auto prng = make_prng(prng_seed);
            auto coin = std::discrete_distribution<int> {{p0, p1}};
            const int outcome = coin(prng);
            const double norm = std::sqrt(1.0 / (outcome == 0 ? p0 : p1));
            check(kt_dm_collapse(h, static_cast<uint32_t>(qubit), outcome, norm));
            cregister_->set(bit, outcome);
        },
        [&](const CircuitLogger&) {
            // simulate_density_matrix.cpp:391-392
            throw std::runtime_error {"DEV ERROR: loggers haven't been implemented yet for the density matrix simulator.\n"};
        });
    state.mark_device_modified();
    has_been_run_ = true;
}

auto DensityMatrixSimulator::classical_register() const -> const ClassicalRegister&
{
    if (!cregister_) {
        throw std::runtime_error {"ERROR: Cannot access classical register; no simulation has been run\n"};
    }
    return *cregister_;
}

void simulate(const QuantumCircuit& circuit, Statevector& state, std::optional<int> prng_seed)
{
    auto sim = StatevectorSimulator {};
    sim.run(circuit, state, prng_seed);
}

void simulate(const QuantumCircuit& circuit, DensityMatrix& state, std::optional<int> prng_seed)
{
    auto sim = DensityMatrixSimulator {state.n_qubits()};
    sim.run(circuit, state, prng_seed);
}

void StatevectorPauliStringSimulator::run(const SparsePauliString& pauli_string, Statevector& state)
{
    // simulation/simulate_pauli.cpp:91-122: the string's X / Y / Z gates in term
    // order, one fused apply; the string's phase is not applied
    if (pauli_string.n_qubits() != state.n_qubits()) {
        throw std::runtime_error {"Invalid simulation; SparsePauliString and state have different number of qubits."};
    }
    if (pauli_string.n_qubits() == 0) {
        throw std::runtime_error {"Cannot simulate a SparsePauliString or state with zero qubits."};
    }
    std::vector<kt_gate> gates;
    for (const auto& [q, t] : pauli_string.terms()) {
        kt_gate g {};
        g.param = -1;
        g.target = static_cast<uint32_t>(q);
        if (t == PauliTerm::X) {
            g.op = static_cast<uint8_t>(Gate::X);
        } else if (t == PauliTerm::Y) {
            g.op = static_cast<uint8_t>(Gate::Y);
        } else if (t == PauliTerm::Z) {
            g.op = static_cast<uint8_t>(Gate::Z);
        } else {
            continue;
        }
        gates.push_back(g);
    }
    if (!gates.empty()) {
        check(kt_sv_apply(state.device(), gates.data(), static_cast<int64_t>(gates.size()), nullptr, 0, KT_APPLY_FUSED));
        state.mark_device_modified();
    }
    has_been_run_ = true;
}

void simulate(const SparsePauliString& pauli_string, Statevector& state)
{
    auto simulator = StatevectorPauliStringSimulator {};
    simulator.run(pauli_string, state);
}

// ---- Pauli ---------------------------------------------------------------------------------------

const std::unordered_map<PauliPhase, std::complex<double>> PAULI_PHASE_MAP = {
    {PauliPhase::PLUS_ONE, {1.0, 0.0}},
    {PauliPhase::PLUS_EYE, {0.0, 1.0}},
    {PauliPhase::MINUS_ONE, {-1.0, 0.0}},
    {PauliPhase::MINUS_EYE, {0.0, -1.0}},
};

SparsePauliString::SparsePauliString(std::size_t n_qubits, PauliPhase phase)
    : n_qubits_ {n_qubits}
    , phase_ {phase}
{
    if (n_qubits_ == 0) {
        throw std::runtime_error {"ERROR: SparsePauliString cannot be constructed with 0 qubits.\n"};
    }
}

SparsePauliString::SparsePauliString(std::vector<std::pair<std::size_t, PauliTerm>> terms, std::size_t n_qubits,
                                     PauliPhase phase)
    : n_qubits_ {n_qubits}
    , phase_ {phase}
    , terms_ {std::move(terms)}
{
    if (n_qubits_ == 0) {
        throw std::runtime_error {"ERROR: SparsePauliString cannot be constructed with 0 qubits.\n"};
    }
}

SparsePauliString::SparsePauliString(const std::vector<PauliTerm>& pauli_terms, PauliPhase phase)
    : n_qubits_ {pauli_terms.size()}
    , phase_ {phase}
{
    if (n_qubits_ == 0) {
        throw std::runtime_error {"ERROR: SparsePauliString cannot be constructed with 0 qubits.\n"};
    }
    for (std::size_t i = 0; i < pauli_terms.size(); ++i) {
        terms_.emplace_back(i, pauli_terms[i]);
    }
}

SparsePauliString::SparsePauliString(const std::initializer_list<PauliTerm>& pauli_terms, PauliPhase phase)
    : SparsePauliString {std::vector<PauliTerm> {pauli_terms}, phase}
{}

auto SparsePauliString::at(std::size_t qubit_index) const -> PauliTerm
{
    for (const auto& [q, t] : terms_) {
        if (q == qubit_index && qubit_index < n_qubits_) {
            return t;
        }
    }
    throw std::runtime_error {"ERROR: no Pauli term found for provided qubit index.\n"};
}

void SparsePauliString::add(std::size_t qubit_index, PauliTerm term)
{
    if (qubit_index >= n_qubits_) {
        throw std::runtime_error {"ERROR: cannot perform operation on SparsePauliString with index beyond qubit range.\n"};
    }
    if (contains_index(qubit_index)) {
        throw std::runtime_error {"ERROR: Pauli term is already present in the string\n"};
    }
    terms_.emplace_back(qubit_index, term);
}

void SparsePauliString::overwrite(std::size_t qubit_index, PauliTerm term)
{
    if (qubit_index >= n_qubits_) {
        throw std::runtime_error {"ERROR: cannot perform operation on SparsePauliString with index beyond qubit range.\n"};
    }
    for (auto& [q, t] : terms_) {
        if (q == qubit_index) {
            t = term;
            return;
        }
    }
    terms_.emplace_back(qubit_index, term);
}

void SparsePauliString::remove(std::size_t qubit_index)
{
    for (auto it = terms_.begin(); it != terms_.end(); ++it) {
        if (it->first == qubit_index) {
            terms_.erase(it);
            return;
        }
    }
}

auto SparsePauliString::contains_index(std::size_t qubit_index) const noexcept -> bool
{
    return std::any_of(terms_.begin(), terms_.end(), [&](const auto& p) { return p.first == qubit_index; });
}

auto SparsePauliString::equal_up_to_phase(const SparsePauliString& other) const -> bool
{
    // sparse_pauli_string.cpp:165-179: identity terms do not count, and the
    // order the terms were added in does not matter
    if (n_qubits_ != other.n_qubits_) {
        return false;
    }
    const auto canonical = [](const std::vector<std::pair<std::size_t, PauliTerm>>& terms) {
        std::vector<std::pair<std::size_t, PauliTerm>> out;
        for (const auto& t : terms) {
            if (t.second != PauliTerm::I) {
                out.push_back(t);
            }
        }
        std::stable_sort(out.begin(), out.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        return out;
    };
    return canonical(terms_) == canonical(other.terms_);
}

auto operator==(const SparsePauliString& left, const SparsePauliString& right) -> bool
{
    return left.phase_ == right.phase_ && left.equal_up_to_phase(right);
}

auto SparsePauliString::to_record() const -> kt_pauli
{
    // Left-multiply each term onto i^k X^x Z^z in application order:
    //   X: x ^= 1;  Z: (-1)^x, z ^= 1;  Y = i X Z: i (-1)^x, x ^= 1, z ^= 1.
    // The record's convention is i^{#Y} X^x Z^z with Y where x & z, so the
    // record phase is k - popcount(x & z) plus the string's own phase.
    uint64_t x = 0, z = 0;
    int k = 0;
    for (const auto& [q, t] : terms_) {
        if (q >= n_qubits_ || q >= 64) {
            throw std::runtime_error {"ERROR: cannot perform operation on SparsePauliString with index beyond qubit range.\n"};
        }
        const uint64_t b = uint64_t {1} << q;
        switch (t) {
            case PauliTerm::X: x ^= b; break;
            case PauliTerm::Z:
                if (x & b) k += 2;
                z ^= b;
                break;
            case PauliTerm::Y:
                k += 1;
                if (x & b) k += 2;
                x ^= b;
                z ^= b;
                break;
            default: break;
        }
    }
    kt_pauli r {};
    r.x_mask = x;
    r.z_mask = z;
    const int ny = __builtin_popcountll(x & z);
    r.phase = ((static_cast<int>(phase_) + k - ny) % 4 + 4) % 4;
    return r;
}

PauliOperator::PauliOperator(std::size_t n_qubits)
    : n_qubits_ {n_qubits}
{}

PauliOperator::PauliOperator(std::vector<WeightedPauliString> weighted)
    : n_qubits_ {0}
    , strings_ {std::move(weighted)}
{
    if (strings_.empty()) {
        throw std::runtime_error {
            "ERROR: construction of `PauliOperator` with only WeightedPauliString instances requires\n"
            "a non-empty vector.\n"};
    }
    for (std::size_t i = 1; i < strings_.size(); ++i) {
        if (strings_[i].pauli_string.n_qubits() != strings_[0].pauli_string.n_qubits()) {
            throw std::runtime_error {
                "ERROR: construction of `PauliOperator` with WeightedPauliString instances requires\n"
                "all pauli strings to have the same number of qubits.\n"};
        }
    }
    n_qubits_ = strings_[0].pauli_string.n_qubits();
}

PauliOperator::PauliOperator(const std::initializer_list<WeightedPauliString>& weighted)
    : PauliOperator {std::vector<WeightedPauliString> {weighted}}
{}

void PauliOperator::add(WeightedPauliString value)
{
    strings_.emplace_back(std::move(value));
}

void PauliOperator::add(std::complex<double> coefficient, SparsePauliString pauli_string)
{
    strings_.push_back(WeightedPauliString {coefficient, std::move(pauli_string)});
}

void PauliOperator::remove(std::size_t index)
{
    if (index >= strings_.size()) {
        throw std::runtime_error {"ERROR: attempted to remove out of bounds element from PauliOperator.\n"};
    }
    strings_.erase(strings_.begin() + static_cast<std::ptrdiff_t>(index));
}

namespace
{

void records_of(const PauliOperator& op, std::size_t n_state, std::vector<kt_pauli>& recs, std::vector<double>& coeffs)
{
    recs.clear();
    coeffs.clear();
    for (const auto& [c, s] : op.weighted_pauli_strings()) {
        if (s.n_qubits() != n_state) {
            throw std::runtime_error {"Invalid simulation; SparsePauliString and state have different number of qubits."};
        }
        recs.push_back(s.to_record());
        coeffs.push_back(c.real());
        coeffs.push_back(c.imag());
    }
}

}  // namespace

auto expectation_value(const PauliOperator& op, const Statevector& state) -> std::complex<double>
{
    std::vector<kt_pauli> recs;
    std::vector<double> coeffs;
    records_of(op, state.n_qubits(), recs, coeffs);
    double total[2] = {0.0, 0.0};
    check(kt_sv_expect(state.device(), recs.data(), static_cast<int64_t>(recs.size()), coeffs.data(), nullptr, total));
    return {total[0], total[1]};
}

auto expectation_value(const SparsePauliString& s, const Statevector& state) -> std::complex<double>
{
    if (s.n_qubits() != state.n_qubits()) {
        throw std::runtime_error {"Invalid simulation; SparsePauliString and state have different number of qubits."};
    }
    const kt_pauli rec = s.to_record();
    double term[2] = {0.0, 0.0};
    check(kt_sv_expect(state.device(), &rec, 1, nullptr, term, nullptr));
    return {term[0], term[1]};
}

auto expectation_value(const PauliOperator& op, const DensityMatrix& state) -> std::complex<double>
{
    std::vector<kt_pauli> recs;
    std::vector<double> coeffs;
    records_of(op, state.n_qubits(), recs, coeffs);
    double total[2] = {0.0, 0.0};
    check(kt_dm_expect(state.device(), recs.data(), static_cast<int64_t>(recs.size()), coeffs.data(), nullptr, total));
    return {total[0], total[1]};
}

// ---- probabilities and measurements ---------------------------------------------------------

QuantumNoise::QuantumNoise(std::size_t n_qubits)
    : n_qubits_ {n_qubits}
    , noise_(n_qubits, 0.0)
{}

void QuantumNoise::set(std::size_t index, double noise)
{
    if (index >= n_qubits_) {
        throw std::runtime_error {"ERROR: Out-of-bounds access for QuantumNoise probability."};
    }
    if (!(0.0 <= noise && noise <= 1.0)) {
        throw std::runtime_error {"ERROR: Cannot set probability in QuantumNoise object outside of [0, 1]."};
    }
    noise_[index] = noise;
}

auto QuantumNoise::get(std::size_t index) const -> const double&
{
    if (index >= n_qubits_) {
        throw std::runtime_error {"ERROR: Out-of-bounds access for QuantumNoise probability."};
    }
    return noise_[index];
}

auto calculate_probabilities_raw(const Statevector& state, const QuantumNoise* noise) -> std::vector<double>
{
    std::vector<double> out(state.n_states());
    check(kt_sv_probabilities(state.device(), noise ? noise->values().data() : nullptr, out.data()));
    return out;
}

auto calculate_probabilities(const Statevector& state, const QuantumNoise* noise) -> std::map<std::string, double>
{
    const auto raw = calculate_probabilities_raw(state, noise);
    std::map<std::string, double> out;
    for (std::size_t i = 0; i < raw.size(); ++i) {
        out[state_index_to_bitstring(i, state.n_qubits(), Endian::LITTLE)] = raw[i];
    }
    return out;
}

auto perform_measurements_as_memory(const Statevector& state, std::size_t n_shots, const QuantumNoise* noise,
                                    std::optional<int> seed) -> std::vector<std::size_t>
{
    // ProbabilitySampler_ (measurements.cpp:288-311): one mt19937 for all shots,
    // each shot one generate_canonical draw scaled by the CDF bound on the device
    auto prng = make_prng(seed);
    std::vector<double> canon(n_shots);
    for (auto& c : canon) {
        c = std::generate_canonical<double, std::numeric_limits<double>::digits>(prng);
    }
    std::vector<uint64_t> idx(n_shots);
    int32_t rescanned = 0;
    check(kt_sv_sample(state.device(), noise ? noise->values().data() : nullptr, canon.data(),
                       static_cast<int64_t>(n_shots), idx.data(), 0, &rescanned));
    return {idx.begin(), idx.end()};
}

namespace
{

// ProbabilitySampler_ (measurements.cpp:288-311) on a probability vector: one
// mt19937 for all shots, one generate_canonical draw per shot, scaled by the
// CDF bound and searched on the device
auto sample_probabilities(const std::vector<double>& probabilities_raw, std::size_t n_shots, std::optional<int> seed)
    -> std::vector<std::size_t>
{
    auto prng = make_prng(seed);
    std::vector<double> canon(n_shots);
    for (auto& c : canon) {
        c = std::generate_canonical<double, std::numeric_limits<double>::digits>(prng);
    }
    std::vector<uint64_t> idx(n_shots);
    check(kt_sample_probabilities(probabilities_raw.data(), probabilities_raw.size(), canon.data(),
                                  static_cast<int64_t>(n_shots), idx.data(), 0, nullptr));
    return {idx.begin(), idx.end()};
}

auto marginal_mask(const std::vector<std::size_t>& marginal_qubits, std::size_t n) -> std::vector<char>
{
    // build_marginal_bitmask_ (measurements.cpp:269-286)
    std::vector<char> marginal(n, 0);
    for (auto q : marginal_qubits) {
        if (q >= n) {
            throw std::runtime_error {"ERROR: marginal qubit index out of range."};
        }
    }
    for (auto q : marginal_qubits) {
        marginal[q] = 1;
    }
    return marginal;
}

// state_index_to_bitstring_marginal_ (state/marginal.cpp:19-45): character q = qubit q, 'x' if marginal
auto marginal_bitstring(std::size_t i, const std::vector<char>& marginal) -> std::string
{
    const auto n = marginal.size();
    std::string s(n, '0');
    for (std::size_t q = 0; q < n; ++q) {
        s[q] = marginal[q] ? 'x' : (((i >> q) & 1U) ? '1' : '0');
    }
    return s;
}

}  // namespace

auto perform_measurements_as_memory(const std::vector<double>& probabilities_raw, std::size_t n_shots,
                                    std::optional<int> seed) -> std::vector<std::size_t>
{
    return sample_probabilities(probabilities_raw, n_shots, seed);
}

auto perform_measurements_as_counts_raw(const std::vector<double>& probabilities_raw, std::size_t n_shots,
                                        std::optional<int> seed) -> std::map<std::size_t, std::size_t>
{
    return memory_to_counts(sample_probabilities(probabilities_raw, n_shots, seed));
}

auto perform_measurements_as_counts_marginal(const std::vector<double>& probabilities_raw, std::size_t n_shots,
                                             const std::vector<std::size_t>& marginal_qubits, std::optional<int> seed)
    -> std::map<std::string, std::size_t>
{
    if (!is_power_of_2(probabilities_raw.size())) {
        throw std::runtime_error {"The number of probabilities must be a power of 2.\n"};
    }
    const auto n = static_cast<std::size_t>(__builtin_ctzll(probabilities_raw.size()));
    const auto marginal = marginal_mask(marginal_qubits, n);
    std::map<std::string, std::size_t> out;
    for (auto i : sample_probabilities(probabilities_raw, n_shots, seed)) {
        ++out[marginal_bitstring(i, marginal)];
    }
    return out;
}

auto perform_measurements_as_counts_marginal(const QuantumCircuit& circuit, const Statevector& original_state,
                                             std::size_t n_shots, const std::vector<std::size_t>& marginal_qubits,
                                             const QuantumNoise* noise, std::optional<int> seed)
    -> std::map<std::string, std::size_t>
{
    const auto marginal = marginal_mask(marginal_qubits, circuit.n_qubits());
    std::map<std::string, std::size_t> out;
    for (std::size_t shot = 0; shot < n_shots; ++shot) {
        auto state = original_state;
        simulate(circuit, state);
        const auto idx = perform_measurements_as_memory(state, 1, noise, seed);
        ++out[marginal_bitstring(idx[0], marginal)];
    }
    return out;
}

auto perform_measurements_as_counts_raw(const Statevector& state, std::size_t n_shots, const QuantumNoise* noise,
                                        std::optional<int> seed) -> std::map<std::size_t, std::size_t>
{
    return memory_to_counts(perform_measurements_as_memory(state, n_shots, noise, seed));
}

auto perform_measurements_as_counts_marginal(const Statevector& state, std::size_t n_shots,
                                             const std::vector<std::size_t>& marginal_qubits,
                                             const QuantumNoise* noise, std::optional<int> seed)
    -> std::map<std::string, std::size_t>
{
    const auto n = state.n_qubits();
    std::vector<char> marginal(n, 0);
    for (auto q : marginal_qubits) {
        if (q >= n) {
            throw std::runtime_error {"ERROR: marginal qubit index out of range."};
        }
        marginal[q] = 1;
    }
    std::map<std::string, std::size_t> out;
    for (auto i : perform_measurements_as_memory(state, n_shots, noise, seed)) {
        // state_index_to_bitstring_marginal_ (state/marginal.cpp:19-45): character q = qubit q, 'x' if marginal
        std::string s(n, '0');
        for (std::size_t q = 0; q < n; ++q) {
            s[q] = marginal[q] ? 'x' : (((i >> q) & 1U) ? '1' : '0');
        }
        ++out[s];
    }
    return out;
}

auto perform_measurements_as_counts(const Statevector& state, std::size_t n_shots, const QuantumNoise* noise,
                                    std::optional<int> seed) -> std::map<std::string, std::size_t>
{
    return perform_measurements_as_counts_marginal(state, n_shots, {}, noise, seed);
}

auto memory_to_counts(const std::vector<std::size_t>& measurements) -> std::map<std::size_t, std::size_t>
{
    std::map<std::size_t, std::size_t> m;
    for (auto i : measurements) {
        ++m[i];
    }
    return m;
}

auto memory_to_fractions(const std::vector<std::size_t>& measurements) -> std::map<std::size_t, double>
{
    std::map<std::size_t, double> m;
    for (auto i : measurements) {
        m[i] += 1.0;
    }
    const auto n = static_cast<double>(measurements.size());
    for (auto& [k, v] : m) {
        v /= n;
    }
    return m;
}

// ---- adjoint ---------------------------------------------------------------------------------------

auto adjoint_gradient(const QuantumCircuit& circuit, const Statevector& initial, const PauliOperator& hamiltonian,
                      int checkpoint_every) -> EnergyAndGradient
{
    check_valid_number_of_qubits(circuit.n_qubits(), initial.n_qubits());
    // every parameter-bound gate gets its own slot; the chain rule sums slots per parameter
    std::vector<kt_gate> recs;
    std::vector<double> values;
    std::vector<param::ParameterID> slot_id;
    for (const auto& el : circuit.circuit_elements()) {
        if (!el.is_gate()) {
            throw std::runtime_error {"ERROR: the adjoint gradient needs a circuit of gates only (no control flow or loggers).\n"};
        }
        const auto& gi = el.get_gate();
        if (gi.gate == Gate::M) {
            throw std::runtime_error {"ERROR: the adjoint gradient needs a circuit without M gates.\n"};
        }
        kt_gate r = to_record(gi, circuit.parameter_data_map());
        if (gi.parameter) {
            r.param = static_cast<int32_t>(values.size());
            values.push_back(r.angle);
            slot_id.push_back(*gi.parameter);
        }
        recs.push_back(r);
    }
    std::vector<kt_pauli> strs;
    std::vector<double> coeffs;
    records_of(hamiltonian, initial.n_qubits(), strs, coeffs);
    Statevector work {initial};
    kt_adjoint adj = nullptr;
    check(kt_adjoint_create(work.device(), checkpoint_every, &adj));
    EnergyAndGradient out {};
    std::vector<double> grad(values.size(), 0.0);
    int32_t rc = kt_adjoint_forward(adj, recs.data(), static_cast<int64_t>(recs.size()), values.data(),
                                    static_cast<int64_t>(values.size()), strs.data(), static_cast<int64_t>(strs.size()),
                                    coeffs.data(), &out.energy);
    if (rc == KT_OK) {
        rc = kt_adjoint_backward(adj, grad.data(), static_cast<int64_t>(grad.size()));
    }
    kt_adjoint_destroy(adj);
    check(rc);
    for (const auto& [id, data] : circuit.parameter_data_map()) {
        out.gradient[id] = 0.0;
    }
    for (std::size_t s = 0; s < grad.size(); ++s) {
        out.gradient[slot_id[s]] += grad[s];
    }
    return out;
}

}  // namespace ket
