// ket_b200_circuit_ops.cpp — circuit transforms (host side).
#include "kettle/ket_b200_circuit_ops.hpp"

#include <algorithm>
#include <cmath>
#include <optional>
#include <stdexcept>
#include <vector>

namespace ket
{

void extend_circuit(QuantumCircuit& left, const QuantumCircuit& right)
{
    if (left.n_qubits() != right.n_qubits()) {
        throw std::runtime_error {"Cannot append circuits with different numbers of qubits."};
    }
    if (left.n_bits() != right.n_bits()) {
        throw std::runtime_error {"Cannot append circuits with different numbers of bits."};
    }
    left.elements_.insert(left.elements_.end(), right.elements_.begin(), right.elements_.end());
    left.parameter_data_.insert(right.parameter_data_.begin(), right.parameter_data_.end());
}

auto append_circuits(QuantumCircuit left, const QuantumCircuit& right) -> QuantumCircuit
{
    extend_circuit(left, right);
    return left;
}

namespace
{

struct Primitive
{
    Gate gate;
    std::optional<double> angle;
};

// one fixed gate, then one rotation / phase whose angle is read off elem11
// (gates/matrix2x2_gate_decomposition.cpp:23-84)
auto as_single_primitive(const Matrix2X2& u, double tol_sq) -> std::optional<Primitive>
{
    static const std::pair<Gate, Matrix2X2> fixed[] = {
        {Gate::H, h_gate()},       {Gate::X, x_gate()}, {Gate::Y, y_gate()},       {Gate::Z, z_gate()},
        {Gate::S, s_gate()},       {Gate::SDAG, sdag_gate()}, {Gate::T, t_gate()}, {Gate::TDAG, tdag_gate()},
        {Gate::SX, sx_gate()},     {Gate::SXDAG, sxdag_gate()},
    };
    for (const auto& [g, m] : fixed) {
        if (almost_eq(u, m, tol_sq)) {
            return Primitive {g, std::nullopt};
        }
    }
    const double re11 = std::clamp(u.elem11.real(), -1.0, 1.0);
    const double half = std::acos(re11);
    if (almost_eq(u, rx_gate(2.0 * half), tol_sq)) {
        return Primitive {Gate::RX, 2.0 * half};
    }
    if (almost_eq(u, ry_gate(2.0 * half), tol_sq)) {
        return Primitive {Gate::RY, 2.0 * half};
    }
    if (almost_eq(u, rz_gate(2.0 * half), tol_sq)) {
        return Primitive {Gate::RZ, 2.0 * half};
    }
    const double im11 = std::clamp(u.elem11.imag(), -1.0, 1.0);
    const double phase = std::atan2(im11, re11);
    if (almost_eq(u, p_gate(phase), tol_sq)) {
        return Primitive {Gate::P, phase};
    }
    return std::nullopt;
}

// A special unitary as RZ(lambda - mu) RY(2 theta) RZ(lambda + mu), the ZYZ
// decomposition of fedimser/quantum_decomp (decompose_2x2.py) that the
// reference follows (gates/matrix2x2_gate_decomposition.cpp:86-112); factors
// whose angle is within the tolerance of 0 are dropped.
auto zyz(const Matrix2X2& u, double tol_sq) -> std::vector<Primitive>
{
    const double abs00 = std::clamp(std::abs(u.elem00), 0.0, 1.0);
    const double theta = -std::acos(abs00);
    const double lambda = -std::atan2(u.elem00.imag(), u.elem00.real());
    const double mu = -std::atan2(u.elem01.imag(), u.elem01.real());
    std::vector<Primitive> out;
    if (std::fabs(lambda - mu) > tol_sq) {
        out.push_back({Gate::RZ, lambda - mu});
    }
    if (std::fabs(2.0 * theta) > tol_sq) {
        out.push_back({Gate::RY, 2.0 * theta});
    }
    if (std::fabs(lambda + mu) > tol_sq) {
        out.push_back({Gate::RZ, lambda + mu});
    }
    return out;
}

auto decompose(const Matrix2X2& u, double tol_sq) -> std::vector<Primitive>
{
    // the single-gate match uses the default tolerance, as the reference's does
    if (auto one = as_single_primitive(u, COMPLEX_ALMOST_EQ_TOLERANCE_SQ)) {
        return {*one};
    }
    const auto det = determinant(u);
    const double det_angle = std::atan2(det.imag(), det.real());
    if (std::fabs(det_angle) < tol_sq) {
        return zyz(u, tol_sq);
    }
    auto out = zyz(p_gate(-det_angle) * u, tol_sq);
    out.push_back({Gate::P, det_angle});
    return out;
}

auto controlled(Gate g) -> Gate
{
    // H..P (0..13) -> CH..CP (14..27)
    return static_cast<Gate>(static_cast<int>(g) + (static_cast<int>(Gate::CH) - static_cast<int>(Gate::H)));
}

auto is_primitive(Gate g) -> bool
{
    return g != Gate::U && g != Gate::CU && g != Gate::M;
}

}  // namespace

// NOLINTNEXTLINE(misc-no-recursion)
auto transpile_to_primitive(const QuantumCircuit& circuit, double tolerance_sq) -> QuantumCircuit
{
    auto out = QuantumCircuit {circuit.n_qubits(), circuit.n_bits()};
    for (const auto& element : circuit.elements_) {
        if (element.is_circuit_logger()) {
            out.elements_.push_back(element);
        } else if (element.is_control_flow()) {
            const auto& cf = element.get_control_flow();
            if (cf.is_if_statement()) {
                const auto& st = cf.get_if_statement();
                auto sub = std::make_shared<const QuantumCircuit>(transpile_to_primitive(*st.circuit(), tolerance_sq));
                out.elements_.emplace_back(ClassicalIfStatement {st.predicate(), std::move(sub)});
            } else {
                const auto& st = cf.get_if_else_statement();
                auto sub_if = std::make_shared<const QuantumCircuit>(transpile_to_primitive(*st.if_circuit(), tolerance_sq));
                auto sub_else = std::make_shared<const QuantumCircuit>(transpile_to_primitive(*st.else_circuit(), tolerance_sq));
                out.elements_.emplace_back(ClassicalIfElseStatement {st.predicate(), std::move(sub_if), std::move(sub_else)});
            }
        } else {
            const auto& info = element.get_gate();
            if (is_primitive(info.gate) || info.gate == Gate::M) {
                out.elements_.push_back(info);
            } else if (info.gate == Gate::U) {
                for (const auto& p : decompose(*info.unitary_ptr, tolerance_sq)) {
                    out.elements_.push_back(GateInfo {p.gate, info.arg0, 0, p.angle.value_or(0.0), std::nullopt, std::nullopt});
                }
            } else {
                for (const auto& p : decompose(*info.unitary_ptr, tolerance_sq)) {
                    out.elements_.push_back(
                        GateInfo {controlled(p.gate), info.arg0, info.arg1, p.angle.value_or(0.0), std::nullopt, std::nullopt});
                }
            }
        }
    }
    return out;
}

namespace
{

// the matrix a gate applies to its target (the controlled matrix for a
// controlled gate), with a bound parameter's value for its angle
auto target_matrix(const GateInfo& g, const param::ParameterDataMap& params) -> Matrix2X2
{
    if (g.gate == Gate::U || g.gate == Gate::CU) {
        return *g.unitary_ptr;
    }
    const bool angle = (g.gate >= Gate::RX && g.gate <= Gate::P) || (g.gate >= Gate::CRX && g.gate <= Gate::CP);
    if (!angle) {
        return non_angle_gate(g.gate);
    }
    double theta = g.arg2;
    if (g.parameter) {
        theta = *params.at(*g.parameter).value;
    }
    return angle_gate(g.gate, theta);
}

auto is_controlled_gate(Gate g) -> bool
{
    return (g >= Gate::CH && g <= Gate::CP) || g == Gate::CU;
}

auto only_loggers_from(const QuantumCircuit& c, std::size_t i) -> bool
{
    for (; i < c.n_circuit_elements(); ++i) {
        if (!c[i].is_circuit_logger()) {
            return false;
        }
    }
    return true;
}

void require_parameter_values(const param::ParameterDataMap& params)
{
    // parameter/parameter_expression.cpp:84-99: every parameter needs a value
    for (const auto& [id, data] : params) {
        if (!data.value) {
            throw std::runtime_error {"ERROR: cannot perform simulation with an uninitialized parameter value.\n"};
        }
    }
}

}  // namespace

auto almost_eq(const QuantumCircuit& left, const QuantumCircuit& right, double tol_sq) -> bool
{
    // circuit_operations/compare_circuits.cpp:128-231
    if (left.n_qubits() != right.n_qubits() || left.n_bits() != right.n_bits()) {
        return false;
    }
    require_parameter_values(left.parameter_data_map());
    require_parameter_values(right.parameter_data_map());
    std::size_t il = 0;
    std::size_t ir = 0;
    while (il < left.n_circuit_elements() && ir < right.n_circuit_elements()) {
        const auto& a = left[il];
        if (a.is_circuit_logger()) {
            ++il;
            continue;
        }
        const auto& b = right[ir];
        if (b.is_circuit_logger()) {
            ++ir;
            continue;
        }
        if (a.is_control_flow() && b.is_control_flow()) {
            const auto& ca = a.get_control_flow();
            const auto& cb = b.get_control_flow();
            if (ca.is_if_statement() && cb.is_if_statement()) {
                const auto& sa = ca.get_if_statement();
                const auto& sb = cb.get_if_statement();
                if (sa.predicate() != sb.predicate() || !almost_eq(*sa.circuit(), *sb.circuit(), tol_sq)) {
                    return false;
                }
            } else if (ca.is_if_else_statement() && cb.is_if_else_statement()) {
                const auto& sa = ca.get_if_else_statement();
                const auto& sb = cb.get_if_else_statement();
                if (sa.predicate() != sb.predicate() || !almost_eq(*sa.if_circuit(), *sb.if_circuit(), tol_sq) ||
                    !almost_eq(*sa.else_circuit(), *sb.else_circuit(), tol_sq)) {
                    return false;
                }
            } else {
                return false;
            }
        } else if (a.is_gate() && b.is_gate()) {
            const auto& ga = a.get_gate();
            const auto& gb = b.get_gate();
            const bool ma = ga.gate == Gate::M;
            const bool mb = gb.gate == Gate::M;
            if (ma != mb) {
                return false;
            }
            if (ma) {
                if (ga.arg0 != gb.arg0 || ga.arg1 != gb.arg1) {
                    return false;
                }
            } else {
                // both as (controlled) U gates: same kind, same qubits, close matrices
                if (is_controlled_gate(ga.gate) != is_controlled_gate(gb.gate) || ga.arg0 != gb.arg0 ||
                    (is_controlled_gate(ga.gate) && ga.arg1 != gb.arg1)) {
                    return false;
                }
                if (!almost_eq(target_matrix(ga, left.parameter_data_map()),
                               target_matrix(gb, right.parameter_data_map()), tol_sq)) {
                    return false;
                }
            }
        } else {
            return false;
        }
        ++il;
        ++ir;
    }
    if (il == left.n_circuit_elements() && ir < right.n_circuit_elements()) {
        return only_loggers_from(right, ir);
    }
    if (il < left.n_circuit_elements() && ir == right.n_circuit_elements()) {
        return only_loggers_from(left, il);
    }
    return true;
}

}  // namespace ket
