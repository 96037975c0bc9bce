// ket_b200.hpp — the kettle C++20 API on the B200 engine (namespace ket).
//
// A drop-in for the circuit-propagation part of the kettle library: the same
// class and function names, argument meanings and thrown messages as the
// reference headers, implemented as host code over the C-ABI of
// include/kettle_b200.h (libket_b200.so links libkettle_b200.so).  States live
// in GPU memory; element access goes through a host mirror that is refreshed
// lazily (reads download once, writes mark the mirror authoritative and the
// next device operation uploads it).
//
// Interfaces mirrored (reference paths):
//   ket::Gate, ket::Matrix2X2            include/kettle/gates/primitive_gate.hpp:19-79,
//                                        include/kettle/common/matrix2x2.hpp:12-20
//   ket::param::{ParameterID, parameterized, ParameterData}
//                                        include/kettle/parameter/parameter.hpp:14-65
//   ket::QuantumCircuit                  include/kettle/circuit/circuit.hpp:20-419 (primitive gates,
//                                        parameters, M gates, classical if / if-else statements,
//                                        circuit loggers; no compound gates)
//   ket::ControlFlowPredicate, Classical*Statement, CircuitLogger, CircuitElement
//                                        include/kettle/circuit/control_flow*.hpp, circuit_element.hpp,
//                                        include/kettle/circuit_loggers/*.hpp
//   ket::ClassicalRegister               include/kettle/circuit/classical_register.hpp:14-42
//   ket::Statevector                     include/kettle/state/statevector.hpp:14-96
//   ket::DensityMatrix                   include/kettle/state/density_matrix.hpp:22-110 (matrix()
//                                        returns a host column-major view instead of Eigen::MatrixXcd)
//   ket::simulate, *Simulator            include/kettle/simulation/simulate.hpp:16-41,
//                                        include/kettle/simulation/simulate_density_matrix.hpp:18-46
//   ket::SparsePauliString, PauliOperator, expectation_value
//                                        include/kettle/operator/pauli/{sparse_pauli_string,pauli_operator}.hpp
//   ket::QuantumNoise, calculate_probabilities_raw, perform_measurements_*
//                                        include/kettle/calculations/{probabilities,measurements}.hpp
//   bitstring / index conversions, marginal strips, random states and unitaries, projection
//                                        include/kettle/state/{qubit_state_conversion,marginal,random,
//                                        project_state}.hpp, include/kettle/gates/random_u_gates.hpp
// New (no reference counterpart): expectation_value(PauliOperator, DensityMatrix),
// ket::adjoint_gradient, ket::DType (complex64 storage).
#pragma once

#include <array>
#include <compare>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <map>
#include <memory>
#include <optional>
#include <random>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <vector>
#include <variant>

#include "kettle_b200.h"

namespace ket
{

// ---- constants (include/kettle/common/tolerance.hpp:6-12) ----------------------
constexpr inline auto PROJECTION_NORMALIZATION_TOLERANCE = double {1.0e-8};
constexpr inline auto CONSTRUCTION_NORMALIZATION_TOLERANCE = double {1.0e-6};
constexpr inline auto COMPLEX_ALMOST_EQ_TOLERANCE_SQ = double {1.0e-6};
constexpr inline auto MATRIX_2X2_SQRT_TOLERANCE = double {1.0e-6};
constexpr inline auto MATCHING_PARAMETER_VALUE_TOLERANCE = double {1.0e-6};
constexpr inline auto DENSITY_MATRIX_TRACE_TOLERANCE = double {1.0e-8};

enum class Endian : std::uint8_t
{
    LITTLE,
    BIG
};

// Amplitude storage on the device (new): complex128, or complex64 with FP64 reductions.
enum class DType : std::int32_t
{
    C128 = KT_C128,
    C64 = KT_C64
};

enum class Gate : std::uint8_t
{
    H, X, Y, Z, S, SDAG, T, TDAG, SX, SXDAG, RX, RY, RZ, P,
    CH, CX, CY, CZ, CS, CSDAG, CT, CTDAG, CSX, CSXDAG, CRX, CRY, CRZ, CP,
    U, CU, M
};

struct Matrix2X2
{
    std::complex<double> elem00;
    std::complex<double> elem01;
    std::complex<double> elem10;
    std::complex<double> elem11;

    // common/matrix2x2.hpp:19-25: in-place sum, product (this * other) and scaling
    auto operator+=(const Matrix2X2& other) noexcept -> Matrix2X2
    {
        elem00 += other.elem00;
        elem01 += other.elem01;
        elem10 += other.elem10;
        elem11 += other.elem11;
        return *this;
    }
    auto operator*=(const Matrix2X2& other) noexcept -> Matrix2X2
    {
        const auto n00 = elem00 * other.elem00 + elem01 * other.elem10;
        const auto n01 = elem00 * other.elem01 + elem01 * other.elem11;
        const auto n10 = elem10 * other.elem00 + elem11 * other.elem10;
        const auto n11 = elem10 * other.elem01 + elem11 * other.elem11;
        elem00 = n00;
        elem01 = n01;
        elem10 = n10;
        elem11 = n11;
        return *this;
    }
    template <typename Number>
    auto operator*=(Number scalar) noexcept -> Matrix2X2
    {
        elem00 *= scalar;
        elem01 *= scalar;
        elem10 *= scalar;
        elem11 *= scalar;
        return *this;
    }
};

auto conjugate_transpose(const Matrix2X2& mat) -> Matrix2X2;
auto operator*(const Matrix2X2& lhs, const Matrix2X2& rhs) -> Matrix2X2;
auto operator+(const Matrix2X2& lhs, const Matrix2X2& rhs) -> Matrix2X2;
auto operator*(const Matrix2X2& lhs, std::complex<double> scalar) -> Matrix2X2;
auto operator*(std::complex<double> scalar, const Matrix2X2& rhs) -> Matrix2X2;
auto determinant(const Matrix2X2& mat) -> std::complex<double>;
auto trace(const Matrix2X2& mat) -> std::complex<double>;
// common/matrix2x2.cpp:117-135: the square root with the positive roots s, t of
// the general 2x2 formula, switching to -s when |tr + 2s|^2 <= tolerance
auto matrix_square_root(const Matrix2X2& mat, double matrix_sqrt_tolerance = MATRIX_2X2_SQRT_TOLERANCE) -> Matrix2X2;
auto almost_eq(const Matrix2X2& left, const Matrix2X2& right,
               double tolerance_sq = COMPLEX_ALMOST_EQ_TOLERANCE_SQ) noexcept -> bool;
auto almost_eq(const std::complex<double>& left, const std::complex<double>& right,
               double tolerance_sq = COMPLEX_ALMOST_EQ_TOLERANCE_SQ) noexcept -> bool;

// gate matrices (gates/common_u_gates.cpp)
auto i_gate() noexcept -> Matrix2X2;
auto h_gate() noexcept -> Matrix2X2;
auto x_gate() noexcept -> Matrix2X2;
auto y_gate() noexcept -> Matrix2X2;
auto z_gate() noexcept -> Matrix2X2;
auto s_gate() noexcept -> Matrix2X2;
auto sdag_gate() noexcept -> Matrix2X2;
auto t_gate() noexcept -> Matrix2X2;
auto tdag_gate() noexcept -> Matrix2X2;
auto sx_gate() noexcept -> Matrix2X2;
auto sxdag_gate() noexcept -> Matrix2X2;
auto rx_gate(double angle) noexcept -> Matrix2X2;
auto ry_gate(double angle) noexcept -> Matrix2X2;
auto rz_gate(double angle) noexcept -> Matrix2X2;
auto p_gate(double angle) noexcept -> Matrix2X2;
// gates/common_u_gates.hpp:39-41: the matrix of a fixed gate (H .. SXDAG) or
// an angle gate (RX, RY, RZ, P), uncontrolled or controlled; other gates throw
auto non_angle_gate(Gate gate) -> Matrix2X2;
auto angle_gate(Gate gate, double angle) -> Matrix2X2;

// Haar-random U(2) (gates/random_u_gates.hpp:18-34): four uniform [0, 1)
// draws from the generator (three phases, then the mixing angle).  The seeded
// form starts a fresh std::mt19937(seed); the bare form seeds from
// std::random_device.
auto generate_random_unitary2x2(std::mt19937& prng) -> Matrix2X2;
auto generate_random_unitary2x2(int seed) -> Matrix2X2;
auto generate_random_unitary2x2() -> Matrix2X2;

// ---- parameters -------------------------------------------------------------------
namespace param
{

struct parameterized
{
    explicit parameterized() = default;
};

constexpr inline auto PARAMETER_ID_SIZE = std::size_t {16};
using ParameterID = std::array<std::uint8_t, PARAMETER_ID_SIZE>;

struct ParameterIdHash
{
    auto operator()(const ParameterID& id) const noexcept -> std::size_t;
};

struct ParameterData
{
    std::optional<double> value;
    std::string name;
    std::size_t count;
};

using ParameterDataMap = std::unordered_map<ParameterID, ParameterData, ParameterIdHash>;

}  // namespace param

// One primitive gate of a circuit (the fields of ket::GateInfo, primitive_gate.hpp:71-79).
struct GateInfo
{
    Gate gate;
    std::size_t arg0;   // target (one-target gates), control (controlled gates), qubit (M)
    std::size_t arg1;   // target (controlled gates), classical bit (M)
    double arg2;        // angle
    std::optional<Matrix2X2> unitary_ptr;  // the reference's field name; dereferences the same way
    std::optional<param::ParameterID> parameter;  // angle bound to a circuit parameter
};

// ---- classical control flow and circuit loggers ---------------------------------------
// include/kettle/circuit/control_flow_predicate.hpp:12-56, control_flow.hpp:28-157,
// circuit_loggers/*.hpp, circuit/circuit_element.hpp: the same classes and accessors.
// Sub-circuits and logged snapshots are immutable once stored and are held by
// shared pointers (ClonePtr here), which dereference like the reference's ClonePtr.
class QuantumCircuit;
class ClassicalRegister;
class Statevector;
class DensityMatrix;

template <typename T>
using ClonePtr = std::shared_ptr<const T>;

enum class ControlFlowBooleanKind : std::uint8_t
{
    IF,
    IF_NOT
};

class ControlFlowPredicate
{
public:
    ControlFlowPredicate(std::vector<std::size_t> bit_indices_to_check, std::vector<int> expected_bits,
                         ControlFlowBooleanKind control_kind);
    auto operator()(const ClassicalRegister& creg) const -> bool;
    [[nodiscard]] auto bit_indices_to_check() const -> const std::vector<std::size_t>& { return bit_indices_to_check_; }
    [[nodiscard]] auto expected_bits() const -> const std::vector<int>& { return expected_bits_; }
    [[nodiscard]] auto control_kind() const -> ControlFlowBooleanKind { return control_kind_; }
    // circuit/control_flow_predicate.hpp:47: member-wise, in declaration order
    friend auto operator<=>(const ControlFlowPredicate& left, const ControlFlowPredicate& right) noexcept = default;

private:
    std::vector<std::size_t> bit_indices_to_check_;
    std::vector<int> expected_bits_;
    ControlFlowBooleanKind control_kind_;
};

class ClassicalIfStatement
{
public:
    ClassicalIfStatement(ControlFlowPredicate predicate, ClonePtr<QuantumCircuit> circuit)
        : predicate_ {std::move(predicate)}, circuit_ {std::move(circuit)}
    {}
    auto operator()(const ClassicalRegister& c_register) const -> bool { return predicate_(c_register); }
    [[nodiscard]] auto circuit() const -> const ClonePtr<QuantumCircuit>& { return circuit_; }
    [[nodiscard]] auto predicate() const -> const ControlFlowPredicate& { return predicate_; }

private:
    ControlFlowPredicate predicate_;
    ClonePtr<QuantumCircuit> circuit_;
};

class ClassicalIfElseStatement
{
public:
    ClassicalIfElseStatement(ControlFlowPredicate predicate, ClonePtr<QuantumCircuit> if_circuit,
                             ClonePtr<QuantumCircuit> else_circuit)
        : predicate_ {std::move(predicate)}, if_circuit_ {std::move(if_circuit)}, else_circuit_ {std::move(else_circuit)}
    {}
    auto operator()(const ClassicalRegister& c_register) const -> bool { return predicate_(c_register); }
    [[nodiscard]] auto if_circuit() const -> const ClonePtr<QuantumCircuit>& { return if_circuit_; }
    [[nodiscard]] auto else_circuit() const -> const ClonePtr<QuantumCircuit>& { return else_circuit_; }
    [[nodiscard]] auto predicate() const -> const ControlFlowPredicate& { return predicate_; }

private:
    ControlFlowPredicate predicate_;
    ClonePtr<QuantumCircuit> if_circuit_;
    ClonePtr<QuantumCircuit> else_circuit_;
};

class ClassicalControlFlowInstruction
{
public:
    ClassicalControlFlowInstruction(ClassicalIfStatement instruction) : instruction_ {std::move(instruction)} {}  // NOLINT
    ClassicalControlFlowInstruction(ClassicalIfElseStatement instruction) : instruction_ {std::move(instruction)} {}  // NOLINT
    [[nodiscard]] auto is_if_statement() const -> bool { return std::holds_alternative<ClassicalIfStatement>(instruction_); }
    [[nodiscard]] auto is_if_else_statement() const -> bool
    {
        return std::holds_alternative<ClassicalIfElseStatement>(instruction_);
    }
    [[nodiscard]] auto get_if_statement() const -> const ClassicalIfStatement&
    {
        return std::get<ClassicalIfStatement>(instruction_);
    }
    [[nodiscard]] auto get_if_else_statement() const -> const ClassicalIfElseStatement&
    {
        return std::get<ClassicalIfElseStatement>(instruction_);
    }

private:
    std::variant<ClassicalIfStatement, ClassicalIfElseStatement> instruction_;
};

class ClassicalRegisterCircuitLogger
{
public:
    void add_classical_register(ClassicalRegister cregister);
    [[nodiscard]] auto classical_register() const -> const ClassicalRegister&;

private:
    ClonePtr<ClassicalRegister> cregister_;
};

class StatevectorCircuitLogger
{
public:
    void add_statevector(Statevector statevector);
    [[nodiscard]] auto statevector() const -> const Statevector&;

private:
    ClonePtr<Statevector> statevector_;
};

class DensityMatrixCircuitLogger
{
public:
    void add_density_matrix(DensityMatrix density_matrix);
    [[nodiscard]] auto density_matrix() const -> const DensityMatrix&;

private:
    ClonePtr<DensityMatrix> density_matrix_;
};

class CircuitLogger
{
public:
    CircuitLogger(ClassicalRegisterCircuitLogger logger) : logger_ {std::move(logger)} {}  // NOLINT
    CircuitLogger(StatevectorCircuitLogger logger) : logger_ {std::move(logger)} {}  // NOLINT
    CircuitLogger(DensityMatrixCircuitLogger logger) : logger_ {std::move(logger)} {}  // NOLINT
    [[nodiscard]] auto is_classical_register_circuit_logger() const -> bool
    {
        return std::holds_alternative<ClassicalRegisterCircuitLogger>(logger_);
    }
    [[nodiscard]] auto get_classical_register_circuit_logger() const -> const ClassicalRegisterCircuitLogger&
    {
        return std::get<ClassicalRegisterCircuitLogger>(logger_);
    }
    [[nodiscard]] auto is_statevector_circuit_logger() const -> bool
    {
        return std::holds_alternative<StatevectorCircuitLogger>(logger_);
    }
    [[nodiscard]] auto get_statevector_circuit_logger() const -> const StatevectorCircuitLogger&
    {
        return std::get<StatevectorCircuitLogger>(logger_);
    }
    [[nodiscard]] auto is_density_matrix_circuit_logger() const -> bool
    {
        return std::holds_alternative<DensityMatrixCircuitLogger>(logger_);
    }
    [[nodiscard]] auto get_density_matrix_circuit_logger() const -> const DensityMatrixCircuitLogger&
    {
        return std::get<DensityMatrixCircuitLogger>(logger_);
    }

private:
    std::variant<ClassicalRegisterCircuitLogger, StatevectorCircuitLogger, DensityMatrixCircuitLogger> logger_;
};

struct CircuitElement
{
public:
    CircuitElement(const GateInfo& ginfo) : element_ {ginfo} {}  // NOLINT
    CircuitElement(ClassicalIfStatement instruction) : element_ {ClassicalControlFlowInstruction {std::move(instruction)}} {}  // NOLINT
    CircuitElement(ClassicalIfElseStatement instruction)  // NOLINT
        : element_ {ClassicalControlFlowInstruction {std::move(instruction)}}
    {}
    CircuitElement(CircuitLogger logger) : element_ {std::move(logger)} {}  // NOLINT
    CircuitElement(ClassicalRegisterCircuitLogger logger) : element_ {CircuitLogger {std::move(logger)}} {}  // NOLINT
    CircuitElement(StatevectorCircuitLogger logger) : element_ {CircuitLogger {std::move(logger)}} {}  // NOLINT
    [[nodiscard]] auto is_gate() const -> bool { return std::holds_alternative<GateInfo>(element_); }
    [[nodiscard]] auto is_control_flow() const -> bool
    {
        return std::holds_alternative<ClassicalControlFlowInstruction>(element_);
    }
    [[nodiscard]] auto is_circuit_logger() const -> bool { return std::holds_alternative<CircuitLogger>(element_); }
    [[nodiscard]] auto get_gate() const -> const GateInfo& { return std::get<GateInfo>(element_); }
    [[nodiscard]] auto get_control_flow() const -> const ClassicalControlFlowInstruction&
    {
        return std::get<ClassicalControlFlowInstruction>(element_);
    }
    [[nodiscard]] auto get_circuit_logger() const -> const CircuitLogger& { return std::get<CircuitLogger>(element_); }

private:
    std::variant<GateInfo, ClassicalControlFlowInstruction, CircuitLogger> element_;
};

// ---- circuit ------------------------------------------------------------------------
class QuantumCircuit
{
public:
    explicit QuantumCircuit(std::size_t n_qubits, std::size_t n_bits);
    explicit QuantumCircuit(std::size_t n_qubits);

    [[nodiscard]] auto n_qubits() const noexcept -> std::size_t { return n_qubits_; }
    [[nodiscard]] auto n_bits() const noexcept -> std::size_t { return n_bits_; }
    [[nodiscard]] auto n_circuit_elements() const noexcept -> std::size_t { return elements_.size(); }
    [[nodiscard]] auto operator[](std::size_t index) const noexcept -> const CircuitElement& { return elements_[index]; }
    [[nodiscard]] auto begin() const noexcept { return elements_.begin(); }
    [[nodiscard]] auto end() const noexcept { return elements_.end(); }
    [[nodiscard]] auto circuit_elements() const noexcept -> const std::vector<CircuitElement>& { return elements_; }
    [[nodiscard]] auto parameter_data_map() const noexcept -> const param::ParameterDataMap& { return parameter_data_; }
    void pop_back();

    void set_parameter_value(const param::ParameterID& id, double angle);

#define KET_ONE_TARGET(name)                                   \
    void add_##name##_gate(std::size_t target_index);          \
    void add_##name##_gate(const std::vector<std::size_t>& indices); \
    void add_##name##_gate(std::initializer_list<std::size_t> indices) { add_##name##_gate(std::vector<std::size_t>(indices)); }
    KET_ONE_TARGET(h)
    KET_ONE_TARGET(x)
    KET_ONE_TARGET(y)
    KET_ONE_TARGET(z)
    KET_ONE_TARGET(s)
    KET_ONE_TARGET(sdag)
    KET_ONE_TARGET(t)
    KET_ONE_TARGET(tdag)
    KET_ONE_TARGET(sx)
    KET_ONE_TARGET(sxdag)
#undef KET_ONE_TARGET

#define KET_ONE_ANGLE(name)                                                                                  \
    void add_##name##_gate(std::size_t target_index, double angle);                                          \
    auto add_##name##_gate(std::size_t target_index, double initial_angle, param::parameterized key)         \
        -> param::ParameterID;                                                                                \
    void add_##name##_gate(std::size_t target_index, const param::ParameterID& id);                          \
    void add_##name##_gate(const std::vector<std::pair<std::size_t, double>>& pairs);                        \
    void add_##name##_gate(std::initializer_list<std::pair<std::size_t, double>> pairs) { add_##name##_gate(std::vector<std::pair<std::size_t, double>>(pairs)); }
    KET_ONE_ANGLE(rx)
    KET_ONE_ANGLE(ry)
    KET_ONE_ANGLE(rz)
    KET_ONE_ANGLE(p)
#undef KET_ONE_ANGLE

#define KET_CTRL(name)                                                                              \
    void add_##name##_gate(std::size_t control_index, std::size_t target_index);                    \
    void add_##name##_gate(const std::vector<std::pair<std::size_t, std::size_t>>& pairs);          \
    void add_##name##_gate(std::initializer_list<std::pair<std::size_t, std::size_t>> pairs) { add_##name##_gate(std::vector<std::pair<std::size_t, std::size_t>>(pairs)); }
    KET_CTRL(ch)
    KET_CTRL(cx)
    KET_CTRL(cy)
    KET_CTRL(cz)
    KET_CTRL(cs)
    KET_CTRL(csdag)
    KET_CTRL(ct)
    KET_CTRL(ctdag)
    KET_CTRL(csx)
    KET_CTRL(csxdag)
#undef KET_CTRL

#define KET_CTRL_ANGLE(name)                                                                                       \
    void add_##name##_gate(std::size_t control_index, std::size_t target_index, double angle);                     \
    auto add_##name##_gate(std::size_t control_index, std::size_t target_index, double initial_angle,              \
                           param::parameterized key) -> param::ParameterID;                                        \
    void add_##name##_gate(std::size_t control_index, std::size_t target_index, const param::ParameterID& id);     \
    void add_##name##_gate(const std::vector<std::tuple<std::size_t, std::size_t, double>>& tuples);
    KET_CTRL_ANGLE(crx)
    KET_CTRL_ANGLE(cry)
    KET_CTRL_ANGLE(crz)
    KET_CTRL_ANGLE(cp)
#undef KET_CTRL_ANGLE

    void add_u_gate(const Matrix2X2& gate, std::size_t target_index);
    void add_u_gate(const Matrix2X2& gate, const std::vector<std::size_t>& indices);
    void add_cu_gate(const Matrix2X2& gate, std::size_t control_index, std::size_t target_index);
    void add_cu_gate(const Matrix2X2& gate, const std::vector<std::pair<std::size_t, std::size_t>>& pairs);

    // compound gates: the same primitive gates the reference appends
    // (circuit/circuit.cpp:723-900), which the engine fuses like any others
    using Triplets = std::vector<std::tuple<std::size_t, std::size_t, std::size_t>>;
    using TripletsIList = std::initializer_list<std::tuple<std::size_t, std::size_t, std::size_t>>;
    void add_ccx_gate(std::size_t control_index0, std::size_t control_index1, std::size_t target_index);
    void add_ccx_gate(const Triplets& triplets);
    void add_ccx_gate(TripletsIList triplets) { add_ccx_gate(Triplets(triplets)); }
    void add_ccy_gate(std::size_t control_index0, std::size_t control_index1, std::size_t target_index);
    void add_ccy_gate(const Triplets& triplets);
    void add_ccy_gate(TripletsIList triplets) { add_ccy_gate(Triplets(triplets)); }
    void add_ccz_gate(std::size_t control_index0, std::size_t control_index1, std::size_t target_index);
    void add_ccz_gate(const Triplets& triplets);
    void add_ccz_gate(TripletsIList triplets) { add_ccz_gate(Triplets(triplets)); }
    void add_ccu_gate(const Matrix2X2& unitary, std::size_t control_index0, std::size_t control_index1,
                      std::size_t target_index);
    void add_ccu_gate(const Matrix2X2& unitary, const Triplets& triplets);
    void add_ccu_gate(const Matrix2X2& unitary, TripletsIList triplets) { add_ccu_gate(unitary, Triplets(triplets)); }
    void add_swap_gate(std::size_t target_index0, std::size_t target_index1);
    void add_swap_gate(const std::vector<std::pair<std::size_t, std::size_t>>& target_index_pairs);
    void add_swap_gate(std::initializer_list<std::pair<std::size_t, std::size_t>> pairs) { add_swap_gate(std::vector<std::pair<std::size_t, std::size_t>>(pairs)); }
    void add_cswap_gate(std::size_t control_qubit, std::size_t target_index0, std::size_t target_index1);
    void add_cswap_gate(const Triplets& triplets);
    void add_cswap_gate(TripletsIList triplets) { add_cswap_gate(Triplets(triplets)); }
    void add_qft_gate(const std::vector<std::size_t>& indices);
    void add_qft_gate(std::initializer_list<std::size_t> indices) { add_qft_gate(std::vector<std::size_t>(indices)); }
    void add_iqft_gate(const std::vector<std::size_t>& indices);
    void add_iqft_gate(std::initializer_list<std::size_t> indices) { add_iqft_gate(std::vector<std::size_t>(indices)); }

    void add_m_gate(std::size_t target_index);
    void add_m_gate(const std::vector<std::size_t>& indices);
    void add_m_gate(std::initializer_list<std::size_t> indices) { add_m_gate(std::vector<std::size_t>(indices)); }
    void add_m_gate(std::size_t target_index, std::size_t bit_index);

    // non-gate elements (circuit.hpp:280-362 of the reference)
    void add_if_statement(ControlFlowPredicate predicate, QuantumCircuit circuit,
                          double tolerance = MATCHING_PARAMETER_VALUE_TOLERANCE);
    void add_if_statement(std::size_t bit_index, QuantumCircuit subcircuit);
    void add_if_not_statement(std::size_t bit_index, QuantumCircuit subcircuit);
    void add_if_else_statement(ControlFlowPredicate predicate, QuantumCircuit if_subcircuit,
                               QuantumCircuit else_subcircuit);
    void add_if_else_statement(std::size_t bit_index, QuantumCircuit if_subcircuit, QuantumCircuit else_subcircuit);
    void add_if_not_else_statement(std::size_t bit_index, QuantumCircuit if_subcircuit, QuantumCircuit else_subcircuit);
    void add_classical_register_circuit_logger();
    void add_statevector_circuit_logger();
    void add_circuit_logger(CircuitLogger circuit_logger);

private:
    friend void extend_circuit(QuantumCircuit& left, const QuantumCircuit& right);
    friend auto transpile_to_primitive(const QuantumCircuit& circuit, double tolerance_sq) -> QuantumCircuit;

    std::size_t n_qubits_;
    std::size_t n_bits_;
    std::vector<CircuitElement> elements_;
    param::ParameterDataMap parameter_data_;
    std::size_t parameter_count_ {0};

    void check_qubit_range_(std::size_t index, const char* qubit_name, const char* gate_name) const;
    void check_bit_range_(std::size_t bit_index) const;
    void merge_subcircuit_parameters_(const QuantumCircuit& subcircuit, double tolerance);
    void add_one_(Gate g, std::size_t target);
    void add_one_angle_(Gate g, std::size_t target, double angle);
    auto add_one_param_(Gate g, std::size_t target, double angle) -> param::ParameterID;
    void add_one_param_id_(Gate g, std::size_t target, const param::ParameterID& id);
    void add_ctrl_(Gate g, std::size_t control, std::size_t target);
    void add_ctrl_angle_(Gate g, std::size_t control, std::size_t target, double angle);
    auto add_ctrl_param_(Gate g, std::size_t control, std::size_t target, double angle) -> param::ParameterID;
    void add_ctrl_param_id_(Gate g, std::size_t control, std::size_t target, const param::ParameterID& id);
    auto new_parameter_(std::optional<double> value) -> param::ParameterID;
    void use_parameter_(const param::ParameterID& id);
};

class ClassicalRegister
{
public:
    explicit ClassicalRegister(std::size_t n_bits)
        : measured_bits_(n_bits, std::nullopt)
    {}
    [[nodiscard]] auto is_measured(std::size_t index) const -> bool { return measured_bits_[index].has_value(); }
    [[nodiscard]] auto get(std::size_t index) const -> int { return measured_bits_[index].value(); }
    void set(std::size_t index, int value) { measured_bits_[index] = value; }

private:
    std::vector<std::optional<int>> measured_bits_;
};

// ---- states ------------------------------------------------------------------------
auto bitstring_to_state_index(const std::string& bitstring, Endian input_endian = Endian::LITTLE) -> std::size_t;
auto state_index_to_bitstring(std::size_t i_state, std::size_t n_qubits, Endian endian = Endian::LITTLE) -> std::string;
auto endian_flip(std::size_t value, std::size_t n_relevant_bits) -> std::size_t;

// state/qubit_state_conversion.hpp:14-61: a "dynamic bitset" holds one
// std::uint8_t (0 or 1) per qubit, in the order of the bitstring's characters.
auto state_index_to_dynamic_bitset(std::size_t i_state, std::size_t n_qubits, Endian input_endian)
    -> std::vector<std::uint8_t>;
auto dynamic_bitset_to_bitstring(const std::vector<std::uint8_t>& bits) -> std::string;
auto dynamic_bitset_to_state_index(const std::vector<std::uint8_t>& dyn_bitset, Endian input_endian) -> std::size_t;
auto bitstring_to_dynamic_bitset(const std::string& bitstring) -> std::vector<std::uint8_t>;
auto bitstring_to_state_index_little_endian(const std::string& bitstring) -> std::size_t;
auto bitstring_to_state_index_big_endian(const std::string& bitstring) -> std::size_t;
auto state_index_to_bitstring_little_endian(std::size_t i_state, std::size_t n_qubits) -> std::string;
auto state_index_to_bitstring_big_endian(std::size_t i_state, std::size_t n_qubits) -> std::string;
auto state_index_to_dynamic_bitset_little_endian(std::size_t i_state, std::size_t n_qubits) -> std::vector<std::uint8_t>;
auto state_index_to_dynamic_bitset_big_endian(std::size_t i_state, std::size_t n_qubits) -> std::vector<std::uint8_t>;
auto dynamic_bitset_to_state_index_little_endian(const std::vector<std::uint8_t>& dyn_bitset) -> std::size_t;
auto dynamic_bitset_to_state_index_big_endian(const std::vector<std::uint8_t>& dyn_bitset) -> std::size_t;
// 0.b1 b2 b3 ... in base 2, b1 the first character (LITTLE) or the last (BIG)
auto binary_fraction_expansion(const std::string& bitstring, Endian endian = Endian::LITTLE) -> double;

// state/marginal.hpp:9-11: drop the marginal characters ('x') of a marginal
// bitstring from its right (left) end; they must all sit at that end.
auto rstrip_marginal_bits(const std::string& marginal_bitstring) -> std::string;
auto lstrip_marginal_bits(const std::string& marginal_bitstring) -> std::string;

class Statevector
{
public:
    explicit Statevector(std::size_t n_qubits, DType dtype = DType::C128);
    explicit Statevector(std::vector<std::complex<double>> coefficients, Endian input_endian = Endian::LITTLE,
                         double normalization_tolerance = CONSTRUCTION_NORMALIZATION_TOLERANCE,
                         DType dtype = DType::C128);
    explicit Statevector(const std::string& computational_state, Endian input_endian = Endian::LITTLE,
                         DType dtype = DType::C128);
    Statevector(const Statevector& other);
    Statevector(Statevector&& other) noexcept;
    auto operator=(const Statevector& other) -> Statevector&;
    auto operator=(Statevector&& other) noexcept -> Statevector&;
    ~Statevector();

    auto operator[](std::size_t index) const -> const std::complex<double>&;
    auto operator[](std::size_t index) -> std::complex<double>&;
    [[nodiscard]] auto at(std::size_t index) const -> const std::complex<double>&;
    auto at(std::size_t index) -> std::complex<double>&;
    [[nodiscard]] auto at(const std::string& bitstring, Endian endian = Endian::LITTLE) const -> const std::complex<double>&;
    auto at(const std::string& bitstring, Endian endian = Endian::LITTLE) -> std::complex<double>&;

    [[nodiscard]] auto n_states() const noexcept -> std::size_t { return n_states_; }
    [[nodiscard]] auto n_qubits() const noexcept -> std::size_t { return n_qubits_; }
    [[nodiscard]] auto dtype() const noexcept -> DType { return dtype_; }

    // engine access: the device handle, synchronised with the host mirror
    [[nodiscard]] auto device() const -> kt_sv;
    void mark_device_modified() const;   // the host mirror is stale after device work

private:
    std::size_t n_qubits_ {0};
    std::size_t n_states_ {0};
    DType dtype_ {DType::C128};
    kt_sv handle_ {nullptr};
    mutable std::vector<std::complex<double>> host_;
    mutable bool host_valid_ {false};   // host mirror matches the device
    mutable bool host_dirty_ {false};   // host mirror was written through a reference
    void pull_() const;
    void check_index_(std::size_t index) const;
};

auto almost_eq(const Statevector& left, const Statevector& right,
               double tolerance_sq = COMPLEX_ALMOST_EQ_TOLERANCE_SQ) noexcept -> bool;
auto inner_product(const Statevector& bra_state, const Statevector& ket_state) -> std::complex<double>;
auto inner_product_norm_squared(const Statevector& left, const Statevector& right) -> double;
// state/statevector.hpp:115,119: the left state's qubits are the low ones
auto tensor_product(const Statevector& left, const Statevector& right) -> Statevector;
auto diagonal_expectation_value(const std::vector<std::complex<double>>& eigenvalues, const Statevector& state)
    -> std::complex<double>;

// state/random.hpp:15-25: magnitudes uniform in [1e-3, 10) normalised, phases
// uniform in [0, 2 pi), drawn in that order; the state is built on the host
// and uploaded.  The seeded form starts a fresh std::mt19937(seed).
auto generate_random_state(std::size_t n_qubits, std::mt19937& prng) -> Statevector;
auto generate_random_state(std::size_t n_qubits, int seed) -> Statevector;
auto generate_random_state(std::size_t n_qubits) -> Statevector;

// state/project_state.hpp:18-23: the amplitudes whose qubits `qubit_indices`
// hold `expected_measurements`, renormalised, as a state of the remaining
// qubits (in their original order).  Throws when every qubit is projected,
// an index is out of range, a value is not 0 or 1, the two lists differ in
// length, or the remaining norm is below `minimum_norm_tol`.
auto project_statevector(const Statevector& statevector, const std::vector<std::size_t>& qubit_indices,
                         const std::vector<std::uint8_t>& expected_measurements,
                         double minimum_norm_tol = PROJECTION_NORMALIZATION_TOLERANCE) -> Statevector;

// Column-major N x N host matrix (element (r, c) at r + c * N), the element
// order of the reference's Eigen::MatrixXcd.
class HostMatrix
{
public:
    HostMatrix() = default;
    HostMatrix(std::ptrdiff_t rows, std::ptrdiff_t cols) : rows_ {rows}, cols_ {cols}, data_(static_cast<std::size_t>(rows * cols)) {}
    auto operator()(std::ptrdiff_t r, std::ptrdiff_t c) -> std::complex<double>& { return data_[static_cast<std::size_t>(r + c * rows_)]; }
    auto operator()(std::ptrdiff_t r, std::ptrdiff_t c) const -> const std::complex<double>& { return data_[static_cast<std::size_t>(r + c * rows_)]; }
    [[nodiscard]] auto rows() const noexcept -> std::ptrdiff_t { return rows_; }
    [[nodiscard]] auto cols() const noexcept -> std::ptrdiff_t { return cols_; }
    [[nodiscard]] auto size() const noexcept -> std::ptrdiff_t { return rows_ * cols_; }
    auto data() noexcept -> std::complex<double>* { return data_.data(); }
    [[nodiscard]] auto data() const noexcept -> const std::complex<double>* { return data_.data(); }

private:
    std::ptrdiff_t rows_ {0};
    std::ptrdiff_t cols_ {0};
    std::vector<std::complex<double>> data_;
};

struct density_matrix_nocheck
{};

class DensityMatrix
{
public:
    explicit DensityMatrix(HostMatrix matrix, const density_matrix_nocheck& key, DType dtype = DType::C128);
    explicit DensityMatrix(const std::string& bitstring, Endian input_endian = Endian::LITTLE, DType dtype = DType::C128);
    DensityMatrix(const DensityMatrix& other);
    DensityMatrix(DensityMatrix&& other) noexcept;
    auto operator=(const DensityMatrix& other) -> DensityMatrix&;
    auto operator=(DensityMatrix&& other) noexcept -> DensityMatrix&;
    ~DensityMatrix();

    [[nodiscard]] auto matrix() const -> const HostMatrix&;
    auto matrix() -> HostMatrix&;
    [[nodiscard]] auto n_states() const noexcept -> std::size_t { return n_states_; }
    [[nodiscard]] auto n_qubits() const noexcept -> std::size_t { return n_qubits_; }
    [[nodiscard]] auto trace() const -> std::complex<double>;
    // |Tr(rho^2) - 1|^2 <= tolerance (state/density_matrix.cpp, is_pure)
    [[nodiscard]] auto is_pure(double tolerance = DENSITY_MATRIX_TRACE_TOLERANCE) const -> bool;
    [[nodiscard]] auto trace_of_square() const -> std::complex<double>;

    [[nodiscard]] auto device() const -> kt_dm;
    void mark_device_modified() const;

private:
    // adopts a device matrix made by the engine (partial trace, tensor product)
    DensityMatrix(kt_dm handle, std::size_t n_qubits, DType dtype);
    friend auto partial_trace(const DensityMatrix& density_matrix, std::vector<std::size_t> qubit_indices) -> DensityMatrix;
    friend auto tensor_product(const DensityMatrix& left, const DensityMatrix& right) -> DensityMatrix;

    std::size_t n_qubits_ {0};
    std::size_t n_states_ {0};
    DType dtype_ {DType::C128};
    kt_dm handle_ {nullptr};
    mutable HostMatrix host_;
    mutable bool host_valid_ {false};
    mutable bool host_dirty_ {false};
    void pull_() const;
};

auto statevector_to_density_matrix(const Statevector& statevector) -> DensityMatrix;

// state/density_matrix.hpp:115-132.  The left factor's qubits are the low ones.
auto tensor_product(const DensityMatrix& left, const DensityMatrix& right) -> DensityMatrix;
auto tensor_product(const std::vector<DensityMatrix>& density_matrices) -> DensityMatrix;
// Trace over `qubit_indices`; tracing every qubit leaves the trace as a 1 x 1 matrix.
auto partial_trace(const DensityMatrix& density_matrix, std::vector<std::size_t> qubit_indices) -> DensityMatrix;

// ---- simulation ----------------------------------------------------------------------
class StatevectorSimulator
{
public:
    void run(const QuantumCircuit& circuit, Statevector& state, std::optional<int> prng_seed = std::nullopt);
    [[nodiscard]] auto has_been_run() const -> bool { return has_been_run_; }
    [[nodiscard]] auto classical_register() const -> const ClassicalRegister&;
    auto classical_register() -> ClassicalRegister&;
    [[nodiscard]] auto circuit_loggers() const -> const std::vector<CircuitLogger>& { return circuit_loggers_; }

private:
    std::optional<ClassicalRegister> cregister_;
    bool has_been_run_ {false};
    std::vector<CircuitLogger> circuit_loggers_;
};

class DensityMatrixSimulator
{
public:
    explicit DensityMatrixSimulator(std::size_t n_qubits) : n_qubits_ {n_qubits} {}
    void run(const QuantumCircuit& circuit, DensityMatrix& state, std::optional<int> prng_seed = std::nullopt);
    [[nodiscard]] auto has_been_run() const -> bool { return has_been_run_; }
    [[nodiscard]] auto classical_register() const -> const ClassicalRegister&;

private:
    std::size_t n_qubits_;
    std::optional<ClassicalRegister> cregister_;
    bool has_been_run_ {false};
};

void simulate(const QuantumCircuit& circuit, Statevector& state, std::optional<int> prng_seed = std::nullopt);
void simulate(const QuantumCircuit& circuit, DensityMatrix& state, std::optional<int> prng_seed = std::nullopt);

// ---- Pauli operators -------------------------------------------------------------------
class SparsePauliString;
enum class PauliTerm : std::uint8_t
{
    I,
    X,
    Y,
    Z,
};

enum class PauliPhase : std::uint8_t
{
    PLUS_ONE,
    PLUS_EYE,
    MINUS_ONE,
    MINUS_EYE,
};

extern const std::unordered_map<PauliPhase, std::complex<double>> PAULI_PHASE_MAP;

class SparsePauliString
{
public:
    explicit SparsePauliString(std::size_t n_qubits, PauliPhase phase = PauliPhase::PLUS_ONE);
    SparsePauliString(std::vector<std::pair<std::size_t, PauliTerm>> pauli_indexed_terms, std::size_t n_qubits,
                      PauliPhase phase = PauliPhase::PLUS_ONE);
    SparsePauliString(const std::vector<PauliTerm>& pauli_terms, PauliPhase phase = PauliPhase::PLUS_ONE);  // NOLINT
    SparsePauliString(const std::initializer_list<PauliTerm>& pauli_terms, PauliPhase phase = PauliPhase::PLUS_ONE);  // NOLINT

    void set_phase(PauliPhase phase) noexcept { phase_ = phase; }
    [[nodiscard]] auto phase() const noexcept -> PauliPhase { return phase_; }
    [[nodiscard]] auto n_qubits() const noexcept -> std::size_t { return n_qubits_; }
    [[nodiscard]] auto terms() const noexcept -> const std::vector<std::pair<std::size_t, PauliTerm>>& { return terms_; }
    [[nodiscard]] auto size() const noexcept -> std::size_t { return terms_.size(); }
    [[nodiscard]] auto at(std::size_t qubit_index) const -> PauliTerm;
    void add(std::size_t qubit_index, PauliTerm term);
    void overwrite(std::size_t qubit_index, PauliTerm term);
    void remove(std::size_t qubit_index);
    [[nodiscard]] auto contains_index(std::size_t qubit_index) const noexcept -> bool;
    // operator/pauli/sparse_pauli_string.hpp:116-119: the same qubit count and the
    // same non-identity terms on the same qubits (in any order); == also
    // compares the phase
    [[nodiscard]] auto equal_up_to_phase(const SparsePauliString& other) const -> bool;
    friend auto operator==(const SparsePauliString& left, const SparsePauliString& right) -> bool;

    // The string as X/Z masks with its total phase (terms applied in order, as
    // simulate(SparsePauliString) applies them, simulate_pauli.cpp:58-87).
    [[nodiscard]] auto to_record() const -> kt_pauli;

private:
    std::size_t n_qubits_;
    PauliPhase phase_ {};
    std::vector<std::pair<std::size_t, PauliTerm>> terms_;
};

struct WeightedPauliString
{
    std::complex<double> coefficient;
    SparsePauliString pauli_string;
};

class PauliOperator
{
public:
    explicit PauliOperator(std::size_t n_qubits);
    PauliOperator(std::vector<WeightedPauliString> weighted_pauli_strings);  // NOLINT
    PauliOperator(const std::initializer_list<WeightedPauliString>& weighted_pauli_strings);

    [[nodiscard]] auto n_qubits() const noexcept -> std::size_t { return n_qubits_; }
    [[nodiscard]] auto size() const noexcept -> std::size_t { return strings_.size(); }
    [[nodiscard]] auto weighted_pauli_strings() const noexcept -> const std::vector<WeightedPauliString>& { return strings_; }
    [[nodiscard]] auto at(std::size_t index) const -> const WeightedPauliString& { return strings_[index]; }
    auto at(std::size_t index) -> WeightedPauliString& { return strings_[index]; }
    void add(WeightedPauliString value);
    void add(std::complex<double> coefficient, SparsePauliString pauli_string);
    void remove(std::size_t index);

private:
    std::size_t n_qubits_;
    std::vector<WeightedPauliString> strings_;
};

// simulation/simulate_pauli.hpp:11-23: the string's X / Y / Z gates applied to
// the state in term order (its phase is not applied)
class StatevectorPauliStringSimulator
{
public:
    void run(const SparsePauliString& pauli_string, Statevector& state);
    [[nodiscard]] auto has_been_run() const -> bool { return has_been_run_; }

private:
    bool has_been_run_ {false};
};

void simulate(const SparsePauliString& pauli_string, Statevector& state);

auto expectation_value(const PauliOperator& pauli_op, const Statevector& state) -> std::complex<double>;
auto expectation_value(const SparsePauliString& sparse_pauli_string, const Statevector& state) -> std::complex<double>;
auto expectation_value(const PauliOperator& pauli_op, const DensityMatrix& state) -> std::complex<double>;

// ---- probabilities and measurements ----------------------------------------------------
class QuantumNoise
{
public:
    explicit QuantumNoise(std::size_t n_qubits);
    void set(std::size_t index, double noise);
    [[nodiscard]] auto get(std::size_t index) const -> const double&;
    [[nodiscard]] auto values() const noexcept -> const std::vector<double>& { return noise_; }

private:
    std::size_t n_qubits_;
    std::vector<double> noise_;
};

auto calculate_probabilities_raw(const Statevector& state, const QuantumNoise* noise = nullptr) -> std::vector<double>;
auto calculate_probabilities(const Statevector& state, const QuantumNoise* noise = nullptr)
    -> std::map<std::string, double>;

// calculations/measurements.hpp:40-97: the overloads on a probability vector
// sample it on the device with the same sampler as the state overloads
auto perform_measurements_as_memory(const std::vector<double>& probabilities_raw, std::size_t n_shots,
                                    std::optional<int> seed = std::nullopt) -> std::vector<std::size_t>;
auto perform_measurements_as_counts_raw(const std::vector<double>& probabilities_raw, std::size_t n_shots,
                                        std::optional<int> seed = std::nullopt) -> std::map<std::size_t, std::size_t>;
auto perform_measurements_as_counts_marginal(const std::vector<double>& probabilities_raw, std::size_t n_shots,
                                             const std::vector<std::size_t>& marginal_qubits = {},
                                             std::optional<int> seed = std::nullopt)
    -> std::map<std::string, std::size_t>;
// every shot simulates the circuit on a copy of the state and draws one
// index with a sampler seeded anew (calculations/measurements.cpp:179-207)
auto perform_measurements_as_counts_marginal(const QuantumCircuit& circuit, const Statevector& original_state,
                                             std::size_t n_shots, const std::vector<std::size_t>& marginal_qubits = {},
                                             const QuantumNoise* noise = nullptr,
                                             std::optional<int> seed = std::nullopt)
    -> std::map<std::string, std::size_t>;
auto perform_measurements_as_memory(const Statevector& state, std::size_t n_shots, const QuantumNoise* noise = nullptr,
                                    std::optional<int> seed = std::nullopt) -> std::vector<std::size_t>;
auto perform_measurements_as_counts_raw(const Statevector& state, std::size_t n_shots,
                                        const QuantumNoise* noise = nullptr, std::optional<int> seed = std::nullopt)
    -> std::map<std::size_t, std::size_t>;
auto perform_measurements_as_counts_marginal(const Statevector& state, std::size_t n_shots,
                                             const std::vector<std::size_t>& marginal_qubits = {},
                                             const QuantumNoise* noise = nullptr,
                                             std::optional<int> seed = std::nullopt) -> std::map<std::string, std::size_t>;
auto perform_measurements_as_counts(const Statevector& state, std::size_t n_shots, const QuantumNoise* noise = nullptr,
                                    std::optional<int> seed = std::nullopt) -> std::map<std::string, std::size_t>;
auto memory_to_counts(const std::vector<std::size_t>& measurements) -> std::map<std::size_t, std::size_t>;
auto memory_to_fractions(const std::vector<std::size_t>& measurements) -> std::map<std::size_t, double>;

// ---- adjoint gradient (new) ----------------------------------------------------------------
// E = Re <psi|H|psi> with psi = circuit applied to `initial`, and dE/dp for
// every circuit parameter (chain rule over every gate bound to it).
struct EnergyAndGradient
{
    double energy;
    std::unordered_map<param::ParameterID, double, param::ParameterIdHash> gradient;
};

auto adjoint_gradient(const QuantumCircuit& circuit, const Statevector& initial, const PauliOperator& hamiltonian,
                      int checkpoint_every = 0) -> EnergyAndGradient;

}  // namespace ket
