// ket_b200_nlocal.hpp — integer ranges and the n-local ansatz builder, on the host.
//
// Mirrors include/kettle/common/arange.hpp and include/kettle/optimize/n_local.hpp
// of the reference: the same names, results and error messages.  An n-local
// circuit is an ordinary QuantumCircuit whose rotation angles are circuit
// parameters, so ket::adjoint_gradient and the engine's fused blocks take it
// as they take any other circuit.
#pragma once

#include <concepts>
#include <cstdint>
#include <stdexcept>
#include <tuple>
#include <variant>
#include <vector>

#include "kettle/ket_b200.hpp"

namespace ket
{

// common/arange.hpp:23-52: {0, 1, ..., value - 1} (empty for value <= 0), and
// {left, left + step, ...} short of `right` (step > 0) or above it (step < 0);
// step 0 throws; revarange is the same sequence reversed
template <std::integral Integer = std::size_t>
auto arange(Integer left, Integer right, std::int64_t step = 1) -> std::vector<Integer>
{
    if (step == 0) {
        throw std::runtime_error {"The `step` value cannot be 0 in `arange()`"};
    }
    std::vector<Integer> out;
    const auto lo = static_cast<std::int64_t>(left);
    const auto hi = static_cast<std::int64_t>(right);
    if (step > 0) {
        for (std::int64_t v = lo; v < hi; v += step) {
            out.push_back(static_cast<Integer>(v));
        }
    } else {
        for (std::int64_t v = lo; v > hi; v += step) {
            out.push_back(static_cast<Integer>(v));
        }
    }
    return out;
}

template <std::integral Integer = std::size_t>
auto arange(Integer value) -> std::vector<Integer>
{
    if (value <= 0) {
        return {};
    }
    return arange<Integer>(Integer {0}, value, 1);
}

template <std::integral Integer = std::size_t>
auto revarange(Integer value) -> std::vector<Integer>
{
    auto out = arange<Integer>(value);
    return {out.rbegin(), out.rend()};
}

template <std::integral Integer = std::size_t>
auto revarange(Integer left, Integer right, std::int64_t step = 1) -> std::vector<Integer>
{
    auto out = arange<Integer>(left, right, step);
    return {out.rbegin(), out.rend()};
}

// gates/compound_gate.hpp:13-18: gates appended as sequences of primitive gates
enum class CompoundGate : std::uint8_t
{
    CCX,
    CCY,
    CCZ
};

// optimize/n_local.hpp:12-42
inline constexpr auto DEFAULT_NLOCAL_GATE_PARAMETER = double {0.0};

using GeneralGate = std::variant<Gate, CompoundGate>;

enum class NLocalEntangelement : std::uint8_t
{
    FULL,
    LINEAR
};

enum class SkipLastRotationLayerFlag : std::uint8_t
{
    TRUE,
    FALSE
};

// n_qubits qubits; `n_repetitions` times a rotation layer then an
// entanglement layer, then a last rotation layer unless `flag` is TRUE.
// A rotation layer applies each rotation block in order: a one-qubit gate to
// every qubit, a controlled gate to the pairs (0, 1), (2, 3), ..., a doubly
// controlled compound gate to the triples (0, 1, 2), (3, 4, 5), ....  An
// entanglement layer applies each entanglement block (controlled or doubly
// controlled) to neighbouring pairs / triples (LINEAR) or to every ordered
// pair / triple (FULL).  Every angle gate gets a new circuit parameter of
// initial value DEFAULT_NLOCAL_GATE_PARAMETER; their IDs are returned in the
// order the gates were added.  Rotation blocks may not be U, CU or M;
// entanglement blocks must be controlled.
auto n_local(std::size_t n_qubits, const std::vector<GeneralGate>& rotation_blocks,
             const std::vector<GeneralGate>& entanglement_blocks, NLocalEntangelement entanglement_kind,
             std::size_t n_repetitions, SkipLastRotationLayerFlag flag = SkipLastRotationLayerFlag::FALSE)
    -> std::tuple<QuantumCircuit, std::vector<param::ParameterID>>;

}  // namespace ket
