// ket_b200_circuit_ops.hpp — circuit transforms on the host: joining circuits
// and lowering U / CU gates to primitive gates.
//
// Mirrors include/kettle/circuit_operations/{append_circuits,transpile_to_primitive,compare_circuits}.hpp
// of the reference: the same functions, results and error messages.  The
// engine applies U and CU gates natively, so transpiling is never needed to
// simulate; it is here for code that inspects or exports primitive circuits.
#pragma once

#include "kettle/ket_b200.hpp"

namespace ket
{

// circuit_operations/append_circuits.cpp:26-41: the right circuit's elements
// and parameters after the left's; both need the same qubit and bit counts
void extend_circuit(QuantumCircuit& left, const QuantumCircuit& right);
auto append_circuits(QuantumCircuit left, const QuantumCircuit& right) -> QuantumCircuit;

// circuit_operations/transpile_to_primitive.cpp:15-91: every U becomes one
// primitive gate where it matches one within `tolerance_sq`, else RZ RY RZ
// (+ P for the determinant's phase); CU likewise with controlled gates.
// Primitive gates, M gates, loggers and (recursively) control flow are kept.
auto transpile_to_primitive(const QuantumCircuit& circuit, double tolerance_sq = COMPLEX_ALMOST_EQ_TOLERANCE_SQ)
    -> QuantumCircuit;

// circuit_operations/compare_circuits.hpp:42-46: gate by gate, loggers
// skipped.  Two gates match when they act on the same qubits with matrices
// within `tol_sq` (a primitive gate and a U gate of its matrix match);
// M gates match on qubit and bit; if / if-else statements on equal
// predicates and (recursively) matching subcircuits.  Angles bound to
// parameters take the circuit's parameter values (every parameter must have
// one).
auto almost_eq(const QuantumCircuit& left, const QuantumCircuit& right, double tol_sq = COMPLEX_ALMOST_EQ_TOLERANCE_SQ)
    -> bool;

}  // namespace ket
