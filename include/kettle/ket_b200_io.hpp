// ket_b200_io.hpp — kettle's on-disk formats for states and Hamiltonians.
//
// Mirrors include/kettle/io/{statevector,numpy_statevector,read_pauli_operator}.hpp
// of the reference: the same functions, text formats and error messages.  A
// loaded state goes to the device with its first use.
#pragma once

#include <filesystem>
#include <iosfwd>

#include "kettle/ket_b200.hpp"

namespace ket
{

// io/statevector.cpp:60-156: "ENDIANNESS: <LITTLE|BIG>", "NUMBER OF STATES: <n>",
// then one "re   im" line per amplitude, fixed with 14 digits, a space in place
// of the sign of non-negative values.
void save_statevector(std::ostream& outstream, const Statevector& state, Endian endian = Endian::LITTLE);
void save_statevector(const std::filesystem::path& filepath, const Statevector& state, Endian endian = Endian::LITTLE);
auto load_statevector(std::istream& instream) -> Statevector;
auto load_statevector(const std::filesystem::path& filepath) -> Statevector;

// io/numpy_statevector.cpp: the number of qubits, then 2^n values "(re+imj)"
auto read_numpy_statevector(std::istream& instream, Endian input_endian = Endian::LITTLE) -> Statevector;
auto read_numpy_statevector(const std::filesystem::path& filepath, Endian input_endian = Endian::LITTLE) -> Statevector;

// io/read_pauli_operator.cpp:29-79: one term per line, "re im : (q, X) (q, Z) ..."
auto read_pauli_operator(std::istream& instream, std::size_t n_qubits) -> PauliOperator;
auto read_pauli_operator(const std::filesystem::path& filepath, std::size_t n_qubits) -> PauliOperator;

}  // namespace ket
