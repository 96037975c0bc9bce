// ket_b200_io.cpp — kettle's text formats for states and Hamiltonians (host side).
#include "kettle/ket_b200_io.hpp"

#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace ket
{

namespace
{

auto endian_to_string(Endian endian) -> std::string
{
    return endian == Endian::BIG ? "BIG" : "LITTLE";
}

auto string_to_endian(const std::string& endian) -> Endian
{
    if (endian == "BIG") {
        return Endian::BIG;
    }
    if (endian == "LITTLE") {
        return Endian::LITTLE;
    }
    throw std::runtime_error {"UNREACHABLE: dev error in `string_to_endian()`"};
}

// one "re   im" line, as std::fixed << std::setprecision(14) prints it, with a
// space in place of the sign of a non-negative value
void append_complex(std::string& out, const std::complex<double>& v)
{
    char buf[64];
    if (v.real() >= 0.0) {
        out.push_back(' ');
    }
    int k = std::snprintf(buf, sizeof(buf), "%.14f", v.real());
    out.append(buf, static_cast<std::size_t>(k));
    out.append("   ");
    if (v.imag() >= 0.0) {
        out.push_back(' ');
    }
    k = std::snprintf(buf, sizeof(buf), "%.14f", v.imag());
    out.append(buf, static_cast<std::size_t>(k));
    out.push_back('\n');
}

}  // namespace

void save_statevector(std::ostream& outstream, const Statevector& state, Endian endian)
{
    outstream << "ENDIANNESS: " << endian_to_string(endian) << '\n';
    outstream << "NUMBER OF STATES: " << state.n_states() << '\n';
    std::string chunk;
    chunk.reserve(1 << 20);
    for (std::size_t i = 0; i < state.n_states(); ++i) {
        const std::size_t j = (endian == Endian::LITTLE) ? i : endian_flip(i, state.n_qubits());
        append_complex(chunk, state[j]);
        if (chunk.size() > (1u << 20) - 128) {
            outstream << chunk;
            chunk.clear();
        }
    }
    outstream << chunk;
}

void save_statevector(const std::filesystem::path& filepath, const Statevector& state, Endian endian)
{
    auto outstream = std::ofstream {filepath};
    if (!outstream.is_open()) {
        std::ostringstream err;
        err << "ERROR: unable to open file to save statevector: \n";
        err << "'" << filepath << "'\n";
        throw std::ios::failure {err.str()};
    }
    save_statevector(outstream, state, endian);
}

auto load_statevector(std::istream& instream) -> Statevector
{
    std::string dummy;
    std::string endian_str;
    instream >> dummy >> endian_str;  // ENDIANNESS: <endian>
    const Endian endian = string_to_endian(endian_str);
    std::size_t n_states = 0;
    instream >> dummy >> dummy >> dummy >> n_states;  // NUMBER OF STATES: <n>
    std::vector<std::complex<double>> amplitudes;
    amplitudes.reserve(n_states);
    for (std::size_t i = 0; i < n_states; ++i) {
        double re = 0.0, im = 0.0;
        instream >> re >> im;
        amplitudes.emplace_back(re, im);
    }
    return Statevector {std::move(amplitudes), endian};
}

auto load_statevector(const std::filesystem::path& filepath) -> Statevector
{
    auto instream = std::ifstream {filepath};
    if (!instream.is_open()) {
        std::ostringstream err;
        err << "ERROR: unable to open file to load statevector: \n";
        err << "'" << filepath << "'\n";
        throw std::ios::failure {err.str()};
    }
    return load_statevector(instream);
}

auto read_numpy_statevector(std::istream& instream, Endian input_endian) -> Statevector
{
    std::size_t n_qubits = 0;
    instream >> n_qubits;
    const std::size_t n_states = std::size_t {1} << n_qubits;
    std::vector<std::complex<double>> amplitudes;
    amplitudes.reserve(n_states);
    for (std::size_t i = 0; i < n_states; ++i) {
        // "(1.23456e005+5.43210e002j)"
        double re = 0.0, im = 0.0;
        char ch = 0;
        instream >> ch >> re >> im >> ch >> ch;
        amplitudes.emplace_back(re, im);
    }
    return Statevector {std::move(amplitudes), input_endian};
}

auto read_numpy_statevector(const std::filesystem::path& filepath, Endian input_endian) -> Statevector
{
    auto instream = std::ifstream {filepath};
    if (!instream.is_open()) {
        std::ostringstream err;
        err << "ERROR: unable to open file for statevector: \n";
        err << "'" << filepath << "'\n";
        throw std::ios::failure {err.str()};
    }
    return read_numpy_statevector(instream, input_endian);
}

auto read_pauli_operator(std::istream& instream, std::size_t n_qubits) -> PauliOperator
{
    auto pauli_op = PauliOperator {n_qubits};
    std::string line;
    while (std::getline(instream, line)) {
        std::istringstream ls {line};
        double re = 0.0, im = 0.0;
        char ch = 0;
        ls >> re >> im >> ch;  // "re im :"
        auto pauli_string = SparsePauliString {n_qubits};
        while (ls >> ch) {
            if (ch == '(') {
                std::size_t qubit = 0;
                char gate = 0;
                ls >> qubit >> ch >> gate >> ch;  // "q, G)"
                switch (gate) {
                    case 'X': pauli_string.add(qubit, PauliTerm::X); break;
                    case 'Y': pauli_string.add(qubit, PauliTerm::Y); break;
                    case 'Z': pauli_string.add(qubit, PauliTerm::Z); break;
                    default: throw std::out_of_range {"_Map_base::at"};
                }
            }
        }
        pauli_op.add(std::complex<double> {re, im}, std::move(pauli_string));
    }
    return pauli_op;
}

auto read_pauli_operator(const std::filesystem::path& filepath, std::size_t n_qubits) -> PauliOperator
{
    auto instream = std::ifstream {filepath};
    if (!instream.is_open()) {
        throw std::ios::failure {std::string {"ERROR: unable to open: "} + filepath.string()};
    }
    return read_pauli_operator(instream, n_qubits);
}

}  // namespace ket
