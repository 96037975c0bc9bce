// dropin_host_main.cpp — the host-side utilities of the kettle API, built once
// against the reference library and once against the ket:: front end; both
// builds must print the same text.
//
//   dropin_host <mode>
//     host    bitstring / state-index / dynamic-bitset conversions, binary
//             fraction expansions, marginal strips, seeded random 2x2
//             unitaries, and the errors of each (no GPU is touched)
//     states  seeded random states and projections of them (the front end
//             keeps states on the GPU)
//
// Doubles are printed as hexadecimal floating point, so equal text means
// equal bits.  Uses only the public kettle API.
#include <complex>
#include <cstdint>
#include <cstdio>
#include <exception>
#include <random>
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
