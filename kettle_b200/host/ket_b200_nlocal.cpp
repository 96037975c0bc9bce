// ket_b200_nlocal.cpp — the n-local ansatz builder (optimize/n_local.cpp of
// the reference): host-side circuit construction with the same gate order,
// parameter order and error messages.
#include "kettle/ket_b200_nlocal.hpp"

#include <stdexcept>

namespace ket
{
namespace
{

enum class Shape
{
    ONE_TARGET,            // H .. SXDAG
    ONE_TARGET_ANGLE,      // RX, RY, RZ, P
    CONTROLLED,            // CH .. CSXDAG
    CONTROLLED_ANGLE,      // CRX, CRY, CRZ, CP
    OTHER                  // U, CU, M
};

auto shape_of(Gate g) -> Shape
{
    if (g >= Gate::H && g <= Gate::SXDAG) {
        return Shape::ONE_TARGET;
    }
    if (g >= Gate::RX && g <= Gate::P) {
        return Shape::ONE_TARGET_ANGLE;
    }
    if (g >= Gate::CH && g <= Gate::CSXDAG) {
        return Shape::CONTROLLED;
    }
    if (g >= Gate::CRX && g <= Gate::CP) {
        return Shape::CONTROLLED_ANGLE;
    }
    return Shape::OTHER;
}

void add_fixed(QuantumCircuit& c, Gate g, std::size_t t)
{
    switch (g) {
    case Gate::H: c.add_h_gate(t); break;
    case Gate::X: c.add_x_gate(t); break;
    case Gate::Y: c.add_y_gate(t); break;
    case Gate::Z: c.add_z_gate(t); break;
    case Gate::S: c.add_s_gate(t); break;
    case Gate::SDAG: c.add_sdag_gate(t); break;
    case Gate::T: c.add_t_gate(t); break;
    case Gate::TDAG: c.add_tdag_gate(t); break;
    case Gate::SX: c.add_sx_gate(t); break;
    case Gate::SXDAG: c.add_sxdag_gate(t); break;
    default: throw std::runtime_error {"DEV ERROR: invalid `Gate` found when applying rotation gates.\n"};
    }
}

auto add_angle(QuantumCircuit& c, Gate g, std::size_t t) -> param::ParameterID
{
    constexpr auto key = param::parameterized {};
    const double a = DEFAULT_NLOCAL_GATE_PARAMETER;
    switch (g) {
    case Gate::RX: return c.add_rx_gate(t, a, key);
    case Gate::RY: return c.add_ry_gate(t, a, key);
    case Gate::RZ: return c.add_rz_gate(t, a, key);
    case Gate::P: return c.add_p_gate(t, a, key);
    default: throw std::runtime_error {"DEV ERROR: invalid `Gate` found when applying rotation gates.\n"};
    }
}

void add_controlled(QuantumCircuit& c, Gate g, std::size_t ctrl, std::size_t t)
{
    switch (g) {
    case Gate::CH: c.add_ch_gate(ctrl, t); break;
    case Gate::CX: c.add_cx_gate(ctrl, t); break;
    case Gate::CY: c.add_cy_gate(ctrl, t); break;
    case Gate::CZ: c.add_cz_gate(ctrl, t); break;
    case Gate::CS: c.add_cs_gate(ctrl, t); break;
    case Gate::CSDAG: c.add_csdag_gate(ctrl, t); break;
    case Gate::CT: c.add_ct_gate(ctrl, t); break;
    case Gate::CTDAG: c.add_ctdag_gate(ctrl, t); break;
    case Gate::CSX: c.add_csx_gate(ctrl, t); break;
    case Gate::CSXDAG: c.add_csxdag_gate(ctrl, t); break;
    default: throw std::runtime_error {"DEV ERROR: invalid `Gate` found when applying entanglement gates.\n"};
    }
}

auto add_controlled_angle(QuantumCircuit& c, Gate g, std::size_t ctrl, std::size_t t) -> param::ParameterID
{
    constexpr auto key = param::parameterized {};
    const double a = DEFAULT_NLOCAL_GATE_PARAMETER;
    switch (g) {
    case Gate::CRX: return c.add_crx_gate(ctrl, t, a, key);
    case Gate::CRY: return c.add_cry_gate(ctrl, t, a, key);
    case Gate::CRZ: return c.add_crz_gate(ctrl, t, a, key);
    case Gate::CP: return c.add_cp_gate(ctrl, t, a, key);
    default: throw std::runtime_error {"DEV ERROR: invalid `Gate` found when applying entanglement gates.\n"};
    }
}

void add_doubly_controlled(QuantumCircuit& c, CompoundGate g, std::size_t c0, std::size_t c1, std::size_t t)
{
    switch (g) {
    case CompoundGate::CCX: c.add_ccx_gate(c0, c1, t); break;
    case CompoundGate::CCY: c.add_ccy_gate(c0, c1, t); break;
    case CompoundGate::CCZ: c.add_ccz_gate(c0, c1, t); break;
    }
}

// one rotation layer (optimize/n_local.cpp:117-158): one-qubit gates on every
// qubit, controlled gates on the disjoint pairs (2i, 2i + 1), doubly
// controlled gates on the disjoint triples (3i, 3i + 1, 3i + 2)
void rotation_layer(QuantumCircuit& c, const std::vector<GeneralGate>& blocks, std::vector<param::ParameterID>& ids)
{
    const std::size_t n = c.n_qubits();
    for (const auto& block : blocks) {
        if (const auto* cg = std::get_if<CompoundGate>(&block)) {
            for (std::size_t i = 0; i < n / 3; ++i) {
                add_doubly_controlled(c, *cg, 3 * i, 3 * i + 1, 3 * i + 2);
            }
            continue;
        }
        const Gate g = std::get<Gate>(block);
        switch (shape_of(g)) {
        case Shape::ONE_TARGET:
            for (std::size_t q = 0; q < n; ++q) {
                add_fixed(c, g, q);
            }
            break;
        case Shape::ONE_TARGET_ANGLE:
            for (std::size_t q = 0; q < n; ++q) {
                ids.push_back(add_angle(c, g, q));
            }
            break;
        case Shape::CONTROLLED:
            for (std::size_t i = 0; i < n / 2; ++i) {
                add_controlled(c, g, 2 * i, 2 * i + 1);
            }
            break;
        case Shape::CONTROLLED_ANGLE:
            for (std::size_t i = 0; i < n / 2; ++i) {
                ids.push_back(add_controlled_angle(c, g, 2 * i, 2 * i + 1));
            }
            break;
        case Shape::OTHER:
            throw std::runtime_error {"DEV ERROR: invalid `Gate` found when applying rotation gates.\n"};
        }
    }
}

// one entanglement layer (optimize/n_local.cpp:160-267): neighbouring pairs /
// triples (LINEAR) or every increasing pair / triple (FULL)
void entanglement_layer(QuantumCircuit& c, const std::vector<GeneralGate>& blocks, NLocalEntangelement kind,
                        std::vector<param::ParameterID>& ids)
{
    const std::size_t n = c.n_qubits();
    const bool full = kind == NLocalEntangelement::FULL;
    for (const auto& block : blocks) {
        if (const auto* cg = std::get_if<CompoundGate>(&block)) {
            if (!full) {
                // the reference counts to n - 2 in unsigned arithmetic, so one
                // qubit wraps around and its first triple fails the range check
                const std::size_t last = n == 1 ? 1 : (n < 2 ? 0 : n - 2);
                for (std::size_t q = 0; q < last; ++q) {
                    add_doubly_controlled(c, *cg, q, q + 1, q + 2);
                }
            } else {
                for (std::size_t a = 0; a + 2 < n; ++a) {
                    for (std::size_t b = a + 1; b + 1 < n; ++b) {
                        for (std::size_t t = b + 1; t < n; ++t) {
                            add_doubly_controlled(c, *cg, a, b, t);
                        }
                    }
                }
            }
            continue;
        }
        const Gate g = std::get<Gate>(block);
        const auto sh = shape_of(g);
        if (sh != Shape::CONTROLLED && sh != Shape::CONTROLLED_ANGLE) {
            throw std::runtime_error {"DEV ERROR: invalid `Gate` found when applying entanglement gates.\n"};
        }
        const auto add = [&](std::size_t ctrl, std::size_t t) {
            if (sh == Shape::CONTROLLED) {
                add_controlled(c, g, ctrl, t);
            } else {
                ids.push_back(add_controlled_angle(c, g, ctrl, t));
            }
        };
        if (!full) {
            for (std::size_t q = 0; q + 1 < n; ++q) {
                add(q, q + 1);
            }
        } else if (sh == Shape::CONTROLLED) {
            for (std::size_t ctrl = 0; ctrl + 1 < n; ++ctrl) {
                for (std::size_t t = ctrl + 1; t < n; ++t) {
                    add(ctrl, t);
                }
            }
        } else {
            // The reference's FULL loop for angle gates (n_local.cpp:188-192)
            // tests the control index where it means the target, so its target
            // runs past the last qubit and the adder's range check throws after
            // the pairs (0, 1) .. (0, n - 1); with one qubit it adds nothing.
            // The drop-in keeps both outcomes.
            for (std::size_t t = 1; n >= 2 && t <= n; ++t) {
                add(0, t);
            }
        }
    }
}

}  // namespace

auto n_local(std::size_t n_qubits, const std::vector<GeneralGate>& rotation_blocks,
             const std::vector<GeneralGate>& entanglement_blocks, NLocalEntangelement entanglement_kind,
             std::size_t n_repetitions, SkipLastRotationLayerFlag flag)
    -> std::tuple<QuantumCircuit, std::vector<param::ParameterID>>
{
    // optimize/n_local.cpp:19-50: the blocks are checked before anything is built
    for (const auto& block : rotation_blocks) {
        if (const auto* g = std::get_if<Gate>(&block); g && (*g == Gate::U || *g == Gate::CU || *g == Gate::M)) {
            throw std::runtime_error {"ERROR: cannot create n-local circuit with U, CU, or M gates.\n"};
        }
    }
    for (const auto& block : entanglement_blocks) {
        if (const auto* g = std::get_if<Gate>(&block)) {
            const auto sh = shape_of(*g);
            if (sh != Shape::CONTROLLED && sh != Shape::CONTROLLED_ANGLE) {
                throw std::runtime_error {"ERROR: entanglement gate must be controlled\n"};
            }
        }
    }
    auto circuit = QuantumCircuit {n_qubits};
    std::vector<param::ParameterID> ids;
    for (std::size_t r = 0; r < n_repetitions; ++r) {
        rotation_layer(circuit, rotation_blocks, ids);
        entanglement_layer(circuit, entanglement_blocks, entanglement_kind, ids);
    }
    if (flag == SkipLastRotationLayerFlag::FALSE) {
        rotation_layer(circuit, rotation_blocks, ids);
    }
    return {circuit, ids};
}

}  // namespace ket
