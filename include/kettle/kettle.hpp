// kettle.hpp — umbrella header of the B200 engine's kettle-compatible C++20 API.
// Code written against the reference's <kettle/kettle.hpp> (namespace ket)
// compiles against this header for the circuit-propagation API it covers.
#pragma once

#include "kettle/ket_b200.hpp"
#include "kettle/ket_b200_io.hpp"
#include "kettle/ket_b200_circuit_ops.hpp"
#include "kettle/ket_b200_nlocal.hpp"
