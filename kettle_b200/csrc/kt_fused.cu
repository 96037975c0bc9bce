// kt_fused.cu — fused gate blocks (placeholder: one sweep per gate until the
// tiled kernel lands).
#include "kt_internal.cuh"

namespace kt
{

int32_t apply_fused(State& s, const std::vector<LGate>& gates)
{
    for (const auto& g : gates) {
        if (const int32_t rc = launch_gate_sweep(s, g); rc != KT_OK) {
            return rc;
        }
    }
    return KT_OK;
}

}  // namespace kt
