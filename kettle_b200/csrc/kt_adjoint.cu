// kt_adjoint.cu — adjoint differentiation (entry points; kernels follow).
#include "kt_internal.cuh"

extern "C" {
int32_t kt_adjoint_create(kt_sv, int32_t, kt_adjoint* out)
{
    if (out) *out = nullptr;
    kt::set_error(KT_ERR_UNSUPPORTED, "adjoint not built yet");
    return KT_ERR_UNSUPPORTED;
}
int32_t kt_adjoint_destroy(kt_adjoint) { return KT_OK; }
int32_t kt_adjoint_forward(kt_adjoint, const kt_gate*, int64_t, const double*, int64_t, const kt_pauli*, int64_t,
                           const double*, double*)
{
    kt::set_error(KT_ERR_UNSUPPORTED, "adjoint not built yet");
    return KT_ERR_UNSUPPORTED;
}
int32_t kt_adjoint_backward(kt_adjoint, double*, int64_t)
{
    kt::set_error(KT_ERR_UNSUPPORTED, "adjoint not built yet");
    return KT_ERR_UNSUPPORTED;
}
int32_t kt_batch_run(const kt_batch_item*, int64_t, const kt_gate*, int64_t, const double*, int64_t, const kt_pauli*,
                     const double*, int64_t, int32_t, double*, double*, void*)
{
    kt::set_error(KT_ERR_UNSUPPORTED, "batch not built yet");
    return KT_ERR_UNSUPPORTED;
}
}
