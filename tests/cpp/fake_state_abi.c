/* fake_state_abi.c — host-memory stand-ins for the six state calls of the
 * C-ABI that the ket:: front end's Statevector uses to hold a state
 * (kt_sv_create, kt_sv_destroy, kt_sv_set_basis, kt_sv_upload, kt_sv_download,
 * kt_sv_copy), complex128 only.  Test infrastructure: preloaded into the
 * front end's host-utility program, it lets the CPU suite check the front
 * end's host-side state logic (random states, projections) without a GPU.
 * The engine itself is checked on the GPU through the real library.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "kettle_b200.h"

struct kt_sv_s
{
    uint64_t n_amps;
    double* amps; /* interleaved re, im */
};

int32_t kt_sv_create(int32_t n_qubits, int32_t dtype, kt_sv* out)
{
    if (n_qubits < 1 || n_qubits > 30 || dtype != KT_C128 || !out) {
        return KT_ERR_INVALID;
    }
    struct kt_sv_s* s = (struct kt_sv_s*)calloc(1, sizeof(struct kt_sv_s));
    if (!s) {
        return KT_ERR_NOMEM;
    }
    s->n_amps = (uint64_t)1 << n_qubits;
    s->amps = (double*)calloc(2 * s->n_amps, sizeof(double));
    if (!s->amps) {
        free(s);
        return KT_ERR_NOMEM;
    }
    s->amps[0] = 1.0;
    *out = s;
    return KT_OK;
}

int32_t kt_sv_destroy(kt_sv sv)
{
    if (sv) {
        free(sv->amps);
        free(sv);
    }
    return KT_OK;
}

int32_t kt_sv_set_basis(kt_sv sv, uint64_t index)
{
    if (!sv || index >= sv->n_amps) {
        return KT_ERR_INVALID;
    }
    memset(sv->amps, 0, 2 * sv->n_amps * sizeof(double));
    sv->amps[2 * index] = 1.0;
    return KT_OK;
}

int32_t kt_sv_upload(kt_sv sv, const double* host_amps, uint64_t n_amps)
{
    if (!sv || !host_amps || n_amps != sv->n_amps) {
        return KT_ERR_INVALID;
    }
    memcpy(sv->amps, host_amps, 2 * n_amps * sizeof(double));
    return KT_OK;
}

int32_t kt_sv_download(kt_sv sv, double* host_amps, uint64_t n_amps)
{
    if (!sv || !host_amps || n_amps != sv->n_amps) {
        return KT_ERR_INVALID;
    }
    memcpy(host_amps, sv->amps, 2 * n_amps * sizeof(double));
    return KT_OK;
}

int32_t kt_sv_copy(kt_sv dst, kt_sv src)
{
    if (!dst || !src || dst->n_amps != src->n_amps) {
        return KT_ERR_INVALID;
    }
    memcpy(dst->amps, src->amps, 2 * src->n_amps * sizeof(double));
    return KT_OK;
}
