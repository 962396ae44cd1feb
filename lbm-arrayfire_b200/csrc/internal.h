// internal.h — declarations shared by the host-side translation units of liblbm_b200.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/lbm.h"
#include "mrt.cuh"

namespace lbm {

// Thread-local error message for lbm_last_error(); returns `code`.
int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);

#define LBM_CK(call)                                              \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return ::lbm::cuda_error(e_, #call); \
    } while (0)

// Relaxation coefficients (scale of the inverse transform folded in) for a basis and rates.
void mrt_coefficients(int basis, const double s[27], MrtCoef<double>& out);

// Validation of a descriptor; returns LBM_OK or an error (message set).
int validate_desc(const lbm_desc* d);

// Number of cells, populations per cell, bytes per stored population.
long long desc_cells(const lbm_desc* d);
int desc_q(const lbm_desc* d);
int storage_bytes(int storage);
double default_scale(int storage);

// Internals of a context used by the ensemble: fixed buffers f[0], f[1] and the device mask, and
// the current-buffer index after the ensemble has stepped it.
int ctx_buffers(lbm_ctx* c, void** f0, void** f1, const uint8_t** mask);
void ctx_set_current(lbm_ctx* c, int cur, bool has_prev, long long steps_added);

}  // namespace lbm
