// fm_adjoint.hpp — launchers of the exact-Jacobian and adjoint kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fm_kernels.hpp"

namespace fm {

// y = K_exact v (transpose = 0) or K_exact^T v (transpose = 1), full DOF set
void launch_exact_apply(const MeshDev& m, const double* u, const double* v, double* y,
                        int transpose, cudaStream_t s);
// per-element dL/dmu, dL/dlambda from an adjoint vector w
void launch_param_grads(const MeshDev& m, const double* u, const double* w, double* gmu,
                        double* glam, cudaStream_t s);
// r = g - y on free DOFs (0 on constrained), ||r||^2 into *out2
void launch_adj_residual(uint32_t n, const uint8_t* mask, const double* g, const double* y,
                         double* r, double* partials, unsigned* counter, double* out2,
                         cudaStream_t s);
// w += dw on free DOFs
void launch_adj_update(uint32_t n, const uint8_t* mask, const double* dw, double* w,
                       cudaStream_t s);

}  // namespace fm
