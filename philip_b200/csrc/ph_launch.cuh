// Launch entry points, one explicit instantiation set per polynomial order
// (ph_inst.cu is compiled once per N1 = p + 1 so the orders build in parallel).
#pragma once
#include <cuda_runtime.h>
#include "ph_kernels.cuh"
#include "ph_integrals.cuh"

namespace ph {

// residual / mass-inverse / RK stage for one stage input
template <int N1>
cudaError_t launch_stage(const StageArgs& a, int fp32, bool visc, bool split, cudaStream_t s);
// auxiliary (lifted gradient) equation, emitting the nodal viscous flux
template <int N1>
cudaError_t launch_aux(const double* U, const int* nbr, const OpTab* ops, int nc, double inv_h,
                       const PhysConst& pc, int fp32, double* Fv, cudaStream_t s);
// DGBase::apply_inverse_global_mass_matrix on its own
template <int N1>
cudaError_t launch_inverse_mass(const double* in, double* out, const OpTab* ops, int nc, double inv_detj,
                                const double* metric, cudaStream_t s);
// Taylor-Green integrals, per-cell partial sums
// X: node coordinates [nc][3][NP] of curvilinear cells, nullptr on affine meshes
template <int N1>
cudaError_t launch_integrals(const double* U, const double* X, const IntegralTab* tab, int nc, double h, double gam,
                             double gm1, double* partial, cudaStream_t s);
// shared memory and threads of the residual kernel (for reporting / tests)
template <int N1>
void stage_launch_shape(int fp32, bool visc, bool split, int* threads, int* cells_per_cta, size_t* smem);

} // namespace ph
