// Launch entry points, one explicit instantiation set per polynomial order
// (ph_inst.cu is compiled once per N1 = p + 1 so the orders build in parallel).
#pragma once
#include <cuda_runtime.h>
#include "ph_kernels.cuh"
#include "ph_gl.cuh"
#include "ph_limiter.cuh"
#include "ph_integrals.cuh"

namespace ph {

// residual / mass-inverse / RK stage for one stage input, cells [a.cell_begin, a.nc)
template <int N1>
cudaError_t launch_stage(const StageArgs& a, int fp32, bool visc, bool split, cudaStream_t s);
// auxiliary (lifted gradient) equation, emitting the viscous terms of the stage kernel
// (viscous_terms_per_cell) of cells [cell_begin, nc); ops: the host copy of the operator table;
// metric: the curvilinear cells' metric rows (nullptr on affine cells)
// bnd: the boundary faces of a non-periodic mesh (nullptr on periodic meshes)
struct BoundaryArgs {
    const int* btype;   // boundary_id per boundary face (nullptr: the periodic kernel over `tiles`)
    void* Fb;           // [nb][4][NF] boundary viscous fluxes (in the arithmetic type)
    double pen;         // SIPG penalty of a boundary face (the cell's own)
    const int* tiles;   // first cell of each CTA's tile (ntiles CTAs)
    int ntiles;
};
template <int N1>
cudaError_t launch_aux(const double* U, const int* nbr, const OpTab& ops, int cell_begin, int nc, double inv_h,
                       const PhysConst& pc, int fp32, void* Fv, const double* metric, cudaStream_t s,
                       const BoundaryArgs* bnd = nullptr);
// DGBase::apply_inverse_global_mass_matrix on its own
template <int N1>
cudaError_t launch_inverse_mass(const double* in, double* out, const OpTab* ops, int nc, double inv_detj,
                                const double* metric, int fr, cudaStream_t s);
// Taylor-Green integrals, per-cell partial sums (integral_partials<full>() per cell)
// X: node coordinates [nc][3][NP] of curvilinear cells, nullptr on affine meshes;
// origin: lower corner [nc][3] of affine cells (the full set's angular momentum)
template <int N1>
cudaError_t launch_integrals(const double* U, const double* X, const double* origin, const IntegralTab* tab, int nc,
                             const IntegralConst& ic, bool full, double* partial, cudaStream_t s);
// Relaxation RK: integrated numerical entropy of u_n + gamma (u1 - u_n), per cell
template <int N1>
cudaError_t launch_rrk_entropy(const double* Un, const double* U1, double gamma, const OpTab* ops, int nc, double h3,
                               const double* metric, double gam, double* partial, cudaStream_t s);
// Batched (many-solve) stage: split-form Euler tiles of several discretisations of the same
// order. `variant` selects the cells-per-CTA tile shape (batched_shape lists them); grid <= 0
// sizes the persistent grid to the resident CTAs of the whole GPU; bnd: solves with boundary
// faces (the boundary-face instance).
template <int N1>
cudaError_t launch_stage_batched(const StageArgs* inst, const BatchTile* tiles, int ntiles, int fp32, bool curv,
                                 bool hot, int variant, int grid, cudaStream_t s, bool bnd = false);
// tile shape of a batched variant: cells per CTA, threads, dynamic shared memory and resident
// CTAs per SM; returns false when the variant does not exist
template <int N1>
bool batched_shape(int fp32, bool curv, int variant, int* cpc, int* threads, size_t* smem, int* ctas_per_sm);
// Uncollocated path (GL flux nodes / overintegration), N1 = p + 1 solution nodes and nq flux
// nodes per direction (N1 <= nq <= min(N1 + 2, 7)): kernel 0 = face values (gl_trace_kernel),
// 1 = auxiliary equation and viscous terms (gl_aux_kernel), 2 = residual / RK stage
// (gl_stage_kernel), 3 = the weight-adjusted inverse mass of curvilinear cells (gl_minv_kernel,
// a.U in, a.out out); one CTA per cell of [a.cell_begin, a.nc). g.vmet != nullptr: curvilinear.
template <int N1>
cudaError_t launch_gl(int kernel, int nq, const StageArgs& a, const GlArgs& g, const GlTab& ht, bool visc, bool split,
                      cudaStream_t s);
// Relaxation RK on uncollocated flux nodes (nq per direction): the integrated numerical entropy
// of u_n + gamma (u_1 - u_n) at the flux nodes, per cell (vmet: curvilinear cells' metric rows)
template <int N1>
cudaError_t launch_gl_rrk_entropy(int nq, const double* Un, const double* U1, double gamma, const GlTab& ht, int nc,
                                  double h3, const double* vmet, double gam, double* partial, cudaStream_t s);
// dKE/dt of state U with time derivative K, per-cell partial sums (affine cells)
template <int N1>
cudaError_t launch_ke_rate(const double* U, const double* K, const IntegralTab* tab, int nc, double h3,
                           double* partial, cudaStream_t s);
// positivity-preserving limiter on a.U, one CTA per cell
template <int N1>
cudaError_t launch_limiter(const LimiterArgs& a, cudaStream_t s);
// shared memory and threads of the residual kernel (for reporting / tests)
template <int N1>
void stage_launch_shape(int fp32, bool visc, bool split, int* threads, int* cells_per_cta, size_t* smem);

} // namespace ph
