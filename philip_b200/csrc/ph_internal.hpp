// Host-side building blocks shared by the single-solve context (ph_capi.cu) and the
// batch of solves (ph_batch.cu): parameter checks, 1-D operators, physics constants,
// periodic-cube connectivity, node geometry / curvilinear metric terms and the RK
// stage arguments. Not part of the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/philip_b200.h"
#include "ph_gl.cuh"
#include "ph_integrals.cuh"
#include "ph_kernels.cuh"

namespace ph_host {

int fail(int code, const std::string& msg);   // records the message for ph_last_error

// Argument checks shared by every entry point that takes a mesh / parameters: PH_OK, or
// PH_ERR_INVALID with the message recorded (mesh size and bounds, cell_order 0..2 and the
// recursive-children order only for a power-of-two n; enumerations within their ranges).
int check_mesh(const ph_mesh_desc* mesh);
bool has_boundaries(const ph_mesh_desc* mesh);
// non-periodic meshes: nullptr when the boundary types are on the path, else the reason
const char* boundary_reason(const ph_mesh_desc* mesh, const ph_params* prm);
// boundary faces of the cube's non-periodic sides: nbr = -1 - k for boundary face k, btype[k] its type
void apply_boundaries(int n, const std::vector<int>& ijk, const int types[6], std::vector<int>& nbr,
                      std::vector<int>& btype);
int check_param_ranges(const ph_params* prm);

// Configuration checks shared by every entry point that builds a discretisation;
// returns nullptr when the configuration is on the GPU path, else the reason.
// unsupported_reason: the collocated kernels (GLL flux nodes, no overintegration);
// uncollocated_reason: a context on GL flux nodes or with overintegration.
const char* unsupported_reason(const ph_mesh_desc* mesh, const ph_params* prm);
bool uncollocated(const ph_params* prm);
const char* uncollocated_reason(const ph_mesh_desc* mesh, const ph_params* prm);
// 1-D operators of the uncollocated path; also sets ops.Minv to its FR mass inverse
int build_gl_operators(const ph_params* prm, ph::GlTab& t, ph::OpTab& ops);

// 1-D operators on the GLL nodes: D, skew D, FR mass inverse (M+K)^-1 and B = (M+K)^-1 W.
// x, D are the nodes and derivative matrix (N1 and N1 x N1). Returns PH_OK or an error.
int build_operators(const ph_params* prm, ph::OpTab& tab, bool& fr, std::vector<double>& x, std::vector<double>& D);

// QGauss(p + 11) tables of the TGV integrals for solution nodes x
void build_integral_table(const std::vector<double>& x, int p, ph::IntegralTab& tab);

// Physics constants of the kernels; the SIPG penalty (dg_base.cpp:397-413) for cell size h.
ph::PhysConst physics_constants(const ph_params* prm, double h, double& penalty);

// deal.II cell order (ijk, 3 per cell) and the 6 periodic neighbours of each cell.
void periodic_connectivity(int n, int order, std::vector<int>& ijk, std::vector<int>& nbr);

// Node coordinates [cell][node][3] and, for a curvilinear mesh (warp != 0 or given support
// points [cell][3][NP]), the metric rows [cell][10][NP];
// cells are processed by host threads. Returns PH_OK or an error (folded cell).
int node_geometry(int n, const std::vector<int>& ijk, const std::vector<double>& x, const std::vector<double>& D,
                  double left, double right, double warp, std::vector<double>& xyz, std::vector<double>& metric,
                  const double* support = nullptr);

// A solve's host-side set-up for a batch (operators, connectivity, geometry / metric terms),
// computed without the batch, so that it can run on the thread that submits the solve.
struct BatchPrep {
    ph::OpTab ops{};
    bool fr = false;
    bool ready = false;
    std::vector<int> nbr;
    std::vector<int> btype;   // boundary face k's type (nbr = -1 - k); empty on periodic meshes
    std::vector<double> metric;
};
int batch_prepare(const ph_mesh_desc* mesh, const ph_params* prm, BatchPrep& out);
// ph_batch_admit with the set-up done beforehand (prep may be nullptr: done here)
int batch_admit_prepared(ph_batch* b, const ph_mesh_desc* mesh, const ph_params* prm, const BatchPrep* prep,
                         const double* U0, double dt, int nsteps, int* slot);

// Device state of a context (its current solution, ndofs doubles) and the stream it is ordered on;
// of a batch slot likewise (the batch stream). For the snapshot matrix's device-to-device copies.
int ctx_state(ph_ctx* c, const double** d, size_t* n, cudaStream_t* stream);
int batch_state(ph_batch* b, int slot, const double** d, size_t* n, cudaStream_t* stream);

// a curvilinear mesh: warped, or given by its mapping support points
inline bool is_curvilinear(const ph_mesh_desc* mesh) {
    return mesh->warp != 0.0 || mesh->mapping_support_points != nullptr;
}

// Butcher tableau of the explicit RK method (runge_kutta_methods.cpp:7-47).
void rk_tableau(int method, int& ns, double A[4][4], double b[4]);

// Low-storage 3S* / 3S*+ tableau (low_storage_runge_kutta_methods.cpp; Ketcheson 2010 for
// RK4(3)5[3S*], Ranocha, Dalcin, Parsani and Ketcheson 2021 for the [3S*+] methods).
struct LowStorageTableau {
    int ns = 0;                 // stages
    int num_delta = 0;          // delta entries summed for the embedded solution (3S*)
    int order = 0;
    bool plus = false;          // 3S*+: FSAL error register S4
    double gamma[11][3] = {};
    double beta[11] = {};
    double delta[11] = {};
    double bhat[11] = {};
};
// false when `method` is not a low-storage method (parameters_ode_solver.h:66-78 numbering)
bool low_storage_tableau(int method, LowStorageTableau& t);

// Device vectors of one explicit RK integration of one discretisation.
struct RkBuffers {
    double* sol;     // u_n, and u_{n+1} after the last stage
    double* stA;     // stage inputs (ping-pong)
    double* stB;
    double* acc;     // running sum of the stage derivatives
    double* carry;   // SSPRK3 carry (nullptr otherwise)
    double* comp;    // Kahan compensation of the precision form (nullptr otherwise)
};

// Stage input of stage i, and the RK epilogue arguments of stage i (mode 2) into a.
const double* rk_stage_input(const RkBuffers& B, int i);
void rk_stage_args(ph::StageArgs& a, const RkBuffers& B, int i, int ns, const double A[4][4], const double b[4],
                   double dt, bool fp32);
// Stage i of a low-storage step (i == ns: the 3S*+ FSAL evaluation). S2 lives in B.acc,
// S4 in B.carry, S3 = u_n = B.sol. Returns the stage input.
const double* lsrk_stage_args(ph::StageArgs& a, const RkBuffers& B, int i, const LowStorageTableau& t, double dt,
                              double atol, double rtol, double* err_partial);

} // namespace ph_host
