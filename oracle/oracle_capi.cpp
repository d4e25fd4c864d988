// C entry points of the CPU oracle, loaded by the test-suite and by the CPU-baseline
// leg of bench.py through ctypes. TEST INFRASTRUCTURE ONLY: nothing in the product
// library links against this file.
#include <cstring>
#include <exception>
#include <cstdio>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "dg_oracle.hpp"

using oracle::Params;
using oracle::Solver;

extern "C" {

struct orc_params {
    int poly_degree, overintegration, flux_nodes, pde, use_split_form, two_point, conv_flux, diss_flux;
    int fr_type, fr_aux_type, rk_method, use_constant_viscosity, non_physical, use_rrk;
    double fr_user_value, gamma, mach_inf, reynolds_inf, prandtl, temperature_inf, constant_viscosity,
        sipg_penalty_factor, atol, rtol, rrk_tol;
    int limiter;
    double min_density;
    double angle_of_attack, side_slip_angle;   // radians
    int thermal_bc;
    double wall_temperature;
    int bc_projected;
};

static Params to_params(const orc_params* p) {
    Params q;
    q.poly_degree = p->poly_degree; q.overintegration = p->overintegration; q.flux_nodes = p->flux_nodes;
    q.pde = p->pde; q.use_split_form = p->use_split_form; q.two_point = p->two_point;
    q.conv_flux = p->conv_flux; q.diss_flux = p->diss_flux; q.fr_type = p->fr_type;
    q.fr_aux_type = p->fr_aux_type; q.fr_user_value = p->fr_user_value; q.rk_method = p->rk_method;
    q.gamma = p->gamma; q.mach_inf = p->mach_inf; q.reynolds_inf = p->reynolds_inf; q.prandtl = p->prandtl;
    q.temperature_inf = p->temperature_inf; q.use_constant_viscosity = p->use_constant_viscosity;
    q.constant_viscosity = p->constant_viscosity; q.sipg_penalty_factor = p->sipg_penalty_factor;
    q.non_physical = p->non_physical;
    q.atol = p->atol; q.rtol = p->rtol;
    q.use_rrk = p->use_rrk; q.rrk_tol = p->rrk_tol;
    q.limiter = p->limiter; q.min_density = p->min_density;
    q.angle_of_attack = p->angle_of_attack; q.side_slip_angle = p->side_slip_angle;
    q.thermal_bc = p->thermal_bc; q.wall_temperature = p->wall_temperature;
    q.bc_projected = p->bc_projected;
    return q;
}

int orc_create(const orc_params* p, int n, double left, double right, int order, void** out) {
    try {
        Solver* s = new Solver();
        s->init(to_params(p), n, left, right, order);
        *out = s;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "orc_create: %s\n", e.what());
        return 1;
    }
}
// curvilinear periodic cube: sine warp of amplitude `warp`, mapping of degree grid_degree
int orc_create_curved(const orc_params* p, int n, double left, double right, int order, double warp,
                      int grid_degree, void** out) {
    try {
        Solver* s = new Solver();
        s->init(to_params(p), n, left, right, order, warp, grid_degree);
        *out = s;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "orc_create_curved: %s\n", e.what());
        return 1;
    }
}
// non-periodic sides of the cube (types[6]: x-, x+, y-, y+, z-, z+; 0 periodic)
int orc_set_boundaries(void* h, const int* types) {
    try {
        static_cast<Solver*>(h)->set_boundaries(types);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "orc_set_boundaries: %s\n", e.what());
        return 1;
    }
}
// the boundary states at one face node: g and gb_visc are [5][3]
int orc_boundary_values(void* h, int type, const double* n, const double* u, const double* g, double* ub_conv,
                        double* ub_visc, double* gb_visc) {
    try {
        static_cast<Solver*>(h)->boundary_values(type, n, u, g, ub_conv, ub_visc, gb_visc);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "orc_boundary_values: %s\n", e.what());
        return 1;
    }
}
// weighted RMS error estimate of the last low-storage step
double orc_rk_error(void* h) { return static_cast<Solver*>(h)->last_error; }
double orc_rrk_gamma(void* h) { return static_cast<Solver*>(h)->rrk_gamma; }
double orc_numerical_entropy(void* h, const double* U) { return static_cast<Solver*>(h)->numerical_entropy(U); }
void orc_destroy(void* h) { delete static_cast<Solver*>(h); }
long long orc_ndofs(void* h) { return (long long)static_cast<Solver*>(h)->ndofs(); }
int orc_nd(void* h) { return static_cast<Solver*>(h)->ops.nd; }
int orc_nq(void* h) { return static_cast<Solver*>(h)->ops.nq; }
int orc_status(void* h) { return static_cast<Solver*>(h)->status; }
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_cell_ijk(void* h, int* ijk) {
    Solver* s = static_cast<Solver*>(h);
    for (int c = 0; c < s->mesh.nc; ++c) for (int d = 0; d < 3; ++d) ijk[3 * c + d] = s->mesh.ijk[c][d];
}
void orc_node_xyz(void* h, double* xyz) {
    Solver* s = static_cast<Solver*>(h);
    std::memcpy(xyz, s->mesh.xnode.data(), s->mesh.xnode.size() * sizeof(double));
}
void orc_ops(void* h, double* xs, double* xq, double* wq) {
    Solver* s = static_cast<Solver*>(h);
    std::memcpy(xs, s->ops.xs.data(), s->ops.nd * sizeof(double));
    std::memcpy(xq, s->ops.xq.data(), s->ops.nq * sizeof(double));
    std::memcpy(wq, s->ops.wq.data(), s->ops.nq * sizeof(double));
}
void orc_minv(void* h, double* minv, double* minv_aux) {
    Solver* s = static_cast<Solver*>(h);
    std::memcpy(minv, s->ops.minv.data(), s->ops.minv.size() * sizeof(double));
    std::memcpy(minv_aux, s->ops.minv_aux.data(), s->ops.minv_aux.size() * sizeof(double));
}
void orc_initial_condition(void* h, double* U, int ic, const double* icp) { static_cast<Solver*>(h)->interpolate_ic(U, ic, icp); }
void orc_residual(void* h, const double* U, double* R) { static_cast<Solver*>(h)->assemble_residual(U, R); }
void orc_aux(void* h, double* out) {
    Solver* s = static_cast<Solver*>(h);
    std::memcpy(out, s->aux.data(), s->aux.size() * sizeof(double));
}
void orc_inverse_mass(void* h, const double* in, double* out) { static_cast<Solver*>(h)->apply_inverse_mass(in, out); }
int orc_rk_step(void* h, double* U, double dt) {
    try {
        static_cast<Solver*>(h)->rk_step(U, dt);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return 1;
    }
}
void orc_integrals(void* h, const double* U, double* out) { static_cast<Solver*>(h)->integrals(U, out); }
void orc_limit(void* h, double* U, double dt) { static_cast<Solver*>(h)->limit(U, dt); }
void orc_integrated_quantities(void* h, const double* U, double* out) {
    static_cast<Solver*>(h)->integrated_quantities(U, out);
}

}  // extern "C"
