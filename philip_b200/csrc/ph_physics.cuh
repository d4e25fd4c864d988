// Device-side Euler / Navier-Stokes physics and numerical fluxes for the GLL
// collocated strong-form DG/FR residual. Templated on the arithmetic type `R`
// (double for the plain path, float for the precision form).
//
// Reference behaviour followed:
//   pressure / primitive conversions ........ src/physics/euler.cpp:177-500
//   two-point split fluxes KG/IR/CH/Ra ...... src/physics/euler.cpp:563-809
//   Ismail-Roe logarithmic mean ............. src/physics/euler.cpp:628-646
//   convective flux ......................... src/physics/euler.cpp:915-938
//   Roe-Pike dissipation + Harten fix ....... src/numerical_flux/convective_numerical_flux.cpp:215-480
//   Lax-Friedrichs dissipation .............. src/numerical_flux/convective_numerical_flux.cpp:190-214
//   viscous flux (Sutherland, Stokes) ....... src/physics/navier_stokes.cpp:241-395, :755-830, :1198-1350
//   SIPG / BR2 auxiliary fluxes ............. src/numerical_flux/viscous_numerical_flux.cpp:146-328
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace ph {

enum TwoPointType { TP_KG = 0, TP_IR = 1, TP_CH = 2, TP_RA = 3 };
enum ConvFluxType { CF_LXF = 0, CF_ROE = 1, CF_CENTRAL = 2, CF_EC = 3, CF_EC_LXF = 4, CF_EC_ROE = 5 };
enum DissFluxType { DF_SIPG = 0, DF_BR2 = 1, DF_CENTRAL = 2 };

// status bits written by kernels (host reads them through ph_status)
// ST_COPY_TIMEOUT: a bulk copy into shared memory did not complete within the kernel's wait
// limit (the tile's outputs were not written)
enum StatusBits : unsigned { ST_NONPHYSICAL = 1u, ST_COPY_TIMEOUT = 2u };

constexpr double BIG_NUMBER = 1e100;   // physics.h:270

struct PhysConst {
    double gam, gm1, mach2, temp_ratio, inv_re, prandtl, const_visc, sipg_pen;
    double pressure_shift;   // precision form: reference pressure taken out of the momentum fluxes
    int use_const_visc, two_point, conv_flux, diss_flux, navier_stokes;
    // boundary conditions: the free stream (density 1, velocities v_inf, pressure 1/(gam M^2),
    // Euler::Euler, euler.cpp:14-70), the inlet totals of boundary_face_values (:1515-1516), the
    // Mach number, and the wall's thermal condition (isothermal: wall temperature t_wall)
    double bc_v_inf[3], bc_p_inf, bc_total_p, bc_total_t, bc_mach_inf, bc_t_wall;
    int bc_isothermal;
    int bc_projected;   // use_projected_entropy_variables_for_nsfr_boundary_term (uncollocated split form)
};

template <typename R> struct Cst {
    // p0: the constant subtracted from the pressure in every momentum flux of the precision
    // form. A constant pressure adds the same amount to the volume and the face terms, which
    // cancel exactly, so the residual is unchanged; in FP32 the large mean pressure of a
    // low-Mach flow (1/(gamma M^2) = 71 at M = 0.1) no longer swamps its O(1) variations.
    // Zero in FP64, whose arithmetic stays the reference's.
    R gam, gm1, mach2, temp_ratio, inv_re, prandtl, const_visc, kappa_fac, inv2gm1, p0;
    __device__ __forceinline__ void load(const PhysConst& c) {
        gam = (R)c.gam; gm1 = (R)c.gm1; mach2 = (R)c.mach2; temp_ratio = (R)c.temp_ratio;
        inv_re = (R)c.inv_re; prandtl = (R)c.prandtl; const_visc = (R)c.const_visc;
        kappa_fac = (R)(1.0 / (c.gm1 * c.mach2 * c.prandtl));
        inv2gm1 = (R)(0.5 / c.gm1);
        p0 = sizeof(R) == 4 ? (R)c.pressure_shift : R(0);
    }
    // the shift as the flux code uses it: a compile-time zero in FP64
    __device__ __forceinline__ R shift() const { return sizeof(R) == 4 ? p0 : R(0); }
};

template <typename R> __device__ __forceinline__ R rlog(R x);
template <> __device__ __forceinline__ double rlog<double>(double x) { return log(x); }
template <> __device__ __forceinline__ float rlog<float>(float x) { return logf(x); }
template <typename R> __device__ __forceinline__ R rsqrt_(R x);
template <> __device__ __forceinline__ double rsqrt_<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float rsqrt_<float>(float x) { return sqrtf(x); }
template <typename R> __device__ __forceinline__ R rpow(R x, R y);
template <> __device__ __forceinline__ double rpow<double>(double x, double y) { return pow(x, y); }
template <> __device__ __forceinline__ float rpow<float>(float x, float y) { return powf(x, y); }
template <typename R> __device__ __forceinline__ R rabs(R x) { return x < R(0) ? -x : x; }

// Quotient used inside the flux functions. PH_FAST_DIV=0: IEEE division. Otherwise the
// numerator times the hardware approximate reciprocal (PTX rcp.approx.ftz.f64/.f32,
// relative error about 1e-6 in FP64) refined by Newton-Raphson steps
// r <- r + r (1 - b r), each of which squares the relative error: two steps in FP64
// (about 2 ulp, measured against IEEE division in tests/test_gpu_quotient.py), none
// in FP32 (the f32 approximation is within about 1 ulp already).
#ifndef PH_FAST_DIV
#define PH_FAST_DIV 1
#endif
__device__ __forceinline__ double rcp_approx(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <typename R> __device__ __forceinline__ R qrcp(R b);
template <> __device__ __forceinline__ double qrcp<double>(double b) {
#if PH_FAST_DIV == 0
    return 1.0 / b;
#else
    double r = rcp_approx(b);
    r = fma(r, fma(-b, r, 1.0), r);
    r = fma(r, fma(-b, r, 1.0), r);
    return r;
#endif
}
template <> __device__ __forceinline__ float qrcp<float>(float b) {
#if PH_FAST_DIV == 0
    return 1.0f / b;
#else
    return rcp_approx(b);
#endif
}
template <typename R> __device__ __forceinline__ R qdiv(R a, R b) {
#if PH_FAST_DIV == 0
    return a / b;
#else
    return a * qrcp<R>(b);
#endif
}

// Non-physical handling: a negative density/pressure sets a status bit and is
// replaced by BIG_NUMBER, as check_positive_quantity does (euler.cpp:155-172).
template <typename R> __device__ __forceinline__ R positive(R q, unsigned* status) {
    if (q < R(0)) {
        if (status) atomicOr(status, ST_NONPHYSICAL);
        return (R)BIG_NUMBER;
    }
    return q;
}

template <typename R> __device__ __forceinline__ R pressure(const R u[5], R gm1, unsigned* st) {
    const R rho = u[0];
    R v2 = R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) { const R v = qdiv<R>(u[1 + d], rho); v2 = v2 + v * v; }
    return positive<R>(gm1 * (u[4] - R(0.5) * rho * v2), st);
}

// the same with IEEE division (boundary states)
template <typename R> __device__ __forceinline__ R pressure_ieee(const R u[5], R gm1, unsigned* st) {
    const R rho = u[0];
    R v2 = R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) { const R v = u[1 + d] / rho; v2 = v2 + v * v; }
    return positive<R>(gm1 * (u[4] - R(0.5) * rho * v2), st);
}

// Per-node quantities reused by every two-point flux that touches the node.
template <typename R> struct NodeQ {
    R rho, v[3], p, E;
    R a, b, la, lb;   // log-mean arguments and their logarithms (type dependent)
    R vsq;            // |v|^2 (CH, Ra) or specific total energy (KG)
};

template <typename R>
__device__ __forceinline__ void node_prepare(const R u[5], int tp, R gm1, NodeQ<R>& q, unsigned* st) {
    q.rho = u[0];
    R v2 = R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) { q.v[d] = qdiv<R>(u[1 + d], u[0]); v2 = v2 + q.v[d] * q.v[d]; }
    q.E = u[4];
    q.p = positive<R>(gm1 * (u[4] - R(0.5) * u[0] * v2), st);
    if (tp == TP_CH) {
        q.a = q.rho; q.b = qdiv<R>(q.rho, R(2) * q.p);
        q.la = rlog<R>(q.a); q.lb = rlog<R>(q.b);
        q.vsq = q.v[0] * q.v[0] + q.v[1] * q.v[1] + q.v[2] * q.v[2];
    } else if (tp == TP_RA) {
        q.a = q.rho; q.b = qdiv<R>(q.rho, q.p);
        q.la = rlog<R>(q.a); q.lb = rlog<R>(q.b);
        q.vsq = q.v[0] * q.v[0] + q.v[1] * q.v[1] + q.v[2] * q.v[2];
    } else if (tp == TP_IR) {
        const R rho = positive<R>(q.rho, st);
        q.a = rsqrt_<R>(qdiv<R>(rho, q.p));      // z_0
        q.b = rsqrt_<R>(rho * q.p);      // z_4
        q.la = rlog<R>(q.a); q.lb = rlog<R>(q.b);
        q.vsq = R(0);
    } else {   // KG
        q.a = q.b = q.la = q.lb = R(0);
        q.vsq = qdiv<R>(q.E, q.rho);
    }
}

// Logarithmic mean with the Ismail-Roe series branch (euler.cpp:628-646). The
// logarithms of the two arguments are taken once per node, so the log of the ratio
// is their difference; the branch test uses the reference's own ratio form.
//
// Division count: f = (a-b)/(a+b) equals the reference's (zeta-1)/(zeta+1) with
// zeta = a/b up to rounding, the series is evaluated in Horner form with the constant
// reciprocals, and (a+b) f / log(zeta) = (a-b)/(log a - log b); two divisions per call.
template <typename R>
__device__ __forceinline__ R log_mean(R a, R b, R la, R lb) {
    const R s = a + b, d = a - b;
    const R f = qdiv<R>(d, s);
    const R u = f * f;
    if (u < R(1.0e-2)) {
        const R F = R(1) + u * (R(1.0 / 3.0) + u * (R(1.0 / 5.0) + u * R(1.0 / 7.0)));
        return qdiv<R>(s, R(2) * F);
    }
    return qdiv<R>(d, la - lb);
}

// The series of log_mean: F(u) = 1 + u/3 + u^2/5 + u^3/7, Horner form.
template <typename R> __device__ __forceinline__ R log_mean_series(R u) {
    return R(1) + u * (R(1.0 / 3.0) + u * (R(1.0 / 5.0) + u * R(1.0 / 7.0)));
}

// Averages of the Chandrashekar flux (Euler::compute_chandrashekar_flux, euler.cpp): the
// logarithmic mean rho_log of the density, p_hat = mean(rho) / (2 mean(b)) and the scalar
// part of the enthalpy, h0 = 1 / (2 (gamma - 1) b_log) + p_hat / rho_log - mean(|v|^2) / 2.
// Both logarithmic means follow log_mean (the same branch test, series for u < 1e-2), with
// the quotients rearranged to share reciprocals: three when both means take the series
// branch (smooth flow), at most five, where the plain form divides six times.
template <typename R>
__device__ __forceinline__ void ch_means(const NodeQ<R>& i, const NodeQ<R>& j, const Cst<R>& c, R& rho_log,
                                         R& p_hat, R& h0) {
    const R srho = i.rho + j.rho, drho = i.rho - j.rho;
    const R sb = i.b + j.b, db = i.b - j.b;
    const R rsb = qrcp<R>(sb);
    p_hat = R(0.5) * srho * rsb;
    R inv_blog;
    {
        const R f = db * rsb, u = f * f;
        if (u < R(1.0e-2)) inv_blog = R(2) * log_mean_series<R>(u) * rsb;
        else inv_blog = (i.lb - j.lb) * qrcp<R>(db);
    }
    R inv_rlog;
    {
        const R rs = qrcp<R>(srho);
        const R f = drho * rs, u = f * f;
        if (u < R(1.0e-2)) {
            const R F = log_mean_series<R>(u);
            inv_rlog = R(2) * F * rs;
            rho_log = R(0.5) * srho * qrcp<R>(F);
        } else {
            const R dl = i.la - j.la;
            rho_log = drho * qrcp<R>(dl);
            inv_rlog = dl * qrcp<R>(drho);
        }
    }
    h0 = inv_blog * c.inv2gm1 + p_hat * inv_rlog - R(0.25) * (i.vsq + j.vsq);
}

// Two-point flux component along direction d (compile time) for all 5 equations.
template <typename R, int d>
__device__ __forceinline__ void two_point_dir(const NodeQ<R>& i, const NodeQ<R>& j, int tp,
                                              const Cst<R>& c, R F[5]) {
    if (tp == TP_CH) {
        R rho_log, p_hat, h0;
        ch_means<R>(i, j, c, rho_log, p_hat, h0);
        R va[3], vsq = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) { va[k] = R(0.5) * (i.v[k] + j.v[k]); vsq += va[k] * va[k]; }
        const R m = rho_log * va[d];
        F[0] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[1 + k] = m * va[k];
        F[1 + d] += p_hat - c.shift();
        F[4] = m * (h0 + vsq);
    } else if (tp == TP_RA) {
        const R rho_log = log_mean<R>(i.a, j.a, i.la, j.la);
        const R b_log = log_mean<R>(i.b, j.b, i.lb, j.lb);
        R va[3], vsq = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) { va[k] = R(0.5) * (i.v[k] + j.v[k]); vsq += va[k] * va[k]; }
        const R p_hat = R(0.5) * (i.p + j.p);
        const R gb = b_log * c.gm1;
        R H = qdiv<R>(rho_log + R(2) * gb * p_hat, gb * rho_log) + vsq;
        H -= R(0.5) * (R(0.5) * (i.vsq + j.vsq));
        const R m = rho_log * va[d];
        F[0] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[1 + k] = m * va[k];
        F[1 + d] += p_hat - c.shift();
        F[4] = m * H - R(0.5) * (i.p * i.v[d] + j.p * j.v[d]);
    } else if (tp == TP_IR) {
        const R z0a = R(0.5) * (i.a + j.a), z4a = R(0.5) * (i.b + j.b);
        const R l0 = log_mean<R>(i.a, j.a, i.la, j.la);
        const R l4 = log_mean<R>(i.b, j.b, i.lb, j.lb);
        const R rho = z0a * l4;
        R v[3], vv = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const R zk = R(0.5) * (i.a * i.v[k] + j.a * j.v[k]);
            v[k] = qdiv<R>(zk, z0a); vv += v[k] * v[k];
        }
        const R p = qdiv<R>(z4a, z0a);
        R H = (c.gam + R(1)) * qdiv<R>(l4, l0) + c.gm1 * p;
        H /= R(2) * c.gam;
        H *= qdiv<R>(c.gam, rho * c.gm1);
        H += R(0.5) * vv;
        const R m = rho * v[d];
        F[0] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[1 + k] = m * v[k];
        F[1 + d] += p - c.shift();
        F[4] = m * H;
    } else {   // KG
        const R rho = (i.rho + j.rho) / R(2);
        const R p = (i.p + j.p) / R(2);
        R v[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) v[k] = R(0.5) * (i.v[k] + j.v[k]);
        const R e = (i.vsq + j.vsq) / R(2);
        const R m = rho * v[d];
        F[0] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[1 + k] = m * v[k];
        F[1 + d] += p - c.shift();
        F[4] = m * e + p * v[d];
    }
}

// Physical convective flux along direction d (p0: the precision form's pressure shift).
template <typename R, int d>
__device__ __forceinline__ void conv_flux_dir(const NodeQ<R>& q, R p0, R F[5]) {
    const R H = qdiv<R>(q.E, q.rho) + qdiv<R>(q.p, q.rho);
    const R m = q.rho * q.v[d];
    F[0] = m;
#pragma unroll
    for (int k = 0; k < 3; ++k) F[1 + k] = m * q.v[k];
    F[1 + d] += q.p - p0;
    F[4] = m * H;
}

// Roe-Pike dissipation -1/2 |A_roe| (uR - uL) for the axis normal n = +e_d.
template <typename R, int d>
__device__ __forceinline__ void roe_dissipation(const NodeQ<R>& L, const NodeQ<R>& Rq,
                                                const Cst<R>& c, R out[5]) {
    const R n[3] = {R(d == 0), R(d == 1), R(d == 2)};
    const R vnL = L.v[d], vnR = Rq.v[d];
    const R hL = qdiv<R>(L.E + L.p, L.rho), hR = qdiv<R>(Rq.E + Rq.p, Rq.rho);
    const R r = rsqrt_<R>(qdiv<R>(Rq.rho, L.rho)), rp1 = r + R(1);
    const R rho_a = r * L.rho;
    R va[3], v2a = R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) { va[k] = qdiv<R>(r * Rq.v[k] + L.v[k], rp1); v2a = v2a + va[k] * va[k]; }
    const R ha = qdiv<R>(r * hR + hL, rp1);
    const R vna = va[d];
    const R c2a = c.gm1 * (ha - R(0.5) * v2a);
    R ca = R(1e10);
    if (c2a > R(0)) ca = rsqrt_<R>(c2a);
    R eig[3] = {rabs(vna - ca), rabs(vna), rabs(vna + ca)};
    const R cL = rsqrt_<R>(qdiv<R>(L.p * c.gam, L.rho)), cR = rsqrt_<R>(qdiv<R>(Rq.p * c.gam, Rq.rho));
    const R eL[3] = {rabs(vnL - cL), rabs(vnL), rabs(vnL + cL)};
    const R eR[3] = {rabs(vnR - cR), rabs(vnR), rabs(vnR + cR)};
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const R a1 = rabs(eig[e] - eL[e]), a2 = rabs(eR[e] - eig[e]);
        const R eps = a1 > a2 ? a1 : a2;
        if (eig[e] < eps) {
            // eig^2 / eps < eps; when eps is below the normal range the flushed approximate
            // reciprocal is infinite and the quotient inf or NaN (0 * inf): the term is then
            // below eps and is dropped (IEEE division would give a value of order eps too)
            R t = qdiv<R>(eig[e] * eig[e], eps);
            if (!(t <= R(2) * eps)) t = R(0);
            eig[e] = R(0.5) * (t + eps);
        }
    }
    const R dp = Rq.p - L.p, drho = Rq.rho - L.rho, dvn = vnR - vnL;
    R dvt[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) dvt[k] = (Rq.v[k] - L.v[k]) - dvn * n[k];
    const R inv2c2 = qdiv<R>(R(1), R(2) * c2a);
    const R c0 = eig[0] * (dp - rho_a * ca * dvn) * inv2c2;
    const R c1 = eig[1] * (drho - R(2) * dp * inv2c2);
    const R c2 = eig[1] * rho_a;
    const R c3 = eig[2] * (dp + rho_a * ca * dvn) * inv2c2;
    R A[5];
    A[0] = c0 + c1 + c3;
    R dvtv = R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        A[1 + k] = c0 * (va[k] - ca * n[k]) + c1 * va[k] + c2 * dvt[k] + c3 * (va[k] + ca * n[k]);
        dvtv += va[k] * dvt[k];
    }
    A[4] = c0 * (ha - ca * vna) + c1 * v2a * R(0.5) + c2 * dvtv + c3 * (ha + ca * vna);
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = R(-0.5) * A[k];
}

// Convective numerical flux dot n for n = +e_d, evaluated with L = minus side.
// (convective_numerical_flux.cpp:35-54 composition of baseline + dissipation)
template <typename R, int d>
__device__ __forceinline__ void conv_num_flux(const R uL[5], const R uR[5], const NodeQ<R>& L, const NodeQ<R>& Rq,
                                              int tp, int cf, const Cst<R>& c, R out[5]) {
    if (cf == CF_EC || cf == CF_EC_LXF || cf == CF_EC_ROE) {
        two_point_dir<R, d>(L, Rq, tp, c, out);
    } else {
        R FL[5], FR[5];
        conv_flux_dir<R, d>(L, c.shift(), FL);
        conv_flux_dir<R, d>(Rq, c.shift(), FR);
#pragma unroll
        for (int k = 0; k < 5; ++k) out[k] = R(0.5) * (FL[k] + FR[k]);
    }
    if (cf == CF_LXF || cf == CF_EC_LXF) {
        const R eLv = rabs(L.v[d]) + rsqrt_<R>(qdiv<R>(L.p * c.gam, L.rho));
        const R eRv = rabs(Rq.v[d]) + rsqrt_<R>(qdiv<R>(Rq.p * c.gam, Rq.rho));
        const R e = eLv > eRv ? eLv : eRv;
#pragma unroll
        for (int k = 0; k < 5; ++k) out[k] += R(-0.5) * e * (uR[k] - uL[k]);
    } else if (cf == CF_ROE || cf == CF_EC_ROE) {
        R diss[5];
        roe_dissipation<R, d>(L, Rq, c, diss);
#pragma unroll
        for (int k = 0; k < 5; ++k) out[k] += diss[k];
    }
}

// ---- general-normal forms, for curvilinear cells: the flux dotted with a vector n
// (sum_k n_k F_k), with n the metric-averaged reference direction in the volume and the
// unit physical normal on faces (strong_dg.cpp:1235-1515, :3354-3452).

// Two-point flux dotted with n.
template <typename R>
__device__ __forceinline__ void two_point_n(const NodeQ<R>& i, const NodeQ<R>& j, const R n[3], int tp,
                                            const Cst<R>& c, R F[5]) {
    if (tp == TP_CH) {
        R rho_log, p_hat, h0;
        ch_means<R>(i, j, c, rho_log, p_hat, h0);
        R va[3], vsq = R(0), vn = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) { va[k] = R(0.5) * (i.v[k] + j.v[k]); vsq += va[k] * va[k]; vn += va[k] * n[k]; }
        const R m = rho_log * vn;
        F[0] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[1 + k] = m * va[k] + (p_hat - c.shift()) * n[k];
        F[4] = m * (h0 + vsq);
    } else if (tp == TP_RA) {
        const R rho_log = log_mean<R>(i.a, j.a, i.la, j.la);
        const R b_log = log_mean<R>(i.b, j.b, i.lb, j.lb);
        R va[3], vsq = R(0), vn = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) { va[k] = R(0.5) * (i.v[k] + j.v[k]); vsq += va[k] * va[k]; vn += va[k] * n[k]; }
        const R p_hat = R(0.5) * (i.p + j.p);
        const R gb = b_log * c.gm1;
        R H = qdiv<R>(rho_log + R(2) * gb * p_hat, gb * rho_log) + vsq;
        H -= R(0.5) * (R(0.5) * (i.vsq + j.vsq));
        const R m = rho_log * vn;
        F[0] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[1 + k] = m * va[k] + (p_hat - c.shift()) * n[k];
        F[4] = m * H;
        R vni = R(0), vnj = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) { vni += i.v[k] * n[k]; vnj += j.v[k] * n[k]; }
        F[4] -= R(0.5) * (i.p * vni + j.p * vnj);
    } else if (tp == TP_IR) {
        const R z0a = R(0.5) * (i.a + j.a), z4a = R(0.5) * (i.b + j.b);
        const R l0 = log_mean<R>(i.a, j.a, i.la, j.la);
        const R l4 = log_mean<R>(i.b, j.b, i.lb, j.lb);
        const R rho = z0a * l4;
        R v[3], vv = R(0), vn = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const R zk = R(0.5) * (i.a * i.v[k] + j.a * j.v[k]);
            v[k] = qdiv<R>(zk, z0a); vv += v[k] * v[k]; vn += v[k] * n[k];
        }
        const R p = qdiv<R>(z4a, z0a);
        R H = (c.gam + R(1)) * qdiv<R>(l4, l0) + c.gm1 * p;
        H /= R(2) * c.gam;
        H *= qdiv<R>(c.gam, rho * c.gm1);
        H += R(0.5) * vv;
        const R m = rho * vn;
        F[0] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[1 + k] = m * v[k] + (p - c.shift()) * n[k];
        F[4] = m * H;
    } else {   // KG
        const R rho = (i.rho + j.rho) / R(2);
        const R p = (i.p + j.p) / R(2);
        R v[3], vn = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) { v[k] = R(0.5) * (i.v[k] + j.v[k]); vn += v[k] * n[k]; }
        const R e = (i.vsq + j.vsq) / R(2);
        const R m = rho * vn;
        F[0] = m;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[1 + k] = m * v[k] + (p - c.shift()) * n[k];
        F[4] = m * e + p * vn;
    }
}

// Physical convective flux dotted with n.
template <typename R>
__device__ __forceinline__ void conv_flux_n(const NodeQ<R>& q, const R n[3], R p0, R F[5]) {
    const R H = qdiv<R>(q.E, q.rho) + qdiv<R>(q.p, q.rho);
    const R vn = q.v[0] * n[0] + q.v[1] * n[1] + q.v[2] * n[2];
    const R m = q.rho * vn;
    F[0] = m;
#pragma unroll
    for (int k = 0; k < 3; ++k) F[1 + k] = m * q.v[k] + (q.p - p0) * n[k];
    F[4] = m * H;
}

// Roe-Pike dissipation -1/2 |A_roe(n)| (uR - uL) for a unit normal n
// (convective_numerical_flux.cpp:333-480 with the entropy fix of :215-232).
template <typename R>
__device__ __forceinline__ void roe_dissipation_n(const NodeQ<R>& L, const NodeQ<R>& Rq, const R n[3],
                                                  const Cst<R>& c, R out[5]) {
    const R vnL = L.v[0] * n[0] + L.v[1] * n[1] + L.v[2] * n[2];
    const R vnR = Rq.v[0] * n[0] + Rq.v[1] * n[1] + Rq.v[2] * n[2];
    const R hL = qdiv<R>(L.E + L.p, L.rho), hR = qdiv<R>(Rq.E + Rq.p, Rq.rho);
    const R r = rsqrt_<R>(qdiv<R>(Rq.rho, L.rho)), rp1 = r + R(1);
    const R rho_a = r * L.rho;
    R va[3], v2a = R(0), vna = R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        va[k] = qdiv<R>(r * Rq.v[k] + L.v[k], rp1); v2a = v2a + va[k] * va[k]; vna = vna + va[k] * n[k];
    }
    const R ha = qdiv<R>(r * hR + hL, rp1);
    const R c2a = c.gm1 * (ha - R(0.5) * v2a);
    R ca = R(1e10);
    if (c2a > R(0)) ca = rsqrt_<R>(c2a);
    R eig[3] = {rabs(vna - ca), rabs(vna), rabs(vna + ca)};
    const R cL = rsqrt_<R>(qdiv<R>(L.p * c.gam, L.rho)), cR = rsqrt_<R>(qdiv<R>(Rq.p * c.gam, Rq.rho));
    const R eL[3] = {rabs(vnL - cL), rabs(vnL), rabs(vnL + cL)};
    const R eR[3] = {rabs(vnR - cR), rabs(vnR), rabs(vnR + cR)};
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const R a1 = rabs(eig[e] - eL[e]), a2 = rabs(eR[e] - eig[e]);
        const R eps = a1 > a2 ? a1 : a2;
        if (eig[e] < eps) eig[e] = R(0.5) * (qdiv<R>(eig[e] * eig[e], eps) + eps);
    }
    const R dp = Rq.p - L.p, drho = Rq.rho - L.rho, dvn = vnR - vnL;
    R dvt[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) dvt[k] = (Rq.v[k] - L.v[k]) - dvn * n[k];
    const R inv2c2 = qdiv<R>(R(1), R(2) * c2a);
    const R c0 = eig[0] * (dp - rho_a * ca * dvn) * inv2c2;
    const R c1 = eig[1] * (drho - R(2) * dp * inv2c2);
    const R c2 = eig[1] * rho_a;
    const R c3 = eig[2] * (dp + rho_a * ca * dvn) * inv2c2;
    R A[5];
    A[0] = c0 + c1 + c3;
    R dvtv = R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        A[1 + k] = c0 * (va[k] - ca * n[k]) + c1 * va[k] + c2 * dvt[k] + c3 * (va[k] + ca * n[k]);
        dvtv += va[k] * dvt[k];
    }
    A[4] = c0 * (ha - ca * vna) + c1 * v2a * R(0.5) + c2 * dvtv + c3 * (ha + ca * vna);
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = R(-0.5) * A[k];
}

// Convective numerical flux dotted with the unit normal n (L = the side n points away from).
template <typename R>
__device__ __forceinline__ void conv_num_flux_n(const R uL[5], const R uR[5], const NodeQ<R>& L, const NodeQ<R>& Rq,
                                                const R n[3], int tp, int cf, const Cst<R>& c, R out[5]) {
    if (cf == CF_EC || cf == CF_EC_LXF || cf == CF_EC_ROE) {
        two_point_n<R>(L, Rq, n, tp, c, out);
    } else {
        R FL[5], FR[5];
        conv_flux_n<R>(L, n, c.shift(), FL);
        conv_flux_n<R>(Rq, n, c.shift(), FR);
#pragma unroll
        for (int k = 0; k < 5; ++k) out[k] = R(0.5) * (FL[k] + FR[k]);
    }
    if (cf == CF_LXF || cf == CF_EC_LXF) {
        const R vnL = L.v[0] * n[0] + L.v[1] * n[1] + L.v[2] * n[2];
        const R vnR = Rq.v[0] * n[0] + Rq.v[1] * n[1] + Rq.v[2] * n[2];
        const R eLv = rabs(vnL) + rsqrt_<R>(qdiv<R>(L.p * c.gam, L.rho));
        const R eRv = rabs(vnR) + rsqrt_<R>(qdiv<R>(Rq.p * c.gam, Rq.rho));
        const R e = eLv > eRv ? eLv : eRv;
#pragma unroll
        for (int k = 0; k < 5; ++k) out[k] += R(-0.5) * e * (uR[k] - uL[k]);
    } else if (cf == CF_ROE || cf == CF_EC_ROE) {
        R diss[5];
        roe_dissipation_n<R>(L, Rq, n, c, diss);
#pragma unroll
        for (int k = 0; k < 5; ++k) out[k] += diss[k];
    }
}

// Navier-Stokes viscous flux ("LHS" sign) for state u and conservative gradient
// g[s][k] (navier_stokes.cpp:1198-1350). F[d][0..3] = (momentum x3, energy) along
// direction d; the density component is zero. `dmask` selects the directions.
template <typename R>
__device__ __forceinline__ void viscous_flux(const R u[5], const R g[5][3], int use_const_visc,
                                             const Cst<R>& c, R F[3][4], int dmask, unsigned* st,
                                             bool no_heat = false) {
    const R rho_raw = u[0];
    R w[5];
#pragma unroll
    for (int k = 0; k < 3; ++k) w[1 + k] = qdiv<R>(u[1 + k], rho_raw);
    R v2 = R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) v2 = v2 + w[1 + k] * w[1 + k];
    w[4] = positive<R>(positive<R>(c.gm1 * (u[4] - R(0.5) * rho_raw * v2), st), st);
    w[0] = positive<R>(rho_raw, st);
    const R rho = w[0];
    const R inv_rho = qdiv<R>(R(1), rho);
    R gv[3][3], gp[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int k = 0; k < 3; ++k) gv[a][k] = (g[1 + a][k] - w[1 + a] * g[0][k]) * inv_rho;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        R t = g[4][k];
#pragma unroll
        for (int m = 0; m < 3; ++m) t -= R(0.5) * (w[1 + m] * g[1 + m][k] + u[1 + m] * gv[m][k]);
        gp[k] = t * c.gm1;
    }
    const R T = c.gam * c.mach2 * (w[4] * inv_rho);
    // Sutherland's law mu = (1 + T_r)/(T + T_r) T^{3/2}, with T^{3/2} = T sqrt(T)
    R mu = use_const_visc ? c.const_visc : qdiv<R>(R(1) + c.temp_ratio, T + c.temp_ratio) * (T * rsqrt_<R>(T));
    mu = mu * c.inv_re;
    const R kappa = mu * c.kappa_fac;
    const R div = gv[0][0] + gv[1][1] + gv[2][2];
    const R mu2 = (R(-2) / R(3)) * mu;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (!(dmask & (1 << d))) continue;
        R tau_d[3];   // tau[k][d] (symmetric)
#pragma unroll
        for (int k = 0; k < 3; ++k) tau_d[k] = R(2) * mu * (R(0.5) * (gv[k][d] + gv[d][k]));
        tau_d[d] += mu2 * div;
        const R dT = (c.gam * c.mach2 * gp[d] - T * g[0][d]) * inv_rho;
        const R q = -kappa * dT;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[d][k] = -tau_d[k];
        F[d][3] = -(w[1] * tau_d[0] + w[2] * tau_d[1] + w[3] * tau_d[2]) + (no_heat ? R(0) : q);
    }
}

// ---------------------------------------------------------------------------------------
// Boundary conditions at one face node with outward unit normal n (boundary_id values of
// euler.cpp:1508-1560). IEEE division throughout (few nodes; the flux code's quotient is for
// the volume loops).
// ---------------------------------------------------------------------------------------
enum BoundaryType { BC_WALL = 1001, BC_PRESSURE_OUTFLOW = 1002, BC_INFLOW = 1003, BC_RIEMANN = 1004,
                    BC_FARFIELD = 1005, BC_SLIP_WALL = 1006, BC_EXTRAPOLATION = 1007 };

// primitive (rho, v, p) with the density and pressure checks of convert_conservative_to_primitive
// (euler.cpp:177-198)
template <typename R> __device__ __forceinline__ void bc_primitive(const R u[5], R gm1, R w[5], unsigned* st) {
    const R rho = u[0];
    R v2 = R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) { w[1 + d] = u[1 + d] / rho; v2 = v2 + w[1 + d] * w[1 + d]; }
    const R p = positive<R>(gm1 * (u[4] - R(0.5) * rho * v2), st);
    w[0] = positive<R>(rho, st);
    w[4] = positive<R>(p, st);
}
// convert_primitive_to_conservative with compute_total_energy (euler.cpp:206-222, :357-374)
template <typename R> __device__ __forceinline__ void bc_conservative(const R w[5], R gm1, R u[5]) {
    u[0] = w[0];
    R v2 = R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) { u[1 + d] = w[0] * w[1 + d]; v2 = v2 + w[1 + d] * w[1 + d]; }
    u[4] = w[4] / gm1 + R(0.5) * w[0] * v2;
}

// Euler::boundary_face_values: the exterior state of the convective numerical flux.
// 1001 (boundary_wall) and 1006: slip wall, the normal velocity reflected (:1171-1229);
// 1002 pressure outflow at back pressure 0.99 (:1287-1327); 1003 inflow (:1329-1434);
// 1004 characteristic (Riemann) farfield (:1096-1169); 1005 the free stream (:1436-1450);
// 1007 the interior state (:1452-1464).
template <typename R>
__device__ void boundary_state(int type, const R n[3], const R u[5], const PhysConst& pc, R ub[5], unsigned* st) {
    const R gam = (R)pc.gam, gm1 = (R)pc.gm1, mach2 = (R)pc.mach2;
    R wi[5], wb[5];
    if (type == BC_EXTRAPOLATION) {
#pragma unroll
        for (int s = 0; s < 5; ++s) ub[s] = u[s];
        return;
    }
    if (type == BC_FARFIELD) {
        wb[0] = R(1);
#pragma unroll
        for (int d = 0; d < 3; ++d) wb[1 + d] = (R)pc.bc_v_inf[d];
        wb[4] = R(1) / (gam * mach2);
        bc_conservative<R>(wb, gm1, ub);
        return;
    }
    if (type == BC_PRESSURE_OUTFLOW) {   // compute_mach_number (:555-563) first
        R v2 = R(0);
#pragma unroll
        for (int d = 0; d < 3; ++d) { const R v = u[1 + d] / u[0]; v2 = v2 + v * v; }
        const R rho_c = positive<R>(u[0], st);
        const R p_c = pressure_ieee<R>(u, gm1, st);
        const R mach = rsqrt_<R>(v2) / rsqrt_<R>(p_c * gam / rho_c);
        if (mach > R(1)) {
#pragma unroll
            for (int s = 0; s < 5; ++s) ub[s] = u[s];
            return;
        }
        bc_primitive<R>(u, gm1, wi, st);
        const R radicant = R(1) + R(0.5) * gm1 * mach2;
        const R p_inlet = (R)pc.bc_total_p * rpow<R>(radicant, -gam / gm1);
        const R ge1 = (mach >= R(1)) ? R(1) : R(0);
        const R p_bc = ge1 * wi[4] + (R(1) - ge1) * R(0.99) * p_inlet;
        const R t_int = gam * mach2 * (wi[4] / wi[0]);
        wb[0] = gam * mach2 * (p_bc / t_int);
#pragma unroll
        for (int d = 0; d < 3; ++d) wb[1 + d] = wi[1 + d];
        wb[4] = p_bc;
        bc_conservative<R>(wb, gm1, ub);
        return;
    }
    bc_primitive<R>(u, gm1, wi, st);
    if (type == BC_INFLOW) {
        const R nrm[3] = {-n[0], -n[1], -n[2]};
        R vni = R(0);
#pragma unroll
        for (int d = 0; d < 3; ++d) vni += wi[1 + d] * nrm[d];
        const R rho_c = positive<R>(u[0], st);
        const R ci = rsqrt_<R>(pressure_ieee<R>(u, gm1, st) * gam / rho_c);   // compute_sound (:535-543)
        const R mach_inf = (R)pc.bc_mach_inf;
        R p_bc, t_bc, vmag;
        if (mach_inf < R(1)) {
            const R rpos = vni + R(2) * ci / gm1;
            const R H = u[4] / wi[0] + wi[4] / wi[0];
            const R a = R(1) + R(2) / gm1;
            const R b = R(-2) * rpos;
            const R c = R(0.5) * gm1 * (rpos * rpos - R(2) * H);
            const R t1 = R(-0.5) * b / a;
            const R t2 = R(0.5) * rsqrt_<R>(b * b - R(4) * a * c) / a;
            const R cb = fmax(t1 + t2, t1 - t2);
            vmag = rpos - R(2) * cb / gm1;
            const R mach_bc = vmag / cb;
            const R radicant = R(1) + R(0.5) * gm1 * mach_bc * mach_bc;
            p_bc = (R)pc.bc_total_p * rpow<R>(radicant, -gam / gm1);
            t_bc = (R)pc.bc_total_t * rpow<R>(radicant, R(-1));
            wb[0] = gam * mach2 * (p_bc / t_bc);
#pragma unroll
            for (int d = 0; d < 3; ++d) wb[1 + d] = vmag * nrm[d];
        } else {
            const R radicant = R(1) + R(0.5) * gm1 * mach2;
            p_bc = (R)pc.bc_total_p * rpow<R>(radicant, -gam / gm1);
            t_bc = (R)pc.bc_total_t * rpow<R>(radicant, R(-1));
            wb[0] = gam * mach2 * (p_bc / t_bc);
            const R cb = rsqrt_<R>(gam * p_bc / wb[0]);
            vmag = mach_inf * cb;
#pragma unroll
            for (int d = 0; d < 3; ++d) wb[1 + d] = -vmag * n[d];
        }
        wb[4] = p_bc;
        bc_conservative<R>(wb, gm1, ub);
        return;
    }
    if (type == BC_RIEMANN) {
        R we[5];
        we[0] = R(1);
#pragma unroll
        for (int d = 0; d < 3; ++d) we[1 + d] = (R)pc.bc_v_inf[d];
        we[4] = R(1) / (gam * mach2);
        const R ci = rsqrt_<R>(wi[4] * gam / wi[0]), ce = rsqrt_<R>(we[4] * gam / we[0]);
        R vni = R(0), vne = R(0);
#pragma unroll
        for (int d = 0; d < 3; ++d) { vni = vni + wi[1 + d] * n[d]; vne = vne + we[1 + d] * n[d]; }
        const R rout = vni + R(2) / gm1 * ci, rinc = vne - R(2) / gm1 * ce;
        const R vnb = R(0.5) * (rout + rinc), cb = R(0.25) * gm1 * (rout - rinc);
        if (rabs<R>(vnb) >= rabs<R>(cb)) {
#pragma unroll
            for (int s = 0; s < 5; ++s) wb[s] = vnb < R(0) ? we[s] : wi[s];
        } else {
            const R* w = vnb < R(0) ? we : wi;
            const R vn = vnb < R(0) ? vne : vni;
            // compute_entropy_measure (:414-421): p rho^-gam of a checked density
            const R ent = w[0] < R(0) ? (R)BIG_NUMBER : w[4] * rpow<R>(w[0], -gam);
            if (w[0] < R(0) && st) atomicOr(st, ST_NONPHYSICAL);
            const R rb = rpow<R>(R(1) / gam * cb * cb / ent, R(1) / gm1);
#pragma unroll
            for (int d = 0; d < 3; ++d) wb[1 + d] = (w[1 + d] - vn * n[d]) + vnb * n[d];
            wb[4] = R(1) / gam * cb * cb * rb;
            wb[0] = rb;
        }
        bc_conservative<R>(wb, gm1, ub);
        return;
    }
    // slip wall (1001 in Euler::boundary_face_values, 1006)
    wb[0] = wi[0]; wb[4] = wi[4];
    const R sn[3] = {-n[0], -n[1], -n[2]};
    R vn = R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) vn = vn + wi[1 + d] * sn[d];
#pragma unroll
    for (int d = 0; d < 3; ++d) wb[1 + d] = wi[1 + d] - R(2) * vn * sn[d];
    bc_conservative<R>(wb, gm1, ub);
}

// boundary_state for the outward normal of reference face f (+/- e_{f/2}), out of line: the kernels
// that call it for their boundary faces keep their registers
template <typename R>
__device__ __noinline__ void boundary_state_face(int type, int f, const R* u, const PhysConst& pc, R* ub,
                                                 unsigned* st) {
    const int dn = f >> 1;
    const R sg = (f & 1) ? R(1) : R(-1);
    const R nrm[3] = {dn == 0 ? sg : R(0), dn == 1 ? sg : R(0), dn == 2 ? sg : R(0)};
    R ui[5], uo[5];
#pragma unroll
    for (int s = 0; s < 5; ++s) ui[s] = u[s];
    boundary_state<R>(type, nrm, ui, pc, uo, st);
#pragma unroll
    for (int s = 0; s < 5; ++s) ub[s] = uo[s];
}

// the same for a given outward unit normal (curvilinear faces)
template <typename R>
__device__ __noinline__ void boundary_state_normal(int type, const R* nrm, const R* u, const PhysConst& pc, R* ub,
                                                   unsigned* st) {
    const R n[3] = {nrm[0], nrm[1], nrm[2]};
    R ui[5], uo[5];
#pragma unroll
    for (int s = 0; s < 5; ++s) ui[s] = u[s];
    boundary_state<R>(type, n, ui, pc, uo, st);
#pragma unroll
    for (int s = 0; s < 5; ++s) ub[s] = uo[s];
}

// NavierStokes::boundary_face_values_viscous_flux (navier_stokes.cpp:1354-1432): the exterior state
// of the dissipative fluxes. 1001: no-slip, the momentum negated (its gradient is the interior's,
// the energy gradient zero on an adiabatic wall; isothermal: the exterior temperature 2 T_wall - T);
// 1006: the interior state and gradient.
template <typename R>
__device__ __forceinline__ void boundary_viscous_state(int type, const R u[5], const PhysConst& pc, R ub[5],
                                                       unsigned* st) {
#pragma unroll
    for (int s = 0; s < 5; ++s) ub[s] = u[s];
    if (type != BC_WALL) return;
#pragma unroll
    for (int d = 0; d < 3; ++d) ub[1 + d] = -u[1 + d];
    if (pc.bc_isothermal) {
        const R gam = (R)pc.gam, gm1 = (R)pc.gm1, mach2 = (R)pc.mach2;
        R wi[5], we[5];
        bc_primitive<R>(u, gm1, wi, st);
        bc_primitive<R>(ub, gm1, we, st);
        const R t_int = gam * mach2 * (wi[4] / wi[0]);
        const R t_ext = R(2) * (R)pc.bc_t_wall - t_int;
        we[4] = we[0] * t_ext / (gam * mach2);
        R w2[5];
        bc_conservative<R>(we, gm1, w2);
        ub[4] = w2[4];
    }
}

} // namespace ph
