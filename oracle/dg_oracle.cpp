// CPU oracle (test infrastructure): restatement of PHiLiP's explicit strong-form
// DG/FR residual. Each function cites the reference file:line it follows.
#include <array>
#include "dg_oracle.hpp"

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

static const double BIG_NUMBER = 1e100;   // physics.h:270
static const double PI = 3.14159265358979323846;

// ---------------------------------------------------------------------------------
// 1-D quadrature and Lagrange bases (stand-ins for deal.II QGauss / QGaussLobatto /
// FE_DGQ / FE_DGQArbitraryNodes, which the reference builds in dg_base.cpp:131-261).
// ---------------------------------------------------------------------------------
static void legendre(int n, double x, double& p, double& dp) {
    // P_n(x) and P_n'(x) on [-1,1] by the three-term recurrence.
    double p0 = 1.0, p1 = x;
    if (n == 0) { p = 1.0; dp = 0.0; return; }
    for (int k = 2; k <= n; ++k) {
        double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1; p1 = pk;
    }
    p = p1;
    dp = (std::fabs(x) < 1.0) ? n * (x * p1 - p0) / (x * x - 1.0) : 0.5 * n * (n + 1) * std::pow(x, n + 1);
}

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0); w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it) {
            double p, dp; legendre(n, z, p, dp);
            double dz = p / dp; z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p, dp; legendre(n, z, p, dp);
        // ascending order on [0,1]
        x[n - 1 - i] = 0.5 * (z + 1.0);
        w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);   // (2/((1-z^2)P'^2)) / 2
    }
}

void gauss_lobatto(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0); w.assign(n, 0.0);
    if (n < 2) throw std::runtime_error("Gauss-Lobatto needs n >= 2");
    const int m = n - 1;  // interior nodes are roots of P_m'
    x[0] = 0.0; x[n - 1] = 1.0;
    for (int i = 1; i < n - 1; ++i) {
        double z = -std::cos(PI * i / m);   // Chebyshev-Gauss-Lobatto guess (ascending)
        for (int it = 0; it < 100; ++it) {
            // Newton on q(z) = P_m'(z); q' = (2 z P_m' - m(m+1) P_m)/(1-z^2)
            double p, dp; legendre(m, z, p, dp);
            double d2p = (2.0 * z * dp - m * (m + 1.0) * p) / (1.0 - z * z);
            double dz = dp / d2p; z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[i] = 0.5 * (z + 1.0);
    }
    for (int i = 0; i < n; ++i) {
        double z = 2.0 * x[i] - 1.0, p, dp; legendre(m, z, p, dp);
        w[i] = 1.0 / (m * (m + 1.0) * p * p);    // (2/(m(m+1)P_m^2)) / 2
    }
}

void lagrange_eval(const std::vector<double>& nodes, double x, double* val, double* der) {
    const int n = (int)nodes.size();
    for (int j = 0; j < n; ++j) {
        double v = 1.0, d = 0.0;
        for (int m = 0; m < n; ++m) {
            if (m == j) continue;
            const double inv = 1.0 / (nodes[j] - nodes[m]);
            d = d * (x - nodes[m]) * inv + v * inv;
            v *= (x - nodes[m]) * inv;
        }
        if (val) val[j] = v;
        if (der) der[j] = d;
    }
}

static std::vector<double> matmul(const std::vector<double>& A, const std::vector<double>& B, int n, int k, int m) {
    std::vector<double> C((size_t)n * m, 0.0);
    for (int i = 0; i < n; ++i)
        for (int l = 0; l < k; ++l)
            for (int j = 0; j < m; ++j) C[i * m + j] += A[i * k + l] * B[l * m + j];
    return C;
}

static std::vector<double> invert(std::vector<double> A, int n) {
    // Gauss-Jordan with partial pivoting (deal.II FullMatrix::invert equivalent).
    std::vector<double> I((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r) if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        if (piv != c) for (int j = 0; j < n; ++j) { std::swap(A[c * n + j], A[piv * n + j]); std::swap(I[c * n + j], I[piv * n + j]); }
        const double d = 1.0 / A[c * n + c];
        for (int j = 0; j < n; ++j) { A[c * n + j] *= d; I[c * n + j] *= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = A[r * n + c];
            if (f == 0.0) continue;
            for (int j = 0; j < n; ++j) { A[r * n + j] -= f * A[c * n + j]; I[r * n + j] -= f * I[c * n + j]; }
        }
    }
    return I;
}

static double factorial(int k) { double f = 1.0; for (int i = 2; i <= k; ++i) f *= i; return f; }

// FR correction parameter c (operators.cpp:1559-1661); reference element [0,1].
double fr_correction_parameter(int fr_type, int p, double user_value) {
    const double pf = factorial(p), pf2 = factorial(2 * p);
    const double cp = pf2 / (pf * pf);
    double c = 0.0;
    switch (fr_type) {
    case C_HU: case C_HU_LUMPED:
        c = 2.0 * (p + 1) / (p * ((2.0 * p + 1.0) * std::pow(pf * cp, 2))); c /= 2.0; break;
    case C_SD:
        c = 2.0 * p / ((p + 1.0) * ((2.0 * p + 1.0) * std::pow(pf * cp, 2))); c /= 2.0; break;
    case C_NEGATIVE:
        c = -2.0 / std::pow((2.0 * p + 1.0) * std::pow(pf * cp, 2), 1.0); c /= 2.0; break;
    case C_NEGATIVE2:
        c = -2.0 / std::pow((2.0 * p + 1.0) * std::pow(pf * cp, 2), 1.0); c /= 2.0; c /= 2.0; break;
    case C_DG: c = 0.0; break;
    case C_10THOUSAND: c = 10000.0; break;
    case C_PLUS:
        if (p == 2) c = 0.186; else if (p == 3) c = 3.67e-3; else if (p == 4) c = 4.79e-5; else if (p == 5) c = 4.24e-7;
        else throw std::runtime_error("cPlus defined for p=2..5 only");
        c /= 2.0; c /= std::pow(std::pow(2.0, p), 2); break;
    case C_USER:
        c = user_value; c /= 2.0; c /= std::pow(std::pow(2.0, p), 2); break;
    default: throw std::runtime_error("unknown FR type");
    }
    return c;
}

static double fr_aux_parameter(int k_type, int p) {
    switch (k_type) {
    case K_DG: return 0.0;
    case K_SD: return fr_correction_parameter(C_SD, p, 0.0);
    case K_HU: return fr_correction_parameter(C_HU, p, 0.0);
    case K_NEGATIVE: return fr_correction_parameter(C_NEGATIVE, p, 0.0);
    case K_NEGATIVE2: return fr_correction_parameter(C_NEGATIVE2, p, 0.0);
    case K_PLUS: return fr_correction_parameter(C_PLUS, p, 0.0);
    case K_10THOUSAND: return 10000.0;
    }
    throw std::runtime_error("unknown FR aux type");
}

Ops1D build_ops(const Params& prm) {
    Ops1D o;
    const int p = prm.poly_degree;
    o.nd = p + 1;
    o.nq = p + 1 + prm.overintegration;
    if (prm.flux_nodes == GLL) gauss_lobatto(o.nq, o.xq, o.wq); else gauss_legendre(o.nq, o.xq, o.wq);
    // FE_DGQ(p) support points: Gauss-Lobatto points of p+1 (0.5 for p=0).
    if (p == 0) o.xs = {0.5};
    else { std::vector<double> dummy; gauss_lobatto(o.nd, o.xs, dummy); }
    const int nd = o.nd, nq = o.nq;
    o.chi.assign((size_t)nq * nd, 0.0); o.dchi.assign((size_t)nq * nd, 0.0);
    for (int q = 0; q < nq; ++q) lagrange_eval(o.xs, o.xq[q], &o.chi[q * nd], &o.dchi[q * nd]);
    for (int s = 0; s < 2; ++s) { o.chi_s[s].assign(nd, 0.0); lagrange_eval(o.xs, (double)s, o.chi_s[s].data(), nullptr); }
    o.phi.assign((size_t)nq * nq, 0.0); o.dphi.assign((size_t)nq * nq, 0.0);
    for (int q = 0; q < nq; ++q) lagrange_eval(o.xq, o.xq[q], &o.phi[q * nq], &o.dphi[q * nq]);
    for (int s = 0; s < 2; ++s) { o.phi_s[s].assign(nq, 0.0); lagrange_eval(o.xq, (double)s, o.phi_s[s].data(), nullptr); }
    // stiffness S_ij = sum_q phi_i(x_q) phi_j'(x_q) w_q, skew = S - S^T (operators.cpp:1440-1477)
    std::vector<double> S((size_t)nq * nq, 0.0);
    for (int i = 0; i < nq; ++i)
        for (int j = 0; j < nq; ++j) {
            double v = 0.0;
            for (int q = 0; q < nq; ++q) v += o.phi[q * nq + i] * o.dphi[q * nq + j] * o.wq[q];
            S[i * nq + j] = v;
        }
    o.skew.assign((size_t)nq * nq, 0.0);
    for (int i = 0; i < nq; ++i) for (int j = 0; j < nq; ++j) o.skew[i * nq + j] = S[i * nq + j] - S[j * nq + i];
    // mass M_ij = sum_q chi_i chi_j w_q (operators.cpp:1354-1385)
    std::vector<double> M((size_t)nd * nd, 0.0);
    for (int i = 0; i < nd; ++i) for (int j = 0; j < nd; ++j) {
        double v = 0.0;
        for (int q = 0; q < nq; ++q) v += o.chi[q * nd + i] * o.chi[q * nd + j] * o.wq[q];
        M[i * nd + j] = v;
    }
    // modal differential operator M^{-1} S_chi, p-th derivative (operators.cpp:1491-1540)
    std::vector<double> Schi((size_t)nd * nd, 0.0);
    for (int i = 0; i < nd; ++i) for (int j = 0; j < nd; ++j) {
        double v = 0.0;
        for (int q = 0; q < nq; ++q) v += o.chi[q * nd + i] * o.dchi[q * nd + j] * o.wq[q];
        Schi[i * nd + j] = v;
    }
    std::vector<double> Minv = invert(M, nd);
    std::vector<double> Dm = matmul(Minv, Schi, nd, nd, nd);
    std::vector<double> Dp((size_t)nd * nd, 0.0);
    for (int i = 0; i < nd; ++i) Dp[i * nd + i] = 1.0;
    for (int k = 0; k < p; ++k) Dp = matmul(Dm, Dp, nd, nd, nd);
    auto fr_oper = [&](double c) {   // K = c (D^p)^T M D^p  (operators.cpp:1663-1675)
        std::vector<double> DpT((size_t)nd * nd);
        for (int i = 0; i < nd; ++i) for (int j = 0; j < nd; ++j) DpT[i * nd + j] = c * Dp[j * nd + i];
        return matmul(matmul(DpT, M, nd, nd, nd), Dp, nd, nd, nd);
    };
    const double c = fr_correction_parameter(prm.fr_type, p, prm.fr_user_value);
    const double k = fr_aux_parameter(prm.fr_aux_type, p);
    std::vector<double> K = fr_oper(c), Ka = fr_oper(k);
    std::vector<double> MK(M), MKa(M);
    for (size_t i = 0; i < M.size(); ++i) { MK[i] += K[i]; MKa[i] += Ka[i]; }
    o.minv = invert(MK, nd);
    o.minv_aux = invert(MKa, nd);
    // projection Pi = M^{-1} chi^T W (operators.cpp:1864-1889), plain M (not FR)
    o.proj.assign((size_t)nd * nq, 0.0);
    for (int i = 0; i < nd; ++i) for (int q = 0; q < nq; ++q) {
        double v = 0.0;
        for (int j = 0; j < nd; ++j) v += Minv[i * nd + j] * o.chi[q * nd + j] * o.wq[q];
        o.proj[i * nq + q] = v;
    }
    return o;
}

// ---------------------------------------------------------------------------------
// Sum-factorised tensor-product application (operators.cpp:294-398, :575-636).
// A_d is (r_d x c_d) row-major; input is c_z*c_y*c_x (x fastest), output r_z*r_y*r_x.
// ---------------------------------------------------------------------------------
static void apply3(const double* Ax, int rx, int cx, const double* Ay, int ry, int cy,
                   const double* Az, int rz, int cz, const double* in, double* out,
                   bool adding, double factor) {
    std::vector<double> t1((size_t)rx * cy * cz), t2((size_t)rx * ry * cz);
    for (int z = 0; z < cz; ++z) for (int y = 0; y < cy; ++y) for (int x = 0; x < rx; ++x) {
        double v = 0.0;
        for (int s = 0; s < cx; ++s) v += Ax[x * cx + s] * in[(z * cy + y) * cx + s];
        t1[(z * cy + y) * rx + x] = v;
    }
    for (int z = 0; z < cz; ++z) for (int y = 0; y < ry; ++y) for (int x = 0; x < rx; ++x) {
        double v = 0.0;
        for (int s = 0; s < cy; ++s) v += Ay[y * cy + s] * t1[(z * cy + s) * rx + x];
        t2[(z * ry + y) * rx + x] = v;
    }
    for (int z = 0; z < rz; ++z) for (int y = 0; y < ry; ++y) for (int x = 0; x < rx; ++x) {
        double v = adding ? out[(z * ry + y) * rx + x] : 0.0;
        for (int s = 0; s < cz; ++s) v += factor * Az[z * cz + s] * t2[(s * ry + y) * rx + x];
        out[(z * ry + y) * rx + x] = v;
    }
}

static std::vector<double> transpose(const double* A, int r, int c) {
    std::vector<double> T((size_t)r * c);
    for (int i = 0; i < r; ++i) for (int j = 0; j < c; ++j) T[j * r + i] = A[i * c + j];
    return T;
}

// inner product: out = (Ax^T (x) Ay^T (x) Az^T)(in .* w)
static void inner3(const double* Ax, int rx, int cx, const double* Ay, int ry, int cy,
                   const double* Az, int rz, int cz, const double* in, const double* w, double* out,
                   bool adding, double factor) {
    const int n = rx * ry * rz;
    std::vector<double> wi(n);
    for (int i = 0; i < n; ++i) wi[i] = in[i] * (w ? w[i] : 1.0);
    std::vector<double> Tx = transpose(Ax, rx, cx), Ty = transpose(Ay, ry, cy), Tz = transpose(Az, rz, cz);
    apply3(Tx.data(), cx, rx, Ty.data(), cy, ry, Tz.data(), cz, rz, wi.data(), out, adding, factor);
}

// ---------------------------------------------------------------------------------
// Physics (euler.cpp, navier_stokes.cpp)
// ---------------------------------------------------------------------------------
struct Physics {
    const Params* prm;
    double gam, gm1, mach2, temp_ratio;
    int* status;
    explicit Physics(const Params* p, int* st) : prm(p), status(st) {
        gam = p->gamma; gm1 = gam - 1.0; mach2 = p->mach_inf * p->mach_inf;
        temp_ratio = 110.4 / p->temperature_inf;     // navier_stokes.cpp:50-52
    }
    double positive(double q) const {   // euler.cpp:155-172 + physics.cpp:298-317
        // with a positivity-preserving limiter selected the check passes every value through
        // unchanged (check_positive_quantity, euler.cpp:153-172)
        if (prm->limiter == PPL_ZHANG2010 || prm->limiter == PPL_WANG2012) return q;
        if (q < 0.0) {
            if (status) __atomic_fetch_or(status, 1, __ATOMIC_RELAXED);
            if (prm->non_physical == ABORT_RUN) { std::fprintf(stderr, "oracle: non-physical state\n"); std::abort(); }
            return BIG_NUMBER;
        }
        return q;
    }
    double pressure(const double* u) const {   // euler.cpp:486-500
        const double rho = u[0];
        double v2 = 0.0;
        for (int d = 0; d < 3; ++d) { const double v = u[1 + d] / rho; v2 = v2 + v * v; }
        return positive(gm1 * (u[4] - 0.5 * rho * v2));
    }
    void primitive(const double* u, double* w) const {   // euler.cpp:177-198
        const double rho = u[0];
        for (int d = 0; d < 3; ++d) w[1 + d] = u[1 + d] / rho;
        const double p = pressure(u);
        w[0] = positive(rho);
        w[4] = positive(p);
    }
    void conservative_from_primitive(const double* w, double* u) const {  // euler.cpp:207-222
        const double rho = w[0];
        u[0] = rho;
        double v2 = 0.0;
        for (int d = 0; d < 3; ++d) { u[1 + d] = rho * w[1 + d]; v2 += w[1 + d] * w[1 + d]; }
        u[4] = w[4] / gm1 + 0.5 * rho * v2;
    }
    double sound(double rho, double p) const { return std::sqrt(p * gam / rho); }
    void convective_flux(const double* u, double F[5][3]) const {   // euler.cpp:915-938
        const double rho = u[0];
        const double p = pressure(u);
        double v[3]; for (int d = 0; d < 3; ++d) v[d] = u[1 + d] / rho;
        const double H = u[4] / u[0] + p / rho;
        for (int fd = 0; fd < 3; ++fd) {
            F[0][fd] = u[1 + fd];
            for (int vd = 0; vd < 3; ++vd) F[1 + vd][fd] = rho * v[fd] * v[vd];
            F[1 + fd][fd] += p;
            F[4][fd] = rho * v[fd] * H;
        }
    }
    static double log_mean(double a, double b) {   // euler.cpp:628-646
        const double zeta = a / b;
        const double f = (zeta - 1.0) / (zeta + 1.0);
        const double u = f * f;
        double F;
        if (u < 1.0e-2) F = 1.0 + u / 3.0 + u * u / 5.0 + u * u * u / 7.0;
        else F = std::log(zeta) / 2.0 / f;
        return (a + b) / (2.0 * F);
    }
    void two_point(const double* u1, const double* u2, double F[5][3]) const {   // euler.cpp:563-809
        const int type = prm->two_point;
        if (type == KG) {
            const double rho = (u1[0] + u2[0]) / 2.;
            const double p = (pressure(u1) + pressure(u2)) / 2.;
            double v[3]; for (int d = 0; d < 3; ++d) v[d] = 0.5 * (u1[1 + d] / u1[0] + u2[1 + d] / u2[0]);
            const double e = ((u1[4] / u1[0]) + (u2[4] / u2[0])) / 2.;
            for (int fd = 0; fd < 3; ++fd) {
                F[0][fd] = rho * v[fd];
                for (int vd = 0; vd < 3; ++vd) F[1 + vd][fd] = rho * v[fd] * v[vd];
                F[1 + fd][fd] += p;
                F[4][fd] = rho * v[fd] * e + p * v[fd];
            }
        } else if (type == IR) {
            double w1[5], w2[5], z1[5], z2[5];
            primitive(u1, w1); primitive(u2, w2);
            auto param = [](const double* w, double* z) {
                z[0] = std::sqrt(w[0] / w[4]);
                for (int d = 0; d < 3; ++d) z[1 + d] = z[0] * w[1 + d];
                z[4] = std::sqrt(w[0] * w[4]);
            };
            param(w1, z1); param(w2, z2);
            double avg[5], lm[5];
            for (int s = 0; s < 5; ++s) avg[s] = 0.5 * (z1[s] + z2[s]);
            for (int s = 0; s < 5; ++s) lm[s] = log_mean(z1[s], z2[s]);
            double v[3];
            const double rho = avg[0] * lm[4];
            for (int d = 0; d < 3; ++d) v[d] = avg[1 + d] / avg[0];
            const double p = avg[4] / avg[0];
            double H = (gam + 1.0) * (lm[4] / lm[0]) + gm1 * p;
            H /= 2.0 * gam;
            H *= gam / (rho * gm1);
            double vv = 0.0; for (int d = 0; d < 3; ++d) vv += v[d] * v[d];
            H += 0.5 * vv;
            for (int fd = 0; fd < 3; ++fd) {
                F[0][fd] = rho * v[fd];
                for (int vd = 0; vd < 3; ++vd) F[1 + vd][fd] = rho * v[fd] * v[vd];
                F[1 + fd][fd] += p;
                F[4][fd] = rho * v[fd] * H;
            }
        } else {   // CH or Ra
            const bool ra = (type == RA);
            const double rho_log = log_mean(u1[0], u2[0]);
            const double p1 = pressure(u1), p2 = pressure(u2);
            const double b1 = ra ? u1[0] / p1 : u1[0] / (2.0 * p1);
            const double b2 = ra ? u2[0] / p2 : u2[0] / (2.0 * p2);
            const double b_log = log_mean(b1, b2);
            double v1[3], v2[3], va[3];
            for (int d = 0; d < 3; ++d) { v1[d] = u1[1 + d] / u1[0]; v2[d] = u2[1 + d] / u2[0]; }
            double p_hat = ra ? 0.5 * (p1 + p2) : 0.5 * (u1[0] + u2[0]) / (2.0 * 0.5 * (b1 + b2));
            double vsq = 0.0;
            for (int d = 0; d < 3; ++d) { va[d] = 0.5 * (v1[d] + v2[d]); vsq += (0.5 * (v1[d] + v2[d])) * (0.5 * (v1[d] + v2[d])); }
            double H = ra ? 1.0 / (b_log * gm1) + vsq + 2.0 * p_hat / rho_log
                          : 1.0 / (2.0 * b_log * gm1) + vsq + p_hat / rho_log;
            for (int d = 0; d < 3; ++d) H -= 0.5 * (0.5 * (v1[d] * v1[d] + v2[d] * v2[d]));
            for (int fd = 0; fd < 3; ++fd) {
                F[0][fd] = rho_log * va[fd];
                for (int vd = 0; vd < 3; ++vd) F[1 + vd][fd] = rho_log * va[fd] * va[vd];
                F[1 + fd][fd] += p_hat;
                F[4][fd] = rho_log * va[fd] * H;
                if (ra) F[4][fd] -= (0.5 * (p1 * v1[fd] + p2 * v2[fd]));
            }
        }
    }
    void entropy_vars(const double* u, double* v) const {   // euler.cpp:811-830
        const double rho = u[0];
        const double p = pressure(u);
        double s;
        {   // compute_entropy (euler.cpp:510-531)
            double rc = rho, pc = p;
            rc = positive(rc); pc = positive(pc);
            s = std::log(p * std::pow(rho, -gam));
        }
        const double rt = p / gm1;
        v[0] = (rt * (gam + 1.0 - s) - u[4]) / rt;
        for (int d = 0; d < 3; ++d) v[1 + d] = u[1 + d] / rt;
        v[4] = -rho / rt;
    }
    void cons_from_entropy(const double* v, double* u) const {   // euler.cpp:833-855
        double vv = 0.0;
        for (int d = 0; d < 3; ++d) vv += v[1 + d] * v[1 + d];
        const double s = gam - v[0] + 0.5 * vv / v[4];
        const double rt = std::pow((gm1 / std::pow(-v[4], gam)), 1.0 / gm1) * std::exp(-s / gm1);
        u[0] = -rt * v[4];
        for (int d = 0; d < 3; ++d) u[1 + d] = rt * v[1 + d];
        u[4] = rt * (1.0 - 0.5 * vv / v[4]);
    }
    double max_normal_eig(const double* u, const double* n) const {   // euler.cpp:1048-1063
        double v[3]; for (int d = 0; d < 3; ++d) v[d] = u[1 + d] / u[0];
        const double rho = positive(u[0]);
        const double c = std::sqrt(pressure(u) * gam / rho);
        double vn = 0.0; for (int d = 0; d < 3; ++d) vn += v[d] * n[d];
        return std::fabs(vn) + c;
    }
    double max_eig(const double* u) const {   // euler.cpp:1034-1046
        double v2 = 0.0; for (int d = 0; d < 3; ++d) { const double v = u[1 + d] / u[0]; v2 += v * v; }
        const double rho = positive(u[0]);
        const double c = std::sqrt(pressure(u) * gam / rho);
        return std::sqrt(v2) + c;
    }
    // Navier-Stokes viscous flux, "LHS" sign (navier_stokes.cpp:1198-1350); no_heat: the heat flux
    // set to zero (dissipative_flux_dot_normal_on_adiabatic_boundary, :1268-1317)
    void viscous_flux(const double* u, const double g[5][3], double F[5][3], bool no_heat = false) const {
        if (prm->pde != NAVIER_STOKES) { for (int s = 0; s < 5; ++s) for (int d = 0; d < 3; ++d) F[s][d] = 0.0; return; }
        double w[5]; primitive(u, w);
        const double rho = w[0];
        double gw[5][3];
        for (int d = 0; d < 3; ++d) gw[0][d] = g[0][d];
        for (int a = 0; a < 3; ++a) for (int d = 0; d < 3; ++d) gw[1 + a][d] = (g[1 + a][d] - w[1 + a] * g[0][d]) / rho;
        for (int d = 0; d < 3; ++d) {
            gw[4][d] = g[4][d];
            for (int k = 0; k < 3; ++k) gw[4][d] -= 0.5 * (w[1 + k] * g[1 + k][d] + u[1 + k] * gw[1 + k][d]);
            gw[4][d] *= gm1;
        }
        const double T = gam * mach2 * (w[4] / rho);
        double mu = prm->use_constant_viscosity ? 1.0 * prm->constant_viscosity
                                                : ((1.0 + temp_ratio) / (T + temp_ratio)) * std::pow(T, 1.5);
        mu = mu / prm->reynolds_inf;
        const double kappa = mu / (gm1 * mach2 * prm->prandtl);
        double S[3][3], div = 0.0;
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) S[a][b] = 0.5 * (gw[1 + a][b] + gw[1 + b][a]);
        for (int d = 0; d < 3; ++d) div += S[d][d];
        double tau[3][3];
        const double mu2 = (-2.0 / 3.0) * mu;
        for (int a = 0; a < 3; ++a) {
            for (int b = 0; b < 3; ++b) tau[a][b] = 2.0 * mu * S[a][b];
            tau[a][a] += mu2 * div;
        }
        double q[3];
        for (int d = 0; d < 3; ++d) {
            const double dT = (gam * mach2 * gw[4][d] - T * gw[0][d]) / rho;
            q[d] = -kappa * dT;
        }
        for (int fd = 0; fd < 3; ++fd) {
            F[0][fd] = 0.0;
            for (int sd = 0; sd < 3; ++sd) F[1 + sd][fd] = -tau[sd][fd];
            F[4][fd] = 0.0;
            for (int sd = 0; sd < 3; ++sd) F[4][fd] -= w[1 + sd] * tau[fd][sd];
            F[4][fd] += no_heat ? 0.0 : q[fd];
        }
    }
    void viscous_flux_dot_n(const double* u, const double g[5][3], const double* n, double* out,
                            bool no_heat = false) const {
        double F[5][3]; viscous_flux(u, g, F, no_heat);
        for (int s = 0; s < 5; ++s) { out[s] = 0.0; for (int d = 0; d < 3; ++d) out[s] += F[s][d] * n[d]; }
    }
    // convective numerical flux dot n (convective_numerical_flux.cpp:35-480)
    void conv_num_flux(const double* uL, const double* uR, const double* n, double* out) const {
        const int t = prm->conv_flux;
        double base[5] = {0, 0, 0, 0, 0};
        if (t == TWO_POINT || t == TWO_POINT_LXF || t == TWO_POINT_ROE) {
            double F[5][3]; two_point(uL, uR, F);
            for (int s = 0; s < 5; ++s) { double v = 0.0; for (int d = 0; d < 3; ++d) v += F[s][d] * n[d]; base[s] = v; }
        } else {
            double FL[5][3], FR[5][3]; convective_flux(uL, FL); convective_flux(uR, FR);
            for (int s = 0; s < 5; ++s) {
                double v = 0.0;
                for (int d = 0; d < 3; ++d) v += 0.5 * (FL[s][d] + FR[s][d]) * n[d];
                base[s] = v;
            }
        }
        double diss[5] = {0, 0, 0, 0, 0};
        if (t == LAX_FRIEDRICHS || t == TWO_POINT_LXF) {
            const double eL = max_normal_eig(uL, n), eR = max_normal_eig(uR, n);
            const double e = (eL > eR) ? eL : eR;
            for (int s = 0; s < 5; ++s) diss[s] = -0.5 * e * (uR[s] - uL[s]);
        } else if (t == ROE || t == TWO_POINT_ROE) {
            roe_dissipation(uL, uR, n, diss);
        }
        for (int s = 0; s < 5; ++s) out[s] = base[s] + diss[s];
    }
    void roe_dissipation(const double* uL, const double* uR, const double* n, double* out) const {
        double wL[5], wR[5]; primitive(uL, wL); primitive(uR, wR);
        const double rL = wL[0], pL = wL[4], rR = wR[0], pR = wR[4];
        double vnL = 0.0, vnR = 0.0;
        for (int d = 0; d < 3; ++d) { vnL += wL[1 + d] * n[d]; vnR += wR[1 + d] * n[d]; }
        const double hL = (uL[4] + pL) / uL[0], hR = (uR[4] + pR) / uR[0];
        const double r = std::sqrt(rR / rL), rp1 = r + 1.0;
        const double rho_a = r * rL;
        double va[3];
        for (int d = 0; d < 3; ++d) va[d] = (r * wR[1 + d] + wL[1 + d]) / rp1;
        const double ha = (r * hR + hL) / rp1;
        double v2a = 0.0; for (int d = 0; d < 3; ++d) v2a = v2a + va[d] * va[d];
        double vna = 0.0; for (int d = 0; d < 3; ++d) vna += va[d] * n[d];
        const double c2a = gm1 * (ha - 0.5 * v2a);
        double ca = 1e10;
        if (c2a > 0.0) ca = std::sqrt(c2a);
        double eig[3] = {std::fabs(vna - ca), std::fabs(vna), std::fabs(vna + ca)};
        const double cL = sound(rL, pL), cR = sound(rR, pR);
        const double eL[3] = {std::fabs(vnL - cL), std::fabs(vnL), std::fabs(vnL + cL)};
        const double eR[3] = {std::fabs(vnR - cR), std::fabs(vnR), std::fabs(vnR + cR)};
        const double dp = pR - pL, drho = rR - rL, dvn = vnR - vnL;
        double dvt[3];
        for (int d = 0; d < 3; ++d) dvt[d] = (wR[1 + d] - wL[1 + d]) - dvn * n[d];
        for (int e = 0; e < 3; ++e) {   // Harten entropy fix (convective_numerical_flux.cpp:215-232)
            const double eps = std::max(std::fabs(eig[e] - eL[e]), std::fabs(eR[e] - eig[e]));
            if (eig[e] < eps) eig[e] = 0.5 * (eig[e] * eig[e] / eps + eps);
        }
        const double c0 = eig[0] * (dp - rho_a * ca * dvn) / (2.0 * c2a);
        const double c1 = eig[1] * (drho - dp / c2a);
        const double c2 = eig[1] * rho_a;
        const double c3 = eig[2] * (dp + rho_a * ca * dvn) / (2.0 * c2a);
        double A[5];
        A[0] = c0 * 1.0;
        for (int d = 0; d < 3; ++d) A[1 + d] = c0 * (va[d] - ca * n[d]);
        A[4] = c0 * (ha - ca * vna);
        A[0] += c1 * 1.0;
        for (int d = 0; d < 3; ++d) A[1 + d] += c1 * va[d];
        A[4] += c1 * v2a * 0.5;
        A[0] += c2 * 0.0;
        double dvtv = 0.0;
        for (int d = 0; d < 3; ++d) { A[1 + d] += c2 * dvt[d]; dvtv += va[d] * dvt[d]; }
        A[4] += c2 * dvtv;
        A[0] += c3 * 1.0;
        for (int d = 0; d < 3; ++d) A[1 + d] += c3 * (va[d] + ca * n[d]);
        A[4] += c3 * (ha + ca * vna);
        for (int s = 0; s < 5; ++s) out[s] = -0.5 * A[s];
    }
    // dissipative numerical (auxiliary) flux dot n (viscous_numerical_flux.cpp:146-328)
    void diss_num_flux(const double* uL, const double* uR, const double gL[5][3], const double gR[5][3],
                       const double* n, double penalty, double* out) const {
        double fL[5], fR[5];
        viscous_flux_dot_n(uL, gL, n, fL);
        viscous_flux_dot_n(uR, gR, n, fR);
        for (int s = 0; s < 5; ++s) out[s] = 0.5 * (fL[s] + fR[s]);
        if (prm->diss_flux == SIPG) {
            double jump[5][3];
            for (int s = 0; s < 5; ++s) for (int d = 0; d < 3; ++d) jump[s][d] = (uL[s] - uR[s]) * n[d];
            double aL[5], aR[5];
            viscous_flux_dot_n(uL, jump, n, aL);
            viscous_flux_dot_n(uR, jump, n, aR);
            for (int s = 0; s < 5; ++s) out[s] = out[s] - penalty * (0.5 * (aL[s] + aR[s]));
        }
    }

    // ---- boundary conditions
    // free-stream primitive state (Euler::Euler, euler.cpp:14-70): density 1, velocities
    // (cos a cos b, sin a cos b, sin b) for the angle of attack a and side slip b, pressure 1/(gam M^2)
    void free_stream(double* w) const {
        w[0] = 1.0;
        w[1] = std::cos(prm->angle_of_attack) * std::cos(prm->side_slip_angle);
        w[2] = std::sin(prm->angle_of_attack) * std::cos(prm->side_slip_angle);
        w[3] = std::sin(prm->side_slip_angle);
        w[4] = 1.0 / (gam * mach2);
    }
    double entropy_measure(double rho, double p) const {   // euler.cpp:414-421
        double rc = rho;
        if (rc < 0.0) { positive(rc); return BIG_NUMBER; }
        return p * std::pow(rho, -gam);
    }
    double sound_of(const double* u) const {   // compute_sound(conservative), euler.cpp:535-543
        const double rho = positive(u[0]);
        const double p = pressure(u);
        return std::sqrt(p * gam / rho);
    }
    // boundary_slip_wall (euler.cpp:1171-1217): the normal velocity reflected
    void slip_wall(const double* n, const double* u, double* ub) const {
        double w[5], wb[5];
        primitive(u, w);
        wb[0] = w[0]; wb[4] = w[4];
        const double sn[3] = {-n[0], -n[1], -n[2]};
        double vn = 0.0;
        for (int d = 0; d < 3; ++d) vn = vn + w[1 + d] * sn[d];
        for (int d = 0; d < 3; ++d) wb[1 + d] = w[1 + d] - 2.0 * vn * sn[d];
        conservative_from_primitive(wb, ub);
    }
    // boundary_riemann (euler.cpp:1096-1169): characteristic farfield
    void riemann(const double* n, const double* u, double* ub) const {
        double wi[5], we[5], wb[5];
        primitive(u, wi);
        free_stream(we);
        const double ci = sound(wi[0], wi[4]), ce = sound(we[0], we[4]);
        double vni = 0.0, vne = 0.0;
        for (int d = 0; d < 3; ++d) { vni = vni + wi[1 + d] * n[d]; vne = vne + we[1 + d] * n[d]; }
        const double rout = vni + 2.0 / gm1 * ci, rinc = vne - 2.0 / gm1 * ce;
        const double vnb = 0.5 * (rout + rinc), cb = 0.25 * gm1 * (rout - rinc);
        if (std::fabs(vnb) >= std::fabs(cb)) {          // supersonic: inlet or outlet
            for (int s = 0; s < 5; ++s) wb[s] = vnb < 0.0 ? we[s] : wi[s];
        } else {                                       // subsonic
            double rb, vt[3];
            if (vnb < 0.0) {
                rb = std::pow(1.0 / gam * cb * cb / entropy_measure(we[0], we[4]), 1.0 / gm1);
                for (int d = 0; d < 3; ++d) vt[d] = we[1 + d] - vne * n[d];
            } else {
                rb = std::pow(1.0 / gam * cb * cb / entropy_measure(wi[0], wi[4]), 1.0 / gm1);
                for (int d = 0; d < 3; ++d) vt[d] = wi[1 + d] - vni * n[d];
            }
            for (int d = 0; d < 3; ++d) wb[1 + d] = vt[d] + vnb * n[d];
            wb[4] = 1.0 / gam * cb * cb * rb;
            wb[0] = rb;
        }
        conservative_from_primitive(wb, ub);
    }
    // boundary_pressure_outflow (euler.cpp:1287-1327), back pressure 0.99 (boundary_face_values)
    void pressure_outflow(double total_p, double back_p, const double* u, double* ub) const {
        double v2 = 0.0;
        for (int d = 0; d < 3; ++d) { const double v = u[1 + d] / u[0]; v2 = v2 + v * v; }
        const double mach = std::sqrt(v2) / sound_of(u);   // compute_mach_number, euler.cpp:555-563
        if (mach > 1.0) { for (int s = 0; s < 5; ++s) ub[s] = u[s]; return; }
        double wi[5], wb[5];
        primitive(u, wi);
        const double radicant = 1.0 + 0.5 * gm1 * mach2;
        const double p_inlet = total_p * std::pow(radicant, -gam / gm1);
        const double ge1 = (mach >= 1) ? 1.0 : 0.0;
        const double p_bc = ge1 * wi[4] + (1 - ge1) * back_p * p_inlet;
        const double t_int = gam * mach2 * (wi[4] / wi[0]);    // compute_temperature, :452-459
        wb[0] = gam * mach2 * (p_bc / t_int);                  // compute_density_from_pressure_temperature
        for (int d = 0; d < 3; ++d) wb[1 + d] = wi[1 + d];
        wb[4] = p_bc;
        conservative_from_primitive(wb, ub);
    }
    // boundary_inflow (euler.cpp:1329-1434), subsonic (mach_inf < 1) or supersonic
    void inflow(double total_p, double total_t, const double* n, const double* u, double* ub) const {
        double wi[5], wb[5];
        primitive(u, wi);
        const double nrm[3] = {-n[0], -n[1], -n[2]};
        double vni = 0.0;
        for (int d = 0; d < 3; ++d) vni += wi[1 + d] * nrm[d];
        const double ci = sound_of(u);
        const double mach_inf = prm->mach_inf;
        if (mach_inf < 1.0) {
            const double rpos = vni + 2.0 * ci / gm1;
            const double H = u[4] / wi[0] + wi[4] / wi[0];
            const double a = 1.0 + 2.0 / gm1;
            const double b = -2.0 * rpos;
            const double c = 0.5 * gm1 * (rpos * rpos - 2.0 * H);
            const double t1 = -0.5 * b / a;
            const double t2 = 0.5 * std::sqrt(b * b - 4.0 * a * c) / a;
            const double cb = std::max(t1 + t2, t1 - t2);
            const double vmag = rpos - 2.0 * cb / gm1;
            const double mach_bc = vmag / cb;
            const double radicant = 1.0 + 0.5 * gm1 * mach_bc * mach_bc;
            const double p_bc = total_p * std::pow(radicant, -gam / gm1);
            const double t_bc = total_t * std::pow(radicant, -1.0);
            wb[0] = gam * mach2 * (p_bc / t_bc);
            for (int d = 0; d < 3; ++d) wb[1 + d] = vmag * nrm[d];
            wb[4] = p_bc;
        } else {
            const double radicant = 1.0 + 0.5 * gm1 * mach2;
            const double p_bc = total_p * std::pow(radicant, -gam / gm1);
            const double t_bc = total_t * std::pow(radicant, -1.0);
            wb[0] = gam * mach2 * (p_bc / t_bc);
            const double cb = std::sqrt(gam * p_bc / wb[0]);
            const double vmag = mach_inf * cb;
            for (int d = 0; d < 3; ++d) wb[1 + d] = -vmag * n[d];
            wb[4] = p_bc;
        }
        conservative_from_primitive(wb, ub);
    }
    // Euler::boundary_face_values (euler.cpp:1508-1560): the exterior state of the convective flux
    void boundary_state(int type, const double* n, const double* u, double* ub) const {
        const double p_inf = 1.0 / (gam * mach2);
        const double t_inf = gam * p_inf / 1.0 * mach2;                       // euler.cpp:44
        const double total_p = p_inf * std::pow(1.0 + 0.5 * gm1 * mach2, gam / gm1);
        const double total_t = t_inf * std::pow(total_p / p_inf, gm1 / gam);
        switch (type) {
        case BC_WALL: case BC_SLIP_WALL: slip_wall(n, u, ub); break;   // boundary_wall = slip wall
        case BC_PRESSURE_OUTFLOW: pressure_outflow(total_p, 0.99, u, ub); break;
        case BC_INFLOW: inflow(total_p, total_t, n, u, ub); break;
        case BC_RIEMANN: riemann(n, u, ub); break;
        case BC_FARFIELD: {                                            // boundary_farfield, :1436-1450
            double w[5]; free_stream(w);
            conservative_from_primitive(w, ub);
            break;
        }
        case BC_EXTRAPOLATION: for (int s = 0; s < 5; ++s) ub[s] = u[s]; break;   // boundary_p0_extrapolation
        default: throw std::runtime_error("oracle: boundary type not restated");
        }
    }
    // NavierStokes::boundary_face_values_viscous_flux (navier_stokes.cpp:1354-1432): the exterior
    // state and gradient of the dissipative flux. 1001: no-slip (momentum negated, gradient the
    // interior's; adiabatic: energy gradient zero; isothermal: the exterior temperature
    // 2 T_wall - T_int); 1006: the interior state and gradient
    void boundary_viscous_state(int type, const double* u, const double g[5][3], double* ub, double gb[5][3]) const {
        if (type != BC_WALL && type != BC_SLIP_WALL)
            throw std::runtime_error("oracle: Navier-Stokes boundary type without a viscous exterior state");
        for (int s = 0; s < 5; ++s) for (int d = 0; d < 3; ++d) gb[s][d] = g[s][d];
        if (type == BC_SLIP_WALL) { for (int s = 0; s < 5; ++s) ub[s] = u[s]; return; }
        ub[0] = u[0]; ub[4] = u[4];
        for (int d = 0; d < 3; ++d) ub[1 + d] = -u[1 + d];
        if (prm->thermal_bc == THERMAL_ADIABATIC) for (int d = 0; d < 3; ++d) gb[4][d] = 0.0;
        if (prm->thermal_bc == THERMAL_ISOTHERMAL) {
            double wi[5], we[5];
            primitive(u, wi);
            primitive(ub, we);
            const double t_int = gam * mach2 * (wi[4] / wi[0]);
            const double t_ext = 2.0 * prm->wall_temperature - t_int;
            we[4] = we[0] * t_ext / (gam * mach2);   // compute_pressure_from_density_temperature
            double w2[5]; conservative_from_primitive(we, w2);
            ub[4] = w2[4];                          // compute_total_energy
        }
    }
    // evaluate_auxiliary_flux on a boundary face (viscous_numerical_flux.cpp:66-328, on_boundary):
    // BR2 and SIPG take the exterior gradient, the central flux the interior one; on an adiabatic
    // 1001 wall both sides' fluxes drop the heat flux (navier_stokes.cpp:1224-1264)
    void diss_boundary_flux(int type, const double* ui, const double* ub, const double gi[5][3],
                            const double gb[5][3], const double* n, double penalty, double* out) const {
        const bool ad = prm->thermal_bc == THERMAL_ADIABATIC && type == BC_WALL;
        double fi[5], fb[5];
        viscous_flux_dot_n(ui, gi, n, fi, ad);
        viscous_flux_dot_n(ub, prm->diss_flux == CENTRAL_VISC ? gi : gb, n, fb, ad);
        for (int s = 0; s < 5; ++s) out[s] = 0.5 * (fi[s] + fb[s]);
        if (prm->diss_flux == SIPG) {
            double jump[5][3];
            for (int s = 0; s < 5; ++s) for (int d = 0; d < 3; ++d) jump[s][d] = (ui[s] - ub[s]) * n[d];
            double aL[5], aR[5];
            viscous_flux_dot_n(ui, jump, n, aL, ad);
            viscous_flux_dot_n(ub, jump, n, aR, ad);
            for (int s = 0; s < 5; ++s) out[s] = out[s] - penalty * (0.5 * (aL[s] + aR[s]));
        }
    }
};

// ---------------------------------------------------------------------------------
// Mesh: deal.II cell order for the periodic cube (straight_periodic_cube.cpp:17-68).
// hyper_cube + refine_global(log2 n) gives recursive-child (Morton, child = x+2y+4z)
// order; subdivided_hyper_cube(n) gives lexicographic order (x fastest).
// ---------------------------------------------------------------------------------
static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Sine warp of the periodic cube [l, r]^3 (L = r - l, k = 2 pi / L): every coordinate is
// moved by the same amount a/k sin(k(x-l)) sin(k(y-l)) sin(k(z-l)), which vanishes on the
// cube's faces, so periodic faces still match (for [0, 2 pi]^3: x_i += a sin x sin y sin z).
// Not a reference grid: the reference's curved periodic grids (curved_periodic_grid.cpp,
// nonsymmetric_curved_periodic_grid.cpp) use other warps; the construction is the same:
// the mapping support points are the manifold's images of the straight-sided points.
static void warp_point(double left, double right, double a, double X[3]) {
    const double k = 2.0 * PI / (right - left);
    const double s = a / k * std::sin(k * (X[0] - left)) * std::sin(k * (X[1] - left)) * std::sin(k * (X[2] - left));
    X[0] += s; X[1] += s; X[2] += s;
}

// Metric cofactor by the conservative curl form (operators.cpp:2738-2884) at the points
// selected by the 1-D operators A[d] (mapping basis values there, r[d] rows each) and
// dA[d] (their derivatives). P holds the nine products X_l dX_m/dxi_j at the grid nodes:
// P[0..2] = z dy/dxi_j, P[3..5] = x dz/dxi_j, P[6..8] = y dx/dxi_j. C is [npts][9].
static void cofactor_at(const double* const A[3], const double* const dA[3], const int r[3], int ng,
                        const std::vector<double> P[9], double* C) {
    const int npts = r[0] * r[1] * r[2];
    std::vector<double> t(npts), acc(npts);
    auto D = [&](int e, const std::vector<double>& f, bool adding, double factor) {
        const double* B[3] = {A[0], A[1], A[2]};
        B[e] = dA[e];
        apply3(B[0], r[0], ng, B[1], r[1], ng, B[2], r[2], ng, f.data(), acc.data(), adding, factor);
    };
    // row l of C from the products of row l: C[l][0] = -D_eta(f_zeta) + D_zeta(f_eta),
    // C[l][1] = D_xi(f_zeta) - D_zeta(f_xi), C[l][2] = -D_xi(f_eta) + D_eta(f_xi)
    for (int l = 0; l < 3; ++l) {
        const std::vector<double>* f = &P[3 * l];
        D(1, f[2], false, -1.0); D(2, f[1], true, 1.0);
        for (int q = 0; q < npts; ++q) C[q * 9 + l * 3 + 0] = acc[q];
        D(0, f[2], false, 1.0); D(2, f[0], true, -1.0);
        for (int q = 0; q < npts; ++q) C[q * 9 + l * 3 + 1] = acc[q];
        D(0, f[1], false, -1.0); D(1, f[0], true, 1.0);
        for (int q = 0; q < npts; ++q) C[q * 9 + l * 3 + 2] = acc[q];
    }
}

static double det3(const double J[3][3]) {
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

// Curvilinear metric terms of cell c: mapping support points on the GLL points of degree
// grid_degree (FE_Q support points in lexicographic order, strong_dg.cpp:68-75), det J at
// the volume flux nodes (operators.cpp:2591-2672), cofactor at the volume flux nodes and
// at every face's flux nodes (operators.cpp:2444-2589), and the physical positions of the
// solution support points.
static void build_curvilinear_cell(Mesh& m, const Ops1D& ops, int c) {
    const int ng = m.grid_degree + 1, ng3 = ng * ng * ng;
    const int nq = ops.nq, nd = ops.nd, nq3 = nq * nq * nq, nf = nq * nq;
    std::vector<double> xg, wg; gauss_lobatto(ng, xg, wg);
    std::vector<double> Bg(ng * ng), dBg(ng * ng), Bf(nq * ng), dBf(nq * ng), Bx(nd * ng);
    std::vector<double> Bs[2] = {std::vector<double>(ng), std::vector<double>(ng)};
    std::vector<double> dBs[2] = {std::vector<double>(ng), std::vector<double>(ng)};
    for (int a = 0; a < ng; ++a) lagrange_eval(xg, xg[a], &Bg[a * ng], &dBg[a * ng]);
    for (int q = 0; q < nq; ++q) lagrange_eval(xg, ops.xq[q], &Bf[q * ng], &dBf[q * ng]);
    for (int i = 0; i < nd; ++i) lagrange_eval(xg, ops.xs[i], &Bx[i * ng], nullptr);
    lagrange_eval(xg, 0.0, Bs[0].data(), dBs[0].data());
    lagrange_eval(xg, 1.0, Bs[1].data(), dBs[1].data());
    const auto t = m.ijk[c];
    std::vector<double> X[3] = {std::vector<double>(ng3), std::vector<double>(ng3), std::vector<double>(ng3)};
    for (int k = 0; k < ng; ++k) for (int j = 0; j < ng; ++j) for (int i = 0; i < ng; ++i) {
        double p[3] = {m.left + m.h * (t[0] + xg[i]), m.left + m.h * (t[1] + xg[j]), m.left + m.h * (t[2] + xg[k])};
        warp_point(m.left, m.right, m.warp, p);
        for (int d = 0; d < 3; ++d) X[d][(k * ng + j) * ng + i] = p[d];
    }
    // gradient of the support points at the grid nodes (the Jacobian there)
    std::vector<double> GX[3][3];
    for (int mm = 0; mm < 3; ++mm)
        for (int j = 0; j < 3; ++j) {
            GX[mm][j].resize(ng3);
            const double* B[3] = {Bg.data(), Bg.data(), Bg.data()};
            B[j] = dBg.data();
            apply3(B[0], ng, ng, B[1], ng, ng, B[2], ng, ng, X[mm].data(), GX[mm][j].data(), false, 1.0);
        }
    std::vector<double> P[9];
    for (int j = 0; j < 3; ++j) {
        P[j].resize(ng3); P[3 + j].resize(ng3); P[6 + j].resize(ng3);
        for (int g = 0; g < ng3; ++g) {
            P[j][g] = X[2][g] * GX[1][j][g];        // z dy/dxi_j
            P[3 + j][g] = X[0][g] * GX[2][j][g];    // x dz/dxi_j
            P[6 + j][g] = X[1][g] * GX[0][j][g];    // y dx/dxi_j
        }
    }
    // volume flux nodes
    {
        const double* A[3] = {Bf.data(), Bf.data(), Bf.data()};
        const double* dA[3] = {dBf.data(), dBf.data(), dBf.data()};
        const int r[3] = {nq, nq, nq};
        cofactor_at(A, dA, r, ng, P, &m.cof[(size_t)c * nq3 * 9]);
        std::vector<double> Jm[3][3];
        for (int mm = 0; mm < 3; ++mm)
            for (int j = 0; j < 3; ++j) {
                Jm[mm][j].resize(nq3);
                const double* B[3] = {Bf.data(), Bf.data(), Bf.data()};
                B[j] = dBf.data();
                apply3(B[0], nq, ng, B[1], nq, ng, B[2], nq, ng, X[mm].data(), Jm[mm][j].data(), false, 1.0);
            }
        for (int q = 0; q < nq3; ++q) {
            double J[3][3];
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) J[a][b] = Jm[a][b][q];
            const double dj = det3(J);
            if (dj <= 1e-14) throw std::runtime_error("oracle: non-positive det J (operators.cpp:2667-2670)");
            m.detj[(size_t)c * nq3 + q] = dj;
        }
    }
    // facet flux nodes of each face, interior side (operators.cpp:2501-2589)
    for (int f = 0; f < 6; ++f) {
        const int dn = f / 2, side = f % 2;
        const double* A[3] = {Bf.data(), Bf.data(), Bf.data()};
        const double* dA[3] = {dBf.data(), dBf.data(), dBf.data()};
        int r[3] = {nq, nq, nq};
        A[dn] = Bs[side].data(); dA[dn] = dBs[side].data(); r[dn] = 1;
        cofactor_at(A, dA, r, ng, P, &m.cof_face[((size_t)c * 6 + f) * nf * 9]);
    }
    // solution support points in physical space
    const int nd3 = nd * nd * nd;
    std::vector<double> xs(nd3);
    for (int d = 0; d < 3; ++d) {
        apply3(Bx.data(), nd, ng, Bx.data(), nd, ng, Bx.data(), nd, ng, X[d].data(), xs.data(), false, 1.0);
        for (int i = 0; i < nd3; ++i) m.xnode[((size_t)c * nd3 + i) * 3 + d] = xs[i];
    }
}

Mesh build_periodic_cube(int n, double left, double right, int order, const Ops1D& ops,
                         double warp, int grid_degree) {
    Mesh m;
    m.n = n; m.nc = n * n * n; m.left = left; m.right = right;
    m.order = (order == ORDER_AUTO) ? (is_pow2(n) ? ORDER_MORTON : ORDER_LEXICOGRAPHIC) : order;
    m.h = (right - left) / n;
    m.ijk.resize(m.nc); m.cell_of.assign(m.nc, -1); m.nbr.resize(m.nc);
    m.bnd.assign(m.nc, {0, 0, 0, 0, 0, 0});
    if (m.order == ORDER_MORTON) {
        int levels = 0; while ((1 << levels) < n) ++levels;
        for (int c = 0; c < m.nc; ++c) {
            int ix = 0, iy = 0, iz = 0;
            for (int l = 0; l < levels; ++l) {
                const int child = (c >> (3 * (levels - 1 - l))) & 7;
                ix = 2 * ix + (child & 1); iy = 2 * iy + ((child >> 1) & 1); iz = 2 * iz + ((child >> 2) & 1);
            }
            m.ijk[c] = {ix, iy, iz};
        }
    } else {
        for (int c = 0; c < m.nc; ++c) m.ijk[c] = {c % n, (c / n) % n, c / (n * n)};
    }
    for (int c = 0; c < m.nc; ++c) { auto& t = m.ijk[c]; m.cell_of[(t[2] * n + t[1]) * n + t[0]] = c; }
    for (int c = 0; c < m.nc; ++c) {
        auto t = m.ijk[c];
        for (int f = 0; f < 6; ++f) {
            auto u = t; const int d = f / 2; const int s = (f % 2) ? 1 : -1;
            u[d] = (u[d] + s + n) % n;
            m.nbr[c][f] = m.cell_of[(u[2] * n + u[1]) * n + u[0]];
        }
    }
    const int nq = ops.nq, nq3 = nq * nq * nq, nd = ops.nd;
    m.cof.assign((size_t)m.nc * nq3 * 9, 0.0);
    m.detj.assign((size_t)m.nc * nq3, 0.0);
    m.cof_face.assign((size_t)m.nc * 6 * nq * nq * 9, 0.0);
    m.xnode.assign((size_t)m.nc * nd * nd * nd * 3, 0.0);
    m.warp = warp; m.grid_degree = grid_degree;
    m.affine = (warp == 0.0);
    if (!m.affine) {
        if (grid_degree < 1) throw std::runtime_error("oracle: grid_degree must be >= 1");
#pragma omp parallel for schedule(static)
        for (int c = 0; c < m.nc; ++c) build_curvilinear_cell(m, ops, c);
        return m;
    }
    const double h = m.h;
    for (int c = 0; c < m.nc; ++c) {
        for (int q = 0; q < nq3; ++q) {
            double* C = &m.cof[((size_t)c * nq3 + q) * 9];
            C[0] = C[4] = C[8] = h * h;
            m.detj[(size_t)c * nq3 + q] = h * h * h;
        }
        for (int f = 0; f < 6 * nq * nq; ++f) {
            double* C = &m.cof_face[((size_t)c * 6 * nq * nq + f) * 9];
            C[0] = C[4] = C[8] = h * h;
        }
        const auto t = m.ijk[c];
        for (int k = 0; k < nd; ++k) for (int j = 0; j < nd; ++j) for (int i = 0; i < nd; ++i) {
            double* X = &m.xnode[(((size_t)c * nd + k) * nd + j) * nd * 3 + i * 3];
            X[0] = left + h * (t[0] + ops.xs[i]);
            X[1] = left + h * (t[1] + ops.xs[j]);
            X[2] = left + h * (t[2] + ops.xs[k]);
        }
    }
    return m;
}

void Solver::init(const Params& p, int n, double left, double right, int order, double warp, int grid_degree) {
    prm = p;
    ops = build_ops(prm);
    mesh = build_periodic_cube(n, left, right, order, ops, warp, grid_degree);
    nd3 = ops.nd * ops.nd * ops.nd;
    nq3 = ops.nq * ops.nq * ops.nq;
    ndofs_cell = NSTATE * nd3;
    aux.assign(3 * ndofs(), 0.0);
    status = 0;
}

void Solver::set_boundaries(const int types[6]) {
    for (int d = 0; d < 3; ++d)
        if ((types[2 * d] == 0) != (types[2 * d + 1] == 0))
            throw std::runtime_error("oracle: a pair of cube sides is periodic on both sides or on neither");
    for (int f = 0; f < 6; ++f) {
        const int t = types[f];
        if (t != 0 && (t < BC_WALL || t > BC_EXTRAPOLATION))
            throw std::runtime_error("oracle: boundary type not restated");
        // the Navier-Stokes viscous boundary state exists for 1000, 1001 and 1006 only
        // (navier_stokes.cpp:1354-1390)
        if (t != 0 && prm.pde == NAVIER_STOKES && t != BC_WALL && t != BC_SLIP_WALL)
            throw std::runtime_error("oracle: Navier-Stokes takes wall (1001) and slip-wall (1006) boundaries");
    }
    const int n = mesh.n;
    for (int c = 0; c < mesh.nc; ++c) {
        const auto t = mesh.ijk[c];
        for (int f = 0; f < 6; ++f) {
            const int d = f / 2;
            const bool side = (f % 2) ? t[d] == n - 1 : t[d] == 0;
            if (types[f] != 0 && side) { mesh.nbr[c][f] = -1; mesh.bnd[c][f] = types[f]; }
        }
    }
}

void Solver::boundary_values(int type, const double* n, const double* u, const double* g, double* ub_conv,
                             double* ub_visc, double* gb_visc) {
    Physics phys(&prm, &status);
    phys.boundary_state(type, n, u, ub_conv);
    double gi[5][3], gb[5][3] = {};
    for (int s = 0; s < 5; ++s) for (int d = 0; d < 3; ++d) gi[s][d] = g[s * 3 + d];
    if (type == BC_WALL || type == BC_SLIP_WALL) phys.boundary_viscous_state(type, u, gi, ub_visc, gb);
    else for (int s = 0; s < 5; ++s) ub_visc[s] = ub_conv[s];
    for (int s = 0; s < 5; ++s) for (int d = 0; d < 3; ++d) gb_visc[s * 3 + d] = gb[s][d];
}

// ---------------------------------------------------------------------------------
// Residual assembly
// ---------------------------------------------------------------------------------
namespace {

struct Face {   // geometry helper for a face of the reference cube
    int dn, side;
};

// surface interpolation: dir dn uses the 1 x c surface row; others the volume op
inline void surf_apply(const Ops1D& o, const double* vol_op, int r, int c, const double* surf_row,
                       int iface, const double* in, double* out, bool adding, double factor) {
    const int dn = iface / 2;
    const double* A[3] = {vol_op, vol_op, vol_op};
    int R[3] = {r, r, r};
    A[dn] = surf_row; R[dn] = 1;
    (void)o;
    apply3(A[0], R[0], c, A[1], R[1], c, A[2], R[2], c, in, out, adding, factor);
}
inline void surf_inner(const double* vol_op, int r, int c, const double* surf_row, int iface,
                       const double* in, const double* w, double* out, bool adding, double factor) {
    const int dn = iface / 2;
    const double* A[3] = {vol_op, vol_op, vol_op};
    int R[3] = {r, r, r};
    A[dn] = surf_row; R[dn] = 1;
    inner3(A[0], R[0], c, A[1], R[1], c, A[2], R[2], c, in, w, out, adding, factor);
}
// volume node on the normal line through face node f at position l
inline int line_node(int dn, int f, int l, int n) {
    int c[3];
    const int t1 = (dn == 0) ? 1 : 0, t2 = (dn == 2) ? 1 : 2;
    c[dn] = l; c[t1] = f % n; c[t2] = f / n;
    return (c[2] * n + c[1]) * n + c[0];
}

} // namespace

void Solver::assemble_residual(const double* U, double* R) {
    const Ops1D& o = ops;
    const int nd = o.nd, nq = o.nq, nf = nq * nq;
    const int nc = mesh.nc;
    const size_t ndc = (size_t)ndofs_cell;
    Physics phys(&prm, &status);
    const bool viscous = (prm.pde == NAVIER_STOKES);
    const bool split = prm.use_split_form != 0;
    const double* chi = o.chi.data();
    const double* dphi = o.dphi.data();
    const double* phi = o.phi.data();
    std::vector<double> Wvol(nq3), Wface(nf), ones_vol(nq3, 1.0), ones_face(nf, 1.0);
    for (int k = 0; k < nq; ++k) for (int j = 0; j < nq; ++j) for (int i = 0; i < nq; ++i)
        Wvol[(k * nq + j) * nq + i] = o.wq[i] * o.wq[j] * o.wq[k];
    for (int j = 0; j < nq; ++j) for (int i = 0; i < nq; ++i) Wface[j * nq + i] = o.wq[i] * o.wq[j];
    const double* nref[6];
    static const double NREF[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int f = 0; f < 6; ++f) nref[f] = NREF[f];

    auto penalty_of = [&](int /*c*/, int /*f*/) {   // dg_base.cpp:397-413
        const int p = prm.poly_degree;
        const double degsq = (p == 0) ? 1.0 : (double)p * (p + 1);
        return degsq / mesh.h * prm.sipg_penalty_factor;
    };

    // ------------------------------ auxiliary equation (strong_dg.cpp:498-1008)
    if (viscous) {
        std::vector<double> aux_rhs(3 * ndofs(), 0.0);
#pragma omp parallel for schedule(static)
        for (int c = 0; c < nc; ++c) {
            const double* Uc = U + (size_t)c * ndc;
            std::vector<double> uq(nq3), g(nq3), pg(nq3), rhs(nd3);
            std::vector<std::vector<double>> rg(3, std::vector<double>(nq3));
            double* out[3];
            for (int d = 0; d < 3; ++d) out[d] = aux_rhs.data() + d * ndofs() + (size_t)c * ndc;
            for (int s = 0; s < NSTATE; ++s) {
                // volume part (strong_dg.cpp:666-724)
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, Uc + s * nd3, uq.data(), false, 1.0);
                apply3(dphi, nq, nq, phi, nq, nq, phi, nq, nq, uq.data(), rg[0].data(), false, 1.0);
                apply3(phi, nq, nq, dphi, nq, nq, phi, nq, nq, uq.data(), rg[1].data(), false, 1.0);
                apply3(phi, nq, nq, phi, nq, nq, dphi, nq, nq, uq.data(), rg[2].data(), false, 1.0);
                for (int d = 0; d < 3; ++d) {
                    for (int q = 0; q < nq3; ++q) {
                        const double* C = &mesh.cof[((size_t)c * nq3 + q) * 9];
                        double v = 0.0;
                        for (int j = 0; j < 3; ++j) v += C[d * 3 + j] * rg[j][q];
                        pg[q] = v;
                    }
                    inner3(chi, nq, nd, chi, nq, nd, chi, nq, nd, pg.data(), Wvol.data(), rhs.data(), false, 1.0);
                    for (int i = 0; i < nd3; ++i) out[d][s * nd3 + i] += rhs[i];
                }
            }
            // face part: this cell's side of each of its 6 faces (strong_dg.cpp:871-1008)
            for (int f = 0; f < 6; ++f) {
                const int bt = mesh.bnd[c][f];
                const int cn = bt ? c : mesh.nbr[c][f];
                const int fn = (f % 2) ? f - 1 : f + 1;
                const double* Un = U + (size_t)cn * ndc;
                // int = owner (lower index) as in dg_base.cpp:417-449; this cell may be either side.
                // A boundary face (strong_dg.cpp:725-866): this cell is the interior side and the
                // exterior state is the viscous boundary state of its face values
                const bool owner = bt || c < cn;
                const int ci = owner ? c : cn, fi = owner ? f : fn, ce = owner ? cn : c, fe = owner ? fn : f;
                const double* Ui = owner ? Uc : Un; const double* Ue = owner ? Un : Uc;
                std::vector<double> si(NSTATE * nf), se(NSTATE * nf);
                for (int s = 0; s < NSTATE; ++s) {
                    surf_apply(o, chi, nq, nd, o.chi_s[fi % 2].data(), fi, Ui + s * nd3, &si[s * nf], false, 1.0);
                    surf_apply(o, chi, nq, nd, o.chi_s[fe % 2].data(), fe, Ue + s * nd3, &se[s * nf], false, 1.0);
                }
                if (bt) {
                    for (int q = 0; q < nf; ++q) {
                        double ui[5], ub[5], g0[5][3] = {}, gb[5][3];
                        for (int s = 0; s < 5; ++s) ui[s] = si[s * nf + q];
                        phys.boundary_viscous_state(bt, ui, g0, ub, gb);
                        for (int s = 0; s < 5; ++s) se[s * nf + q] = ub[s];
                    }
                }
                std::vector<double> term(nf);
                for (int d = 0; d < 3; ++d) {
                    for (int s = 0; s < NSTATE; ++s) {
                        for (int q = 0; q < nf; ++q) {
                            const double* C = &mesh.cof_face[(((size_t)ci * 6 + fi) * nf + q) * 9];
                            double np[3];
                            for (int a = 0; a < 3; ++a) { np[a] = 0.0; for (int b = 0; b < 3; ++b) np[a] += C[a * 3 + b] * nref[fi][b]; }
                            double J = std::sqrt(np[0] * np[0] + np[1] * np[1] + np[2] * np[2]);
                            for (int a = 0; a < 3; ++a) np[a] /= J;
                            const double ustar = 0.5 * (si[s * nf + q] + se[s * nf + q]);
                            if (owner) term[q] = (ustar - si[s * nf + q]) * np[d] * J;
                            else term[q] = (ustar - se[s * nf + q]) * (-np[d]) * J;
                        }
                        const int fme = owner ? fi : fe;
                        surf_inner(chi, nq, nd, o.chi_s[fme % 2].data(), fme, term.data(), Wface.data(), rhs.data(), false, 1.0);
                        for (int i = 0; i < nd3; ++i) out[d][s * nd3 + i] += rhs[i];
                    }
                }
                (void)ce;
            }
        }
        // aux = M_aux^{-1} aux_rhs per dimension
        for (int d = 0; d < 3; ++d) apply_inverse_mass(aux_rhs.data() + d * ndofs(), aux.data() + d * ndofs(), true);
    }

    // ------------------------------ primary equations
    std::fill(R, R + ndofs(), 0.0);
    // entropy-projected states per cell (volume nodes), computed once per cell
#pragma omp parallel for schedule(dynamic, 4)
    for (int c = 0; c < nc; ++c) {
        const double* Uc = U + (size_t)c * ndc;
        double* Rc = R + (size_t)c * ndc;
        auto auxc = [&](int cell, int d) { return aux.data() + d * ndofs() + (size_t)cell * ndc; };
        // ---- volume term (strong_dg.cpp:1016-1579)
        std::vector<double> uq(NSTATE * nq3), aq(NSTATE * 3 * nq3), ev(NSTATE * nq3), ecoef(nd3), pe(NSTATE * nq3);
        for (int s = 0; s < NSTATE; ++s) {
            apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, Uc + s * nd3, &uq[s * nq3], false, 1.0);
            for (int d = 0; d < 3; ++d)
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, auxc(c, d) + s * nd3, &aq[(s * 3 + d) * nq3], false, 1.0);
        }
        std::vector<double> ucons(NSTATE * nq3);   // conservative state from projected entropy variables
        if (split) {
            for (int q = 0; q < nq3; ++q) {
                double u[5], v[5];
                for (int s = 0; s < 5; ++s) u[s] = uq[s * nq3 + q];
                phys.entropy_vars(u, v);
                for (int s = 0; s < 5; ++s) ev[s * nq3 + q] = v[s];
            }
            for (int s = 0; s < NSTATE; ++s) {
                apply3(o.proj.data(), nd, nq, o.proj.data(), nd, nq, o.proj.data(), nd, nq, &ev[s * nq3], ecoef.data(), false, 1.0);
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, ecoef.data(), &pe[s * nq3], false, 1.0);
            }
            for (int q = 0; q < nq3; ++q) {
                double v[5], u[5];
                for (int s = 0; s < 5; ++s) v[s] = pe[s * nq3 + q];
                phys.cons_from_entropy(v, u);
                for (int s = 0; s < 5; ++s) ucons[s * nq3 + q] = u[s];
            }
        }
        std::vector<double> conv_ref(NSTATE * 3 * nq3, 0.0), diff_ref(NSTATE * 3 * nq3, 0.0);
        std::vector<double> twopt;
        if (split) twopt.assign((size_t)NSTATE * 3 * nq3 * nq, 0.0);
        for (int q = 0; q < nq3; ++q) {
            double u[5], g[5][3];
            for (int s = 0; s < 5; ++s) { u[s] = uq[s * nq3 + q]; for (int d = 0; d < 3; ++d) g[s][d] = aq[(s * 3 + d) * nq3 + q]; }
            const double* Ci = &mesh.cof[((size_t)c * nq3 + q) * 9];
            if (split) {
                for (int s = 0; s < 5; ++s) u[s] = ucons[s * nq3 + q];
                const int xi[3] = {q % nq, (q / nq) % nq, q / (nq * nq)};
                for (int l = 0; l < nq; ++l) {
                    for (int rd = 0; rd < 3; ++rd) {
                        int xj[3] = {xi[0], xi[1], xi[2]}; xj[rd] = l;
                        const int j = (xj[2] * nq + xj[1]) * nq + xj[0];
                        const double* Cj = &mesh.cof[((size_t)c * nq3 + j) * 9];
                        double uj[5]; for (int s = 0; s < 5; ++s) uj[s] = ucons[s * nq3 + j];
                        double F[5][3]; phys.two_point(u, uj, F);
                        for (int s = 0; s < 5; ++s) {
                            double v = 0.0;
                            for (int k = 0; k < 3; ++k) v += 0.5 * (Ci[k * 3 + rd] + Cj[k * 3 + rd]) * F[s][k];
                            twopt[((size_t)(s * 3 + rd) * nq3 + q) * nq + l] = v;
                        }
                    }
                }
            } else {
                double F[5][3]; phys.convective_flux(u, F);
                for (int s = 0; s < 5; ++s) for (int d = 0; d < 3; ++d) {
                    double v = 0.0; for (int k = 0; k < 3; ++k) v += Ci[k * 3 + d] * F[s][k];
                    conv_ref[(s * 3 + d) * nq3 + q] = v;
                }
            }
            if (viscous) {
                double F[5][3]; phys.viscous_flux(u, g, F);
                for (int s = 0; s < 5; ++s) for (int d = 0; d < 3; ++d) {
                    double v = 0.0; for (int k = 0; k < 3; ++k) v += Ci[k * 3 + d] * F[s][k];
                    diff_ref[(s * 3 + d) * nq3 + q] = v;
                }
            }
        }
        std::vector<double> div(nq3), ddiv(nq3), rhs(nd3);
        for (int s = 0; s < NSTATE; ++s) {
            if (split) {
                for (int q = 0; q < nq3; ++q) {
                    const int xi[3] = {q % nq, (q / nq) % nq, q / (nq * nq)};
                    double v = 0.0;
                    for (int rd = 0; rd < 3; ++rd) {
                        const int a = (rd + 1) % 3, b = (rd + 2) % 3;
                        // skew row of the node's coordinate in rd, times the two perpendicular weights
                        for (int l = 0; l < nq; ++l) {
                            const double Q = o.skew[xi[rd] * nq + l] * o.wq[xi[std::min(a, b)]] * o.wq[xi[std::max(a, b)]];
                            v += Q * twopt[((size_t)(s * 3 + rd) * nq3 + q) * nq + l];
                        }
                    }
                    div[q] = v;
                }
                inner3(chi, nq, nd, chi, nq, nd, chi, nq, nd, div.data(), ones_vol.data(), rhs.data(), false, -1.0);
            } else {
                apply3(dphi, nq, nq, phi, nq, nq, phi, nq, nq, &conv_ref[(s * 3 + 0) * nq3], div.data(), false, 1.0);
                apply3(phi, nq, nq, dphi, nq, nq, phi, nq, nq, &conv_ref[(s * 3 + 1) * nq3], div.data(), true, 1.0);
                apply3(phi, nq, nq, phi, nq, nq, dphi, nq, nq, &conv_ref[(s * 3 + 2) * nq3], div.data(), true, 1.0);
                inner3(chi, nq, nd, chi, nq, nd, chi, nq, nd, div.data(), Wvol.data(), rhs.data(), false, -1.0);
            }
            if (viscous) {
                apply3(dphi, nq, nq, phi, nq, nq, phi, nq, nq, &diff_ref[(s * 3 + 0) * nq3], ddiv.data(), false, 1.0);
                apply3(phi, nq, nq, dphi, nq, nq, phi, nq, nq, &diff_ref[(s * 3 + 1) * nq3], ddiv.data(), true, 1.0);
                apply3(phi, nq, nq, phi, nq, nq, dphi, nq, nq, &diff_ref[(s * 3 + 2) * nq3], ddiv.data(), true, 1.0);
                inner3(chi, nq, nd, chi, nq, nd, chi, nq, nd, ddiv.data(), Wvol.data(), rhs.data(), true, -1.0);
            } else {
                // the reference adds -chi^T W div(F_v) with F_v == 0 for Euler: a no-op
            }
            for (int i = 0; i < nd3; ++i) Rc[s * nd3 + i] += rhs[i];
        }

        // ---- face terms (strong_dg.cpp:2367-3576); this cell's side of each face
        for (int f = 0; f < 6; ++f) {
            // a boundary face (assemble_boundary_term_strong, strong_dg.cpp:1582-2366): this cell is
            // the interior side with its own hybrid and volume-flux terms; the numerical fluxes take
            // the boundary states at the face nodes (the "exterior" arrays below are unused)
            const int bt = mesh.bnd[c][f];
            const int cn = bt ? c : mesh.nbr[c][f];
            const int fn = (f % 2) ? f - 1 : f + 1;
            const bool owner = bt || c < cn;
            const int ci = owner ? c : cn, fi = owner ? f : fn, ce = bt ? c : (owner ? cn : c);
            const int fe = bt ? f : (owner ? fn : f);
            const double* Ui = U + (size_t)ci * ndc;
            const double* Ue = U + (size_t)ce * ndc;
            const int dni = fi / 2, dne = fe / 2;
            // interpolations (strong_dg.cpp:2420-2470)
            std::vector<double> vi(NSTATE * nq3), ve(NSTATE * nq3), si(NSTATE * nf), se(NSTATE * nf);
            std::vector<double> avi(NSTATE * 3 * nq3), ave(NSTATE * 3 * nq3), asi(NSTATE * 3 * nf), ase(NSTATE * 3 * nf);
            for (int s = 0; s < NSTATE; ++s) {
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, Ui + s * nd3, &vi[s * nq3], false, 1.0);
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, Ue + s * nd3, &ve[s * nq3], false, 1.0);
                surf_apply(o, chi, nq, nd, o.chi_s[fi % 2].data(), fi, Ui + s * nd3, &si[s * nf], false, 1.0);
                surf_apply(o, chi, nq, nd, o.chi_s[fe % 2].data(), fe, Ue + s * nd3, &se[s * nf], false, 1.0);
                for (int d = 0; d < 3; ++d) {
                    apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, auxc(ci, d) + s * nd3, &avi[(s * 3 + d) * nq3], false, 1.0);
                    apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, auxc(ce, d) + s * nd3, &ave[(s * 3 + d) * nq3], false, 1.0);
                    surf_apply(o, chi, nq, nd, o.chi_s[fi % 2].data(), fi, auxc(ci, d) + s * nd3, &asi[(s * 3 + d) * nf], false, 1.0);
                    surf_apply(o, chi, nq, nd, o.chi_s[fe % 2].data(), fe, auxc(ce, d) + s * nd3, &ase[(s * 3 + d) * nf], false, 1.0);
                }
            }
            // reference volume fluxes interpolated to the face, dotted with the unit reference normal (:2836-3041)
            std::vector<double> cfi(NSTATE * nf, 0.0), cfe(NSTATE * nf, 0.0), dfi(NSTATE * nf, 0.0), dfe(NSTATE * nf, 0.0);
            {
                std::vector<double> cri(NSTATE * nq3), cre(NSTATE * nq3), dri(NSTATE * nq3), dre(NSTATE * nq3);
                for (int side = 0; side < 2; ++side) {
                    const int cc = side ? ce : ci; const int dn = side ? dne : dni;
                    const std::vector<double>& vv = side ? ve : vi; const std::vector<double>& aa = side ? ave : avi;
                    std::vector<double>& cr = side ? cre : cri; std::vector<double>& dr = side ? dre : dri;
                    for (int q = 0; q < nq3; ++q) {
                        double u[5], g[5][3];
                        for (int s = 0; s < 5; ++s) { u[s] = vv[s * nq3 + q]; for (int d = 0; d < 3; ++d) g[s][d] = aa[(s * 3 + d) * nq3 + q]; }
                        const double* C = &mesh.cof[((size_t)cc * nq3 + q) * 9];
                        if (!split) {
                            double F[5][3]; phys.convective_flux(u, F);
                            for (int s = 0; s < 5; ++s) { double v = 0.0; for (int k = 0; k < 3; ++k) v += C[k * 3 + dn] * F[s][k]; cr[s * nq3 + q] = v; }
                        }
                        double F[5][3]; phys.viscous_flux(u, g, F);
                        for (int s = 0; s < 5; ++s) { double v = 0.0; for (int k = 0; k < 3; ++k) v += C[k * 3 + dn] * F[s][k]; dr[s * nq3 + q] = v; }
                    }
                }
                for (int s = 0; s < NSTATE; ++s) {
                    if (!split) {
                        surf_apply(o, phi, nq, nq, o.phi_s[fi % 2].data(), fi, &cri[s * nq3], &cfi[s * nf], false, nref[fi][dni]);
                        surf_apply(o, phi, nq, nq, o.phi_s[fe % 2].data(), fe, &cre[s * nq3], &cfe[s * nf], false, nref[fe][dne]);
                    }
                    surf_apply(o, phi, nq, nq, o.phi_s[fi % 2].data(), fi, &dri[s * nq3], &dfi[s * nf], false, nref[fi][dni]);
                    surf_apply(o, phi, nq, nq, o.phi_s[fe % 2].data(), fe, &dre[s * nq3], &dfe[s * nf], false, nref[fe][dne]);
                }
            }
            // entropy projection (:3050-3142)
            std::vector<double> pvi(NSTATE * nq3), pve(NSTATE * nq3), psi(NSTATE * nf), pse(NSTATE * nf);
            {
                std::vector<double> evi(NSTATE * nq3), eve(NSTATE * nq3), coef(nd3);
                for (int q = 0; q < nq3; ++q) {
                    double u[5], v[5];
                    for (int s = 0; s < 5; ++s) u[s] = vi[s * nq3 + q];
                    phys.entropy_vars(u, v);
                    for (int s = 0; s < 5; ++s) evi[s * nq3 + q] = v[s];
                    for (int s = 0; s < 5; ++s) u[s] = ve[s * nq3 + q];
                    phys.entropy_vars(u, v);
                    for (int s = 0; s < 5; ++s) eve[s * nq3 + q] = v[s];
                }
                for (int s = 0; s < NSTATE; ++s) {
                    apply3(o.proj.data(), nd, nq, o.proj.data(), nd, nq, o.proj.data(), nd, nq, &evi[s * nq3], coef.data(), false, 1.0);
                    apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, coef.data(), &pvi[s * nq3], false, 1.0);
                    surf_apply(o, chi, nq, nd, o.chi_s[fi % 2].data(), fi, coef.data(), &psi[s * nf], false, 1.0);
                    apply3(o.proj.data(), nd, nq, o.proj.data(), nd, nq, o.proj.data(), nd, nq, &eve[s * nq3], coef.data(), false, 1.0);
                    apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, coef.data(), &pve[s * nq3], false, 1.0);
                    surf_apply(o, chi, nq, nd, o.chi_s[fe % 2].data(), fe, coef.data(), &pse[s * nf], false, 1.0);
                }
            }
            // hybrid surface-volume two-point terms (:3144-3350)
            std::vector<double> hsi(NSTATE * nf, 0.0), hse(NSTATE * nf, 0.0), hvi(NSTATE * nq3, 0.0), hve(NSTATE * nq3, 0.0);
            if (split) {
                std::vector<double> s2i((size_t)NSTATE * nf * nq), s2e((size_t)NSTATE * nf * nq);
                for (int q = 0; q < nf; ++q) {
                    const double* Cs = &mesh.cof_face[(((size_t)ci * 6 + fi) * nf + q) * 9];
                    double vfi[5], vfe[5], ufi[5], ufe[5];
                    for (int s = 0; s < 5; ++s) { vfi[s] = psi[s * nf + q]; vfe[s] = pse[s * nf + q]; }
                    phys.cons_from_entropy(vfi, ufi); phys.cons_from_entropy(vfe, ufe);
                    for (int side = 0; side < 2; ++side) {
                        const int dn = side ? dne : dni; const int cc = side ? ce : ci;
                        const std::vector<double>& pv = side ? pve : pvi;
                        const double* uf = side ? ufe : ufi;
                        std::vector<double>& s2 = side ? s2e : s2i;
                        for (int l = 0; l < nq; ++l) {
                            const int jv = line_node(dn, q, l, nq);
                            const double* Cv = &mesh.cof[((size_t)cc * nq3 + jv) * 9];
                            double ev5[5], uv[5];
                            for (int s = 0; s < 5; ++s) ev5[s] = pv[s * nq3 + jv];
                            phys.cons_from_entropy(ev5, uv);
                            double F[5][3]; phys.two_point(uv, uf, F);
                            for (int s = 0; s < 5; ++s) {
                                double v = 0.0;
                                for (int k = 0; k < 3; ++k) v += 0.5 * (Cs[k * 3 + dn] + Cv[k * 3 + dn]) * F[s][k];
                                s2[((size_t)s * nf + q) * nq + l] = v;
                            }
                        }
                    }
                }
                for (int side = 0; side < 2; ++side) {
                    const int ff = side ? fe : fi; const int dn = ff / 2;
                    const std::vector<double>& s2 = side ? s2e : s2i;
                    std::vector<double>& hs = side ? hse : hsi; std::vector<double>& hv = side ? hve : hvi;
                    const double nn = nref[ff][dn];
                    for (int s = 0; s < NSTATE; ++s)
                        for (int q = 0; q < nf; ++q)
                            for (int l = 0; l < nq; ++l) {
                                const double Hop = o.phi_s[ff % 2][l] * o.wq[q % nq] * o.wq[q / nq];
                                const double Hv = Hop * s2[((size_t)s * nf + q) * nq + l];
                                hs[s * nf + q] -= Hv * nn;
                                hv[s * nq3 + line_node(dn, q, l, nq)] += Hv * nn;
                            }
                }
            }
            // numerical fluxes at face nodes (:3354-3452)
            std::vector<double> cn_(NSTATE * nf), dn_(NSTATE * nf);
            const double pen = 0.5 * (penalty_of(ci, fi) + penalty_of(ce, fe));
            for (int q = 0; q < nf; ++q) {
                const double* Cs = &mesh.cof_face[(((size_t)ci * 6 + fi) * nf + q) * 9];
                double ui[5], ue[5], ri[5], re[5], gi[5][3], ge[5][3];
                for (int s = 0; s < 5; ++s) {
                    ri[s] = si[s * nf + q]; re[s] = se[s * nf + q];
                    for (int d = 0; d < 3; ++d) { gi[s][d] = asi[(s * 3 + d) * nf + q]; ge[s][d] = ase[(s * 3 + d) * nf + q]; }
                }
                {
                    double vfi[5], vfe[5];
                    for (int s = 0; s < 5; ++s) { vfi[s] = psi[s * nf + q]; vfe[s] = pse[s * nf + q]; }
                    phys.cons_from_entropy(vfi, ui); phys.cons_from_entropy(vfe, ue);
                }
                if (!split) for (int s = 0; s < 5; ++s) { ui[s] = ri[s]; ue[s] = re[s]; }
                double np[3];
                for (int a = 0; a < 3; ++a) { np[a] = 0.0; for (int b = 0; b < 3; ++b) np[a] += Cs[a * 3 + b] * nref[fi][b]; }
                double J = 0.0; for (int a = 0; a < 3; ++a) J += np[a] * np[a];
                J = std::sqrt(J);
                for (int a = 0; a < 3; ++a) np[a] /= J;
                double cf[5], df[5] = {0, 0, 0, 0, 0};
                if (bt) {
                    // the interior state interpolated to the face, or with
                    // use_projected_entropy_variables_for_nsfr_boundary_term (split form) the state of the
                    // projected entropy variables (strong_dg.cpp:2255-2273); the dissipative flux's
                    // interior side stays the interpolated state (:2291-2298); the penalty is this
                    // cell's (dg_base.cpp:563)
                    const double* us = (split && prm.bc_projected) ? ui : ri;
                    double ub[5];
                    phys.boundary_state(bt, np, us, ub);
                    phys.conv_num_flux(us, ub, np, cf);
                    if (viscous) {
                        double uv[5], gv[5][3];
                        phys.boundary_viscous_state(bt, us, gi, uv, gv);
                        phys.diss_boundary_flux(bt, ri, uv, gi, gv, np, penalty_of(c, f), df);
                    }
                } else {
                    phys.conv_num_flux(ui, ue, np, cf);
                    if (viscous) phys.diss_num_flux(ri, re, gi, ge, np, pen, df);
                }
                for (int s = 0; s < 5; ++s) { cn_[s * nf + q] = J * cf[s]; dn_[s * nf + q] = J * df[s]; }
            }
            // lift this cell's side (:3454-3576)
            std::vector<double> r(nd3);
            const bool me_int = owner;
            const int fme = me_int ? fi : fe;
            for (int s = 0; s < NSTATE; ++s) {
                const double* crow = o.chi_s[fme % 2].data();
                if (split) {
                    surf_inner(chi, nq, nd, crow, fme, me_int ? &hsi[s * nf] : &hse[s * nf], ones_face.data(), r.data(), false, -1.0);
                    inner3(chi, nq, nd, chi, nq, nd, chi, nq, nd, me_int ? &hvi[s * nq3] : &hve[s * nq3], ones_vol.data(), r.data(), true, -1.0);
                } else {
                    surf_inner(chi, nq, nd, crow, fme, me_int ? &cfi[s * nf] : &cfe[s * nf], Wface.data(), r.data(), false, 1.0);
                }
                surf_inner(chi, nq, nd, crow, fme, me_int ? &dfi[s * nf] : &dfe[s * nf], Wface.data(), r.data(), true, 1.0);
                surf_inner(chi, nq, nd, crow, fme, &cn_[s * nf], Wface.data(), r.data(), true, me_int ? -1.0 : 1.0);
                surf_inner(chi, nq, nd, crow, fme, &dn_[s * nf], Wface.data(), r.data(), true, me_int ? -1.0 : 1.0);
                for (int i = 0; i < nd3; ++i) Rc[s * nd3 + i] += r[i];
            }
        }
    }
}

void Solver::apply_inverse_mass(const double* in, double* out, bool aux_eq) {
    // affine: (M+K)^{-1} (x) (M+K)^{-1} (x) (M+K)^{-1} / det J  (dg_base.cpp:4207-4219)
    const int nd = ops.nd;
    const double* Mi = aux_eq ? ops.minv_aux.data() : ops.minv.data();
    const size_t ndc = (size_t)ndofs_cell;
    if (!mesh.affine) {
        // curvilinear: weight-adjusted inverse P diag(1/(w J)) P^T with the FR projection
        // P = (M+K)^{-1} chi^T W (dg_base.cpp:4217-4249, operators.cpp:1909-1932)
        const int nq = ops.nq;
        std::vector<double> P((size_t)nd * nq, 0.0);
        for (int i = 0; i < nd; ++i)
            for (int q = 0; q < nq; ++q) {
                double v = 0.0;
                for (int j = 0; j < nd; ++j) v += Mi[i * nd + j] * ops.chi[q * nd + j];
                P[i * nq + q] = v * ops.wq[q];
            }
        const std::vector<double> PT = transpose(P.data(), nd, nq);
#pragma omp parallel for schedule(static)
        for (int c = 0; c < mesh.nc; ++c) {
            std::vector<double> t(nq3), jw(nq3);
            for (int k = 0; k < nq; ++k) for (int j = 0; j < nq; ++j) for (int i = 0; i < nq; ++i) {
                const int q = (k * nq + j) * nq + i;
                jw[q] = 1.0 / (ops.wq[i] * ops.wq[j] * ops.wq[k] * mesh.detj[(size_t)c * nq3 + q]);
            }
            for (int s = 0; s < NSTATE; ++s) {
                apply3(PT.data(), nq, nd, PT.data(), nq, nd, PT.data(), nq, nd, in + c * ndc + s * nd3, t.data(), false, 1.0);
                for (int q = 0; q < nq3; ++q) t[q] *= jw[q];
                apply3(P.data(), nd, nq, P.data(), nd, nq, P.data(), nd, nq, t.data(), out + c * ndc + s * nd3, false, 1.0);
            }
        }
        return;
    }
#pragma omp parallel for schedule(static)
    for (int c = 0; c < mesh.nc; ++c) {
        const double dj = mesh.detj[(size_t)c * nq3];
        for (int s = 0; s < NSTATE; ++s)
            apply3(Mi, nd, nd, Mi, nd, nd, Mi, nd, nd, in + c * ndc + s * nd3, out + c * ndc + s * nd3, false, 1.0 / dj);
    }
}

// ---------------------------------------------------------------------------------
// Positivity-preserving limiter (PositivityPreservingLimiter, limiter/positivity_preserving_limiter.cpp),
// restated with its index behaviour: the solution is interpolated to three mixed point sets
// (GLL along direction d, GL along the other two; the sum-factorised interpolation applies its
// first operator along x, operators.cpp:355-395), and each directional "cell average" loops
// over GLL/GL weights with an unbraced innermost loop, so its point index advances once per
// (i, j) pair: the average of set d sums the first n^2 points only (the z = 0 plane), with the
// weight of the loop's i on y and of its j on x (:264-298). The averages are combined with the
// wave-speed weights of Zhang & Shu (:300-345).
// ---------------------------------------------------------------------------------
namespace {

// Smallest-modulus root of s3 + s2 t + s1 t^2, real part (Eigen::PolynomialSolver<double,2>
// smallestRoot().real(), as get_theta2_Zhang2010 takes it, :95-98)
double smallest_root_real(double s3, double s2, double s1) {
    if (s1 == 0.0) return -s3 / s2;
    const double disc = s2 * s2 - 4.0 * s1 * s3;
    if (disc < 0.0) return -s2 / (2.0 * s1);      // complex pair: equal moduli, same real part
    const double q = -0.5 * (s2 + (s2 >= 0.0 ? std::sqrt(disc) : -std::sqrt(disc)));
    const double r1 = q / s1, r2 = (q != 0.0) ? s3 / q : r1;
    return std::fabs(r1) <= std::fabs(r2) ? r1 : r2;
}

}  // namespace

void Solver::limit(double* U, double dt) {
    if (prm.limiter != PPL_ZHANG2010 && prm.limiter != PPL_WANG2012) return;
    const int n = ops.nd, n3 = n * n * n;
    std::vector<double> xgl, wgl, xgll, wgll;
    gauss_legendre(n, xgl, wgl);
    gauss_lobatto(n, xgll, wgll);
    std::vector<double> Bgl((size_t)n * n), Bgll((size_t)n * n);   // FE_DGQ basis at the GL / GLL points
    for (int q = 0; q < n; ++q) {
        lagrange_eval(ops.xs, xgl[q], &Bgl[q * n], nullptr);
        lagrange_eval(ops.xs, xgll[q], &Bgll[q * n], nullptr);
    }
    const double dx = mesh.h;   // (right - left) / cells, the same in every direction
    const double lam = dt / dx;
    const double gam = prm.gamma, gm1 = gam - 1.0;
    auto pressure = [&](const double* u) {   // compute_pressure, no non-physical replacement here
        const double rho = u[0];
        double v2 = 0.0;
        for (int d = 0; d < 3; ++d) { const double v = u[1 + d] / rho; v2 = v2 + v * v; }
        return gm1 * (u[4] - 0.5 * rho * v2);
    };
    auto max_eig = [&](const double* u) {   // max_convective_eigenvalue (euler.cpp:1034-1046)
        double v2 = 0.0;
        for (int d = 0; d < 3; ++d) { const double v = u[1 + d] / u[0]; v2 += v * v; }
        return std::sqrt(v2) + std::sqrt(pressure(u) * gam / u[0]);
    };
    const bool zhang = prm.limiter == PPL_ZHANG2010;
    const double lower = prm.min_density;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < mesh.nc; ++c) {
        double* Uc = U + (size_t)c * ndofs_cell;
        std::vector<double> coeff(Uc, Uc + ndofs_cell);
        bool nan = false;
        for (double v : coeff) nan |= std::isnan(v);
        if (nan) continue;   // the reference aborts here (:430-442)
        // the three mixed point sets: q[d][s][n3]
        std::vector<double> q[3];
        auto interp = [&](int d, int s) {
            const double* A[3] = {d == 0 ? Bgll.data() : Bgl.data(), d == 1 ? Bgll.data() : Bgl.data(),
                                  d == 2 ? Bgll.data() : Bgl.data()};
            apply3(A[0], n, n, A[1], n, n, A[2], n, n, &coeff[(size_t)s * n3], &q[d][(size_t)s * n3], false, 1.0);
        };
        for (int d = 0; d < 3; ++d) { q[d].assign((size_t)NSTATE * n3, 0.0); for (int s = 0; s < NSTATE; ++s) interp(d, s); }
        double min_rho = 1e6;
        for (int d = 0; d < 3; ++d)
            for (int i = 0; i < n3; ++i) {
                if (coeff[i] < min_rho) min_rho = coeff[i];
                if (q[d][i] < min_rho) min_rho = q[d][i];
            }
        // directional averages with the reference's point indexing (see above)
        double avg_dim[3][NSTATE] = {};
        for (int s = 0; s < NSTATE; ++s) {
            int qp = 0;
            for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) {
                for (int k = 0; k < n; ++k) avg_dim[0][s] += wgll[i] * wgl[j] * wgl[k] * q[0][(size_t)s * n3 + qp];
                qp++;
            }
            qp = 0;
            for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) {
                for (int k = 0; k < n; ++k) avg_dim[1][s] += wgl[i] * wgll[j] * wgl[k] * q[1][(size_t)s * n3 + qp];
                qp++;
            }
            qp = 0;
            for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) {
                for (int k = 0; k < n; ++k) avg_dim[2][s] += wgl[i] * wgl[j] * wgll[k] * q[2][(size_t)s * n3 + qp];
                qp++;
            }
        }
        double ws[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < n3; ++i)
            for (int d = 0; d < 3; ++d) {
                double u[NSTATE];
                for (int s = 0; s < NSTATE; ++s) u[s] = q[d][(size_t)s * n3 + i];
                const double w = max_eig(u);
                if (w > ws[d]) ws[d] = w;
            }
        const double mu = ws[0] * lam + ws[1] * lam + ws[2] * lam;
        const double aw[3] = {(ws[0] * lam) / mu, (ws[1] * lam) / mu, (ws[2] * lam) / mu};
        double avg[NSTATE];
        for (int s = 0; s < NSTATE; ++s) {
            avg[s] = aw[0] * avg_dim[0][s] + aw[1] * avg_dim[1][s];
            avg[s] += aw[2] * avg_dim[2][s];
        }
        const double p_avg = pressure(avg);
        // get_density_scaling_value (:170-186)
        double eps = std::min({lower, avg[0], p_avg});
        if (eps < 0) eps = lower;
        double theta = 1.0;
        if (avg[0] - min_rho > 1e-13)
            theta = (avg[0] - min_rho == 0) ? 1.0 : std::min((avg[0] - eps) / (avg[0] - min_rho), 1.0);
        if (theta < 0 || theta > 1) theta = 0;
        for (int i = 0; i < n3; ++i) coeff[i] = theta * (coeff[i] - avg[0]) + avg[0];
        for (int d = 0; d < 3; ++d) interp(d, 0);
        if (!zhang) {   // Wang 2012 (:597-618)
            auto theta2_of = [&](const double* base) {
                double th = 1.0;
                for (int i = 0; i < n3; ++i) {
                    double u[NSTATE];
                    for (int s = 0; s < NSTATE; ++s) u[s] = base[(size_t)s * n3 + i];
                    const double pl = pressure(u);
                    const double t2 = (pl >= 0) ? 1.0 : p_avg / (p_avg - pl);
                    if (t2 != 1 && t2 >= 0 && t2 <= 1 && t2 < th) th = t2;
                }
                return th;
            };
            double theta2 = 1.0;
            for (int d = 0; d < 3; ++d) theta2 = std::min(theta2, theta2_of(q[d].data()));
            const double t_soln = theta2_of(coeff.data());
            if (t_soln < theta2) theta2 = t_soln;
            for (int s = 0; s < NSTATE; ++s)
                for (int i = 0; i < n3; ++i) coeff[(size_t)s * n3 + i] = theta2 * (coeff[(size_t)s * n3 + i] - avg[s]) + avg[s];
        } else {   // Zhang 2010 (:620-668); gamma 1.4 as the reference passes it
            auto theta2_of = [&](const double* base, double* out) {
                const double e = lower / 1.4;
                for (int i = 0; i < n3; ++i) {
                    double u[NSTATE];
                    for (int s = 0; s < NSTATE; ++s) u[s] = base[(size_t)s * n3 + i];
                    if (pressure(u) >= lower) { out[i] = 1.0; continue; }
                    double s1 = (u[4] - avg[4]) * (u[0] - avg[0]) - 0.5 * std::pow(u[1] - avg[1], 2);
                    double s2 = avg[0] * (u[4] - avg[4]) + avg[4] * (u[0] - avg[0]) - avg[1] * (u[1] - avg[1]) -
                                e * (u[0] - avg[0]);
                    double s3 = (avg[4] * avg[0]) - 0.5 * std::pow(avg[1], 2) - e * avg[0];
                    s1 -= 0.5 * std::pow(u[2] - avg[2], 2);
                    s2 -= avg[2] * (u[2] - avg[2]);
                    s3 -= 0.5 * std::pow(avg[2], 2);
                    s1 -= 0.5 * std::pow(u[3] - avg[3], 2);
                    s2 -= avg[3] * (u[3] - avg[3]);
                    s3 -= 0.5 * std::pow(avg[3], 2);
                    out[i] = smallest_root_real(s3, s2, s1);
                }
            };
            std::vector<double> tq((size_t)3 * n3), tsol(n3);
            for (int d = 0; d < 3; ++d) theta2_of(q[d].data(), &tq[(size_t)d * n3]);
            theta2_of(coeff.data(), tsol.data());
            for (int s = 0; s < NSTATE; ++s)
                for (int i = 0; i < n3; ++i) {
                    double mq = 1e6;
                    for (int d = 0; d < 3; ++d) if (tq[(size_t)d * n3 + i] < mq) mq = tq[(size_t)d * n3 + i];
                    const double th = std::min(mq, tsol[i]);
                    coeff[(size_t)s * n3 + i] = th * (coeff[(size_t)s * n3 + i] - avg[s]) + avg[s];
                }
        }
        std::copy(coeff.begin(), coeff.end(), Uc);
    }
}

// ---------------------------------------------------------------------------------
// Low-storage 3S* / 3S*+ step (LowStorageRungeKuttaODESolver,
// low_storage_runge_kutta_ode_solver.cpp:20-110; tableaux low_storage_runge_kutta_methods.cpp,
// the published RK4(3)5[3S*] of Ketcheson 2010 and the [3S*+] family of Ranocha et al. 2021).
// ---------------------------------------------------------------------------------
namespace {
struct LsTableau {
    int ns, num_delta, order;
    bool plus;
    std::vector<std::array<double, 3>> gamma;
    std::vector<double> beta, delta, bhat;
};

LsTableau ls_tableau(int m) {
    LsTableau t;
    if (m == LS_RK4_3_5) {
        t.ns = 5; t.num_delta = 7; t.order = 4; t.plus = false;
        t.gamma = {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {-0.497531095840104, 1.384996869124138, 0.0},
                   {1.010070514199942, 3.878155713328178, 0.0}, {-3.196559004608766, -2.324512951813145, 1.642598936063715},
                   {1.717835630267259, -0.514633322274467, 0.188295940828347}};
        t.beta = {0.0, 0.075152045700771, 0.211361016946069, 1.100713347634329, 0.728537814675568, 0.393172889823198};
        t.delta = {1.0, 0.081252332929194, -1.083849060586449, -1.096110881845602, 2.859440022030827,
                   -0.655568367959557, -0.194421504490852};
        t.bhat = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    } else if (m == LS_RK3_2_5F) {
        t.ns = 5; t.num_delta = 5; t.order = 3; t.plus = true;
        t.gamma = {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0},
                   {0.2587771979725733308135192812685323706, 0.5528354909301389892439698870483746541, 0.0},
                   {-0.1324380360140723382965420909764953437, 0.6731871608203061824849561782794643600, 0.0},
                   {0.05056033948190826045833606441415585735, 0.2803103963297672407841316576323901761,
                    0.2752563273304676380891217287572780582},
                   {0.5670532000739313812633197158607642990, 0.5521525447020610386070346724931300367,
                    -0.8950526174674033822276061734289327568}};
        t.beta = {0.0, 0.2300298624518076223899418286314123354, 0.3021434166948288809034402119555380003,
                  0.8025606185416310937583009085873554681, 0.4362158943603440930655148245148766471,
                  0.11292725304550591};
        t.delta = {1.0, 0.34076558793345252, 0.34143826550033862, 0.72292753667879872, 0.0};
        t.bhat = {0.094841667050357029, 0.17263713394303537, 0.39982431890843712, 0.17180168075801786,
                  0.058819144221557401, 0.1020760551185952388626787099944507877};
    } else if (m == LS_RK4_3_9F) {
        t.ns = 9; t.num_delta = 9; t.order = 4; t.plus = true;
        t.gamma = {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0},
                   {-4.655641447335068552684422206224169103, 2.499262792574495009336242992898153462, 0.0},
                   {-0.7720265099645871829248487209517314217, 0.5866820377718875577451517985847920081, 0.0},
                   {-4.024436690519806086742256154738379161, 1.205146086523094569925592464380295241,
                    0.7621006678721315291614677352949377871},
                   {-0.02129676284018530966221583708648634733, 0.3474793722186732780030762737753849272,
                    -0.1981182504339400567765766904309673119},
                   {-2.435022509790109546199372365866450709, 1.321346060965113109321230804210670518,
                    -0.6228959218699007450469629366684127462},
                   {0.01985627297131987000579523283542615256, 0.3119636464694193615946633676950358444,
                    -0.3752248380775956442989480369774937099},
                   {-0.2810791146791038566946663374735713961, 0.4351419539684379261368971206040518552,
                    -0.3355438309135169811915662336248989661},
                   {0.1689434168754859644351230590422137972, 0.2359698130028753572503744518147537768,
                    -0.04560955005031121479972862973705108039}};
        t.beta = {0.0, 0.2836343005184365275160654678626695428, 0.9736500104654741223716056170419660217,
                  0.3382359225242515288768487569778320563, -0.3584943611106183357043212309791897386,
                  -0.004113944068471528211627210454497620358, 1.427968894048586363415504654313371031,
                  0.01808470948394314017665968411915568633, 0.1605770645946802213926893453819236685,
                  0.2952227015964591648775833803635147962};
        t.delta = {1.0, 1.262923876648114432874834923838556100, 0.7574967189685911558308119415539596711,
                   0.5163589453140728104667573195005629833, -0.02746327421802609557034437892013640319,
                   -0.4382673178127944142238606608356542890, 1.273587294602656522645691372699677063,
                   -0.6294740283927400326554066998751383342, 0.0};
        t.bhat = {0.02483675912451591196775756814283216443, 0.1866327774562103796990092260942180726,
                  0.05671080795936984495604436622517631183, -0.003447695439149287702616943808570747099,
                  0.003602245056516636472203469198006404016, 0.4545570622145088936800484247980581766,
                  -0.0002434665289427612407531544765622888855, 0.06642755361103549971517945063138312147,
                  0.1613697079523505006226025497715177578, 0.04955424859358438183052504342394102722};
    } else {   // LS_RK5_4_10F
        t.ns = 10; t.num_delta = 10; t.order = 5; t.plus = true;
        t.gamma = {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0},
                   {0.4043660121685749695640462197806189975, 0.6871467028161416909922221357014564412, 0.0},
                   {-0.8503427289575839690883191973980814832, 1.093024748914750833700799552463885117, 0.0},
                   {-6.950894175262117526410215315179482885, 3.225975379607193001678365742708874597,
                    -2.393405133244194727221124311276648940},
                   {0.9238765192731084931855438934978371889, 1.041153702510101386914019859778740444,
                    -1.902854422421760920850597670305403139},
                   {-2.563178056509891340215942413817786020, 1.292821487912164945157744726076279306,
                    -2.820042207399977261483046412236557428},
                   {0.2545744879365226143946122067064118430, 0.7391462755788122847651304143259254381,
                    -1.832698465277380999601896111079977378},
                   {0.3125831707411998258746812355492206137, 0.1239129251371800313941948224441873274,
                    -0.2199094483084671192328083958346519535},
                   {-0.7007114414440507927791249989236719346, 0.1842753472370123193132193302369345580,
                    -0.4082430635847870963724591602173546218},
                   {0.4839621016023833375810172323297465039, 0.05712788998796583446479387686662738843,
                    -0.1377669797880289713535665985132703979}};
        t.beta = {0.0, 0.2597883554788674084039539165398464630, 0.01777008889438867858759149597539211023,
                  0.2481636629715501931294746189266601496, 0.7941736871152005775821844297293296135,
                  0.3885391285642019129575902994397298066, 0.1455051657916305055730603387469193768,
                  0.1587517385964749337690916959584348979, 0.1650605617880053419242434594242509601,
                  0.2118093284937153836908655490906875007, 0.1559392342362059886106995325687547506};
        t.delta = {1.0, -0.1331778419508803397033287009506932673, 0.8260422814750207498262063505871077303,
                   1.513700425755728332485300719652378197, -1.305810059935023735972298885749903694,
                   3.036678802924163246003321318996156380, -1.449458274398895177922690618003584514,
                   3.834313899176362315089976408899373409, 4.122293760012985409330881631526514714, 0.0};
        t.bhat = {-0.02019255440012066080909442770590267512, 0.02737903480959184339932730854141598275,
                  0.3028818636145965534365173822296811090, -0.03656843880622222190071445247906780540,
                  0.3982664774676767729863101188528827405, -0.05715959421140685436681459970502471634,
                  0.09849855103848558320961101178888983150, 0.06654601552456084978615342374581437947,
                  0.09073479542748112726465375642050504556, 0.08432289325330803924891866923939606351,
                  0.04529095628204896774513180907141004447};
    }
    return t;
}
} // namespace

void Solver::lsrk_step(double* U, double dt) {
    const LsTableau t = ls_tableau(prm.rk_method);
    const size_t N = ndofs();
    // prep_for_step_in_time (:207-217): S1 = S3 = S4 = u_n, S2 = 0
    std::vector<double> s1(U, U + N), s2(N, 0.0), s3(U, U + N), s4(U, U + N), rhs(N), R(N);
    for (int i = 0; i < t.ns; ++i) {
        for (size_t m = 0; m < N; ++m) s2[m] += t.delta[i] * s1[m];            // calculate_stage_solution
        assemble_residual(s1.data(), R.data());                                // calculate_stage_derivative
        apply_inverse_mass(R.data(), rhs.data());
        for (size_t m = 0; m < N; ++m) {
            double v = s1[m] * t.gamma[i + 1][0];
            v += t.gamma[i + 1][1] * s2[m];
            v += t.gamma[i + 1][2] * s3[m];
            const double r = rhs[m] * dt;
            v += t.beta[i + 1] * r;
            s1[m] = v;
            if (t.plus) s4[m] += t.bhat[i] * r;
        }
    }
    // sum_stages (:47-72)
    if (!t.plus) {
        double sum_delta = 0.0;
        for (int i = 0; i < t.num_delta; ++i) sum_delta += t.delta[i];
        for (size_t m = 0; m < N; ++m) {
            s2[m] += t.delta[t.ns] * s1[m];
            s2[m] += t.delta[t.ns + 1] * s3[m];
            s2[m] /= sum_delta;
        }
    } else {
        assemble_residual(s1.data(), R.data());
        apply_inverse_mass(R.data(), rhs.data());
        for (size_t m = 0; m < N; ++m) s4[m] += t.bhat[t.ns] * (rhs[m] * dt);
    }
    // get_automatic_error_adaptive_step_size (:80-110), before the controller
    const std::vector<double>& other = t.plus ? s4 : s2;
    double w = 0.0;
    for (size_t m = 0; m < N; ++m) {
        const double e = s1[m] - other[m];
        const double q = e / (prm.atol + prm.rtol * std::max(std::abs(s1[m]), std::abs(other[m])));
        w += q * q;
    }
    last_error = std::sqrt(w / (double)N);
    std::copy(s1.begin(), s1.end(), U);
    current_time += dt;
}

void Solver::rk_step(double* U, double dt) {
    if (prm.rk_method >= LS_RK4_3_5) { lsrk_step(U, dt); return; }
    // Butcher tableaux (runge_kutta_methods.cpp:7-47), stage loop (runge_kutta_base.cpp:21-39,
    // runge_kutta_ode_solver.cpp:15-100)
    int ns; double a[4][4] = {{0}}, b[4] = {0}, cc[4] = {0};
    if (prm.rk_method == RK4) {
        ns = 4; a[1][0] = 0.5; a[2][1] = 0.5; a[3][2] = 1.0;
        b[0] = 1.0 / 6.0; b[1] = 1.0 / 3.0; b[2] = 1.0 / 3.0; b[3] = 1.0 / 6.0;
        cc[1] = 0.5; cc[2] = 0.5; cc[3] = 1.0;
    } else if (prm.rk_method == SSPRK3) {
        ns = 3; a[1][0] = 1.0; a[2][0] = 0.25; a[2][1] = 0.25;
        b[0] = 1.0 / 6.0; b[1] = 1.0 / 6.0; b[2] = 2.0 / 3.0;
        cc[1] = 1.0; cc[2] = 0.5;
    } else if (prm.rk_method == HEUN2) {   // HeunExplicit (runge_kutta_methods.cpp:73-92)
        ns = 2; a[1][0] = 1.0; b[0] = 0.5; b[1] = 0.5; cc[1] = 1.0;
    } else { ns = 1; b[0] = 1.0; }
    const size_t N = ndofs();
    std::vector<double> un(U, U + N), R(N);
    std::vector<std::vector<double>> k(ns, std::vector<double>(N));
    double est = 0.0;   // relaxation RK: dt sum_i b_i v(u_i)^T M k_i
    for (int i = 0; i < ns; ++i) {
        std::vector<double>& st = k[i];
        std::fill(st.begin(), st.end(), 0.0);
        for (int j = 0; j < i; ++j)
            if (a[i][j] != 0.0) for (size_t m = 0; m < N; ++m) st[m] += a[i][j] * k[j][m];
        for (size_t m = 0; m < N; ++m) { st[m] *= dt; st[m] += 1.0 * un[m]; }
        limit(st.data(), dt);   // RungeKuttaBase::apply_limiter at every stage (runge_kutta_base.cpp:26)
        assemble_residual(st.data(), R.data());
        if (prm.use_rrk) est += b[i] * entropy_vars_dot_mass(st.data(), R.data());
        apply_inverse_mass(R.data(), st.data());
    }
    double step = dt;
    if (prm.use_rrk) step = dt * relaxation_parameter(un.data(), k, b, ns, dt, dt * est);
    for (int i = 0; i < ns; ++i)
        for (size_t m = 0; m < N; ++m) un[m] += step * b[i] * k[i][m];
    std::copy(un.begin(), un.end(), U);
    limit(U, dt);   // and on the new solution (runge_kutta_base.cpp:34)
    current_time += step;
    (void)cc;
}

// ---- relaxation Runge-Kutta, root-finding form for the Euler / Navier-Stokes entropy
// (RootFindingRRKODESolver, root_finding_rrk_ode_solver.cpp:15-180, :182-390;
// RKNumEntropy::compute_entropy_vars, runge_kutta_store_entropy.cpp:27-100). Collocated GLL flux
// nodes: the volume quadrature is the solution nodes, so the entropy variables' projection onto
// the solution basis is the identity and the mass matrix of the M norm is diag(W det J); other
// flux nodes interpolate to them and project back.

// Euler::compute_entropy (euler.cpp:512-530) and compute_numerical_entropy_function (:437-447)
static double numerical_entropy_fn(const double u[5], double gam) {
    const double p = (gam - 1.0) * (u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]);
    const double s = std::log(p * std::pow(u[0], -gam));
    return -u[0] * s;
}

// Euler::compute_entropy_variables (euler.cpp:811-829)
static void entropy_variables(const double u[5], double gam, double v[5]) {
    const double p = (gam - 1.0) * (u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]);
    const double s = std::log(p * std::pow(u[0], -gam));
    const double rt = p / (gam - 1.0);
    v[0] = (rt * (gam + 1.0 - s) - u[4]) / rt;
    for (int d = 0; d < 3; ++d) v[1 + d] = u[1 + d] / rt;
    v[4] = -u[0] / rt;
}

// W det J of every solution node of cell c (GLL collocation)
static double node_mass(const Mesh& mesh, const Ops1D& ops, int c, int node) {
    const int nd = ops.nd;
    const double W = ops.wq[node % nd] * ops.wq[(node / nd) % nd] * ops.wq[node / (nd * nd)];
    const double J = mesh.affine ? mesh.h * mesh.h * mesh.h : mesh.detj[(size_t)c * nd * nd * nd + node];
    return W * J;
}

// W det J at flux node q of cell c (uncollocated flux nodes)
static double flux_node_mass(const Mesh& mesh, const Ops1D& ops, int c, int q) {
    const int nq = ops.nq;
    const double W = ops.wq[q % nq] * ops.wq[(q / nq) % nq] * ops.wq[q / (nq * nq)];
    const double J = mesh.affine ? mesh.h * mesh.h * mesh.h : mesh.detj[(size_t)c * nq * nq * nq + q];
    return W * J;
}

static bool collocated(const Params& p) { return p.flux_nodes == GLL && p.overintegration == 0; }

double Solver::numerical_entropy(const double* U) const {
    double sum = 0.0;
    if (!collocated(prm)) {   // the volume quadrature: the state interpolated to the flux nodes
        // (compute_integrated_numerical_entropy, root_finding_rrk_ode_solver.cpp:211-350)
        const int nd = ops.nd, nq = ops.nq;
        const double* chi = ops.chi.data();
        std::vector<double> uq((size_t)NSTATE * nq3);
        for (int c = 0; c < mesh.nc; ++c) {
            for (int s = 0; s < NSTATE; ++s)
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, U + (size_t)c * ndofs_cell + s * nd3, &uq[s * nq3],
                       false, 1.0);
            for (int q = 0; q < nq3; ++q) {
                double u[5];
                for (int s = 0; s < 5; ++s) u[s] = uq[s * nq3 + q];
                sum += flux_node_mass(mesh, ops, c, q) * numerical_entropy_fn(u, prm.gamma);
            }
        }
        return sum;
    }
    for (int c = 0; c < mesh.nc; ++c)
        for (int i = 0; i < nd3; ++i) {
            double u[5];
            for (int s = 0; s < 5; ++s) u[s] = U[(size_t)c * ndofs_cell + s * nd3 + i];
            sum += node_mass(mesh, ops, c, i) * numerical_entropy_fn(u, prm.gamma);
        }
    return sum;
}

// v(u)^T M k with M k = R for the residual R of this stage: M (M+K)^{-1} R is R for cDG; the
// reference's M-norm form applies M to k, which for FR differs from R, so it is M k here.
double Solver::entropy_vars_dot_mass(const double* st, const double* R) {
    std::vector<double> kk((size_t)ndofs());
    apply_inverse_mass(R, kk.data());
    double sum = 0.0;
    if (!collocated(prm)) {
        // uncollocated flux nodes: v_hat = M^-1 chi^T W v(chi u), the entropy variables projected on
        // the solution basis (compute_entropy_vars, runge_kutta_store_entropy.cpp:30-100), dotted with
        // M k, M = chi^T W J chi (compute_entropy_change_estimate, root_finding_rrk_ode_solver.cpp:353-388):
        // sum over the flux nodes of W J (chi v_hat)(chi k)
        const int nd = ops.nd, nq = ops.nq;
        const double* chi = ops.chi.data();
        const double* proj = ops.proj.data();
        std::vector<double> uq((size_t)NSTATE * nq3), vh(nd3), vq((size_t)NSTATE * nq3), kq(nq3);
        for (int c = 0; c < mesh.nc; ++c) {
            for (int s = 0; s < NSTATE; ++s)
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, st + (size_t)c * ndofs_cell + s * nd3, &uq[s * nq3],
                       false, 1.0);
            for (int q = 0; q < nq3; ++q) {
                double u[5], v[5];
                for (int s = 0; s < 5; ++s) u[s] = uq[s * nq3 + q];
                entropy_variables(u, prm.gamma, v);
                for (int s = 0; s < 5; ++s) vq[s * nq3 + q] = v[s];
            }
            for (int s = 0; s < NSTATE; ++s) {
                apply3(proj, nd, nq, proj, nd, nq, proj, nd, nq, &vq[s * nq3], vh.data(), false, 1.0);
                std::vector<double> vhq(nq3);
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, vh.data(), vhq.data(), false, 1.0);
                apply3(chi, nq, nd, chi, nq, nd, chi, nq, nd, kk.data() + (size_t)c * ndofs_cell + s * nd3, kq.data(),
                       false, 1.0);
                for (int q = 0; q < nq3; ++q) sum += flux_node_mass(mesh, ops, c, q) * vhq[q] * kq[q];
            }
        }
        return sum;
    }
    for (int c = 0; c < mesh.nc; ++c)
        for (int i = 0; i < nd3; ++i) {
            double u[5], v[5];
            for (int s = 0; s < 5; ++s) u[s] = st[(size_t)c * ndofs_cell + s * nd3 + i];
            entropy_variables(u, prm.gamma, v);
            const double m = node_mass(mesh, ops, c, i);
            for (int s = 0; s < 5; ++s) sum += v[s] * m * kk[(size_t)c * ndofs_cell + s * nd3 + i];
        }
    return sum;
}

double Solver::relaxation_parameter(const double* un, const std::vector<std::vector<double>>& k, const double* b,
                                    int ns, double dt, double est) {
    const size_t N = ndofs();
    std::vector<double> d(N, 0.0), tmp(N);
    for (int i = 0; i < ns; ++i)
        for (size_t m = 0; m < N; ++m) d[m] += b[i] * k[i][m];
    for (size_t m = 0; m < N; ++m) d[m] *= dt;
    const double eta_n = numerical_entropy(un);
    auto root = [&](double g) {
        for (size_t m = 0; m < N; ++m) tmp[m] = un[m] + g * d[m];
        return numerical_entropy(tmp.data()) - eta_n - g * est;
    };
    // secant from the previous parameter, with the reference's safeguards; bisection if it fails
    const int iter_limit = 100;
    int iter = 0;
    double g_kp1 = 0.0;
    bool secant_failed = false;
    {
        double residual = 1.0;
        double g_k = rrk_gamma + 1e-5, g_km1 = rrk_gamma - 1e-5;
        double r_k = root(g_k), r_km1 = root(g_km1);
        while (residual > prm.rrk_tol && iter < iter_limit) {
            if (r_km1 == r_k) { g_k *= 1.001; r_km1 = root(g_km1); r_k = root(g_k); }
            if (g_k < 0.5 || g_k > 1.5) { g_k = 1.0; r_k = root(g_k); }
            g_kp1 = g_k - r_k * (g_k - g_km1) / (r_k - r_km1);
            residual = std::fabs(g_kp1 - g_k);
            ++iter;
            g_km1 = g_k; g_k = g_kp1; r_km1 = r_k; r_k = root(g_k);
            if (std::isnan(g_k) || std::isnan(g_km1)) {
                g_k = 1.0 - 1e-5; r_k = root(g_k); g_km1 = 1.0 + 1e-5; r_km1 = root(g_km1); residual = 1.0;
            }
        }
        if (iter == iter_limit) secant_failed = true;
    }
    if (secant_failed) {
        iter = 0;
        double lo = rrk_gamma - 0.1, hi = rrk_gamma + 0.1;
        double r_lo = root(lo), r_hi = root(hi), residual = 1.0;
        while (residual > prm.rrk_tol && iter < iter_limit) {
            if (r_lo * r_hi > 0) { lo -= 0.1; hi += 0.1; }
            g_kp1 = 0.5 * (lo + hi);
            const double r = root(g_kp1);
            if (r < 0) { lo = g_kp1; r_lo = r; } else { hi = g_kp1; r_hi = r; }
            residual = hi - lo;
            ++iter;
        }
        if (iter == iter_limit) throw std::runtime_error("relaxation RK: root finding failed");
    }
    if (g_kp1 < 0.5) throw std::runtime_error("relaxation RK: no reasonable relaxation factor");
    rrk_gamma = g_kp1;
    return g_kp1;
}

void Solver::interpolate_ic(double* U, int ic, const double* icp) {
    Physics phys(&prm, &status);
    for (int c = 0; c < mesh.nc; ++c)
        for (int i = 0; i < nd3; ++i) {
            const double* X = &mesh.xnode[((size_t)c * nd3 + i) * 3];
            double w[5], u[5];
            if (ic == IC_TGV) {   // initial_condition_function.cpp:261-310
                const double x = X[0], y = X[1], z = X[2];
                w[0] = 1.0;
                w[1] = std::sin(x) * std::cos(y) * std::cos(z);
                w[2] = -std::cos(x) * std::sin(y) * std::cos(z);
                w[3] = 0.0;
                w[4] = 1.0 / (prm.gamma * prm.mach_inf * prm.mach_inf) + (1.0 / 16.0) * (std::cos(2.0 * x) + std::cos(2.0 * y)) * (std::cos(2.0 * z) + 2.0);
                phys.conservative_from_primitive(w, u);
            } else {
                // isentropic vortex (initial_condition_function.cpp:643-690); IC_VORTEX_PARAM takes
                // icp = {beta, mach, dir_x, dir_y, dir_z, x0, y0, t, L} and translates with the flow.
                const double gam = prm.gamma;
                double Minf, beta, dir[3], x0 = 0.0, y0 = 0.0, t = 0.0, L = 0.0;
                if (ic == IC_ISENTROPIC_VORTEX) {
                    Minf = std::sqrt(2.0 / gam);
                    beta = Minf * 5 * std::sqrt(2.0) / 4.0 / PI * std::exp(1.0 / 2.0);
                    dir[0] = std::cos(PI / 4); dir[1] = std::sin(PI / 4); dir[2] = 0.0;
                } else {
                    beta = icp[0]; Minf = icp[1]; dir[0] = icp[2]; dir[1] = icp[3]; dir[2] = icp[4];
                    x0 = icp[5]; y0 = icp[6]; t = icp[7]; L = icp[8];
                }
                double x = X[0] - x0 - Minf * dir[0] * t, y = X[1] - y0 - Minf * dir[1] * t;
                if (L > 0.0) { x -= L * std::round(x / L); y -= L * std::round(y / L); }
                const double Om = beta * std::exp(-0.5 * (x * x + y * y));
                const double dT = -(gam - 1.0) / 2.0 * Om * Om;
                w[0] = std::pow(1 + dT, 1.0 / (gam - 1.0));
                w[1] = Minf * dir[0] - y * Om;
                w[2] = Minf * dir[1] + x * Om;
                w[3] = Minf * dir[2];
                w[4] = 1.0 / gam * std::pow(1 + dT, gam / (gam - 1.0));
                phys.conservative_from_primitive(w, u);
            }
            for (int s = 0; s < 5; ++s) U[(size_t)c * ndofs_cell + s * nd3 + i] = u[s];
        }
}

void Solver::integrated_quantities(const double* U, double* out) {
    // PeriodicTurbulence::compute_and_update_integrated_quantities (periodic_turbulence.cpp:439-672)
    // with QGauss(p+11) over-integration. The integrands follow the NavierStokes physics of
    // navier_stokes.cpp:399-740 and euler.cpp:378-402; the palinstrophy takes the gradient of the
    // vorticity after its L2 projection onto the solution basis on the reference cell
    // (vol_projection_operator, operators.cpp:1865-1889).
    Physics phys(&prm, &status);
    const int nd = ops.nd;
    const int ne = prm.poly_degree + 1 + 10;
    std::vector<double> xe, we; gauss_legendre(ne, xe, we);
    std::vector<double> B((size_t)ne * nd), dB((size_t)ne * nd);
    for (int q = 0; q < ne; ++q) lagrange_eval(ops.xs, xe[q], &B[q * nd], &dB[q * nd]);
    // 1-D projection P = M^-1 (W B)^T with the mass matrix of the same quadrature
    std::vector<double> M((size_t)nd * nd, 0.0), P((size_t)nd * ne);
    for (int i = 0; i < nd; ++i) for (int j = 0; j < nd; ++j)
        for (int q = 0; q < ne; ++q) M[i * nd + j] += we[q] * B[q * nd + i] * B[q * nd + j];
    const std::vector<double> Minv = invert(M, nd);
    for (int i = 0; i < nd; ++i) for (int q = 0; q < ne; ++q) {
        double v = 0.0;
        for (int j = 0; j < nd; ++j) v += Minv[i * nd + j] * we[q] * B[q * nd + j];
        P[i * ne + q] = v;
    }
    const int ne3 = ne * ne * ne;
    // curvilinear: the mapping (degree grid_degree on its GLL support points) at the Gauss points
    const int ng = mesh.grid_degree + 1, ng3 = ng * ng * ng;
    std::vector<double> xg, wg, Bm, dBm;
    if (!mesh.affine) {
        gauss_lobatto(ng, xg, wg);
        Bm.resize((size_t)ne * ng); dBm.resize((size_t)ne * ng);
        for (int q = 0; q < ne; ++q) lagrange_eval(xg, xe[q], &Bm[q * ng], &dBm[q * ng]);
    }
    const double gam = prm.gamma, mach2 = prm.mach_inf * prm.mach_inf;
    const double temp_ratio = 110.4 / prm.temperature_inf;   // navier_stokes.cpp:50-52
    double acc[NUM_INTEGRATED] = {0.0};
    double wave = 0.0;
    const int nq = NUM_INTEGRATED;
#pragma omp parallel for reduction(+ : acc[:nq]) reduction(max : wave)
    for (int c = 0; c < mesh.nc; ++c) {
        const double h = mesh.h, dj = h * h * h;
        const auto t = mesh.ijk[c];
        std::vector<double> jac, dje, xq;   // curvilinear: J^{-1} [ne3][3][3], det J, positions [3][ne3]
        if (!mesh.affine) {
            std::vector<double> X(ng3), Jm((size_t)9 * ne3);
            xq.resize((size_t)3 * ne3);
            for (int mm = 0; mm < 3; ++mm) {
                for (int k = 0; k < ng; ++k) for (int j = 0; j < ng; ++j) for (int i = 0; i < ng; ++i) {
                    double p[3] = {mesh.left + h * (t[0] + xg[i]), mesh.left + h * (t[1] + xg[j]), mesh.left + h * (t[2] + xg[k])};
                    warp_point(mesh.left, mesh.right, mesh.warp, p);
                    X[(k * ng + j) * ng + i] = p[mm];
                }
                apply3(Bm.data(), ne, ng, Bm.data(), ne, ng, Bm.data(), ne, ng, X.data(), &xq[(size_t)mm * ne3], false, 1.0);
                for (int j = 0; j < 3; ++j) {
                    const double* Bd[3] = {Bm.data(), Bm.data(), Bm.data()};
                    Bd[j] = dBm.data();
                    apply3(Bd[0], ne, ng, Bd[1], ne, ng, Bd[2], ne, ng, X.data(), &Jm[(size_t)(mm * 3 + j) * ne3], false, 1.0);
                }
            }
            jac.resize((size_t)9 * ne3); dje.resize(ne3);
            for (int q = 0; q < ne3; ++q) {
                double J[3][3];
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) J[a][b] = Jm[(size_t)(a * 3 + b) * ne3 + q];
                const double d = det3(J);
                dje[q] = d;
                // inverse by the cofactor (adjugate) formula
                double* I = &jac[(size_t)q * 9];
                I[0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / d;
                I[1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / d;
                I[2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / d;
                I[3] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / d;
                I[4] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / d;
                I[5] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / d;
                I[6] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / d;
                I[7] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / d;
                I[8] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / d;
            }
        }
        // physical gradient of a field from its reference gradient at cubature point q
        auto physical = [&](const double* gref, int q, double* g) {
            if (mesh.affine) {
                for (int d = 0; d < 3; ++d) g[d] = (h * h) * gref[d] / dj;
            } else {   // d/dx_d = sum_j (J^{-1})[j][d] d/dxi_j
                const double* I = &jac[(size_t)q * 9];
                for (int d = 0; d < 3; ++d) {
                    double v = 0.0;
                    for (int j = 0; j < 3; ++j) v += I[j * 3 + d] * gref[j];
                    g[d] = v;
                }
            }
        };
        auto gradient_at_points = [&](const double* coef, double* val, double* grad) {
            apply3(B.data(), ne, nd, B.data(), ne, nd, B.data(), ne, nd, coef, val, false, 1.0);
            apply3(dB.data(), ne, nd, B.data(), ne, nd, B.data(), ne, nd, coef, &grad[0], false, 1.0);
            apply3(B.data(), ne, nd, dB.data(), ne, nd, B.data(), ne, nd, coef, &grad[ne3], false, 1.0);
            apply3(B.data(), ne, nd, B.data(), ne, nd, dB.data(), ne, nd, coef, &grad[2 * (size_t)ne3], false, 1.0);
        };
        std::vector<double> uq(5 * ne3), gq(15 * ne3), omq(3 * ne3);
        for (int s = 0; s < 5; ++s)
            gradient_at_points(U + (size_t)c * ndofs_cell + s * nd3, &uq[s * ne3], &gq[(size_t)s * 3 * ne3]);
        double loc[NUM_INTEGRATED] = {0.0};
        for (int q = 0; q < ne3; ++q) {
            double u[5], g[5][3], w[5];
            for (int s = 0; s < 5; ++s) {
                u[s] = uq[s * ne3 + q];
                const double gref[3] = {gq[(s * 3 + 0) * ne3 + q], gq[(s * 3 + 1) * ne3 + q], gq[(s * 3 + 2) * ne3 + q]};
                physical(gref, q, g[s]);
            }
            phys.primitive(u, w);
            double v2 = 0.0; for (int d = 0; d < 3; ++d) v2 += w[1 + d] * w[1 + d];
            double gv[3][3];
            for (int a = 0; a < 3; ++a) for (int d = 0; d < 3; ++d) gv[a][d] = (g[1 + a][d] - w[1 + a] * g[0][d]) / w[0];
            const double om[3] = {gv[2][1] - gv[1][2], gv[0][2] - gv[2][0], gv[1][0] - gv[0][1]};
            const double om2 = om[0] * om[0] + om[1] * om[1] + om[2] * om[2];
            for (int d = 0; d < 3; ++d) omq[d * ne3 + q] = om[d];
            double S[3][3], dil = 0.0;
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) S[a][b] = 0.5 * (gv[a][b] + gv[b][a]);
            for (int d = 0; d < 3; ++d) dil += gv[d][d];
            double s2 = 0.0, sd2 = 0.0;
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) {
                const double dv = S[a][b] - (a == b ? dil / 3.0 : 0.0);
                s2 += S[a][b] * S[a][b];
                sd2 += dv * dv;
            }
            const double T = gam * mach2 * (w[4] / w[0]);
            const double mu = prm.use_constant_viscosity ? 1.0 * prm.constant_viscosity
                                                         : ((1.0 + temp_ratio) / (T + temp_ratio)) * std::pow(T, 1.5);
            double r2 = 0.0;
            for (int d = 0; d < 3; ++d) {
                const double x = mesh.affine ? mesh.left + h * (t[d] + xe[d == 0 ? q % ne : d == 1 ? (q / ne) % ne : q / (ne * ne)])
                                             : xq[(size_t)d * ne3 + q];
                r2 += x * x;
            }
            const double val[NUM_INTEGRATED] = {
                0.5 * w[0] * v2,                 // kinetic energy
                0.5 * w[0] * om2,                // enstrophy
                w[4] * dil,                      // pressure dilatation
                mu * sd2,                        // viscosity x |deviatoric strain rate|^2
                mu * s2,                         // viscosity x |strain rate|^2
                0.5 * v2,                        // incompressible kinetic energy
                0.5 * om2,                       // incompressible enstrophy
                0.0,                             // incompressible palinstrophy (below)
                0.5 * r2 * std::sqrt(om2)};      // angular momentum
            const double wt = we[q % ne] * we[(q / ne) % ne] * we[q / (ne * ne)] * (mesh.affine ? dj : dje[q]);
            for (int i = 0; i < NUM_INTEGRATED; ++i) loc[i] += val[i] * wt;
            const double mw = phys.max_eig(u);
            if (mw > wave) wave = mw;
        }
        // palinstrophy: project the vorticity onto the solution basis, then take its gradient
        std::vector<double> coef(nd3), oval(ne3), ograd(3 * (size_t)ne3);
        for (int d = 0; d < 3; ++d) {
            apply3(P.data(), nd, ne, P.data(), nd, ne, P.data(), nd, ne, &omq[(size_t)d * ne3], coef.data(), false, 1.0);
            gradient_at_points(coef.data(), oval.data(), ograd.data());
            for (int q = 0; q < ne3; ++q) {
                const double gref[3] = {ograd[q], ograd[ne3 + q], ograd[2 * (size_t)ne3 + q]};
                double g[3];
                physical(gref, q, g);
                const double wt = we[q % ne] * we[(q / ne) % ne] * we[q / (ne * ne)] * (mesh.affine ? dj : dje[q]);
                loc[7] += 0.5 * (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) * wt;
            }
        }
        for (int i = 0; i < NUM_INTEGRATED; ++i) acc[i] += loc[i];
    }
    const double vol = std::pow(mesh.right - mesh.left, 3);
    for (int i = 0; i < NUM_INTEGRATED; ++i) out[i] = acc[i] / vol;
    out[NUM_INTEGRATED] = wave;
}

void Solver::integrals(const double* U, double* out) {
    double q[NUM_INTEGRATED + 1];
    integrated_quantities(U, q);
    out[0] = q[0];
    out[1] = q[1];
    // zero for inviscid flow (periodic_turbulence.cpp:717-725)
    out[2] = (prm.pde == NAVIER_STOKES) ? 2.0 * out[1] / prm.reynolds_inf : 0.0;
    out[3] = q[NUM_INTEGRATED];
}

} // namespace oracle
