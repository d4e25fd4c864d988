// C-ABI of the B200 strong-form DG/FR residual and explicit RK stage: context set-up
// (host index maps, 1-D operators, device buffers) and stage orchestration.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <initializer_list>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/philip_b200.h"
#include "ph_internal.hpp"
#include "ph_launch.cuh"

namespace ph_host {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define PH_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(PH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------------------
// 1-D nodes, bases and FR operators (host, double)
// ---------------------------------------------------------------------------------------
void legendre_pd(int n, double x, double& p, double& dp) {
    double pm = 1.0, pc = x;
    if (n == 0) { p = 1.0; dp = 0.0; return; }
    for (int k = 2; k <= n; ++k) {
        const double pn = ((2 * k - 1) * x * pc - (k - 1) * pm) / k;
        pm = pc; pc = pn;
    }
    p = pc;
    dp = n * (x * pc - pm) / (x * x - 1.0);
}

// Gauss-Lobatto-Legendre nodes/weights on [0,1], ascending (deal.II QGaussLobatto<1>)
void gll(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0); w.assign(n, 0.0);
    const int m = n - 1;
    for (int i = 0; i < n; ++i) {
        double z = -std::cos(M_PI * i / m);
        if (i > 0 && i < m) {
            for (int it = 0; it < 64; ++it) {
                double p, dp; legendre_pd(m, z, p, dp);
                const double d2p = (2.0 * z * dp - m * (m + 1.0) * p) / (1.0 - z * z);
                const double dz = dp / d2p;
                z -= dz;
                if (std::fabs(dz) < 1e-17) break;
            }
        }
        double p, dp; legendre_pd(m, z, p, dp);
        x[i] = 0.5 * (z + 1.0);
        w[i] = 1.0 / (m * (m + 1.0) * p * p);
    }
    x[0] = 0.0; x[m] = 1.0;
}

// Gauss-Legendre nodes/weights on [0,1], ascending (deal.II QGauss<1>)
void gauss(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0); w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = -std::cos(M_PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 64; ++it) {
            double p, dp; legendre_pd(n, z, p, dp);
            const double dz = p / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-17) break;
        }
        double p, dp; legendre_pd(n, z, p, dp);
        x[i] = 0.5 * (z + 1.0);
        w[i] = 1.0 / ((1.0 - z * z) * dp * dp);
    }
}

// Lagrange basis on `nodes` at x: values and derivatives (product rule, exact at nodes)
void lagrange(const std::vector<double>& nodes, double x, double* v, double* dv) {
    const int n = (int)nodes.size();
    for (int j = 0; j < n; ++j) {
        double val = 1.0, der = 0.0;
        for (int m = 0; m < n; ++m) {
            if (m == j) continue;
            const double r = 1.0 / (nodes[j] - nodes[m]);
            der = der * (x - nodes[m]) * r + val * r;
            val *= (x - nodes[m]) * r;
        }
        v[j] = val; dv[j] = der;
    }
}

std::vector<double> mat_mul(const std::vector<double>& A, const std::vector<double>& B, int n) {
    std::vector<double> C(n * n, 0.0);
    for (int i = 0; i < n; ++i) for (int k = 0; k < n; ++k) for (int j = 0; j < n; ++j) C[i * n + j] += A[i * n + k] * B[k * n + j];
    return C;
}

bool mat_inv(std::vector<double> A, int n, std::vector<double>& Ai) {
    Ai.assign(n * n, 0.0);
    for (int i = 0; i < n; ++i) Ai[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r) if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        if (A[piv * n + c] == 0.0) return false;
        for (int j = 0; j < n; ++j) { std::swap(A[c * n + j], A[piv * n + j]); std::swap(Ai[c * n + j], Ai[piv * n + j]); }
        const double inv = 1.0 / A[c * n + c];
        for (int j = 0; j < n; ++j) { A[c * n + j] *= inv; Ai[c * n + j] *= inv; }
        for (int r = 0; r < n; ++r) if (r != c && A[r * n + c] != 0.0) {
            const double f = A[r * n + c];
            for (int j = 0; j < n; ++j) { A[r * n + j] -= f * A[c * n + j]; Ai[r * n + j] -= f * Ai[c * n + j]; }
        }
    }
    return true;
}

double fact(int k) { double f = 1.0; for (int i = 2; i <= k; ++i) f *= i; return f; }

// FR correction parameter for the reference element [0,1]
// (local_Flux_Reconstruction_operator::get_FR_correction_parameter, operators.cpp:1559-1661)
int fr_parameter(int type, int p, double user, double& c) {
    const double pf = fact(p), cp = fact(2 * p) / (pf * pf);
    switch (type) {
    case 0: c = 0.0; return 0;                                                                          // cDG
    case 1: c = 2.0 * p / ((p + 1.0) * ((2.0 * p + 1.0) * std::pow(pf * cp, 2))) / 2.0; return 0;     // cSD
    case 2: case 7: c = 2.0 * (p + 1) / (p * ((2.0 * p + 1.0) * std::pow(pf * cp, 2))) / 2.0; return 0; // cHU
    case 3: c = -2.0 / ((2.0 * p + 1.0) * std::pow(pf * cp, 2)) / 2.0; return 0;                        // cNegative
    case 4: c = -2.0 / ((2.0 * p + 1.0) * std::pow(pf * cp, 2)) / 2.0 / 2.0; return 0;                  // cNegative2
    case 5: {                                                                                            // cPlus
        static const double tab[6] = {0, 0, 0.186, 3.67e-3, 4.79e-5, 4.24e-7};
        if (p < 2 || p > 5) return 1;
        c = tab[p] / 2.0 / std::pow(std::pow(2.0, p), 2);
        return 0;
    }
    case 6: c = 10000.0; return 0;                                                                     // c10Thousand
    case 8: c = user / 2.0 / std::pow(std::pow(2.0, p), 2); return 0;                                  // user value
    }
    return 1;
}

// FR auxiliary correction parameter (local_Flux_Reconstruction_operator_aux::
// get_FR_aux_correction_parameter, operators.cpp:1809-1835): kDG, kSD, kHU, kNegative, kNegative2,
// kPlus, k10Thousand (indices 0..6) take the values of cDG, cSD, cHU, cNegative, cNegative2, cPlus,
// c10Thousand, which have the same indices in fr_parameter
int fr_aux_parameter(int type, int p, double& k) {
    if (type < 0 || type > 6) return 1;
    return fr_parameter(type, p, 0.0, k);
}

// deal.II active-cell order of the periodic cube: recursive children (child = x+2y+4z)
// for hyper_cube + refine_global, lexicographic for subdivided_hyper_cube
// (straight_periodic_cube.cpp:38-67).
void cell_order(int n, int order, std::vector<int>& ijk) {
    const int nc = n * n * n;
    ijk.assign(3 * nc, 0);
    const bool pow2 = n > 0 && (n & (n - 1)) == 0;
    const bool morton = (order == 2) || (order == 0 && pow2);
    int levels = 0;
    while ((1 << levels) < n) ++levels;
    for (int c = 0; c < nc; ++c) {
        int ix, iy, iz;
        if (morton) {
            ix = iy = iz = 0;
            for (int l = 0; l < levels; ++l) {
                const int ch = (c >> (3 * (levels - 1 - l))) & 7;
                ix = 2 * ix + (ch & 1); iy = 2 * iy + ((ch >> 1) & 1); iz = 2 * iz + ((ch >> 2) & 1);
            }
        } else {
            ix = c % n; iy = (c / n) % n; iz = c / (n * n);
        }
        ijk[3 * c] = ix; ijk[3 * c + 1] = iy; ijk[3 * c + 2] = iz;
    }
}

// Sine warp of the periodic cube [l, r]^3: each coordinate moves by
// a/k sin(k(x-l)) sin(k(y-l)) sin(k(z-l)), k = 2 pi / (r - l); zero on the cube's faces.
void warp_point(double l, double r, double a, double X[3]) {
    const double k = 2.0 * M_PI / (r - l);
    const double s = a / k * std::sin(k * (X[0] - l)) * std::sin(k * (X[1] - l)) * std::sin(k * (X[2] - l));
    X[0] += s; X[1] += s; X[2] += s;
}

// d/dxi_dir of a nodal field f on the N1^3 GLL nodes (x fastest): out = (D along dir) f
void nodal_derivative(const std::vector<double>& D, int N1, int dir, const double* f, double* out) {
    const int st = dir == 0 ? 1 : dir == 1 ? N1 : N1 * N1;
    const int NP = N1 * N1 * N1;
    for (int node = 0; node < NP; ++node) {
        const int pos = (node / st) % N1, base = node - pos * st;
        double v = 0.0;
        for (int l = 0; l < N1; ++l) v += D[pos * N1 + l] * f[base + l * st];
        out[node] = v;
    }
}

// Metric terms of one curvilinear cell whose mapping has the solution's degree, so the
// mapping support points, the flux nodes and the solution nodes are the same GLL points
// and every tensor-product operator is a 1-D derivative along one direction.
// Cofactor by the conservative curl form (operators.cpp:2738-2884):
//   C[l][0] = d_zeta(f_eta) - d_eta(f_zeta), C[l][1] = d_xi(f_zeta) - d_zeta(f_xi),
//   C[l][2] = d_eta(f_xi) - d_xi(f_eta),
// with f_j = z dy/dxi_j (l = 0), x dz/dxi_j (l = 1), y dx/dxi_j (l = 2); det J of the
// mapping Jacobian (operators.cpp:2629-2672). Writes metric rows 0..8 (C[k][d] at k*3+d),
// row 9 = 1 / det J, and the node coordinates; returns false on a non-positive det J.
bool curvilinear_cell(const std::vector<double>& x, const std::vector<double>& D, int N1, double h, double left,
                      double right, double warp, const int ijk[3], double* metric, double* xyz,
                      const double* support /* [3][NP] or nullptr */) {
    const int NP = N1 * N1 * N1;
    std::vector<double> X(3 * NP), G(9 * NP), P(9 * NP), t(NP);
    for (int node = 0; node < NP; ++node) {
        const int i = node % N1, j = (node / N1) % N1, k = node / (N1 * N1);
        double p[3] = {left + h * (ijk[0] + x[i]), left + h * (ijk[1] + x[j]), left + h * (ijk[2] + x[k])};
        if (support) { for (int d = 0; d < 3; ++d) p[d] = support[d * NP + node]; }
        else warp_point(left, right, warp, p);
        for (int d = 0; d < 3; ++d) { X[d * NP + node] = p[d]; xyz[node * 3 + d] = p[d]; }
    }
    for (int m = 0; m < 3; ++m)
        for (int j = 0; j < 3; ++j) nodal_derivative(D, N1, j, &X[m * NP], &G[(m * 3 + j) * NP]);
    // products at the nodes: row l uses (X_a, dX_b) = (z, y), (x, z), (y, x)
    const int pa[3] = {2, 0, 1}, pb[3] = {1, 2, 0};
    for (int l = 0; l < 3; ++l)
        for (int j = 0; j < 3; ++j)
            for (int node = 0; node < NP; ++node)
                P[(l * 3 + j) * NP + node] = X[pa[l] * NP + node] * G[(pb[l] * 3 + j) * NP + node];
    for (int l = 0; l < 3; ++l) {
        const double* f0 = &P[(l * 3 + 0) * NP];
        const double* f1 = &P[(l * 3 + 1) * NP];
        const double* f2 = &P[(l * 3 + 2) * NP];
        double* C0 = metric + (l * 3 + 0) * NP;
        double* C1 = metric + (l * 3 + 1) * NP;
        double* C2 = metric + (l * 3 + 2) * NP;
        nodal_derivative(D, N1, 1, f2, C0);
        nodal_derivative(D, N1, 2, f1, t.data());
        for (int q = 0; q < NP; ++q) C0[q] = t[q] - C0[q];
        nodal_derivative(D, N1, 0, f2, C1);
        nodal_derivative(D, N1, 2, f0, t.data());
        for (int q = 0; q < NP; ++q) C1[q] = C1[q] - t[q];
        nodal_derivative(D, N1, 0, f1, C2);
        nodal_derivative(D, N1, 1, f0, t.data());
        for (int q = 0; q < NP; ++q) C2[q] = t[q] - C2[q];
    }
    for (int q = 0; q < NP; ++q) {
        double J[3][3];
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) J[a][b] = G[(a * 3 + b) * NP + q];
        const double dj = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                          J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        if (!(dj > 1e-14)) return false;
        metric[9 * NP + q] = 1.0 / dj;
    }
    return true;
}


// Tensor-product evaluation on the host: out[z][y][x] = sum A_z[z][k] A_y[y][j] A_x[x][i] in[k][j][i]
// (x first), A_e of r_e rows and n columns; in is n^3 values.
static void host_apply3(const double* Ax, int rx, const double* Ay, int ry, const double* Az, int rz, int n,
                        const double* in, double* out) {
    std::vector<double> t1((size_t)rx * n * n), t2((size_t)rx * ry * n);
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int x = 0; x < rx; ++x) {
                double v = 0.0;
                for (int i = 0; i < n; ++i) v += Ax[x * n + i] * in[(k * n + j) * n + i];
                t1[(k * n + j) * rx + x] = v;
            }
    for (int k = 0; k < n; ++k)
        for (int y = 0; y < ry; ++y)
            for (int x = 0; x < rx; ++x) {
                double v = 0.0;
                for (int j = 0; j < n; ++j) v += Ay[y * n + j] * t1[(k * n + j) * rx + x];
                t2[(k * ry + y) * rx + x] = v;
            }
    for (int z = 0; z < rz; ++z)
        for (int y = 0; y < ry; ++y)
            for (int x = 0; x < rx; ++x) {
                double v = 0.0;
                for (int k = 0; k < n; ++k) v += Az[z * n + k] * t2[(k * ry + y) * rx + x];
                out[(z * ry + y) * rx + x] = v;
            }
}

// Metric terms of one curvilinear cell at uncollocated flux nodes: the mapping of degree p on
// the GLL support points (the solution's, grid_degree = poly_degree) with coordinates X
// [3][nd^3]; the cofactor by the conservative curl form (operators.cpp:2738-2884) evaluated at
// the nq^3 volume flux nodes and at each face's nq^2 flux nodes (operators.cpp:2444-2589), det J
// at the volume flux nodes (operators.cpp:2591-2672). Out: vmet [10][nq^3] (C[k][d] at row
// k * 3 + d, 1 / det J at row 9) and fnrm [6][3][nq^2] (face f's metric column C[:, f / 2]);
// returns false on a non-positive det J.
bool gl_curvilinear_cell(const std::vector<double>& xs, const std::vector<double>& xq, const double* X,
                         double* vmet, double* fnrm) {
    const int nd = (int)xs.size(), nq = (int)xq.size(), nd3 = nd * nd * nd, nq3 = nq * nq * nq, nf = nq * nq;
    std::vector<double> Bg((size_t)nd * nd), dBg((size_t)nd * nd), Bf((size_t)nq * nd), dBf((size_t)nq * nd);
    std::vector<double> Bs[2], dBs[2];
    for (int a = 0; a < nd; ++a) lagrange(xs, xs[a], &Bg[a * nd], &dBg[a * nd]);
    for (int q = 0; q < nq; ++q) lagrange(xs, xq[q], &Bf[q * nd], &dBf[q * nd]);
    for (int side = 0; side < 2; ++side) {
        Bs[side].assign(nd, 0.0); dBs[side].assign(nd, 0.0);
        lagrange(xs, (double)side, Bs[side].data(), dBs[side].data());
    }
    // the Jacobian at the support points and the nine products X_a dX_b/dxi_j there:
    // P[0..2] = z dy/dxi_j, P[3..5] = x dz/dxi_j, P[6..8] = y dx/dxi_j
    std::vector<double> GX[3][3], P[9];
    for (int m = 0; m < 3; ++m)
        for (int j = 0; j < 3; ++j) {
            GX[m][j].resize(nd3);
            const double* B[3] = {Bg.data(), Bg.data(), Bg.data()};
            B[j] = dBg.data();
            host_apply3(B[0], nd, B[1], nd, B[2], nd, nd, X + (size_t)m * nd3, GX[m][j].data());
        }
    for (int j = 0; j < 3; ++j) {
        P[j].resize(nd3); P[3 + j].resize(nd3); P[6 + j].resize(nd3);
        for (int g = 0; g < nd3; ++g) {
            P[j][g] = X[2 * nd3 + g] * GX[1][j][g];
            P[3 + j][g] = X[0 * nd3 + g] * GX[2][j][g];
            P[6 + j][g] = X[1 * nd3 + g] * GX[0][j][g];
        }
    }
    // the cofactor at the points selected by A (derivatives dA): row l from the products of row l,
    // C[l][0] = D_zeta(f_eta) - D_eta(f_zeta), C[l][1] = D_xi(f_zeta) - D_zeta(f_xi),
    // C[l][2] = D_eta(f_xi) - D_xi(f_eta)
    auto cofactor = [&](const double* const A[3], const double* const dA[3], const int r[3], double* C, int cs) {
        const int npts = r[0] * r[1] * r[2];
        std::vector<double> t1(npts), t2(npts);
        auto D = [&](int e, const std::vector<double>& f, std::vector<double>& out) {
            const double* B[3] = {A[0], A[1], A[2]};
            B[e] = dA[e];
            host_apply3(B[0], r[0], B[1], r[1], B[2], r[2], nd, f.data(), out.data());
        };
        for (int l = 0; l < 3; ++l) {
            const std::vector<double>* f = &P[3 * l];
            D(2, f[1], t1); D(1, f[2], t2);
            for (int q = 0; q < npts; ++q) C[(l * 3 + 0) * cs + q] = t1[q] - t2[q];
            D(0, f[2], t1); D(2, f[0], t2);
            for (int q = 0; q < npts; ++q) C[(l * 3 + 1) * cs + q] = t1[q] - t2[q];
            D(1, f[0], t1); D(0, f[1], t2);
            for (int q = 0; q < npts; ++q) C[(l * 3 + 2) * cs + q] = t1[q] - t2[q];
        }
    };
    {
        const double* A[3] = {Bf.data(), Bf.data(), Bf.data()};
        const double* dA[3] = {dBf.data(), dBf.data(), dBf.data()};
        const int r[3] = {nq, nq, nq};
        cofactor(A, dA, r, vmet, nq3);
        std::vector<double> Jm[3][3];
        for (int m = 0; m < 3; ++m)
            for (int j = 0; j < 3; ++j) {
                Jm[m][j].resize(nq3);
                const double* B[3] = {Bf.data(), Bf.data(), Bf.data()};
                B[j] = dBf.data();
                host_apply3(B[0], nq, B[1], nq, B[2], nq, nd, X + (size_t)m * nd3, Jm[m][j].data());
            }
        for (int q = 0; q < nq3; ++q) {
            double J[3][3];
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) J[a][b] = Jm[a][b][q];
            const double dj = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                              J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                              J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
            if (!(dj > 1e-14)) return false;
            vmet[9 * nq3 + q] = 1.0 / dj;
        }
    }
    std::vector<double> Cf((size_t)9 * nf);
    for (int f = 0; f < 6; ++f) {
        const int dn = f / 2, side = f % 2;
        const double* A[3] = {Bf.data(), Bf.data(), Bf.data()};
        const double* dA[3] = {dBf.data(), dBf.data(), dBf.data()};
        int r[3] = {nq, nq, nq};
        A[dn] = Bs[side].data(); dA[dn] = dBs[side].data(); r[dn] = 1;
        cofactor(A, dA, r, Cf.data(), nf);
        for (int k = 0; k < 3; ++k)
            for (int q = 0; q < nf; ++q) fnrm[((size_t)f * 3 + k) * nf + q] = Cf[(k * 3 + dn) * nf + q];
    }
    return true;
}

int check_mesh(const ph_mesh_desc* mesh) {
    const int n = mesh->n_cells_per_direction;
    if (n < 1 || !(mesh->right > mesh->left)) return fail(PH_ERR_INVALID, "bad mesh");
    if (mesh->cell_order < 0 || mesh->cell_order > 2) return fail(PH_ERR_INVALID, "cell_order must be 0, 1 or 2");
    // the recursive-children order exists only for hyper_cube + refine_global: n = 2^levels
    if (mesh->cell_order == 2 && (n & (n - 1)) != 0)
        return fail(PH_ERR_INVALID, "cell_order 2 (recursive children) needs n_cells_per_direction a power of two");
    for (int f = 0; f < 6; ++f) {
        const int t = mesh->boundary_type[f];
        if (t != 0 && (t < ph::BC_WALL || t > ph::BC_EXTRAPOLATION))
            return fail(PH_ERR_INVALID, "boundary_type: 0 (periodic) or a boundary_id 1001..1007");
    }
    for (int d = 0; d < 3; ++d)
        if ((mesh->boundary_type[2 * d] == 0) != (mesh->boundary_type[2 * d + 1] == 0))
            return fail(PH_ERR_INVALID, "boundary_type: a pair of cube sides is periodic on both sides or on neither");
    return PH_OK;
}

bool has_boundaries(const ph_mesh_desc* mesh) {
    for (int f = 0; f < 6; ++f)
        if (mesh->boundary_type[f] != 0) return true;
    return false;
}

// Non-periodic meshes: what the boundary terms take (nullptr when supported).
const char* boundary_reason(const ph_mesh_desc* mesh, const ph_params* prm) {
    if (!has_boundaries(mesh)) return nullptr;
    if (prm->pde_type == 1)
        for (int f = 0; f < 6; ++f) {
            const int t = mesh->boundary_type[f];
            // NavierStokes::boundary_face_values_viscous_flux defines the exterior state of 1000, 1001
            // and 1006 only (navier_stokes.cpp:1354-1390); for the others the reference's auxiliary
            // boundary term reads an unset state
            if (t != 0 && t != ph::BC_WALL && t != ph::BC_SLIP_WALL)
                return "boundary conditions: Navier-Stokes takes wall (1001) and slip wall (1006) boundaries";
        }
    return nullptr;
}

int check_param_ranges(const ph_params* prm) {
    if (prm->pde_type < 0 || prm->pde_type > 1 || prm->two_point_num_flux_type < 0 || prm->two_point_num_flux_type > 3 ||
        prm->conv_num_flux < 0 || prm->conv_num_flux > 5 || prm->diss_num_flux < 0 || prm->diss_num_flux > 2 ||
        prm->runge_kutta_method < 0 || prm->runge_kutta_method > 10 ||
        (prm->runge_kutta_method >= 4 && prm->runge_kutta_method <= 6) || prm->precision < 0 || prm->precision > 1 ||
        prm->flux_nodes_type < 0 || prm->flux_nodes_type > 1 || prm->flux_reconstruction_aux < 0 ||
        prm->flux_reconstruction_aux > 6 || prm->thermal_boundary_condition_type < 0 ||
        prm->thermal_boundary_condition_type > 1)
        return fail(PH_ERR_INVALID, "parameter out of range");
    // Euler::Euler aborts on a side slip (euler.cpp:47-51)
    if (std::fabs(prm->side_slip_angle * (std::atan(1.0) * 4.0) / 180.0) >= 1e-14)
        return fail(PH_ERR_INVALID, "side_slip_angle must be zero");
    return PH_OK;
}

bool uncollocated(const ph_params* prm) { return prm->flux_nodes_type != 1 || prm->overintegration != 0; }

const char* uncollocated_reason(const ph_mesh_desc* mesh, const ph_params* prm) {
    if (prm->overintegration < 0 || prm->overintegration > 2) return "overintegration must be 0, 1 or 2";
    if (prm->poly_degree < 1 || prm->poly_degree + 1 + prm->overintegration > ph::GL_MAXQ)
        return "uncollocated flux nodes: poly_degree >= 1 and poly_degree + 1 + overintegration <= 7";
    if (is_curvilinear(mesh)) {
        if (mesh->mapping_support_points == nullptr && mesh->grid_degree != prm->poly_degree)
            return "curvilinear meshes take grid_degree = poly_degree";
        if (prm->pde_type != 0 && prm->diss_num_flux == 0)
            return "curvilinear Navier-Stokes takes bassi_rebay_2 or central_visc_flux (the SIPG penalty's cell "
                   "extent on curved cells is not restated)";
    }
    if (prm->precision != PH_FP64) return "uncollocated flux nodes take the FP64 path";
    return nullptr;
}

const char* unsupported_reason(const ph_mesh_desc* mesh, const ph_params* prm) {
    if (uncollocated(prm))
        return "this entry point is collocated: flux_nodes_type = GLL and overintegration = 0 (contexts take both)";
    if (prm->poly_degree < 1 || prm->poly_degree > 6) return "poly_degree must be 1..6";
    if (is_curvilinear(mesh)) {
        if (mesh->mapping_support_points == nullptr && mesh->grid_degree != prm->poly_degree)
            return "curvilinear meshes take grid_degree = poly_degree";
        if (prm->pde_type != 0 && prm->diss_num_flux == 0)
            return "curvilinear Navier-Stokes takes bassi_rebay_2 or central_visc_flux (the SIPG penalty's cell "
                   "extent on curved cells is not restated)";
        if (prm->pde_type != 0 && prm->flux_reconstruction_aux != 0)
            return "curvilinear Navier-Stokes takes flux_reconstruction_aux = kDG";
    }
    return nullptr;
}

int build_operators(const ph_params* prm, ph::OpTab& tab, bool& fr, std::vector<double>& x, std::vector<double>& D) {
    const int N1 = prm->poly_degree + 1;
    std::vector<double> w;
    gll(N1, x, w);
    D.assign(N1 * N1, 0.0);
    std::vector<double> v(N1), dv(N1);
    for (int a = 0; a < N1; ++a) {
        lagrange(x, x[a], v.data(), dv.data());
        for (int l = 0; l < N1; ++l) D[a * N1 + l] = dv[l];
    }
    double cfr = 0.0, kaux = 0.0;
    if (fr_parameter(prm->flux_reconstruction, prm->poly_degree, prm->FR_user_specified_correction_parameter_value, cfr))
        return fail(PH_ERR_UNSUPPORTED, "flux_reconstruction type not defined for this degree");
    if (fr_aux_parameter(prm->flux_reconstruction_aux, prm->poly_degree, kaux))
        return fail(PH_ERR_UNSUPPORTED, "flux_reconstruction_aux type not defined for this degree");
    std::vector<double> Dp(N1 * N1, 0.0);
    for (int i = 0; i < N1; ++i) Dp[i * N1 + i] = 1.0;
    for (int k = 0; k < prm->poly_degree; ++k) Dp = mat_mul(D, Dp, N1);
    // K = (D^p)^T M D^p without its parameter; M + c K for the primary equation, M + k K for the
    // auxiliary one (local_Flux_Reconstruction_operator(_aux)::build_1D_volume_operator)
    std::vector<double> MK(N1 * N1, 0.0), MKa(N1 * N1, 0.0);
    for (int i = 0; i < N1; ++i)
        for (int j = 0; j < N1; ++j) {
            double kij = 0.0;
            for (int q = 0; q < N1; ++q) kij += Dp[q * N1 + i] * w[q] * Dp[q * N1 + j];
            MK[i * N1 + j] = (i == j ? w[i] : 0.0) + cfr * kij;
            MKa[i * N1 + j] = (i == j ? w[i] : 0.0) + kaux * kij;
        }
    std::vector<double> Minv, Minva;
    if (!mat_inv(MK, N1, Minv)) return fail(PH_ERR_INVALID, "singular FR mass matrix");
    if (!mat_inv(MKa, N1, Minva)) return fail(PH_ERR_INVALID, "singular auxiliary FR mass matrix");
    fr = (cfr != 0.0);
    std::memset(&tab, 0, sizeof(tab));
    tab.aux_fr = kaux != 0.0;
    for (int a = 0; a < N1; ++a) {
        tab.w[a] = w[a];
        for (int l = 0; l < N1; ++l) {
            tab.D[a * ph::MAXN1 + l] = D[a * N1 + l];
            tab.Dsk[a * ph::MAXN1 + l] = (w[a] * D[a * N1 + l] - w[l] * D[l * N1 + a]) / w[a];
            tab.Minv[a * ph::MAXN1 + l] = Minv[a * N1 + l];
            tab.B[a * ph::MAXN1 + l] = Minv[a * N1 + l] * w[l];
            tab.Baux[a * ph::MAXN1 + l] = Minva[a * N1 + l] * w[l];
        }
    }
    return PH_OK;
}

// 1-D operators of the uncollocated path (GL flux nodes, or overintegration): solution basis
// on the p + 1 GLL support points, nq flux nodes (QGauss, or QGaussLobatto with
// overintegration); the sets of DGBase::create_collection_tuple (dg_base.cpp:131-261) and
// OPERATOR::basis_functions / local_mass / local_basis_stiffness / vol_projection_operator /
// local_Flux_Reconstruction_operator (operators.cpp:1206-2005): chi, its face rows, the
// flux-node derivative and skew operator, M = chi^T W chi, the projection chi M^-1 chi^T W,
// and (M + K)^-1 with K = c (D^p)^T M D^p, D = M^-1 chi^T W chi'. The FR mass inverse also
// goes into ops.Minv for ph_apply_inverse_mass.
int build_gl_operators(const ph_params* prm, ph::GlTab& t, ph::OpTab& ops) {
    const int p = prm->poly_degree, nd = p + 1, nq = p + 1 + prm->overintegration;
    std::vector<double> xs, ws, xq, wq;
    gll(nd, xs, ws);
    if (prm->flux_nodes_type == 1) gll(nq, xq, wq); else gauss(nq, xq, wq);
    std::memset(&t, 0, sizeof(t));
    std::vector<double> chi((size_t)nq * nd), dchi((size_t)nq * nd), phi(nq), dph(nq);
    for (int q = 0; q < nq; ++q) {
        lagrange(xs, xq[q], &chi[q * nd], &dchi[q * nd]);
        lagrange(xq, xq[q], phi.data(), dph.data());
        for (int l = 0; l < nq; ++l) t.dphi[q * nq + l] = dph[l];
        t.wq[q] = wq[q];
    }
    for (int i = 0; i < nq * nd; ++i) t.chi[i] = chi[i];
    std::vector<double> tmp(std::max(nd, nq)), dtmp(std::max(nd, nq));
    for (int side = 0; side < 2; ++side) {
        lagrange(xs, (double)side, tmp.data(), dtmp.data());
        for (int i = 0; i < nd; ++i) t.chis[side][i] = tmp[i];
        lagrange(xq, (double)side, tmp.data(), dtmp.data());
        for (int l = 0; l < nq; ++l) t.phis[side][l] = tmp[l];
    }
    // S_ij = sum_q phi_i(x_q) phi_j'(x_q) w_q = w_i dphi[i][j] on the flux nodes
    for (int i = 0; i < nq; ++i)
        for (int j = 0; j < nq; ++j) t.skew[i * nq + j] = wq[i] * t.dphi[i * nq + j] - wq[j] * t.dphi[j * nq + i];
    std::vector<double> M((size_t)nd * nd, 0.0), Schi((size_t)nd * nd, 0.0);
    for (int i = 0; i < nd; ++i)
        for (int j = 0; j < nd; ++j)
            for (int q = 0; q < nq; ++q) {
                M[i * nd + j] += chi[q * nd + i] * chi[q * nd + j] * wq[q];
                Schi[i * nd + j] += chi[q * nd + i] * dchi[q * nd + j] * wq[q];
            }
    std::vector<double> Mi;
    if (!mat_inv(M, nd, Mi)) return fail(PH_ERR_INVALID, "singular mass matrix");
    // projection M^-1 chi^T W (nd x nq), then P = chi proj and the face rows chis proj
    std::vector<double> proj((size_t)nd * nq, 0.0);
    for (int i = 0; i < nd; ++i)
        for (int q = 0; q < nq; ++q) {
            double v = 0.0;
            for (int j = 0; j < nd; ++j) v += Mi[i * nd + j] * chi[q * nd + j] * wq[q];
            proj[i * nq + q] = v;
        }
    for (int a = 0; a < nq; ++a)
        for (int q = 0; q < nq; ++q) {
            double v = 0.0;
            for (int i = 0; i < nd; ++i) v += chi[a * nd + i] * proj[i * nq + q];
            t.P[a * nq + q] = v;
        }
    for (int side = 0; side < 2; ++side)
        for (int q = 0; q < nq; ++q) {
            double v = 0.0;
            for (int i = 0; i < nd; ++i) v += t.chis[side][i] * proj[i * nq + q];
            t.ps[side][q] = v;
        }
    // FR: D = M^-1 Schi, K = c (D^p)^T M D^p; the auxiliary equation's K_aux takes k for c
    double cfr = 0.0, kaux = 0.0;
    if (fr_parameter(prm->flux_reconstruction, p, prm->FR_user_specified_correction_parameter_value, cfr))
        return fail(PH_ERR_UNSUPPORTED, "flux_reconstruction type not defined for this degree");
    if (fr_aux_parameter(prm->flux_reconstruction_aux, p, kaux))
        return fail(PH_ERR_UNSUPPORTED, "flux_reconstruction_aux type not defined for this degree");
    const std::vector<double> Dm = mat_mul(Mi, Schi, nd);
    std::vector<double> Dp((size_t)nd * nd, 0.0);
    for (int i = 0; i < nd; ++i) Dp[i * nd + i] = 1.0;
    for (int k = 0; k < p; ++k) Dp = mat_mul(Dm, Dp, nd);
    std::vector<double> MK(M), MKa(M);
    for (int i = 0; i < nd; ++i)
        for (int j = 0; j < nd; ++j) {
            double kij = 0.0;
            for (int a = 0; a < nd; ++a)
                for (int b = 0; b < nd; ++b) kij += Dp[a * nd + i] * M[a * nd + b] * Dp[b * nd + j];
            MK[i * nd + j] += cfr * kij;
            MKa[i * nd + j] += kaux * kij;
        }
    std::vector<double> MKi, MKai;
    if (!mat_inv(MK, nd, MKi)) return fail(PH_ERR_INVALID, "singular FR mass matrix");
    if (kaux == 0.0) MKai = Mi;
    else if (!mat_inv(MKa, nd, MKai)) return fail(PH_ERR_INVALID, "singular auxiliary FR mass matrix");
    for (int i = 0; i < nd * nd; ++i) { t.minv[i] = MKi[i]; t.minv_aux[i] = MKai[i]; }
    // chi (M + K_aux)^-1 chi^T (nq x nq): the auxiliary equation's inverse mass seen from the flux
    // nodes (solution values at the flux nodes of (M + K_aux)^-1 chi^T applied to flux-node data)
    for (int a = 0; a < nq; ++a)
        for (int b = 0; b < nq; ++b) {
            double v = 0.0;
            for (int i = 0; i < nd; ++i) {
                double w = 0.0;
                for (int j = 0; j < nd; ++j) w += MKai[i * nd + j] * chi[b * nd + j];
                v += chi[a * nd + i] * w;
            }
            t.haux[a * nq + b] = v;
        }
    for (int a = 0; a < nd; ++a)
        for (int l = 0; l < nd; ++l) ops.Minv[a * ph::MAXN1 + l] = MKi[a * nd + l];
    // the projection of the weight-adjusted inverse mass on curvilinear cells, (M+K)^-1 chi^T W
    for (int i = 0; i < nd; ++i)
        for (int q = 0; q < nq; ++q) {
            double v = 0.0;
            for (int j = 0; j < nd; ++j) v += MKi[i * nd + j] * chi[q * nd + j];
            t.pwa[i * nq + q] = v * wq[q];
        }
    return PH_OK;
}

void build_integral_table(const std::vector<double>& x, int p, ph::IntegralTab& itab) {
    const int N1 = p + 1, ne = p + 11;
    std::memset(&itab, 0, sizeof(itab));
    std::vector<double> xe, we, v(N1), dv(N1);
    gauss(ne, xe, we);
    for (int q = 0; q < ne; ++q) {
        lagrange(x, xe[q], v.data(), dv.data());
        for (int a = 0; a < N1; ++a) { itab.B[q * N1 + a] = v[a]; itab.dB[q * N1 + a] = dv[a]; }
        itab.w[q] = we[q];
        itab.x[q] = xe[q];
    }
    // 1-D L2 projection onto the solution basis, P = M^-1 (W B)^T with the mass matrix of the
    // same quadrature (vol_projection_operator::build_1D_volume_operator, operators.cpp:1873-1889)
    std::vector<double> M((size_t)N1 * N1, 0.0), Mi;
    for (int i = 0; i < N1; ++i)
        for (int j = 0; j < N1; ++j)
            for (int q = 0; q < ne; ++q) M[i * N1 + j] += we[q] * itab.B[q * N1 + i] * itab.B[q * N1 + j];
    mat_inv(M, N1, Mi);   // a Gauss mass matrix of the Lagrange basis: symmetric positive definite
    for (int i = 0; i < N1; ++i)
        for (int q = 0; q < ne; ++q) {
            double acc = 0.0;
            for (int j = 0; j < N1; ++j) acc += Mi[i * N1 + j] * we[q] * itab.B[q * N1 + j];
            itab.P[i * ne + q] = acc;
        }
}

ph::PhysConst physics_constants(const ph_params* prm, double h, double& penalty) {
    ph::PhysConst pc{};
    pc.gam = prm->gamma_gas; pc.gm1 = prm->gamma_gas - 1.0;
    pc.mach2 = prm->mach_infinity * prm->mach_infinity;
    pc.temp_ratio = 110.4 / prm->temperature_inf;
    pc.inv_re = 1.0 / prm->reynolds_number_inf;
    pc.prandtl = prm->prandtl_number;
    pc.const_visc = prm->nondimensionalized_constant_viscosity;
    pc.use_const_visc = prm->use_constant_viscosity;
    pc.pressure_shift = prm->pressure_shift;
    pc.two_point = prm->two_point_num_flux_type;
    pc.conv_flux = prm->conv_num_flux;
    pc.diss_flux = prm->diss_num_flux;
    pc.navier_stokes = prm->pde_type == 1;
    double sipg = prm->sipg_penalty_factor;
    if (prm->diss_num_flux == 1) sipg = 0.0;   // all_parameters.cpp:611-614
    pc.sipg_pen = sipg;
    // SIPG penalty (dg_base.cpp:397-413), averaged over both (identical) cells
    penalty = (double)prm->poly_degree * (prm->poly_degree + 1) / h * sipg;
    // boundary conditions: the free stream of Euler::Euler (euler.cpp:14-70; angles in degrees as in the
    // .prm, parameters_euler.cpp:41-43) and the inlet totals of boundary_face_values (:1515-1516)
    const double pi = std::atan(1.0) * 4.0;
    const double aoa = prm->angle_of_attack * pi / 180.0, ss = prm->side_slip_angle * pi / 180.0;
    pc.bc_v_inf[0] = std::cos(aoa) * std::cos(ss);
    pc.bc_v_inf[1] = std::sin(aoa) * std::cos(ss);
    pc.bc_v_inf[2] = std::sin(ss);
    pc.bc_p_inf = 1.0 / (pc.gam * pc.mach2);
    const double t_inf = pc.gam * pc.bc_p_inf / 1.0 * pc.mach2;
    pc.bc_total_p = pc.bc_p_inf * std::pow(1.0 + 0.5 * pc.gm1 * pc.mach2, pc.gam / pc.gm1);
    pc.bc_total_t = t_inf * std::pow(pc.bc_total_p / pc.bc_p_inf, pc.gm1 / pc.gam);
    pc.bc_mach_inf = prm->mach_infinity;
    pc.bc_t_wall = prm->isothermal_wall_temperature;
    pc.bc_isothermal = prm->thermal_boundary_condition_type == 1;
    pc.bc_projected = prm->use_split_form && prm->use_projected_entropy_variables_for_nsfr_boundary_term;
    return pc;
}

// Boundary faces of a non-periodic cube: a cell face on a side with boundary_type[f] != 0 gets
// nbr = -1 - k, k numbering the boundary faces cell by cell, and btype[k] = boundary_type[f]
// (the boundary_id a flow case's grid gives those faces, e.g. channel_flow.cpp:324-343).
void apply_boundaries(int n, const std::vector<int>& ijk, const int types[6], std::vector<int>& nbr,
                      std::vector<int>& btype) {
    btype.clear();
    const int nc = (int)(ijk.size() / 3);
    for (int cc = 0; cc < nc; ++cc)
        for (int f = 0; f < 6; ++f) {
            const int d = f / 2;
            const int t = ijk[3 * cc + d];
            if (types[f] != 0 && ((f & 1) ? t == n - 1 : t == 0)) {
                nbr[6 * (size_t)cc + f] = -1 - (int)btype.size();
                btype.push_back(types[f]);
            }
        }
}

void periodic_connectivity(int n, int order, std::vector<int>& ijk, std::vector<int>& nbr) {
    const int nc = n * n * n;
    cell_order(n, order, ijk);
    std::vector<int> lex2cell(nc);
    nbr.assign(6 * (size_t)nc, 0);
    for (int cc = 0; cc < nc; ++cc) lex2cell[(ijk[3 * cc + 2] * n + ijk[3 * cc + 1]) * n + ijk[3 * cc]] = cc;
    for (int cc = 0; cc < nc; ++cc)
        for (int f = 0; f < 6; ++f) {
            int t[3] = {ijk[3 * cc], ijk[3 * cc + 1], ijk[3 * cc + 2]};
            const int d = f / 2;
            t[d] = (t[d] + ((f & 1) ? 1 : -1) + n) % n;
            nbr[6 * cc + f] = lex2cell[(t[2] * n + t[1]) * n + t[0]];
        }
}

// Slab z0 .. z0 + nz - 1 of the periodic cube, owned cells lexicographic (x, y, then z from
// z0). The lower ghost layer (layer z0 - 1) follows the owned cells, then the upper one
// (layer z0 + nz), each in (y, x) order; a ghost's own row names itself (no kernel evaluates
// a ghost). With nz = n the ghosts stand for the slab's own last and first layers.
void slab_connectivity(int n, int z0, int nz, std::vector<int>& ijk, std::vector<int>& nbr) {
    const int L = n * n, nown = nz * L;
    const int ntot = nown + 2 * L;
    ijk.assign(3 * (size_t)nown, 0);
    nbr.assign(6 * (size_t)ntot, 0);
    for (int cc = 0; cc < nown; ++cc) {
        const int i = cc % n, j = (cc / n) % n, kz = cc / L;
        ijk[3 * cc] = i; ijk[3 * cc + 1] = j; ijk[3 * cc + 2] = (z0 + kz) % n;
        const int in = j * n + i;
        nbr[6 * cc + 0] = kz * L + j * n + (i + n - 1) % n;
        nbr[6 * cc + 1] = kz * L + j * n + (i + 1) % n;
        nbr[6 * cc + 2] = kz * L + ((j + n - 1) % n) * n + i;
        nbr[6 * cc + 3] = kz * L + ((j + 1) % n) * n + i;
        nbr[6 * cc + 4] = kz > 0 ? cc - L : nown + in;
        nbr[6 * cc + 5] = kz < nz - 1 ? cc + L : nown + L + in;
    }
    for (int g = nown; g < ntot; ++g)
        for (int f = 0; f < 6; ++f) nbr[6 * (size_t)g + f] = g;
}

int node_geometry(int n, const std::vector<int>& ijk, const std::vector<double>& x, const std::vector<double>& D,
                  double left, double right, double warp, std::vector<double>& xyz, std::vector<double>& metric,
                  const double* support) {
    const int N1 = (int)x.size(), NP = N1 * N1 * N1, nc = (int)(ijk.size() / 3);
    const double h = (right - left) / n;
    const bool curv = warp != 0.0 || support != nullptr;
    xyz.assign((size_t)nc * NP * 3, 0.0);
    if (curv) metric.assign((size_t)nc * 10 * NP, 0.0);
    else metric.clear();
    const unsigned nthr = std::max(1u, std::min(32u, std::min(std::thread::hardware_concurrency(), (unsigned)nc)));
    std::vector<std::thread> pool;
    std::vector<int> ok(nthr, 1);
    for (unsigned tI = 0; tI < nthr; ++tI)
        pool.emplace_back([&, tI]() {
            for (int cc = (int)tI; cc < nc; cc += (int)nthr) {
                const int* t = &ijk[3 * cc];
                double* X = &xyz[(size_t)cc * NP * 3];
                if (curv) {
                    if (!curvilinear_cell(x, D, N1, h, left, right, warp, t, &metric[(size_t)cc * 10 * NP], X,
                                          support ? support + (size_t)cc * 3 * NP : nullptr))
                        ok[tI] = 0;
                } else {
                    for (int node = 0; node < NP; ++node) {
                        const int ii[3] = {node % N1, (node / N1) % N1, node / (N1 * N1)};
                        for (int d = 0; d < 3; ++d) X[node * 3 + d] = left + h * (t[d] + x[ii[d]]);
                    }
                }
            }
        });
    for (auto& th : pool) th.join();
    for (int v : ok)
        if (!v) return fail(PH_ERR_INVALID, "non-positive det J: the warp folds a cell");
    return PH_OK;
}

void rk_tableau(int method, int& ns, double A[4][4], double b[4]) {
    for (int i = 0; i < 4; ++i) { b[i] = 0.0; for (int j = 0; j < 4; ++j) A[i][j] = 0.0; }
    if (method == 0) {          // rk4_ex
        ns = 4; A[1][0] = 0.5; A[2][1] = 0.5; A[3][2] = 1.0;
        b[0] = 1.0 / 6.0; b[1] = 1.0 / 3.0; b[2] = 1.0 / 3.0; b[3] = 1.0 / 6.0;
    } else if (method == 1) {   // ssprk3_ex
        ns = 3; A[1][0] = 1.0; A[2][0] = 0.25; A[2][1] = 0.25;
        b[0] = 1.0 / 6.0; b[1] = 1.0 / 6.0; b[2] = 2.0 / 3.0;
    } else if (method == 2) {   // heun2_ex
        ns = 2; A[1][0] = 1.0;
        b[0] = 0.5; b[1] = 0.5;
    } else {                    // euler_ex
        ns = 1; b[0] = 1.0;
    }
}

const double* rk_stage_input(const RkBuffers& B, int i) {
    return (i == 0) ? B.sol : ((i - 1) % 2 == 0 ? B.stA : B.stB);
}

// Stage i of RungeKuttaODESolver::step_in_time (runge_kutta_ode_solver.cpp:15-100) fused
// into the residual epilogue: u_{i+1} = u_n + dt sum_j a_{i+1,j} k_j written as the next
// stage input, the b-weighted sum accumulated in acc, u_{n+1} written by the last stage.
void rk_stage_args(ph::StageArgs& a, const RkBuffers& B, int i, int ns, const double A[4][4], const double b[4],
                   double dt, bool fp32) {
    a.mode = 2;
    a.dt = dt;
    a.Un = B.sol;
    a.inc_mode = fp32 ? 1 : 0;
    a.acc_in = (i == 0) ? nullptr : B.acc;
    a.c_acc = dt * b[i];
    const bool last = (i == ns - 1);
    if (!last) {
        a.acc_out = B.acc;
        a.next = (i % 2 == 0) ? B.stA : B.stB;
        a.a_next = A[i + 1][i];
        if (B.carry && i >= 1 && A[i + 1][i - 1] != 0.0) a.carry_in = B.carry;
        if (B.carry && i + 2 < ns && A[i + 2][i] != 0.0) { a.carry_out = B.carry; a.a_carry = A[i + 2][i]; }
    } else {
        // the stage input is read by neighbouring CTAs, so a one-stage method writes elsewhere
        a.final_out = (ns == 1) ? B.stA : B.sol;
        a.comp = B.comp;
    }
}

// Low-storage tableaux: published coefficients (restated from
// src/ode_solver/runge_kutta_methods/low_storage_runge_kutta_methods.cpp).
bool low_storage_tableau(int method, LowStorageTableau& t) {
    t = LowStorageTableau();
    auto set = [&](int ns, int nd, int order, bool plus, std::initializer_list<std::array<double, 3>> g,
                   std::initializer_list<double> b, std::initializer_list<double> d, std::initializer_list<double> bh) {
        t.ns = ns; t.num_delta = nd; t.order = order; t.plus = plus;
        int i = 0;
        for (const auto& row : g) { t.gamma[i][0] = row[0]; t.gamma[i][1] = row[1]; t.gamma[i][2] = row[2]; ++i; }
        i = 0; for (double v : b) t.beta[i++] = v;
        i = 0; for (double v : d) t.delta[i++] = v;
        i = 0; for (double v : bh) t.bhat[i++] = v;
    };
    switch (method) {
    case 7:   // RK4(3)5[3S*]
        set(5, 7, 4, false,
            {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {-0.497531095840104, 1.384996869124138, 0.0},
             {1.010070514199942, 3.878155713328178, 0.0}, {-3.196559004608766, -2.324512951813145, 1.642598936063715},
             {1.717835630267259, -0.514633322274467, 0.188295940828347}},
            {0.0, 0.075152045700771, 0.211361016946069, 1.100713347634329, 0.728537814675568, 0.393172889823198},
            {1.0, 0.081252332929194, -1.083849060586449, -1.096110881845602, 2.859440022030827, -0.655568367959557,
             -0.194421504490852},
            {0.0, 0.0, 0.0, 0.0, 0.0, 0.0});
        return true;
    case 8:   // RK3(2)5F[3S*+]
        set(5, 5, 3, true,
            {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0},
             {0.2587771979725733308135192812685323706, 0.5528354909301389892439698870483746541, 0.0},
             {-0.1324380360140723382965420909764953437, 0.6731871608203061824849561782794643600, 0.0},
             {0.05056033948190826045833606441415585735, 0.2803103963297672407841316576323901761,
              0.2752563273304676380891217287572780582},
             {0.5670532000739313812633197158607642990, 0.5521525447020610386070346724931300367,
              -0.8950526174674033822276061734289327568}},
            {0.0, 0.2300298624518076223899418286314123354, 0.3021434166948288809034402119555380003,
             0.8025606185416310937583009085873554681, 0.4362158943603440930655148245148766471, 0.11292725304550591},
            {1.0, 0.34076558793345252, 0.34143826550033862, 0.72292753667879872, 0.0},
            {0.094841667050357029, 0.17263713394303537, 0.39982431890843712, 0.17180168075801786,
             0.058819144221557401, 0.1020760551185952388626787099944507877});
        return true;
    case 9:   // RK4(3)9F[3S*+]
        set(9, 9, 4, true,
            {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0},
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
              -0.04560955005031121479972862973705108039}},
            {0.0, 0.2836343005184365275160654678626695428, 0.9736500104654741223716056170419660217,
             0.3382359225242515288768487569778320563, -0.3584943611106183357043212309791897386,
             -0.004113944068471528211627210454497620358, 1.427968894048586363415504654313371031,
             0.01808470948394314017665968411915568633, 0.1605770645946802213926893453819236685,
             0.2952227015964591648775833803635147962},
            {1.0, 1.262923876648114432874834923838556100, 0.7574967189685911558308119415539596711,
             0.5163589453140728104667573195005629833, -0.02746327421802609557034437892013640319,
             -0.4382673178127944142238606608356542890, 1.273587294602656522645691372699677063,
             -0.6294740283927400326554066998751383342, 0.0},
            {0.02483675912451591196775756814283216443, 0.1866327774562103796990092260942180726,
             0.05671080795936984495604436622517631183, -0.003447695439149287702616943808570747099,
             0.003602245056516636472203469198006404016, 0.4545570622145088936800484247980581766,
             -0.0002434665289427612407531544765622888855, 0.06642755361103549971517945063138312147,
             0.1613697079523505006226025497715177578, 0.04955424859358438183052504342394102722});
        return true;
    case 10:  // RK5(4)10F[3S*+]
        set(10, 10, 5, true,
            {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0},
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
              -0.1377669797880289713535665985132703979}},
            {0.0, 0.2597883554788674084039539165398464630, 0.01777008889438867858759149597539211023,
             0.2481636629715501931294746189266601496, 0.7941736871152005775821844297293296135,
             0.3885391285642019129575902994397298066, 0.1455051657916305055730603387469193768,
             0.1587517385964749337690916959584348979, 0.1650605617880053419242434594242509601,
             0.2118093284937153836908655490906875007, 0.1559392342362059886106995325687547506},
            {1.0, -0.1331778419508803397033287009506932673, 0.8260422814750207498262063505871077303,
             1.513700425755728332485300719652378197, -1.305810059935023735972298885749903694,
             3.036678802924163246003321318996156380, -1.449458274398895177922690618003584514,
             3.834313899176362315089976408899373409, 4.122293760012985409330881631526514714, 0.0},
            {-0.02019255440012066080909442770590267512, 0.02737903480959184339932730854141598275,
             0.3028818636145965534365173822296811090, -0.03656843880622222190071445247906780540,
             0.3982664774676767729863101188528827405, -0.05715959421140685436681459970502471634,
             0.09849855103848558320961101178888983150, 0.06654601552456084978615342374581437947,
             0.09073479542748112726465375642050504556, 0.08432289325330803924891866923939606351,
             0.04529095628204896774513180907141004447});
        return true;
    }
    return false;
}

const double* lsrk_stage_args(ph::StageArgs& a, const RkBuffers& B, int i, const LowStorageTableau& t, double dt,
                              double atol, double rtol, double* err_partial) {
    const int ns = t.ns;
    a.mode = 3;
    a.dt = dt;
    a.atol = atol; a.rtol = rtol;
    a.ls_s2 = B.acc; a.ls_s3 = B.sol; a.ls_s4 = t.plus ? B.carry : nullptr;
    if (i == ns) {   // 3S*+: the first-same-as-last evaluation at u_{n+1} feeds the error register only
        a.ls_s1_out = nullptr;
        a.ls_bhat = t.bhat[ns];
        a.err_partial = err_partial;
        return B.sol;
    }
    const double* in = (i == 0) ? B.sol : ((i - 1) % 2 == 0 ? B.stA : B.stB);
    a.ls_s1_out = (i == ns - 1) ? B.sol : (i % 2 == 0 ? B.stA : B.stB);
    a.ls_g0 = t.gamma[i + 1][0]; a.ls_g1 = t.gamma[i + 1][1]; a.ls_g2 = t.gamma[i + 1][2];
    a.ls_beta = t.beta[i + 1];
    a.ls_delta = t.delta[i];
    a.ls_bhat = t.bhat[i];
    a.ls_first = (i == 0);
    if (!t.plus && i == ns - 1) {
        double sum = 0.0;
        for (int j = 0; j < t.num_delta; ++j) sum += t.delta[j];
        a.ls_embedded = 1;
        a.ls_delta_s = t.delta[ns]; a.ls_delta_s1 = t.delta[ns + 1];
        a.ls_inv_sum_delta = 1.0 / sum;
        a.err_partial = err_partial;
    }
    return in;
}

} // namespace ph_host

using namespace ph_host;

struct ph_ctx {
    ph_params prm{};
    int n = 0, nc = 0, p = 0, N1 = 0, NP = 0;
    double left = 0, right = 1, h = 1;
    cudaStream_t stream = nullptr;
    int device = 0;
    bool visc = false, split = false, fp32 = false, fr = false, curv = false;
    double warp = 0.0;
    std::vector<double> xyz;            // physical node coordinates [cell][node][3]
    double* d_metric = nullptr;         // curvilinear: [nc][10][NP] cofactor rows + 1/det J
    double* d_xnode = nullptr;          // curvilinear: node coordinates [nc][3][NP] (integrals)
    double* d_origin = nullptr;         // affine: lower corner of each cell [nc][3] (integrals)
    size_t ndofs = 0;
    std::vector<int> ijk;
    int* d_nbr = nullptr;
    ph::OpTab h_ops{};
    ph::OpTab* d_ops = nullptr;
    ph::IntegralTab* d_itab = nullptr;
    double *d_sol = nullptr, *d_stA = nullptr, *d_stB = nullptr, *d_acc = nullptr, *d_carry = nullptr;
    double *d_fv = nullptr, *d_comp = nullptr, *d_tmpA = nullptr, *d_tmpB = nullptr, *d_partial = nullptr;
    unsigned* d_status = nullptr;
    ph::PhysConst pc{};
    double pen = 0.0;
    int ns = 0;
    double A[4][4] = {{0}}, b[4] = {0};
    bool lowstorage = false;            // 3S* / 3S*+ low-storage method
    LowStorageTableau ls;
    double* d_err = nullptr;            // per-tile squared scaled errors of the last low-storage step
    int err_tiles = 0;
    // relaxation RK: per-stage per-tile sums of v^T M k, per-cell entropy partials, the last
    // parameter (the next step's initial guess) and the time advanced by the last call
    bool rrk = false;
    double* d_ent = nullptr;
    double* d_ent_cell = nullptr;
    int ent_tiles = 0;
    double rrk_gamma = 1.0, rrk_elapsed = 0.0;
    std::vector<double> h_ent;
    std::vector<double> h_partial;
    // positivity-preserving limiter (2 Zhang 2010, 3 Wang 2012; 0 none) and its 1-D tables
    int limiter = 0;
    ph::LimiterTab* d_ltab = nullptr;
    // uncollocated path (GL flux nodes / overintegration): nq flux nodes per direction, the
    // operator table and the face / viscous buffers of its kernels
    bool gl = false;
    int NQ = 0;
    ph::GlTab h_gl{};
    ph::GlTab* d_gl = nullptr;
    double* d_t1 = nullptr;
    double* d_t2 = nullptr;
    double* d_vis = nullptr;
    double* d_glvm = nullptr;           // curvilinear uncollocated: [nc][10][nq^3] cofactor + 1 / det J
    double* d_glfn = nullptr;           // curvilinear uncollocated: [nc][6][3][nq^2] face metric columns
    // optional per-kernel timing: 1 = CUDA events around every direct launch, the stream
    // synchronised after each; 2 = event-record nodes between the kernels of the captured
    // RK step, a fresh set of events for every replay (the replays themselves are timed)
    int timing = 0;
    double t_ms[3] = {0, 0, 0};      // residual/stage kernel, auxiliary kernel, other
    long long t_n[3] = {0, 0, 0};
    long long launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool capturing = false;                        // inside capture_step_graph
    cudaStream_t tside = nullptr;                  // mode 2: the event nodes' side branch of the graph
    cudaEvent_t tfork = nullptr;                   // mode 2: fork / join points of that branch
    std::vector<cudaEvent_t> tcap;                 // mode 2: events recorded at capture, kernels + 1
    std::vector<int> tcls;                         // mode 2: class of kernel j of the step
    std::vector<cudaGraphNode_t> tnodes;           // mode 2: the event-record node of tcap[j]
    std::vector<std::vector<cudaEvent_t>> tpool;   // mode 2: the events of replay r
    size_t treplays = 0;                           // mode 2: replays since the last reset
    // one RK step captured as a CUDA graph, replayed by ph_rk_step while dt stays the same
    // (only on a caller-given stream: the legacy default stream cannot be captured)
    cudaGraphExec_t step_graph = nullptr;
    cudaGraph_t step_graph_src = nullptr;          // mode 2: kept for its node handles
    double step_graph_dt = 0.0;
    int step_graph_launches = 0;
    // ph_run: device table of integrals rows, its row counter, and the captured graph of one
    // record interval (record_every steps, the integrals and the row reduction)
    double* d_table = nullptr;
    int table_rows = 0;
    int* d_counter = nullptr;
    cudaGraphExec_t run_graph = nullptr;
    double run_graph_dt = 0.0;
    int run_graph_every = 0;
    int run_graph_launches = 0;
    // slab of a mesh shared by several GPUs: the owned layers z_first .. z_first + z_count - 1,
    // the ghost layers (2 n^2 cells, face data only) stored after the owned cells in every
    // stage-input state buffer and in the viscous terms
    bool slab = false;
    int z_first = 0, z_count = 0, layer = 0, nc_ghost = 0;
    // non-periodic mesh: boundary faces (nbr = -1 - k), their boundary_id and (Navier-Stokes) the
    // boundary viscous fluxes of the auxiliary kernel
    int nb = 0;
    int* d_btype = nullptr;
    double* d_fb = nullptr;
    // tile lists (first cell of each CTA's tile): the nt_int tiles without a boundary face, then
    // the nt_bnd tiles with one
    int* d_tiles = nullptr;
    int nt_int = 0, nt_bnd = 0;
    std::vector<int> h_tiles;
    size_t nalloc = 0;                  // doubles per stage-input buffer, ghost slots included
    // stage tiles [0, lo_end) and [hi_begin, nc) read ghost data (CPC-aligned, so the tiles and
    // their partial sums are those of one launch over all cells); [lo_end, hi_begin) do not
    int lo_end = 0, hi_begin = 0;
    ph_halo_fn halo_fn = nullptr;
    void* halo_user = nullptr;
    ph_rank_sum_fn sum_fn = nullptr;    // slab contexts with relaxation RK
    void* sum_user = nullptr;
    unsigned char* d_halo = nullptr;    // send_lo | send_hi | recv_lo | recv_hi, halo_stride bytes each
    size_t halo_stride = 0, halo_state_bytes = 0, halo_visc_bytes = 0;
    // the interior cells' kernels run on a second stream, concurrently with the exchange and the
    // first and last layers' kernels; events fork it from and join it to the context stream
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_aux = nullptr, ev_join = nullptr;
};

namespace {

// NVTX range for the profilers' timelines (a no-op unless a tool is attached): one per RK
// step, per stage and per kernel launch
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

constexpr size_t TIMED_KERNELS_PER_STEP = 64;

void drop_step_graph(ph_ctx* c) {
    if (c->step_graph) { cudaGraphExecDestroy(c->step_graph); c->step_graph = nullptr; }
    if (c->step_graph_src) { cudaGraphDestroy(c->step_graph_src); c->step_graph_src = nullptr; }
    c->tnodes.clear();
}

// Mode 2: an event-record node of the captured graph on a side branch that forks from the
// context stream at this point, so the kernels that follow do not wait for the event.
void timer_mark(ph_ctx* c, cudaEvent_t ev) {
    cudaEventRecord(c->tfork, c->stream);
    cudaStreamWaitEvent(c->tside, c->tfork, 0);
    cudaEventRecordWithFlags(ev, c->tside, cudaEventRecordExternal);
}

void timer_begin(ph_ctx* c) {
    if (c->timing == 1) cudaEventRecord(c->ev0, c->stream);
    else if (c->timing == 2 && c->capturing && c->tcls.empty()) timer_mark(c, c->tcap[0]);
}
void timer_end(ph_ctx* c, int cls) {
    ++c->launches;
    if (c->timing == 2) {
        if (c->capturing && c->tcls.size() + 1 < c->tcap.size()) {
            c->tcls.push_back(cls);
            timer_mark(c, c->tcap[c->tcls.size()]);
        }
        return;
    }
    if (c->timing != 1) return;
    cudaEventRecord(c->ev1, c->stream);
    cudaEventSynchronize(c->ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->t_ms[cls] += ms;
    c->t_n[cls] += 1;
}

// The tiles of list `list` (0: without a boundary face, 1: with one) whose first cell lies in
// [b, e): their offset in the device tile array and their count (each list ascends; launch ranges
// are whole tiles).
void tile_span(const ph_ctx* c, int list, int b, int e, int* off, int* cnt) {
    const int base = list ? c->nt_int : 0, n = list ? c->nt_bnd : c->nt_int;
    const int* t = c->h_tiles.data() + base;
    const int i0 = (int)(std::lower_bound(t, t + n, b) - t), i1 = (int)(std::lower_bound(t, t + n, e) - t);
    *off = base + i0;
    *cnt = i1 - i0;
}

// cells per CTA of the stage and auxiliary kernels (the uncollocated ones: one)
int cells_per_tile(const ph_ctx* c) {
    if (c->gl) return 1;
    int threads = 0, cpc = 1;
    size_t smem = 0;
    switch (c->N1) {
    case 2: ph::stage_launch_shape<2>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    case 3: ph::stage_launch_shape<3>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    case 4: ph::stage_launch_shape<4>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    case 5: ph::stage_launch_shape<5>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    case 6: ph::stage_launch_shape<6>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    default: ph::stage_launch_shape<7>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    }
    return cpc;
}

int dispatch_stage(ph_ctx* c, const ph::StageArgs& a) {
    if (c->nb && !a.tiles) {   // non-periodic mesh: the periodic kernel on the range's tiles without a
                               // boundary face, the boundary-face kernel on the others
        int oi, ni, ob, nbt;
        tile_span(c, 0, a.cell_begin, a.nc, &oi, &ni);
        tile_span(c, 1, a.cell_begin, a.nc, &ob, &nbt);
        ph::StageArgs ai = a, ab = a;
        ai.btype = nullptr; ai.tiles = c->d_tiles + oi; ai.ntiles = ni;
        ab.btype = c->d_btype; ab.tiles = c->d_tiles + ob; ab.ntiles = nbt;
        if (ni) if (int rc = dispatch_stage(c, ai)) return rc;
        if (nbt) return dispatch_stage(c, ab);
        return PH_OK;
    }
    NvtxRange nvtx("stage kernel");
    cudaError_t e;
    timer_begin(c);
    switch (c->N1) {
    case 2: e = ph::launch_stage<2>(a, c->fp32, c->visc, c->split, c->stream); break;
    case 3: e = ph::launch_stage<3>(a, c->fp32, c->visc, c->split, c->stream); break;
    case 4: e = ph::launch_stage<4>(a, c->fp32, c->visc, c->split, c->stream); break;
    case 5: e = ph::launch_stage<5>(a, c->fp32, c->visc, c->split, c->stream); break;
    case 6: e = ph::launch_stage<6>(a, c->fp32, c->visc, c->split, c->stream); break;
    case 7: e = ph::launch_stage<7>(a, c->fp32, c->visc, c->split, c->stream); break;
    default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree outside 1..6");
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string("residual launch: ") + cudaGetErrorString(e));
    timer_end(c, 0);
    return PH_OK;
}

// one auxiliary-kernel launch (bnd: a tile list, with btype set the boundary-face kernel)
static int aux_launch(ph_ctx* c, const double* U, int cell_begin, int cell_end, const ph::BoundaryArgs* bnd) {
    NvtxRange nvtx("auxiliary kernel");
    cudaError_t e;
    const double inv_h = 1.0 / c->h;
    timer_begin(c);
    switch (c->N1) {
    case 2: e = ph::launch_aux<2>(U, c->d_nbr, c->h_ops, cell_begin, cell_end, inv_h, c->pc, c->fp32, c->d_fv, c->curv ? c->d_metric : nullptr, c->stream, bnd); break;
    case 3: e = ph::launch_aux<3>(U, c->d_nbr, c->h_ops, cell_begin, cell_end, inv_h, c->pc, c->fp32, c->d_fv, c->curv ? c->d_metric : nullptr, c->stream, bnd); break;
    case 4: e = ph::launch_aux<4>(U, c->d_nbr, c->h_ops, cell_begin, cell_end, inv_h, c->pc, c->fp32, c->d_fv, c->curv ? c->d_metric : nullptr, c->stream, bnd); break;
    case 5: e = ph::launch_aux<5>(U, c->d_nbr, c->h_ops, cell_begin, cell_end, inv_h, c->pc, c->fp32, c->d_fv, c->curv ? c->d_metric : nullptr, c->stream, bnd); break;
    case 6: e = ph::launch_aux<6>(U, c->d_nbr, c->h_ops, cell_begin, cell_end, inv_h, c->pc, c->fp32, c->d_fv, c->curv ? c->d_metric : nullptr, c->stream, bnd); break;
    case 7: e = ph::launch_aux<7>(U, c->d_nbr, c->h_ops, cell_begin, cell_end, inv_h, c->pc, c->fp32, c->d_fv, c->curv ? c->d_metric : nullptr, c->stream, bnd); break;
    default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree outside 1..6");
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string("aux launch: ") + cudaGetErrorString(e));
    timer_end(c, 1);
    return PH_OK;
}

int dispatch_aux(ph_ctx* c, const double* U, int cell_begin, int cell_end) {
    if (!c->nb) return aux_launch(c, U, cell_begin, cell_end, nullptr);
    // non-periodic mesh: the periodic kernel on the tiles without a boundary face, then the
    // boundary-face kernel on the others (it stores the boundary viscous fluxes)
    int oi, ni, ob, nbt;
    tile_span(c, 0, cell_begin, cell_end, &oi, &ni);
    tile_span(c, 1, cell_begin, cell_end, &ob, &nbt);
    const ph::BoundaryArgs bi{nullptr, c->d_fb, c->pen, c->d_tiles + oi, ni};
    const ph::BoundaryArgs bb{c->d_btype, c->d_fb, c->pen, c->d_tiles + ob, nbt};
    if (ni) if (int rc = aux_launch(c, U, cell_begin, cell_end, &bi)) return rc;
    if (nbt) return aux_launch(c, U, cell_begin, cell_end, &bb);
    return PH_OK;
}

// One kernel of the uncollocated path on the stage input a.U: 0 face values, 1 auxiliary
// equation, 2 residual / RK stage, 3 the curvilinear weight-adjusted inverse mass (timing classes:
// other, auxiliary, stage, other).
int dispatch_gl(ph_ctx* c, int kernel, const ph::StageArgs& a) {
    if (c->nb && (kernel == 1 || kernel == 2) && !a.tiles) {
        // non-periodic mesh: the periodic kernel on the cells without a boundary face, the
        // boundary-face kernel on the others
        int oi, ni, ob, nbt;
        tile_span(c, 0, a.cell_begin, a.nc, &oi, &ni);
        tile_span(c, 1, a.cell_begin, a.nc, &ob, &nbt);
        ph::StageArgs ai = a, ab = a;
        ai.btype = nullptr; ai.tiles = c->d_tiles + oi; ai.ntiles = ni;
        ab.btype = c->d_btype; ab.tiles = c->d_tiles + ob; ab.ntiles = nbt;
        if (ni) if (int rc = dispatch_gl(c, kernel, ai)) return rc;
        if (nbt) return dispatch_gl(c, kernel, ab);
        return PH_OK;
    }
    static const char* const kName[] = {"face-value kernel", "auxiliary kernel", "stage kernel",
                                        "inverse-mass kernel"};
    NvtxRange nvtx(kName[kernel]);
    const ph::GlArgs g{c->d_gl, c->d_t1, c->d_t2, c->d_vis, c->d_glvm, c->d_glfn, c->d_fb};
    cudaError_t e;
    timer_begin(c);
    switch (c->N1) {
    case 2: e = ph::launch_gl<2>(kernel, c->NQ, a, g, c->h_gl, c->visc, c->split, c->stream); break;
    case 3: e = ph::launch_gl<3>(kernel, c->NQ, a, g, c->h_gl, c->visc, c->split, c->stream); break;
    case 4: e = ph::launch_gl<4>(kernel, c->NQ, a, g, c->h_gl, c->visc, c->split, c->stream); break;
    case 5: e = ph::launch_gl<5>(kernel, c->NQ, a, g, c->h_gl, c->visc, c->split, c->stream); break;
    case 6: e = ph::launch_gl<6>(kernel, c->NQ, a, g, c->h_gl, c->visc, c->split, c->stream); break;
    case 7: e = ph::launch_gl<7>(kernel, c->NQ, a, g, c->h_gl, c->visc, c->split, c->stream); break;
    default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree outside 1..6");
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string(kName[kernel]) + " launch: " + cudaGetErrorString(e));
    timer_end(c, kernel == 2 ? 0 : kernel == 1 ? 1 : 2);   // (the inverse mass alone: other)
    return PH_OK;
}

// The positivity-preserving limiter on a state of this context (in place), for a stage of dt.
int dispatch_limiter(ph_ctx* c, double* U, double dt) {
    NvtxRange nvtx("limiter kernel");
    ph::LimiterArgs la{U, c->d_ltab, c->nc, dt / c->h, c->prm.gamma_gas, c->prm.min_density, c->limiter == 2 ? 1 : 0};
    cudaError_t e;
    timer_begin(c);
    switch (c->N1) {
    case 2: e = ph::launch_limiter<2>(la, c->stream); break;
    case 3: e = ph::launch_limiter<3>(la, c->stream); break;
    case 4: e = ph::launch_limiter<4>(la, c->stream); break;
    case 5: e = ph::launch_limiter<5>(la, c->stream); break;
    case 6: e = ph::launch_limiter<6>(la, c->stream); break;
    case 7: e = ph::launch_limiter<7>(la, c->stream); break;
    default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree outside 1..6");
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string("limiter launch: ") + cudaGetErrorString(e));
    timer_end(c, 2);
    return PH_OK;
}

// Halo copy of a slab context: rows of `width` 8-byte words for both partition faces at once
// (blockIdx.y = side), from a strided source to a strided destination.
struct HaloCopy {
    const unsigned long long* src[2];
    unsigned long long* dst[2];
    long long src_pitch, dst_pitch;   // words between rows
    int rows, width;
};

__global__ void halo_copy_kernel(const HaloCopy h) {
    const int side = blockIdx.y;
    const long long total = (long long)h.rows * h.width;
    const unsigned long long* __restrict__ src = h.src[side];
    unsigned long long* __restrict__ dst = h.dst[side];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / h.width, w = i - r * h.width;
        dst[r * h.dst_pitch + w] = src[r * h.src_pitch + w];
    }
}

// Packs (pack = true) the first owned layer's bottom-face data into send_lo and the last
// layer's top-face data into send_hi, or unpacks recv_lo into the lower ghost layer (its top
// face, read by the first layer's z- faces) and recv_hi into the upper ghost layer (its
// bottom face). STATE: the 5 components at the face's (p+1)^2 nodes of the state buffer U;
// VISCOUS: the face's block of the viscous terms (4 (p+1)^2 values of the arithmetic type).
// Uncollocated flux nodes: STATE is the face's block of the face-value buffer (the state's and
// the projected entropy variables' face values, written by the face-value kernel), VISCOUS the
// first four rows of the face's viscous block (each side's F_v . n).
int halo_copy(ph_ctx* c, int what, bool pack, const double* U) {
    const int N1 = c->N1, NF = N1 * N1, NP = c->NP, L = c->layer, nc = c->nc;
    unsigned char* hb = c->d_halo;
    unsigned long long* buf[4];
    for (int i = 0; i < 4; ++i) buf[i] = reinterpret_cast<unsigned long long*>(hb + i * c->halo_stride);
    HaloCopy h{};
    const unsigned long long* vol[2];
    unsigned long long* volw[2];
    long long vpitch;
    if (c->gl) {   // uncollocated: the face blocks of the face-value / viscous buffers
        const int NQF = c->NQ * c->NQ, T1W = c->split ? 10 : 5;
        const size_t cw = (size_t)6 * (what == PH_HALO_STATE ? T1W : ph::GL_T2W) * NQF;   // words per cell
        const size_t fw = cw / 6;                                                          // per face
        auto* w = reinterpret_cast<unsigned long long*>(what == PH_HALO_STATE ? c->d_t1 : c->d_t2);
        h.rows = L; h.width = (int)(what == PH_HALO_STATE ? fw : (size_t)4 * NQF); vpitch = (long long)cw;
        if (pack) { vol[0] = w + 4 * fw; vol[1] = w + (size_t)(nc - L) * cw + 5 * fw; }
        else { volw[0] = w + (size_t)nc * cw + 5 * fw; volw[1] = w + (size_t)(nc + L) * cw + 4 * fw; }
    } else if (what == PH_HALO_STATE) {
        auto* w = reinterpret_cast<unsigned long long*>(const_cast<double*>(U));
        h.rows = 5 * L; h.width = NF; vpitch = NP;
        if (pack) { vol[0] = w; vol[1] = w + (size_t)(nc - L) * 5 * NP + (size_t)(N1 - 1) * NF; }
        else { volw[0] = w + (size_t)nc * 5 * NP + (size_t)(N1 - 1) * NF; volw[1] = w + (size_t)(nc + L) * 5 * NP; }
    } else {
        const size_t es = c->fp32 ? sizeof(float) : sizeof(double);
        const size_t VT = (size_t)4 * NP + (size_t)24 * NF;
        auto* w = reinterpret_cast<unsigned long long*>(c->d_fv);
        const size_t vtw = VT * es / 8, blk = (size_t)4 * NF * es / 8;
        auto off = [&](int f) { return ((size_t)4 * NP + (size_t)f * 4 * NF) * es / 8; };
        h.rows = L; h.width = (int)blk; vpitch = (long long)vtw;
        if (pack) { vol[0] = w + off(4); vol[1] = w + (size_t)(nc - L) * vtw + off(5); }
        else { volw[0] = w + (size_t)nc * vtw + off(5); volw[1] = w + (size_t)(nc + L) * vtw + off(4); }
    }
    if (pack) {
        h.src[0] = vol[0]; h.src[1] = vol[1]; h.dst[0] = buf[0]; h.dst[1] = buf[1];
        h.src_pitch = vpitch; h.dst_pitch = h.width;
    } else {
        h.src[0] = buf[2]; h.src[1] = buf[3]; h.dst[0] = volw[0]; h.dst[1] = volw[1];
        h.src_pitch = h.width; h.dst_pitch = vpitch;
    }
    const long long total = (long long)h.rows * h.width;
    const int gx = (int)std::min<long long>((total + 255) / 256, 4 * 148);
    timer_begin(c);
    halo_copy_kernel<<<dim3(gx, 2), 256, 0, c->stream>>>(h);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string("halo copy: ") + cudaGetErrorString(e));
    timer_end(c, 2);
    return PH_OK;
}

int halo_call(ph_ctx* c, int what, int phase) {
    if (!c->halo_fn) return fail(PH_ERR_INVALID, "a slab context needs ph_set_halo_exchange before it evaluates a residual");
    unsigned char* b = c->d_halo;
    const size_t st = c->halo_stride;
    const size_t bytes = what == PH_HALO_STATE ? c->halo_state_bytes : c->halo_visc_bytes;
    const int rc = c->halo_fn(c->halo_user, what, phase, b, b + st, b + 2 * st, b + 3 * st, bytes, (void*)c->stream);
    if (rc) return fail(PH_ERR_EXCHANGE, "halo exchange callback returned " + std::to_string(rc));
    return PH_OK;
}

// values[0..n) summed over the ranks of the mesh (slab contexts; a whole mesh is its own sum)
int rank_sum(ph_ctx* c, double* values, int n) {
    if (!c->nc_ghost) return PH_OK;
    if (!c->sum_fn) return fail(PH_ERR_INVALID, "a slab context with relaxation RK needs ph_set_rank_sum");
    const int rc = c->sum_fn(c->sum_user, values, n);
    if (rc) return fail(PH_ERR_EXCHANGE, "rank sum callback returned " + std::to_string(rc));
    return PH_OK;
}

ph::StageArgs base_args(ph_ctx* c, const double* U) {
    ph::StageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.U = U; a.Fv = c->d_fv; a.nbr = c->d_nbr; a.ops = c->d_ops; a.nc = c->nc;
    a.h = c->h; a.inv_h = 1.0 / c->h; a.pen = c->pen; a.pc = c->pc; a.status = c->d_status;
    a.fr = c->fr ? 1 : 0;
    a.metric = c->d_metric;
    a.btype = c->nb ? c->d_btype : nullptr;
    a.Fb = c->d_fb;
    return a;
}

template <typename T>
int dalloc(T** p, size_t count) {
    if (cudaMalloc((void**)p, count * sizeof(T)) != cudaSuccess) { *p = nullptr; return 1; }
    return 0;
}

int stage_range(ph_ctx* c, ph::StageArgs a, int begin, int end) {
    if (begin >= end) return PH_OK;
    a.cell_begin = begin; a.nc = end;
    return dispatch_stage(c, a);
}

// One residual evaluation on the stage input `in` (auxiliary kernel, then the stage kernel with
// the epilogue `a` asks for). In a slab context with neighbours the ghost layers of `in` and of
// the viscous terms are refreshed through the halo callback; the cells that read no ghost data
// run while each transfer is in flight, the first and last layer after it. Every cell runs the
// same code on the same inputs as in one launch over all cells.
// Runs `launch` on the interior stream after everything queued so far on the context stream
// (or on the context stream itself when `fork` is false); `done`, when given, is recorded on
// the interior stream after it.
template <typename F>
int on_interior(ph_ctx* c, bool fork, F launch, cudaEvent_t done) {
    if (!fork) return launch();
    PH_CUDA(cudaEventRecord(c->ev_fork, c->stream));
    PH_CUDA(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    cudaStream_t main = c->stream;
    c->stream = c->side;
    const int rc = launch();
    c->stream = main;
    if (rc) return rc;
    if (done) PH_CUDA(cudaEventRecord(done, c->side));
    return PH_OK;
}

int eval_residual(ph_ctx* c, const double* in, ph::StageArgs a) {
    a.U = in;
    if (c->gl) {   // face values, (auxiliary equation,) residual: every kernel over all cells
        a.cell_begin = 0; a.nc = c->nc;
        if (int rc = dispatch_gl(c, 0, a)) return rc;
        if (c->nc_ghost) {   // a slab: the partition faces' face values to and from the neighbours
            if (int rc = halo_copy(c, PH_HALO_STATE, true, in)) return rc;
            if (int rc = halo_call(c, PH_HALO_STATE, PH_HALO_BEGIN)) return rc;
            if (int rc = halo_call(c, PH_HALO_STATE, PH_HALO_END)) return rc;
            if (int rc = halo_copy(c, PH_HALO_STATE, false, in)) return rc;
        }
        if (c->visc) {
            if (int rc = dispatch_gl(c, 1, a)) return rc;
            if (c->nc_ghost) {
                if (int rc = halo_copy(c, PH_HALO_VISCOUS, true, in)) return rc;
                if (int rc = halo_call(c, PH_HALO_VISCOUS, PH_HALO_BEGIN)) return rc;
                if (int rc = halo_call(c, PH_HALO_VISCOUS, PH_HALO_END)) return rc;
                if (int rc = halo_copy(c, PH_HALO_VISCOUS, false, in)) return rc;
            }
        }
        return dispatch_gl(c, 2, a);
    }
    if (!c->nc_ghost) {
        if (c->visc) if (int rc = dispatch_aux(c, in, 0, c->nc)) return rc;
        return stage_range(c, a, 0, c->nc);
    }
    const int lo = c->lo_end, hi = c->hi_begin, nc = c->nc;
    // the interior runs concurrently unless there is none or every launch is being timed
    const bool fork = lo < hi && c->timing != 1;
    if (int rc = halo_copy(c, PH_HALO_STATE, true, in)) return rc;
    if (int rc = halo_call(c, PH_HALO_STATE, PH_HALO_BEGIN)) return rc;
    if (lo < hi) {
        if (c->visc) {
            if (int rc = on_interior(c, fork, [&] { return dispatch_aux(c, in, lo, hi); }, c->ev_aux)) return rc;
        } else if (int rc = on_interior(c, fork, [&] { return stage_range(c, a, lo, hi); }, c->ev_join)) {
            return rc;
        }
    }
    if (int rc = halo_call(c, PH_HALO_STATE, PH_HALO_END)) return rc;
    if (int rc = halo_copy(c, PH_HALO_STATE, false, in)) return rc;
    if (c->visc) {
        if (int rc = dispatch_aux(c, in, 0, lo)) return rc;
        if (hi < nc) if (int rc = dispatch_aux(c, in, hi, nc)) return rc;
        if (int rc = halo_copy(c, PH_HALO_VISCOUS, true, in)) return rc;
        if (int rc = halo_call(c, PH_HALO_VISCOUS, PH_HALO_BEGIN)) return rc;
        // the interior stage reads the first and last layers' viscous terms: forked after them
        if (int rc = on_interior(c, fork, [&] { return stage_range(c, a, lo, hi); }, c->ev_join)) return rc;
        if (int rc = halo_call(c, PH_HALO_VISCOUS, PH_HALO_END)) return rc;
        if (int rc = halo_copy(c, PH_HALO_VISCOUS, false, in)) return rc;
        // ... and the first and last layers read the interior's
        if (fork) PH_CUDA(cudaStreamWaitEvent(c->stream, c->ev_aux, 0));
    }
    if (int rc = stage_range(c, a, 0, lo)) return rc;
    if (int rc = stage_range(c, a, hi, nc)) return rc;
    if (fork) PH_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    return PH_OK;
}

} // namespace

extern "C" {

const char* ph_last_error(void) { return g_err.c_str(); }

// ph_ctx_create (nz = 0: the whole mesh in mesh->cell_order) and ph_ctx_create_slab
static int create_context(const ph_mesh_desc* mesh, const ph_params* prm, void* cuda_stream, int z0, int nz,
                          ph_ctx** out) {
    if (!mesh || !prm || !out) return fail(PH_ERR_INVALID, "null argument");
    *out = nullptr;
    if (int rc = check_mesh(mesh)) return rc;
    if (int rc = check_param_ranges(prm)) return rc;
    const bool gl = uncollocated(prm);
    if (const char* why = boundary_reason(mesh, prm)) return fail(PH_ERR_UNSUPPORTED, why);
    if (const char* why = gl ? uncollocated_reason(mesh, prm) : unsupported_reason(mesh, prm))
        return fail(PH_ERR_UNSUPPORTED, why);
    const bool ec = prm->conv_num_flux >= 3;
    if (ec && !prm->use_split_form)
        return fail(PH_ERR_INVALID, "two point flux and not using split form are not compatible");   // numerical_flux_factory.cpp
    if (prm->use_relaxation_runge_kutta) {
        // ode_solver_factory.cpp:343-369: Euler / Navier-Stokes take the root-finding form, KG has no
        // assigned numerical entropy
        if (prm->two_point_num_flux_type == ph::TP_KG)
            return fail(PH_ERR_UNSUPPORTED, "relaxation RK: the KG two-point flux has no numerical entropy");
        if (prm->runge_kutta_method >= 7) return fail(PH_ERR_UNSUPPORTED, "relaxation RK: the Butcher methods");
        if (prm->precision != PH_FP64) return fail(PH_ERR_UNSUPPORTED, "relaxation RK: the FP64 path");
        if (is_curvilinear(mesh) && prm->flux_reconstruction != 0)
            return fail(PH_ERR_UNSUPPORTED, "relaxation RK on curvilinear meshes takes cDG");
        if (!(prm->relaxation_runge_kutta_root_tolerance > 0.0))
            return fail(PH_ERR_INVALID, "relaxation_runge_kutta_root_tolerance must be positive");
    }
    if (prm->bound_preserving_limiter < 0 || prm->bound_preserving_limiter > 3)
        return fail(PH_ERR_INVALID, "bound_preserving_limiter out of range");
    if (prm->bound_preserving_limiter == 1)
        return fail(PH_ERR_UNSUPPORTED, "the maximum-principle limiter applies to scalar equations, not Euler / Navier-Stokes");
    if (prm->bound_preserving_limiter >= 2) {
        if (prm->runge_kutta_method > 3 || prm->use_relaxation_runge_kutta)
            return fail(PH_ERR_UNSUPPORTED, "the positivity-preserving limiter: Butcher RK methods without relaxation");
        if (!(prm->min_density > 0.0)) return fail(PH_ERR_INVALID, "min_density must be positive");
        if (is_curvilinear(mesh)) return fail(PH_ERR_UNSUPPORTED, "the positivity-preserving limiter: affine meshes");
    }
    const bool slab = nz > 0;
    if (slab) {
        if (z0 < 0 || z0 >= mesh->n_cells_per_direction || nz > mesh->n_cells_per_direction)
            return fail(PH_ERR_INVALID, "slab outside the mesh: 0 <= z_first < n and 1 <= z_count <= n");
    }
    ph_ctx* c = new ph_ctx();
    c->prm = *prm;
    c->n = mesh->n_cells_per_direction;
    c->slab = slab;
    c->layer = c->n * c->n;
    c->z_first = slab ? z0 : 0;
    c->z_count = slab ? nz : c->n;
    c->nc = c->z_count * c->layer;
    c->nc_ghost = slab ? 2 * c->layer : 0;
    c->p = prm->poly_degree;
    c->N1 = c->p + 1;
    c->NP = c->N1 * c->N1 * c->N1;
    c->left = mesh->left; c->right = mesh->right;
    c->h = (mesh->right - mesh->left) / c->n;
    c->stream = (cudaStream_t)cuda_stream;
    c->visc = prm->pde_type == 1;
    c->split = prm->use_split_form != 0;
    c->fp32 = prm->precision == PH_FP32_RESIDUAL;
    c->ndofs = (size_t)c->nc * 5 * c->NP;
    c->nalloc = (size_t)(c->nc + c->nc_ghost) * 5 * c->NP;
    c->warp = mesh->warp;
    c->curv = is_curvilinear(mesh);
    cudaGetDevice(&c->device);

    // ---- 1-D operators, integral tables, physics, RK tableau, connectivity, geometry
    std::vector<double> x, D;
    if (int rc = build_operators(prm, c->h_ops, c->fr, x, D)) { delete c; return rc; }
    c->gl = gl;
    if (gl) {
        c->NQ = c->N1 + prm->overintegration;
        if (int rc = build_gl_operators(prm, c->h_gl, c->h_ops)) { delete c; return rc; }
    }
    ph::IntegralTab itab;
    build_integral_table(x, c->p, itab);
    c->pc = physics_constants(prm, c->h, c->pen);
    if (low_storage_tableau(prm->runge_kutta_method, c->ls)) {
        c->lowstorage = true;
        c->ns = c->ls.ns;
    } else {
        rk_tableau(prm->runge_kutta_method, c->ns, c->A, c->b);
    }
    std::vector<int> nbr, btype;
    if (slab) slab_connectivity(c->n, c->z_first, c->z_count, c->ijk, nbr);
    else periodic_connectivity(c->n, mesh->cell_order, c->ijk, nbr);
    if (has_boundaries(mesh)) apply_boundaries(c->n, c->ijk, mesh->boundary_type, nbr, btype);
    c->nb = (int)btype.size();
    std::vector<double> metric;
    if (int rc = node_geometry(c->n, c->ijk, x, D, c->left, c->right, c->warp, c->xyz, metric,
                               mesh->mapping_support_points)) { delete c; return rc; }

    // ---- device buffers
    const size_t N = c->ndofs;
    int bad = 0;
    bad |= dalloc(&c->d_nbr, nbr.size());
    bad |= dalloc(&c->d_ops, 1);
    bad |= dalloc(&c->d_itab, 1);
    bad |= dalloc(&c->d_sol, c->nalloc);
    bad |= dalloc(&c->d_stA, c->nalloc);
    bad |= dalloc(&c->d_stB, c->nalloc);
    bad |= dalloc(&c->d_acc, N);
    if (c->ns == 3 || (c->lowstorage && c->ls.plus)) bad |= dalloc(&c->d_carry, N);   // SSPRK3 carry / 3S*+ S4
    if (c->lowstorage) bad |= dalloc(&c->d_err, (size_t)c->nc);
    c->rrk = prm->use_relaxation_runge_kutta != 0;
    if (c->rrk) {
        c->ent_tiles = c->nc;   // at most one tile per cell
        bad |= dalloc(&c->d_ent, (size_t)c->ns * c->ent_tiles);
        bad |= dalloc(&c->d_ent_cell, (size_t)c->nc);
    }
    if (c->visc) {   // viscous terms, stored in the arithmetic type (floats in the precision form)
        const size_t vt = (size_t)(c->nc + c->nc_ghost) * (4 * c->NP + 24 * c->N1 * c->N1);
        bad |= dalloc(&c->d_fv, c->fp32 ? (vt + 1) / 2 : vt);
    }
    if (c->fp32) bad |= dalloc(&c->d_comp, N);
    bad |= dalloc(&c->d_partial, (size_t)ph::integral_partials<true>() * c->nc);
    bad |= dalloc(&c->d_status, 1);
    if (c->nc_ghost) {   // per side: the face state (5 NF doubles) or viscous block (4 NF values) per layer cell
        const int NF = c->N1 * c->N1;
        c->halo_state_bytes = (size_t)c->layer * 5 * NF * sizeof(double);
        c->halo_visc_bytes = c->visc ? (size_t)c->layer * 4 * NF * (c->fp32 ? sizeof(float) : sizeof(double)) : 0;
        if (gl) {   // the face blocks of the face-value buffer, and four rows of the viscous one
            const int NQF = (c->N1 + prm->overintegration) * (c->N1 + prm->overintegration);
            c->halo_state_bytes = (size_t)c->layer * (c->split ? 10 : 5) * NQF * sizeof(double);
            c->halo_visc_bytes = c->visc ? (size_t)c->layer * 4 * NQF * sizeof(double) : 0;
        }
        c->halo_stride = (std::max(c->halo_state_bytes, c->halo_visc_bytes) + 255) / 256 * 256;
        bad |= dalloc(&c->d_halo, 4 * c->halo_stride);
    }
    c->limiter = prm->bound_preserving_limiter;
    if (c->limiter) bad |= dalloc(&c->d_ltab, 1);
    std::vector<int> tiles;
    if (c->nb) {   // the stage / auxiliary tiles without a boundary face first, then those with one
        const int tc = cells_per_tile(c);
        std::vector<int> tb;
        for (int t0 = 0; t0 < c->nc; t0 += tc) {
            bool b = false;
            for (int cc = t0; cc < std::min(c->nc, t0 + tc); ++cc)
                for (int f = 0; f < 6; ++f) b = b || nbr[6 * (size_t)cc + f] < 0;
            (b ? tb : tiles).push_back(t0);
        }
        c->nt_int = (int)tiles.size();
        c->nt_bnd = (int)tb.size();
        tiles.insert(tiles.end(), tb.begin(), tb.end());
        c->h_tiles = tiles;
        bad |= dalloc(&c->d_tiles, tiles.size());
    }
    if (c->nb) {   // boundary faces: their types, and (Navier-Stokes) their viscous fluxes in the arithmetic type
        bad |= dalloc(&c->d_btype, (size_t)c->nb);
        if (c->visc) {   // per boundary face 4 values at each face flux node
            const int nf = gl ? c->NQ * c->NQ : c->N1 * c->N1;
            const size_t fb = (size_t)c->nb * 4 * nf;
            bad |= dalloc(&c->d_fb, c->fp32 ? (fb + 1) / 2 : fb);
        }
    }
    if (gl) {   // (slabs: the ghost cells' face blocks too, filled by the exchange)
        const size_t faces = (size_t)(c->nc + c->nc_ghost) * 6 * c->NQ * c->NQ;
        bad |= dalloc(&c->d_gl, 1);
        bad |= dalloc(&c->d_t1, faces * (c->split ? 10 : 5));
        if (c->visc) {
            bad |= dalloc(&c->d_t2, faces * ph::GL_T2W);
            bad |= dalloc(&c->d_vis, (size_t)c->nc * 4 * c->NP);
        }
        if (c->curv) {
            const size_t q3 = (size_t)c->NQ * c->NQ * c->NQ;
            bad |= dalloc(&c->d_glvm, (size_t)c->nc * 10 * q3);
            bad |= dalloc(&c->d_glfn, (size_t)c->nc * 6 * 3 * c->NQ * c->NQ);
        }
    }
    if (c->curv) bad |= dalloc(&c->d_metric, metric.size());
    if (c->curv) bad |= dalloc(&c->d_xnode, (size_t)3 * c->nc * c->NP);
    else bad |= dalloc(&c->d_origin, (size_t)3 * c->nc);
    if (bad) { ph_ctx_destroy(c); return fail(PH_ERR_NOMEM, "device allocation failed"); }
    cudaError_t e = cudaSuccess;
    e = cudaMemcpy(c->d_nbr, nbr.data(), nbr.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && c->nb)
        e = cudaMemcpy(c->d_btype, btype.data(), btype.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && c->nb)
        e = cudaMemcpy(c->d_tiles, tiles.data(), tiles.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_ops, &c->h_ops, sizeof(ph::OpTab), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_itab, &itab, sizeof(ph::IntegralTab), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && c->d_gl) e = cudaMemcpy(c->d_gl, &c->h_gl, sizeof(ph::GlTab), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && c->d_glvm) {   // metric terms at the uncollocated flux nodes, cell by cell
        const int nq = c->NQ, nq3 = nq * nq * nq, nf = nq * nq, NP = c->NP;
        std::vector<double> xq, wq;
        if (prm->flux_nodes_type == 1) gll(nq, xq, wq); else gauss(nq, xq, wq);
        std::vector<double> vm((size_t)c->nc * 10 * nq3), fnm((size_t)c->nc * 18 * nf);
        std::atomic<int> ok{1};
        const unsigned nthr = std::max(1u, std::min(32u, std::min(std::thread::hardware_concurrency(), (unsigned)c->nc)));
        std::vector<std::thread> pool;
        for (unsigned tI = 0; tI < nthr; ++tI)
            pool.emplace_back([&, tI]() {
                std::vector<double> X((size_t)3 * NP);
                for (int cc = (int)tI; cc < c->nc; cc += (int)nthr) {
                    for (int node = 0; node < NP; ++node)
                        for (int d = 0; d < 3; ++d) X[(size_t)d * NP + node] = c->xyz[((size_t)cc * NP + node) * 3 + d];
                    if (!gl_curvilinear_cell(x, xq, X.data(), &vm[(size_t)cc * 10 * nq3], &fnm[(size_t)cc * 18 * nf]))
                        ok = 0;
                }
            });
        for (auto& th : pool) th.join();
        if (!ok) { ph_ctx_destroy(c); return fail(PH_ERR_INVALID, "non-positive det J at a flux node: the warp folds a cell"); }
        e = cudaMemcpy(c->d_glvm, vm.data(), vm.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(c->d_glfn, fnm.data(), fnm.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && c->d_ltab) {   // the FE_DGQ basis at the Gauss and Gauss-Lobatto points of p + 1
        ph::LimiterTab lt;
        std::memset(&lt, 0, sizeof(lt));
        std::vector<double> xg, wg, xl, wl, v(c->N1), dv(c->N1);
        gauss(c->N1, xg, wg);
        gll(c->N1, xl, wl);
        for (int q = 0; q < c->N1; ++q) {
            lagrange(x, xg[q], v.data(), dv.data());
            for (int i = 0; i < c->N1; ++i) lt.Bgl[q * c->N1 + i] = v[i];
            lagrange(x, xl[q], v.data(), dv.data());
            for (int i = 0; i < c->N1; ++i) lt.Bgll[q * c->N1 + i] = v[i];
            lt.wgl[q] = wg[q];
            lt.wgll[q] = wl[q];
        }
        e = cudaMemcpy(c->d_ltab, &lt, sizeof(lt), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(c->d_status, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(c->d_sol, 0, c->nalloc * sizeof(double));
    if (e == cudaSuccess && c->d_comp) e = cudaMemset(c->d_comp, 0, N * sizeof(double));
    if (e == cudaSuccess && c->d_metric)
        e = cudaMemcpy(c->d_metric, metric.data(), metric.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && c->d_xnode) {
        std::vector<double> xn((size_t)3 * c->nc * c->NP);
        for (int cc = 0; cc < c->nc; ++cc)
            for (int d = 0; d < 3; ++d)
                for (int node = 0; node < c->NP; ++node)
                    xn[((size_t)cc * 3 + d) * c->NP + node] = c->xyz[((size_t)cc * c->NP + node) * 3 + d];
        e = cudaMemcpy(c->d_xnode, xn.data(), xn.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && c->d_origin) {   // node 0 sits at the cell's lower corner
        std::vector<double> o((size_t)3 * c->nc);
        for (int cc = 0; cc < c->nc; ++cc)
            for (int d = 0; d < 3; ++d) o[(size_t)cc * 3 + d] = c->xyz[(size_t)cc * c->NP * 3 + d];
        e = cudaMemcpy(c->d_origin, o.data(), o.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) { ph_ctx_destroy(c); return fail(PH_ERR_CUDA, cudaGetErrorString(e)); }
    c->h_partial.resize((size_t)ph::integral_partials<true>() * c->nc);
    {   // stage tiles that read ghost data: the first and last layer, rounded out to whole tiles
        int threads = 0, cpc = 1;
        size_t smem = 0;
        switch (c->N1) {
        case 2: ph::stage_launch_shape<2>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
        case 3: ph::stage_launch_shape<3>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
        case 4: ph::stage_launch_shape<4>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
        case 5: ph::stage_launch_shape<5>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
        case 6: ph::stage_launch_shape<6>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
        default: ph::stage_launch_shape<7>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
        }
        c->lo_end = (c->layer + cpc - 1) / cpc * cpc;
        c->hi_begin = (c->nc - c->layer) / cpc * cpc;
        if (c->lo_end >= c->hi_begin) c->lo_end = c->hi_begin = c->nc;   // no cell is free of ghost data
    }
    if (c->nc_ghost) {
        cudaError_t se = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking);
        if (se == cudaSuccess) se = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
        if (se == cudaSuccess) se = cudaEventCreateWithFlags(&c->ev_aux, cudaEventDisableTiming);
        if (se == cudaSuccess) se = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
        if (se != cudaSuccess) { ph_ctx_destroy(c); return fail(PH_ERR_CUDA, cudaGetErrorString(se)); }
    }
    *out = c;
    return PH_OK;
}

int ph_ctx_create(const ph_mesh_desc* mesh, const ph_params* prm, void* cuda_stream, ph_ctx** out) {
    return create_context(mesh, prm, cuda_stream, 0, 0, out);
}

int ph_ctx_create_slab(const ph_mesh_desc* mesh, const ph_params* prm, int z_first, int z_count, void* cuda_stream,
                       ph_ctx** out) {
    if (z_count < 1) return fail(PH_ERR_INVALID, "slab outside the mesh: 0 <= z_first < n and 1 <= z_count <= n");
    return create_context(mesh, prm, cuda_stream, z_first, z_count, out);
}

int ph_set_halo_exchange(ph_ctx* c, ph_halo_fn fn, void* user) {
    if (!c) return fail(PH_ERR_INVALID, "null argument");
    c->halo_fn = fn;
    c->halo_user = user;
    return PH_OK;
}

int ph_set_rank_sum(ph_ctx* c, ph_rank_sum_fn fn, void* user) {
    if (!c) return fail(PH_ERR_INVALID, "null argument");
    c->sum_fn = fn;
    c->sum_user = user;
    return PH_OK;
}

int ph_slab_connectivity(int n, int z_first, int z_count, int32_t* ijk, int32_t* nbr) {
    if (n < 1 || z_first < 0 || z_first >= n || z_count < 1 || z_count > n || !ijk || !nbr)
        return fail(PH_ERR_INVALID, "bad slab");
    std::vector<int> h_ijk, h_nbr;
    slab_connectivity(n, z_first, z_count, h_ijk, h_nbr);
    std::memcpy(ijk, h_ijk.data(), h_ijk.size() * sizeof(int32_t));
    std::memcpy(nbr, h_nbr.data(), (size_t)6 * z_count * n * n * sizeof(int32_t));
    return PH_OK;
}

int ph_ctx_destroy(ph_ctx* c) {
    if (!c) return PH_OK;
    if (c->step_graph || c->run_graph) {
        if (c->stream) cudaStreamSynchronize(c->stream);
        drop_step_graph(c);
        if (c->run_graph) cudaGraphExecDestroy(c->run_graph);
    }
    for (cudaEvent_t ev : c->tcap) if (ev) cudaEventDestroy(ev);
    if (c->tfork) cudaEventDestroy(c->tfork);
    if (c->tside) cudaStreamDestroy(c->tside);
    for (auto& set : c->tpool) for (cudaEvent_t ev : set) if (ev) cudaEventDestroy(ev);
    void* ptrs[] = {c->d_nbr, c->d_ops, c->d_itab, c->d_sol, c->d_stA, c->d_stB, c->d_acc, c->d_carry,
                    c->d_fv, c->d_comp, c->d_tmpA, c->d_tmpB, c->d_partial, c->d_status, c->d_metric, c->d_xnode, c->d_origin, c->d_err,
                    c->d_table, c->d_counter, c->d_ent, c->d_ent_cell, c->d_halo, c->d_gl, c->d_t1, c->d_t2,
                    c->d_vis, c->d_ltab, c->d_glvm, c->d_glfn, c->d_btype, c->d_fb, c->d_tiles};
    if (c->side) cudaStreamSynchronize(c->side);
    for (void* p : ptrs) if (p) cudaFree(p);
    if (c->side) cudaStreamDestroy(c->side);
    for (cudaEvent_t ev : {c->ev_fork, c->ev_aux, c->ev_join}) if (ev) cudaEventDestroy(ev);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    delete c;
    return PH_OK;
}

int64_t ph_ndofs(const ph_ctx* c) { return c ? (int64_t)c->ndofs : -1; }

}  // extern "C"

int ph_host::ctx_state(ph_ctx* c, const double** d, size_t* n, cudaStream_t* stream) {
    if (!c) return fail(PH_ERR_INVALID, "null argument");
    *d = c->d_sol; *n = c->ndofs; *stream = c->stream;
    return PH_OK;
}

extern "C" {

int ph_node_xyz(const ph_ctx* c, double* xyz) {
    if (!c || !xyz) return fail(PH_ERR_INVALID, "null argument");
    std::memcpy(xyz, c->xyz.data(), c->xyz.size() * sizeof(double));
    return PH_OK;
}

int ph_cell_ijk(const ph_ctx* c, int32_t* ijk) {
    if (!c || !ijk) return fail(PH_ERR_INVALID, "null argument");
    std::memcpy(ijk, c->ijk.data(), c->ijk.size() * sizeof(int32_t));
    return PH_OK;
}

int ph_set_state(ph_ctx* c, const double* U, int where) {
    if (!c || !U) return fail(PH_ERR_INVALID, "null argument");
    PH_CUDA(cudaMemcpyAsync(c->d_sol, U, c->ndofs * sizeof(double),
                            where == PH_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c->stream));
    if (c->d_comp) PH_CUDA(cudaMemsetAsync(c->d_comp, 0, c->ndofs * sizeof(double), c->stream));
    if (where == PH_HOST) PH_CUDA(cudaStreamSynchronize(c->stream));
    return PH_OK;
}

int ph_get_state(ph_ctx* c, double* U, int where) {
    if (!c || !U) return fail(PH_ERR_INVALID, "null argument");
    PH_CUDA(cudaMemcpyAsync(U, c->d_sol, c->ndofs * sizeof(double),
                            where == PH_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, c->stream));
    if (where == PH_HOST) PH_CUDA(cudaStreamSynchronize(c->stream));
    return PH_OK;
}

static int ensure_tmp(ph_ctx* c) {
    if (!c->d_tmpA && dalloc(&c->d_tmpA, c->nalloc)) return fail(PH_ERR_NOMEM, "device allocation failed");
    if (!c->d_tmpB && dalloc(&c->d_tmpB, c->nalloc)) return fail(PH_ERR_NOMEM, "device allocation failed");
    return PH_OK;
}

int ph_residual(ph_ctx* c, const double* U, double* R, int where) {
    if (!c || !U || !R) return fail(PH_ERR_INVALID, "null argument");
    NvtxRange nvtx("ph_residual");
    const double* dU = U;
    double* dR = R;
    if (where == PH_HOST) {
        if (int rc = ensure_tmp(c)) return rc;
        PH_CUDA(cudaMemcpyAsync(c->d_tmpA, U, c->ndofs * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        dU = c->d_tmpA; dR = c->d_tmpB;
    } else if (c->nc_ghost) {   // the ghost layers need room after the owned cells
        if (int rc = ensure_tmp(c)) return rc;
        PH_CUDA(cudaMemcpyAsync(c->d_tmpA, U, c->ndofs * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        dU = c->d_tmpA;
    }
    ph::StageArgs a = base_args(c, dU);
    a.mode = 0; a.out = dR;
    if (int rc = eval_residual(c, dU, a)) return rc;
    if (where == PH_HOST) {
        PH_CUDA(cudaMemcpyAsync(R, dR, c->ndofs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        PH_CUDA(cudaStreamSynchronize(c->stream));
    }
    return PH_OK;
}

int ph_apply_inverse_mass(ph_ctx* c, const double* R, double* out, int where) {
    if (!c || !R || !out) return fail(PH_ERR_INVALID, "null argument");
    const double* dR = R;
    double* dO = out;
    if (where == PH_HOST) {
        if (int rc = ensure_tmp(c)) return rc;
        PH_CUDA(cudaMemcpyAsync(c->d_tmpA, R, c->ndofs * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        dR = c->d_tmpA; dO = c->d_tmpB;
    }
    if (c->gl && c->curv) {   // the weight-adjusted inverse mass at the uncollocated flux nodes
        ph::StageArgs a = base_args(c, dR);
        a.out = dO;
        a.cell_begin = 0;
        a.nc = c->nc;
        if (int rc = dispatch_gl(c, 3, a)) return rc;
        if (where == PH_HOST) {
            PH_CUDA(cudaMemcpyAsync(out, dO, c->ndofs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            PH_CUDA(cudaStreamSynchronize(c->stream));
        }
        return PH_OK;
    }
    const double inv_detj = 1.0 / (c->h * c->h * c->h);
    cudaError_t e;
    switch (c->N1) {
    case 2: e = ph::launch_inverse_mass<2>(dR, dO, c->d_ops, c->nc, inv_detj, c->d_metric, c->fr ? 1 : 0, c->stream); break;
    case 3: e = ph::launch_inverse_mass<3>(dR, dO, c->d_ops, c->nc, inv_detj, c->d_metric, c->fr ? 1 : 0, c->stream); break;
    case 4: e = ph::launch_inverse_mass<4>(dR, dO, c->d_ops, c->nc, inv_detj, c->d_metric, c->fr ? 1 : 0, c->stream); break;
    case 5: e = ph::launch_inverse_mass<5>(dR, dO, c->d_ops, c->nc, inv_detj, c->d_metric, c->fr ? 1 : 0, c->stream); break;
    case 6: e = ph::launch_inverse_mass<6>(dR, dO, c->d_ops, c->nc, inv_detj, c->d_metric, c->fr ? 1 : 0, c->stream); break;
    case 7: e = ph::launch_inverse_mass<7>(dR, dO, c->d_ops, c->nc, inv_detj, c->d_metric, c->fr ? 1 : 0, c->stream); break;
    default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree");
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, cudaGetErrorString(e));
    if (where == PH_HOST) {
        PH_CUDA(cudaMemcpyAsync(out, dO, c->ndofs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        PH_CUDA(cudaStreamSynchronize(c->stream));
    }
    return PH_OK;
}

// One explicit Butcher step (RungeKuttaBase::step_in_time, runge_kutta_base.cpp:21-39):
// stage i reads its stage state, computes k_i = M^{-1} R and, in the same kernel,
// updates the running sum and writes the next stage state.
static int rk_one_step(ph_ctx* c, double dt) {
    static const char* const kStage[] = {"RK stage 0", "RK stage 1", "RK stage 2", "RK stage 3", "RK stage 4",
                                         "RK stage 5", "RK stage 6", "RK stage 7", "RK stage 8", "RK stage 9",
                                         "RK stage 10"};
    NvtxRange nvtx("RK step");
    const int ns = c->ns;
    const RkBuffers B{c->d_sol, c->d_stA, c->d_stB, c->d_acc, c->d_carry, c->d_comp};
    if (c->lowstorage) {   // LowStorageRungeKuttaODESolver: ns stages (+ the FSAL evaluation of 3S*+)
        const int last = c->ls.plus ? ns : ns - 1;
        for (int i = 0; i <= last; ++i) {
            NvtxRange stage(kStage[i < 10 ? i : 10]);
            ph::StageArgs a = base_args(c, nullptr);
            const double* in = lsrk_stage_args(a, B, i, c->ls, dt, c->prm.rk_atol, c->prm.rk_rtol, c->d_err);
            if (int rc = eval_residual(c, in, a)) return rc;
        }
        return PH_OK;
    }
    for (int i = 0; i < ns; ++i) {
        NvtxRange stage(kStage[i]);
        const double* in = rk_stage_input(B, i);
        if (c->limiter && i == 0) {
            // RungeKuttaBase::step_in_time limits every stage solution before its derivative
            // (runge_kutta_base.cpp:24-28): stage 0's is u_n, limited in a copy (stB is free
            // during stage 0) so that the step's sum still starts from u_n itself
            PH_CUDA(cudaMemcpyAsync(c->d_stB, c->d_sol, c->ndofs * sizeof(double), cudaMemcpyDeviceToDevice,
                                    c->stream));
            if (int rc = dispatch_limiter(c, c->d_stB, dt)) return rc;
            in = c->d_stB;
        }
        ph::StageArgs a = base_args(c, in);
        rk_stage_args(a, B, i, ns, c->A, c->b, dt, c->fp32);
        if (int rc = eval_residual(c, in, a)) return rc;
        if (c->limiter) {   // the next stage's solution, or the new solution (runge_kutta_base.cpp:34)
            double* out = (i == ns - 1) ? a.final_out : a.next;
            if (int rc = dispatch_limiter(c, out, dt)) return rc;
        }
    }
    if (ns == 1) std::swap(c->d_sol, c->d_stA);
    return PH_OK;
}

// tiles (CTAs) of one stage-kernel launch
static int stage_tiles(const ph_ctx* c) {
    if (c->gl) return c->nc;   // the uncollocated kernels: one cell per CTA
    int threads = 0, cpc = 1;
    size_t smem = 0;
    switch (c->N1) {
    case 2: ph::stage_launch_shape<2>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    case 3: ph::stage_launch_shape<3>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    case 4: ph::stage_launch_shape<4>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    case 5: ph::stage_launch_shape<5>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    case 6: ph::stage_launch_shape<6>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    default: ph::stage_launch_shape<7>(c->fp32, c->visc, c->split, &threads, &cpc, &smem); break;
    }
    return (c->nc + cpc - 1) / cpc;
}

static __global__ void rrk_apply_kernel(double* __restrict__ sol, const double* __restrict__ u1, double g, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        sol[i] = sol[i] + g * (u1[i] - sol[i]);
}

// Integrated numerical entropy of u_n + g (u1 - u_n): per-cell partials on the device,
// summed on the host in cell order (the same value on every run).
static int rrk_entropy(ph_ctx* c, const double* u1, double g, double* out) {
    const double h3 = c->h * c->h * c->h;
    const double* metric = c->curv ? c->d_metric : nullptr;
    cudaError_t e;
    if (c->gl) {   // at the flux nodes
        const double* vm = c->curv ? c->d_glvm : nullptr;
        switch (c->N1) {
#define PH_RRK_GL_CASE(n) \
        case n: e = ph::launch_gl_rrk_entropy<n>(c->NQ, c->d_sol, u1, g, c->h_gl, c->nc, h3, vm, c->prm.gamma_gas, \
                                                 c->d_ent_cell, c->stream); break;
        PH_RRK_GL_CASE(2) PH_RRK_GL_CASE(3) PH_RRK_GL_CASE(4) PH_RRK_GL_CASE(5) PH_RRK_GL_CASE(6) PH_RRK_GL_CASE(7)
#undef PH_RRK_GL_CASE
        default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree");
        }
    } else {       // at the solution nodes
        switch (c->N1) {
#define PH_RRK_CASE(n) \
        case n: e = ph::launch_rrk_entropy<n>(c->d_sol, u1, g, c->d_ops, c->nc, h3, metric, c->prm.gamma_gas, \
                                              c->d_ent_cell, c->stream); break;
        PH_RRK_CASE(2) PH_RRK_CASE(3) PH_RRK_CASE(4) PH_RRK_CASE(5) PH_RRK_CASE(6) PH_RRK_CASE(7)
#undef PH_RRK_CASE
        default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree");
        }
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, cudaGetErrorString(e));
    ++c->launches;
    c->h_ent.resize((size_t)c->nc);
    PH_CUDA(cudaMemcpyAsync(c->h_ent.data(), c->d_ent_cell, c->nc * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PH_CUDA(cudaStreamSynchronize(c->stream));
    double sum = 0.0;
    for (int i = 0; i < c->nc; ++i) sum += c->h_ent[i];
    if (int rc = rank_sum(c, &sum, 1)) return rc;   // a slab's share -> the mesh's
    *out = sum;
    return PH_OK;
}

// One relaxation-RK step (RungeKuttaBase::step_in_time with RootFindingRRKODESolver,
// runge_kutta_base.cpp:21-39, root_finding_rrk_ode_solver.cpp:15-180): the stages as
// rk_one_step takes them, with v(u_i)^T M k_i reduced in each stage's epilogue and the last
// stage's u_n + dt sum b_i k_i written beside u_n; the relaxation parameter gamma is the root of
// eta(u_n + gamma d) - eta(u_n) - gamma dt sum_i b_i v_i^T M k_i (secant from the previous
// gamma, the reference's safeguards, bisection as the fallback), and u_{n+1} = u_n + gamma d.
static int rrk_one_step(ph_ctx* c, double dt) {
    const int ns = c->ns;
    const RkBuffers B{c->d_sol, c->d_stA, c->d_stB, c->d_acc, c->d_carry, c->d_comp};
    // the last stage reads stA (ns even) or stB (ns odd, > 1); its output goes to the other one
    double* u1 = (ns == 1) ? B.stA : ((ns - 2) % 2 == 0 ? B.stB : B.stA);
    const int tiles = stage_tiles(c);
    for (int i = 0; i < ns; ++i) {
        const double* in = rk_stage_input(B, i);
        ph::StageArgs a = base_args(c, in);
        rk_stage_args(a, B, i, ns, c->A, c->b, dt, c->fp32);
        if (i == ns - 1) a.final_out = u1;
        a.ent_partial = c->d_ent + (size_t)i * c->ent_tiles;
        if (int rc = eval_residual(c, in, a)) return rc;
    }
    std::vector<double> part((size_t)ns * c->ent_tiles);
    PH_CUDA(cudaMemcpyAsync(part.data(), c->d_ent, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PH_CUDA(cudaStreamSynchronize(c->stream));
    double si[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < ns; ++i)
        for (int t = 0; t < tiles; ++t) si[i] += part[(size_t)i * c->ent_tiles + t];
    if (int rc = rank_sum(c, si, ns)) return rc;
    double est = 0.0;
    for (int i = 0; i < ns; ++i) est += c->b[i] * si[i];
    est *= dt;
    double eta_n = 0.0;
    if (int rc = rrk_entropy(c, u1, 0.0, &eta_n)) return rc;
    int rc = PH_OK;
    auto root = [&](double g) {
        double eta = 0.0;
        if (!rc) rc = rrk_entropy(c, u1, g, &eta);
        return eta - eta_n - g * est;
    };
    const double tol = c->prm.relaxation_runge_kutta_root_tolerance;
    const int iter_limit = 100;
    int iter = 0;
    double g_kp1 = 0.0;
    bool secant_failed = false;
    {
        double residual = 1.0;
        double g_k = c->rrk_gamma + 1e-5, g_km1 = c->rrk_gamma - 1e-5;
        double r_k = root(g_k), r_km1 = root(g_km1);
        while (residual > tol && iter < iter_limit && !rc) {
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
    if (secant_failed && !rc) {
        iter = 0;
        double lo = c->rrk_gamma - 0.1, hi = c->rrk_gamma + 0.1;
        double r_lo = root(lo), r_hi = root(hi), residual = 1.0;
        while (residual > tol && iter < iter_limit && !rc) {
            if (r_lo * r_hi > 0) { lo -= 0.1; hi += 0.1; }
            g_kp1 = 0.5 * (lo + hi);
            const double r = root(g_kp1);
            if (r < 0) { lo = g_kp1; r_lo = r; } else { hi = g_kp1; r_hi = r; }
            residual = hi - lo;
            ++iter;
        }
        if (iter == iter_limit && !rc) return fail(PH_ERR_INVALID, "relaxation RK: root finding did not converge");
    }
    if (rc) return rc;
    if (!(g_kp1 >= 0.5)) return fail(PH_ERR_INVALID, "relaxation RK: no reasonable relaxation parameter (< 0.5)");
    rrk_apply_kernel<<<1184, 256, 0, c->stream>>>(c->d_sol, u1, g_kp1, c->ndofs);
    PH_CUDA(cudaGetLastError());
    ++c->launches;
    c->rrk_gamma = g_kp1;
    c->rrk_elapsed += g_kp1 * dt;
    return PH_OK;
}

// Capture one RK step (all stages, auxiliary kernels included) as a graph for this dt.
// Timing mode 2: the event-record nodes of the captured step, in kernel order (matched to the
// capture events they record).
static int find_timing_nodes(ph_ctx* c, cudaGraph_t g) {
    size_t n = 0;
    PH_CUDA(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    PH_CUDA(cudaGraphGetNodes(g, nodes.data(), &n));
    c->tnodes.assign(c->tcls.size() + 1, nullptr);
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        PH_CUDA(cudaGraphNodeGetType(node, &type));
        if (type != cudaGraphNodeTypeEventRecord) continue;
        cudaEvent_t ev = nullptr;
        PH_CUDA(cudaGraphEventRecordNodeGetEvent(node, &ev));
        for (size_t j = 0; j < c->tnodes.size(); ++j)
            if (c->tcap[j] == ev) c->tnodes[j] = node;
    }
    for (cudaGraphNode_t node : c->tnodes)
        if (!node) return fail(PH_ERR_CUDA, "step capture: a timing event node is missing");
    return PH_OK;
}

static int capture_step_graph(ph_ctx* c, double dt) {
    drop_step_graph(c);
    const long long before = c->launches;
    cudaGraph_t g = nullptr;
    c->tcls.clear();
    PH_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    c->capturing = true;
    int rc = rk_one_step(c, dt);
    c->capturing = false;
    if (c->timing == 2 && !c->tcls.empty()) {   // join the event branch back before the capture ends
        cudaEventRecord(c->tfork, c->tside);
        cudaStreamWaitEvent(c->stream, c->tfork, 0);
    }
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        c->launches = before;
        return rc ? rc : fail(PH_ERR_CUDA, std::string("step capture: ") + cudaGetErrorString(e));
    }
    if (c->timing == 2) {
        if (int rc2 = find_timing_nodes(c, g)) { cudaGraphDestroy(g); return rc2; }
    }
    const cudaError_t e2 = cudaGraphInstantiate(&c->step_graph, g, 0);
    if (c->timing == 2) c->step_graph_src = g;
    else cudaGraphDestroy(g);
    if (e2 != cudaSuccess) { c->step_graph = nullptr; drop_step_graph(c); return fail(PH_ERR_CUDA, cudaGetErrorString(e2)); }
    c->step_graph_launches = (int)(c->launches - before);
    c->launches = before;
    c->step_graph_dt = dt;
    return PH_OK;
}

int ph_rk_step(ph_ctx* c, double dt, int nsteps) {
    if (!c || nsteps < 0) return fail(PH_ERR_INVALID, "bad argument");
    NvtxRange nvtx("ph_rk_step");
    if (c->rrk) {   // the root finding reads sums back after every step: direct launches
        c->rrk_elapsed = 0.0;
        for (int s = 0; s < nsteps; ++s)
            if (int rc = rrk_one_step(c, dt)) return rc;
        return PH_OK;
    }
    c->rrk_elapsed = dt * nsteps;
    // several steps of one dt on a caller-given stream replay a graph of one step; the
    // per-launch timing mode and one-stage methods (which swap buffers) launch directly
    const bool graph = c->stream != nullptr && c->timing != 1 && c->ns > 1 && nsteps > 1 && !c->nc_ghost;
    if (graph) {
        int s = 0;
        if (!c->step_graph || c->step_graph_dt != dt) {
            // the first step runs directly, so every kernel is configured before the capture
            if (int rc = rk_one_step(c, dt)) return rc;
            s = 1;
            if (int rc = capture_step_graph(c, dt)) return rc;
        }
        for (; s < nsteps; ++s) {
            if (c->timing == 2) {   // this replay records its own events
                if (c->tpool.size() <= c->treplays) {
                    c->tpool.emplace_back(c->tnodes.size(), nullptr);
                    for (cudaEvent_t& ev : c->tpool.back()) PH_CUDA(cudaEventCreate(&ev));
                }
                std::vector<cudaEvent_t>& evs = c->tpool[c->treplays];
                for (size_t j = 0; j < c->tnodes.size(); ++j)
                    PH_CUDA(cudaGraphExecEventRecordNodeSetEvent(c->step_graph, c->tnodes[j], evs[j]));
                ++c->treplays;
            }
            PH_CUDA(cudaGraphLaunch(c->step_graph, c->stream));
            c->launches += c->step_graph_launches;
        }
        return PH_OK;
    }
    for (int s = 0; s < nsteps; ++s)
        if (int rc = rk_one_step(c, dt)) return rc;
    return PH_OK;
}

static int launch_integrals_async(ph_ctx* c, bool full) {
    ph::IntegralConst ic{};
    ic.h = c->h;
    ic.gam = c->prm.gamma_gas; ic.gm1 = ic.gam - 1.0;
    ic.mach2 = c->pc.mach2; ic.temp_ratio = c->pc.temp_ratio;
    ic.const_visc = c->pc.const_visc; ic.use_const_visc = c->pc.use_const_visc;
    cudaError_t e;
    switch (c->N1) {
#define PH_INTEGRALS_CASE(n)                                                                                   \
    case n: e = ph::launch_integrals<n>(c->d_sol, c->d_xnode, c->d_origin, c->d_itab, c->nc, ic, full, c->d_partial, \
                                        c->stream); break;
    PH_INTEGRALS_CASE(2) PH_INTEGRALS_CASE(3) PH_INTEGRALS_CASE(4) PH_INTEGRALS_CASE(5) PH_INTEGRALS_CASE(6)
    PH_INTEGRALS_CASE(7)
#undef PH_INTEGRALS_CASE
    default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree");
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, cudaGetErrorString(e));
    ++c->launches;
    return PH_OK;
}

static int run_integrals(ph_ctx* c, bool full) {
    if (int rc = launch_integrals_async(c, full)) return rc;
    const size_t nq = full ? ph::integral_partials<true>() : ph::integral_partials<false>();
    PH_CUDA(cudaMemcpyAsync(c->h_partial.data(), c->d_partial, nq * c->nc * sizeof(double),
                            cudaMemcpyDeviceToHost, c->stream));
    PH_CUDA(cudaStreamSynchronize(c->stream));
    return PH_OK;
}

int ph_integrals(ph_ctx* c, double out[4]) {
    if (!c || !out) return fail(PH_ERR_INVALID, "null argument");
    if (int rc = run_integrals(c, false)) return rc;
    double ke = 0.0, ens = 0.0, wave = 0.0;
    for (int i = 0; i < c->nc; ++i) {
        ke += c->h_partial[3 * i]; ens += c->h_partial[3 * i + 1];
        wave = std::max(wave, c->h_partial[3 * i + 2]);
    }
    const double vol = std::pow(c->right - c->left, 3);
    out[0] = ke / vol;
    out[1] = ens / vol;
    // zero for inviscid flow (PeriodicTurbulence::get_vorticity_based_dissipation_rate,
    // periodic_turbulence.cpp:717-725)
    out[2] = c->visc ? 2.0 * out[1] / c->prm.reynolds_number_inf : 0.0;
    out[3] = wave;
    return PH_OK;
}

int ph_integrated_quantities(ph_ctx* c, double out[PH_N_INTEGRATED_QUANTITIES]) {
    if (!c || !out) return fail(PH_ERR_INVALID, "null argument");
    if (int rc = run_integrals(c, true)) return rc;
    constexpr int NQ = ph::integral_partials<true>();
    static_assert(NQ == PH_N_INTEGRATED_QUANTITIES + 1, "partials: the quantities then the wave speed");
    double acc[PH_N_INTEGRATED_QUANTITIES] = {0.0};
    for (int i = 0; i < c->nc; ++i)
        for (int q = 0; q < PH_N_INTEGRATED_QUANTITIES; ++q) acc[q] += c->h_partial[(size_t)NQ * i + q];
    const double vol = std::pow(c->right - c->left, 3);
    for (int q = 0; q < PH_N_INTEGRATED_QUANTITIES; ++q) out[q] = acc[q] / vol;
    return PH_OK;
}

// One record interval: record_every RK steps, then the integrals and their row on the device.
static int run_interval(ph_ctx* c, double dt, int record_every) {
    for (int s = 0; s < record_every; ++s)
        if (int rc = rk_one_step(c, dt)) return rc;
    if (int rc = launch_integrals_async(c, false)) return rc;
    const double vol = std::pow(c->right - c->left, 3);
    ph::integrals_row_kernel<<<1, ph::ROW_THREADS, 0, c->stream>>>(
        c->d_partial, c->nc, vol, c->visc ? c->prm.reynolds_number_inf : 0.0, c->d_counter, c->table_rows,
        c->d_table);
    PH_CUDA(cudaGetLastError());
    ++c->launches;
    return PH_OK;
}

static int capture_run_graph(ph_ctx* c, double dt, int record_every) {
    if (c->run_graph) { cudaGraphExecDestroy(c->run_graph); c->run_graph = nullptr; }
    const long long before = c->launches;
    cudaGraph_t g = nullptr;
    PH_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = run_interval(c, dt, record_every);
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        c->launches = before;
        return rc ? rc : fail(PH_ERR_CUDA, std::string("run capture: ") + cudaGetErrorString(e));
    }
    const cudaError_t e2 = cudaGraphInstantiate(&c->run_graph, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) { c->run_graph = nullptr; return fail(PH_ERR_CUDA, cudaGetErrorString(e2)); }
    c->run_graph_launches = (int)(c->launches - before);
    c->launches = before;
    c->run_graph_dt = dt;
    c->run_graph_every = record_every;
    return PH_OK;
}

int ph_rk_relaxation(ph_ctx* c, double* gamma, double* elapsed) {
    if (!c || !gamma || !elapsed) return fail(PH_ERR_INVALID, "null argument");
    *gamma = c->rrk ? c->rrk_gamma : 1.0;
    *elapsed = c->rrk_elapsed;
    return PH_OK;
}

int ph_run(ph_ctx* c, double dt, int nsteps, int record_every, double* rows) {
    if (!c || nsteps < 0 || record_every < 0) return fail(PH_ERR_INVALID, "bad argument");
    if (c->rrk) return fail(PH_ERR_UNSUPPORTED, "ph_run: relaxation RK steps have variable length; use ph_rk_step");
    if (c->nc_ghost) return fail(PH_ERR_UNSUPPORTED, "ph_run: slab contexts exchange halos on the host; use ph_rk_step");
    const int nrec = record_every > 0 ? nsteps / record_every : 0;
    if (nrec > 0 && !rows) return fail(PH_ERR_INVALID, "null rows");
    if (nrec > c->table_rows) {   // grow the device table (synchronises the stream)
        if (c->run_graph) {
            PH_CUDA(cudaStreamSynchronize(c->stream));
            cudaGraphExecDestroy(c->run_graph);
            c->run_graph = nullptr;
        }
        if (c->d_table) cudaFree(c->d_table);
        c->d_table = nullptr;
        c->table_rows = 0;
        if (cudaMalloc(&c->d_table, (size_t)nrec * 4 * sizeof(double)) != cudaSuccess) {
            c->d_table = nullptr;
            return fail(PH_ERR_NOMEM, "integrals table");
        }
        c->table_rows = nrec;
    }
    if (nrec > 0 && !c->d_counter) {
        if (cudaMalloc(&c->d_counter, sizeof(int)) != cudaSuccess) {
            c->d_counter = nullptr;
            return fail(PH_ERR_NOMEM, "row counter");
        }
    }
    if (nrec > 0) PH_CUDA(cudaMemsetAsync(c->d_counter, 0, sizeof(int), c->stream));
    // intervals on a caller-given stream replay a captured graph (the first one runs
    // directly so that every kernel is configured before the capture)
    const bool graph = c->stream != nullptr && c->timing == 0 && c->ns > 1 && nrec > 1;
    int r = 0;
    if (graph) {
        if (!c->run_graph || c->run_graph_dt != dt || c->run_graph_every != record_every) {
            if (int rc = run_interval(c, dt, record_every)) return rc;
            r = 1;
            if (int rc = capture_run_graph(c, dt, record_every)) return rc;
        }
        for (; r < nrec; ++r) {
            PH_CUDA(cudaGraphLaunch(c->run_graph, c->stream));
            c->launches += c->run_graph_launches;
        }
    } else {
        for (; r < nrec; ++r)
            if (int rc = run_interval(c, dt, record_every)) return rc;
    }
    for (int s = nrec * record_every; s < nsteps; ++s)
        if (int rc = rk_one_step(c, dt)) return rc;
    if (nrec > 0) {
        PH_CUDA(cudaMemcpyAsync(rows, c->d_table, (size_t)nrec * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    }
    PH_CUDA(cudaStreamSynchronize(c->stream));
    return PH_OK;
}

int ph_rk_error_norm(ph_ctx* c, double* w) {
    if (!c || !w) return fail(PH_ERR_INVALID, "null argument");
    if (!c->lowstorage) return fail(PH_ERR_INVALID, "the error estimate belongs to the low-storage methods");
    const int tiles = stage_tiles(c);   // one partial per stage-kernel tile
    std::vector<double> part(tiles);
    PH_CUDA(cudaMemcpyAsync(part.data(), c->d_err, tiles * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PH_CUDA(cudaStreamSynchronize(c->stream));
    double sum = 0.0;
    for (double v : part) sum += v;   // tile order: deterministic
    *w = std::sqrt(sum / (double)c->ndofs);
    return PH_OK;
}

int ph_status(ph_ctx* c, uint32_t* flags) {
    if (!c || !flags) return fail(PH_ERR_INVALID, "null argument");
    unsigned v = 0;
    PH_CUDA(cudaMemcpyAsync(&v, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    PH_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
    PH_CUDA(cudaStreamSynchronize(c->stream));
    *flags = v;
    return PH_OK;
}

int ph_kinetic_energy_rate(ph_ctx* c, double* out) {
    if (!c || !out) return fail(PH_ERR_INVALID, "null argument");
    if (c->curv || c->nc_ghost) return fail(PH_ERR_UNSUPPORTED, "ph_kinetic_energy_rate: whole affine meshes");
    if (int rc = ensure_tmp(c)) return rc;
    // K = M^-1 R(u) of the current solution, by the stage kernel's mode 1
    ph::StageArgs a = base_args(c, c->d_sol);
    a.mode = 1; a.out = c->d_tmpB;
    if (int rc = eval_residual(c, c->d_sol, a)) return rc;
    cudaError_t e;
    const double h3 = c->h * c->h * c->h;
    switch (c->N1) {
#define PH_KE_CASE(n) case n: e = ph::launch_ke_rate<n>(c->d_sol, c->d_tmpB, c->d_itab, c->nc, h3, c->d_partial, c->stream); break;
    PH_KE_CASE(2) PH_KE_CASE(3) PH_KE_CASE(4) PH_KE_CASE(5) PH_KE_CASE(6) PH_KE_CASE(7)
#undef PH_KE_CASE
    default: return fail(PH_ERR_UNSUPPORTED, "polynomial degree");
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string("kinetic energy rate: ") + cudaGetErrorString(e));
    ++c->launches;
    PH_CUDA(cudaMemcpyAsync(c->h_partial.data(), c->d_partial, c->nc * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    PH_CUDA(cudaStreamSynchronize(c->stream));
    double sum = 0.0;
    for (int i = 0; i < c->nc; ++i) sum += c->h_partial[i];
    const double L = c->right - c->left;
    *out = sum / (L * L * L);
    return PH_OK;
}

int ph_limit(ph_ctx* c, double dt) {
    if (!c) return fail(PH_ERR_INVALID, "null argument");
    if (!c->limiter) return fail(PH_ERR_INVALID, "the context has no positivity-preserving limiter");
    if (c->nc_ghost) return fail(PH_ERR_UNSUPPORTED, "ph_limit on a slab context");
    if (int rc = dispatch_limiter(c, c->d_sol, dt)) return rc;
    return PH_OK;
}

int ph_set_timing(ph_ctx* c, int enable) {
    if (!c) return fail(PH_ERR_INVALID, "null argument");
    if (enable < 0 || enable > 2) return fail(PH_ERR_INVALID, "timing mode must be 0, 1 or 2");
    if (enable == 1 && !c->ev0) {
        PH_CUDA(cudaEventCreate(&c->ev0));
        PH_CUDA(cudaEventCreate(&c->ev1));
    }
    if (enable == 2 && c->tcap.empty()) {
        c->tcap.assign(TIMED_KERNELS_PER_STEP + 1, nullptr);
        for (cudaEvent_t& ev : c->tcap) PH_CUDA(cudaEventCreate(&ev));
        PH_CUDA(cudaStreamCreateWithFlags(&c->tside, cudaStreamNonBlocking));
        PH_CUDA(cudaEventCreateWithFlags(&c->tfork, cudaEventDisableTiming));
    }
    // a step graph captured in another mode has (or lacks) the timing nodes: capture again
    if ((enable == 2) != (c->timing == 2) && c->step_graph) {
        PH_CUDA(cudaStreamSynchronize(c->stream));
        drop_step_graph(c);
    }
    c->timing = enable;
    for (int i = 0; i < 3; ++i) { c->t_ms[i] = 0.0; c->t_n[i] = 0; }
    c->treplays = 0;
    c->launches = 0;
    return PH_OK;
}

int ph_get_timing(ph_ctx* c, double out[7]) {
    if (!c || !out) return fail(PH_ERR_INVALID, "null argument");
    if (c->timing == 2 && c->treplays) {   // the replays' kernel durations, summed per class
        PH_CUDA(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < 3; ++i) { c->t_ms[i] = 0.0; c->t_n[i] = 0; }
        for (size_t r = 0; r < c->treplays; ++r)
            for (size_t j = 0; j < c->tcls.size(); ++j) {
                float ms = 0.f;
                PH_CUDA(cudaEventElapsedTime(&ms, c->tpool[r][j], c->tpool[r][j + 1]));
                c->t_ms[c->tcls[j]] += ms;
                c->t_n[c->tcls[j]] += 1;
            }
    }
    for (int i = 0; i < 3; ++i) { out[2 * i] = c->t_ms[i]; out[2 * i + 1] = (double)c->t_n[i]; }
    out[6] = (double)c->launches;
    return PH_OK;
}

int ph_quotient_selftest(uint64_t seed, int n, double out[2]) {
    if (n <= 0 || !out) return fail(PH_ERR_INVALID, "bad argument");
    const int blocks = (n + 255) / 256;
    double* d = nullptr;
    PH_CUDA(cudaMalloc(&d, 2 * (size_t)blocks * sizeof(double)));
    ph::quotient_selftest_kernel<<<blocks, 256>>>(seed, n, d);
    cudaError_t e = cudaGetLastError();
    std::vector<double> h(2 * (size_t)blocks);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, cudaGetErrorString(e));
    out[0] = out[1] = 0.0;
    for (int b = 0; b < blocks; ++b) { out[0] = std::max(out[0], h[2 * b]); out[1] = std::max(out[1], h[2 * b + 1]); }
    return PH_OK;
}

int ph_sync(ph_ctx* c) {
    if (!c) return fail(PH_ERR_INVALID, "null argument");
    PH_CUDA(cudaStreamSynchronize(c->stream));
    return PH_OK;
}

}  // extern "C"

// =======================================================================================
// Residual evaluation that allocates no device memory.
//
// Some callers cannot call cudaMalloc: solver loops that must never synchronise the
// device (cudaMalloc and cudaFree may), and host frameworks that reserve the device memory
// up front through their own pool and forbid any later allocation. For them
// ph_residual_noalloc computes R(U) on caller-owned device buffers without a context:
// its scratch (the viscous terms between the auxiliary and residual kernels), the
// neighbour table and the operator tables live in file-scope device arrays of fixed
// size, which every GPU that loads this library holds until the process exits.
// Nothing has to start at zero: each call rebuilds the tables, clears the status word,
// writes the whole viscous-flux scratch before reading it and writes every entry of R.
// The status word keeps the call's non-physical flag until the next call
// (ph_residual_noalloc_status reads it). All calls share these arrays, so calls that
// overlap on the GPU race.
// =======================================================================================
namespace {

constexpr size_t NOALLOC_FV_DOUBLES = (size_t)4 << 20;      // 4 Mi doubles = 32 MiB viscous-term scratch
constexpr int NOALLOC_MAX_CELLS = 32768;                     // 32^3 cells (neighbour table 768 KiB)

static __device__ __align__(256) double g_noalloc_fv[NOALLOC_FV_DOUBLES];
static __device__ __align__(256) int g_noalloc_nbr[6 * NOALLOC_MAX_CELLS];
static __device__ __align__(256) ph::OpTab g_noalloc_ops;
static __device__ __align__(256) unsigned g_noalloc_status;

// Device addresses of the arrays above, resolved once per device with that device current.
// In host code the array names are host-side stand-ins, never device addresses. The first
// call on a device takes the mutex; later calls see `ready` set (release / acquire).
struct NoallocSymbols {
    std::atomic<bool> ready{false};
    double* fv = nullptr;
    int* nbr = nullptr;
    ph::OpTab* ops = nullptr;
    unsigned* status = nullptr;
};
NoallocSymbols g_noalloc_sym[64];
std::mutex g_noalloc_setup_mutex;

int noalloc_setup(int dev) {
    if (dev < 0 || dev >= 64) return fail(PH_ERR_INVALID, "device ordinal out of range");
    NoallocSymbols& s = g_noalloc_sym[dev];
    if (s.ready.load(std::memory_order_acquire)) return PH_OK;
    std::lock_guard<std::mutex> lock(g_noalloc_setup_mutex);
    if (s.ready.load(std::memory_order_relaxed)) return PH_OK;
    PH_CUDA(cudaGetSymbolAddress((void**)&s.fv, g_noalloc_fv));
    PH_CUDA(cudaGetSymbolAddress((void**)&s.nbr, g_noalloc_nbr));
    PH_CUDA(cudaGetSymbolAddress((void**)&s.ops, g_noalloc_ops));
    PH_CUDA(cudaGetSymbolAddress((void**)&s.status, g_noalloc_status));
    s.ready.store(true, std::memory_order_release);
    return PH_OK;
}

// Writes this call's operator table and clears the status word. The table travels as a
// kernel argument (copied into the launch), so no host buffer has to outlive the call.
__global__ void noalloc_set_tables(const ph::OpTab tab) {
    const double* src = reinterpret_cast<const double*>(&tab);
    double* dst = reinterpret_cast<double*>(&g_noalloc_ops);
    for (int i = threadIdx.x; i < (int)(sizeof(ph::OpTab) / sizeof(double)); i += blockDim.x) dst[i] = src[i];
    if (threadIdx.x == 0) g_noalloc_status = 0u;
}

// fixed-size versions of the 1-D helpers (no heap allocation)
void noalloc_gll(int n, double* x, double* w) {
    const int m = n - 1;
    for (int i = 0; i < n; ++i) {
        double z = -std::cos(M_PI * i / m);
        if (i > 0 && i < m) {
            for (int it = 0; it < 64; ++it) {
                double p, dp; legendre_pd(m, z, p, dp);
                const double d2p = (2.0 * z * dp - m * (m + 1.0) * p) / (1.0 - z * z);
                const double dz = dp / d2p;
                z -= dz;
                if (std::fabs(dz) < 1e-17) break;
            }
        }
        double p, dp; legendre_pd(m, z, p, dp);
        x[i] = 0.5 * (z + 1.0);
        w[i] = 1.0 / (m * (m + 1.0) * p * p);
    }
    x[0] = 0.0; x[m] = 1.0;
}
void noalloc_lagrange_derivative(const double* nodes, int n, double xx, double* dv) {
    for (int j = 0; j < n; ++j) {
        double val = 1.0, der = 0.0;
        for (int m = 0; m < n; ++m) {
            if (m == j) continue;
            const double r = 1.0 / (nodes[j] - nodes[m]);
            der = der * (xx - nodes[m]) * r + val * r;
            val *= (xx - nodes[m]) * r;
        }
        dv[j] = der;
    }
}
bool noalloc_invert(const double* A0, int n, double* Ai) {
    double A[ph::MAXN1 * ph::MAXN1];
    for (int i = 0; i < n * n; ++i) { A[i] = A0[i]; Ai[i] = (i % (n + 1) == 0) ? 1.0 : 0.0; }
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r) if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        if (A[piv * n + c] == 0.0) return false;
        for (int j = 0; j < n; ++j) { std::swap(A[c * n + j], A[piv * n + j]); std::swap(Ai[c * n + j], Ai[piv * n + j]); }
        const double inv = 1.0 / A[c * n + c];
        for (int j = 0; j < n; ++j) { A[c * n + j] *= inv; Ai[c * n + j] *= inv; }
        for (int r = 0; r < n; ++r) if (r != c && A[r * n + c] != 0.0) {
            const double f = A[r * n + c];
            for (int j = 0; j < n; ++j) { A[r * n + j] -= f * A[c * n + j]; Ai[r * n + j] -= f * Ai[c * n + j]; }
        }
    }
    return true;
}

// neighbour table of the periodic cube in deal.II cell order, built on the device
__global__ void noalloc_neighbours(int n, int morton, int levels, int* nbr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int nc = n * n * n;
    if (c >= nc) return;
    int t[3];
    if (morton) {
        t[0] = t[1] = t[2] = 0;
        for (int l = 0; l < levels; ++l) {
            const int ch = (c >> (3 * (levels - 1 - l))) & 7;
            t[0] = 2 * t[0] + (ch & 1); t[1] = 2 * t[1] + ((ch >> 1) & 1); t[2] = 2 * t[2] + ((ch >> 2) & 1);
        }
    } else {
        t[0] = c % n; t[1] = (c / n) % n; t[2] = c / (n * n);
    }
    for (int f = 0; f < 6; ++f) {
        int u[3] = {t[0], t[1], t[2]};
        const int d = f >> 1;
        u[d] = (u[d] + ((f & 1) ? 1 : -1) + n) % n;
        int id;
        if (morton) {
            id = 0;
            for (int l = 0; l < levels; ++l) {
                const int b = levels - 1 - l;
                const int ch = ((u[0] >> b) & 1) | (((u[1] >> b) & 1) << 1) | (((u[2] >> b) & 1) << 2);
                id = (id << 3) | ch;
            }
        } else {
            id = (u[2] * n + u[1]) * n + u[0];
        }
        nbr[6 * c + f] = id;
    }
}

} // namespace

extern "C" int ph_residual_noalloc(const ph_mesh_desc* mesh, const ph_params* prm, const double* U, double* R,
                                   void* cuda_stream) {
    if (!mesh || !prm || !U || !R) return fail(PH_ERR_INVALID, "null argument");
    // the checks of ph_ctx_create, before anything is launched
    if (int rc = check_mesh(mesh)) return rc;
    if (int rc = check_param_ranges(prm)) return rc;
    if (is_curvilinear(mesh)) return fail(PH_ERR_UNSUPPORTED, "ph_residual_noalloc: affine meshes only");
    if (has_boundaries(mesh)) return fail(PH_ERR_UNSUPPORTED, "ph_residual_noalloc: periodic meshes only");
    if (const char* why = unsupported_reason(mesh, prm)) return fail(PH_ERR_UNSUPPORTED, why);
    if (prm->conv_num_flux >= 3 && !prm->use_split_form)
        return fail(PH_ERR_INVALID, "two point flux and not using split form are not compatible");
    const int n = mesh->n_cells_per_direction;
    const long long nc = (long long)n * n * n;
    const int N1 = prm->poly_degree + 1, NP = N1 * N1 * N1;
    const bool visc = prm->pde_type == 1;
    if (nc > NOALLOC_MAX_CELLS)
        return fail(PH_ERR_INVALID, "ph_residual_noalloc: " + std::to_string(nc) + " cells exceed the fixed limit of " +
                                        std::to_string(NOALLOC_MAX_CELLS));
    const size_t fv_doubles = (size_t)nc * (4 * NP + 24 * N1 * N1);
    if (visc && fv_doubles > NOALLOC_FV_DOUBLES)
        return fail(PH_ERR_INVALID, "ph_residual_noalloc: the viscous-term scratch needs " +
                                        std::to_string(fv_doubles) + " doubles, above the fixed " +
                                        std::to_string(NOALLOC_FV_DOUBLES));
    int dev = 0;
    PH_CUDA(cudaGetDevice(&dev));
    if (int rc = noalloc_setup(dev)) return rc;
    const NoallocSymbols& sym = g_noalloc_sym[dev];
    cudaStream_t stream = (cudaStream_t)cuda_stream;
    const double h = (mesh->right - mesh->left) / n;

    // 1-D operators (the construction of ph_ctx_create, on fixed-size stack arrays so that
    // this entry point makes no heap allocation either)
    double x[ph::MAXN1], w[ph::MAXN1], D[ph::MAXN1 * ph::MAXN1], Dp[ph::MAXN1 * ph::MAXN1];
    double MK[ph::MAXN1 * ph::MAXN1], Minv[ph::MAXN1 * ph::MAXN1], tmp[ph::MAXN1 * ph::MAXN1];
    double MKa[ph::MAXN1 * ph::MAXN1], Minva[ph::MAXN1 * ph::MAXN1];
    noalloc_gll(N1, x, w);
    for (int a = 0; a < N1; ++a) noalloc_lagrange_derivative(x, N1, x[a], &D[a * N1]);
    double cfr = 0.0, kaux = 0.0;
    if (fr_parameter(prm->flux_reconstruction, prm->poly_degree, prm->FR_user_specified_correction_parameter_value, cfr))
        return fail(PH_ERR_UNSUPPORTED, "flux_reconstruction type not defined for this degree");
    if (fr_aux_parameter(prm->flux_reconstruction_aux, prm->poly_degree, kaux))
        return fail(PH_ERR_UNSUPPORTED, "flux_reconstruction_aux type not defined for this degree");
    for (int i = 0; i < N1 * N1; ++i) Dp[i] = (i % (N1 + 1) == 0) ? 1.0 : 0.0;
    for (int k = 0; k < prm->poly_degree; ++k) {
        for (int i = 0; i < N1; ++i)
            for (int j = 0; j < N1; ++j) {
                double acc = 0.0;
                for (int m = 0; m < N1; ++m) acc += D[i * N1 + m] * Dp[m * N1 + j];
                tmp[i * N1 + j] = acc;
            }
        for (int i = 0; i < N1 * N1; ++i) Dp[i] = tmp[i];
    }
    for (int i = 0; i < N1; ++i)
        for (int j = 0; j < N1; ++j) {
            double kij = 0.0;
            for (int q = 0; q < N1; ++q) kij += Dp[q * N1 + i] * w[q] * Dp[q * N1 + j];
            MK[i * N1 + j] = (i == j ? w[i] : 0.0) + cfr * kij;
            MKa[i * N1 + j] = (i == j ? w[i] : 0.0) + kaux * kij;
        }
    if (!noalloc_invert(MK, N1, Minv)) return fail(PH_ERR_INVALID, "singular FR mass matrix");
    if (!noalloc_invert(MKa, N1, Minva)) return fail(PH_ERR_INVALID, "singular auxiliary FR mass matrix");
    ph::OpTab tab;
    std::memset(&tab, 0, sizeof(tab));
    tab.aux_fr = kaux != 0.0;
    for (int a = 0; a < N1; ++a) {
        tab.w[a] = w[a];
        for (int l = 0; l < N1; ++l) {
            tab.D[a * ph::MAXN1 + l] = D[a * N1 + l];
            tab.Dsk[a * ph::MAXN1 + l] = (w[a] * D[a * N1 + l] - w[l] * D[l * N1 + a]) / w[a];
            tab.Minv[a * ph::MAXN1 + l] = Minv[a * N1 + l];
            tab.B[a * ph::MAXN1 + l] = Minv[a * N1 + l] * w[l];
            tab.Baux[a * ph::MAXN1 + l] = Minva[a * N1 + l] * w[l];
        }
    }
    noalloc_set_tables<<<1, 128, 0, stream>>>(tab);
    PH_CUDA(cudaGetLastError());
    const bool pow2 = (n & (n - 1)) == 0;
    const bool morton = (mesh->cell_order == 2) || (mesh->cell_order == 0 && pow2);
    int levels = 0;
    while ((1 << levels) < n) ++levels;
    noalloc_neighbours<<<(int)((nc + 127) / 128), 128, 0, stream>>>(n, morton ? 1 : 0, levels, sym.nbr);
    PH_CUDA(cudaGetLastError());

    ph::PhysConst pc{};
    pc.gam = prm->gamma_gas; pc.gm1 = prm->gamma_gas - 1.0;
    pc.mach2 = prm->mach_infinity * prm->mach_infinity;
    pc.temp_ratio = 110.4 / prm->temperature_inf;
    pc.inv_re = 1.0 / prm->reynolds_number_inf;
    pc.prandtl = prm->prandtl_number;
    pc.const_visc = prm->nondimensionalized_constant_viscosity;
    pc.use_const_visc = prm->use_constant_viscosity;
    pc.pressure_shift = prm->pressure_shift;
    pc.two_point = prm->two_point_num_flux_type;
    pc.conv_flux = prm->conv_num_flux;
    pc.diss_flux = prm->diss_num_flux;
    pc.navier_stokes = visc;
    const double sipg = prm->diss_num_flux == 1 ? 0.0 : prm->sipg_penalty_factor;
    pc.sipg_pen = sipg;
    const int fp32 = prm->precision == PH_FP32_RESIDUAL;

    cudaError_t e = cudaSuccess;
    if (visc) {
        switch (N1) {
        case 2: e = ph::launch_aux<2>(U, sym.nbr, tab, 0, (int)nc, 1.0 / h, pc, fp32, sym.fv, nullptr, stream); break;
        case 3: e = ph::launch_aux<3>(U, sym.nbr, tab, 0, (int)nc, 1.0 / h, pc, fp32, sym.fv, nullptr, stream); break;
        case 4: e = ph::launch_aux<4>(U, sym.nbr, tab, 0, (int)nc, 1.0 / h, pc, fp32, sym.fv, nullptr, stream); break;
        case 5: e = ph::launch_aux<5>(U, sym.nbr, tab, 0, (int)nc, 1.0 / h, pc, fp32, sym.fv, nullptr, stream); break;
        case 6: e = ph::launch_aux<6>(U, sym.nbr, tab, 0, (int)nc, 1.0 / h, pc, fp32, sym.fv, nullptr, stream); break;
        default: e = ph::launch_aux<7>(U, sym.nbr, tab, 0, (int)nc, 1.0 / h, pc, fp32, sym.fv, nullptr, stream); break;
        }
        if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string("aux launch: ") + cudaGetErrorString(e));
    }
    ph::StageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.U = U; a.Fv = sym.fv; a.nbr = sym.nbr; a.ops = sym.ops; a.nc = (int)nc;
    a.h = h; a.inv_h = 1.0 / h; a.pen = (double)prm->poly_degree * (prm->poly_degree + 1) / h * sipg;
    a.pc = pc; a.status = sym.status; a.mode = 0; a.fr = cfr != 0.0; a.out = R;
    const bool split = prm->use_split_form != 0;
    switch (N1) {
    case 2: e = ph::launch_stage<2>(a, fp32, visc, split, stream); break;
    case 3: e = ph::launch_stage<3>(a, fp32, visc, split, stream); break;
    case 4: e = ph::launch_stage<4>(a, fp32, visc, split, stream); break;
    case 5: e = ph::launch_stage<5>(a, fp32, visc, split, stream); break;
    case 6: e = ph::launch_stage<6>(a, fp32, visc, split, stream); break;
    default: e = ph::launch_stage<7>(a, fp32, visc, split, stream); break;
    }
    if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string("residual launch: ") + cudaGetErrorString(e));
    return PH_OK;
}

extern "C" int ph_residual_noalloc_status(void* cuda_stream, uint32_t* flags) {
    if (!flags) return fail(PH_ERR_INVALID, "null argument");
    int dev = 0;
    PH_CUDA(cudaGetDevice(&dev));
    if (int rc = noalloc_setup(dev)) return rc;
    unsigned v = 0;
    cudaStream_t stream = (cudaStream_t)cuda_stream;
    PH_CUDA(cudaMemcpyAsync(&v, g_noalloc_sym[dev].status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    PH_CUDA(cudaStreamSynchronize(stream));
    *flags = v;
    return PH_OK;
}
