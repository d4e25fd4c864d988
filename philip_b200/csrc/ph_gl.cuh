// sm_100a kernels of the uncollocated strong-form DG/FR residual: solution on the (p+1)^3
// GLL support points of FE_DGQ(p), volume and face integrals on nq = p + 1 +
// overintegration flux nodes per direction (Gauss-Legendre, the reference's default
// flux_nodes_type, or Gauss-Lobatto with overintegration), affine periodic cells, FP64.
//
// Here the 1-D operators are dense: the interpolation chi (nq x nd) from the solution
// nodes to the flux nodes, its face rows, the entropy projection (chi M^-1 chi^T W), the
// flux-node differentiation and the FR mass inverse (M + K)^-1 with M = chi^T W chi. Every
// one is applied direction by direction (sum factorisation, operators.cpp:294-649): one thread
// per 1-D line holds the line in registers, and the operator, a kernel parameter, is read with
// compile-time indices (the extents are template arguments), so its entries are operands of
// the FMAs rather than memory loads.
//
// Three kernels per residual evaluation (one CTA per cell each):
//   gl_trace_kernel  the state's face values (chi_s (x) chi (x) chi U) and, for the split
//                    form, the face values of the projected entropy variables, per face
//   gl_aux_kernel    (Navier-Stokes) the lifted gradient q = (M_aux)^-1 [chi^T W D(chi u)
//                    + face (u* - u) n], kept at the flux nodes, then the viscous volume term
//                    -chi^T W div(F_v), and per face node F_v(u, q) . n and the face-normal
//                    volume viscous flux
//   gl_stage_kernel  volume term (two-point split form with the skew operator on flux-node
//                    lines, or the conservative divergence), hybrid surface-volume two-point
//                    terms, numerical fluxes, lifts, (M+K)^-1 and the RK stage update
// The face data of a neighbour come from the buffers the earlier kernels wrote, so every
// face's numerical flux sees the same two states from either side.
//
// Reference structure restated (the oracle's Solver::assemble_residual follows the same lines):
//   auxiliary equation ................ src/dg/strong_dg.cpp:498-1008
//   volume term, split and conservative src/dg/strong_dg.cpp:1016-1579
//   entropy projection ................ src/dg/strong_dg.cpp:1235-1330, :3044-3142
//   hybrid surface-volume two-point ... src/dg/strong_dg.cpp:3144-3350
//   numerical fluxes and lifts ........ src/dg/strong_dg.cpp:3354-3576
//   inverse mass (affine) ............. src/dg/dg_base.cpp:4207-4219
#pragma once
#include "ph_kernels.cuh"

namespace ph {

constexpr int GL_MAXQ = 7;   // flux nodes per direction
constexpr int GL_MAXD = 7;   // solution nodes per direction

// 1-D operators, packed row-major with the actual sizes (nq, nd).
struct GlTab {
    double chi[GL_MAXQ * GL_MAXD];    // [q][i] solution basis l_i at flux node q
    double chis[2][GL_MAXD];          // solution basis at xi = 0 and xi = 1
    double phis[2][GL_MAXQ];          // flux-node Lagrange basis at xi = 0 and xi = 1
    double dphi[GL_MAXQ * GL_MAXQ];   // [q][l] derivative of flux-node basis l at flux node q
    double skew[GL_MAXQ * GL_MAXQ];   // S - S^T, S_ij = sum_q phi_i phi_j' w_q (operators.cpp:1440-1477)
    double wq[GL_MAXQ];               // flux-node weights on [0, 1]
    double P[GL_MAXQ * GL_MAXQ];      // chi M^-1 chi^T W: flux values -> projected -> flux values
    double ps[2][GL_MAXQ];            // chis[side] M^-1 chi^T W: face value of the projection
    double minv[GL_MAXD * GL_MAXD];   // (M + K)^-1
    double minv_aux[GL_MAXD * GL_MAXD];
    double haux[GL_MAXQ * GL_MAXQ];   // chi (M + K_aux)^-1 chi^T
    double pwa[GL_MAXD * GL_MAXQ];    // (M + K)^-1 chi^T W (nd x nq): the weight-adjusted inverse mass's projection
};

// Device buffers of the uncollocated path (per cell, reference units).
struct GlArgs {
    const GlTab* tab;
    double* t1;    // [nc][6][T1W][nq^2]: state at the face nodes (5), projected entropy variables (5, split)
    double* t2;    // [nc][6][8][nq^2]: the cell's F_v(u, q) . e_dn at its face nodes (4) and its face-normal
                   // volume viscous flux interpolated to them, signed by the side (4)
    double* vis;   // [nc][4][nd^3]: -chi^T W div(F_v), momentum and energy rows
    // curvilinear cells (nullptr on affine ones): at the volume flux nodes [nc][10][nq^3] the
    // cofactor C[k][d] (row k * 3 + d) and 1 / det J (row 9); at each face's flux nodes
    // [nc][6][3][nq^2] the face's metric column C[:, f / 2]
    const double* vmet;
    const double* fnrm;
    // boundary faces of a non-periodic mesh (nbr = -1 - k, a.btype[k]): [nb][4][nq^2] the outward
    // boundary viscous flux F*_v . n at the face nodes, written by the auxiliary kernel
    double* fb;
};

// Boundary faces (out of line: only boundary face nodes call them, and the periodic path keeps its
// register allocation). The viscous boundary state of a face node (component s) from the cell's own
// face values (stride NF), for the auxiliary equation's lift.
static __device__ __noinline__ double gl_bnd_visc_state(int bt, const double* own, int NF, int s,
                                                        const PhysConst& pc) {
    double u[5], ub[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) u[k] = __ldg(&own[k * NF]);
    boundary_viscous_state<double>(bt, u, pc, ub, nullptr);
    return s == 0 ? ub[0] : s == 1 ? ub[1] : s == 2 ? ub[2] : s == 3 ? ub[3] : ub[4];
}
// The outward boundary viscous flux at a face node of face f (evaluate_auxiliary_flux on a boundary,
// viscous_numerical_flux.cpp:66-328): the viscous boundary state of us (the interpolated face state r,
// or the projected one), BR2 / SIPG with its gradient, the central flux with the interior one, no heat
// flux on an adiabatic 1001 wall; the interior side is r.
// Curvilinear faces (m = the face's metric column C[:, f / 2] at the node, else nullptr): the outward
// unit normal sg m / |m| and the flux scaled by |m|.
static __device__ __noinline__ void gl_bnd_visc_flux(int bt, const double r[5], const double us[5],
                                                     const double g[5][3], int f, const PhysConst& pc, double pen,
                                                     double out[4], const double* m) {
    Cst<double> cst; cst.load(pc);
    const int dn = f >> 1;
    const double sg = (f & 1) ? 1.0 : -1.0;
    double ub[5];
    boundary_viscous_state<double>(bt, us, pc, ub, nullptr);
    if (m) {
        const double Jf = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        const double nv[3] = {sg * m[0] / Jf, sg * m[1] / Jf, sg * m[2] / Jf};
        const bool ad = bt == BC_WALL && !pc.bc_isothermal;
        double gb[5][3];
        for (int s = 0; s < 5; ++s)
            for (int e = 0; e < 3; ++e) gb[s][e] = (ad && s == 4) ? 0.0 : g[s][e];
        double Fi[3][4], Fe[3][4];
        viscous_flux<double>(r, g, pc.use_const_visc, cst, Fi, 7, nullptr, ad);
        viscous_flux<double>(ub, pc.diss_flux == DF_CENTRAL ? g : gb, pc.use_const_visc, cst, Fe, 7, nullptr, ad);
        for (int k = 0; k < 4; ++k) {
            const double fi = Fi[0][k] * nv[0] + Fi[1][k] * nv[1] + Fi[2][k] * nv[2];
            const double fe = Fe[0][k] * nv[0] + Fe[1][k] * nv[1] + Fe[2][k] * nv[2];
            out[k] = Jf * (0.5 * (fi + fe));
        }
        return;
    }
    const bool ad = bt == BC_WALL && !pc.bc_isothermal;
    double gb[5][3];
    for (int s = 0; s < 5; ++s)
        for (int e = 0; e < 3; ++e) gb[s][e] = (ad && s == 4) ? 0.0 : g[s][e];
    double Fi[3][4], Fe[3][4];
    viscous_flux<double>(r, g, pc.use_const_visc, cst, Fi, 7, nullptr, ad);
    viscous_flux<double>(ub, pc.diss_flux == DF_CENTRAL ? g : gb, pc.use_const_visc, cst, Fe, 7, nullptr, ad);
    for (int k = 0; k < 4; ++k) out[k] = 0.5 * (sg * Fi[dn][k] + sg * Fe[dn][k]);
    if (pc.diss_flux == DF_SIPG) {
        double J[5][3];
        for (int s = 0; s < 5; ++s)
            for (int e = 0; e < 3; ++e) J[s][e] = (e == dn) ? (r[s] - ub[s]) * sg : 0.0;
        viscous_flux<double>(r, J, pc.use_const_visc, cst, Fi, 7, nullptr, ad);
        viscous_flux<double>(ub, J, pc.use_const_visc, cst, Fe, 7, nullptr, ad);
        for (int k = 0; k < 4; ++k) out[k] = out[k] - pen * (0.5 * (sg * Fi[dn][k] + sg * Fe[dn][k]));
    }
}
// The convective boundary state of a face node (Euler::boundary_face_values) for outward normal
// sg e_dn of face f.
static __device__ __noinline__ void gl_bnd_state(int bt, const double r[5], int f, const PhysConst& pc,
                                                 double ub[5], unsigned* st, const double* nv = nullptr) {
    const int dn = f >> 1;
    const double sg = (f & 1) ? 1.0 : -1.0;
    double nrm[3] = {dn == 0 ? sg : 0.0, dn == 1 ? sg : 0.0, dn == 2 ? sg : 0.0};
    if (nv) { nrm[0] = sg * nv[0]; nrm[1] = sg * nv[1]; nrm[2] = sg * nv[2]; }   // curvilinear: sg times the unit m
    boundary_state<double>(bt, nrm, r, pc, ub, st);
}

template <bool SPLIT> __host__ __device__ constexpr int gl_t1_width() { return SPLIT ? 10 : 5; }
constexpr int GL_T2W = 8;

#ifndef PH_GL_PREFETCH
#define PH_GL_PREFETCH 1
#endif

// L2 prefetch of n doubles at p, one per 128-byte line, addresses clamped inside [p, p + n)
__device__ __forceinline__ void gl_prefetch_span(const double* p, int n, int i0, int stride) {
    const int nl = (n + 15) / 16;
    for (int i = i0; i < nl; i += stride) {
        const int e = i * 16;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p + (e < n ? e : n - 1)));
    }
}

// Warms L2 with the data a cell reads after its volume work: the neighbours' blocks of the
// face-value buffer (the auxiliary kernel: their states; the stage kernel: the whole blocks), and
// in the stage kernel its own face-value blocks, its own and its neighbours' viscous face blocks,
// its viscous volume rows and the RK registers of the epilogue. Each block is one the kernel
// itself reads; a prefetch writes nothing. Boundary faces (nbr < 0) have no neighbour block.
template <int NT, int NF, int D3, int T1W, bool STAGE, bool VISC>
__device__ __forceinline__ void gl_prefetch_l2(const StageArgs& a, const GlArgs& g, int cell) {
    if (!PH_GL_PREFETCH) return;
    const int w = threadIdx.x >> 5, nw = NT / 32, lane = threadIdx.x & 31;
    // warp w takes the blocks w, w + nw, ...: 6 neighbour face-value blocks, then (stage: viscous)
    // 6 neighbour viscous face blocks, the own blocks, (viscous) the viscous rows, the RK registers
    constexpr int NB = STAGE ? 6 + (VISC ? 6 : 0) + 1 + (VISC ? 2 : 0) + 2 : 6;
    for (int b = w; b < NB; b += nw) {
        const double* p = nullptr;
        int n = 0;
        if (b < 6) {
            const int cn = __ldg(&a.nbr[cell * 6 + b]);
            if (cn >= 0) { p = g.t1 + ((size_t)cn * 6 + (b ^ 1)) * T1W * NF; n = (STAGE ? T1W : 5) * NF; }
        } else if (STAGE && VISC && b < 12) {
            const int f = b - 6, cn = __ldg(&a.nbr[cell * 6 + f]);
            if (cn >= 0) { p = g.t2 + ((size_t)cn * 6 + (f ^ 1)) * GL_T2W * NF; n = GL_T2W * NF; }
        } else {
            const int r = b - (STAGE && VISC ? 12 : 6);
            if (r == 0) { p = g.t1 + (size_t)cell * 6 * T1W * NF; n = 6 * T1W * NF; }
            else if (STAGE && VISC && r == 1) { p = g.t2 + (size_t)cell * 6 * GL_T2W * NF; n = 6 * GL_T2W * NF; }
            else if (STAGE && VISC && r == 2) { p = g.vis + (size_t)cell * 4 * D3; n = 4 * D3; }
            else if (STAGE && a.mode == 2) {
                const int k = r - (VISC ? 3 : 1);
                const double* base = k == 0 ? a.Un : a.acc_in;
                if (base) { p = base + (size_t)cell * 5 * D3; n = 5 * D3; }
            }
        }
        if (p) gl_prefetch_span(p, n, lane, 32);
    }
}

// temporaries of the sum-factorised passes on 5 components (and of the six faces' arrays)
template <int ND, int NQ> __host__ __device__ constexpr int gl_temp() {
    constexpr int a = 5 * NQ * NQ * NQ, b = 30 * NQ * NQ, c = 30 * NQ * ND, d = 30 * ND * ND;
    constexpr int ab = a > b ? a : b, cd = c > d ? c : d;
    return ab > cd ? ab : cd;
}

template <int NQ> __host__ __device__ constexpr int gl_threads() {
    return NQ * NQ * NQ <= 64 ? 64 : NQ * NQ * NQ <= 128 ? 128 : 256;
}

// Entropy variables of a conservative state (Euler::compute_entropy_variables, euler.cpp:811-830)
// and the conservative state of entropy variables (:833-855), FP64. The powers are taken through
// logarithms: s = log(p rho^-gamma) = log p - gamma log rho, and
// rho e = (gm1 / (-v4)^gamma)^(1/gm1) exp(-s / gm1) = exp((log gm1 - gamma log(-v4) - s) / gm1),
// one exponential and one or two logarithms instead of the powers' own logarithm-exponential
// pairs (the same values to rounding).
__device__ __forceinline__ void gl_entropy_vars(const double u[5], double gam, double gm1, double v[5],
                                                unsigned* st) {
    const double rho = u[0];
    double v2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) { const double w = u[1 + d] / rho; v2 = v2 + w * w; }
    const double p = positive<double>(gm1 * (u[4] - 0.5 * rho * v2), st);
    const double s = log(p) - gam * log(rho);
    const double rt = p / gm1;
    const double irt = 1.0 / rt;
    v[0] = (rt * (gam + 1.0 - s) - u[4]) * irt;
#pragma unroll
    for (int d = 0; d < 3; ++d) v[1 + d] = u[1 + d] * irt;
    v[4] = -rho * irt;
}
__device__ __forceinline__ void gl_cons_from_entropy(const double v[5], double gam, double gm1, double u[5]) {
    double vv = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) vv += v[1 + d] * v[1 + d];
    const double iv4 = 1.0 / v[4];
    const double s = gam - v[0] + 0.5 * vv * iv4;
    const double rt = exp((log(gm1) - gam * log(-v[4]) - s) / gm1);
    u[0] = -rt * v[4];
#pragma unroll
    for (int d = 0; d < 3; ++d) u[1 + d] = rt * v[1 + d];
    u[4] = rt * (1.0 - 0.5 * vv * iv4);
}

// One sum-factorised pass along direction d: out[s][o] (+)= scale * sum_l A[r * cols + l] in[s][o, r -> l]
// with r the output's coordinate along d. Input dims (n0, n1, n2), n_d = cols; output dims the
// same with n_d = rows. x is the fastest index.
template <int NT>
__device__ __forceinline__ void gl_pass(const double* A, int rows, int cols, int d, int n0, int n1, int n2,
                                            const double* in, int in_ss, double* out, int out_ss, int ns,
                                            double scale, bool acc) {
    const int m0 = d == 0 ? rows : n0, m1 = d == 1 ? rows : n1, m2 = d == 2 ? rows : n2;
    const int osz = m0 * m1 * m2;
    const int st = d == 0 ? 1 : d == 1 ? n0 : n0 * n1;
    for (int it = threadIdx.x; it < ns * osz; it += NT) {
        const int s = it / osz, o = it - s * osz;
        const int x = o % m0, y = (o / m0) % m1, z = o / (m0 * m1);
        const int r = d == 0 ? x : d == 1 ? y : z;
        const int base = ((d == 2 ? 0 : z) * n1 + (d == 1 ? 0 : y)) * n0 + (d == 0 ? 0 : x);
        const double* ip = in + s * in_ss + base;
        const double* ar = A + r * cols;
        double v = 0.0;
        for (int l = 0; l < cols; ++l) v += ar[l] * ip[l * st];
        double* op = out + s * out_ss + o;
        *op = acc ? *op + scale * v : scale * v;
    }
}

// ------------------------------------------------------------------------------------
// Compile-time sum-factorised passes
// ------------------------------------------------------------------------------------
// One pass along direction D of NS arrays with input extents (N0, N1, N2), N_D = COLS, and
// output extents the same with N_D = ROWS (x fastest): one thread per line reads the COLS
// inputs into registers and writes out[o] (+)= scale * sum_l A(o, l) in[l] for each of the ROWS
// outputs, A(o, l) = A[o * COLS + l], or A[l * ROWS + o] with TRANS (the transposed operator
// stored as cols x rows). Summation in ascending l from zero. A line's inputs are all read
// before its outputs are written, so in == out is allowed when ROWS == COLS.
template <int NT, int ROWS, int COLS, int D, int N0, int N1, int N2, int NS, bool TRANS = false>
__device__ __forceinline__ void gl_line(const double* __restrict__ A, const double* in, int in_ss, double* out,
                                        int out_ss, double scale, bool acc) {
    static_assert((D == 0 ? N0 : D == 1 ? N1 : N2) == COLS, "the input extent along D is COLS");
    constexpr int PA = D == 0 ? N1 : N0, PB = D == 2 ? N1 : N2;   // the other two extents, lower first
    constexpr int IST = D == 0 ? 1 : D == 1 ? N0 : N0 * N1;
    constexpr int M0 = D == 0 ? ROWS : N0, M1 = D == 1 ? ROWS : N1;
    constexpr int OST = D == 0 ? 1 : D == 1 ? M0 : M0 * M1;
    constexpr int NL = NS * PA * PB;
#pragma unroll 1
    for (int t = threadIdx.x; t < NL; t += NT) {
        const int s = t / (PA * PB), r = t - s * (PA * PB);
        const int ca = r % PA, cb = r / PA;
        int ib, ob;
        if constexpr (D == 0) { ib = (cb * N1 + ca) * N0; ob = (cb * M1 + ca) * M0; }
        else if constexpr (D == 1) { ib = cb * N1 * N0 + ca; ob = cb * M1 * M0 + ca; }
        else { ib = cb * N0 + ca; ob = ib; }
        const double* ip = in + s * in_ss + ib;
        double* op = out + s * out_ss + ob;
        double v[COLS];
#pragma unroll
        for (int l = 0; l < COLS; ++l) v[l] = ip[l * IST];
#pragma unroll
        for (int o = 0; o < ROWS; ++o) {
            double x = 0.0;
#pragma unroll
            for (int l = 0; l < COLS; ++l) x += (TRANS ? A[l * ROWS + o] : A[o * COLS + l]) * v[l];
            op[o * OST] = acc ? op[o * OST] + scale * x : scale * x;
        }
    }
}

// out = (A (x) A (x) A) in, x first (TRANS: the transpose of A stored NI x NO): input cubes of
// NI per direction, output NO per direction; t0, t1 hold NS NO NI^2 and NS NO^2 NI values.
// Ends with a barrier.
template <int NT, int NO, int NI, int NS, bool TRANS = false>
__device__ __forceinline__ void gl_apply3(const double* A, const double* in, int in_ss, double* out, int out_ss,
                                          double* t0, double* t1, double scale, bool acc) {
    constexpr int S0 = NO * NI * NI, S1 = NO * NO * NI;
    gl_line<NT, NO, NI, 0, NI, NI, NI, NS, TRANS>(A, in, in_ss, t0, S0, 1.0, false);
    __syncthreads();
    gl_line<NT, NO, NI, 1, NO, NI, NI, NS, TRANS>(A, t0, S0, t1, S1, 1.0, false);
    __syncthreads();
    gl_line<NT, NO, NI, 2, NO, NO, NI, NS, TRANS>(A, t1, S1, out, out_ss, scale, acc);
    __syncthreads();
}

// node index of position l along direction dn on the face-node line q2 = t2 * N + t1 (t1 < t2
// the tangential directions: the face-node order of both sides of a face)
template <int N> __device__ __forceinline__ int gl_line_node(int dn, int q2, int l) {
    const int t1c = q2 % N, t2c = q2 / N;
    return dn == 0 ? (t2c * N + t1c) * N + l : dn == 1 ? (t2c * N + l) * N + t1c : (l * N + t2c) * N + t1c;
}

// Face values on all six faces of NS cubes of NIN^3 values: for face f (normal dn = f / 2,
// side f & 1) out[f][s][q2] = sum row[side][i_dn] T[q_t1][i_t1] T[q_t2][i_t2] src[s][i]
// (the surface interpolation of operators.cpp:355-398 with the face's row along the normal),
// q2 = q_t2 * NOUT + q_t1. row0 / row1 (NIN values) are read with run-time indices (shared
// memory); T (NOUT x NIN, a kernel parameter) only with compile-time ones; without HAS_T the
// tangential operator is the identity (NOUT = NIN). w0: 6 NS NIN^2 values, w1: 6 NS NOUT NIN.
// Ends with a barrier.
template <int NT, int NIN, int NOUT, int NS, bool HAS_T>
__device__ __forceinline__ void gl_face_values(const double* src, int src_ss, const double* row0, const double* row1,
                                               const double* T, double* w0, double* w1, double* out, int out_fs,
                                               int out_ss) {
    constexpr int N2 = NIN * NIN;
    for (int it = threadIdx.x; it < 6 * NS * N2; it += NT) {   // along the normal: w0[f][s][b * NIN + a]
        const int f = it / (NS * N2), r = it - f * NS * N2, s = r / N2, ab = r - s * N2;
        const int a = ab % NIN, b = ab / NIN, dn = f >> 1;
        const double* rw = (f & 1) ? row1 : row0;
        const int st = dn == 0 ? 1 : dn == 1 ? NIN : N2;
        const int base = dn == 0 ? (b * NIN + a) * NIN : dn == 1 ? b * N2 + a : b * NIN + a;
        const double* ip = src + s * src_ss + base;
        double v = 0.0;
#pragma unroll
        for (int l = 0; l < NIN; ++l) v += rw[l] * ip[l * st];
        if constexpr (HAS_T) w0[it] = v;
        else out[f * out_fs + s * out_ss + ab] = v;
    }
    __syncthreads();
    if constexpr (HAS_T) {
        for (int it = threadIdx.x; it < 6 * NS * NIN; it += NT) {   // along t1: w1[f][s][b * NOUT + q1]
            const double* ip = w0 + it * NIN;
            double v[NIN];
#pragma unroll
            for (int l = 0; l < NIN; ++l) v[l] = ip[l];
            double* op = w1 + it * NOUT;
#pragma unroll
            for (int o = 0; o < NOUT; ++o) {
                double x = 0.0;
#pragma unroll
                for (int l = 0; l < NIN; ++l) x += T[o * NIN + l] * v[l];
                op[o] = x;
            }
        }
        __syncthreads();
        for (int it = threadIdx.x; it < 6 * NS * NOUT; it += NT) {   // along t2
            const int fs = it / NOUT, q1 = it - fs * NOUT, f = fs / NS, s = fs - f * NS;
            const double* ip = w1 + fs * NOUT * NIN + q1;
            double v[NIN];
#pragma unroll
            for (int l = 0; l < NIN; ++l) v[l] = ip[l * NOUT];
            double* op = out + f * out_fs + s * out_ss + q1;
#pragma unroll
            for (int o = 0; o < NOUT; ++o) {
                double x = 0.0;
#pragma unroll
                for (int l = 0; l < NIN; ++l) x += T[o * NIN + l] * v[l];
                op[o * NOUT] = x;
            }
        }
        __syncthreads();
    }
}

// The lift of six face arrays into NS cubes of ND^3: dst[s][node] (+)= sum_f row[side][i_dn]
// sum_{q1,q2} T[q1][i_t1] T[q2][i_t2] face[f][s][q2] (the surface inner products of
// operators.cpp:575-636 with the solution basis; T is NQ x ND, a kernel parameter; row0 / row1
// in shared memory). w0: 6 NS NQ ND, w1: 6 NS ND^2 values. Ends with a barrier.
template <int NT, int NQ, int ND, int NS>
__device__ __forceinline__ void gl_lift_faces(const double* face, int face_fs, int face_ss, const double* row0,
                                              const double* row1, const double* T, double* w0, double* w1, double* dst,
                                              int dst_ss, double scale) {
    constexpr int MQ = NQ * NQ, D2 = ND * ND, D3 = D2 * ND;
    for (int it = threadIdx.x; it < 6 * NS * NQ; it += NT) {   // along t1: w0[f][s][q2][a]
        const int fs = it / NQ, q2 = it - fs * NQ, f = fs / NS, s = fs - f * NS;
        const double* ip = face + f * face_fs + s * face_ss + q2 * NQ;
        double v[NQ];
#pragma unroll
        for (int l = 0; l < NQ; ++l) v[l] = ip[l];
        double* op = w0 + (fs * NQ + q2) * ND;
#pragma unroll
        for (int o = 0; o < ND; ++o) {
            double x = 0.0;
#pragma unroll
            for (int l = 0; l < NQ; ++l) x += T[l * ND + o] * v[l];
            op[o] = x;
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < 6 * NS * ND; it += NT) {   // along t2: w1[f][s][b * ND + a]
        const int fs = it / ND, a = it - fs * ND;
        const double* ip = w0 + fs * NQ * ND + a;
        double v[NQ];
#pragma unroll
        for (int l = 0; l < NQ; ++l) v[l] = ip[l * ND];
        double* op = w1 + fs * D2 + a;
#pragma unroll
        for (int o = 0; o < ND; ++o) {
            double x = 0.0;
#pragma unroll
            for (int l = 0; l < NQ; ++l) x += T[l * ND + o] * v[l];
            op[o * ND] = x;
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < NS * D3; it += NT) {
        const int s = it / D3, node = it - s * D3;
        const int c[3] = {node % ND, (node / ND) % ND, node / D2};
        double* op = dst + s * dst_ss + node;
#pragma unroll
        for (int dn = 0; dn < 3; ++dn) {
            const int t1 = dn == 0 ? 1 : 0, t2 = dn == 2 ? 1 : 2;
            const int ab = c[t2] * ND + c[t1];
            const double v = row0[c[dn]] * w1[((2 * dn) * NS + s) * D2 + ab] +
                             row1[c[dn]] * w1[((2 * dn + 1) * NS + s) * D2 + ab];
            *op += scale * v;
        }
    }
    __syncthreads();
    (void)MQ;
}

// Shared-memory copy of the operator table (for the reads with run-time indices).
__device__ __forceinline__ void gl_load_tab(const GlTab* g, GlTab* s, int nt) {
    const double* src = reinterpret_cast<const double*>(g);
    double* dst = reinterpret_cast<double*>(s);
    for (int i = threadIdx.x; i < (int)(sizeof(GlTab) / sizeof(double)); i += nt) dst[i] = src[i];
}

// ------------------------------------------------------------------------------------
// Face values of the state (and of the projected entropy variables)
// ------------------------------------------------------------------------------------
template <int ND, int NQ, bool SPLIT>
struct GlTraceLayout {
    static constexpr int NT = gl_threads<NQ>();
    static constexpr int D3 = ND * ND * ND, Q3 = NQ * NQ * NQ;
    static constexpr int oTab = 0, nTab = (int)(sizeof(GlTab) / sizeof(double));
    static constexpr int oU = nTab;                                 // 5 ND^3
    static constexpr int oQ = oU + 5 * D3;                          // 5 NQ^3 (flux-node values / entropy variables)
    static constexpr int nW = gl_temp<ND, NQ>();
    static constexpr int oW0 = oQ + 5 * Q3, oW1 = oW0 + nW;
    static constexpr int total = oW1 + nW;
    static constexpr size_t bytes = (size_t)total * sizeof(double);
};

template <int ND, int NQ, bool SPLIT>
__global__ void __launch_bounds__(gl_threads<NQ>())
gl_trace_kernel(const StageArgs a, const GlArgs g, const __grid_constant__ GlTab T) {
    using L = GlTraceLayout<ND, NQ, SPLIT>;
    constexpr int NT = L::NT, D3 = L::D3, Q3 = L::Q3, T1W = gl_t1_width<SPLIT>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    GlTab* tab = reinterpret_cast<GlTab*>(sm + L::oTab);
    double* sU = sm + L::oU;
    double* sQ = sm + L::oQ;
    double* w0 = sm + L::oW0;
    double* w1 = sm + L::oW1;
    const int cell = a.cell_begin + blockIdx.x;
    gl_load_tab(g.tab, tab, NT);
    for (int i = threadIdx.x; i < 5 * D3; i += NT) sU[i] = __ldg(&a.U[(size_t)cell * 5 * D3 + i]);
    __syncthreads();
    double* out = g.t1 + (size_t)cell * 6 * T1W * NQ * NQ;
    gl_face_values<NT, ND, NQ, 5, true>(sU, D3, tab->chis[0], tab->chis[1], T.chi, w0, w1, out, T1W * NQ * NQ,
                                        NQ * NQ);
    if constexpr (SPLIT) {
        gl_apply3<NT, NQ, ND, 5>(T.chi, sU, D3, sQ, Q3, w0, w1, 1.0, false);
        const double gam = a.pc.gam, gm1 = a.pc.gm1;
        for (int q = threadIdx.x; q < Q3; q += NT) {
            double u[5], v[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) u[s] = sQ[s * Q3 + q];
            gl_entropy_vars(u, gam, gm1, v, a.status);
#pragma unroll
            for (int s = 0; s < 5; ++s) sQ[s * Q3 + q] = v[s];
        }
        __syncthreads();
        gl_face_values<NT, NQ, NQ, 5, true>(sQ, Q3, tab->ps[0], tab->ps[1], T.P, w0, w1, out + 5 * NQ * NQ,
                                            T1W * NQ * NQ, NQ * NQ);
    }
}

// ------------------------------------------------------------------------------------
// Auxiliary equation and the viscous terms (Navier-Stokes)
// ------------------------------------------------------------------------------------
// The lifted gradient is formed at the flux nodes: with H = chi (M + K_aux)^-1 chi^T and
// chi_side = chi^T phi_side (the solution basis is interpolated exactly by the flux-node basis),
//   chi (x3) q_d = (1/h) (H (x) H (x) H) [W D_d (chi u) + sum_side phi_side (x) W_face (u* - u) n_d]
// which is the reference's q_d = (M_aux)^-1 [chi^T W D_d (chi u) + face lifts] taken to the
// flux nodes (strong_dg.cpp:498-1008, dg_base.cpp:4089-4260 with use_auxiliary_eq; C = h^2 I):
// four passes per direction instead of ten. The face values of q are the flux-node values along
// the normal contracted with phi_side (exact for the degree-p gradient).
template <int ND, int NQ, bool SPLIT>
struct GlAuxLayout {
    static constexpr int NT = gl_threads<NQ>();
    static constexpr int D3 = ND * ND * ND, Q3 = NQ * NQ * NQ, NF = NQ * NQ;
    static constexpr int nTab = (int)(sizeof(GlTab) / sizeof(double));
    static constexpr int oU = nTab;                      // 5 NQ^3: the state, later the projected state
    static constexpr int oQ = oU + 5 * Q3;               // 5 NQ^3: state at the flux nodes
    static constexpr int oAQ = oQ + 5 * Q3;              // 15 NQ^3: lifted gradient at the flux nodes
    static constexpr int oF = oAQ + 15 * Q3;             // 12 NQ^3: volume viscous flux
    static constexpr int nT = gl_temp<ND, NQ>();
    static constexpr int oT0 = oF + 12 * Q3, oT1 = oT0 + nT;
    static constexpr int total = oT1 + nT;
    static constexpr size_t bytes = (size_t)total * sizeof(double);
    static_assert(nT >= 30 * NF, "the six faces' terms fit a temporary");
};

// the lifted gradient of all three directions at once (see above), into sAQ[s * 3 + d][Q3]:
// the flux-node derivatives, the six faces' terms, the brackets, then H (x) H (x) H as three
// passes over all fifteen components in place (H is square: each line is read whole before it
// is written). Ends with a barrier.
template <int ND, int NQ, bool SPLIT, bool CURV = false, bool BND = false>
__device__ __forceinline__ void gl_aux_gradient(const StageArgs& a, const GlArgs& g, const GlTab& T,
                                                const GlTab* tab, int cell, const double* sQ, double* face,
                                                double* sAQ) {
    using L = GlAuxLayout<ND, NQ, SPLIT>;
    constexpr int NT = L::NT, Q3 = L::Q3, NF = L::NF, T1W = gl_t1_width<SPLIT>();
    gl_line<NT, NQ, NQ, 0, NQ, NQ, NQ, 5>(T.dphi, sQ, Q3, sAQ + 0 * Q3, 3 * Q3, 1.0, false);
    gl_line<NT, NQ, NQ, 1, NQ, NQ, NQ, 5>(T.dphi, sQ, Q3, sAQ + 1 * Q3, 3 * Q3, 1.0, false);
    gl_line<NT, NQ, NQ, 2, NQ, NQ, NQ, 5>(T.dphi, sQ, Q3, sAQ + 2 * Q3, 3 * Q3, 1.0, false);
    for (int it = threadIdx.x; it < 6 * 5 * NF; it += NT) {   // face[f][s][q2] = W_face (u* - u) n_{f/2}
        const int f = it / (5 * NF), s = (it / NF) % 5, q2 = it % NF;
        const int cn = __ldg(&a.nbr[cell * 6 + f]);
        const double uo = __ldg(&g.t1[(((size_t)cell * 6 + f) * T1W + s) * NF + q2]);
        const double ue = (!BND || cn >= 0) ? __ldg(&g.t1[(((size_t)cn * 6 + (f ^ 1)) * T1W + s) * NF + q2])
                                            : gl_bnd_visc_state(__ldg(&a.btype[-1 - cn]),
                                                                g.t1 + ((size_t)cell * 6 + f) * T1W * NF + q2, NF, s,
                                                                a.pc);
        const double sgn = (f & 1) ? 1.0 : -1.0;
        face[it] = tab->wq[q2 % NQ] * tab->wq[q2 / NQ] * ((0.5 * (uo + ue) - uo) * sgn);
    }
    __syncthreads();
    if constexpr (CURV) {
        // physical components: W sum_j C[d][j] D_j u at the volume flux nodes, and every face's
        // lift (u* - u) (C_face[:, dn])_d (each face reaches every component on a curved cell)
        const double* vm = g.vmet + (size_t)cell * 10 * Q3;
        const double* fm = g.fnrm + (size_t)cell * 18 * NF;
        for (int i = threadIdx.x; i < 5 * Q3; i += NT) {
            const int s = i / Q3, q = i - s * Q3;
            const int c[3] = {q % NQ, (q / NQ) % NQ, q / NF};
            const double W = tab->wq[c[0]] * tab->wq[c[1]] * tab->wq[c[2]];
            double r[3], b[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) r[j] = sAQ[(s * 3 + j) * Q3 + q];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                b[d] = W * (__ldg(&vm[(d * 3 + 0) * Q3 + q]) * r[0] + __ldg(&vm[(d * 3 + 1) * Q3 + q]) * r[1] +
                            __ldg(&vm[(d * 3 + 2) * Q3 + q]) * r[2]);
#pragma unroll
            for (int dn = 0; dn < 3; ++dn) {
                const int a1 = dn == 0 ? 1 : 0, a2 = dn == 2 ? 1 : 2;
                const int q2 = c[a2] * NQ + c[a1];
                const double l0 = tab->phis[0][c[dn]] * face[((2 * dn) * 5 + s) * NF + q2];
                const double l1 = tab->phis[1][c[dn]] * face[((2 * dn + 1) * 5 + s) * NF + q2];
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    b[d] += l0 * __ldg(&fm[((2 * dn) * 3 + d) * NF + q2]) + l1 * __ldg(&fm[((2 * dn + 1) * 3 + d) * NF + q2]);
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) sAQ[(s * 3 + d) * Q3 + q] = b[d];
        }
        __syncthreads();
        // the weight-adjusted inverse at the flux nodes: H (x3) [ (W / det J) H (x3) b ]
        gl_line<NT, NQ, NQ, 0, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, 1.0, false);
        __syncthreads();
        gl_line<NT, NQ, NQ, 1, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, 1.0, false);
        __syncthreads();
        gl_line<NT, NQ, NQ, 2, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, 1.0, false);
        __syncthreads();
        for (int i = threadIdx.x; i < 15 * Q3; i += NT) {
            const int q = i % Q3;
            sAQ[i] *= tab->wq[q % NQ] * tab->wq[(q / NQ) % NQ] * tab->wq[q / NF] * __ldg(&vm[9 * Q3 + q]);
        }
        __syncthreads();
        gl_line<NT, NQ, NQ, 0, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, 1.0, false);
        __syncthreads();
        gl_line<NT, NQ, NQ, 1, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, 1.0, false);
        __syncthreads();
        gl_line<NT, NQ, NQ, 2, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, 1.0, false);
        __syncthreads();
        return;
    }
    for (int i = threadIdx.x; i < 15 * Q3; i += NT) {
        const int k = i / Q3, q = i - k * Q3, s = k / 3, d = k - 3 * s;
        const int c[3] = {q % NQ, (q / NQ) % NQ, q / NF};
        const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
        const int q2 = c[a2] * NQ + c[a1];
        sAQ[i] = tab->wq[c[0]] * tab->wq[c[1]] * tab->wq[c[2]] * sAQ[i] +
                 tab->phis[0][c[d]] * face[((2 * d) * 5 + s) * NF + q2] +
                 tab->phis[1][c[d]] * face[((2 * d + 1) * 5 + s) * NF + q2];
    }
    __syncthreads();
    gl_line<NT, NQ, NQ, 0, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, 1.0, false);
    __syncthreads();
    gl_line<NT, NQ, NQ, 1, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, 1.0, false);
    __syncthreads();
    gl_line<NT, NQ, NQ, 2, NQ, NQ, NQ, 15>(T.haux, sAQ, Q3, sAQ, Q3, a.inv_h, false);
    __syncthreads();
}

// the contravariant viscous flux F~_j = sum_m C[m][j] F_m at volume flux node q (curvilinear)
__device__ __forceinline__ void gl_contravariant(const double* vm, int q, int Q3, double F[3][4]) {
    double C[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) C[i] = __ldg(&vm[i * Q3 + q]);
    double Ft[3][4];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 4; ++k) Ft[j][k] = C[0 * 3 + j] * F[0][k] + C[1 * 3 + j] * F[1][k] + C[2 * 3 + j] * F[2][k];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 4; ++k) F[j][k] = Ft[j][k];
}

// CURV: curvilinear cells (the metric at the flux nodes, g.vmet / g.fnrm): the physical
// gradient through the weight-adjusted inverse (gl_aux_gradient), contravariant volume fluxes,
// and each face node's F_v . C_face[:, dn] (the metric-scaled normal flux)
// BND: the cells with a boundary face (a tile list of them), the boundary states in the lift and the
// boundary viscous fluxes stored for the stage kernel
template <int ND, int NQ, bool SPLIT, bool CURV = false, bool BND = false>
__global__ void __launch_bounds__(gl_threads<NQ>(), 2)
gl_aux_kernel(const StageArgs a, const GlArgs g, const __grid_constant__ GlTab T) {
    using L = GlAuxLayout<ND, NQ, SPLIT>;
    constexpr int NT = L::NT, D3 = L::D3, Q3 = L::Q3, NF = L::NF, T1W = gl_t1_width<SPLIT>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    GlTab* tab = reinterpret_cast<GlTab*>(sm);
    double* sU = sm + L::oU;
    double* sQ = sm + L::oQ;
    double* sAQ = sm + L::oAQ;
    double* sF = sm + L::oF;
    double* t0 = sm + L::oT0;
    double* t1 = sm + L::oT1;
    const int cell = a.tiles ? __ldg(&a.tiles[blockIdx.x]) : a.cell_begin + (int)blockIdx.x;
    Cst<double> cst; cst.load(a.pc);
    const int ucv = a.pc.use_const_visc;
    gl_load_tab(g.tab, tab, NT);
    for (int i = threadIdx.x; i < 5 * D3; i += NT) sU[i] = __ldg(&a.U[(size_t)cell * 5 * D3 + i]);
    gl_prefetch_l2<NT, NF, D3, T1W, false, true>(a, g, cell);
    __syncthreads();
    gl_apply3<NT, NQ, ND, 5>(T.chi, sU, D3, sQ, Q3, t0, t1, 1.0, false);
    gl_aux_gradient<ND, NQ, SPLIT, CURV, BND>(a, g, T, tab, cell, sQ, t0, sAQ);
    const double* vm = CURV ? g.vmet + (size_t)cell * 10 * Q3 : nullptr;
    // per face node of the cell: F_v(u, q) . e_dn with the state's and the gradient's face values
    // (each side's half of the dissipative numerical flux, strong_dg.cpp:3354-3452)
    double* tout = g.t2 + (size_t)cell * 6 * GL_T2W * NF;
    for (int it = threadIdx.x; it < 6 * NF; it += NT) {
        const int f = it / NF, q2 = it - f * NF, dn = f >> 1, side = f & 1;
        const double* rw = tab->phis[side];
        double gq[5][3], r[5];
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            r[s] = __ldg(&g.t1[(((size_t)cell * 6 + f) * T1W + s) * NF + q2]);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double* row = sAQ + (s * 3 + d) * Q3;
                double v = 0.0;
#pragma unroll
                for (int l = 0; l < NQ; ++l) v += rw[l] * row[gl_line_node<NQ>(dn, q2, l)];
                gq[s][d] = v;
            }
        }
        if constexpr (BND) {   // a boundary face: its outward boundary viscous flux for the stage kernel
            const int cn = __ldg(&a.nbr[cell * 6 + f]);
            if (cn < 0) {
                double us[5], out[4];
#pragma unroll
                for (int s = 0; s < 5; ++s) us[s] = r[s];
                if (SPLIT && a.pc.bc_projected) {   // the face state of the projected entropy variables
                    double v[5];
#pragma unroll
                    for (int s = 0; s < 5; ++s) v[s] = __ldg(&g.t1[(((size_t)cell * 6 + f) * T1W + 5 + s) * NF + q2]);
                    gl_cons_from_entropy(v, cst.gam, cst.gm1, us);
                }
                double mc[3];
                if constexpr (CURV) {
                    const double* m = g.fnrm + ((size_t)cell * 6 + f) * 3 * NF + q2;
                    mc[0] = __ldg(&m[0]); mc[1] = __ldg(&m[NF]); mc[2] = __ldg(&m[2 * NF]);
                }
                gl_bnd_visc_flux(__ldg(&a.btype[-1 - cn]), r, us, gq, f, a.pc, a.pen, out, CURV ? mc : nullptr);
#pragma unroll
                for (int k = 0; k < 4; ++k) g.fb[((size_t)(-1 - cn) * 4 + k) * NF + q2] = out[k];
            }
        }
        double F[3][4];
        if constexpr (CURV) {   // F_v . C_face[:, dn]
            viscous_flux<double>(r, gq, ucv, cst, F, 7, nullptr);
            const double* m = g.fnrm + ((size_t)cell * 6 + f) * 3 * NF + q2;
            const double m0 = __ldg(&m[0]), m1 = __ldg(&m[NF]), m2 = __ldg(&m[2 * NF]);
#pragma unroll
            for (int k = 0; k < 4; ++k) tout[(f * GL_T2W + k) * NF + q2] = m0 * F[0][k] + m1 * F[1][k] + m2 * F[2][k];
            continue;
        }
        viscous_flux<double>(r, gq, ucv, cst, F, 1 << dn, nullptr);
#pragma unroll
        for (int k = 0; k < 4; ++k)   // (selects, not a run-time index, keep F in registers)
            tout[(f * GL_T2W + k) * NF + q2] = dn == 0 ? F[0][k] : dn == 1 ? F[1][k] : F[2][k];
    }
    // the split form evaluates the volume viscous flux at the entropy-projected state
    // (strong_dg.cpp:1328 before :1392); the face-normal flux interpolated to the faces uses
    // the state itself (:2836-3041)
    if constexpr (SPLIT) {
        for (int q = threadIdx.x; q < Q3; q += NT) {
            double u[5], v[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) u[s] = sQ[s * Q3 + q];
            gl_entropy_vars(u, cst.gam, cst.gm1, v, a.status);
#pragma unroll
            for (int s = 0; s < 5; ++s) t0[s * Q3 + q] = v[s];
        }
        __syncthreads();
        gl_apply3<NT, NQ, NQ, 5>(T.P, t0, Q3, sU, Q3, t1, sF, 1.0, false);   // sF is free until the fluxes
        for (int q = threadIdx.x; q < Q3; q += NT) {
            double v[5], u[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) v[s] = sU[s * Q3 + q];
            gl_cons_from_entropy(v, cst.gam, cst.gm1, u);
#pragma unroll
            for (int s = 0; s < 5; ++s) sU[s * Q3 + q] = u[s];
        }
        __syncthreads();
    }
    // sF: [d][k][Q3] volume viscous flux
    for (int q = threadIdx.x; q < Q3; q += NT) {
        double u[5], gq[5][3];
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            u[s] = SPLIT ? sU[s * Q3 + q] : sQ[s * Q3 + q];
#pragma unroll
            for (int d = 0; d < 3; ++d) gq[s][d] = sAQ[(s * 3 + d) * Q3 + q];
        }
        double F[3][4];
        viscous_flux<double>(u, gq, ucv, cst, F, 7, nullptr);
        if constexpr (CURV) gl_contravariant(vm, q, Q3, F);
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int k = 0; k < 4; ++k) sF[(d * 4 + k) * Q3 + q] = F[d][k];
    }
    __syncthreads();
    // -chi^T W sum_d D_d F_d, momentum and energy rows
    gl_line<NT, NQ, NQ, 0, NQ, NQ, NQ, 4>(T.dphi, sF, Q3, t0, Q3, 1.0, false);
    __syncthreads();
    gl_line<NT, NQ, NQ, 1, NQ, NQ, NQ, 4>(T.dphi, sF + 4 * Q3, Q3, t0, Q3, 1.0, true);
    __syncthreads();
    gl_line<NT, NQ, NQ, 2, NQ, NQ, NQ, 4>(T.dphi, sF + 8 * Q3, Q3, t0, Q3, 1.0, true);
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * Q3; i += NT) {
        const int q = i % Q3;
        t0[i] *= tab->wq[q % NQ] * tab->wq[(q / NQ) % NQ] * tab->wq[q / NF];
    }
    __syncthreads();
    // (the state rows sU are free now: the fluxes stay in sF for the face values below)
    gl_line<NT, ND, NQ, 0, NQ, NQ, NQ, 4, true>(T.chi, t0, Q3, t1, ND * NQ * NQ, 1.0, false);
    __syncthreads();
    gl_line<NT, ND, NQ, 1, ND, NQ, NQ, 4, true>(T.chi, t1, ND * NQ * NQ, sU, ND * ND * NQ, 1.0, false);
    __syncthreads();
    gl_line<NT, ND, NQ, 2, ND, ND, NQ, 4, true>(T.chi, sU, ND * ND * NQ, g.vis + (size_t)cell * 4 * D3, D3, -1.0,
                                                false);
    // face-normal volume viscous flux at the faces: n_dn sum_l phi_l(side) F_dn(u_l) (state not
    // projected)
    if constexpr (SPLIT) {
        __syncthreads();
        for (int q = threadIdx.x; q < Q3; q += NT) {
            double u[5], gq[5][3];
#pragma unroll
            for (int s = 0; s < 5; ++s) {
                u[s] = sQ[s * Q3 + q];
#pragma unroll
                for (int d = 0; d < 3; ++d) gq[s][d] = sAQ[(s * 3 + d) * Q3 + q];
            }
            double F[3][4];
            viscous_flux<double>(u, gq, ucv, cst, F, 7, nullptr);
            if constexpr (CURV) gl_contravariant(vm, q, Q3, F);
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int k = 0; k < 4; ++k) sF[(d * 4 + k) * Q3 + q] = F[d][k];
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < 6 * 4 * NF; it += NT) {
        const int f = it / (4 * NF), k = (it / NF) % 4, q2 = it % NF;
        const int dn = f >> 1, side = f & 1;
        const double* rw = tab->phis[side];
        const double* row = sF + (dn * 4 + k) * Q3;
        double v = 0.0;
#pragma unroll
        for (int l = 0; l < NQ; ++l) v += rw[l] * row[gl_line_node<NQ>(dn, q2, l)];
        tout[(f * GL_T2W + 4 + k) * NF + q2] = side ? v : -v;
    }
}

// ------------------------------------------------------------------------------------
// Residual (+ mass inverse + RK epilogue)
// ------------------------------------------------------------------------------------
template <int ND, int NQ, bool VISC, bool SPLIT, bool CURV = false>
struct GlStageLayout {
    static constexpr int NT = gl_threads<NQ>();
    static constexpr int D3 = ND * ND * ND, Q3 = NQ * NQ * NQ, NF = NQ * NQ;
    static constexpr int nTab = (int)(sizeof(GlTab) / sizeof(double));
    static constexpr int oU = nTab;                       // 5 ND^3 state, later the right-hand side
    static constexpr int oQ = oU + 5 * D3;                // 5 NQ^3 state at the flux nodes (split: projected)
    static constexpr int oN = oQ + 5 * Q3;                // node quantities (11 NQ^3) or fluxes (15 NQ^3)
    static constexpr int oDiv = oN + 15 * Q3;             // 5 NQ^3 volume divergence (+ hybrid volume terms)
    static constexpr int oF = oDiv + 5 * Q3;              // 6 x 5 x NF face arrays
    static constexpr int nT = gl_temp<ND, NQ>();
    static constexpr int oT0 = oF + 30 * NF, oT1 = oT0 + nT;
    static constexpr int oQF = oT1 + nT;                 // split: the node quantities of two faces' nodes
    static constexpr int oM = oQF + (SPLIT ? 2 * NF * 11 : 0);   // curvilinear: 9 NQ^3 metric cofactor
    static constexpr int total = oM + (CURV ? 9 * Q3 : 0);
    static constexpr size_t bytes = (size_t)total * sizeof(double);
    static_assert(2 * nT >= 2 * NF * NQ * 5, "the hybrid pair fluxes of one direction fit the temporaries");
};

// CURV (split or conservative Euler on curvilinear cells): the volume two-point fluxes are dotted
// with the metric average 1/2 (C_i[:, d] + C_j[:, d]) and the conservative fluxes with C[:, d]
// (strong_dg.cpp:1235-1578), the face fluxes use the face's unit normal C[:, dn] / |C[:, dn]|
// scaled by |C[:, dn]| and the hybrid terms 1/2 (C_face[:, dn] + C_vol[:, dn]) (:3144-3452), and
// the inverse mass is the weight-adjusted P diag(1 / (W det J)) P^T, P = (M+K)^-1 chi^T W
// (dg_base.cpp:4217-4249, operators.cpp:1909-1932). The residual is then in physical units.
template <int ND, int NQ, bool VISC, bool SPLIT, bool CURV = false, bool BND = false>
__global__ void __launch_bounds__(gl_threads<NQ>(), 2)
gl_stage_kernel(const StageArgs a, const GlArgs g, const __grid_constant__ GlTab T) {
    using L = GlStageLayout<ND, NQ, VISC, SPLIT, CURV>;
    constexpr int NT = L::NT, D3 = L::D3, Q3 = L::Q3, NF = L::NF, T1W = gl_t1_width<SPLIT>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    GlTab* tab = reinterpret_cast<GlTab*>(sm);
    double* sU = sm + L::oU;
    double* sQ = sm + L::oQ;
    double* sN = sm + L::oN;
    double* sDiv = sm + L::oDiv;
    double* sF = sm + L::oF;
    double* t0 = sm + L::oT0;
    double* t1 = sm + L::oT1;
    const int cell = a.tiles ? __ldg(&a.tiles[blockIdx.x]) : a.cell_begin + (int)blockIdx.x;
    Cst<double> cst; cst.load(a.pc);
    const int tp = a.pc.two_point, cf = a.pc.conv_flux, df = a.pc.diss_flux, ucv = a.pc.use_const_visc;
    double* sM = sm + L::oM;   // curvilinear: the cofactor at the flux nodes, [k * 3 + d][Q3]
    gl_load_tab(g.tab, tab, NT);
    for (int i = threadIdx.x; i < 5 * D3; i += NT) sU[i] = __ldg(&a.U[(size_t)cell * 5 * D3 + i]);
    if constexpr (CURV)
        for (int i = threadIdx.x; i < 9 * Q3; i += NT) sM[i] = __ldg(&g.vmet[(size_t)cell * 10 * Q3 + i]);
    gl_prefetch_l2<NT, NF, D3, T1W, true, VISC>(a, g, cell);
    __syncthreads();
    gl_apply3<NT, NQ, ND, 5>(T.chi, sU, D3, sQ, Q3, t0, t1, 1.0, false);
    if constexpr (SPLIT) {
        // entropy projection at the flux nodes: u = u(P (x3) v(chi u))  (strong_dg.cpp:1235-1330)
        for (int q = threadIdx.x; q < Q3; q += NT) {
            double u[5], v[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) u[s] = sQ[s * Q3 + q];
            gl_entropy_vars(u, cst.gam, cst.gm1, v, a.status);
#pragma unroll
            for (int s = 0; s < 5; ++s) t0[s * Q3 + q] = v[s];
        }
        __syncthreads();
        gl_apply3<NT, NQ, NQ, 5>(T.P, t0, Q3, sQ, Q3, t1, sDiv, 1.0, false);
        for (int q = threadIdx.x; q < Q3; q += NT) {
            double v[5], u[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) v[s] = sQ[s * Q3 + q];
            gl_cons_from_entropy(v, cst.gam, cst.gm1, u);
#pragma unroll
            for (int s = 0; s < 5; ++s) sQ[s * Q3 + q] = u[s];
            NodeQ<double> nq;
            node_prepare<double>(u, tp, cst.gm1, nq, a.status);
            store_q<double>(sN, Q3, q, nq);
        }
        __syncthreads();
        // two-point volume term: sum over the node's three flux-node lines of
        // skew[x_d][l] w_a w_b F(u_i, u_l) . e_d   (operators.cpp:983-1062), pair-symmetric on
        // warp segments as in the collocated kernel: segments of NQ lanes own the lines along
        // rd; lane pos evaluates the pairs (pos, pos + k), k = 1 .. NQ / 2, in the frame whose x
        // axis is e_rd and receives the pair (pos - k, pos) from lane pos - k of its segment (the
        // two-point fluxes are symmetric); w_a w_b, the same along a line, scales the sum.
        constexpr int SPW = 32 / NQ, NSEG = (NT / 32) * SPW;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int lseg = lane / NQ, pos = lane - lseg * NQ, segbase = lseg * NQ;
#pragma unroll 1
        for (int rd = 0; rd < 3; ++rd) {
            const int st = rd == 0 ? 1 : rd == 1 ? NQ : NF;
#pragma unroll 1
            for (int l0 = 0; l0 < NF; l0 += NSEG) {
                const int lt = l0 + warp * SPW + lseg;
                const bool valid = lseg < SPW && lt < NF;
                const int node = gl_line_node<NQ>(rd, valid ? lt : 0, pos);
                const int base = node - pos * st;
                double acc[5];
                if constexpr (CURV) {   // the pair flux dotted with the averaged metric column
                    NodeQ<double> qi;
                    load_q<double>(sN, Q3, node, qi);
                    const double mi[3] = {sM[(0 * 3 + rd) * Q3 + node], sM[(1 * 3 + rd) * Q3 + node],
                                          sM[(2 * 3 + rd) * Q3 + node]};
#pragma unroll
                    for (int s = 0; s < 5; ++s) acc[s] = 0.0;
#pragma unroll
                    for (int k = 1; k <= NQ / 2; ++k) {
                        const int jp = pos + k < NQ ? pos + k : pos + k - NQ;
                        const int jm = pos - k >= 0 ? pos - k : pos - k + NQ;
                        const bool dup = ((NQ & 1) == 0) && (2 * k == NQ);
                        const int nj = base + jp * st;
                        NodeQ<double> qj;
                        load_q<double>(sN, Q3, nj, qj);
                        const double nv[3] = {0.5 * (mi[0] + sM[(0 * 3 + rd) * Q3 + nj]),
                                              0.5 * (mi[1] + sM[(1 * 3 + rd) * Q3 + nj]),
                                              0.5 * (mi[2] + sM[(2 * 3 + rd) * Q3 + nj])};
                        double F[5];
                        two_point_n<double>(qi, qj, nv, tp, cst, F);
                        const double cj = tab->skew[pos * NQ + jp], cr = tab->skew[pos * NQ + jm];
#pragma unroll
                        for (int s = 0; s < 5; ++s) {
                            const double fr = __shfl_sync(0xffffffffu, F[s], segbase + jm);
                            acc[s] += cj * F[s];
                            if (!dup) acc[s] += cr * fr;
                        }
                    }
                } else {
                    NodeQ<double> qi;
                    load_q_rot<double>(sN, Q3, node, rd, qi);
                    double accr[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
                    for (int k = 1; k <= NQ / 2; ++k) {
                        const int jp = pos + k < NQ ? pos + k : pos + k - NQ;   // (pos + k) mod NQ
                        const int jm = pos - k >= 0 ? pos - k : pos - k + NQ;   // (pos - k) mod NQ
                        const bool dup = ((NQ & 1) == 0) && (2 * k == NQ);
                        NodeQ<double> qj;
                        load_q_rot<double>(sN, Q3, base + jp * st, rd, qj);
                        double F[5];
                        two_point_dir<double, 0>(qi, qj, tp, cst, F);
                        const double cj = tab->skew[pos * NQ + jp], cr = tab->skew[pos * NQ + jm];
#pragma unroll
                        for (int s = 0; s < 5; ++s) {
                            const double fr = __shfl_sync(0xffffffffu, F[s], segbase + jm);
                            accr[s] += cj * F[s];
                            if (!dup) accr[s] += cr * fr;
                        }
                    }
                    // back to (x, y, z) components by selects (a run-time index would put acc in
                    // local memory)
                    acc[0] = accr[0]; acc[4] = accr[4];
                    acc[1] = rd == 0 ? accr[1] : rd == 1 ? accr[3] : accr[2];
                    acc[2] = rd == 0 ? accr[2] : rd == 1 ? accr[1] : accr[3];
                    acc[3] = rd == 0 ? accr[3] : rd == 1 ? accr[2] : accr[1];
                }
                if (valid) {
                    const int t1c = lt % NQ, t2c = lt / NQ;
                    const double wab = tab->wq[t1c] * tab->wq[t2c];
#pragma unroll
                    for (int s = 0; s < 5; ++s) {
                        double* o = sDiv + s * Q3 + node;
                        *o = rd == 0 ? wab * acc[s] : *o + wab * acc[s];
                    }
                }
            }
            __syncthreads();
        }
    } else {
        // conservative: W div(F(chi u)) by the flux-node derivative   (strong_dg.cpp:1546)
        for (int q = threadIdx.x; q < Q3; q += NT) {
            double u[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) u[s] = sQ[s * Q3 + q];
            NodeQ<double> nq;
            node_prepare<double>(u, TP_KG, cst.gm1, nq, a.status);
#pragma unroll
            for (int d = 0; d < 3; ++d) {   // affine: F . e_d; curvilinear: the contravariant F . C[:, d]
                const double nv[3] = {CURV ? sM[(0 * 3 + d) * Q3 + q] : d == 0 ? 1.0 : 0.0,
                                      CURV ? sM[(1 * 3 + d) * Q3 + q] : d == 1 ? 1.0 : 0.0,
                                      CURV ? sM[(2 * 3 + d) * Q3 + q] : d == 2 ? 1.0 : 0.0};
                double F[5];
                conv_flux_n<double>(nq, nv, 0.0, F);
#pragma unroll
                for (int s = 0; s < 5; ++s) sN[(d * 5 + s) * Q3 + q] = F[s];
            }
        }
        __syncthreads();
        gl_line<NT, NQ, NQ, 0, NQ, NQ, NQ, 5>(T.dphi, sN, Q3, sDiv, Q3, 1.0, false);
        __syncthreads();
        gl_line<NT, NQ, NQ, 1, NQ, NQ, NQ, 5>(T.dphi, sN + 5 * Q3, Q3, sDiv, Q3, 1.0, true);
        __syncthreads();
        gl_line<NT, NQ, NQ, 2, NQ, NQ, NQ, 5>(T.dphi, sN + 10 * Q3, Q3, sDiv, Q3, 1.0, true);
        __syncthreads();
        for (int i = threadIdx.x; i < 5 * Q3; i += NT) {
            const int q = i % Q3;
            sDiv[i] *= tab->wq[q % NQ] * tab->wq[(q / NQ) % NQ] * tab->wq[q / NF];
        }
        __syncthreads();
    }

    // ---- faces: numerical fluxes (canonical orientation: the left state is the cell whose
    // +e_dn face it is, the normal +e_dn), and this cell's face array
    // W_face (F_vol.n + F_v,vol.n -/+ F*_conv -/+ F*_diss) [- hybrid surface terms]
    for (int it = threadIdx.x; it < 6 * NF; it += NT) {
        const int f = it / NF, q2 = it % NF;
        const int dn = f >> 1, side = f & 1;
        const double sgn = side ? 1.0 : -1.0;
        const int cn = __ldg(&a.nbr[cell * 6 + f]);
        const bool bnd = BND && cn < 0;   // a boundary face (assemble_boundary_term_strong, strong_dg.cpp:1582-2366)
        const double* to = g.t1 + ((size_t)cell * 6 + f) * T1W * NF + q2;
        const double* te = g.t1 + ((size_t)(bnd ? cell : cn) * 6 + (f ^ 1)) * T1W * NF + q2;
        double uo[5], ue[5], ro[5], re[5];
#pragma unroll
        for (int s = 0; s < 5; ++s) { ro[s] = __ldg(&to[s * NF]); re[s] = __ldg(&te[s * NF]); }
        if (bnd) {
            // the convective flux between the interpolated face state (the projected one with
            // use_projected_entropy_variables_for_nsfr_boundary_term, :2255-2273) and its boundary state
            double ub[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) uo[s] = ro[s];
            if (SPLIT && a.pc.bc_projected) {
                double vo[5];
#pragma unroll
                for (int s = 0; s < 5; ++s) vo[s] = __ldg(&to[(5 + s) * NF]);
                gl_cons_from_entropy(vo, cst.gam, cst.gm1, uo);
            }
            double mnv[3];
            if constexpr (CURV) {   // the face's unit metric normal C[:, dn] / |C[:, dn]|
                const double* m = g.fnrm + ((size_t)cell * 6 + f) * 3 * NF + q2;
                const double m0 = __ldg(&m[0]), m1 = __ldg(&m[NF]), m2 = __ldg(&m[2 * NF]);
                const double J = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
                mnv[0] = m0 / J; mnv[1] = m1 / J; mnv[2] = m2 / J;
            }
            gl_bnd_state(__ldg(&a.btype[-1 - cn]), uo, f, a.pc, ub, a.status, CURV ? mnv : nullptr);
#pragma unroll
            for (int s = 0; s < 5; ++s) ue[s] = ub[s];
        } else if constexpr (SPLIT) {
            double vo[5], ve[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) { vo[s] = __ldg(&to[(5 + s) * NF]); ve[s] = __ldg(&te[(5 + s) * NF]); }
            gl_cons_from_entropy(vo, cst.gam, cst.gm1, uo);
            gl_cons_from_entropy(ve, cst.gam, cst.gm1, ue);
        } else {
#pragma unroll
            for (int s = 0; s < 5; ++s) { uo[s] = ro[s]; ue[s] = re[s]; }
        }
        double nv[3] = {dn == 0 ? 1.0 : 0.0, dn == 1 ? 1.0 : 0.0, dn == 2 ? 1.0 : 0.0};
        double Jf = 1.0;
        if constexpr (CURV) {   // the face's unit normal and |C[:, dn]|
            const double* m = g.fnrm + ((size_t)cell * 6 + f) * 3 * NF + q2;
            const double m0 = __ldg(&m[0]), m1 = __ldg(&m[NF]), m2 = __ldg(&m[2 * NF]);
            Jf = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
            nv[0] = m0 / Jf; nv[1] = m1 / Jf; nv[2] = m2 / Jf;
        }
        const double* uL = side ? uo : ue;
        const double* uR = side ? ue : uo;
        NodeQ<double> qL, qR;
        node_prepare<double>(uL, tp, cst.gm1, qL, nullptr);
        node_prepare<double>(uR, tp, cst.gm1, qR, nullptr);
        double Fc[5];
        conv_num_flux_n<double>(uL, uR, qL, qR, nv, tp, cf, cst, Fc);
        double term[5];
#pragma unroll
        for (int s = 0; s < 5; ++s) term[s] = -sgn * (CURV ? Jf * Fc[s] : Fc[s]);
        if constexpr (VISC) {
            // each side's F_v(u, q) . e_dn at the face node, from the auxiliary kernel
            const double* ao = g.t2 + ((size_t)cell * 6 + f) * GL_T2W * NF + q2;
            const double* ae = g.t2 + ((size_t)(bnd ? cell : cn) * 6 + (f ^ 1)) * GL_T2W * NF + q2;
            double Fo[4], Fe[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) { Fo[k] = __ldg(&ao[k * NF]); Fe[k] = __ldg(&ae[k * NF]); }
            const double* rL = side ? ro : re;
            const double* rR = side ? re : ro;
            const double* FL = side ? Fo : Fe;
            const double* FR = side ? Fe : Fo;
            double Fd[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)   // boundary: F*_v . e_dn = sgn (F*_v . n_out) of the auxiliary kernel
                Fd[k] = bnd ? sgn * __ldg(&g.fb[((size_t)(-1 - cn) * 4 + k) * NF + q2]) : 0.5 * (FL[k] + FR[k]);
            if (df == DF_SIPG && !bnd) {
                double jump[5][3];
#pragma unroll
                for (int s = 0; s < 5; ++s)
#pragma unroll
                    for (int d = 0; d < 3; ++d) jump[s][d] = d == dn ? rL[s] - rR[s] : 0.0;
                double AL[3][4], AR[3][4];
                viscous_flux<double>(rL, jump, ucv, cst, AL, 1 << dn, nullptr);
                viscous_flux<double>(rR, jump, ucv, cst, AR, 1 << dn, nullptr);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double al = dn == 0 ? AL[0][k] : dn == 1 ? AL[1][k] : AL[2][k];
                    const double ar = dn == 0 ? AR[0][k] : dn == 1 ? AR[1][k] : AR[2][k];
                    Fd[k] = Fd[k] - a.pen * (0.5 * (al + ar));
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) term[1 + k] += -sgn * Fd[k] + __ldg(&ao[(4 + k) * NF]);
        }
        if constexpr (!SPLIT) {   // the cell's own convective volume flux at the face: n . sum_l phi_l F(u_l)
            const double* rw = tab->phis[side];
#pragma unroll
            for (int s = 0; s < 5; ++s) {
                const double* row = sN + (dn * 5 + s) * Q3;
                double v = 0.0;
#pragma unroll
                for (int l = 0; l < NQ; ++l) v += rw[l] * row[gl_line_node<NQ>(dn, q2, l)];
                term[s] += sgn * v;
            }
        }
        const double wf = tab->wq[q2 % NQ] * tab->wq[q2 / NQ];
#pragma unroll
        for (int s = 0; s < 5; ++s) sF[(f * 5 + s) * NF + q2] = wf * term[s];
    }
    __syncthreads();
    if constexpr (SPLIT) {
        // hybrid surface-volume two-point terms (strong_dg.cpp:3144-3350): between each face node
        // (its projected state) and the flux nodes of the normal line through it. One direction at
        // a time (its two faces share the volume nodes): the face nodes' quantities, then every
        // (face node, line node) pair flux, then the face sums and the volume sums, in the order
        // face 2 dn before face 2 dn + 1 and line position by position.
        double* sQF = sm + L::oQF;   // [11][2 NF]
        double* s2 = t0;             // [2][NF][NQ][5] (t0 and t1 are contiguous)
#pragma unroll 1
        for (int dn = 0; dn < 3; ++dn) {
            const double nv[3] = {dn == 0 ? 1.0 : 0.0, dn == 1 ? 1.0 : 0.0, dn == 2 ? 1.0 : 0.0};
            for (int it = threadIdx.x; it < 2 * NF; it += NT) {
                const int side = it / NF, q2 = it % NF;
                const double* to = g.t1 + ((size_t)cell * 6 + 2 * dn + side) * T1W * NF + q2;
                double vo[5], uf[5];
#pragma unroll
                for (int s = 0; s < 5; ++s) vo[s] = __ldg(&to[(5 + s) * NF]);
                gl_cons_from_entropy(vo, cst.gam, cst.gm1, uf);
                NodeQ<double> qf;
                node_prepare<double>(uf, tp, cst.gm1, qf, nullptr);
                store_q<double>(sQF, 2 * NF, it, qf);
            }
            __syncthreads();
            for (int it = threadIdx.x; it < 2 * NF * NQ; it += NT) {
                const int side = it / (NF * NQ), r = it % (NF * NQ), q2 = r / NQ, l = r % NQ;
                const int node = gl_line_node<NQ>(dn, q2, l);
                NodeQ<double> qv, qf;
                load_q<double>(sN, Q3, node, qv);
                load_q<double>(sQF, 2 * NF, side * NF + q2, qf);
                double F[5];
                if constexpr (CURV) {   // 1/2 (C_face[:, dn] + C_vol[:, dn])
                    const double* m = g.fnrm + ((size_t)cell * 6 + 2 * dn + side) * 3 * NF + q2;
                    const double mv[3] = {0.5 * (__ldg(&m[0]) + sM[(0 * 3 + dn) * Q3 + node]),
                                          0.5 * (__ldg(&m[NF]) + sM[(1 * 3 + dn) * Q3 + node]),
                                          0.5 * (__ldg(&m[2 * NF]) + sM[(2 * 3 + dn) * Q3 + node])};
                    two_point_n<double>(qv, qf, mv, tp, cst, F);
                } else {
                    two_point_n<double>(qv, qf, nv, tp, cst, F);
                }
#pragma unroll
                for (int s = 0; s < 5; ++s) s2[(size_t)it * 5 + s] = F[s];
            }
            __syncthreads();
            for (int it = threadIdx.x; it < 2 * NF; it += NT) {   // face sums
                const int side = it / NF, q2 = it % NF, f = 2 * dn + side;
                const double sgn = side ? 1.0 : -1.0;
                const double wf = tab->wq[q2 % NQ] * tab->wq[q2 / NQ];
                double hs[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int l = 0; l < NQ; ++l) {
                    const double Hop = tab->phis[side][l] * wf * sgn;
                    const double* F = s2 + ((size_t)(side * NF + q2) * NQ + l) * 5;
#pragma unroll
                    for (int s = 0; s < 5; ++s) hs[s] -= Hop * F[s];
                }
#pragma unroll
                for (int s = 0; s < 5; ++s) sF[(f * 5 + s) * NF + q2] -= hs[s];
            }
            for (int it = threadIdx.x; it < NF * NQ; it += NT) {   // volume sums (other outputs)
                const int q2 = it / NQ, l = it % NQ;
                const int t1c = q2 % NQ, t2c = q2 / NQ;
                const int node = gl_line_node<NQ>(dn, q2, l);
                const double wf = tab->wq[t1c] * tab->wq[t2c];
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                    const double Hop = tab->phis[side][l] * wf * (side ? 1.0 : -1.0);
                    const double* F = s2 + ((size_t)(side * NF + q2) * NQ + l) * 5;
#pragma unroll
                    for (int s = 0; s < 5; ++s) sDiv[s * Q3 + node] += Hop * F[s];
                }
            }
            __syncthreads();
        }
    }
    // ---- assembly: r = -chi^T (x3) [div (+ hybrid)] + sum_f lift(face array) (+ viscous volume)
    gl_apply3<NT, ND, NQ, 5, true>(T.chi, sDiv, Q3, sU, D3, t0, t1, -1.0, false);
    gl_lift_faces<NT, NQ, ND, 5>(sF, 5 * NF, NF, tab->chis[0], tab->chis[1], T.chi, t0, t1, sU, D3, 1.0);
    if constexpr (VISC) {
        for (int i = threadIdx.x; i < 4 * D3; i += NT) sU[D3 + i] += __ldg(&g.vis[(size_t)cell * 4 * D3 + i]);
        __syncthreads();
    }
    // affine: sU = R / h^2 (the affine metric C = h^2 I and J = h^2 factored out); curvilinear: R
    if (a.mode == 0) {
        const double h2 = CURV ? 1.0 : a.h * a.h;
        for (int i = threadIdx.x; i < 5 * D3; i += NT) a.out[(size_t)cell * 5 * D3 + i] = h2 * sU[i];
        return;
    }
    if constexpr (CURV) {   // k = P (x3) [ (1 / (W det J)) P^T (x3) R ]
        gl_apply3<NT, NQ, ND, 5, true>(T.pwa, sU, D3, sDiv, Q3, t0, t1, 1.0, false);
        const double* iJ = g.vmet + ((size_t)cell * 10 + 9) * Q3;
        for (int i = threadIdx.x; i < 5 * Q3; i += NT) {
            const int q = i % Q3;
            sDiv[i] *= __ldg(&iJ[q]) / (tab->wq[q % NQ] * tab->wq[(q / NQ) % NQ] * tab->wq[q / NF]);
        }
        __syncthreads();
        gl_apply3<NT, ND, NQ, 5>(T.pwa, sDiv, Q3, sQ, D3, t0, t1, 1.0, false);
    } else {
        // k = M^-1 R = (1/h) (M+K)^-1 (x3) (R / h^2)
        gl_apply3<NT, ND, ND, 5>(T.minv, sU, D3, sQ, D3, t0, t1, a.inv_h, false);
    }
    if (a.mode == 1) {
        for (int i = threadIdx.x; i < 5 * D3; i += NT) a.out[(size_t)cell * 5 * D3 + i] = sQ[i];
        return;
    }
    if (a.mode == 3) {   // low-storage 3S* / 3S*+ stage (as the collocated kernel's)
        double err2 = 0.0;
        for (int i = threadIdx.x; i < 5 * D3; i += NT) ls_stage_dof(a, (size_t)cell * 5 * D3 + i, sQ[i], err2);
        if (a.err_partial) ls_tile_error<NT>(err2, &a.err_partial[cell]);
        return;
    }
    if (a.ent_partial) {
        // relaxation RK: this cell's v_hat^T M k, v_hat the entropy variables of the stage input
        // projected on the solution basis (compute_entropy_vars, runge_kutta_store_entropy.cpp:30-100)
        // and M = chi^T W J chi (compute_entropy_change_estimate, root_finding_rrk_ode_solver.cpp:353-388):
        // the sum over the flux nodes of W J (chi v_hat)(chi k), chi v_hat = (chi M^-1 chi^T W) v(chi u)
        for (int i = threadIdx.x; i < 5 * D3; i += NT) sU[i] = __ldg(&a.U[(size_t)cell * 5 * D3 + i]);
        __syncthreads();
        gl_apply3<NT, NQ, ND, 5>(T.chi, sU, D3, sDiv, Q3, t0, t1, 1.0, false);
        for (int q = threadIdx.x; q < Q3; q += NT) {
            double u[5], v[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) u[s] = sDiv[s * Q3 + q];
            gl_entropy_vars(u, cst.gam, cst.gm1, v, nullptr);
#pragma unroll
            for (int s = 0; s < 5; ++s) sDiv[s * Q3 + q] = v[s];
        }
        __syncthreads();
        gl_apply3<NT, NQ, NQ, 5>(T.P, sDiv, Q3, sN, Q3, t0, t1, 1.0, false);
        gl_apply3<NT, NQ, ND, 5>(T.chi, sQ, D3, sDiv, Q3, t0, t1, 1.0, false);
        const double h3 = a.h * a.h * a.h;
        double ent = 0.0;
        for (int i = threadIdx.x; i < 5 * Q3; i += NT) {
            const int q = i % Q3;
            const double W = tab->wq[q % NQ] * tab->wq[(q / NQ) % NQ] * tab->wq[q / NF];
            const double J = CURV ? 1.0 / __ldg(&g.vmet[((size_t)cell * 10 + 9) * Q3 + q]) : h3;
            ent += W * J * sN[i] * sDiv[i];
        }
        __shared__ double ered[32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ent += __shfl_down_sync(0xffffffffu, ent, o);
        if ((threadIdx.x & 31) == 0) ered[threadIdx.x >> 5] = ent;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (NT + 31) / 32; ++w) t += ered[w];
            a.ent_partial[cell] = t;
        }
    }
    // Butcher RK stage (as the collocated kernel's epilogue)
    for (int i = threadIdx.x; i < 5 * D3; i += NT) {
        const size_t dof = (size_t)cell * 5 * D3 + i;
        const double k = sQ[i];
        const double un = a.Un[dof];
        const double bs = a.acc_in ? a.acc_in[dof] : (a.inc_mode ? 0.0 : un);
        const double sum = bs + a.c_acc * k;
        if (a.acc_out) a.acc_out[dof] = sum;
        if (a.final_out) a.final_out[dof] = a.inc_mode ? un + sum : sum;
        if (a.next) {
            const double cin = a.carry_in ? a.carry_in[dof] : 0.0;
            a.next[dof] = (cin + a.a_next * k) * a.dt + un;
        }
        if (a.carry_out) a.carry_out[dof] = a.a_carry * k;
    }
}

// ------------------------------------------------------------------------------------
// Relaxation RK on uncollocated flux nodes: the integrated numerical entropy of
// u_n + gamma (u_1 - u_n), the state interpolated to the flux nodes
// (compute_integrated_numerical_entropy, root_finding_rrk_ode_solver.cpp:211-350): per-cell partials
// ------------------------------------------------------------------------------------
template <int ND, int NQ>
struct GlEntropyLayout {
    static constexpr int D3 = ND * ND * ND, Q3 = NQ * NQ * NQ, nT = gl_temp<ND, NQ>();
    static constexpr int oU = 0, oQ = oU + 5 * D3, oT0 = oQ + 5 * Q3, oT1 = oT0 + nT, total = oT1 + nT;
    static constexpr size_t bytes = (size_t)total * sizeof(double);
};

template <int ND, int NQ>
__global__ void __launch_bounds__(gl_threads<NQ>())
gl_rrk_entropy_kernel(const double* __restrict__ Un, const double* __restrict__ U1, double gamma,
                      const __grid_constant__ GlTab T, double h3, const double* __restrict__ vmet, double gam,
                      double* __restrict__ partial) {
    using L = GlEntropyLayout<ND, NQ>;
    constexpr int NT = gl_threads<NQ>(), D3 = L::D3, Q3 = L::Q3, NF = NQ * NQ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    double* sU = sm + L::oU;
    double* sQ = sm + L::oQ;
    const int cell = blockIdx.x;
    for (int i = threadIdx.x; i < 5 * D3; i += NT) {
        const size_t k = (size_t)cell * 5 * D3 + i;
        sU[i] = Un[k] + gamma * (U1[k] - Un[k]);
    }
    __syncthreads();
    gl_apply3<NT, NQ, ND, 5>(T.chi, sU, D3, sQ, Q3, sm + L::oT0, sm + L::oT1, 1.0, false);
    double e = 0.0;
    for (int q = threadIdx.x; q < Q3; q += NT) {
        double u[5];
#pragma unroll
        for (int s = 0; s < 5; ++s) u[s] = sQ[s * Q3 + q];
        const double W = T.wq[q % NQ] * T.wq[(q / NQ) % NQ] * T.wq[q / NF];
        const double J = vmet ? 1.0 / vmet[((size_t)cell * 10 + 9) * Q3 + q] : h3;
        e += W * J * numerical_entropy_fn(u, gam);
    }
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (NT + 31) / 32; ++w) t += red[w];
        partial[cell] = t;
    }
}

// ------------------------------------------------------------------------------------
// The weight-adjusted inverse mass on curvilinear cells on its own (ph_apply_inverse_mass):
// out = P (x3) [ (1 / (W det J)) P^T (x3) in ], one CTA per cell (a.U = in, a.out = out)
// ------------------------------------------------------------------------------------
template <int ND, int NQ>
struct GlMinvLayout {
    static constexpr int NT = gl_threads<NQ>();
    static constexpr int D3 = ND * ND * ND, Q3 = NQ * NQ * NQ;
    static constexpr int nTab = (int)(sizeof(GlTab) / sizeof(double));
    static constexpr int oU = nTab, oQ = oU + 5 * Q3;
    static constexpr int nT = gl_temp<ND, NQ>();
    static constexpr int oT0 = oQ + 5 * Q3, oT1 = oT0 + nT;
    static constexpr int total = oT1 + nT;
    static constexpr size_t bytes = (size_t)total * sizeof(double);
};

template <int ND, int NQ>
__global__ void __launch_bounds__(gl_threads<NQ>())
gl_minv_kernel(const StageArgs a, const GlArgs g, const __grid_constant__ GlTab T) {
    using L = GlMinvLayout<ND, NQ>;
    constexpr int NT = L::NT, D3 = L::D3, Q3 = L::Q3, NF = NQ * NQ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sm = reinterpret_cast<double*>(smem_raw);
    GlTab* tab = reinterpret_cast<GlTab*>(sm);
    double* sU = sm + L::oU;
    double* sQ = sm + L::oQ;
    double* t0 = sm + L::oT0;
    double* t1 = sm + L::oT1;
    const int cell = a.cell_begin + blockIdx.x;
    gl_load_tab(g.tab, tab, NT);
    for (int i = threadIdx.x; i < 5 * D3; i += NT) sU[i] = __ldg(&a.U[(size_t)cell * 5 * D3 + i]);
    __syncthreads();
    gl_apply3<NT, NQ, ND, 5, true>(T.pwa, sU, D3, sQ, Q3, t0, t1, 1.0, false);
    const double* iJ = g.vmet + ((size_t)cell * 10 + 9) * Q3;
    for (int i = threadIdx.x; i < 5 * Q3; i += NT) {
        const int q = i % Q3;
        sQ[i] *= __ldg(&iJ[q]) / (tab->wq[q % NQ] * tab->wq[(q / NQ) % NQ] * tab->wq[q / NF]);
    }
    __syncthreads();
    gl_apply3<NT, ND, NQ, 5>(T.pwa, sQ, Q3, a.out + (size_t)cell * 5 * D3, D3, t0, t1, 1.0, false);
}

} // namespace ph
