// Taylor-Green integrated quantities with QGauss(p+11) over-integration
// (PeriodicTurbulence::compute_and_update_integrated_quantities,
// src/flow_solver/flow_solver_cases/periodic_turbulence.cpp:439-672).
//
// One CTA per cell. The solution is contracted with the 1-D basis in x once and kept
// in shared memory (value and x-derivative); each thread owns one (qx, qy) column of
// cubature points and walks qz, contracting y and z on the fly. Per-cell partial sums
// go to global memory and are summed on the host in cell order (deterministic).
//
// Curvilinear cells (CURV): the node coordinates are three more nodal fields carried
// through the same contractions; their derivatives at a cubature point are the mapping
// Jacobian there (the mapping has the solution's degree), which gives det J for the
// weights and J^-1 for the physical gradients.
//
// FULL: all nine quantities of the reference's IntegratedQuantitiesEnum
// (periodic_turbulence.h:176-186) with the integrands of navier_stokes.cpp:399-740 and
// euler.cpp:378-402. The palinstrophy needs the gradient of the vorticity after its L2
// projection onto the solution basis (vol_projection_operator, operators.cpp:1865-1889):
// each column thread accumulates the qz-projection of the vorticity while it walks qz,
// the qy and qx projections follow in shared memory, and a second pass over the
// cubature points differentiates the projected vorticity.
#pragma once
#include "ph_kernels.cuh"

namespace ph {

constexpr int MAXNE = 20;

struct IntegralTab {
    double B[MAXNE * MAXN1];
    double dB[MAXNE * MAXN1];
    double P[MAXN1 * MAXNE];   // 1-D L2 projection onto the solution basis, [node][cubature point]
    double w[MAXNE];
    double x[MAXNE];           // cubature points on [0, 1]
};

// Viscosity and gas constants of the integrands (the reference evaluates them with a
// NavierStokes physics object whatever the PDE).
struct IntegralConst {
    double h, gam, gm1, mach2, temp_ratio, const_visc;
    int use_const_visc;
};

// partial sums per cell: FULL = the nine quantities then the max wave speed;
// otherwise kinetic energy, enstrophy, max wave speed
template <bool FULL> __host__ __device__ constexpr int integral_partials() { return FULL ? 10 : 3; }

template <int N1, bool CURV, bool FULL>
__host__ __device__ constexpr size_t integrals_smem_bytes() {
    constexpr int NFLD = CURV ? 8 : 5;
    constexpr int NE = N1 + 10;
    constexpr size_t base = NFLD * N1 * N1 * N1 + 2 * NFLD * N1 * N1 * NE;
    constexpr size_t proj = FULL ? 3 * NE * NE * N1 + 3 * NE * N1 * N1 : 0;
    return sizeof(double) * (base + proj);
}

// Physical gradient of nf nodal fields at one cubature point from the x-contracted values
// and x-derivatives (sT0, sT1); fields listed in fld[].
template <int N1, int NE, int NF>
__device__ __forceinline__ void point_fields(const double* sT0, const double* sT1, const double* sB, const double* sdB,
                                             const int (&fld)[NF], int qx, int qy, int qz, double (&u)[NF],
                                             double (&g)[NF][3]) {
    constexpr int NT2 = N1 * N1 * NE;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        const int s = fld[f];
        double v = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
        for (int k = 0; k < N1; ++k) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
            for (int j = 0; j < N1; ++j) {
                const double t0 = sT0[s * NT2 + (k * N1 + j) * NE + qx];
                const double t1 = sT1[s * NT2 + (k * N1 + j) * NE + qx];
                a0 += sB[qy * N1 + j] * t0;
                a1 += sB[qy * N1 + j] * t1;
                a2 += sdB[qy * N1 + j] * t0;
            }
            const double b = sB[qz * N1 + k], db = sdB[qz * N1 + k];
            v += b * a0; gx += b * a1; gy += b * a2; gz += db * a0;
        }
        u[f] = v; g[f][0] = gx; g[f][1] = gy; g[f][2] = gz;
    }
}

// J^-1 and det J from the reference gradients of the three coordinate fields
// (J[m][j] = dX_m/dxi_j; physical gradient = reference gradient times J^-1).
__device__ __forceinline__ double inverse_jacobian(const double (&gx)[3][3], double (&I)[3][3]) {
    const double(&J)[3][3] = gx;
    const double dj = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                      J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                      J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    I[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / dj;
    I[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / dj;
    I[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / dj;
    I[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / dj;
    I[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / dj;
    I[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / dj;
    I[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / dj;
    I[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / dj;
    I[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / dj;
    return dj;
}

template <int NF>
__device__ __forceinline__ void to_physical(double (&g)[NF][3], int nf, const double (&I)[3][3]) {
#pragma unroll
    for (int s = 0; s < NF; ++s) {
        if (s >= nf) break;
        const double r0 = g[s][0], r1 = g[s][1], r2 = g[s][2];
#pragma unroll
        for (int d = 0; d < 3; ++d) g[s][d] = r0 * I[0][d] + r1 * I[1][d] + r2 * I[2][d];
    }
}

template <int N1, bool CURV, bool FULL>
__global__ void integrals_kernel(const double* __restrict__ U, const double* __restrict__ X,
                                 const double* __restrict__ origin, const IntegralTab* tab, int nc, IntegralConst ic,
                                 double* __restrict__ partial) {
    constexpr int NE = N1 + 10;
    constexpr int NP = N1 * N1 * N1;
    constexpr int NT2 = N1 * N1 * NE;
    constexpr int NFLD = CURV ? 8 : 5;   // state (+ node coordinates)
    constexpr int NQ = integral_partials<FULL>();
    constexpr int NACC = FULL ? 9 : 2;   // summed quantities (the wave speed is a max)
    __shared__ double sB[NE * N1], sdB[NE * N1], sP[FULL ? N1 * NE : 1], sw[NE], sx[NE];
    __shared__ double red[NQ][32];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sU = reinterpret_cast<double*>(smem_raw);
    double* sT0 = sU + NFLD * NP;       // [s][(k*N1 + j)*NE + qx], x-contracted values
    double* sT1 = sT0 + NFLD * NT2;     // x-contracted x-derivatives
    double* sWz = sT1 + NFLD * NT2;     // FULL: vorticity projected in z, [c][qy*NE + qx][k]
    double* sWy = sWz + 3 * NE * NE * N1;   // FULL: ... and in y, [c][(k*N1 + j)*NE + qx]
    const int cell = blockIdx.x;
    const int tid = threadIdx.x;
    for (int i = tid; i < NE * N1; i += blockDim.x) { sB[i] = tab->B[i]; sdB[i] = tab->dB[i]; }
    if constexpr (FULL) {
        for (int i = tid; i < N1 * NE; i += blockDim.x) sP[i] = tab->P[i];
    }
    for (int i = tid; i < NE; i += blockDim.x) { sw[i] = tab->w[i]; sx[i] = tab->x[i]; }
    for (int i = tid; i < 5 * NP; i += blockDim.x) sU[i] = U[(size_t)cell * 5 * NP + i];
    if constexpr (CURV) {
        for (int i = tid; i < 3 * NP; i += blockDim.x) sU[5 * NP + i] = X[(size_t)cell * 3 * NP + i];
    }
    __syncthreads();
    for (int i = tid; i < NFLD * NT2; i += blockDim.x) {
        const int qx = i % NE, kj = (i / NE) % (N1 * N1), s = i / NT2;
        double v = 0.0, dv = 0.0;
        for (int a = 0; a < N1; ++a) {
            const double u = sU[s * NP + kj * N1 + a];
            v += sB[qx * N1 + a] * u;
            dv += sdB[qx * N1 + a] * u;
        }
        sT0[i] = v;
        sT1[i] = dv;
    }
    __syncthreads();
    const double h = ic.h, inv_h = 1.0 / h, detj = h * h * h;
    const double gam = ic.gam, gm1 = ic.gm1;
    double acc[NACC];
#pragma unroll
    for (int i = 0; i < NACC; ++i) acc[i] = 0.0;
    double wave = 0.0;
    double o0rg[3] = {0.0, 0.0, 0.0};
    if constexpr (FULL && !CURV) {
        for (int d = 0; d < 3; ++d) o0rg[d] = origin[3 * cell + d];
    }
    int fld[NFLD];
#pragma unroll
    for (int s = 0; s < NFLD; ++s) fld[s] = s;
    for (int col = tid; col < NE * NE; col += blockDim.x) {
        const int qx = col % NE, qy = col / NE;
        double zp[FULL ? 3 : 1][FULL ? N1 : 1];   // FULL: vorticity projected along this column
#pragma unroll
        for (int c = 0; c < (FULL ? 3 : 1); ++c)
#pragma unroll
            for (int k = 0; k < (FULL ? N1 : 1); ++k) zp[c][k] = 0.0;
        for (int qz = 0; qz < NE; ++qz) {
            double u[NFLD], g[NFLD][3];
            point_fields<N1, NE, NFLD>(sT0, sT1, sB, sdB, fld, qx, qy, qz, u, g);
            double wdet = detj;
            if constexpr (CURV) {
                const double gx[3][3] = {{g[5][0], g[5][1], g[5][2]}, {g[6][0], g[6][1], g[6][2]},
                                         {g[7][0], g[7][1], g[7][2]}};
                double I[3][3];
                wdet = inverse_jacobian(gx, I);
                to_physical<NFLD>(g, 5, I);
            } else {
#pragma unroll
                for (int s = 0; s < 5; ++s)
#pragma unroll
                    for (int d = 0; d < 3; ++d) g[s][d] *= inv_h;
            }
            const double rho = u[0];
            double v[3], v2 = 0.0;
#pragma unroll
            for (int d = 0; d < 3; ++d) { v[d] = u[1 + d] / rho; v2 += v[d] * v[d]; }
            double gv[3][3];
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d) gv[a][d] = (g[1 + a][d] - v[a] * g[0][d]) / rho;
            const double o0 = gv[2][1] - gv[1][2], o1 = gv[0][2] - gv[2][0], o2 = gv[1][0] - gv[0][1];
            const double om2 = o0 * o0 + o1 * o1 + o2 * o2;
            const double wt = sw[qx] * sw[qy] * sw[qz] * wdet;
            acc[0] += 0.5 * rho * v2 * wt;
            acc[1] += 0.5 * rho * om2 * wt;
            const double p = gm1 * (u[4] - 0.5 * rho * v2);
            if constexpr (FULL) {
                double S[3][3], dil = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) S[a][b] = 0.5 * (gv[a][b] + gv[b][a]);
#pragma unroll
                for (int d = 0; d < 3; ++d) dil += gv[d][d];
                double s2 = 0.0, sd2 = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        const double dv = S[a][b] - (a == b ? dil / 3.0 : 0.0);
                        s2 += S[a][b] * S[a][b];
                        sd2 += dv * dv;
                    }
                // Sutherland's law in the nondimensional temperature (navier_stokes.cpp:241-300)
                const double T = gam * ic.mach2 * (p / rho);
                const double mu = ic.use_const_visc ? 1.0 * ic.const_visc
                                                    : ((1.0 + ic.temp_ratio) / (T + ic.temp_ratio)) * pow(T, 1.5);
                double r2 = 0.0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    double xd;
                    if constexpr (CURV) xd = u[5 + d];
                    else xd = o0rg[d] + h * sx[d == 0 ? qx : d == 1 ? qy : qz];
                    r2 += xd * xd;
                }
                acc[2] += p * dil * wt;
                acc[3] += mu * sd2 * wt;
                acc[4] += mu * s2 * wt;
                acc[5] += 0.5 * v2 * wt;
                acc[6] += 0.5 * om2 * wt;
                acc[8] += 0.5 * r2 * sqrt(om2) * wt;
#pragma unroll
                for (int k = 0; k < N1; ++k) {
                    const double pk = sP[k * NE + qz];
                    zp[0][k] += pk * o0; zp[1][k] += pk * o1; zp[2][k] += pk * o2;
                }
            }
            const double c = sqrt(p * gam / rho);
            const double ws = sqrt(v2) + c;
            wave = ws > wave ? ws : wave;
        }
        if constexpr (FULL) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < N1; ++k) sWz[(c * NE * NE + col) * N1 + k] = zp[c][k];
        }
    }
    if constexpr (FULL) {
        __syncthreads();
        // projection in y: sWy[c][(k*N1 + j)*NE + qx] = sum_qy P[j][qy] sWz[c][qy*NE + qx][k]
        for (int i = tid; i < 3 * N1 * N1 * NE; i += blockDim.x) {
            const int qx = i % NE, j = (i / NE) % N1, k = (i / (NE * N1)) % N1, c = i / (NE * N1 * N1);
            double v = 0.0;
            for (int qy = 0; qy < NE; ++qy) v += sP[j * NE + qy] * sWz[(c * NE * NE + qy * NE + qx) * N1 + k];
            sWy[i] = v;
        }
        __syncthreads();
        // projection in x: coefficients into the (no longer needed) state slots 0..2 of sU
        for (int i = tid; i < 3 * NP; i += blockDim.x) {
            const int a = i % N1, kj = (i / N1) % (N1 * N1), c = i / NP;
            double v = 0.0;
            for (int qx = 0; qx < NE; ++qx) v += sP[a * NE + qx] * sWy[(c * N1 * N1 + kj) * NE + qx];
            sU[i] = v;
        }
        __syncthreads();
        // x-contraction of the projected vorticity into slots 0..2 (coordinates stay in 5..7)
        for (int i = tid; i < 3 * NT2; i += blockDim.x) {
            const int qx = i % NE, kj = (i / NE) % (N1 * N1), s = i / NT2;
            double v = 0.0, dv = 0.0;
            for (int a = 0; a < N1; ++a) {
                const double u = sU[s * NP + kj * N1 + a];
                v += sB[qx * N1 + a] * u;
                dv += sdB[qx * N1 + a] * u;
            }
            sT0[i] = v;
            sT1[i] = dv;
        }
        __syncthreads();
        constexpr int NF2 = CURV ? 6 : 3;
        int fld2[NF2];
#pragma unroll
        for (int f = 0; f < NF2; ++f) fld2[f] = f < 3 ? f : f + 2;
        double pal = 0.0;
        for (int pt = tid; pt < NE * NE * NE; pt += blockDim.x) {
            const int qx = pt % NE, qy = (pt / NE) % NE, qz = pt / (NE * NE);
            double u[NF2], g[NF2][3];
            point_fields<N1, NE, NF2>(sT0, sT1, sB, sdB, fld2, qx, qy, qz, u, g);
            double wdet = detj;
            if constexpr (CURV) {
                const double gx[3][3] = {{g[3][0], g[3][1], g[3][2]}, {g[4][0], g[4][1], g[4][2]},
                                         {g[5][0], g[5][1], g[5][2]}};
                double I[3][3];
                wdet = inverse_jacobian(gx, I);
                to_physical<NF2>(g, 3, I);
            } else {
#pragma unroll
                for (int s = 0; s < 3; ++s)
#pragma unroll
                    for (int d = 0; d < 3; ++d) g[s][d] *= inv_h;
            }
            double gg = 0.0;
#pragma unroll
            for (int s = 0; s < 3; ++s)
#pragma unroll
                for (int d = 0; d < 3; ++d) gg += g[s][d] * g[s][d];
            pal += 0.5 * gg * sw[qx] * sw[qy] * sw[qz] * wdet;
        }
        acc[7] = pal;
    }
    // block reduction in a fixed order (warp shuffles, then warp 0)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int i = 0; i < NACC; ++i) acc[i] += __shfl_down_sync(0xffffffffu, acc[i], o);
        const double wo = __shfl_down_sync(0xffffffffu, wave, o);
        wave = wo > wave ? wo : wave;
    }
    const int warp = tid >> 5, lane = tid & 31, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < NACC; ++i) red[i][warp] = acc[i];
        red[NQ - 1][warp] = wave;
    }
    __syncthreads();
    if (tid == 0) {
        double a[NQ];
#pragma unroll
        for (int i = 0; i < NQ; ++i) a[i] = 0.0;
        for (int w = 0; w < nw; ++w) {
#pragma unroll
            for (int i = 0; i < NACC; ++i) a[i] += red[i][w];
            a[NQ - 1] = red[NQ - 1][w] > a[NQ - 1] ? red[NQ - 1][w] : a[NQ - 1];
        }
#pragma unroll
        for (int i = 0; i < NQ; ++i) partial[(size_t)NQ * cell + i] = a[i];
    }
}

// Kinetic energy, enstrophy and wave speed on affine cells (the integrals_kernel's partials
// without FULL) with the y-contraction hoisted out of the point loop: the x- and then the
// y-contracted values (and x-, y-derivatives of the four fields whose gradient the enstrophy
// needs) of all columns are built once per cell in shared memory, so a cubature point only
// contracts along z (4 N1-term sums per field instead of N1 (3 N1 + 4)). Each point's values
// are the same products summed in the same order as in integrals_kernel. Used while two CTAs
// fit an SM (p <= 3: 82 KB at p = 3): 2.5 ms against 3.9 ms per evaluation at 32^3 cells,
// p = 3 on B200; at p = 5 (178 KB, one CTA per SM) it was slower than integrals_kernel.
constexpr int AFF_THREADS = 256;
template <int N1> __host__ __device__ constexpr size_t integrals_affine_smem_bytes() {
    constexpr int NE = N1 + 10;
    return sizeof(double) * (5 * N1 * N1 * N1 + 2 * N1 * N1 * NE + 13 * N1 * NE * NE);
}
template <int N1> __host__ __device__ constexpr bool integrals_affine_fits() {
    return integrals_affine_smem_bytes<N1>() <= 100 * 1024;
}

template <int N1>
__global__ void __launch_bounds__(AFF_THREADS)
integrals_affine_kernel(const double* __restrict__ U, const IntegralTab* tab, int nc, IntegralConst ic,
                        double* __restrict__ partial) {
    constexpr int NE = N1 + 10;
    constexpr int NP = N1 * N1 * N1;
    constexpr int NT2 = N1 * N1 * NE;    // x-contracted entries of one field
    constexpr int NY = N1 * NE * NE;     // x- and y-contracted entries of one field
    __shared__ double sB[NE * N1], sdB[NE * N1], sw[NE];
    __shared__ double red[3][32];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sU = reinterpret_cast<double*>(smem_raw);   // [5][NP]
    double* sTv = sU + 5 * NP;                          // [(k*N1 + j)*NE + qx], one field at a time
    double* sTx = sTv + NT2;
    // rows 0-4: values of the five fields; 5-8: x-derivatives and 9-12: y-derivatives of
    // density and momentum; each row [k][qy*NE + qx]
    double* sY = sTx + NT2;
    const int cell = blockIdx.x;
    const int tid = threadIdx.x;
    for (int i = tid; i < NE * N1; i += AFF_THREADS) { sB[i] = tab->B[i]; sdB[i] = tab->dB[i]; }
    for (int i = tid; i < NE; i += AFF_THREADS) sw[i] = tab->w[i];
    for (int i = tid; i < 5 * NP; i += AFF_THREADS) sU[i] = U[(size_t)cell * 5 * NP + i];
    __syncthreads();
    for (int f = 0; f < 5; ++f) {
        for (int i = tid; i < NT2; i += AFF_THREADS) {
            const int qx = i % NE, kj = i / NE;
            double v = 0.0, dv = 0.0;
            for (int a = 0; a < N1; ++a) {
                const double u = sU[f * NP + kj * N1 + a];
                v += sB[qx * N1 + a] * u;
                dv += sdB[qx * N1 + a] * u;
            }
            sTv[i] = v;
            sTx[i] = dv;
        }
        __syncthreads();
        for (int i = tid; i < NY; i += AFF_THREADS) {
            const int qx = i % NE, qy = (i / NE) % NE, k = i / (NE * NE);
            double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
            for (int j = 0; j < N1; ++j) {
                const double t0 = sTv[(k * N1 + j) * NE + qx];
                const double t1 = sTx[(k * N1 + j) * NE + qx];
                a0 += sB[qy * N1 + j] * t0;
                a1 += sB[qy * N1 + j] * t1;
                a2 += sdB[qy * N1 + j] * t0;
            }
            sY[f * NY + i] = a0;
            if (f < 4) { sY[(5 + f) * NY + i] = a1; sY[(9 + f) * NY + i] = a2; }
        }
        __syncthreads();
    }
    const double inv_h = 1.0 / ic.h, detj = ic.h * ic.h * ic.h;
    const double gam = ic.gam, gm1 = ic.gm1;
    double ke = 0.0, ens = 0.0, wave = 0.0;
    for (int pt = tid; pt < NE * NE * NE; pt += AFF_THREADS) {
        const int col = pt % (NE * NE), qz = pt / (NE * NE);
        const int qx = col % NE, qy = col / NE;
        double u[5], g[4][3];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            double v = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
            for (int k = 0; k < N1; ++k) {
                const double b = sB[qz * N1 + k], db = sdB[qz * N1 + k];
                const double a0 = sY[f * NY + k * NE * NE + col];
                if (f < 4) {
                    const double a1 = sY[(5 + f) * NY + k * NE * NE + col];
                    const double a2 = sY[(9 + f) * NY + k * NE * NE + col];
                    v += b * a0; gx += b * a1; gy += b * a2; gz += db * a0;
                } else {
                    v += b * a0;
                }
            }
            u[f] = v;
            if (f < 4) { g[f][0] = gx * inv_h; g[f][1] = gy * inv_h; g[f][2] = gz * inv_h; }
        }
        const double rho = u[0];
        double v[3], v2 = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) { v[d] = u[1 + d] / rho; v2 += v[d] * v[d]; }
        double gv[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) gv[a][d] = (g[1 + a][d] - v[a] * g[0][d]) / rho;
        const double o0 = gv[2][1] - gv[1][2], o1 = gv[0][2] - gv[2][0], o2 = gv[1][0] - gv[0][1];
        const double wt = sw[qx] * sw[qy] * sw[qz] * detj;
        ke += 0.5 * rho * v2 * wt;
        ens += 0.5 * rho * (o0 * o0 + o1 * o1 + o2 * o2) * wt;
        const double p = gm1 * (u[4] - 0.5 * rho * v2);
        const double c = sqrt(p * gam / rho);
        const double ws = sqrt(v2) + c;
        wave = ws > wave ? ws : wave;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ke += __shfl_down_sync(0xffffffffu, ke, o);
        ens += __shfl_down_sync(0xffffffffu, ens, o);
        const double wo = __shfl_down_sync(0xffffffffu, wave, o);
        wave = wo > wave ? wo : wave;
    }
    const int warp = tid >> 5, lane = tid & 31;
    if (lane == 0) { red[0][warp] = ke; red[1][warp] = ens; red[2][warp] = wave; }
    __syncthreads();
    if (tid == 0) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int w = 0; w < AFF_THREADS / 32; ++w) {
            a0 += red[0][w]; a1 += red[1][w];
            a2 = red[2][w] > a2 ? red[2][w] : a2;
        }
        partial[3 * (size_t)cell + 0] = a0;
        partial[3 * (size_t)cell + 1] = a1;
        partial[3 * (size_t)cell + 2] = a2;
    }
}

// One row of the integrals table on the device: the per-cell partials of integrals_kernel
// (not FULL: kinetic energy, enstrophy, max wave speed per cell) reduced to
// {KE / V, enstrophy / V, 2 enstrophy / (Re V) (re > 0; zero otherwise), max wave speed}, the
// values ph_integrals returns. One block of ROW_THREADS: each thread sums a fixed strided share of the cells in
// order, then a fixed-order tree, so a row is the same on every run. The row index comes
// from a device counter that the kernel advances, so one captured launch serves every row.
constexpr int ROW_THREADS = 512;
static __global__ void __launch_bounds__(ROW_THREADS)
integrals_row_kernel(const double* __restrict__ partial, int nc, double vol, double re, int* __restrict__ counter,
                     int max_rows, double* __restrict__ table) {
    __shared__ double ske[ROW_THREADS], sen[ROW_THREADS], swv[ROW_THREADS];
    const int tid = threadIdx.x;
    double ke = 0.0, en = 0.0, wv = 0.0;
    for (int i = tid; i < nc; i += ROW_THREADS) {
        ke += partial[3 * (size_t)i];
        en += partial[3 * (size_t)i + 1];
        const double w = partial[3 * (size_t)i + 2];
        wv = w > wv ? w : wv;
    }
    ske[tid] = ke; sen[tid] = en; swv[tid] = wv;
    __syncthreads();
    for (int h = ROW_THREADS / 2; h > 0; h >>= 1) {
        if (tid < h) {
            ske[tid] += ske[tid + h];
            sen[tid] += sen[tid + h];
            swv[tid] = swv[tid + h] > swv[tid] ? swv[tid + h] : swv[tid];
        }
        __syncthreads();
    }
    if (tid == 0) {
        const int r = *counter;
        if (r < max_rows) {
            double* row = table + 4 * (size_t)r;
            row[0] = ske[0] / vol;
            row[1] = sen[0] / vol;
            row[2] = re > 0.0 ? 2.0 * row[1] / re : 0.0;
            row[3] = swv[0];
        }
        *counter = r + 1;
    }
}

// ------------------------------------------------------------------------------------
// Rate of change of the kinetic energy, dKE/dt = integral of dKE/dU . dU/dt over the cell with
// the same QGauss(p+11) cubature as the kinetic energy itself (so its time integral is that
// KE), from a state U and its time derivative K = M^-1 R(U): the integrand is
// v . K_m - |v|^2 / 2 K_rho (rho |v|^2 / 2 with m = rho v; the energy does not enter). Affine
// cells; per-cell partial sums (W det J included), summed on the host in cell order. One CTA
// per cell; one thread per (qx, qy) column walks qz.
// ------------------------------------------------------------------------------------
template <int N1> __host__ __device__ constexpr int ke_rate_threads() {
    return (N1 + 10) * (N1 + 10) <= 256 ? 256 : 512;
}
template <int N1> __host__ __device__ constexpr size_t ke_rate_smem() {
    constexpr int NE = N1 + 10;
    return sizeof(double) * (8 * (size_t)N1 * N1 * N1 + 8 * (size_t)N1 * N1 * NE + 8 * (size_t)N1 * NE * NE);
}

template <int N1>
__global__ void __launch_bounds__(ke_rate_threads<N1>())
ke_rate_kernel(const double* __restrict__ U, const double* __restrict__ K, const IntegralTab* __restrict__ tab,
               int nc, double h3, double* __restrict__ partial) {
    constexpr int NE = N1 + 10, NP = N1 * N1 * N1, NT = ke_rate_threads<N1>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sF = reinterpret_cast<double*>(smem_raw);   // [8][NP]: rho, m (3) of U, then of K
    double* t0 = sF + 8 * NP;                           // [8][N1][N1][NE] after x
    double* t1 = t0 + 8 * N1 * N1 * NE;                 // [8][N1][NE][NE] after y
    __shared__ double sB[NE * N1], sw[NE], red[NT / 32];
    const int cell = blockIdx.x, tid = threadIdx.x;
    for (int i = tid; i < NE * N1; i += NT) sB[i] = tab->B[i];
    for (int i = tid; i < NE; i += NT) sw[i] = tab->w[i];
    for (int i = tid; i < 8 * NP; i += NT) {
        const int f = i / NP, node = i % NP;
        const double* src = f < 4 ? U : K;
        sF[i] = src[((size_t)cell * 5 + (f % 4)) * NP + node];
    }
    __syncthreads();
    for (int i = tid; i < 8 * N1 * N1 * NE; i += NT) {   // x: [f][z][y][qx]
        const int qx = i % NE, r = i / NE;              // r = (f * N1 + z) * N1 + y
        double v = 0.0;
        for (int a = 0; a < N1; ++a) v += sB[qx * N1 + a] * sF[r * N1 + a];
        t0[i] = v;
    }
    __syncthreads();
    for (int i = tid; i < 8 * N1 * NE * NE; i += NT) {   // y: [f][z][qy][qx]
        const int qx = i % NE, qy = (i / NE) % NE, fz = i / (NE * NE);
        double v = 0.0;
        for (int b = 0; b < N1; ++b) v += sB[qy * N1 + b] * t0[(fz * N1 + b) * NE + qx];
        t1[i] = v;
    }
    __syncthreads();
    double acc = 0.0;
    for (int col = tid; col < NE * NE; col += NT) {
        const int qx = col % NE, qy = col / NE;
        for (int qz = 0; qz < NE; ++qz) {
            double f[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                double v = 0.0;
                for (int c = 0; c < N1; ++c) v += sB[qz * N1 + c] * t1[((k * N1 + c) * NE + qy) * NE + qx];
                f[k] = v;
            }
            const double v0 = f[1] / f[0], v1 = f[2] / f[0], v2 = f[3] / f[0];
            const double rate = v0 * f[5] + v1 * f[6] + v2 * f[7] - 0.5 * (v0 * v0 + v1 * v1 + v2 * v2) * f[4];
            acc += sw[qx] * sw[qy] * sw[qz] * rate;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < NT / 32; ++w) t += red[w];
        partial[cell] = t * h3;
    }
}

} // namespace ph
