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
#pragma once
#include "ph_kernels.cuh"

namespace ph {

constexpr int MAXNE = 20;

struct IntegralTab {
    double B[MAXNE * MAXN1];
    double dB[MAXNE * MAXN1];
    double w[MAXNE];
};

template <int N1, bool CURV>
__host__ __device__ constexpr size_t integrals_smem_bytes() {
    constexpr int NFLD = CURV ? 8 : 5;
    return sizeof(double) * (NFLD * N1 * N1 * N1 + 2 * NFLD * N1 * N1 * (N1 + 10));
}

template <int N1, bool CURV>
__global__ void integrals_kernel(const double* __restrict__ U, const double* __restrict__ X, const IntegralTab* tab,
                                 int nc, double h, double gam, double gm1, double* __restrict__ partial) {
    constexpr int NE = N1 + 10;
    constexpr int NP = N1 * N1 * N1;
    constexpr int NT2 = N1 * N1 * NE;
    constexpr int NFLD = CURV ? 8 : 5;   // state (+ node coordinates)
    __shared__ double sB[NE * N1], sdB[NE * N1], sw[NE];
    __shared__ double red[3][32];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sU = reinterpret_cast<double*>(smem_raw);
    double* sT0 = sU + NFLD * NP;       // [s][(k*N1 + j)*NE + qx], x-contracted values
    double* sT1 = sT0 + NFLD * NT2;     // x-contracted x-derivatives
    const int cell = blockIdx.x;
    const int tid = threadIdx.x;
    for (int i = tid; i < NE * N1; i += blockDim.x) { sB[i] = tab->B[i]; sdB[i] = tab->dB[i]; }
    for (int i = tid; i < NE; i += blockDim.x) sw[i] = tab->w[i];
    for (int i = tid; i < 5 * NP; i += blockDim.x) sU[i] = U[(size_t)cell * 5 * NP + i];
    if constexpr (CURV)
        for (int i = tid; i < 3 * NP; i += blockDim.x) sU[5 * NP + i] = X[(size_t)cell * 3 * NP + i];
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
    const double inv_h = 1.0 / h, detj = h * h * h;
    double ke = 0.0, ens = 0.0, wave = 0.0;
    for (int pt = tid; pt < NE * NE * NE; pt += blockDim.x) {
        const int qx = pt % NE, qy = (pt / NE) % NE, qz = pt / (NE * NE);
        double u[NFLD], g[NFLD][3];
#pragma unroll
        for (int s = 0; s < NFLD; ++s) {
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
            u[s] = v; g[s][0] = gx; g[s][1] = gy; g[s][2] = gz;
        }
        double wdet = detj;
        if constexpr (CURV) {
            // J[m][j] = dX_m/dxi_j; physical gradient = reference gradient times J^-1
            double J[3][3];
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int j = 0; j < 3; ++j) J[m][j] = g[5 + m][j];
            const double dj = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                              J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                              J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
            double I[3][3];
            I[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / dj;
            I[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / dj;
            I[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / dj;
            I[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / dj;
            I[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / dj;
            I[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / dj;
            I[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / dj;
            I[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / dj;
            I[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / dj;
#pragma unroll
            for (int s = 0; s < 5; ++s) {
                const double r0 = g[s][0], r1 = g[s][1], r2 = g[s][2];
#pragma unroll
                for (int d = 0; d < 3; ++d) g[s][d] = r0 * I[0][d] + r1 * I[1][d] + r2 * I[2][d];
            }
            wdet = dj;
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
        const double wt = sw[qx] * sw[qy] * sw[qz] * wdet;
        ke += 0.5 * rho * v2 * wt;
        ens += 0.5 * rho * (o0 * o0 + o1 * o1 + o2 * o2) * wt;
        const double p = gm1 * (u[4] - 0.5 * rho * v2);
        const double c = sqrt(p * gam / rho);
        const double ws = sqrt(v2) + c;
        wave = ws > wave ? ws : wave;
    }
    // block reduction in a fixed order (warp shuffles, then warp 0)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ke += __shfl_down_sync(0xffffffffu, ke, o);
        ens += __shfl_down_sync(0xffffffffu, ens, o);
        const double wo = __shfl_down_sync(0xffffffffu, wave, o);
        wave = wo > wave ? wo : wave;
    }
    const int warp = tid >> 5, lane = tid & 31, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) { red[0][warp] = ke; red[1][warp] = ens; red[2][warp] = wave; }
    __syncthreads();
    if (tid == 0) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int w = 0; w < nw; ++w) { a0 += red[0][w]; a1 += red[1][w]; a2 = red[2][w] > a2 ? red[2][w] : a2; }
        partial[3 * cell + 0] = a0; partial[3 * cell + 1] = a1; partial[3 * cell + 2] = a2;
    }
}

} // namespace ph
