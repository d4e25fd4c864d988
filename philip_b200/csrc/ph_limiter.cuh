// Positivity-preserving limiter of the RK stage solutions (PositivityPreservingLimiter::limit,
// src/limiter/positivity_preserving_limiter.cpp:381-678, applied by RungeKuttaBase::apply_limiter
// to every stage solution and to the new solution, src/ode_solver/runge_kutta_base.cpp:21-56).
// One CTA per cell, FP64, in place on a state vector.
//
// Per cell, as the reference computes it:
//   - the solution interpolated to three mixed point sets: Gauss-Lobatto points along direction
//     d and Gauss points along the other two (the sum-factorised interpolation applies its
//     first operator along x, operators.cpp:355-395);
//   - the minimum density over the nodal values and the three sets;
//   - three directional "cell averages" whose innermost weight loop has no braces, so the
//     point index advances once per (i, j) pair: each sums the first n^2 points of its set
//     (the z = 0 plane) with the weight of the loop's i on y and of its j on x (:264-298);
//   - the averages combined with the weights lambda_d max|v|+c of each set (Zhang & Shu,
//     :300-345), the density scaled towards the average (theta, :170-186), the density of the
//     sets interpolated again, and the whole state scaled towards the average by theta2:
//     one value per cell from the pressure ratios (Wang 2012, :597-618) or one per node from
//     the root of the quadratic pressure condition (Zhang 2010, :620-668, gamma taken as 1.4
//     there as in the reference).
#pragma once
#include "ph_gl.cuh"

namespace ph {

struct LimiterTab {
    double Bgl[MAXN1 * MAXN1];    // [q][i] FE_DGQ basis i at Gauss point q (n x n)
    double Bgll[MAXN1 * MAXN1];   // at the Gauss-Lobatto points
    double wgl[MAXN1], wgll[MAXN1];
};

struct LimiterArgs {
    double* U;               // state, limited in place
    const LimiterTab* tab;
    int nc;
    double lam;              // dt / dx (the same cell size in every direction)
    double gam;
    double min_density;      // limiter/min_density
    int zhang;               // 1: positivity_preservingZhang2010, 0: positivity_preservingWang2012
};

template <int N1> __host__ __device__ constexpr int limiter_threads() {
    return N1 * N1 * N1 <= 64 ? 64 : N1 * N1 * N1 <= 128 ? 128 : 256;
}
template <int N1> __host__ __device__ constexpr size_t limiter_smem() {
    // coefficients, three point sets, two pass temporaries (5 NP each), per-node theta2 (4 NP)
    return sizeof(double) * ((size_t)(1 + 3 + 2) * 5 * N1 * N1 * N1 + 4 * N1 * N1 * N1);
}

__device__ __forceinline__ double limiter_pressure(const double u[5], double gm1) {
    const double rho = u[0];
    double v2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) { const double v = u[1 + d] / rho; v2 = v2 + v * v; }
    return gm1 * (u[4] - 0.5 * rho * v2);
}

// Smallest-modulus root of s3 + s2 t + s1 t^2, its real part.
__device__ __forceinline__ double limiter_smallest_root(double s3, double s2, double s1) {
    if (s1 == 0.0) return -s3 / s2;
    const double disc = s2 * s2 - 4.0 * s1 * s3;
    if (disc < 0.0) return -s2 / (2.0 * s1);
    const double q = -0.5 * (s2 + (s2 >= 0.0 ? sqrt(disc) : -sqrt(disc)));
    const double r1 = q / s1, r2 = (q != 0.0) ? s3 / q : r1;
    return fabs(r1) <= fabs(r2) ? r1 : r2;
}

template <int N1>
__global__ void __launch_bounds__(limiter_threads<N1>()) limiter_kernel(const LimiterArgs a) {
    constexpr int NT = limiter_threads<N1>(), NP = N1 * N1 * N1, n = N1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sC = reinterpret_cast<double*>(smem_raw);   // [5][NP] coefficients (nodal values)
    double* sQ = sC + 5 * NP;                            // [3][5][NP] mixed point sets
    double* t0 = sQ + 15 * NP;
    double* t1 = t0 + 5 * NP;
    double* sT = t1 + 5 * NP;                            // [4][NP] per-node theta2 (Zhang)
    __shared__ double red[3][32];
    __shared__ double avg_dim[3][5], avg[5], scal[4];
    __shared__ int nanflag;
    const int cell = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const LimiterTab* tb = a.tab;
    const double gm1 = a.gam - 1.0;
    double* Uc = a.U + (size_t)cell * 5 * NP;
    if (tid == 0) nanflag = 0;
    __syncthreads();
    for (int i = tid; i < 5 * NP; i += NT) {
        const double v = Uc[i];
        sC[i] = v;
        if (isnan(v)) nanflag = 1;
    }
    __syncthreads();
    if (nanflag) return;   // the reference aborts on a NaN state (:430-442); the state is left as it is
    auto interp = [&](int d, int ns) {   // sQ[d][s] for s < ns, x then y then z
        const double* Ax = d == 0 ? tb->Bgll : tb->Bgl;
        const double* Ay = d == 1 ? tb->Bgll : tb->Bgl;
        const double* Az = d == 2 ? tb->Bgll : tb->Bgl;
        gl_pass<NT>(Ax, n, n, 0, n, n, n, sC, NP, t0, NP, ns, 1.0, false);
        __syncthreads();
        gl_pass<NT>(Ay, n, n, 1, n, n, n, t0, NP, t1, NP, ns, 1.0, false);
        __syncthreads();
        gl_pass<NT>(Az, n, n, 2, n, n, n, t1, NP, sQ + d * 5 * NP, NP, ns, 1.0, false);
        __syncthreads();
    };
    for (int d = 0; d < 3; ++d) interp(d, 5);
    // minimum density and maximum wave speed of each set (order-independent reductions)
    double mn = 1e6, ws[3] = {0.0, 0.0, 0.0};
    for (int i = tid; i < NP; i += NT) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (sC[i] < mn) mn = sC[i];
            const double* q = sQ + d * 5 * NP;
            if (q[i] < mn) mn = q[i];
            double u[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) u[s] = q[s * NP + i];
            double v2 = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) { const double v = u[1 + k] / u[0]; v2 += v * v; }
            const double w = sqrt(v2) + sqrt(limiter_pressure(u, gm1) * a.gam / u[0]);
            if (w > ws[d]) ws[d] = w;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
#pragma unroll
        for (int d = 0; d < 3; ++d) ws[d] = fmax(ws[d], __shfl_xor_sync(0xffffffffu, ws[d], o));
    }
    __shared__ double redmin[32];
    if (lane == 0) {
        redmin[warp] = mn;
#pragma unroll
        for (int d = 0; d < 3; ++d) red[d][warp] = ws[d];
    }
    // directional averages, each summed by one thread in the reference's order
    if (tid < 15) {
        const int d = tid / 5, s = tid % 5;
        const double* q = sQ + d * 5 * NP + s * NP;
        const double* wi = d == 0 ? tb->wgll : tb->wgl;
        const double* wj = d == 1 ? tb->wgll : tb->wgl;
        const double* wk = d == 2 ? tb->wgll : tb->wgl;
        double acc = 0.0;
        int qp = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                for (int k = 0; k < n; ++k) acc += wi[i] * wj[j] * wk[k] * q[qp];
                qp++;
            }
        avg_dim[d][s] = acc;
    }
    __syncthreads();
    if (tid == 0) {
        double m = 1e6, w[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < (NT + 31) / 32; ++i) {
            m = fmin(m, redmin[i]);
            for (int d = 0; d < 3; ++d) w[d] = fmax(w[d], red[d][i]);
        }
        const double mu = w[0] * a.lam + w[1] * a.lam + w[2] * a.lam;
        const double aw[3] = {(w[0] * a.lam) / mu, (w[1] * a.lam) / mu, (w[2] * a.lam) / mu};
        for (int s = 0; s < 5; ++s) {
            double v = aw[0] * avg_dim[0][s] + aw[1] * avg_dim[1][s];
            v += aw[2] * avg_dim[2][s];
            avg[s] = v;
        }
        const double p_avg = limiter_pressure(avg, gm1);
        double eps = fmin(fmin(a.min_density, avg[0]), p_avg);
        if (eps < 0) eps = a.min_density;
        double theta = 1.0;
        if (avg[0] - m > 1e-13) theta = (avg[0] - m == 0) ? 1.0 : fmin((avg[0] - eps) / (avg[0] - m), 1.0);
        if (theta < 0 || theta > 1) theta = 0;
        scal[0] = theta;
        scal[1] = p_avg;
    }
    __syncthreads();
    const double theta = scal[0], p_avg = scal[1];
    for (int i = tid; i < NP; i += NT) sC[i] = theta * (sC[i] - avg[0]) + avg[0];
    __syncthreads();
    for (int d = 0; d < 3; ++d) interp(d, 1);
    if (!a.zhang) {
        double th = 1.0;
        for (int i = tid; i < 4 * NP; i += NT) {
            const int set = i / NP, node = i % NP;
            const double* base = set < 3 ? sQ + set * 5 * NP : sC;
            double u[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) u[s] = base[s * NP + node];
            const double pl = limiter_pressure(u, gm1);
            const double t2 = (pl >= 0) ? 1.0 : p_avg / (p_avg - pl);
            if (t2 != 1 && t2 >= 0 && t2 <= 1 && t2 < th) th = t2;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) th = fmin(th, __shfl_xor_sync(0xffffffffu, th, o));
        if (lane == 0) redmin[warp] = th;
        __syncthreads();
        if (tid == 0) {
            double t = 1.0;
            for (int i = 0; i < (NT + 31) / 32; ++i) t = fmin(t, redmin[i]);
            scal[2] = t;
        }
        __syncthreads();
        const double theta2 = scal[2];
        for (int i = tid; i < 5 * NP; i += NT) {
            const int s = i / NP;
            Uc[i] = theta2 * (sC[i] - avg[s]) + avg[s];
        }
        return;
    }
    // Zhang 2010: theta2 per point of each set and per node; node i takes the smallest of the
    // four values with index i
    const double e = a.min_density / 1.4;
    for (int i = tid; i < 4 * NP; i += NT) {
        const int set = i / NP, node = i % NP;
        const double* base = set < 3 ? sQ + set * 5 * NP : sC;
        double u[5];
#pragma unroll
        for (int s = 0; s < 5; ++s) u[s] = base[s * NP + node];
        double t = 1.0;
        if (!(limiter_pressure(u, gm1) >= a.min_density)) {
            double s1 = (u[4] - avg[4]) * (u[0] - avg[0]) - 0.5 * ((u[1] - avg[1]) * (u[1] - avg[1]));
            double s2 = avg[0] * (u[4] - avg[4]) + avg[4] * (u[0] - avg[0]) - avg[1] * (u[1] - avg[1]) -
                        e * (u[0] - avg[0]);
            double s3 = (avg[4] * avg[0]) - 0.5 * (avg[1] * avg[1]) - e * avg[0];
            s1 -= 0.5 * ((u[2] - avg[2]) * (u[2] - avg[2]));
            s2 -= avg[2] * (u[2] - avg[2]);
            s3 -= 0.5 * (avg[2] * avg[2]);
            s1 -= 0.5 * ((u[3] - avg[3]) * (u[3] - avg[3]));
            s2 -= avg[3] * (u[3] - avg[3]);
            s3 -= 0.5 * (avg[3] * avg[3]);
            t = limiter_smallest_root(s3, s2, s1);
        }
        sT[i] = t;
    }
    __syncthreads();
    for (int i = tid; i < 5 * NP; i += NT) {
        const int s = i / NP, node = i % NP;
        double mq = 1e6;
#pragma unroll
        for (int d = 0; d < 3; ++d) if (sT[d * NP + node] < mq) mq = sT[d * NP + node];
        const double th = fmin(mq, sT[3 * NP + node]);
        Uc[i] = th * (sC[i] - avg[s]) + avg[s];
    }
}

} // namespace ph
