// Snapshot matrix on the device and its POD basis (OnlinePOD::addSnapshot / computeBasis,
// src/reduced_order/pod_basis_online.cpp:28-89, fed by FlowSolver::run every
// output_snapshot_every_x_timesteps, src/flow_solver/flow_solver.cpp:110-120, :675-679, and by
// the adaptive-sampling snapshot solves, src/reduced_order/adaptive_sampling_base.cpp:249).
//
// The snapshots stay resident as the columns of an ndofs x capacity matrix (column-major), each
// appended by a device copy from the solver's state, so no snapshot crosses to the host. The POD
// basis follows the reference's definition: reference state = the row mean, snapshots centred
// on it, the thin SVD's left singular vectors. It is computed by the method of snapshots: the
// Gram matrix G = Sc^T Sc (cuBLAS DSYRK), its eigen-decomposition G = V diag(sigma^2) V^T on the
// host (cyclic Jacobi rotations), then U = Sc V diag(1 / sigma) (cuBLAS DGEMM).
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <initializer_list>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/philip_b200.h"
#include "ph_internal.hpp"

using namespace ph_host;

#define PH_SCUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(PH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct ph_snapshots {
    size_t ndofs = 0;
    int capacity = 0, count = 0;
    double* d_S = nullptr;            // [capacity][ndofs]: column j at d_S + j * ndofs
    cudaStream_t stream = nullptr;
    cublasHandle_t blas = nullptr;
};

namespace {

__global__ void row_mean_kernel(const double* __restrict__ S, size_t ndofs, int m, double* __restrict__ mean) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < ndofs; i += (size_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < m; ++j) acc += S[(size_t)j * ndofs + i];
        mean[i] = acc / m;
    }
}

__global__ void center_kernel(const double* __restrict__ S, const double* __restrict__ mean, size_t ndofs, int m,
                              double* __restrict__ Sc) {
    const size_t n = ndofs * (size_t)m;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        Sc[k] = S[k] - mean[k % ndofs];
}

// per column: the index of the entry of largest magnitude (first such entry), for the sign rule
__global__ void column_argmax_kernel(const double* __restrict__ U, size_t ndofs, long long* __restrict__ idx,
                                     double* __restrict__ val) {
    const int col = blockIdx.x;
    const double* u = U + (size_t)col * ndofs;
    double best = -1.0;
    long long bi = 0;
    for (size_t i = threadIdx.x; i < ndofs; i += blockDim.x) {
        const double a = fabs(u[i]);
        if (a > best) { best = a; bi = (long long)i; }
    }
    __shared__ double sb[256];
    __shared__ long long si[256];
    sb[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double o = sb[threadIdx.x + s];
            const long long oi = si[threadIdx.x + s];
            if (o > sb[threadIdx.x] || (o == sb[threadIdx.x] && oi < si[threadIdx.x])) { sb[threadIdx.x] = o; si[threadIdx.x] = oi; }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { idx[col] = si[0]; val[col] = u[si[0]]; }
}

__global__ void scale_columns_kernel(double* __restrict__ U, size_t ndofs, int r, const double* __restrict__ sign) {
    const size_t n = ndofs * (size_t)r;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        U[k] *= sign[k / ndofs];
}

int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

// Eigen-decomposition of the symmetric m x m matrix A (row-major, overwritten) by cyclic Jacobi
// rotations (Golub and Van Loan, Matrix Computations, sec. 8.5): eigenvalues in w, eigenvectors
// in the columns of V (row-major m x m).
void jacobi_eigen(std::vector<double>& A, int m, std::vector<double>& w, std::vector<double>& V) {
    V.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; ++i) V[(size_t)i * m + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < m; ++i) {
            diag += A[(size_t)i * m + i] * A[(size_t)i * m + i];
            for (int j = i + 1; j < m; ++j) off += A[(size_t)i * m + j] * A[(size_t)i * m + j];
        }
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < m - 1; ++p)
            for (int q = p + 1; q < m; ++q) {
                const double apq = A[(size_t)p * m + q];
                if (apq == 0.0) continue;
                const double app = A[(size_t)p * m + p], aqq = A[(size_t)q * m + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < m; ++k) {   // A <- J^T A J
                    const double akp = A[(size_t)k * m + p], akq = A[(size_t)k * m + q];
                    A[(size_t)k * m + p] = c * akp - s * akq;
                    A[(size_t)k * m + q] = s * akp + c * akq;
                }
                for (int k = 0; k < m; ++k) {
                    const double apk = A[(size_t)p * m + k], aqk = A[(size_t)q * m + k];
                    A[(size_t)p * m + k] = c * apk - s * aqk;
                    A[(size_t)q * m + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < m; ++k) {
                    const double vkp = V[(size_t)k * m + p], vkq = V[(size_t)k * m + q];
                    V[(size_t)k * m + p] = c * vkp - s * vkq;
                    V[(size_t)k * m + q] = s * vkp + c * vkq;
                }
            }
    }
    w.resize(m);
    for (int i = 0; i < m; ++i) w[i] = A[(size_t)i * m + i];
}

int append(ph_snapshots* s, const double* src, cudaMemcpyKind kind, cudaStream_t stream) {
    if (s->count >= s->capacity) {   // grow: twice the columns, the old ones copied over
        const int cap = s->capacity * 2;
        double* d = nullptr;
        if (cudaMalloc((void**)&d, s->ndofs * (size_t)cap * sizeof(double)) != cudaSuccess)
            return fail(PH_ERR_NOMEM, "the snapshot matrix is full and cannot grow");
        PH_SCUDA(cudaMemcpyAsync(d, s->d_S, s->ndofs * (size_t)s->count * sizeof(double), cudaMemcpyDeviceToDevice,
                                 s->stream));
        PH_SCUDA(cudaStreamSynchronize(s->stream));
        cudaFree(s->d_S);
        s->d_S = d;
        s->capacity = cap;
    }
    PH_SCUDA(cudaMemcpyAsync(s->d_S + (size_t)s->count * s->ndofs, src, s->ndofs * sizeof(double), kind, stream));
    if (stream != s->stream) {   // later work on the matrix waits for this copy
        cudaEvent_t ev;
        PH_SCUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        PH_SCUDA(cudaEventRecord(ev, stream));
        PH_SCUDA(cudaStreamWaitEvent(s->stream, ev, 0));
        cudaEventDestroy(ev);
    }
    ++s->count;
    return PH_OK;
}

}  // namespace

extern "C" {

int ph_snapshots_create(int64_t ndofs, int capacity, ph_snapshots** out) {
    if (!out) return fail(PH_ERR_INVALID, "null argument");
    *out = nullptr;
    if (ndofs < 1 || capacity < 1) return fail(PH_ERR_INVALID, "ndofs and capacity must be positive");
    if (ndofs > INT_MAX) return fail(PH_ERR_INVALID, "ndofs above the 32-bit dimensions of the cuBLAS calls");
    ph_snapshots* s = new ph_snapshots();
    s->ndofs = (size_t)ndofs;
    s->capacity = capacity;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->d_S, s->ndofs * (size_t)capacity * sizeof(double));
    if (e != cudaSuccess) {
        ph_snapshots_destroy(s);
        return fail(e == cudaErrorMemoryAllocation ? PH_ERR_NOMEM : PH_ERR_CUDA, cudaGetErrorString(e));
    }
    if (cublasCreate(&s->blas) != CUBLAS_STATUS_SUCCESS) {
        ph_snapshots_destroy(s);
        return fail(PH_ERR_CUDA, "cublasCreate failed");
    }
    cublasSetStream(s->blas, s->stream);
    *out = s;
    return PH_OK;
}

int ph_snapshots_destroy(ph_snapshots* s) {
    if (!s) return PH_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->blas) cublasDestroy(s->blas);
    if (s->d_S) cudaFree(s->d_S);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return PH_OK;
}

int ph_snapshots_add(ph_snapshots* s, const double* U, int where) {
    if (!s || !U) return fail(PH_ERR_INVALID, "null argument");
    return append(s, U, where == PH_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s->stream);
}

int ph_snapshots_add_state(ph_snapshots* s, ph_ctx* ctx) {
    if (!s || !ctx) return fail(PH_ERR_INVALID, "null argument");
    const double* d = nullptr;
    size_t n = 0;
    cudaStream_t st = nullptr;
    if (int rc = ctx_state(ctx, &d, &n, &st)) return rc;
    if (n != s->ndofs) return fail(PH_ERR_INVALID, "the context's state size differs from the snapshot length");
    return append(s, d, cudaMemcpyDeviceToDevice, st);
}

int ph_snapshots_add_batch(ph_snapshots* s, ph_batch* b, int slot) {
    if (!s || !b) return fail(PH_ERR_INVALID, "null argument");
    const double* d = nullptr;
    size_t n = 0;
    cudaStream_t st = nullptr;
    if (int rc = batch_state(b, slot, &d, &n, &st)) return rc;
    if (n != s->ndofs) return fail(PH_ERR_INVALID, "the solve's state size differs from the snapshot length");
    return append(s, d, cudaMemcpyDeviceToDevice, st);
}

int ph_snapshots_count(const ph_snapshots* s, int* m) {
    if (!s || !m) return fail(PH_ERR_INVALID, "null argument");
    *m = s->count;
    return PH_OK;
}

int ph_snapshots_get(ph_snapshots* s, double* S, int where) {
    if (!s || !S) return fail(PH_ERR_INVALID, "null argument");
    const size_t bytes = s->ndofs * (size_t)s->count * sizeof(double);
    PH_SCUDA(cudaMemcpyAsync(S, s->d_S, bytes, where == PH_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                             s->stream));
    PH_SCUDA(cudaStreamSynchronize(s->stream));
    return PH_OK;
}

int ph_snapshots_pod(ph_snapshots* s, double rel_tol, double* reference_state, double* singular_values, double* basis,
                     int where, int* rank) {
    if (!s || !rank) return fail(PH_ERR_INVALID, "null argument");
    if (!(rel_tol >= 0.0)) return fail(PH_ERR_INVALID, "rel_tol must be >= 0");
    const int m = s->count;
    const size_t n = s->ndofs;
    *rank = 0;
    if (m < 1) return fail(PH_ERR_INVALID, "no snapshots");
    const cudaMemcpyKind out_kind = where == PH_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    double *d_mean = nullptr, *d_Sc = nullptr, *d_G = nullptr, *d_W = nullptr, *d_U = nullptr, *d_aux = nullptr;
    long long* d_idx = nullptr;
    auto release = [&] {
        cudaStreamSynchronize(s->stream);
        for (void* p : {(void*)d_mean, (void*)d_Sc, (void*)d_G, (void*)d_W, (void*)d_U, (void*)d_aux, (void*)d_idx})
            if (p) cudaFree(p);
    };
    int rc = PH_OK;
    cudaError_t e = cudaMalloc((void**)&d_mean, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_Sc, n * (size_t)m * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_G, (size_t)m * m * sizeof(double));
    if (e != cudaSuccess) { release(); return fail(PH_ERR_NOMEM, cudaGetErrorString(e)); }
    // reference state and centred snapshots (pod_basis_online.cpp:52-59)
    row_mean_kernel<<<grid_for(n), 256, 0, s->stream>>>(s->d_S, n, m, d_mean);
    center_kernel<<<grid_for(n * (size_t)m), 256, 0, s->stream>>>(s->d_S, d_mean, n, m, d_Sc);
    if ((e = cudaGetLastError()) != cudaSuccess) { release(); return fail(PH_ERR_CUDA, cudaGetErrorString(e)); }
    // G = Sc^T Sc, lower triangle (column-major m x m)
    const double one = 1.0, zero = 0.0;
    if (cublasDsyrk(s->blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, m, (int)n, &one, d_Sc, (int)n, &zero, d_G, m) !=
        CUBLAS_STATUS_SUCCESS) {
        release();
        return fail(PH_ERR_CUDA, "cublasDsyrk failed");
    }
    std::vector<double> G((size_t)m * m);
    e = cudaMemcpyAsync(G.data(), d_G, G.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && reference_state) e = cudaMemcpyAsync(reference_state, d_mean, n * sizeof(double), out_kind, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) { release(); return fail(PH_ERR_CUDA, cudaGetErrorString(e)); }
    std::vector<double> A((size_t)m * m);   // row-major symmetric copy of the lower triangle
    for (int j = 0; j < m; ++j)
        for (int i = j; i < m; ++i) A[(size_t)i * m + j] = A[(size_t)j * m + i] = G[(size_t)j * m + i];
    std::vector<double> w, V;
    jacobi_eigen(A, m, w, V);
    std::vector<int> order(m);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return w[a] > w[b]; });
    std::vector<double> sig(m);
    for (int k = 0; k < m; ++k) sig[k] = std::sqrt(std::max(w[order[k]], 0.0));
    int r = 0;
    while (r < m && sig[r] > rel_tol * sig[0] && sig[r] > 0.0) ++r;
    if (singular_values) for (int k = 0; k < m; ++k) singular_values[k] = k < r ? sig[k] : 0.0;
    *rank = r;
    if (basis && r > 0) {
        // W = V_r diag(1 / sigma_r) (column-major m x r); U = Sc W
        std::vector<double> W((size_t)m * r);
        for (int k = 0; k < r; ++k)
            for (int i = 0; i < m; ++i) W[(size_t)k * m + i] = V[(size_t)i * m + order[k]] / sig[k];
        e = cudaMalloc((void**)&d_W, W.size() * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc((void**)&d_U, n * (size_t)r * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc((void**)&d_aux, 2 * (size_t)r * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc((void**)&d_idx, (size_t)r * sizeof(long long));
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_W, W.data(), W.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream);
        if (e != cudaSuccess) { release(); return fail(PH_ERR_NOMEM, cudaGetErrorString(e)); }
        if (cublasDgemm(s->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, r, m, &one, d_Sc, (int)n, d_W, m, &zero, d_U, (int)n) !=
            CUBLAS_STATUS_SUCCESS) {
            release();
            return fail(PH_ERR_CUDA, "cublasDgemm failed");
        }
        // sign rule: the entry of largest magnitude of each basis vector is positive
        column_argmax_kernel<<<r, 256, 0, s->stream>>>(d_U, n, d_idx, d_aux);
        std::vector<double> val(r), sign(r);
        e = cudaMemcpyAsync(val.data(), d_aux, r * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) { release(); return fail(PH_ERR_CUDA, cudaGetErrorString(e)); }
        for (int k = 0; k < r; ++k) sign[k] = val[k] < 0.0 ? -1.0 : 1.0;
        e = cudaMemcpyAsync(d_aux + r, sign.data(), r * sizeof(double), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) {
            scale_columns_kernel<<<grid_for(n * (size_t)r), 256, 0, s->stream>>>(d_U, n, r, d_aux + r);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(basis, d_U, n * (size_t)r * sizeof(double), out_kind, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) rc = fail(PH_ERR_CUDA, cudaGetErrorString(e));
    }
    release();
    return rc;
}

}  // extern "C"
