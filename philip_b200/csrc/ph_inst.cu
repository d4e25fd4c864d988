// Explicit instantiation of the kernels for one polynomial order. Compiled once per
// N1 (= p + 1) with -DPH_N1=<N1>.
#include "ph_launch.cuh"

#ifndef PH_N1
#error "PH_N1 must be defined"
#endif

namespace ph {

template <int N1> constexpr int cells_per_cta() { return N1 == 2 ? 16 : N1 == 3 ? 4 : N1 == 4 ? 2 : 1; }

template <typename R, int N1, bool VISC, bool SPLIT, int FS, bool CURV = false, bool BND = false>
static cudaError_t launch_one(const StageArgs& a, cudaStream_t s) {
    constexpr int CPC = cells_per_cta<N1>();
    using L = Layout<R, N1, CPC, VISC, SPLIT, CURV>;
    auto kern = residual_kernel<R, N1, CPC, VISC, SPLIT, FS, CURV, BND>;
    int dev = 0;
    cudaGetDevice(&dev);
    static bool configured[64] = {false};
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    const int grid = a.tiles ? a.ntiles : (a.nc - a.cell_begin + CPC - 1) / CPC;
    if (grid <= 0) return a.tiles ? cudaSuccess : cudaErrorInvalidValue;
    kern<<<grid, L::NT, L::bytes, s>>>(a);
    return cudaGetLastError();
}

template <typename R, int N1>
static cudaError_t launch_prec(const StageArgs& a, bool visc, bool split, cudaStream_t s) {
    // the Chandrashekar + EC/Roe (+ BR2) combination has its own compile-time instance; the
    // relaxation RK's entropy estimate lives in the generic instance only
    const bool hot = split && a.pc.two_point == TP_CH && a.pc.conv_flux == CF_EC_ROE &&
                     (!visc || a.pc.diss_flux == DF_BR2) && a.ent_partial == nullptr;
    if (a.btype && a.metric) {   // boundary faces of curvilinear cells
        if (visc) return split ? launch_one<R, N1, true, true, 0, true, true>(a, s)
                               : launch_one<R, N1, true, false, 0, true, true>(a, s);
        return split ? launch_one<R, N1, false, true, 0, true, true>(a, s)
                     : launch_one<R, N1, false, false, 0, true, true>(a, s);
    }
    if (a.btype) {    // boundary faces (affine cells)
        if (visc) {
            if (split) return hot ? launch_one<R, N1, true, true, 1, false, true>(a, s)
                                  : launch_one<R, N1, true, true, 0, false, true>(a, s);
            return launch_one<R, N1, true, false, 0, false, true>(a, s);
        }
        if (split) return hot ? launch_one<R, N1, false, true, 1, false, true>(a, s)
                              : launch_one<R, N1, false, true, 0, false, true>(a, s);
        return launch_one<R, N1, false, false, 0, false, true>(a, s);
    }
    if (a.metric) {   // curvilinear cells
        if (!split) return visc ? launch_one<R, N1, true, false, 0, true>(a, s) : launch_one<R, N1, false, false, 0, true>(a, s);
        if (visc) return hot ? launch_one<R, N1, true, true, 1, true>(a, s) : launch_one<R, N1, true, true, 0, true>(a, s);
        return hot ? launch_one<R, N1, false, true, 1, true>(a, s) : launch_one<R, N1, false, true, 0, true>(a, s);
    }
    if (visc) {
        if (split) return hot ? launch_one<R, N1, true, true, 1>(a, s) : launch_one<R, N1, true, true, 0>(a, s);
        return launch_one<R, N1, true, false, 0>(a, s);
    }
    if (split) return hot ? launch_one<R, N1, false, true, 1>(a, s) : launch_one<R, N1, false, true, 0>(a, s);
    return launch_one<R, N1, false, false, 0>(a, s);
}

template <int N1>
cudaError_t launch_stage(const StageArgs& a, int fp32, bool visc, bool split, cudaStream_t s) {
    return fp32 ? launch_prec<float, N1>(a, visc, split, s) : launch_prec<double, N1>(a, visc, split, s);
}

// ---- batched stage kernels: tile-shape variants per order (cells per CTA)
template <int N1> constexpr int batched_variants() { return (N1 == 2 || N1 >= 6) ? 1 : 2; }
template <int N1, int V> constexpr int batched_cpc() {
    return N1 == 2 ? 16 : N1 == 3 ? (V == 0 ? 4 : 8) : N1 == 4 ? (V == 0 ? 2 : 4) : N1 == 5 ? (V == 0 ? 1 : 2) : 1;
}

template <typename R, int N1, int V, int FS, bool CURV, bool BND>
static cudaError_t launch_batched_one(const StageArgs* inst, const BatchTile* tiles, int ntiles, int grid,
                                      cudaStream_t s) {
    constexpr int CPC = batched_cpc<N1, V>();
    using L = Layout<R, N1, CPC, false, true, CURV>;
    auto kern = residual_kernel_batched<R, N1, CPC, false, true, FS, CURV, BND>;
    int dev = 0;
    cudaGetDevice(&dev);
    static bool configured[64] = {false};
    static int resident[64] = {0};
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, L::NT, L::bytes);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        resident[dev] = per_sm * sms;
        configured[dev] = true;
    }
    if (ntiles <= 0) return cudaSuccess;
    if (grid <= 0) grid = resident[dev < 64 ? dev : 0];
    if (grid <= 0 || grid > ntiles) grid = ntiles;
    kern<<<grid, L::NT, L::bytes, s>>>(inst, tiles, ntiles);
    return cudaGetLastError();
}

template <typename R, int N1, int V, bool BND>
static cudaError_t launch_batched_vb(const StageArgs* inst, const BatchTile* tiles, int ntiles, bool curv, bool hot,
                                     int grid, cudaStream_t s) {
    if (curv) return hot ? launch_batched_one<R, N1, V, 1, true, BND>(inst, tiles, ntiles, grid, s)
                         : launch_batched_one<R, N1, V, 0, true, BND>(inst, tiles, ntiles, grid, s);
    return hot ? launch_batched_one<R, N1, V, 1, false, BND>(inst, tiles, ntiles, grid, s)
               : launch_batched_one<R, N1, V, 0, false, BND>(inst, tiles, ntiles, grid, s);
}

template <typename R, int N1, int V>
static cudaError_t launch_batched_v(const StageArgs* inst, const BatchTile* tiles, int ntiles, bool curv, bool hot,
                                    bool bnd, int grid, cudaStream_t s) {
    return bnd ? launch_batched_vb<R, N1, V, true>(inst, tiles, ntiles, curv, hot, grid, s)
               : launch_batched_vb<R, N1, V, false>(inst, tiles, ntiles, curv, hot, grid, s);
}

template <typename R, int N1>
static cudaError_t launch_batched_prec(const StageArgs* inst, const BatchTile* tiles, int ntiles, bool curv, bool hot,
                                       bool bnd, int variant, int grid, cudaStream_t s) {
    if constexpr (batched_variants<N1>() > 1) {
        if (variant == 1) return launch_batched_v<R, N1, 1>(inst, tiles, ntiles, curv, hot, bnd, grid, s);
    }
    if (variant != 0) return cudaErrorInvalidValue;
    return launch_batched_v<R, N1, 0>(inst, tiles, ntiles, curv, hot, bnd, grid, s);
}

template <int N1>
cudaError_t launch_stage_batched(const StageArgs* inst, const BatchTile* tiles, int ntiles, int fp32, bool curv,
                                 bool hot, int variant, int grid, cudaStream_t s, bool bnd) {
    return fp32 ? launch_batched_prec<float, N1>(inst, tiles, ntiles, curv, hot, bnd, variant, grid, s)
                : launch_batched_prec<double, N1>(inst, tiles, ntiles, curv, hot, bnd, variant, grid, s);
}

template <typename R, int N1, int V, bool CURV>
static bool batched_shape_one(int* cpc, int* threads, size_t* smem, int* ctas_per_sm) {
    constexpr int CPC = batched_cpc<N1, V>();
    using L = Layout<R, N1, CPC, false, true, CURV>;
    *cpc = CPC; *threads = L::NT; *smem = L::bytes;
    auto kern = residual_kernel_batched<R, N1, CPC, false, true, 1, CURV>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes) != cudaSuccess) return false;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, kern, L::NT, L::bytes) == cudaSuccess;
}

template <typename R, int N1>
static bool batched_shape_prec(bool curv, int variant, int* cpc, int* threads, size_t* smem, int* ctas_per_sm) {
    if constexpr (batched_variants<N1>() > 1) {
        if (variant == 1) return curv ? batched_shape_one<R, N1, 1, true>(cpc, threads, smem, ctas_per_sm)
                                      : batched_shape_one<R, N1, 1, false>(cpc, threads, smem, ctas_per_sm);
    }
    if (variant != 0) return false;
    return curv ? batched_shape_one<R, N1, 0, true>(cpc, threads, smem, ctas_per_sm)
                : batched_shape_one<R, N1, 0, false>(cpc, threads, smem, ctas_per_sm);
}

template <int N1>
bool batched_shape(int fp32, bool curv, int variant, int* cpc, int* threads, size_t* smem, int* ctas_per_sm) {
    return fp32 ? batched_shape_prec<float, N1>(curv, variant, cpc, threads, smem, ctas_per_sm)
                : batched_shape_prec<double, N1>(curv, variant, cpc, threads, smem, ctas_per_sm);
}

template <typename R, int N1, bool VISC, bool SPLIT>
static void shape_one(int* threads, int* cpc, size_t* smem) {  // same shape for every flux set
    constexpr int CPC = cells_per_cta<N1>();
    using L = Layout<R, N1, CPC, VISC, SPLIT>;
    *threads = L::NT; *cpc = CPC; *smem = L::bytes;
}

template <int N1>
void stage_launch_shape(int fp32, bool visc, bool split, int* threads, int* cpc, size_t* smem) {
    if (fp32) {
        if (visc) split ? shape_one<float, N1, true, true>(threads, cpc, smem) : shape_one<float, N1, true, false>(threads, cpc, smem);
        else split ? shape_one<float, N1, false, true>(threads, cpc, smem) : shape_one<float, N1, false, false>(threads, cpc, smem);
    } else {
        if (visc) split ? shape_one<double, N1, true, true>(threads, cpc, smem) : shape_one<double, N1, true, false>(threads, cpc, smem);
        else split ? shape_one<double, N1, false, true>(threads, cpc, smem) : shape_one<double, N1, false, false>(threads, cpc, smem);
    }
}

template <typename R, int N1, bool FRA, bool CURV, bool BND = false>
static cudaError_t launch_aux_prec(const double* U, const int* nbr, const OpTab& ops, int cell_begin, int nc,
                                   double inv_h, const PhysConst& pc, void* Fv, const double* metric, cudaStream_t s,
                                   const BoundaryArgs* bnd = nullptr) {
    constexpr int CPC = cells_per_cta<N1>();
    using L = AuxLayout<N1, CPC, FRA>;
    constexpr size_t bytes = L::template bytes<R>();
    auto kern = aux_kernel<R, N1, CPC, FRA, CURV, BND>;
    int dev = 0;
    cudaGetDevice(&dev);
    static bool configured[64] = {false};
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    AuxCoef<R> co{};
    for (int i = 0; i < MAXN1 * MAXN1; ++i) { co.D[i] = (R)ops.D[i]; co.Ba[i] = (R)ops.Baux[i]; }
    co.inv_wend = R(1) / (R)ops.w[0];
    const int* tiles = bnd ? bnd->tiles : nullptr;
    const int grid = tiles ? bnd->ntiles : (nc - cell_begin + CPC - 1) / CPC;
    if (grid <= 0) return tiles ? cudaSuccess : cudaErrorInvalidValue;
    kern<<<grid, L::NT, bytes, s>>>(U, nbr, cell_begin, nc, CURV ? R(1) : (R)inv_h, pc, co, static_cast<R*>(Fv),
                                    metric, bnd ? bnd->btype : nullptr, bnd ? static_cast<R*>(bnd->Fb) : nullptr,
                                    bnd ? (R)bnd->pen : R(0), tiles);
    return cudaGetLastError();
}

template <int N1>
cudaError_t launch_aux(const double* U, const int* nbr, const OpTab& ops, int cell_begin, int nc, double inv_h,
                       const PhysConst& pc, int fp32, void* Fv, const double* metric, cudaStream_t s,
                       const BoundaryArgs* bnd) {
    if (bnd && bnd->btype && metric) {   // the boundary tiles of curvilinear cells (kDG)
        if (ops.aux_fr) return cudaErrorInvalidValue;
        return fp32 ? launch_aux_prec<float, N1, false, true, true>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, metric, s, bnd)
                    : launch_aux_prec<double, N1, false, true, true>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, metric, s, bnd);
    }
    if (bnd && bnd->btype) {   // the boundary tiles (affine cells)
        if (ops.aux_fr)
            return fp32 ? launch_aux_prec<float, N1, true, false, true>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, nullptr, s, bnd)
                        : launch_aux_prec<double, N1, true, false, true>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, nullptr, s, bnd);
        return fp32 ? launch_aux_prec<float, N1, false, false, true>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, nullptr, s, bnd)
                    : launch_aux_prec<double, N1, false, false, true>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, nullptr, s, bnd);
    }
    if (metric) {   // curvilinear cells (kDG, checked by the host)
        if (ops.aux_fr) return cudaErrorInvalidValue;
        return fp32 ? launch_aux_prec<float, N1, false, true>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, metric, s, bnd)
                    : launch_aux_prec<double, N1, false, true>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, metric, s, bnd);
    }
    if (ops.aux_fr)   // (bnd without btype: the periodic kernel over bnd->tiles)
        return fp32 ? launch_aux_prec<float, N1, true, false>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, nullptr, s, bnd)
                    : launch_aux_prec<double, N1, true, false>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, nullptr, s, bnd);
    return fp32 ? launch_aux_prec<float, N1, false, false>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, nullptr, s, bnd)
                : launch_aux_prec<double, N1, false, false>(U, nbr, ops, cell_begin, nc, inv_h, pc, Fv, nullptr, s, bnd);
}

template <int N1>
cudaError_t launch_inverse_mass(const double* in, double* out, const OpTab* ops, int nc, double inv_detj,
                                const double* metric, int fr, cudaStream_t s) {
    inverse_mass_kernel<N1><<<nc, 128, 0, s>>>(in, out, ops, nc, inv_detj, metric, fr);
    return cudaGetLastError();
}

template <int N1, bool CURV, bool FULL>
static cudaError_t launch_integrals_one(const double* U, const double* X, const double* origin, const IntegralTab* tab,
                                       int nc, const IntegralConst& ic, double* partial, cudaStream_t s) {
    auto kern = integrals_kernel<N1, CURV, FULL>;
    constexpr size_t bytes = integrals_smem_bytes<N1, CURV, FULL>();
    int dev = 0;
    cudaGetDevice(&dev);
    static bool configured[64] = {false};
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    kern<<<nc, 256, bytes, s>>>(U, X, origin, tab, nc, ic, partial);
    return cudaGetLastError();
}

template <int N1>
cudaError_t launch_integrals(const double* U, const double* X, const double* origin, const IntegralTab* tab, int nc,
                             const IntegralConst& ic, bool full, double* partial, cudaStream_t s) {
    if constexpr (integrals_affine_fits<N1>()) {
        if (!full && !X) {   // affine cells, the three partials: the hoisted-contraction kernel
            auto kern = integrals_affine_kernel<N1>;
            constexpr size_t bytes = integrals_affine_smem_bytes<N1>();
            int dev = 0;
            cudaGetDevice(&dev);
            static bool configured[64] = {false};
            if (dev < 64 && !configured[dev]) {
                cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
                if (e != cudaSuccess) return e;
                configured[dev] = true;
            }
            kern<<<nc, AFF_THREADS, bytes, s>>>(U, tab, nc, ic, partial);
            return cudaGetLastError();
        }
    }
    if (full)
        return X ? launch_integrals_one<N1, true, true>(U, X, origin, tab, nc, ic, partial, s)
                 : launch_integrals_one<N1, false, true>(U, X, origin, tab, nc, ic, partial, s);
    return X ? launch_integrals_one<N1, true, false>(U, X, origin, tab, nc, ic, partial, s)
             : launch_integrals_one<N1, false, false>(U, X, origin, tab, nc, ic, partial, s);
}

template <int N1>
cudaError_t launch_rrk_entropy(const double* Un, const double* U1, double gamma, const OpTab* ops, int nc, double h3,
                               const double* metric, double gam, double* partial, cudaStream_t s) {
    constexpr int NP = N1 * N1 * N1;
    rrk_entropy_kernel<N1><<<nc, ((NP + 31) / 32) * 32, 0, s>>>(Un, U1, gamma, ops, nc, h3, metric, gam, partial);
    return cudaGetLastError();
}

template cudaError_t launch_rrk_entropy<PH_N1>(const double*, const double*, double, const OpTab*, int, double,
                                               const double*, double, double*, cudaStream_t);
template cudaError_t launch_stage<PH_N1>(const StageArgs&, int, bool, bool, cudaStream_t);
template void stage_launch_shape<PH_N1>(int, bool, bool, int*, int*, size_t*);
template cudaError_t launch_stage_batched<PH_N1>(const StageArgs*, const BatchTile*, int, int, bool, bool, int, int,
                                                 cudaStream_t, bool);
template bool batched_shape<PH_N1>(int, bool, int, int*, int*, size_t*, int*);
template cudaError_t launch_aux<PH_N1>(const double*, const int*, const OpTab&, int, int, double, const PhysConst&, int,
                                       void*, const double*, cudaStream_t, const BoundaryArgs*);
template cudaError_t launch_inverse_mass<PH_N1>(const double*, double*, const OpTab*, int, double, const double*, int,
                                                cudaStream_t);
template cudaError_t launch_integrals<PH_N1>(const double*, const double*, const double*, const IntegralTab*, int,
                                             const IntegralConst&, bool, double*, cudaStream_t);

// ---- uncollocated path
template <typename K>
static cudaError_t launch_gl_kernel(K kern, size_t bytes, int threads, const StageArgs& a, const GlArgs& g,
                                   const GlTab& ht, bool& configured, cudaStream_t s) {
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int grid = a.tiles ? a.ntiles : a.nc - a.cell_begin;
    if (grid <= 0) return a.tiles ? cudaSuccess : cudaErrorInvalidValue;
    kern<<<grid, threads, bytes, s>>>(a, g, ht);
    return cudaGetLastError();
}

template <int ND, int NQ>
static cudaError_t launch_gl_nq(int kernel, const StageArgs& a, const GlArgs& g, const GlTab& ht, bool visc,
                                bool split, cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    constexpr int NT = gl_threads<NQ>();
    static bool cfg[27][64] = {};
    if (kernel == 0) {
        if (split) return launch_gl_kernel(gl_trace_kernel<ND, NQ, true>, GlTraceLayout<ND, NQ, true>::bytes, NT, a, g, ht,
                                           cfg[0][dev], s);
        return launch_gl_kernel(gl_trace_kernel<ND, NQ, false>, GlTraceLayout<ND, NQ, false>::bytes, NT, a, g, ht,
                                cfg[1][dev], s);
    }
    if (kernel == 1) {
        if (g.vmet && a.btype) {   // curvilinear cells with a boundary face
            if (split) return launch_gl_kernel(gl_aux_kernel<ND, NQ, true, true, true>, GlAuxLayout<ND, NQ, true>::bytes,
                                               NT, a, g, ht, cfg[21][dev], s);
            return launch_gl_kernel(gl_aux_kernel<ND, NQ, false, true, true>, GlAuxLayout<ND, NQ, false>::bytes, NT, a,
                                    g, ht, cfg[22][dev], s);
        }
        if (g.vmet) {   // curvilinear cells
            if (split) return launch_gl_kernel(gl_aux_kernel<ND, NQ, true, true>, GlAuxLayout<ND, NQ, true>::bytes, NT, a,
                                               g, ht, cfg[11][dev], s);
            return launch_gl_kernel(gl_aux_kernel<ND, NQ, false, true>, GlAuxLayout<ND, NQ, false>::bytes, NT, a, g, ht,
                                    cfg[12][dev], s);
        }
        if (a.btype) {   // the cells with a boundary face
            if (split) return launch_gl_kernel(gl_aux_kernel<ND, NQ, true, false, true>, GlAuxLayout<ND, NQ, true>::bytes,
                                               NT, a, g, ht, cfg[15][dev], s);
            return launch_gl_kernel(gl_aux_kernel<ND, NQ, false, false, true>, GlAuxLayout<ND, NQ, false>::bytes, NT, a,
                                    g, ht, cfg[16][dev], s);
        }
        if (split) return launch_gl_kernel(gl_aux_kernel<ND, NQ, true>, GlAuxLayout<ND, NQ, true>::bytes, NT, a, g, ht,
                                           cfg[2][dev], s);
        return launch_gl_kernel(gl_aux_kernel<ND, NQ, false>, GlAuxLayout<ND, NQ, false>::bytes, NT, a, g, ht,
                                cfg[3][dev], s);
    }
    if (kernel == 3)   // curvilinear: the weight-adjusted inverse mass alone
        return launch_gl_kernel(gl_minv_kernel<ND, NQ>, GlMinvLayout<ND, NQ>::bytes, NT, a, g, ht, cfg[8][dev], s);
    if (g.vmet && a.btype) {   // curvilinear cells with a boundary face
        if (visc) {
            if (split) return launch_gl_kernel(gl_stage_kernel<ND, NQ, true, true, true, true>,
                                               GlStageLayout<ND, NQ, true, true, true>::bytes, NT, a, g, ht, cfg[23][dev],
                                               s);
            return launch_gl_kernel(gl_stage_kernel<ND, NQ, true, false, true, true>,
                                    GlStageLayout<ND, NQ, true, false, true>::bytes, NT, a, g, ht, cfg[24][dev], s);
        }
        if (split) return launch_gl_kernel(gl_stage_kernel<ND, NQ, false, true, true, true>,
                                           GlStageLayout<ND, NQ, false, true, true>::bytes, NT, a, g, ht, cfg[25][dev], s);
        return launch_gl_kernel(gl_stage_kernel<ND, NQ, false, false, true, true>,
                                GlStageLayout<ND, NQ, false, false, true>::bytes, NT, a, g, ht, cfg[26][dev], s);
    }
    if (g.vmet) {      // curvilinear cells
        if (visc) {
            if (split) return launch_gl_kernel(gl_stage_kernel<ND, NQ, true, true, true>,
                                               GlStageLayout<ND, NQ, true, true, true>::bytes, NT, a, g, ht, cfg[13][dev],
                                               s);
            return launch_gl_kernel(gl_stage_kernel<ND, NQ, true, false, true>,
                                    GlStageLayout<ND, NQ, true, false, true>::bytes, NT, a, g, ht, cfg[14][dev], s);
        }
        if (split) return launch_gl_kernel(gl_stage_kernel<ND, NQ, false, true, true>,
                                           GlStageLayout<ND, NQ, false, true, true>::bytes, NT, a, g, ht, cfg[9][dev], s);
        return launch_gl_kernel(gl_stage_kernel<ND, NQ, false, false, true>,
                                GlStageLayout<ND, NQ, false, false, true>::bytes, NT, a, g, ht, cfg[10][dev], s);
    }
    if (a.btype) {     // the cells with a boundary face
        if (visc) {
            if (split) return launch_gl_kernel(gl_stage_kernel<ND, NQ, true, true, false, true>,
                                               GlStageLayout<ND, NQ, true, true>::bytes, NT, a, g, ht, cfg[17][dev], s);
            return launch_gl_kernel(gl_stage_kernel<ND, NQ, true, false, false, true>,
                                    GlStageLayout<ND, NQ, true, false>::bytes, NT, a, g, ht, cfg[18][dev], s);
        }
        if (split) return launch_gl_kernel(gl_stage_kernel<ND, NQ, false, true, false, true>,
                                           GlStageLayout<ND, NQ, false, true>::bytes, NT, a, g, ht, cfg[19][dev], s);
        return launch_gl_kernel(gl_stage_kernel<ND, NQ, false, false, false, true>,
                                GlStageLayout<ND, NQ, false, false>::bytes, NT, a, g, ht, cfg[20][dev], s);
    }
    if (visc) {
        if (split) return launch_gl_kernel(gl_stage_kernel<ND, NQ, true, true>, GlStageLayout<ND, NQ, true, true>::bytes,
                                           NT, a, g, ht, cfg[4][dev], s);
        return launch_gl_kernel(gl_stage_kernel<ND, NQ, true, false>, GlStageLayout<ND, NQ, true, false>::bytes, NT, a,
                                g, ht, cfg[5][dev], s);
    }
    if (split) return launch_gl_kernel(gl_stage_kernel<ND, NQ, false, true>, GlStageLayout<ND, NQ, false, true>::bytes,
                                       NT, a, g, ht, cfg[6][dev], s);
    return launch_gl_kernel(gl_stage_kernel<ND, NQ, false, false>, GlStageLayout<ND, NQ, false, false>::bytes, NT, a,
                            g, ht, cfg[7][dev], s);
}

template <int N1>
cudaError_t launch_gl(int kernel, int nq, const StageArgs& a, const GlArgs& g, const GlTab& ht, bool visc, bool split,
                      cudaStream_t s) {
    if (nq == N1) return launch_gl_nq<N1, N1>(kernel, a, g, ht, visc, split, s);
    if constexpr (N1 + 1 <= GL_MAXQ) {
        if (nq == N1 + 1) return launch_gl_nq<N1, N1 + 1>(kernel, a, g, ht, visc, split, s);
    }
    if constexpr (N1 + 2 <= GL_MAXQ) {
        if (nq == N1 + 2) return launch_gl_nq<N1, N1 + 2>(kernel, a, g, ht, visc, split, s);
    }
    return cudaErrorInvalidValue;
}
template <int ND, int NQ>
static cudaError_t launch_gl_rrk_entropy_nq(const double* Un, const double* U1, double gamma, const GlTab& ht, int nc,
                                            double h3, const double* vmet, double gam, double* partial, cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    static bool configured[64] = {};
    auto kern = gl_rrk_entropy_kernel<ND, NQ>;
    constexpr size_t bytes = GlEntropyLayout<ND, NQ>::bytes;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (nc <= 0) return cudaErrorInvalidValue;
    kern<<<nc, gl_threads<NQ>(), bytes, s>>>(Un, U1, gamma, ht, h3, vmet, gam, partial);
    return cudaGetLastError();
}

template <int N1>
cudaError_t launch_gl_rrk_entropy(int nq, const double* Un, const double* U1, double gamma, const GlTab& ht, int nc,
                                  double h3, const double* vmet, double gam, double* partial, cudaStream_t s) {
    if (nq == N1) return launch_gl_rrk_entropy_nq<N1, N1>(Un, U1, gamma, ht, nc, h3, vmet, gam, partial, s);
    if constexpr (N1 + 1 <= GL_MAXQ) {
        if (nq == N1 + 1) return launch_gl_rrk_entropy_nq<N1, N1 + 1>(Un, U1, gamma, ht, nc, h3, vmet, gam, partial, s);
    }
    if constexpr (N1 + 2 <= GL_MAXQ) {
        if (nq == N1 + 2) return launch_gl_rrk_entropy_nq<N1, N1 + 2>(Un, U1, gamma, ht, nc, h3, vmet, gam, partial, s);
    }
    return cudaErrorInvalidValue;
}
template cudaError_t launch_gl_rrk_entropy<PH_N1>(int, const double*, const double*, double, const GlTab&, int, double,
                                                  const double*, double, double*, cudaStream_t);

template cudaError_t launch_gl<PH_N1>(int, int, const StageArgs&, const GlArgs&, const GlTab&, bool, bool,
                                      cudaStream_t);

template <int N1>
cudaError_t launch_limiter(const LimiterArgs& a, cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    static bool configured[64] = {false};
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(limiter_kernel<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)limiter_smem<N1>());
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (a.nc <= 0) return cudaErrorInvalidValue;
    limiter_kernel<N1><<<a.nc, limiter_threads<N1>(), limiter_smem<N1>(), s>>>(a);
    return cudaGetLastError();
}
template cudaError_t launch_limiter<PH_N1>(const LimiterArgs&, cudaStream_t);

template <int N1>
cudaError_t launch_ke_rate(const double* U, const double* K, const IntegralTab* tab, int nc, double h3,
                           double* partial, cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    static bool configured[64] = {false};
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(ke_rate_kernel<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)ke_rate_smem<N1>());
        if (e != cudaSuccess) return e;
        configured[dev] = true;
    }
    if (nc <= 0) return cudaErrorInvalidValue;
    ke_rate_kernel<N1><<<nc, ke_rate_threads<N1>(), ke_rate_smem<N1>(), s>>>(U, K, tab, nc, h3, partial);
    return cudaGetLastError();
}
template cudaError_t launch_ke_rate<PH_N1>(const double*, const double*, const IntegralTab*, int, double, double*,
                                           cudaStream_t);

} // namespace ph
