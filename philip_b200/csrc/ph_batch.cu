// Batch of independent explicit solves on one GPU: the served / parameter-swept form.
//
// Memory. One device arena of the HBM budget is reserved when the batch is created; every
// admitted solve takes one contiguous, 256-byte aligned range of it (state, RK stage
// vectors, metric terms, neighbour table, operator table, status word) from a first-fit
// free list, and gives it back when released. Admission never calls cudaMalloc.
//
// Work. For every RK stage, all unfinished solves of one (order, mesh kind, flux set) group
// run as ONE persistent launch of residual_kernel_batched over a tile list (instance, first
// cell). The stage arguments of every solve live in a device table [stage][slot]. One RK
// step of all groups is captured as a CUDA graph whose groups are parallel branches (they
// share nothing), replayed step after step; the graph and the tile list are rebuilt only
// when a solve joins or finishes (continuous batching). All copies and launches are ordered
// on the batch stream, so a range that a finished solve gives back is reused only after the
// work that read it.
//
// Tile shapes. Each (order, precision, mesh kind) has 1-2 cells-per-CTA variants; the
// autotuner times them on a synthetic solve and keeps the fastest for the process.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/philip_b200.h"
#include "ph_internal.hpp"
#include "ph_launch.cuh"

using namespace ph_host;

#define PH_BCUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(PH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

constexpr size_t ALIGN = 256;
constexpr int MAX_SLOTS = 4096;
constexpr int MAX_STAGES = 4;
constexpr int MAX_BRANCHES = 16;

size_t align_up(size_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }

// byte offsets of one solve's arrays inside its arena range
struct SlotLayout {
    size_t sol, stA, stB, acc, carry, comp, metric, nbr, btype, ops, status, total;
};

// boundary faces of a mesh: n^2 on every non-periodic side
int boundary_face_count(const ph_mesh_desc* mesh) {
    const int n = mesh->n_cells_per_direction;
    int nb = 0;
    for (int f = 0; f < 6; ++f)
        if (mesh->boundary_type[f] != 0) nb += n * n;
    return nb;
}

SlotLayout slot_layout(size_t ndofs, int nc, int NP, bool curv, bool carry, bool comp, int nb) {
    SlotLayout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o = align_up(o + bytes); return at; };
    const size_t vec = ndofs * sizeof(double);
    L.sol = take(vec); L.stA = take(vec); L.stB = take(vec); L.acc = take(vec);
    L.carry = carry ? take(vec) : SIZE_MAX;
    L.comp = comp ? take(vec) : SIZE_MAX;
    L.metric = curv ? take((size_t)nc * 10 * NP * sizeof(double)) : SIZE_MAX;
    L.nbr = take((size_t)nc * 6 * sizeof(int));
    L.btype = nb > 0 ? take((size_t)nb * sizeof(int)) : SIZE_MAX;
    L.ops = take(sizeof(ph::OpTab));
    L.status = take(sizeof(unsigned));
    L.total = o;
    return L;
}

// tile-shape choice per (N1, precision, curvilinear) for the process; -1 = not chosen yet
int g_variant[8][2][2];
bool g_variant_init = false;
std::mutex g_variant_mu;

int variant_of(int N1, int fp32, int curv) {
    std::lock_guard<std::mutex> lk(g_variant_mu);
    if (!g_variant_init) {
        for (auto& a : g_variant) for (auto& b : a) for (int& v : b) v = -1;
        g_variant_init = true;
    }
    return g_variant[N1][fp32][curv];
}
void set_variant(int N1, int fp32, int curv, int v) {
    variant_of(N1, fp32, curv);
    std::lock_guard<std::mutex> lk(g_variant_mu);
    g_variant[N1][fp32][curv] = v;
}

cudaError_t launch_group(int N1, const ph::StageArgs* inst, const ph::BatchTile* tiles, int ntiles, int fp32,
                         bool curv, bool hot, int variant, cudaStream_t s, bool bnd = false) {
    switch (N1) {
    case 2: return ph::launch_stage_batched<2>(inst, tiles, ntiles, fp32, curv, hot, variant, 0, s, bnd);
    case 3: return ph::launch_stage_batched<3>(inst, tiles, ntiles, fp32, curv, hot, variant, 0, s, bnd);
    case 4: return ph::launch_stage_batched<4>(inst, tiles, ntiles, fp32, curv, hot, variant, 0, s, bnd);
    case 5: return ph::launch_stage_batched<5>(inst, tiles, ntiles, fp32, curv, hot, variant, 0, s, bnd);
    case 6: return ph::launch_stage_batched<6>(inst, tiles, ntiles, fp32, curv, hot, variant, 0, s, bnd);
    case 7: return ph::launch_stage_batched<7>(inst, tiles, ntiles, fp32, curv, hot, variant, 0, s, bnd);
    }
    return cudaErrorInvalidValue;
}

bool shape_of(int N1, int fp32, bool curv, int variant, int* cpc, int* threads, size_t* smem, int* per_sm) {
    switch (N1) {
    case 2: return ph::batched_shape<2>(fp32, curv, variant, cpc, threads, smem, per_sm);
    case 3: return ph::batched_shape<3>(fp32, curv, variant, cpc, threads, smem, per_sm);
    case 4: return ph::batched_shape<4>(fp32, curv, variant, cpc, threads, smem, per_sm);
    case 5: return ph::batched_shape<5>(fp32, curv, variant, cpc, threads, smem, per_sm);
    case 6: return ph::batched_shape<6>(fp32, curv, variant, cpc, threads, smem, per_sm);
    case 7: return ph::batched_shape<7>(fp32, curv, variant, cpc, threads, smem, per_sm);
    }
    return false;
}

int cells_per_tile(int N1, int fp32, bool curv, int variant) {
    int cpc = 1, threads = 0, per_sm = 0;
    size_t smem = 0;
    if (!shape_of(N1, fp32, curv, variant, &cpc, &threads, &smem, &per_sm)) return 0;
    return cpc;
}

struct Slot {
    bool used = false, finished = false;
    int N1 = 0, NP = 0, nc = 0, ns = 0;
    bool curv = false, hot = false, bnd = false;
    size_t ndofs = 0, off = 0, bytes = 0;
    int nsteps = 0, done = 0;
    cudaEvent_t done_ev = nullptr;      // recorded after the step that finishes the solve
    bool done_recorded = false;
    RkBuffers B{};
    unsigned* status = nullptr;
    ph::StageArgs args[MAX_STAGES];
};

struct Group {
    int N1 = 0;
    bool curv = false, hot = false, bnd = false;
    int variant = 0, ns = 0;
    size_t tile_off = 0;
    int ntiles = 0;
};

// TGV nodal state (initial_condition_function.cpp:261-310) for the autotuner's solve
void tgv_state(const std::vector<double>& xyz, int nc, int NP, double gam, double mach, std::vector<double>& U) {
    U.assign((size_t)nc * 5 * NP, 0.0);
    for (int c = 0; c < nc; ++c)
        for (int q = 0; q < NP; ++q) {
            const double* X = &xyz[((size_t)c * NP + q) * 3];
            const double x = X[0], y = X[1], z = X[2];
            const double u = std::sin(x) * std::cos(y) * std::cos(z), v = -std::cos(x) * std::sin(y) * std::cos(z);
            const double p = 1.0 / (gam * mach * mach) + (std::cos(2 * x) + std::cos(2 * y)) * (std::cos(2 * z) + 2) / 16.0;
            double* Uc = &U[(size_t)c * 5 * NP];
            Uc[q] = 1.0; Uc[NP + q] = u; Uc[2 * NP + q] = v; Uc[3 * NP + q] = 0.0;
            Uc[4 * NP + q] = p / (gam - 1.0) + 0.5 * (u * u + v * v);
        }
}

} // namespace

struct ph_batch {
    cudaStream_t stream = nullptr;
    int device = 0;
    int fp32 = 0;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    std::map<size_t, size_t> free_blocks;   // offset -> bytes
    std::vector<Slot> slots;
    ph::StageArgs* d_args = nullptr;        // [MAX_STAGES][MAX_SLOTS]
    ph::BatchTile* d_tiles = nullptr;
    size_t tiles_cap = 0;
    std::vector<Group> groups;
    bool dirty = true;
    cudaGraphExec_t graph = nullptr;
    std::vector<cudaGraphExec_t> retired;   // replaced graphs, destroyed after the next synchronisation
    cudaStream_t branch[MAX_BRANCHES] = {};
    cudaStream_t copy = nullptr;            // read-back of finished solves, waits on their events only
    std::vector<cudaEvent_t> fences;        // ring of step fences handed to the caller
    long long fence_next = 0;
    // pinned staging ring for uploads: a pageable source would make an asynchronous copy
    // wait for the work already queued on the stream
    char* stage = nullptr;
    size_t stage_cap = 0, stage_head = 0;
    struct Pending { size_t off, bytes; cudaEvent_t ev; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> spare_events;
    bool own_stream = false;
    cudaEvent_t ev_fork = nullptr, ev_join[MAX_BRANCHES] = {};
    long long launches = 0;
    int launches_per_step = 0;
};

namespace {

bool arena_alloc(ph_batch* b, size_t bytes, size_t& off) {
    for (auto it = b->free_blocks.begin(); it != b->free_blocks.end(); ++it) {
        if (it->second < bytes) continue;
        off = it->first;
        const size_t rest = it->second - bytes;
        b->free_blocks.erase(it);
        if (rest) b->free_blocks[off + bytes] = rest;
        return true;
    }
    return false;
}

void arena_free(ph_batch* b, size_t off, size_t bytes) {
    auto it = b->free_blocks.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != b->free_blocks.end() && it->first + it->second == next->first) {
        it->second += next->second;
        b->free_blocks.erase(next);
    }
    if (it != b->free_blocks.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            b->free_blocks.erase(it);
        }
    }
}

void destroy_retired(ph_batch* b) {
    for (auto g : b->retired) cudaGraphExecDestroy(g);
    b->retired.clear();
}

// Copy `bytes` from host memory to the device through the pinned staging ring, ordered on
// the batch stream; returns once the source may be reused. The ring space of earlier
// uploads is reclaimed when their copies have completed.
int staged_upload(ph_batch* b, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return PH_OK;
    if (bytes > b->stage_cap) {   // larger than the ring: a plain (possibly waiting) copy
        PH_BCUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, b->stream));
        return PH_OK;
    }
    const size_t need = align_up(bytes);
    size_t off = b->stage_head;
    if (off + need > b->stage_cap) off = 0;
    // wait for (and retire) the pending copies that overlap [off, off + need)
    for (size_t i = 0; i < b->pending.size();) {
        const auto& pd = b->pending[i];
        if (pd.off < off + need && off < pd.off + pd.bytes) {
            PH_BCUDA(cudaEventSynchronize(pd.ev));
            b->spare_events.push_back(pd.ev);
            b->pending.erase(b->pending.begin() + i);
        } else {
            ++i;
        }
    }
    std::memcpy(b->stage + off, src, bytes);
    PH_BCUDA(cudaMemcpyAsync(dst, b->stage + off, bytes, cudaMemcpyHostToDevice, b->stream));
    cudaEvent_t ev = nullptr;
    if (!b->spare_events.empty()) { ev = b->spare_events.back(); b->spare_events.pop_back(); }
    else PH_BCUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    PH_BCUDA(cudaEventRecord(ev, b->stream));
    b->pending.push_back({off, need, ev});
    b->stage_head = off + need;
    return PH_OK;
}

// Rebuild the tile lists of the unfinished solves and capture one RK step as a graph.
int rebuild(ph_batch* b) {
    std::map<std::tuple<int, int, int, int>, std::vector<ph::BatchTile>> lists;
    std::map<std::tuple<int, int, int, int>, Group> info;
    for (int s = 0; s < (int)b->slots.size(); ++s) {
        const Slot& sl = b->slots[s];
        if (!sl.used || sl.finished) continue;
        const auto key = std::make_tuple(sl.N1, (int)sl.curv, (int)sl.hot, (int)sl.bnd);
        Group& g = info[key];
        if (g.N1 == 0) {
            g.N1 = sl.N1; g.curv = sl.curv; g.hot = sl.hot; g.bnd = sl.bnd; g.ns = sl.ns;
            g.variant = std::max(0, variant_of(sl.N1, b->fp32, sl.curv));
        }
        g.ns = std::max(g.ns, sl.ns);
        const int cpc = cells_per_tile(sl.N1, b->fp32, sl.curv, g.variant);
        if (cpc <= 0) return fail(PH_ERR_CUDA, "batched kernel shape query failed");
        auto& L = lists[key];
        for (int c0 = 0; c0 < sl.nc; c0 += cpc) L.push_back(ph::BatchTile{s, c0});
    }
    std::vector<ph::BatchTile> all;
    b->groups.clear();
    for (auto& kv : lists) {
        Group g = info[kv.first];
        g.tile_off = all.size();
        g.ntiles = (int)kv.second.size();
        all.insert(all.end(), kv.second.begin(), kv.second.end());
        b->groups.push_back(g);
    }
    if ((int)b->groups.size() > MAX_BRANCHES) return fail(PH_ERR_UNSUPPORTED, "too many (order, mesh, flux) groups");
    if (all.size() > b->tiles_cap) {
        if (b->d_tiles) PH_BCUDA(cudaFreeAsync(b->d_tiles, b->stream));
        b->tiles_cap = std::max(all.size(), 2 * b->tiles_cap);
        PH_BCUDA(cudaMallocAsync((void**)&b->d_tiles, b->tiles_cap * sizeof(ph::BatchTile), b->stream));
    }
    if (int rc = staged_upload(b, b->d_tiles, all.data(), all.size() * sizeof(ph::BatchTile))) return rc;
    // configure every kernel before capture (attributes and occupancy are not stream work)
    for (const Group& g : b->groups)
        PH_BCUDA(launch_group(g.N1, b->d_args, b->d_tiles, 0, b->fp32, g.curv, g.hot, g.variant, b->stream, g.bnd));
    if (b->graph) { b->retired.push_back(b->graph); b->graph = nullptr; }
    b->launches_per_step = 0;
    if (!b->groups.empty()) {
        cudaGraph_t graph = nullptr;
        PH_BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaEventRecord(b->ev_fork, b->stream);
        for (int gi = 0; gi < (int)b->groups.size() && e == cudaSuccess; ++gi) {
            const Group& g = b->groups[gi];
            cudaStream_t st = b->branch[gi];
            e = cudaStreamWaitEvent(st, b->ev_fork, 0);
            for (int i = 0; i < g.ns && e == cudaSuccess; ++i) {
                e = launch_group(g.N1, b->d_args + (size_t)i * MAX_SLOTS, b->d_tiles + g.tile_off, g.ntiles, b->fp32,
                                 g.curv, g.hot, g.variant, st, g.bnd);
                ++b->launches_per_step;
            }
            if (e == cudaSuccess) e = cudaEventRecord(b->ev_join[gi], st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->ev_join[gi], 0);
        }
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return fail(PH_ERR_CUDA, std::string("batch graph capture: ") +
                                         cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        e = cudaGraphInstantiate(&b->graph, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(PH_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e));
    }
    if (b->retired.size() > 8) {   // bound the retired graphs: they are idle after a synchronisation
        PH_BCUDA(cudaStreamSynchronize(b->stream));
        destroy_retired(b);
    }
    b->dirty = false;
    return PH_OK;
}

int check_batch_params(const ph_batch* b, const ph_mesh_desc* mesh, const ph_params* prm) {
    if (int rc = check_mesh(mesh)) return rc;
    if (const char* why = boundary_reason(mesh, prm)) return fail(PH_ERR_UNSUPPORTED, why);
    if (const char* why = unsupported_reason(mesh, prm)) return fail(PH_ERR_UNSUPPORTED, why);
    if (prm->pde_type != 0 || !prm->use_split_form)
        return fail(PH_ERR_UNSUPPORTED, "a batch takes split-form Euler solves");
    if (prm->runge_kutta_method < 0 || prm->runge_kutta_method > 2)
        return fail(PH_ERR_UNSUPPORTED, "a batch takes rk4_ex, ssprk3_ex or heun2_ex");
    if (prm->use_relaxation_runge_kutta)
        return fail(PH_ERR_UNSUPPORTED, "a batch takes fixed-step solves (no relaxation RK)");
    if (prm->bound_preserving_limiter != 0) return fail(PH_ERR_UNSUPPORTED, "a batch takes solves without a limiter");
    if (prm->two_point_num_flux_type < 0 || prm->two_point_num_flux_type > 3 || prm->conv_num_flux < 0 ||
        prm->conv_num_flux > 5)
        return fail(PH_ERR_INVALID, "parameter out of range");
    if (b && (prm->precision == PH_FP32_RESIDUAL) != (b->fp32 != 0))
        return fail(PH_ERR_INVALID, "the solve's precision differs from the batch's");
    return PH_OK;
}

} // namespace

extern "C" {

int ph_batch_create(size_t hbm_budget_bytes, int precision, void* cuda_stream, ph_batch** out) {
    if (!out) return fail(PH_ERR_INVALID, "null argument");
    *out = nullptr;
    if (hbm_budget_bytes < ALIGN) return fail(PH_ERR_INVALID, "budget too small");
    ph_batch* b = new ph_batch();
    b->stream = (cudaStream_t)cuda_stream;
    b->fp32 = precision == PH_FP32_RESIDUAL ? 1 : 0;
    cudaGetDevice(&b->device);
    b->arena_bytes = align_up(hbm_budget_bytes);
    cudaError_t e = cudaSuccess;
    if (!b->stream) {   // graphs cannot be captured on the legacy default stream
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        b->own_stream = e == cudaSuccess;
    }
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->arena, b->arena_bytes);
    b->stage_cap = std::min<size_t>(b->arena_bytes, (size_t)512 << 20);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&b->stage, b->stage_cap, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_args, sizeof(ph::StageArgs) * MAX_STAGES * MAX_SLOTS);
    for (int i = 0; i < MAX_BRANCHES && e == cudaSuccess; ++i) {
        e = cudaStreamCreateWithFlags(&b->branch[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->copy, cudaStreamNonBlocking);
    b->fences.assign(64, nullptr);
    for (auto& f : b->fences)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        ph_batch_destroy(b);
        return fail(e == cudaErrorMemoryAllocation ? PH_ERR_NOMEM : PH_ERR_CUDA,
                    std::string("batch creation: ") + cudaGetErrorString(e));
    }
    b->free_blocks[0] = b->arena_bytes;
    *out = b;
    return PH_OK;
}

int ph_batch_destroy(ph_batch* b) {
    if (!b) return PH_OK;
    if (b->stream || b->arena) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    destroy_retired(b);
    if (b->d_tiles) cudaFree(b->d_tiles);
    if (b->d_args) cudaFree(b->d_args);
    if (b->arena) cudaFree(b->arena);
    for (int i = 0; i < MAX_BRANCHES; ++i) {
        if (b->branch[i]) cudaStreamDestroy(b->branch[i]);
        if (b->ev_join[i]) cudaEventDestroy(b->ev_join[i]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->copy) cudaStreamDestroy(b->copy);
    for (auto& pd : b->pending) cudaEventDestroy(pd.ev);
    for (auto ev : b->spare_events) cudaEventDestroy(ev);
    if (b->stage) cudaFreeHost(b->stage);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    for (auto f : b->fences) if (f) cudaEventDestroy(f);
    for (auto& sl : b->slots) if (sl.done_ev) cudaEventDestroy(sl.done_ev);
    delete b;
    return PH_OK;
}

int ph_batch_bytes(const ph_mesh_desc* mesh, const ph_params* prm, size_t* bytes) {
    if (!mesh || !prm || !bytes) return fail(PH_ERR_INVALID, "null argument");
    if (int rc = check_batch_params(nullptr, mesh, prm)) return rc;
    const int n = mesh->n_cells_per_direction, nc = n * n * n, N1 = prm->poly_degree + 1, NP = N1 * N1 * N1;
    const SlotLayout L = slot_layout((size_t)nc * 5 * NP, nc, NP, is_curvilinear(mesh), prm->runge_kutta_method == 1,
                                     prm->precision == PH_FP32_RESIDUAL, boundary_face_count(mesh));
    *bytes = L.total;
    return PH_OK;
}

}  // extern "C"

int ph_host::batch_prepare(const ph_mesh_desc* mesh, const ph_params* prm, BatchPrep& out) {
    if (!mesh || !prm) return fail(PH_ERR_INVALID, "null argument");
    if (int rc = check_batch_params(nullptr, mesh, prm)) return rc;
    std::vector<double> x, D, xyz;
    std::vector<int> ijk;
    int rc = build_operators(prm, out.ops, out.fr, x, D);
    if (!rc) {
        periodic_connectivity(mesh->n_cells_per_direction, mesh->cell_order, ijk, out.nbr);
        out.btype.clear();
        if (has_boundaries(mesh)) apply_boundaries(mesh->n_cells_per_direction, ijk, mesh->boundary_type, out.nbr, out.btype);
        rc = node_geometry(mesh->n_cells_per_direction, ijk, x, D, mesh->left, mesh->right, mesh->warp, xyz,
                           out.metric, mesh->mapping_support_points);
    }
    out.ready = rc == PH_OK;
    return rc;
}

int ph_host::batch_admit_prepared(ph_batch* b, const ph_mesh_desc* mesh, const ph_params* prm, const BatchPrep* prep,
                                  const double* U0, double dt, int nsteps, int* slot) {
    if (!b || !mesh || !prm || !U0 || !slot) return fail(PH_ERR_INVALID, "null argument");
    *slot = -1;
    if (int rc = check_batch_params(b, mesh, prm)) return rc;
    if (nsteps < 0 || !(dt > 0.0)) return fail(PH_ERR_INVALID, "dt must be > 0 and nsteps >= 0");
    const int n = mesh->n_cells_per_direction, nc = n * n * n, N1 = prm->poly_degree + 1, NP = N1 * N1 * N1;
    const bool curv = is_curvilinear(mesh);
    const size_t ndofs = (size_t)nc * 5 * NP;
    int ns = 0;
    double A[4][4], bw[4];
    rk_tableau(prm->runge_kutta_method, ns, A, bw);
    const int nb = boundary_face_count(mesh);
    const SlotLayout L = slot_layout(ndofs, nc, NP, curv, ns == 3, b->fp32 != 0, nb);
    size_t off = 0;
    if (!arena_alloc(b, L.total, off)) return fail(PH_ERR_NOMEM, "the batch's HBM budget has no room for this solve now");
    // the tile shape of this (order, mesh kind): tuned once per process
    if (variant_of(N1, b->fp32, curv) < 0) {
        int best = 0, nv = 0;
        double ms[4];
        cudaStreamSynchronize(b->stream);
        if (ph_batch_autotune(prm->poly_degree, b->fp32 ? PH_FP32_RESIDUAL : PH_FP64, curv ? 1 : 0, &best, ms, &nv))
            set_variant(N1, b->fp32, curv, 0);
    }
    // host set-up: operators, connectivity, geometry (here, unless the caller prepared them)
    BatchPrep local;
    if (!prep || !prep->ready) {
        if (int rc = batch_prepare(mesh, prm, local)) { arena_free(b, off, L.total); return rc; }
        prep = &local;
    }
    const ph::OpTab& ops = prep->ops;
    const bool fr = prep->fr;
    const std::vector<int>& nbr = prep->nbr;
    const std::vector<int>& btype = prep->btype;
    const std::vector<double>& metric = prep->metric;
    if ((int)btype.size() != nb) { arena_free(b, off, L.total); return fail(PH_ERR_INVALID, "the prepared mesh differs"); }
    int s = -1;
    for (int i = 0; i < (int)b->slots.size(); ++i)
        if (!b->slots[i].used) { s = i; break; }
    if (s < 0) {
        if ((int)b->slots.size() >= MAX_SLOTS) { arena_free(b, off, L.total); return fail(PH_ERR_NOMEM, "too many solves"); }
        s = (int)b->slots.size();
        b->slots.emplace_back();
    }
    Slot& sl = b->slots[s];
    const cudaEvent_t kept_ev = sl.done_ev;
    sl = Slot();
    sl.done_ev = kept_ev;
    sl.used = true;
    sl.N1 = N1; sl.NP = NP; sl.nc = nc; sl.ns = ns; sl.curv = curv; sl.bnd = nb > 0;
    sl.hot = prm->two_point_num_flux_type == ph::TP_CH && prm->conv_num_flux == ph::CF_EC_ROE;
    sl.ndofs = ndofs; sl.off = off; sl.bytes = L.total;
    sl.nsteps = nsteps; sl.done = 0; sl.finished = (nsteps == 0);
    char* base = b->arena + off;
    auto ptr = [&](size_t o) { return o == SIZE_MAX ? nullptr : (double*)(base + o); };
    sl.B = RkBuffers{ptr(L.sol), ptr(L.stA), ptr(L.stB), ptr(L.acc), ptr(L.carry), ptr(L.comp)};
    sl.status = (unsigned*)(base + L.status);
    double* d_metric = ptr(L.metric);
    int* d_nbr = (int*)(base + L.nbr);
    int* d_btype = nb > 0 ? (int*)(base + L.btype) : nullptr;
    ph::OpTab* d_ops = (ph::OpTab*)(base + L.ops);
    const double h = (mesh->right - mesh->left) / n;
    double pen = 0.0;
    const ph::PhysConst pc = physics_constants(prm, h, pen);
    for (int i = 0; i < ns; ++i) {
        ph::StageArgs& a = sl.args[i];
        std::memset(&a, 0, sizeof(a));
        a.U = rk_stage_input(sl.B, i);
        a.nbr = d_nbr; a.ops = d_ops; a.nc = nc;
        a.h = h; a.inv_h = 1.0 / h; a.pen = pen; a.pc = pc; a.status = sl.status;
        a.fr = fr ? 1 : 0;
        a.metric = d_metric;
        a.btype = d_btype;   // (Euler: no boundary viscous flux, a.Fb stays null)
        rk_stage_args(a, sl.B, i, ns, A, bw, dt, b->fp32 != 0);
    }
    // uploads through the pinned ring, ordered on the batch stream after the work already queued
    int up = staged_upload(b, sl.B.sol, U0, ndofs * sizeof(double));
    if (!up) up = staged_upload(b, d_nbr, nbr.data(), nbr.size() * sizeof(int));
    if (!up && d_btype) up = staged_upload(b, d_btype, btype.data(), btype.size() * sizeof(int));
    if (!up) up = staged_upload(b, d_ops, &ops, sizeof(ops));
    if (!up && d_metric) up = staged_upload(b, d_metric, metric.data(), metric.size() * sizeof(double));
    for (int i = 0; i < ns && !up; ++i)
        up = staged_upload(b, b->d_args + (size_t)i * MAX_SLOTS + s, &sl.args[i], sizeof(ph::StageArgs));
    if (up) { arena_free(b, off, L.total); sl = Slot(); return up; }
    if (sl.B.comp) PH_BCUDA(cudaMemsetAsync(sl.B.comp, 0, ndofs * sizeof(double), b->stream));
    PH_BCUDA(cudaMemsetAsync(sl.status, 0, sizeof(unsigned), b->stream));
    if (sl.finished) {   // nothing to step: complete once its state is uploaded
        if (!sl.done_ev) PH_BCUDA(cudaEventCreateWithFlags(&sl.done_ev, cudaEventDisableTiming));
        PH_BCUDA(cudaEventRecord(sl.done_ev, b->stream));
        sl.done_recorded = true;
    }
    if (!sl.finished) b->dirty = true;
    *slot = s;
    return PH_OK;
}

int ph_host::batch_state(ph_batch* b, int slot, const double** d, size_t* n, cudaStream_t* stream) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) return fail(PH_ERR_INVALID, "bad slot");
    *d = b->slots[slot].B.sol; *n = b->slots[slot].ndofs; *stream = b->stream;
    return PH_OK;
}

extern "C" {

int ph_batch_admit(ph_batch* b, const ph_mesh_desc* mesh, const ph_params* prm, const double* U0, double dt,
                   int nsteps, int* slot) {
    return batch_admit_prepared(b, mesh, prm, nullptr, U0, dt, nsteps, slot);
}

int ph_batch_step(ph_batch* b, int nsteps) {
    if (!b) return fail(PH_ERR_INVALID, "null argument");
    int remaining = nsteps;
    while (remaining > 0) {
        int k = remaining, active = 0;
        for (const Slot& sl : b->slots)
            if (sl.used && !sl.finished) { ++active; k = std::min(k, sl.nsteps - sl.done); }
        if (!active) break;
        if (b->dirty)
            if (int rc = rebuild(b)) return rc;
        for (int r = 0; r < k; ++r) PH_BCUDA(cudaGraphLaunch(b->graph, b->stream));
        b->launches += (long long)k * b->launches_per_step;
        for (Slot& sl : b->slots)
            if (sl.used && !sl.finished) {
                sl.done += k;
                if (sl.done >= sl.nsteps) {
                    sl.finished = true;
                    b->dirty = true;
                    if (!sl.done_ev) PH_BCUDA(cudaEventCreateWithFlags(&sl.done_ev, cudaEventDisableTiming));
                    PH_BCUDA(cudaEventRecord(sl.done_ev, b->stream));
                    sl.done_recorded = true;
                }
            }
        remaining -= k;
    }
    return PH_OK;
}

int ph_batch_progress(ph_batch* b, int slot, int* steps_done, int* nsteps) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) return fail(PH_ERR_INVALID, "bad slot");
    if (steps_done) *steps_done = b->slots[slot].done;
    if (nsteps) *nsteps = b->slots[slot].nsteps;
    return PH_OK;
}

int ph_batch_active(ph_batch* b, int* active) {
    if (!b || !active) return fail(PH_ERR_INVALID, "null argument");
    int n = 0;
    for (const Slot& sl : b->slots) n += (sl.used && !sl.finished) ? 1 : 0;
    *active = n;
    return PH_OK;
}

int ph_batch_get_state(ph_batch* b, int slot, double* U) {
    if (!b || !U || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
        return fail(PH_ERR_INVALID, "bad slot");
    const Slot& sl = b->slots[slot];
    if (sl.finished && sl.done_recorded) {
        // wait for this solve's last step only, not for the work queued after it
        PH_BCUDA(cudaStreamWaitEvent(b->copy, sl.done_ev, 0));
        PH_BCUDA(cudaMemcpyAsync(U, sl.B.sol, sl.ndofs * sizeof(double), cudaMemcpyDeviceToHost, b->copy));
        PH_BCUDA(cudaStreamSynchronize(b->copy));
        return PH_OK;
    }
    PH_BCUDA(cudaMemcpyAsync(U, sl.B.sol, sl.ndofs * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    PH_BCUDA(cudaStreamSynchronize(b->stream));
    destroy_retired(b);
    return PH_OK;
}

int ph_batch_status(ph_batch* b, int slot, uint32_t* flags) {
    if (!b || !flags || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
        return fail(PH_ERR_INVALID, "bad slot");
    unsigned v = 0;
    const Slot& sl = b->slots[slot];
    PH_BCUDA(cudaMemcpyAsync(&v, sl.status, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream));
    PH_BCUDA(cudaMemsetAsync(sl.status, 0, sizeof(unsigned), b->stream));
    PH_BCUDA(cudaStreamSynchronize(b->stream));
    *flags = v;
    return PH_OK;
}

int ph_batch_release(ph_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) return fail(PH_ERR_INVALID, "bad slot");
    Slot& sl = b->slots[slot];
    if (!sl.finished) b->dirty = true;
    arena_free(b, sl.off, sl.bytes);
    cudaEvent_t ev = sl.done_ev;   // events are reused by the slot's next solve
    sl = Slot();
    sl.done_ev = ev;
    return PH_OK;
}

int ph_batch_poll(ph_batch* b, int slot, int* complete) {
    if (!b || !complete || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
        return fail(PH_ERR_INVALID, "bad slot");
    const Slot& sl = b->slots[slot];
    *complete = 0;
    if (!sl.finished || !sl.done_recorded) return PH_OK;
    const cudaError_t e = cudaEventQuery(sl.done_ev);
    if (e == cudaSuccess) *complete = 1;
    else if (e != cudaErrorNotReady) return fail(PH_ERR_CUDA, cudaGetErrorString(e));
    return PH_OK;
}

int ph_batch_fence(ph_batch* b, long long* ticket) {
    if (!b || !ticket) return fail(PH_ERR_INVALID, "null argument");
    const long long t = b->fence_next++;
    PH_BCUDA(cudaEventRecord(b->fences[t % b->fences.size()], b->stream));
    *ticket = t;
    return PH_OK;
}

int ph_batch_fence_wait(ph_batch* b, long long ticket) {
    if (!b || ticket < 0 || ticket >= b->fence_next) return fail(PH_ERR_INVALID, "bad ticket");
    if (b->fence_next - ticket > (long long)b->fences.size()) return PH_OK;   // long past: its event was reused
    PH_BCUDA(cudaEventSynchronize(b->fences[ticket % b->fences.size()]));
    return PH_OK;
}

int ph_mesh_node_xyz(const ph_mesh_desc* mesh, int poly_degree, double* xyz) {
    if (!mesh || !xyz) return fail(PH_ERR_INVALID, "null argument");
    if (poly_degree < 1 || poly_degree > 6) return fail(PH_ERR_UNSUPPORTED, "poly_degree must be 1..6");
    if (int rc = check_mesh(mesh)) return rc;
    ph_params prm{};
    prm.poly_degree = poly_degree;
    ph::OpTab ops;
    bool fr;
    std::vector<double> x, D, X, metric;
    std::vector<int> ijk, nbr;
    if (int rc = build_operators(&prm, ops, fr, x, D)) return rc;
    periodic_connectivity(mesh->n_cells_per_direction, mesh->cell_order, ijk, nbr);
    if (int rc = node_geometry(mesh->n_cells_per_direction, ijk, x, D, mesh->left, mesh->right, mesh->warp, X, metric,
                               mesh->mapping_support_points))
        return rc;
    std::memcpy(xyz, X.data(), X.size() * sizeof(double));
    return PH_OK;
}

int ph_batch_launches(ph_batch* b, long long* launches) {
    if (!b || !launches) return fail(PH_ERR_INVALID, "null argument");
    *launches = b->launches;
    return PH_OK;
}

int ph_batch_set_variant(int poly_degree, int precision, int curvilinear, int variant) {
    const int N1 = poly_degree + 1;
    if (N1 < 2 || N1 > 7) return fail(PH_ERR_UNSUPPORTED, "poly_degree must be 1..6");
    const int fp32 = precision == PH_FP32_RESIDUAL ? 1 : 0;
    if (cells_per_tile(N1, fp32, curvilinear != 0, variant) <= 0) return fail(PH_ERR_INVALID, "no such tile variant");
    set_variant(N1, fp32, curvilinear ? 1 : 0, variant);
    return PH_OK;
}

int ph_batch_autotune(int poly_degree, int precision, int curvilinear, int* best, double ms[4], int* nvariants) {
    const int N1 = poly_degree + 1;
    if (N1 < 2 || N1 > 7) return fail(PH_ERR_UNSUPPORTED, "poly_degree must be 1..6");
    const int fp32 = precision == PH_FP32_RESIDUAL ? 1 : 0;
    const bool curv = curvilinear != 0;
    int nv = 0;
    while (nv < 4 && cells_per_tile(N1, fp32, curv, nv) > 0) ++nv;
    if (nvariants) *nvariants = nv;
    // synthetic solve: TGV on the periodic cube, large enough to fill the GPU several times
    const int n = poly_degree <= 3 ? 24 : 16;
    ph_mesh_desc mesh{n, 0, 0.0, 2.0 * M_PI, curv ? 0.1 : 0.0, poly_degree, nullptr};
    ph_params prm{};
    prm.poly_degree = poly_degree; prm.flux_nodes_type = 1; prm.pde_type = 0; prm.use_split_form = 1;
    prm.two_point_num_flux_type = ph::TP_CH; prm.conv_num_flux = ph::CF_EC_ROE; prm.diss_num_flux = 0;
    prm.runge_kutta_method = 0; prm.precision = precision; prm.gamma_gas = 1.4; prm.mach_infinity = 0.1;
    prm.reynolds_number_inf = 1600.0; prm.prandtl_number = 0.71; prm.temperature_inf = 273.15;
    prm.sipg_penalty_factor = 1.0; prm.nondimensionalized_constant_viscosity = 1.0;
    prm.rk_atol = 1e-3; prm.rk_rtol = 1e-3;
    prm.pressure_shift = 1.0 / (1.4 * 0.1 * 0.1);
    size_t bytes = 0;
    if (int rc = ph_batch_bytes(&mesh, &prm, &bytes)) return rc;
    cudaStream_t s = nullptr;
    PH_BCUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    ph_batch* b = nullptr;
    int rc = ph_batch_create(bytes, precision, s, &b);
    std::vector<double> U, xyz, metric, x, D;
    int slot = -1;
    if (!rc) {
        ph::OpTab ops;
        bool fr;
        std::vector<int> ijk, nbr;
        rc = build_operators(&prm, ops, fr, x, D);
        if (!rc) {
            periodic_connectivity(n, 0, ijk, nbr);
            rc = node_geometry(n, ijk, x, D, mesh.left, mesh.right, mesh.warp, xyz, metric);
        }
        if (!rc) {
            tgv_state(xyz, n * n * n, N1 * N1 * N1, prm.gamma_gas, prm.mach_infinity, U);
            set_variant(N1, fp32, curv, 0);   // admission must not recurse into the tuner
            rc = ph_batch_admit(b, &mesh, &prm, U.data(), 1e-4, 1, &slot);
        }
    }
    double best_ms = 1e300;
    int best_v = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!rc) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        const Slot& sl = b->slots[slot];
        for (int v = 0; v < nv && !rc; ++v) {
            const int cpc = cells_per_tile(N1, fp32, curv, v);
            std::vector<ph::BatchTile> tiles;
            for (int c0 = 0; c0 < sl.nc; c0 += cpc) tiles.push_back(ph::BatchTile{slot, c0});
            ph::BatchTile* d_tiles = nullptr;
            if (cudaMalloc((void**)&d_tiles, tiles.size() * sizeof(ph::BatchTile)) != cudaSuccess) {
                rc = fail(PH_ERR_NOMEM, "autotune tiles");
                break;
            }
            cudaMemcpy(d_tiles, tiles.data(), tiles.size() * sizeof(ph::BatchTile), cudaMemcpyHostToDevice);
            const int nt = (int)tiles.size();
            cudaError_t e = cudaSuccess;
            for (int r = 0; r < 3 && e == cudaSuccess; ++r)
                e = launch_group(N1, b->d_args, d_tiles, nt, fp32, curv, true, v, s);
            cudaEventRecord(e0, s);
            const int reps = 10;
            for (int r = 0; r < reps && e == cudaSuccess; ++r)
                e = launch_group(N1, b->d_args, d_tiles, nt, fp32, curv, true, v, s);
            cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float t = 0.f;
            if (e == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
            cudaFree(d_tiles);
            if (e != cudaSuccess) { rc = fail(PH_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e)); break; }
            const double per = (double)t / reps;
            if (ms) ms[v] = per;
            if (per < best_ms) { best_ms = per; best_v = v; }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (b) ph_batch_destroy(b);
    cudaStreamDestroy(s);
    if (rc) return rc;
    set_variant(N1, fp32, curv, best_v);
    if (best) *best = best_v;
    return PH_OK;
}

}  // extern "C"
