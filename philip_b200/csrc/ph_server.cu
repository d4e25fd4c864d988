// Native continuous-batching server over a ph_batch (host code only).
//
// The reference runs one FlowSolver per snapshot (AdaptiveSamplingBase::solveSnapshotFOM,
// src/reduced_order/adaptive_sampling_base.cpp:255-265). Here callers on any host thread submit
// solves; one worker thread owns the batch. Each pass of its loop admits queued solves in FIFO
// order while the HBM budget holds them (a solve that does not fit waits and holds the ones
// behind it, so large solves are not starved), enqueues chunk_steps RK steps of every resident
// solve (one graph replay per step) with at most two chunks in flight, and retires every solve
// whose last step the GPU has finished: its final state and status word are copied to host
// memory and its arena range is released.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/philip_b200.h"
#include "ph_internal.hpp"

using namespace ph_host;

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    long long ticket = 0;
    ph_mesh_desc mesh{};
    std::vector<double> support;     // copy of mesh.mapping_support_points (when given)
    ph_params prm{};
    std::vector<double> U;           // initial state, then the final state
    double dt = 0.0;
    int nsteps = 0;
    BatchPrep prep;                  // host set-up, built on the submitting thread
    int state = PH_SOLVE_QUEUED;
    int rc = PH_OK;
    std::string error;
    uint32_t flags = 0;
    Clock::time_point submitted, admitted, completed;
};

size_t state_size(const ph_mesh_desc& m, const ph_params& p) {
    const size_t n = (size_t)m.n_cells_per_direction, n1 = (size_t)p.poly_degree + 1;
    return n * n * n * 5 * n1 * n1 * n1;
}

}  // namespace

struct ph_server {
    ph_batch* batch = nullptr;
    int device = 0;
    int chunk = 16;
    double admit_slice = 0.004;        // seconds of host time per pass spent admitting while solves run
    std::mutex mu;
    std::condition_variable work_cv;   // the worker waits here for submissions
    std::condition_variable done_cv;   // callers of ph_server_wait wait here
    std::deque<Job*> queue;            // submitted, not admitted (FIFO)
    std::map<long long, Job*> jobs;    // every ticket not yet collected
    long long next_ticket = 1;
    bool stop = false;
    long long admissions_deferred = 0;
    int max_resident = 0;
    long long launches = 0;            // kernel launches the batch has issued (graph nodes counted)
    std::thread worker;

    void run();
};

void ph_server::run() {
    cudaSetDevice(device);
    std::map<int, Job*> resident;      // batch slot -> job
    std::deque<long long> fences;
    for (;;) {
        Job* head = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (stop && !queue.empty()) {   // stopping: solves never admitted are cancelled
                for (Job* j : queue) {
                    j->state = PH_SOLVE_FAILED;
                    j->rc = PH_ERR_INVALID;
                    j->error = "server stopped before the solve was admitted";
                    j->completed = Clock::now();
                }
                queue.clear();
                done_cv.notify_all();
            }
            if (resident.empty() && queue.empty()) {
                if (stop) break;
                work_cv.wait_for(lk, std::chrono::milliseconds(50));
                continue;
            }
            if (!queue.empty()) head = queue.front();
        }
        // admission, FIFO; the batch is touched by this thread only. While solves are resident it
        // takes at most admit_slice of host time per pass (an admission builds the solve's
        // geometry on the host), so the loop returns to queue steps before the GPU runs dry.
        auto slice_end = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                            std::chrono::duration<double>(admit_slice));
        while (head && (resident.empty() || Clock::now() < slice_end)) {
            const double* u0 = head->U.data();
            if (!head->support.empty()) head->mesh.mapping_support_points = head->support.data();
            int slot = -1;
            const int rc = batch_admit_prepared(batch, &head->mesh, &head->prm, &head->prep, u0, head->dt, head->nsteps,
                                                &slot);
            std::unique_lock<std::mutex> lk(mu);
            if (rc == PH_ERR_NOMEM && !resident.empty()) {   // no room now: retry once solves retire
                ++admissions_deferred;
                break;
            }
            queue.pop_front();
            if (rc != PH_OK) {
                head->rc = rc;
                head->error = ph_last_error();
                head->state = PH_SOLVE_FAILED;
                head->completed = Clock::now();
                done_cv.notify_all();
            } else {
                head->state = PH_SOLVE_RUNNING;
                head->admitted = Clock::now();
                if (resident.empty())   // the first resident solve opens the slice
                    slice_end = head->admitted + std::chrono::duration_cast<Clock::duration>(
                                                     std::chrono::duration<double>(admit_slice));
                resident[slot] = head;
                if ((int)resident.size() > max_resident) max_resident = (int)resident.size();
            }
            head = queue.empty() ? nullptr : queue.front();
        }
        if (resident.empty()) continue;
        int active = 0;
        ph_batch_active(batch, &active);
        if (active > 0) {
            long long t = 0;
            int rc = ph_batch_step(batch, chunk);
            if (rc == PH_OK) rc = ph_batch_fence(batch, &t);
            if (rc == PH_OK) fences.push_back(t);
            if (rc == PH_OK && fences.size() > 2) { rc = ph_batch_fence_wait(batch, fences.front()); fences.pop_front(); }
            if (rc != PH_OK) {   // the batch cannot advance: every resident solve fails with its error
                const std::string why = ph_last_error();
                for (auto& kv : resident) {
                    ph_batch_release(batch, kv.first);
                    std::lock_guard<std::mutex> lk(mu);
                    kv.second->rc = rc;
                    kv.second->error = "stepping failed: " + why;
                    kv.second->state = PH_SOLVE_FAILED;
                    kv.second->completed = Clock::now();
                }
                resident.clear();
                fences.clear();
                done_cv.notify_all();
                continue;
            }
            long long n = 0;
            ph_batch_launches(batch, &n);
            std::lock_guard<std::mutex> lk(mu);
            launches = n;
        }
        for (auto it = resident.begin(); it != resident.end();) {
            int complete = 0;
            ph_batch_poll(batch, it->first, &complete);
            if (!complete) { ++it; continue; }
            Job* j = it->second;
            const int rc = ph_batch_get_state(batch, it->first, j->U.data());
            uint32_t flags = 0;
            ph_batch_status(batch, it->first, &flags);
            ph_batch_release(batch, it->first);
            {
                std::lock_guard<std::mutex> lk(mu);
                j->flags = flags;
                j->rc = rc;
                if (rc != PH_OK) j->error = ph_last_error();
                j->state = rc == PH_OK ? PH_SOLVE_DONE : PH_SOLVE_FAILED;
                j->completed = Clock::now();
            }
            done_cv.notify_all();
            it = resident.erase(it);
        }
        if (active == 0 && !resident.empty())   // everything resident is enqueued to its end
            while (!fences.empty()) { ph_batch_fence_wait(batch, fences.front()); fences.pop_front(); }
    }
}

extern "C" {

int ph_server_create(size_t hbm_budget_bytes, int precision, int chunk_steps, double admit_slice_s, ph_server** out) {
    if (!out) return fail(PH_ERR_INVALID, "null argument");
    *out = nullptr;
    if (chunk_steps < 1) return fail(PH_ERR_INVALID, "chunk_steps must be positive");
    if (!(admit_slice_s >= 0.0)) return fail(PH_ERR_INVALID, "admit_slice_s must be >= 0");
    if (precision != PH_FP64 && precision != PH_FP32_RESIDUAL) return fail(PH_ERR_INVALID, "precision");
    if (hbm_budget_bytes == 0) return fail(PH_ERR_INVALID, "budget too small");
    ph_server* s = new ph_server();
    s->chunk = chunk_steps;
    s->admit_slice = admit_slice_s;
    cudaGetDevice(&s->device);
    if (int rc = ph_batch_create(hbm_budget_bytes, precision, nullptr, &s->batch)) { delete s; return rc; }
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return PH_OK;
}

int ph_server_submit(ph_server* s, const ph_mesh_desc* mesh, const ph_params* prm, const double* U0, double dt,
                     int nsteps, long long* ticket) {
    if (!s || !mesh || !prm || !U0 || !ticket) return fail(PH_ERR_INVALID, "null argument");
    if (nsteps < 1 || !(dt > 0.0) || mesh->n_cells_per_direction < 1 || prm->poly_degree < 1 || prm->poly_degree > 6)
        return fail(PH_ERR_INVALID, "bad solve");
    Job* j = new Job();
    j->mesh = *mesh;
    j->prm = *prm;
    j->dt = dt;
    j->nsteps = nsteps;
    const size_t n = state_size(*mesh, *prm);
    j->U.assign(U0, U0 + n);
    if (mesh->mapping_support_points) {
        const size_t ns = n / 5 * 3;   // [cell][3][(p+1)^3]
        j->support.assign(mesh->mapping_support_points, mesh->mapping_support_points + ns);
    }
    j->mesh.mapping_support_points = j->support.empty() ? nullptr : j->support.data();
    j->submitted = Clock::now();
    // the solve's geometry on this thread, not on the worker's (which keeps the GPU fed)
    if (int rc = batch_prepare(&j->mesh, &j->prm, j->prep)) { delete j; return rc; }
    j->mesh.mapping_support_points = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) { delete j; return fail(PH_ERR_INVALID, "server is stopping"); }
        j->ticket = s->next_ticket++;
        s->jobs[j->ticket] = j;
        s->queue.push_back(j);
        *ticket = j->ticket;
    }
    s->work_cv.notify_one();
    return PH_OK;
}

int ph_server_poll(ph_server* s, long long ticket, int* state) {
    if (!s || !state) return fail(PH_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return fail(PH_ERR_INVALID, "unknown ticket");
    *state = it->second->state;
    return PH_OK;
}

int ph_server_wait(ph_server* s, long long ticket, double timeout_s, int* state) {
    if (!s || !state) return fail(PH_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return fail(PH_ERR_INVALID, "unknown ticket");
    Job* j = it->second;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(timeout_s > 0.0 ? timeout_s : 0.0));
    s->done_cv.wait_until(lk, until, [j] { return j->state == PH_SOLVE_DONE || j->state == PH_SOLVE_FAILED; });
    *state = j->state;
    return PH_OK;
}

int ph_server_result(ph_server* s, long long ticket, double* U, uint32_t* flags, double seconds[2]) {
    if (!s) return fail(PH_ERR_INVALID, "null argument");
    Job* j = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->jobs.find(ticket);
        if (it == s->jobs.end()) return fail(PH_ERR_INVALID, "unknown ticket");
        j = it->second;
        if (j->state != PH_SOLVE_DONE && j->state != PH_SOLVE_FAILED) return fail(PH_ERR_INVALID, "solve not finished");
        s->jobs.erase(it);
    }
    int rc = PH_OK;
    if (j->state == PH_SOLVE_FAILED) {
        rc = fail(j->rc ? j->rc : PH_ERR_INVALID, j->error);
    } else {
        if (U) std::memcpy(U, j->U.data(), j->U.size() * sizeof(double));
        if (flags) *flags = j->flags;
        if (seconds) {
            seconds[0] = std::chrono::duration<double>(j->admitted - j->submitted).count();
            seconds[1] = std::chrono::duration<double>(j->completed - j->submitted).count();
        }
    }
    delete j;
    return rc;
}

int ph_server_stats(ph_server* s, long long out[4]) {
    if (!s || !out) return fail(PH_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = (long long)s->queue.size();
    out[1] = s->admissions_deferred;
    out[2] = s->max_resident;
    out[3] = s->launches;
    return PH_OK;
}

int ph_server_destroy(ph_server* s) {
    if (!s) return PH_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->work_cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    ph_batch_destroy(s->batch);
    for (auto& kv : s->jobs) delete kv.second;
    delete s;
    return PH_OK;
}

}  // extern "C"
