// Serving (include/alea_gpu.h, "serving"): a job queue in front of per-job
// walker contexts.  No reference counterpart: the reference runs one input
// per process.
//
// A packed server (alea_gpu_server_create_packed) steps the admitted VMC
// jobs together by sweep body: preparer threads admit queued VMC jobs as
// memory frees up and build each one's context (system tables, walkers,
// first evaluation), and one packing thread per body class runs its jobs
// through its own packed engine (alea_capi.cu, "packed VMC runs"), one sweep
// launch per step for all of that class's walkers.  The classes step
// independently, so a class of cheap sweeps is not held to the pace of a
// class of expensive ones; DMC jobs still take worker contexts.
//
// Each admitted job gets its own alea_gpu_ctx (own CUDA stream, own device
// records, own random streams keyed by the job's seed) on one of max_running
// worker threads, so several jobs' kernels are in flight on the device at
// once.  Admission is first-fit in arrival order against an HBM budget, by
// the context's footprint estimate; a finishing job returns its bytes and
// wakes the workers, so requests that arrived meanwhile are admitted as soon
// as a slot and the memory are free.  A job's arithmetic is that of
// alea_gpu_vmc_run / alea_gpu_dmc_run on its own context, independent of
// what else runs.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "alea_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
    uint64_t id = 0;
    alea_gpu_job spec{};
    int capacity = 0;
    size_t bytes = 0;
    std::atomic<int> cancel{0};
    bool running = false, done = false;
    alea_gpu_job_result res{};
    Clock::time_point t_submit, t_admit;
};

// A job's AoS walkers [w][p][d] as the SoA planes alea_gpu_upload_walkers
// reads, [p*dim*nw + d*nw + w].
std::vector<double> soa_of(const alea_gpu_job& j) {
    const int row = j.system->n_particles * j.system->dim, nw = j.n_walkers;
    std::vector<double> soa(static_cast<size_t>(row) * nw);
    for (int w = 0; w < nw; ++w)
        for (int i = 0; i < row; ++i) soa[static_cast<size_t>(i) * nw + w] = j.positions[static_cast<size_t>(w) * row + i];
    return soa;
}

}  // namespace

struct alea_gpu_server {
    int device = 0;
    bool packed = false;           // VMC jobs go to the packing scheduler
    size_t budget = 0, in_use = 0;
    int max_running = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    std::deque<uint64_t> queue;
    uint64_t next_id = 1;
    bool stop = false;
    std::vector<std::thread> workers;
    std::string err;
    // packed: contexts built by the preparers, by body class, for the packers
    std::deque<std::pair<Job*, alea_gpu_ctx*>> ready[alea_gpu::kPackedClasses];
    int preparing = 0;
    std::condition_variable cv_ready;

    // First queued job that fits the budget left (caller holds mu); a packed
    // server's scheduler takes the VMC jobs of two-dimensional systems (what
    // the packed sweeps run), its workers every other job.
    Job* admissible(bool vmc_packer = false) {
        for (uint64_t id : queue) {
            Job* j = jobs[id].get();
            const bool packs = j->spec.mode == ALEA_JOB_VMC && j->spec.system->dim == 2;
            if (packed && packs != vmc_packer) continue;
            if (j->bytes <= budget - std::min(budget, in_use)) return j;
        }
        return nullptr;
    }

    void admit(Job* j) {   // caller holds mu
        queue.erase(std::find(queue.begin(), queue.end(), j->id));
        in_use += j->bytes;
        j->running = true;
        j->t_admit = Clock::now();
    }

    // A preparer: admits a queued VMC job, builds its context and hands it to
    // the packer of its body class.
    void preparer() {
        cudaSetDevice(device);
        for (;;) {
            Job* j = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || admissible(true) != nullptr; });
                if (stop) return;
                j = admissible(true);
                admit(j);
                ++preparing;
            }
            alea_gpu_ctx* ctx = nullptr;
            int rc = j->cancel.load() ? ALEA_ERR_CANCELLED : ALEA_OK;
            if (rc == ALEA_OK) rc = alea_gpu_create(j->spec.system, device, j->capacity, &ctx);
            if (rc == ALEA_OK) rc = alea_gpu_upload_walkers(ctx, soa_of(j->spec).data(), j->spec.n_walkers);
            if (rc != ALEA_OK && ctx) {
                alea_gpu_destroy(ctx);
                ctx = nullptr;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                if (rc == ALEA_OK) ready[alea_gpu::packed_class(ctx)].emplace_back(j, ctx);
                --preparing;
            }
            if (rc != ALEA_OK) finish(j, rc, nullptr);
            cv_ready.notify_all();
        }
    }

    // The packer of body class `cls`: its prepared jobs step together.
    void packer(int cls) {
        cudaSetDevice(device);
        alea_gpu_packed* P = nullptr;
        const int prc = alea_gpu::packed_create(device, &P);
        std::vector<std::pair<Job*, alea_gpu_ctx*>> slots;   // in the engine's run order
        for (;;) {
            std::vector<std::pair<Job*, alea_gpu_ctx*>> fresh;
            {
                std::unique_lock<std::mutex> lk(mu);
                const auto drained = [&] { return stop && preparing == 0 && ready[cls].empty(); };
                if (slots.empty()) cv_ready.wait(lk, [&] { return drained() || !ready[cls].empty(); });
                if (slots.empty() && drained()) break;
                for (; !ready[cls].empty(); ready[cls].pop_front()) fresh.push_back(ready[cls].front());
            }
            for (auto& jc : fresh) {
                Job* j = jc.first;
                int rc = prc != ALEA_OK ? prc : j->cancel.load() ? ALEA_ERR_CANCELLED : ALEA_OK;
                if (rc == ALEA_OK) rc = alea_gpu::packed_add(P, jc.second, j->spec.run, nullptr);
                if (rc != ALEA_OK) {
                    alea_gpu_destroy(jc.second);
                    finish(j, rc, nullptr);
                    continue;
                }
                slots.push_back(jc);
            }
            if (slots.empty()) continue;
            for (size_t i = 0; i < slots.size(); ++i)
                if (slots[i].first->cancel.load()) alea_gpu::packed_cancel(P, static_cast<int>(i));
            const int rc = alea_gpu::packed_step(P);
            std::vector<std::pair<Job*, alea_gpu_ctx*>> keep;
            for (size_t i = 0; i < slots.size(); ++i) {
                int status = ALEA_OK;
                alea_gpu_run_result r{};
                const bool done = alea_gpu::packed_done(P, static_cast<int>(i), &status, &r);
                if (!done && rc == ALEA_OK) {
                    keep.push_back(slots[i]);
                    continue;
                }
                if (!done) {
                    status = rc;
                    alea_gpu::packed_cancel(P, static_cast<int>(i));
                }
                alea_gpu_destroy(slots[i].second);
                finish(slots[i].first, status, status == ALEA_OK ? &r : nullptr);
            }
            if (keep.size() != slots.size()) alea_gpu::packed_prune(P);
            slots.swap(keep);
        }
        alea_gpu::packed_destroy(P);
    }

    void finish(Job* j, int status, const alea_gpu_run_result* r) {
        std::lock_guard<std::mutex> lk(mu);
        const auto now = Clock::now();
        j->res.status = status;
        if (r) j->res.result = *r;
        j->res.footprint_bytes = j->bytes;
        if (j->running) {
            j->res.queue_ms = ms_between(j->t_submit, j->t_admit);
            j->res.run_ms = ms_between(j->t_admit, now);
            in_use -= std::min(in_use, j->bytes);
        } else {
            j->res.queue_ms = ms_between(j->t_submit, now);
        }
        j->res.latency_ms = ms_between(j->t_submit, now);
        j->running = false;
        j->done = true;
        cv_done.notify_all();
        cv_work.notify_all();
    }

    void run(Job* j) {
        const alea_gpu_job& sp = j->spec;
        alea_gpu_ctx* ctx = nullptr;
        alea_gpu_run_result r{};
        int rc = j->cancel.load() ? ALEA_ERR_CANCELLED : ALEA_OK;
        if (rc == ALEA_OK) rc = alea_gpu_create(sp.system, device, j->capacity, &ctx);
        if (rc == ALEA_OK) {
            alea_gpu::set_cancel_flag(ctx, &j->cancel);
            rc = alea_gpu_upload_walkers(ctx, soa_of(sp).data(), sp.n_walkers);
        }
        if (rc == ALEA_OK)
            rc = sp.mode == ALEA_JOB_DMC ? alea_gpu_dmc_run(ctx, &sp.run, &r, nullptr)
                                         : alea_gpu_vmc_run(ctx, &sp.run, &r, nullptr);
        if (rc == ALEA_OK && j->cancel.load()) rc = ALEA_ERR_CANCELLED;
        // the context's memory goes back to the device before the job's bytes
        // go back to the budget, so the next admission cannot overcommit
        if (ctx) alea_gpu_destroy(ctx);
        finish(j, rc, rc == ALEA_OK ? &r : nullptr);
    }

    void worker() {
        cudaSetDevice(device);
        for (;;) {
            Job* j = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || admissible() != nullptr; });
                if (stop) return;
                j = admissible();
                admit(j);
            }
            run(j);
        }
    }
};

extern "C" {

static int server_create(int device, size_t hbm_budget_bytes, int max_running, bool packed,
                         alea_gpu_server** out) {
    if (!out || max_running < 1) return ALEA_ERR_INVALID;
    *out = nullptr;
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) return ALEA_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return ALEA_ERR_CUDA;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return ALEA_ERR_CUDA;
    auto* s = new alea_gpu_server();
    s->device = device;
    s->budget = hbm_budget_bytes ? std::min(hbm_budget_bytes, free_b) : free_b / 10 * 8;
    s->max_running = max_running;
    s->packed = packed;
    for (int i = 0; i < max_running; ++i) s->workers.emplace_back([s] { s->worker(); });
    if (packed) {
        for (int i = 0; i < 2; ++i) s->workers.emplace_back([s] { s->preparer(); });
        for (int k = 0; k < alea_gpu::kPackedClasses; ++k) s->workers.emplace_back([s, k] { s->packer(k); });
    }
    *out = s;
    return ALEA_OK;
}

int alea_gpu_server_create(int device, size_t hbm_budget_bytes, int max_running, alea_gpu_server** out) {
    return server_create(device, hbm_budget_bytes, max_running, false, out);
}

int alea_gpu_server_create_packed(int device, size_t hbm_budget_bytes, int max_running, alea_gpu_server** out) {
    return server_create(device, hbm_budget_bytes, max_running, true, out);
}

int alea_gpu_submit_job(alea_gpu_server* s, const alea_gpu_job* job, uint64_t* job_id) {
    if (!s || !job || !job_id || !job->system || !job->positions || job->n_walkers < 1 ||
        (job->mode != ALEA_JOB_VMC && job->mode != ALEA_JOB_DMC))
        return ALEA_ERR_INVALID;
    auto j = std::make_unique<Job>();
    j->spec = *job;
    const int target = job->run.target_walkers > 0 ? job->run.target_walkers : job->n_walkers;
    j->capacity = job->mode == ALEA_JOB_DMC ? std::max(2 * target + 2, job->n_walkers) : job->n_walkers;
    j->bytes = alea_gpu::footprint_bytes(job->system, j->capacity, job->run.n_substeps);
    std::lock_guard<std::mutex> lk(s->mu);
    if (j->bytes > s->budget) {
        s->err = "job needs " + std::to_string(j->bytes) + " bytes, over the server's budget of " +
                 std::to_string(s->budget);
        return ALEA_ERR_NOMEM;
    }
    j->id = s->next_id++;
    j->t_submit = Clock::now();
    *job_id = j->id;
    s->queue.push_back(j->id);
    s->jobs[j->id] = std::move(j);
    s->cv_work.notify_all();   // a packed server's workers and scheduler wait on different jobs
    return ALEA_OK;
}

int alea_gpu_poll(alea_gpu_server* s, uint64_t job_id, int timeout_ms, alea_gpu_job_result* out) {
    if (!s || !out) return ALEA_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return ALEA_ERR_INVALID;
    Job* j = it->second.get();
    if (!j->done && timeout_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return j->done; });
    if (!j->done) return ALEA_ERR_TIMEOUT;
    *out = j->res;
    s->jobs.erase(it);   // a finished job's result is handed out once
    return ALEA_OK;
}

int alea_gpu_cancel(alea_gpu_server* s, uint64_t job_id) {
    if (!s) return ALEA_ERR_INVALID;
    Job* j = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->jobs.find(job_id);
        if (it == s->jobs.end() || it->second->done) return ALEA_ERR_INVALID;
        j = it->second.get();
        j->cancel.store(1);
        if (j->running) return ALEA_OK;   // its worker stops at the next step
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), job_id));
    }
    s->finish(j, ALEA_ERR_CANCELLED, nullptr);
    return ALEA_OK;
}

int alea_gpu_server_destroy(alea_gpu_server* s) {
    if (!s) return ALEA_OK;
    std::vector<Job*> queued;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (auto& kv : s->jobs) kv.second->cancel.store(1);
        for (uint64_t id : s->queue) queued.push_back(s->jobs[id].get());
        s->queue.clear();
        s->cv_work.notify_all();
        s->cv_ready.notify_all();
    }
    for (Job* j : queued) s->finish(j, ALEA_ERR_CANCELLED, nullptr);
    for (std::thread& t : s->workers) t.join();
    delete s;
    return ALEA_OK;
}

const char* alea_gpu_server_last_error(const alea_gpu_server* s) { return s ? s->err.c_str() : ""; }

}  // extern "C"
