/*
 * php_serve.cu -- the serving loop of php_serve.h.
 *
 * Host threads per server:
 *  - admission threads (kBuilders) take queued jobs in arrival order while the
 *    memory budget and max_active allow, builds their contexts
 *    (php_create, the DFT plane, php_prepare of both chunk lengths) and
 *    hands them to the stepping thread; building a context (medium census,
 *    uploads, graph capture) takes milliseconds and must not starve the GPU;
 *  - the stepping thread keeps up to two chunks of every running job queued
 *    on the job's own stream and retires chunks as their events complete;
 *  - the finisher thread reads a finished job's DFT plane back and destroys
 *    its context (stream-ordered frees, pooled page-locked buffers: nothing
 *    waits for the other jobs).
 * All device work of a job is that of a php_ctx stepped alone.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "php_fdtd.h"
#include "php_serve.h"

namespace {

constexpr int kDefaultChunk = 256;
constexpr int kQueuedChunks = 2;
constexpr int kBuilders = 4; /* admission threads building contexts in parallel */

struct Job {
    int64_t id = 0;
    uint64_t tag = 0;
    /* owned copy of the description */
    php_desc desc{};
    std::vector<php_material_desc> mats;
    std::vector<std::vector<double>> ion;
    std::vector<int32_t> medium;
    std::vector<php_source_desc> srcs;
    int32_t nsteps = 0;
    bool has_dft = false;
    php_dft_request dft{};
    std::vector<double> freqs;

    uint64_t bytes = 0;
    php_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    int dft_id = -1;
    cudaEvent_t ev[kQueuedChunks] = {};
    int chunk_n[kQueuedChunks] = {};
    int head = 0, inflight = 0;
    int32_t issued = 0, done = 0;

    php_job_info info{};
    std::vector<double> plane;
};

double now_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void set_error(Job* j, int rc, const char* msg)
{
    j->info.status = rc;
    snprintf(j->info.error, sizeof(j->info.error), "%s", msg ? msg : "");
}

} // namespace

struct php_server {
    php_server_desc d{};
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_admit, cv_step, cv_done, cv_finish;
    std::deque<Job*> queued;      /* submitted, not admitted */
    std::deque<Job*> ready;       /* admitted and built, not yet stepping */
    std::vector<Job*> running;    /* owned by the stepping thread */
    std::deque<Job*> finishing;   /* all chunks done, teardown pending */
    std::deque<Job*> finished;    /* not yet polled */
    std::map<int64_t, Job*> polled;
    int building = 0;
    int active = 0;               /* admitted and not finished */
    uint64_t used = 0, peak_bytes = 0;
    int peak_running = 0;
    int64_t next_id = 1, submitted = 0, completed = 0;
    bool stop = false;
    std::string err;
    std::vector<std::thread> admit_thr;
    std::thread step_thr, finish_thr;
    bool stepping_done = false;
};

namespace {

/* php_create + DFT plane + graphs; false on failure (status set) */
bool build_job(php_server* s, Job* j)
{
    j->desc.device = s->d.device;
    /* the device is shared by the running jobs: a small grid keeps 8-plane z
     * chunks (fewer halo re-reads) instead of splitting its z range until its
     * own blocks fill the GPU */
    if (j->desc.z_chunk <= 0) j->desc.z_chunk = 8;
    int rc = php_create(&j->desc, &j->ctx);
    if (rc) {
        set_error(j, rc, php_last_error(nullptr));
        return false;
    }
    auto bail = [&](int code) {
        set_error(j, code, php_last_error(j->ctx));
        php_destroy(j->ctx);
        j->ctx = nullptr;
        return false;
    };
    if (j->has_dft) {
        int32_t id = -1;
        rc = php_dft_add(j->ctx, j->dft.component, j->dft.z_plane, j->dft.first_step, j->dft.interval, j->dft.nfreq,
                         j->freqs.data(), j->dft.cast_f32, &id);
        if (rc) return bail(rc);
        j->dft_id = id;
    }
    const int chunk = s->d.chunk_steps > 0 ? s->d.chunk_steps : kDefaultChunk;
    if (j->nsteps >= chunk && (rc = php_prepare(j->ctx, chunk))) return bail(rc);
    if (j->nsteps % chunk && (rc = php_prepare(j->ctx, j->nsteps % chunk))) return bail(rc);
    void* st = nullptr;
    php_stream(j->ctx, &st);
    j->stream = (cudaStream_t)st;
    for (int q = 0; q < kQueuedChunks; q++)
        if (cudaEventCreateWithFlags(&j->ev[q], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return bail(PHP_ERR_CUDA);
        }
    return true;
}

/* DFT read-back and teardown of a job whose chunks have all completed */
void finish_job(Job* j)
{
    if (j->ctx) {
        int rc = php_sync(j->ctx);
        if (rc && j->info.status == PHP_OK) set_error(j, rc, php_last_error(j->ctx));
        if (j->info.status == PHP_OK && j->dft_id >= 0) {
            const size_t n = (size_t)j->dft.nfreq * j->desc.nx * j->desc.ny * 2;
            j->plane.resize(n);
            int32_t ns = 0;
            rc = php_dft_read(j->ctx, j->dft_id, j->plane.data(), &ns);
            if (rc) set_error(j, rc, php_last_error(j->ctx));
            j->info.dft_samples = ns;
        }
        int32_t t = 0;
        php_get_step(j->ctx, &t);
        j->info.steps = t;
        php_destroy(j->ctx);
        j->ctx = nullptr;
    }
    for (int q = 0; q < kQueuedChunks; q++)
        if (j->ev[q]) cudaEventDestroy(j->ev[q]);
}

void admission_loop(php_server* s)
{
    cudaSetDevice(s->d.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_admit.wait(lk, [&] {
            if (s->queued.empty()) return s->stop;
            Job* j = s->queued.front();
            const bool slot = s->d.max_active <= 0 || s->active < s->d.max_active;
            const bool mem = s->active == 0 || s->used + j->bytes <= s->d.memory_budget;
            return slot && mem;
        });
        if (s->queued.empty() && s->stop) return;
        Job* j = s->queued.front();
        s->queued.pop_front();
        s->active++;
        s->used += j->bytes;
        s->peak_bytes = std::max(s->peak_bytes, s->used);
        j->info.t_admit = now_since(s->t0);
        s->building++;
        if (!s->queued.empty()) s->cv_admit.notify_one(); /* the next job may fit too */
        lk.unlock();
        const bool ok = build_job(s, j);
        lk.lock();
        s->building--;
        s->cv_step.notify_one();
        j->info.t_start = now_since(s->t0);
        if (ok) {
            s->ready.push_back(j);
        } else {
            finish_job(j);
            s->active--;
            s->used -= j->bytes;
            j->info.t_done = now_since(s->t0);
            s->finished.push_back(j);
            s->completed++;
            s->cv_done.notify_all();
            s->cv_admit.notify_one();
        }
    }
}

void stepping_loop(php_server* s)
{
    cudaSetDevice(s->d.device);
    const int chunk = s->d.chunk_steps > 0 ? s->d.chunk_steps : kDefaultChunk;
    std::vector<Job*>& run = s->running;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (run.empty())
                s->cv_step.wait(lk, [&] { return !s->ready.empty() || (s->stop && s->queued.empty() && s->building == 0); });
            while (!s->ready.empty()) {
                Job* j = s->ready.front();
                s->ready.pop_front();
                run.push_back(j);
            }
            s->peak_running = std::max(s->peak_running, (int)run.size());
            if (run.empty() && s->stop && s->queued.empty() && s->building == 0) {
                s->stepping_done = true;
                s->cv_finish.notify_one();
                return;
            }
        }
        bool progressed = false;
        std::vector<Job*> fin;
        for (Job* j : run) {
            /* retire completed chunks */
            while (j->inflight > 0) {
                const cudaError_t e = cudaEventQuery(j->ev[j->head]);
                if (e == cudaErrorNotReady) break;
                if (e != cudaSuccess) {
                    cudaGetLastError();
                    set_error(j, PHP_ERR_CUDA, cudaGetErrorString(e));
                }
                j->done += j->chunk_n[j->head];
                j->head = (j->head + 1) % kQueuedChunks;
                j->inflight--;
                progressed = true;
            }
            /* keep kQueuedChunks chunks queued */
            while (j->info.status == PHP_OK && j->inflight < kQueuedChunks && j->issued < j->nsteps) {
                const int n = std::min(chunk, j->nsteps - j->issued);
                const int rc = php_step(j->ctx, n);
                if (rc) {
                    set_error(j, rc, php_last_error(j->ctx));
                    break;
                }
                const int tail = (j->head + j->inflight) % kQueuedChunks;
                cudaEventRecord(j->ev[tail], j->stream);
                j->chunk_n[tail] = n;
                j->inflight++;
                j->issued += n;
                progressed = true;
            }
            if (j->inflight == 0 && (j->done >= j->nsteps || j->info.status != PHP_OK)) fin.push_back(j);
        }
        if (!fin.empty()) {
            /* the read-back and teardown run on the finisher thread, so that
             * the other jobs keep their chunks queued meanwhile */
            std::lock_guard<std::mutex> g(s->mu);
            for (Job* j : fin) {
                run.erase(std::find(run.begin(), run.end(), j));
                s->finishing.push_back(j);
            }
            s->cv_finish.notify_one();
        }
        if (!progressed && fin.empty()) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

void finisher_loop(php_server* s)
{
    cudaSetDevice(s->d.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_finish.wait(lk, [&] { return !s->finishing.empty() || s->stepping_done; });
        if (s->finishing.empty()) return;
        Job* j = s->finishing.front();
        s->finishing.pop_front();
        lk.unlock();
        finish_job(j);
        lk.lock();
        s->active--;
        s->used -= j->bytes;
        j->info.t_done = now_since(s->t0);
        s->finished.push_back(j);
        s->completed++;
        s->cv_done.notify_all();
        s->cv_admit.notify_one();
    }
}

int copy_desc(Job* j, const php_desc* d)
{
    j->desc = *d;
    if (d->nx < 2 || d->ny < 2 || d->nz < 1 || d->num_materials < 1 || !d->materials || !d->medium ||
        d->num_sources < 0 || (d->num_sources > 0 && !d->sources))
        return PHP_ERR_INPUT;
    j->mats.assign(d->materials, d->materials + d->num_materials);
    j->ion.resize(d->num_materials * 3);
    for (int m = 0; m < d->num_materials; m++) {
        php_material_desc& md = j->mats[m];
        const int N = md.natom;
        if (N > 0) {
            if (!md.qezv || !md.qezm || !md.dmm) return PHP_ERR_INPUT;
            j->ion[3 * m].assign(md.qezv, md.qezv + 9 * N);
            j->ion[3 * m + 1].assign(md.qezm, md.qezm + 9 * N);
            j->ion[3 * m + 2].assign(md.dmm, md.dmm + 9 * (size_t)N * N);
            md.qezv = j->ion[3 * m].data();
            md.qezm = j->ion[3 * m + 1].data();
            md.dmm = j->ion[3 * m + 2].data();
        }
    }
    j->medium.assign(d->medium, d->medium + (size_t)d->nx * d->ny * d->nz);
    j->srcs.assign(d->sources, d->sources + d->num_sources);
    j->desc.materials = j->mats.data();
    j->desc.medium = j->medium.data();
    j->desc.sources = j->srcs.empty() ? nullptr : j->srcs.data();
    return PHP_OK;
}

} // namespace

extern "C" {

int php_server_create(const php_server_desc* desc, php_server** out)
{
    if (!desc || !out) return PHP_ERR_INPUT;
    *out = nullptr;
    if (desc->abi_version != PHP_ABI_VERSION || desc->memory_budget == 0 || desc->chunk_steps < 0) return PHP_ERR_INPUT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PHP_ERR_NODEVICE;
    }
    if (desc->device < 0 || desc->device >= ndev) return PHP_ERR_INPUT;
    if (cudaSetDevice(desc->device) != cudaSuccess) return PHP_ERR_CUDA;
    /* freed job buffers stay in the device pool for the next job instead of
     * going back to the driver at every synchronisation */
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, desc->device) == cudaSuccess) {
        uint64_t thr = desc->memory_budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    php_server* s = new php_server();
    s->d = *desc;
    s->t0 = std::chrono::steady_clock::now();
    for (int b = 0; b < kBuilders; b++) s->admit_thr.emplace_back(admission_loop, s);
    s->step_thr = std::thread(stepping_loop, s);
    s->finish_thr = std::thread(finisher_loop, s);
    *out = s;
    return PHP_OK;
}

int php_server_destroy(php_server* s)
{
    if (!s) return PHP_ERR_INPUT;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_admit.notify_all();
    s->cv_step.notify_all();
    for (auto& t : s->admit_thr) t.join();
    s->cv_step.notify_all();
    s->step_thr.join();
    s->finish_thr.join();
    for (Job* j : s->finished) delete j;
    for (auto& kv : s->polled) delete kv.second;
    delete s;
    return PHP_OK;
}

const char* php_server_last_error(const php_server* s)
{
    return s ? s->err.c_str() : "null server";
}

int php_server_clock(const php_server* s, double* seconds)
{
    if (!s || !seconds) return PHP_ERR_INPUT;
    *seconds = now_since(s->t0);
    return PHP_OK;
}

int php_server_stats_read(php_server* s, php_server_stats* o)
{
    if (!s || !o) return PHP_ERR_INPUT;
    std::lock_guard<std::mutex> g(s->mu);
    o->queued = (int32_t)s->queued.size();
    o->running = s->active;
    o->finished_unpolled = (int32_t)s->finished.size();
    o->peak_running = s->peak_running;
    o->bytes_in_use = s->used;
    o->peak_bytes = s->peak_bytes;
    o->submitted = s->submitted;
    o->completed = s->completed;
    return PHP_OK;
}

int php_batch_submit(php_server* s, const php_desc* desc, int32_t nsteps, const php_dft_request* dft, uint64_t tag,
                     int64_t* job)
{
    if (!s || !desc || !job || nsteps < 0) return PHP_ERR_INPUT;
    Job* j = new Job();
    int rc = copy_desc(j, desc);
    if (!rc && dft) {
        if (dft->nfreq < 1 || !dft->freq_hz) rc = PHP_ERR_INPUT;
        else {
            j->has_dft = true;
            j->dft = *dft;
            j->freqs.assign(dft->freq_hz, dft->freq_hz + dft->nfreq);
            j->dft.freq_hz = j->freqs.data();
        }
    }
    uint64_t est = 0;
    if (!rc) rc = php_estimate_bytes(&j->desc, &est);
    if (rc) {
        std::lock_guard<std::mutex> g(s->mu);
        s->err = "php_batch_submit: invalid description";
        delete j;
        return rc;
    }
    if (j->has_dft) est += (uint64_t)j->dft.nfreq * desc->nx * desc->ny * 16;
    j->bytes = est;
    if (est > s->d.memory_budget) {
        std::lock_guard<std::mutex> g(s->mu);
        s->err = "php_batch_submit: the job alone needs more than the memory budget";
        delete j;
        return PHP_ERR_OOM;
    }
    j->nsteps = nsteps;
    j->tag = tag;
    std::lock_guard<std::mutex> g(s->mu);
    j->id = s->next_id++;
    j->info.job = j->id;
    j->info.tag = tag;
    j->info.t_submit = now_since(s->t0);
    j->info.device_bytes = est;
    j->info.nx = desc->nx;
    j->info.ny = desc->ny;
    j->info.nfreq = j->has_dft ? j->dft.nfreq : 0;
    s->queued.push_back(j);
    s->submitted++;
    *job = j->id;
    s->cv_admit.notify_one();
    return PHP_OK;
}

int php_batch_poll(php_server* s, php_job_info* out, int32_t max, int32_t timeout_ms, int32_t* n)
{
    if (!s || !n || max < 0 || (max > 0 && !out)) return PHP_ERR_INPUT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto have = [&] { return !s->finished.empty(); };
    if (!have() && timeout_ms != 0) {
        if (timeout_ms < 0) s->cv_done.wait(lk, have);
        else s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), have);
    }
    int32_t k = 0;
    while (k < max && !s->finished.empty()) {
        Job* j = s->finished.front();
        s->finished.pop_front();
        out[k++] = j->info;
        s->polled[j->id] = j;
    }
    *n = k;
    return PHP_OK;
}

int php_batch_fetch_dft(php_server* s, int64_t job, double* out)
{
    if (!s || !out) return PHP_ERR_INPUT;
    Job* j;
    {
        std::lock_guard<std::mutex> g(s->mu);
        auto it = s->polled.find(job);
        if (it == s->polled.end()) return PHP_ERR_STATE;
        j = it->second;
        if (j->plane.empty()) return PHP_ERR_STATE;
        s->polled.erase(it);
    }
    memcpy(out, j->plane.data(), j->plane.size() * sizeof(double));
    delete j;
    return PHP_OK;
}

int php_batch_release(php_server* s, int64_t job)
{
    if (!s) return PHP_ERR_INPUT;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->polled.find(job);
    if (it == s->polled.end()) return PHP_ERR_STATE;
    delete it->second;
    s->polled.erase(it);
    return PHP_OK;
}

} // extern "C"
