// combiner.cu -- shared elemental launches across concurrent Newton solves.
//
// A serving loop runs many independent hdgx_solve calls at once, each on its own host thread and
// CUDA stream.  Each Newton step re-assembles (kernel/hdg_assemble.m:42 calls hdg_elemental once
// per assembly), and a small request's elemental launch fills only part of the GPU.  A combiner
// collects the assemblies that concurrent solves submit and evaluates every group of one element
// shape (equal master tables) and one kind of physics (viscous or not) as ONE segmented launch
// (hdgx_elemental_shared): each solve keeps its own physics, arrays and status, and its results
// are bitwise those of its own launch.
//
// Batching is leader/follower, without a thread of its own: the first solve to submit while no
// batch is being formed becomes the leader; it waits until every attached solve of its group has
// submitted or `window_us` has passed, takes the queue, launches each group of two or more on one of
// the combiner's streams (after an event of every member's stream) and makes every member's stream
// wait for its group's launch; a group of one is launched on its own solve's stream.
// Solves whose submissions arrive during a launch form the next batch.  With window_us = 0 the
// leader takes whatever is queued at once (no solve ever waits for another to submit).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <chrono>
#include <new>
#include <condition_variable>
#include <map>
#include <mutex>
#include <vector>
#include "hdgx_common.cuh"

namespace hdgx {
int elemental_launch(const hdgx_master *m, const hdgx_app *app, int ne, const double *dgnodes,
                     const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                     double *FE, double *DUDG, double *DUDG_DUH, int *status, cudaStream_t st, bool mixed,
                     int grid, double *QDG, double *RU);
int elemental_launch_shared(int nb, const hdgx_elem_bucket *b, cudaStream_t st, int grid);
int elemental_shared_max_segments();
int elemental_check_master(const hdgx_master *m);
}  // namespace hdgx

namespace {

struct Submission {
    hdgx_elem_bucket b;
    uint64_t key;              // master tables, shape and physics kind
    cudaStream_t st;           // the submitting solve's stream (its inputs are queued on it)
    int rc = 0;
    bool done = false;
};

uint64_t fnv1a(uint64_t h, const void *p, size_t n) {
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < n; i++) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

}  // namespace

struct hdgx_combiner {
    std::mutex mu;
    std::condition_variable cv;
    int window_us = 0;
    int device = 0;
    int attached = 0;
    std::map<uint64_t, int> attached_by_key;  // attached solves per group key
    bool leading = false;
    std::vector<Submission *> queue;
    static constexpr int kStreams = 8;
    cudaStream_t ls[kStreams] = {};          // the shared launches' streams, used in turn
    int next = 0;
    std::vector<cudaEvent_t> done;           // one per launch of a batch (grown on demand)
    std::vector<cudaEvent_t> ready;          // one per member of a batch's shared launches
    long long batches = 0, launches = 0, submissions = 0;
    double key_s = 0.0, submit_s = 0.0;      // host time in combiner_key / combiner_submit, all solves

    static cudaEvent_t pooled(std::vector<cudaEvent_t> &pool, size_t i) {
        while (pool.size() <= i) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) e = nullptr;
            pool.push_back(e);
        }
        return pool[i];
    }

    // Launch one batch (called by the leader without the lock held); returns the launch count.
    // The members' threads are blocked in combiner_submit meanwhile, so the last work queued on
    // a member's stream is that assembly's input (the trace gather); the leader records the
    // member's ready event there itself.
    long long run(std::vector<Submission *> &batch) {
        std::vector<bool> taken(batch.size(), false);
        const int maxseg = hdgx::elemental_shared_max_segments();
        size_t ev = 0, nr = 0;
        long long nl = 0;
        std::vector<hdgx_elem_bucket> bk;
        std::vector<Submission *> grp;
        for (size_t i = 0; i < batch.size(); i++) {
            if (taken[i]) continue;
            grp.clear();
            for (size_t j = i; j < batch.size() && (int)grp.size() < maxseg; j++)
                if (!taken[j] && batch[j]->key == batch[i]->key) {
                    taken[j] = true;
                    grp.push_back(batch[j]);
                }
            if (grp.size() == 1) {
                // a group of one: its own launch on its own stream (no cross-stream events)
                Submission *x = grp[0];
                const hdgx_elem_bucket &q = x->b;
                x->rc = hdgx::elemental_launch(q.master, q.app, q.ne, q.dgnodes, q.bf, q.UDG, q.UH, q.SH, q.AE, q.FE,
                                               q.DUDG, q.DUDG_DUH, q.status, x->st, false, 0, nullptr, nullptr);
                nl++;
                continue;
            }
            bk.clear();
            int rc = 0;
            // launches on different streams in turn, so that consecutive batches (and the groups
            // of one batch) run concurrently, as the solves' own launches would
            cudaStream_t ls_k = ls[next];
            next = (next + 1) % kStreams;
            for (Submission *s : grp) {
                bk.push_back(s->b);
                cudaEvent_t r = pooled(ready, nr++);
                if (!r || cudaEventRecord(r, s->st) != cudaSuccess || cudaStreamWaitEvent(ls_k, r, 0) != cudaSuccess)
                    rc = -12;
            }
            if (!rc) rc = hdgx::elemental_launch_shared((int)bk.size(), bk.data(), ls_k, 0);
            cudaEvent_t e = pooled(done, ev++);
            // A later batch re-records the event only after these waits were issued, and a wait
            // takes the event's state at the time of the call.
            if (!e || cudaEventRecord(e, ls_k) != cudaSuccess) rc = rc ? rc : -12;
            for (Submission *s : grp) {
                if (e && cudaStreamWaitEvent(s->st, e, 0) != cudaSuccess && !rc) rc = -12;
                s->rc = rc;
            }
            nl++;
        }
        return nl;
    }
};

namespace hdgx {

// Register a solve of group `key` with the combiner (it is then counted among the submissions a
// batch of its group waits for).
int combiner_attach(hdgx_combiner *c, uint64_t key) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -12;
    if (dev != c->device) return -2;
    std::lock_guard<std::mutex> lk(c->mu);
    c->attached++;
    c->attached_by_key[key]++;
    return 0;
}

void combiner_detach(hdgx_combiner *c, uint64_t key) {
    std::lock_guard<std::mutex> lk(c->mu);
    c->attached--;
    if (--c->attached_by_key[key] <= 0) c->attached_by_key.erase(key);
    c->cv.notify_all();
}

static double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Group key of a solve: a 64-bit FNV-1a hash of its master's tables (read from the device once per
// solve) and sizes, so that only masters with equal tables share a launch, and whether the physics
// is viscous (which selects the kernel).

int combiner_key(hdgx_combiner *c, const hdgx_master *m, const hdgx_app *app, cudaStream_t st, uint64_t *key) {
    const auto t0 = std::chrono::steady_clock::now();
    if (int rc = elemental_check_master(m)) return rc;
    const size_t nd1 = (size_t)m->nd + 1;
    const size_t nv = (size_t)m->ngv * m->npv * nd1, nf = (size_t)m->ngf * m->npf * m->nd;
    std::vector<double> t(3 * nv + 3 * nf);
    std::vector<int> perm((size_t)m->npf * m->nfe);
    const double *src[6] = {m->shapvt, m->shapvg, m->shapmv, m->shapft, m->shapfg, m->shapmf};
    size_t off = 0;
    for (int i = 0; i < 6; i++) {
        const size_t n = i < 3 ? nv : nf;
        if (cudaMemcpyAsync(t.data() + off, src[i], n * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return -12;
        off += n;
    }
    if (cudaMemcpyAsync(perm.data(), m->perm, perm.size() * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return -12;
    if (cudaStreamSynchronize(st) != cudaSuccess) return -12;
    const int dims[7] = {m->nd, m->porder, m->npv, m->npf, m->nfe, m->ngv, m->ngf};
    uint64_t h = 1469598103934665603ull;
    h = fnv1a(h, dims, sizeof(dims));
    h = fnv1a(h, t.data(), t.size() * sizeof(double));
    h = fnv1a(h, perm.data(), perm.size() * sizeof(int));
    const double re = app->param[2];
    *key = h * 2 + ((re > 0.0 && isfinite(re)) ? 1 : 0);
    const double dt = seconds_since(t0);
    std::lock_guard<std::mutex> lk(c->mu);
    c->key_s += dt;
    return 0;
}

// Submit one assembly's elemental evaluation (FP64) queued on stream `st`; returns when it has been
// launched (not completed): `st` then waits for the shared launch that holds it.
int combiner_submit(hdgx_combiner *c, const hdgx_elem_bucket &b, uint64_t key, cudaStream_t st) {
    const auto t0 = std::chrono::steady_clock::now();
    Submission s;
    s.b = b;
    s.key = key;
    s.st = st;
    std::unique_lock<std::mutex> lk(c->mu);
    c->queue.push_back(&s);
    c->submissions++;
    c->cv.notify_all();
    while (!s.done) {
        if (!c->leading) {
            c->leading = true;
            // wait for the other solves of this group (the batch takes every group's submissions)
            const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(c->window_us);
            auto queued_of_group = [&] {
                int n = 0;
                for (const Submission *x : c->queue) n += x->key == s.key;
                return n;
            };
            while (std::chrono::steady_clock::now() < deadline && queued_of_group() < c->attached_by_key[s.key])
                c->cv.wait_until(lk, deadline);
            std::vector<Submission *> batch;
            batch.swap(c->queue);
            lk.unlock();
            const long long nl = c->run(batch);
            lk.lock();
            c->launches += nl;
            c->batches++;
            for (Submission *x : batch) x->done = true;
            c->leading = false;
            c->cv.notify_all();
        } else {
            c->cv.wait(lk);
        }
    }
    c->submit_s += seconds_since(t0);
    return s.rc;
}

}  // namespace hdgx

extern "C" int hdgx_combiner_create(int window_us, hdgx_combiner **out) {
    if (!out || window_us < 0) return -1;
    *out = nullptr;
    hdgx_combiner *c = new (std::nothrow) hdgx_combiner;
    if (!c) return -13;
    c->window_us = window_us;
    bool ok = cudaGetDevice(&c->device) == cudaSuccess;
    for (int k = 0; k < hdgx_combiner::kStreams && ok; k++)
        ok = cudaStreamCreateWithFlags(&c->ls[k], cudaStreamNonBlocking) == cudaSuccess;
    if (!ok) {
        for (cudaStream_t s : c->ls)
            if (s) cudaStreamDestroy(s);
        delete c;
        return -12;
    }
    *out = c;
    return 0;
}

extern "C" int hdgx_combiner_times(const hdgx_combiner *c, double *key_s, double *submit_s) {
    if (!c) return -1;
    hdgx_combiner *m = const_cast<hdgx_combiner *>(c);
    std::lock_guard<std::mutex> lk(m->mu);
    if (key_s) *key_s = m->key_s;
    if (submit_s) *submit_s = m->submit_s;
    return 0;
}

extern "C" int hdgx_combiner_stats(const hdgx_combiner *c, long long *batches, long long *launches,
                                   long long *submissions) {
    if (!c) return -1;
    hdgx_combiner *m = const_cast<hdgx_combiner *>(c);
    std::lock_guard<std::mutex> lk(m->mu);
    if (batches) *batches = m->batches;
    if (launches) *launches = m->launches;
    if (submissions) *submissions = m->submissions;
    return 0;
}

extern "C" int hdgx_combiner_destroy(hdgx_combiner *c) {
    if (!c) return 0;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        if (c->attached != 0) return -1;
    }
    int rc = 0;
    for (cudaStream_t s : c->ls) {
        if (!s) continue;
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = -12;
        cudaStreamDestroy(s);
    }
    for (cudaEvent_t e : c->done)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : c->ready)
        if (e) cudaEventDestroy(e);
    delete c;
    return rc;
}
