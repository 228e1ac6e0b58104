// server.cu -- request loop with continuous batching over one index.
//
// The reference has no serving layer: its driver runs searches, inserts and
// deletes one call at a time on the default stream (vamana.cu:1782-1895).
// Here a worker thread owns the index.  Search requests (host queries, each
// with its own k and L) queue up; whenever one of the batch slots is free, all
// queued searches up to max_batch queries are admitted into it as ONE uneven
// launch (vann_search_uneven) with its host->device copy and result copy on the
// slot's own stream, so several batches are on the GPU at once and requests that
// arrive meanwhile join the next free slot.  Writes (insert, delete, consolidate)
// keep their place in the request order: a write runs once every search admitted
// before it has completed, and searches after it are admitted only when it is
// done, so each search sees exactly the writes submitted before it, the same as
// running the requests one by one.  Device memory for batches is fixed at
// creation: the number of slots is capped by the HBM budget.
//
// With a commit interval (group commit), writes wait in their own queue while
// searches keep being admitted against the last committed state; at most once
// per interval (or as soon as no search is waiting) the in-flight batches drain
// and every queued write is applied, in submission order.  Each request reports
// its epoch: a search served at epoch e sees exactly the first e writes, so
// replaying writes in order and running each search after its epoch's writes
// reproduces every result.  One drain then serves many writes.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/vann.h"
#include "kernels.h"

namespace {

using Clock = std::chrono::steady_clock;

enum Kind { kSearch = 0, kInsert = 1, kDelete = 2, kConsolidate = 3 };

struct Request {
    uint64_t              ticket = 0;
    int                   kind   = kSearch;
    uint32_t              n = 0, k = 0, L = 0;
    std::vector<float>    vecs;
    std::vector<uint32_t> ids;
    std::vector<uint32_t> out_ids;  // search: n x k; insert: n new ids
    std::vector<float>    out_d;
    Clock::time_point     t_submit, t_done;
    vann_status           status = VANN_OK;
    bool                  done   = false;
    uint64_t              epoch  = 0;  // writes applied before this request was served
};

struct Slot {
    cudaStream_t                          st   = nullptr;
    cudaEvent_t                           done = nullptr;
    float*                                d_q  = nullptr;
    uint32_t *                            d_ids = nullptr, *d_L = nullptr, *d_k = nullptr;
    float*                                d_d  = nullptr;
    float*                                h_q  = nullptr;  // pinned
    uint32_t *                            h_ids = nullptr, *h_L = nullptr, *h_k = nullptr;
    float*                                h_d  = nullptr;
    uint32_t                              kmax = 0;
    bool                                  busy = false;
    std::vector<std::pair<Request*, uint32_t>> reqs;  // request, first row
};

}  // namespace

struct vann_server {
    vann_index*          idx = nullptr;
    vann_server_params   p{};
    uint32_t             dim = 0;
    std::vector<Slot>    slots;
    std::deque<Request*> queue;
    std::deque<Request*> wqueue;      // group commit: writes waiting for the next commit
    uint64_t             epoch = 0;   // writes applied so far
    std::unordered_map<uint64_t, Request*> all;
    std::mutex              mu;
    std::condition_variable cv_work, cv_done;
    std::thread             worker;
    bool                    stop        = false;
    uint64_t                next_ticket = 1;
    size_t                  slot_bytes  = 0;
    // write staging (grow-only device buffers)
    cudaStream_t wst      = nullptr;
    void*        d_stage  = nullptr;
    size_t       stage_sz = 0;
    // counters
    uint64_t n_batches = 0, n_searched = 0, n_writes = 0, max_inflight = 0;
    std::string last_error;

    bool any_busy() const {
        for (const Slot& s : slots)
            if (s.busy) return true;
        return false;
    }

    void complete(Request* r, vann_status st) {
        r->status = st;
        r->t_done = Clock::now();
        r->done   = true;
    }

    // harvest finished slots (lock held)
    void harvest() {
        for (Slot& s : slots) {
            if (!s.busy) continue;
            cudaError_t q = cudaEventQuery(s.done);
            if (q == cudaErrorNotReady) continue;
            vann_status st = q == cudaSuccess ? VANN_OK : VANN_ERR_CUDA;
            for (auto& rr : s.reqs) {
                Request* r = rr.first;
                r->out_ids.resize((size_t)r->n * r->k);
                r->out_d.resize((size_t)r->n * r->k);
                for (uint32_t i = 0; i < r->n; ++i) {
                    memcpy(&r->out_ids[(size_t)i * r->k], s.h_ids + (size_t)(rr.second + i) * s.kmax,
                           sizeof(uint32_t) * r->k);
                    memcpy(&r->out_d[(size_t)i * r->k], s.h_d + (size_t)(rr.second + i) * s.kmax,
                           sizeof(float) * r->k);
                }
                complete(r, st);
            }
            s.reqs.clear();
            s.busy = false;
            cv_done.notify_all();
        }
    }

    // admit queued searches into a free slot (lock held); returns true if launched
    bool admit(Slot& s) {
        uint32_t rows = 0, kmax = 1, Lmax = 1;
        while (!queue.empty() && queue.front()->kind == kSearch) {
            Request* r = queue.front();
            if (rows > 0 && rows + r->n > p.max_batch) break;
            queue.pop_front();
            memcpy(s.h_q + (size_t)rows * dim, r->vecs.data(), sizeof(float) * r->n * dim);
            for (uint32_t i = 0; i < r->n; ++i) {
                s.h_L[rows + i] = r->L;
                s.h_k[rows + i] = r->k;
            }
            kmax = r->k > kmax ? r->k : kmax;
            Lmax = r->L > Lmax ? r->L : Lmax;
            r->epoch = epoch;
            s.reqs.emplace_back(r, rows);
            rows += r->n;
        }
        if (rows == 0) return false;
        s.kmax = kmax;
        vann_search_params sp{Lmax, kmax, p.store, p.rerank, 0, 0};
        cudaError_t ce = cudaMemcpyAsync(s.d_q, s.h_q, sizeof(float) * rows * dim, cudaMemcpyHostToDevice, s.st);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(s.d_L, s.h_L, sizeof(uint32_t) * rows, cudaMemcpyHostToDevice, s.st);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(s.d_k, s.h_k, sizeof(uint32_t) * rows, cudaMemcpyHostToDevice, s.st);
        vann_status st = ce == cudaSuccess
                             ? vann_search_uneven(idx, s.d_q, rows, &sp, s.d_L, s.d_k, s.d_ids, s.d_d, s.st)
                             : VANN_ERR_CUDA;
        if (st != VANN_OK) {
            for (auto& rr : s.reqs) complete(rr.first, st);
            s.reqs.clear();
            last_error = vann_last_error();
            cv_done.notify_all();
            return false;
        }
        ce = cudaMemcpyAsync(s.h_ids, s.d_ids, sizeof(uint32_t) * rows * kmax, cudaMemcpyDeviceToHost, s.st);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(s.h_d, s.d_d, sizeof(float) * rows * kmax, cudaMemcpyDeviceToHost, s.st);
        if (ce == cudaSuccess) ce = cudaEventRecord(s.done, s.st);
        if (ce != cudaSuccess) {  // the results would never arrive: fail the batch now
            for (auto& rr : s.reqs) complete(rr.first, VANN_ERR_CUDA);
            s.reqs.clear();
            last_error = cudaGetErrorString(ce);
            cv_done.notify_all();
            return false;
        }
        s.busy = true;
        ++n_batches;
        n_searched += rows;
        uint64_t inflight = 0;
        for (const Slot& t : slots) inflight += t.busy;
        if (inflight > max_inflight) max_inflight = inflight;
        return true;
    }

    void stage(size_t bytes) {
        if (bytes <= stage_sz) return;
        if (d_stage) cudaFree(d_stage);
        d_stage  = nullptr;
        stage_sz = 0;
        if (cudaMalloc(&d_stage, bytes) == cudaSuccess) stage_sz = bytes;
    }

    // run a write with the lock released; every earlier search has completed
    vann_status write(Request* r) {
        vann_status st = VANN_OK;
        if (r->kind == kInsert) {
            stage(sizeof(float) * r->n * dim + sizeof(uint32_t) * r->n);
            if (stage_sz == 0) return VANN_ERR_OOM;
            float*    dv = static_cast<float*>(d_stage);
            uint32_t* di = reinterpret_cast<uint32_t*>(dv + (size_t)r->n * dim);
            if (cudaMemcpyAsync(dv, r->vecs.data(), sizeof(float) * r->n * dim, cudaMemcpyHostToDevice, wst) !=
                cudaSuccess)
                return VANN_ERR_CUDA;
            st = vann_insert(idx, dv, r->n, di, wst);
            if (st == VANN_OK) {
                r->out_ids.resize(r->n);
                if (cudaMemcpyAsync(r->out_ids.data(), di, sizeof(uint32_t) * r->n, cudaMemcpyDeviceToHost, wst) !=
                        cudaSuccess ||
                    cudaStreamSynchronize(wst) != cudaSuccess)
                    st = VANN_ERR_CUDA;
            }
        } else if (r->kind == kDelete) {
            stage(sizeof(uint32_t) * r->n);
            if (stage_sz == 0) return VANN_ERR_OOM;
            if (cudaMemcpyAsync(d_stage, r->ids.data(), sizeof(uint32_t) * r->n, cudaMemcpyHostToDevice, wst) !=
                cudaSuccess)
                return VANN_ERR_CUDA;
            st = vann_delete(idx, static_cast<uint32_t*>(d_stage), r->n, wst);
            if (st == VANN_OK && cudaStreamSynchronize(wst) != cudaSuccess) st = VANN_ERR_CUDA;
        } else {
            st = vann_consolidate(idx, wst);
        }
        if (st != VANN_OK) last_error = vann_last_error();
        return st;
    }

    void apply_write(std::unique_lock<std::mutex>& lk, Request* r) {
        lk.unlock();
        vann_status st = write(r);
        lk.lock();
        ++n_writes;
        r->epoch = ++epoch;
        complete(r, st);
        cv_done.notify_all();
    }

    void loop() {
        std::unique_lock<std::mutex> lk(mu);
        const auto interval = std::chrono::microseconds(p.commit_interval_us);
        while (!stop) {
            harvest();
            if (p.commit_interval_us == 0) {
                // strict order: a write waits for the searches before it
                if (!queue.empty() && queue.front()->kind != kSearch) {
                    if (any_busy()) {
                        cv_work.wait_for(lk, std::chrono::microseconds(20));
                        continue;
                    }
                    Request* r = queue.front();
                    queue.pop_front();
                    apply_write(lk, r);
                    continue;
                }
            } else if (!wqueue.empty() &&
                       (queue.empty() || Clock::now() - wqueue.front()->t_submit >= interval)) {
                // group commit: drain, then apply every queued write in order
                if (any_busy()) {
                    cv_work.wait_for(lk, std::chrono::microseconds(20));
                    continue;
                }
                for (size_t w = wqueue.size(); w > 0; --w) {  // writes queued by now
                    Request* r = wqueue.front();
                    wqueue.pop_front();
                    apply_write(lk, r);
                }
                continue;
            }
            bool launched = false;
            for (Slot& s : slots)
                if (!s.busy && !queue.empty() && queue.front()->kind == kSearch) launched |= admit(s);
            if (launched) continue;
            if (any_busy() || !wqueue.empty())
                cv_work.wait_for(lk, std::chrono::microseconds(20));  // poll slot events / commit timer
            else
                cv_work.wait(lk, [&] { return stop || !queue.empty() || !wqueue.empty(); });
        }
    }

    uint64_t submit(Request* r) {
        std::lock_guard<std::mutex> lk(mu);
        r->ticket   = next_ticket++;
        r->t_submit = Clock::now();
        all[r->ticket] = r;
        if (p.commit_interval_us > 0 && r->kind != kSearch)
            wqueue.push_back(r);
        else
            queue.push_back(r);
        cv_work.notify_one();
        return r->ticket;
    }
};

extern "C" {

vann_status vann_server_create(vann_index* idx, const vann_server_params* params, vann_server** out) {
    if (!idx || !params || !out) return VANN_ERR_INVALID;
    const vann_server_params& p = *params;
    if (p.max_batch == 0 || p.slots == 0 || p.max_k == 0 || p.max_k > 1024 || p.store > 4)
        return VANN_ERR_INVALID;
    vann_info info{};
    vann_status st = vann_get_info(idx, &info);
    if (st != VANN_OK) return st;
    auto* s       = new vann_server();
    s->idx        = idx;
    s->p          = p;
    s->dim        = info.dim;
    const size_t B = p.max_batch;
    s->slot_bytes = B * (sizeof(float) * info.dim + (sizeof(uint32_t) + sizeof(float)) * p.max_k + 8);
    uint32_t nslots = p.slots;
    if (p.hbm_budget > 0) {
        uint64_t fit = p.hbm_budget / s->slot_bytes;
        if (fit == 0) {
            delete s;
            vann::set_last_error("hbm_budget holds no batch slot");
            return VANN_ERR_CAPACITY;
        }
        if (fit < nslots) nslots = (uint32_t)fit;
    }
    s->slots.resize(nslots);
    bool ok = cudaStreamCreateWithFlags(&s->wst, cudaStreamNonBlocking) == cudaSuccess;
    for (Slot& sl : s->slots) {
        ok = ok && cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) == cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaMalloc(&sl.d_q, sizeof(float) * B * info.dim) == cudaSuccess;
        ok = ok && cudaMalloc(&sl.d_ids, sizeof(uint32_t) * B * p.max_k) == cudaSuccess;
        ok = ok && cudaMalloc(&sl.d_d, sizeof(float) * B * p.max_k) == cudaSuccess;
        ok = ok && cudaMalloc(&sl.d_L, sizeof(uint32_t) * B) == cudaSuccess;
        ok = ok && cudaMalloc(&sl.d_k, sizeof(uint32_t) * B) == cudaSuccess;
        ok = ok && cudaMallocHost(&sl.h_q, sizeof(float) * B * info.dim) == cudaSuccess;
        ok = ok && cudaMallocHost(&sl.h_ids, sizeof(uint32_t) * B * p.max_k) == cudaSuccess;
        ok = ok && cudaMallocHost(&sl.h_d, sizeof(float) * B * p.max_k) == cudaSuccess;
        ok = ok && cudaMallocHost(&sl.h_L, sizeof(uint32_t) * B) == cudaSuccess;
        ok = ok && cudaMallocHost(&sl.h_k, sizeof(uint32_t) * B) == cudaSuccess;
    }
    if (!ok) {
        vann_server_destroy(s);
        vann::set_last_error("server slot allocation failed");
        return VANN_ERR_OOM;
    }
    s->worker = std::thread([s] { s->loop(); });
    *out      = s;
    return VANN_OK;
}

vann_status vann_server_destroy(vann_server* s) {
    if (!s) return VANN_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    cudaDeviceSynchronize();
    for (Slot& sl : s->slots) {
        if (sl.st) cudaStreamDestroy(sl.st);
        if (sl.done) cudaEventDestroy(sl.done);
        cudaFree(sl.d_q);
        cudaFree(sl.d_ids);
        cudaFree(sl.d_d);
        cudaFree(sl.d_L);
        cudaFree(sl.d_k);
        cudaFreeHost(sl.h_q);
        cudaFreeHost(sl.h_ids);
        cudaFreeHost(sl.h_d);
        cudaFreeHost(sl.h_L);
        cudaFreeHost(sl.h_k);
    }
    if (s->wst) cudaStreamDestroy(s->wst);
    if (s->d_stage) cudaFree(s->d_stage);
    for (auto& kv : s->all) delete kv.second;  // every request, queued or done, is in `all`
    delete s;
    return VANN_OK;
}

vann_status vann_server_submit_search(vann_server* s, const float* h_q, uint32_t n, uint32_t k, uint32_t L,
                                      uint64_t* ticket) {
    if (!s || !h_q || !ticket || n == 0 || n > s->p.max_batch || k == 0 || k > s->p.max_k || L < k ||
        L > 1024)
        return VANN_ERR_INVALID;
    auto* r = new Request();
    r->kind = kSearch;
    r->n = n;
    r->k = k;
    r->L = L;
    r->vecs.assign(h_q, h_q + (size_t)n * s->dim);
    *ticket = s->submit(r);
    return VANN_OK;
}

vann_status vann_server_submit_insert(vann_server* s, const float* h_vecs, uint32_t n, uint64_t* ticket) {
    if (!s || !h_vecs || !ticket || n == 0) return VANN_ERR_INVALID;
    auto* r = new Request();
    r->kind = kInsert;
    r->n = n;
    r->vecs.assign(h_vecs, h_vecs + (size_t)n * s->dim);
    *ticket = s->submit(r);
    return VANN_OK;
}

vann_status vann_server_submit_delete(vann_server* s, const uint32_t* h_ids, uint32_t n, uint64_t* ticket) {
    if (!s || !h_ids || !ticket || n == 0) return VANN_ERR_INVALID;
    auto* r = new Request();
    r->kind = kDelete;
    r->n = n;
    r->ids.assign(h_ids, h_ids + n);
    *ticket = s->submit(r);
    return VANN_OK;
}

vann_status vann_server_submit_consolidate(vann_server* s, uint64_t* ticket) {
    if (!s || !ticket) return VANN_ERR_INVALID;
    auto* r = new Request();
    r->kind = kConsolidate;
    *ticket = s->submit(r);
    return VANN_OK;
}

vann_status vann_server_wait(vann_server* s, uint64_t ticket, uint32_t* h_ids, float* h_dists,
                             double* latency_us, uint64_t* epoch, uint32_t timeout_ms) {
    if (!s) return VANN_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return VANN_ERR_NOT_FOUND;
    Request* r = it->second;
    bool done = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms ? timeout_ms : 600000),
                                    [&] { return r->done; });
    if (!done) return VANN_ERR_TIMEOUT;
    if (h_ids && !r->out_ids.empty()) memcpy(h_ids, r->out_ids.data(), sizeof(uint32_t) * r->out_ids.size());
    if (h_dists && !r->out_d.empty()) memcpy(h_dists, r->out_d.data(), sizeof(float) * r->out_d.size());
    if (latency_us)
        *latency_us = std::chrono::duration<double, std::micro>(r->t_done - r->t_submit).count();
    if (epoch) *epoch = r->epoch;
    vann_status st = r->status;
    if (st != VANN_OK) vann::set_last_error(s->last_error.c_str());
    s->all.erase(it);
    delete r;
    return st;
}

vann_status vann_server_get_stats(vann_server* s, vann_server_stats* out) {
    if (!s || !out) return VANN_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    out->slots        = (uint32_t)s->slots.size();
    out->slot_bytes   = s->slot_bytes;
    out->batches      = s->n_batches;
    out->queries      = s->n_searched;
    out->writes       = s->n_writes;
    out->max_inflight = s->max_inflight;
    out->queued       = s->queue.size() + s->wqueue.size();
    out->epoch        = s->epoch;
    return VANN_OK;
}

}  // extern "C"
