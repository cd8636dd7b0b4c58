// Serving: independent HigFlow cases stepping concurrently on one device, one
// engine case per request (requests that can share a batch go to the
// continuous-batching server, higflow_b200/serve.py, instead).
//
// A request is a step program, its options, an optional initial state and a
// step count.  The server
//   - queues requests in arrival order and admits the oldest ones while the
//     device memory they will hold fits the HBM budget and fewer than
//     max_active cases are stepping;
//   - creates admitted cases on a pool of host threads (program upload, AMG
//     set-up), so host set-up overlaps the device work of the running cases;
//   - steps every running case on its own CUDA stream, chunk_steps steps at a
//     time (one CUDA graph launch per step), so the kernels of different
//     cases overlap on the device; a case's fields stay resident from
//     admission to release;
//   - reports per request the time from submission to completion (queue +
//     run).
// Each case is an engine case of its own (hf_case_*), so its result does not
// depend on what else is running: the same bits alone and in any mix.
//
// The dispatcher is one host thread; completion is detected with CUDA events
// (no device-wide synchronisation).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "higflow_b200.h"

namespace {

using clock_t_ = std::chrono::steady_clock;

double since(clock_t_::time_point t0) { return std::chrono::duration<double>(clock_t_::now() - t0).count(); }

thread_local std::string g_srv_err;
int srv_fail(int code, const std::string &m)
{
    g_srv_err = m;
    return code;
}

// An owned copy of a step program (the caller's arrays may go away after submit).
struct ProgCopy {
    hf_program p{};
    std::vector<std::vector<char>> bufs;

    template <typename T>
    const T *keep(const T *src, size_t n)
    {
        if (!src || n == 0) return nullptr;
        bufs.emplace_back((const char *)src, (const char *)src + n * sizeof(T));
        return (const T *)bufs.back().data();
    }

    explicit ProgCopy(const hf_program &s)
    {
        p = s;
        const int D = s.par.dim;
        const size_t nc = (size_t)s.ncell;
        p.delta = keep(s.delta, (size_t)s.ndelta * D);
        p.row_tmpl = keep(s.row_tmpl, (size_t)s.nrows);
        p.row_base = keep(s.row_base, (size_t)s.nrows);
        p.row_rhs = keep(s.row_rhs, (size_t)s.nrows);
        p.tmpl_ptr = keep(s.tmpl_ptr, (size_t)s.ntmpl + 1);
        p.tmpl_col = keep(s.tmpl_col, (size_t)s.nnz);
        p.tmpl_w = keep(s.tmpl_w, (size_t)s.nnz);
        for (int d = 0; d < 3; d++) {
            const size_t nf = d < D ? (size_t)s.nfacet[d] : 0;
            p.vel_slots[d] = keep(s.vel_slots[d], (size_t)s.vel_nslot * nf);
            p.vel_flags[d] = keep(s.vel_flags[d], nf);
            p.vel_delta[d] = keep(s.vel_delta[d], nf);
        }
        p.div_slots = keep(s.div_slots, (size_t)HF_P_NSLOT(D) * nc);
        p.cell_delta = keep(s.cell_delta, nc);
        p.p_ptr = keep(s.p_ptr, nc + 1);
        p.p_col = keep(s.p_col, (size_t)s.pnnz);
        p.p_val = keep(s.p_val, (size_t)s.pnnz);
        p.p_brhs = keep(s.p_brhs, nc);
        p.cell_slots = keep(s.cell_slots, (size_t)s.cell_nslot * nc);
        p.cell_flags = keep(s.cell_flags, s.cell_nslot ? nc : 0);
        const size_t ni = s.ninst > 0 ? (size_t)s.ninst : 0;
        p.inst_par = keep(s.inst_par, ni);
        p.cell_off = keep(s.cell_off, ni ? ni + 1 : 0);
        for (int d = 0; d < 3; d++) p.facet_off[d] = keep(s.facet_off[d], d < D && ni ? ni + 1 : 0);
        p.inst_pin = keep(s.inst_pin, ni);
        p.inst_pin_value = keep(s.inst_pin_value, ni);
    }
};

struct FieldCopy {
    int32_t field, comp;
    std::vector<double> data;
};

enum class St { Queued, Creating, Running, Done };

struct Request {
    int64_t id = 0;
    std::unique_ptr<ProgCopy> prog;
    hf_options opt{};
    int32_t nsteps = 0, remaining = 0, inflight = 0;
    std::vector<FieldCopy> init;
    St state = St::Queued;
    int status = HF_OK;
    std::string error;
    hf_case *c = nullptr;
    cudaEvent_t ev = nullptr;
    int64_t reserve = 0, bytes = 0, cells = 0;
    clock_t_::time_point t_submit, t_admit, t_done;
};

}  // namespace

struct hf_server {
    hf_server_options opt{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<int64_t, std::shared_ptr<Request>> all;
    std::deque<std::shared_ptr<Request>> queue, to_create;
    std::vector<std::shared_ptr<Request>> running;
    int64_t next_id = 1, budget = 0, reserved = 0;
    int active = 0;   // creating + running
    bool stop = false;
    std::thread dispatcher;
    std::vector<std::thread> workers;
    hf_server_counts st{};
    clock_t_::time_point t0;
};

namespace {

// admit from the queue head while memory and slots allow (lock held)
void admit(hf_server *S)
{
    while (!S->queue.empty() && S->active < S->opt.max_active) {
        auto r = S->queue.front();
        if (S->reserved + r->reserve > S->budget && S->active > 0) break;   // the oldest waits for memory
        S->queue.pop_front();
        S->reserved += r->reserve;
        S->active++;
        r->state = St::Creating;
        r->t_admit = clock_t_::now();
        S->to_create.push_back(r);
    }
    S->cv_work.notify_all();
}

void finish(hf_server *S, const std::shared_ptr<Request> &r, int status, const std::string &err)
{
    // lock held by the caller
    r->state = St::Done;
    r->status = status;
    r->error = err;
    r->t_done = clock_t_::now();
    S->active--;
    S->st.completed++;
    if (status) S->st.failed++;
    S->st.cell_steps += r->cells * (int64_t)(r->nsteps - r->remaining);
    S->cv_done.notify_all();
    admit(S);
}

void worker_main(hf_server *S)
{
    cudaSetDevice(S->opt.device);
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stop || !S->to_create.empty(); });
            if (S->stop) return;
            r = S->to_create.front();
            S->to_create.pop_front();
        }
        hf_case *c = nullptr;
        int rc = hf_case_create(&r->prog->p, &r->opt, &c);
        std::string err = rc ? hf_last_error() : "";
        for (size_t k = 0; rc == HF_OK && k < r->init.size(); k++) {
            const FieldCopy &f = r->init[k];
            rc = hf_case_set_field(c, f.field, f.comp, f.data.data(), (int64_t)f.data.size());
            if (rc) err = hf_last_error();
        }
        hf_stats hs{};
        if (rc == HF_OK) rc = hf_case_stats(c, &hs);
        if (rc == HF_OK && cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming) != cudaSuccess) {
            rc = HF_ERR_CUDA;
            err = "event";
        }
        std::lock_guard<std::mutex> lk(S->mu);
        r->prog.reset();   // the engine holds its own copy now
        r->init.clear();
        if (rc) {
            if (c) hf_case_destroy(c);
            S->reserved -= r->reserve;
            r->reserve = 0;
            finish(S, r, rc, err);
            continue;
        }
        r->c = c;
        r->bytes = (int64_t)hs.device_bytes;
        S->reserved += r->bytes - r->reserve;   // the estimate replaced by what the case holds
        r->reserve = r->bytes;
        r->state = St::Running;
        S->running.push_back(r);
        S->cv_work.notify_all();
    }
}

void dispatcher_main(hf_server *S)
{
    cudaSetDevice(S->opt.device);
    std::vector<std::shared_ptr<Request>> mine;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->running.empty() && mine.empty())
                S->cv_work.wait(lk, [&] { return S->stop || !S->running.empty(); });
            if (S->stop) return;
            for (auto &r : S->running) mine.push_back(r);
            S->running.clear();
        }
        bool progressed = false;
        for (size_t k = 0; k < mine.size();) {
            auto &r = mine[k];
            if (r->inflight > 0) {
                const cudaError_t q = cudaEventQuery(r->ev);
                if (q == cudaErrorNotReady) { k++; continue; }
                r->remaining -= r->inflight;
                r->inflight = 0;
                progressed = true;
            }
            int rc = HF_OK;
            std::string err;
            if (r->remaining > 0) {
                const int n = std::min(r->remaining, S->opt.chunk_steps);
                rc = hf_case_step_async(r->c, n);
                if (rc == HF_OK) {
                    void *st = nullptr;
                    hf_case_stream(r->c, &st);
                    if (cudaEventRecord(r->ev, (cudaStream_t)st) != cudaSuccess) rc = HF_ERR_CUDA;
                    r->inflight = n;
                }
                if (rc == HF_OK) { k++; continue; }
                err = hf_last_error();
            } else {
                rc = hf_case_synchronize(r->c);   // the solves' status
                if (rc) err = hf_last_error();
            }
            {
                std::lock_guard<std::mutex> lk(S->mu);
                finish(S, r, rc, err);
            }
            mine.erase(mine.begin() + (long)k);
            progressed = true;
        }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

}  // namespace

extern "C" const char *hf_server_last_error(void) { return g_srv_err.c_str(); }

extern "C" int hf_server_create(const hf_server_options *opt, hf_server **out)
{
    if (!out) return srv_fail(HF_ERR_INVALID, "null output");
    *out = nullptr;
    hf_server *S = new hf_server();
    if (opt) S->opt = *opt;
    if (S->opt.hbm_budget_gb <= 0) S->opt.hbm_budget_gb = 150.0;
    if (S->opt.max_active <= 0) S->opt.max_active = 64;
    if (S->opt.chunk_steps <= 0) S->opt.chunk_steps = 16;
    if (S->opt.setup_threads <= 0) S->opt.setup_threads = 8;
    S->budget = (int64_t)(S->opt.hbm_budget_gb * 1e9);
    if (cudaSetDevice(S->opt.device) != cudaSuccess) {
        delete S;
        return srv_fail(HF_ERR_NO_DEVICE, "no CUDA device");
    }
    S->t0 = clock_t_::now();
    S->dispatcher = std::thread(dispatcher_main, S);
    for (int k = 0; k < S->opt.setup_threads; k++) S->workers.emplace_back(worker_main, S);
    *out = S;
    return HF_OK;
}

extern "C" int hf_server_submit(hf_server *S, const hf_program *prog, const hf_options *opt, int32_t nsteps,
                                const hf_field_data *fields, int32_t nfields, int64_t *id)
{
    if (!S || !prog || nsteps <= 0 || nfields < 0 || (nfields && !fields)) return srv_fail(HF_ERR_INVALID, "bad argument");
    auto r = std::make_shared<Request>();
    r->prog.reset(new ProgCopy(*prog));
    if (opt) r->opt = *opt;
    r->opt.device = S->opt.device;
    r->nsteps = r->remaining = nsteps;
    r->cells = prog->ncell;
    for (int32_t k = 0; k < nfields; k++) {
        if (!fields[k].data || fields[k].n < 0) return srv_fail(HF_ERR_INVALID, "bad field data");
        r->init.push_back(FieldCopy{fields[k].field, fields[k].comp,
                                    std::vector<double>(fields[k].data, fields[k].data + fields[k].n)});
    }
    int64_t est = 0;
    if (hf_case_device_bytes(prog, &r->opt, &est)) return srv_fail(HF_ERR_INVALID, hf_last_error());
    r->reserve = est + est / 2;   // AMG hierarchy and graph scratch beyond the estimate
    if (r->reserve > S->budget) return srv_fail(HF_ERR_OOM_BUDGET, "case larger than the HBM budget");
    r->t_submit = clock_t_::now();
    std::lock_guard<std::mutex> lk(S->mu);
    r->id = S->next_id++;
    S->all[r->id] = r;
    S->queue.push_back(r);
    S->st.submitted++;
    admit(S);
    if (id) *id = r->id;
    return HF_OK;
}

extern "C" int hf_server_wait(hf_server *S, int64_t id, int32_t timeout_ms, int32_t *status, double *queue_s,
                              double *total_s)
{
    if (!S) return srv_fail(HF_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return srv_fail(HF_ERR_INVALID, "unknown request");
    auto r = it->second;
    auto done = [&] { return r->state == St::Done; };
    if (timeout_ms < 0) S->cv_done.wait(lk, done);
    else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return HF_ERR_TIMEOUT;
    if (status) *status = r->status;
    if (queue_s) *queue_s = std::chrono::duration<double>(r->t_admit - r->t_submit).count();
    if (total_s) *total_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (r->status) g_srv_err = r->error;
    return HF_OK;
}

extern "C" int hf_server_get_field(hf_server *S, int64_t id, int32_t field, int32_t comp, double *host, int64_t n)
{
    if (!S) return srv_fail(HF_ERR_INVALID, "null server");
    std::shared_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->all.find(id);
        if (it == S->all.end() || it->second->state != St::Done || !it->second->c)
            return srv_fail(HF_ERR_INVALID, "request not finished or released");
        r = it->second;
    }
    const int rc = hf_case_get_field(r->c, field, comp, host, n);
    return rc ? srv_fail(rc, hf_last_error()) : HF_OK;
}

extern "C" int hf_server_release(hf_server *S, int64_t id)
{
    if (!S) return srv_fail(HF_ERR_INVALID, "null server");
    std::shared_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->all.find(id);
        if (it == S->all.end()) return srv_fail(HF_ERR_INVALID, "unknown request");
        if (it->second->state != St::Done) return srv_fail(HF_ERR_INVALID, "request still running");
        r = it->second;
        S->all.erase(it);
        S->reserved -= r->reserve;
        admit(S);
    }
    if (r->ev) cudaEventDestroy(r->ev);
    if (r->c) hf_case_destroy(r->c);
    return HF_OK;
}

extern "C" int hf_server_stats(hf_server *S, hf_server_counts *out)
{
    if (!S || !out) return srv_fail(HF_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->queued = (int64_t)S->queue.size();
    out->active = S->active;
    out->reserved_bytes = S->reserved;
    out->seconds = since(S->t0);
    return HF_OK;
}

extern "C" void hf_server_destroy(hf_server *S)
{
    if (!S) return;
    // requests not yet admitted are dropped; admitted ones run to completion
    {
        std::unique_lock<std::mutex> lk(S->mu);
        for (auto &r : S->queue) S->all.erase(r->id);
        S->queue.clear();
        S->cv_done.wait(lk, [&] { return S->active == 0; });
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
    }
    S->dispatcher.join();
    for (auto &t : S->workers) t.join();
    for (auto &kv : S->all) {
        if (kv.second->ev) cudaEventDestroy(kv.second->ev);
        if (kv.second->c) hf_case_destroy(kv.second->c);
    }
    delete S;
}
