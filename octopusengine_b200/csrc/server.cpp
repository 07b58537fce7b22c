// Serving loop: continuous batching of (scene, steps) requests on one device, built on the
// public C ABI (scenes, batches).  The reference has no server; its host loop steps one
// scene per frame (octopus/src/Script/Dynamic/Cuda_ParticleSystem_Dynamic.cpp:17-31).
//
// Admission: FIFO; the head request is admitted when a slot is free and its estimated device
// footprint (oct_scene_footprint) fits the remaining budget, otherwise it waits; a request
// larger than the whole budget is rejected at submit.  Set-up of admitted scenes (mesh
// graphs, colouring, FP64 precompute, upload) runs on host worker threads while the GPU
// advances the current batch; ready scenes join the batch at the next frame boundary.
// Membership changes are known while a frame runs (the requests on their last step, the
// scenes whose set-up finished), so the next frame's batch is built and its graph captured
// during the current frame; the GPU then goes from one frame to the next without waiting
// on the host.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <future>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/octopus_b200.h"

namespace {

struct Request {
    int64_t id = 0;
    int steps_total = 0, steps_done = 0;
    std::vector<float> X, masses, ype, v0;
    std::vector<int32_t> topo, fixed;
    oct_scene_desc desc{};
    size_t bytes = 0;
    oct_scene* scene = nullptr;
    std::future<oct_status> setup;
    bool done = false;
    oct_status status = OCT_OK;
    std::vector<float> result;
    int64_t free_nodes = 0;
};

int nodes_per_element(int e) {
    switch (e) { case 3: return 4; case 6: return 8; case 7: return 10; case 8: return 20; case 9: return 27; default: return -1; }
}

}  // namespace

struct oct_server {
    oct_ctx* ctx = nullptr;
    oct_server_config cfg{};
    size_t budget = 0, reserved = 0;
    int64_t next_id = 1;
    std::deque<Request*> queue;
    std::vector<Request*> staging, active, joining;   // joining: set up, enter at the next frame
    std::map<int64_t, std::unique_ptr<Request>> all;
    oct_batch* batch = nullptr;
    bool dirty = true;
    std::vector<double> frame_ms;
    double vertex_iterations = 0, busy_ms = 0;
    int64_t submitted = 0, admitted = 0, finished = 0, rejected = 0, failed = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr, prev_end = nullptr;
    bool have_prev = false;
    double gap_ms = 0;   // device idle time between consecutive frames
    cudaStream_t stream = nullptr;
};

extern "C" {

oct_status oct_server_create(oct_ctx* ctx, const oct_server_config* cfg, oct_server** out) {
    if (!ctx || !cfg || !out || cfg->max_scenes <= 0 || !(cfg->frame_dt > 0.f) || cfg->substeps <= 0 || cfg->iterations <= 0)
        return OCT_EINVAL;
    auto* s = new oct_server();
    s->ctx = ctx;
    s->cfg = *cfg;
    size_t used = 0, budget = 0;
    oct_ctx_memory(ctx, &used, &budget);
    s->budget = cfg->hbm_budget ? std::min(cfg->hbm_budget, budget - used) : budget - used;
    void* st = nullptr;
    oct_ctx_stream(ctx, &st);
    s->stream = (cudaStream_t)st;
    if (cudaEventCreate(&s->e0) != cudaSuccess || cudaEventCreate(&s->e1) != cudaSuccess ||
        cudaEventCreate(&s->prev_end) != cudaSuccess) { delete s; return OCT_ECUDA; }
    *out = s;
    return OCT_OK;
}

oct_status oct_server_submit(oct_server* s, const oct_scene_desc* d, int32_t steps, int64_t* id) {
    if (!s || !d || steps <= 0 || !id) return OCT_EINVAL;
    const int ne = nodes_per_element(d->element);
    if (ne < 0 || d->n_nodes <= 0 || d->n_elements <= 0 || !d->positions || !d->topology) return OCT_EINVAL;
    auto r = std::make_unique<Request>();
    r->id = s->next_id++;
    r->steps_total = steps;
    r->desc = *d;
    r->desc.iterations = s->cfg.iterations;
    r->desc.precision = s->cfg.precision;
    r->desc.solver = OCT_SOLVER_VBD;
    r->desc.order_mode = OCT_ORDER_ASCENDING;
    r->X.assign(d->positions, d->positions + 3 * (size_t)d->n_nodes);
    r->topo.assign(d->topology, d->topology + (size_t)ne * d->n_elements);
    r->desc.positions = r->X.data();
    r->desc.topology = r->topo.data();
    if (d->masses) { r->masses.assign(d->masses, d->masses + d->n_nodes); r->desc.masses = r->masses.data(); }
    if (d->young_per_element) {
        r->ype.assign(d->young_per_element, d->young_per_element + d->n_elements);
        r->desc.young_per_element = r->ype.data();
    }
    if (d->initial_velocity) {
        r->v0.assign(d->initial_velocity, d->initial_velocity + 3 * (size_t)d->n_nodes);
        r->desc.initial_velocity = r->v0.data();
    }
    if (d->n_fixed > 0 && d->fixed_ids) {
        r->fixed.assign(d->fixed_ids, d->fixed_ids + d->n_fixed);
        r->desc.fixed_ids = r->fixed.data();
    }
    oct_status st = oct_scene_footprint(&r->desc, &r->bytes);
    if (st) return st;
    s->submitted++;
    *id = r->id;
    if (r->bytes > s->budget) {   // can never fit: reject, nothing queued
        s->rejected++;
        r->done = true;
        r->status = OCT_ENOMEM_BUDGET;
        s->all[r->id] = std::move(r);
        return OCT_ENOMEM_BUDGET;
    }
    s->queue.push_back(r.get());
    s->all[r->id] = std::move(r);
    return OCT_OK;
}

namespace {

void collect_ready(oct_server* s, bool wait_all) {
    for (auto it = s->staging.begin(); it != s->staging.end();) {
        Request* r = *it;
        if (!wait_all && r->setup.wait_for(std::chrono::seconds(0)) != std::future_status::ready) { ++it; continue; }
        r->status = r->setup.get();
        if (r->status == OCT_OK) {
            int32_t nn = 0, nf = 0;
            oct_scene_info(r->scene, &nn, nullptr, nullptr, &nf);
            r->free_nodes = nn - nf;
            s->joining.push_back(r);
        } else {
            r->done = true;
            s->reserved -= r->bytes;
            s->rejected++;
        }
        it = s->staging.erase(it);
    }
}

oct_status build_batch(oct_server* s, const std::vector<Request*>& members, oct_batch** out) {
    *out = nullptr;
    if (members.empty()) return OCT_OK;
    std::vector<oct_scene*> sc;
    for (auto* r : members) sc.push_back(r->scene);
    oct_status st = oct_batch_create(s->ctx, sc.data(), (int)sc.size(), out);
    if (st) return st;
    return oct_batch_prepare(*out, s->cfg.frame_dt, s->cfg.substeps);
}

void admit(oct_server* s) {
    const int threads = s->cfg.setup_threads > 0 ? s->cfg.setup_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    while (!s->queue.empty()) {
        Request* r = s->queue.front();
        const int slots = (int)(s->active.size() + s->staging.size());
        if (slots >= s->cfg.max_scenes || (int)s->staging.size() >= threads || s->reserved + r->bytes > s->budget) break;
        s->queue.pop_front();
        s->reserved += r->bytes;
        s->admitted++;
        oct_ctx* ctx = s->ctx;
        r->setup = std::async(std::launch::async, [ctx, r]() { return oct_scene_create(ctx, &r->desc, &r->scene); });
        s->staging.push_back(r);
    }
}

}  // namespace

oct_status oct_server_tick(oct_server* s, int32_t* n_active) {
    if (!s) return OCT_EINVAL;
    admit(s);
    // scenes join while a frame runs; only an idle server takes them here (waiting for a set-up
    // when there is nothing else to do)
    if (s->active.empty()) {
        collect_ready(s, false);
        if (s->joining.empty() && !s->staging.empty()) collect_ready(s, true);
    }
    if (!s->joining.empty() || s->dirty) {   // membership changed outside a frame
        s->active.insert(s->active.end(), s->joining.begin(), s->joining.end());
        s->joining.clear();
        if (s->batch) { oct_batch_destroy(s->batch); s->batch = nullptr; }
        oct_status st = build_batch(s, s->active, &s->batch);
        if (st) return st;
        s->dirty = false;
    }
    if (!s->active.empty()) {
        cudaEventRecord(s->e0, s->stream);
        oct_status st = oct_batch_step(s->batch, s->cfg.frame_dt, s->cfg.substeps);
        if (st) return st;
        cudaEventRecord(s->e1, s->stream);
        // while the frame runs: start queued set-ups, collect finished ones and build the next
        // frame's batch (members without the requests on their last step, plus the joiners)
        admit(s);
        collect_ready(s, false);
        std::vector<Request*> next;
        bool leaving = false;
        for (auto* r : s->active) {
            if (r->steps_done + 1 >= r->steps_total) leaving = true;
            else next.push_back(r);
        }
        next.insert(next.end(), s->joining.begin(), s->joining.end());
        oct_batch* next_batch = nullptr;
        const bool changed = leaving || !s->joining.empty();
        if (changed && (st = build_batch(s, next, &next_batch))) return st;
        if (cudaEventSynchronize(s->e1) != cudaSuccess) return OCT_ECUDA;
        // per-request failure state of the frame: a request whose state went non-finite or
        // whose work timed out ends with that status; scenes are independent, so the others
        // carry on unchanged
        std::vector<int32_t> flags(s->active.size(), OCT_OK);
        if ((st = oct_batch_status(s->batch, flags.data()))) return st;
        std::vector<Request*> failed;
        for (size_t i = 0; i < s->active.size(); ++i)
            if (flags[i] != OCT_OK) { s->active[i]->status = (oct_status)flags[i]; failed.push_back(s->active[i]); }
        float ms = 0.f, gap = 0.f;
        cudaEventElapsedTime(&ms, s->e0, s->e1);
        if (s->have_prev && cudaEventElapsedTime(&gap, s->prev_end, s->e0) == cudaSuccess) s->gap_ms += gap;
        cudaEventRecord(s->prev_end, s->stream);   // the frame's end, for the next gap
        s->have_prev = true;
        s->frame_ms.push_back(ms);
        s->busy_ms += ms;
        if (changed) {   // the finished frame's batch is no longer needed
            oct_batch_destroy(s->batch);
            s->batch = next_batch;
        }
        for (auto* r : s->active) {
            s->vertex_iterations += (double)r->free_nodes * s->cfg.iterations * s->cfg.substeps;
            const bool bad = r->status != OCT_OK;
            if (++r->steps_done >= r->steps_total || bad) {
                if (!bad) {
                    r->result.resize(3 * (size_t)r->desc.n_nodes);
                    r->status = oct_scene_get_positions(r->scene, r->result.data());
                }
                oct_scene_destroy(r->scene);
                r->scene = nullptr;
                r->done = true;
                s->reserved -= r->bytes;
                if (bad) s->failed++;
                else s->finished++;
            }
        }
        if (changed) {
            s->active = next;
            s->joining.clear();
        }
        if (!failed.empty()) {   // failed requests leave now; the next tick rebuilds the batch
            auto gone = [&](Request* r) { return std::find(failed.begin(), failed.end(), r) != failed.end(); };
            s->active.erase(std::remove_if(s->active.begin(), s->active.end(), gone), s->active.end());
            if (s->batch) { oct_batch_destroy(s->batch); s->batch = nullptr; }
            s->dirty = true;
        }
    }
    if (s->active.empty()) s->have_prev = false;   // idle: the next gap is not a host delay
    if (n_active) *n_active = (int32_t)s->active.size();
    return OCT_OK;
}

oct_status oct_server_poll(oct_server* s, int64_t id, int32_t* done, float* positions) {
    if (!s || !done) return OCT_EINVAL;
    auto it = s->all.find(id);
    if (it == s->all.end()) return OCT_EINVAL;
    Request* r = it->second.get();
    *done = r->done ? 1 : 0;
    if (r->done && positions && !r->result.empty()) std::copy(r->result.begin(), r->result.end(), positions);
    return r->done ? r->status : OCT_OK;
}

oct_status oct_server_get_stats(oct_server* s, oct_server_stats* o) {
    if (!s || !o) return OCT_EINVAL;
    std::memset(o, 0, sizeof(*o));
    o->submitted = s->submitted;
    o->admitted = s->admitted;
    o->finished = s->finished;
    o->rejected = s->rejected;
    o->failed = s->failed;
    o->queued = (int64_t)s->queue.size();
    o->active = (int64_t)s->active.size();
    o->frames = (int64_t)s->frame_ms.size();
    o->vertex_iterations = s->vertex_iterations;
    o->busy_ms = s->busy_ms;
    o->bytes_in_use = s->reserved;
    o->gap_ms = s->gap_ms;
    if (!s->frame_ms.empty()) {
        std::vector<double> v(s->frame_ms);
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const double x = p * (v.size() - 1);
            const size_t i = (size_t)x;
            const double f = x - i;
            return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
        };
        o->p50_step_ms = pct(0.50);
        o->p99_step_ms = pct(0.99);
        double sum = 0;
        for (double x : v) sum += x;
        o->mean_step_ms = sum / v.size();
    }
    return OCT_OK;
}

oct_status oct_server_destroy(oct_server* s) {
    if (!s) return OCT_EINVAL;
    collect_ready(s, true);
    if (s->batch) oct_batch_destroy(s->batch);
    for (auto* r : s->active) if (r->scene) oct_scene_destroy(r->scene);
    for (auto* r : s->joining) if (r->scene) oct_scene_destroy(r->scene);
    cudaEventDestroy(s->e0);
    cudaEventDestroy(s->e1);
    cudaEventDestroy(s->prev_end);
    delete s;
    return OCT_OK;
}

}  // extern "C"
