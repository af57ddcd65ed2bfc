// gc_serve.cu — the serving loop: requests (simulations) arrive at any time,
// are admitted while their estimated device memory fits the budget, and are
// stepped together with every running simulation of the same model
// structure (one packed context per structure, "batch").  Batches of
// different structures run concurrently, each on its own stream and host
// thread.  A batch is repacked at a round boundary when requests join or
// leave; state of the simulations that stay is copied on the device.
//
// Rounds: every batch advances min(round_steps, the fewest steps any of its
// requests still needs) steps, so a request stops exactly at its step
// count.  Its result is then copied to host memory and the request leaves
// the batch at the next repack.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/grasph_cuda.h"

namespace gc {
bool ctx_same_structure(gc_ctx* a, int ia, gc_ctx* b, int ib);
bool ctx_finalized(gc_ctx* c);
int ctx_ninst(gc_ctx* c);
int ctx_set_cfl(gc_ctx* c, int inst, double cfl);
int64_t ctx_particles(gc_ctx* c, int inst);
int64_t ctx_moving_particles(gc_ctx* c, int inst);
int64_t ctx_estimate_bytes(gc_ctx* m, int inst);
int ctx_model_copy(gc_ctx* m, int inst, gc_ctx** out);
int ctx_pack(int device, size_t budget, int precision, const std::vector<std::pair<gc_ctx*, int>>& src,
             gc_ctx** out, std::string* err);
void ctx_result_fields(gc_ctx* c, int inst, std::vector<std::array<int64_t, 3>>& out);
const char* ctx_error(gc_ctx* c);
}  // namespace gc

namespace {

enum { RQ_QUEUED = 0, RQ_RUNNING = 1, RQ_DONE = 2, RQ_FAILED = -1 };

struct Result {
    int handle, field;
    std::vector<char> bytes;
};

struct Request {
    int64_t id = 0;
    gc_ctx* model = nullptr;  // one instance, unfinalized, fields staged
    int nsteps = 0;
    double cfl = 0;
    int state = RQ_QUEUED;
    int64_t done = 0;
    double t_submit = 0, t_admit = -1, t_done = -1;
    int64_t est = 0, particles = 0, moving = 0;
    int batch = -1;
    std::vector<Result> result;
    std::string err;
};

struct Batch {
    gc_ctx* proto = nullptr;  // the structure (model copy, no state)
    gc_ctx* ctx = nullptr;    // packed running context
    std::vector<int64_t> live;     // request ids, instance order of ctx
    std::vector<int64_t> joining;  // admitted, packed at the next repack
    bool dirty = false;            // a request left
    int64_t est = 0;               // estimated bytes of live + joining requests
    int last_status = GC_OK;
    std::string last_err;
};

}  // namespace

struct gc_server {
    int device = 0;
    size_t budget = 0;
    int round_steps = 50;
    int precision = GC_PRECISION_FP32_COMPENSATED;
    std::map<int64_t, Request> reqs;
    std::deque<int64_t> queue;
    std::vector<Batch> batches;
    size_t used = 0;
    size_t max_batch = 0;  // estimated bytes one batch may hold (bounds a repack's peak)
    int64_t next_id = 1;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    gc_serve_stats stats{};
    std::string err;
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

int serr(gc_server* s, int code, const std::string& msg) {
    s->err = msg;
    return code;
}

// A batch of the same structure with room for `est` more bytes, else a new
// one.  A repack holds the old and the new context at once, so batches are
// kept to a fraction of the budget.
int find_batch(gc_server* s, gc_ctx* model, int64_t est) {
    for (size_t b = 0; b < s->batches.size(); ++b) {
        Batch& B = s->batches[b];
        if (!gc::ctx_same_structure(B.proto, 0, model, 0)) continue;
        if (B.est == 0 || (size_t)(B.est + est) <= s->max_batch) return (int)b;
    }
    Batch nb;
    if (gc::ctx_model_copy(model, 0, &nb.proto) != GC_OK) return -1;
    s->batches.push_back(nb);
    return (int)s->batches.size() - 1;
}

// Admission in arrival order; a request that does not fit waits (later,
// smaller ones may still be admitted).  One that can never fit fails.
void admit(gc_server* s) {
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Request& r = s->reqs[*it];
        if (s->budget && (size_t)r.est > s->budget) {
            r.state = RQ_FAILED;
            r.err = "request needs more device memory than the whole budget";
            it = s->queue.erase(it);
            continue;
        }
        if (s->budget && s->used + (size_t)r.est > s->budget) {
            ++it;
            continue;
        }
        const int b = find_batch(s, r.model, r.est);
        if (b < 0) {
            ++it;
            continue;
        }
        s->batches[b].est += r.est;
        s->used += (size_t)r.est;
        r.state = RQ_RUNNING;
        r.t_admit = s->now();
        r.batch = b;
        s->batches[b].joining.push_back(r.id);
        it = s->queue.erase(it);
    }
}

// Rebuild a batch's context: the requests of `live` that still run (state
// copied on the device from the old context) followed by the joining ones
// (staged host fields).
int repack(gc_server* s, Batch& B) {
    if (!B.dirty && B.joining.empty()) return GC_OK;
    std::vector<std::pair<gc_ctx*, int>> src;
    std::vector<int64_t> ids;
    for (size_t k = 0; k < B.live.size(); ++k)
        if (s->reqs[B.live[k]].state == RQ_RUNNING) {
            src.push_back({B.ctx, (int)k});
            ids.push_back(B.live[k]);
        }
    for (int64_t id : B.joining) {
        src.push_back({s->reqs[id].model, 0});
        ids.push_back(id);
    }
    gc_ctx* nc = nullptr;
    if (!src.empty()) {
        std::string e;
        int st = gc::ctx_pack(s->device, 0, s->precision, src, &nc, &e);
        if (st != GC_OK) {
            for (int64_t id : ids) {
                Request& r = s->reqs[id];
                r.state = RQ_FAILED;
                r.err = "repack: " + e;
                s->used -= std::min(s->used, (size_t)r.est);
            }
            B.est = 0;
            if (B.ctx) gc_ctx_destroy(B.ctx);
            B.ctx = nullptr;
            B.live.clear();
            B.joining.clear();
            B.dirty = false;
            return serr(s, st, "repack: " + e);
        }
        for (size_t k = 0; k < ids.size(); ++k) gc::ctx_set_cfl(nc, (int)k, s->reqs[ids[k]].cfl);
    }
    if (B.ctx) gc_ctx_destroy(B.ctx);
    B.ctx = nc;
    B.live = ids;
    B.joining.clear();
    B.dirty = false;
    s->stats.repacks += 1;
    return GC_OK;
}

// After a round of `steps` steps: count them, copy finished results to the
// host, mark the batch for a repack when a request left.
void retire(gc_server* s, Batch& B, int steps, int* ncompleted) {
    for (size_t k = 0; k < B.live.size(); ++k) {
        Request& r = s->reqs[B.live[k]];
        if (r.state != RQ_RUNNING) continue;
        if (B.last_status != GC_OK) {
            r.state = RQ_FAILED;
            r.err = B.last_err;
        } else {
            r.done += steps;
            s->stats.particle_steps += r.moving * steps;
            if (r.done < r.nsteps) continue;
            std::vector<std::array<int64_t, 3>> fields;
            gc::ctx_result_fields(B.ctx, (int)k, fields);
            r.result.clear();
            for (auto& f : fields) {
                Result res;
                res.handle = (int)f[0];
                res.field = (int)f[1];
                res.bytes.resize((size_t)f[2]);
                if (gc_download_field(B.ctx, (int)k, res.handle, res.field, res.bytes.data(), res.bytes.size()) !=
                    GC_OK) {
                    r.state = RQ_FAILED;
                    r.err = gc::ctx_error(B.ctx);
                    break;
                }
                r.result.push_back(std::move(res));
            }
            if (r.state != RQ_FAILED) {
                r.state = RQ_DONE;
                r.t_done = s->now();
                ++*ncompleted;
            }
        }
        s->used -= std::min(s->used, (size_t)r.est);
        B.est -= std::min(B.est, r.est);
        B.dirty = true;
    }
    B.last_status = GC_OK;
}

}  // namespace

extern "C" {

int gc_serve_create(int device, size_t hbm_budget_bytes, int round_steps, int precision, gc_server** out) {
    if (!out || round_steps < 1) return GC_ERR_ARG;
    if (precision != GC_PRECISION_FP64 && precision != GC_PRECISION_FP32_COMPENSATED) return GC_ERR_ARG;
    gc_server* s = new gc_server;
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->round_steps = round_steps;
    s->precision = precision;
    s->max_batch = hbm_budget_bytes ? std::max<size_t>(hbm_budget_bytes / 8, (size_t)1 << 30) : (size_t)16 << 30;
    *out = s;
    return GC_OK;
}

int gc_serve_destroy(gc_server* s) {
    if (!s) return GC_OK;
    for (auto& B : s->batches) {
        if (B.ctx) gc_ctx_destroy(B.ctx);
        if (B.proto) gc_ctx_destroy(B.proto);
    }
    for (auto& kv : s->reqs)
        if (kv.second.model) gc_ctx_destroy(kv.second.model);
    delete s;
    return GC_OK;
}

const char* gc_serve_last_error(gc_server* s) { return s ? s->err.c_str() : "null server"; }

int gc_serve_submit(gc_server* s, gc_ctx* model, int nsteps, double cfl, int64_t* req_out) {
    if (!s || !model || !req_out) return GC_ERR_ARG;
    if (gc::ctx_finalized(model) || gc::ctx_ninst(model) != 1)
        return serr(s, GC_ERR_ARG, "a request is one unfinalized instance with staged fields");
    if (nsteps < 0 || !(cfl > 0.0) || !std::isfinite(cfl)) return serr(s, GC_ERR_ARG, "bad step count or CFL");
    Request r;
    r.id = s->next_id++;
    r.model = model;
    r.nsteps = nsteps;
    r.cfl = cfl;
    r.t_submit = s->now();
    r.est = gc::ctx_estimate_bytes(model, 0);
    r.particles = gc::ctx_particles(model, 0);
    r.moving = gc::ctx_moving_particles(model, 0);
    s->reqs[r.id] = std::move(r);
    s->queue.push_back(*req_out = s->next_id - 1);
    return GC_OK;
}

int gc_serve_pump(gc_server* s, int* ncompleted) {
    if (!s) return GC_ERR_ARG;
    int done = 0;
    admit(s);
    for (auto& B : s->batches) repack(s, B);
    // requests that need no steps at all finish now
    std::vector<Batch*> run;
    std::vector<int> steps;
    for (auto& B : s->batches) {
        if (!B.ctx) continue;
        int64_t left = s->round_steps;
        for (int64_t id : B.live) left = std::min<int64_t>(left, s->reqs[id].nsteps - s->reqs[id].done);
        run.push_back(&B);
        steps.push_back((int)std::max<int64_t>(left, 0));
    }
    std::vector<std::thread> th;
    for (size_t i = 0; i < run.size(); ++i) {
        if (steps[i] == 0) continue;
        th.emplace_back([&, i] {
            Batch& B = *run[i];
            B.last_status = gc_step(B.ctx, steps[i], s->reqs[B.live[0]].cfl);
            if (B.last_status != GC_OK) B.last_err = gc_last_error(B.ctx);
        });
    }
    for (auto& t : th) t.join();
    for (size_t i = 0; i < run.size(); ++i) retire(s, *run[i], steps[i], &done);
    s->stats.rounds += 1;
    if (ncompleted) *ncompleted = done;
    return GC_OK;
}

int gc_serve_poll(gc_server* s, int64_t req, int* state, int64_t* steps_done, double* t_submit, double* t_admit,
                  double* t_done) {
    if (!s) return GC_ERR_ARG;
    auto it = s->reqs.find(req);
    if (it == s->reqs.end()) return serr(s, GC_ERR_ARG, "unknown request");
    const Request& r = it->second;
    if (state) *state = r.state;
    if (steps_done) *steps_done = r.done;
    if (t_submit) *t_submit = r.t_submit;
    if (t_admit) *t_admit = r.t_admit;
    if (t_done) *t_done = r.t_done;
    if (r.state == RQ_FAILED) s->err = r.err;
    return GC_OK;
}

int gc_serve_download(gc_server* s, int64_t req, int handle, int field, void* host, size_t bytes) {
    if (!s || !host) return GC_ERR_ARG;
    auto it = s->reqs.find(req);
    if (it == s->reqs.end()) return serr(s, GC_ERR_ARG, "unknown request");
    const Request& r = it->second;
    if (r.state != RQ_DONE) return serr(s, GC_ERR_STATE, "request not completed");
    for (auto& f : r.result)
        if (f.handle == handle && f.field == field) {
            if (f.bytes.size() != bytes) return serr(s, GC_ERR_ARG, "byte count mismatch");
            memcpy(host, f.bytes.data(), bytes);
            return GC_OK;
        }
    return serr(s, GC_ERR_ARG, "field not present on this system");
}

int gc_serve_release(gc_server* s, int64_t req) {
    if (!s) return GC_ERR_ARG;
    auto it = s->reqs.find(req);
    if (it == s->reqs.end()) return serr(s, GC_ERR_ARG, "unknown request");
    if (it->second.state == RQ_RUNNING || it->second.state == RQ_QUEUED)
        return serr(s, GC_ERR_STATE, "request still queued or running");
    if (it->second.model) gc_ctx_destroy(it->second.model);
    s->reqs.erase(it);
    return GC_OK;
}

int gc_serve_get_stats(gc_server* s, gc_serve_stats* out) {
    if (!s || !out) return GC_ERR_ARG;
    *out = s->stats;
    out->queued = (int64_t)s->queue.size();
    out->running = 0;
    out->batches = 0;
    for (auto& B : s->batches) {
        if (B.ctx) out->batches += 1;
        for (int64_t id : B.live) out->running += s->reqs[id].state == RQ_RUNNING;
        out->running += (int64_t)B.joining.size();
    }
    out->device_bytes_reserved = (int64_t)s->used;
    return GC_OK;
}

}  // extern "C"
