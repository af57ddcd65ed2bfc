// gc_serve.cu — the serving loop: requests (simulations) arrive at any time,
// are admitted while their estimated device memory fits the budget, and are
// stepped together with every running simulation of the same model
// structure (one packed context per structure, "batch").  Batches of
// different structures run concurrently, each on its own stream and host
// thread.  A batch is repacked at a round boundary when requests join or
// leave; state of the simulations that stay is copied on the device.
//
// A step that fails (a non-finite position, say) fails the whole batch's
// context, whichever request caused it: the batch's running requests then
// run again from their submitted state, each in a batch of its own, and
// only a request that fails alone fails.
//
// Rounds: every batch advances min(round_steps, the fewest steps any of its
// running requests still needs) steps, so a request stops exactly at its
// step count.  Its result is then copied to host memory and its instance is
// frozen in place (time step 0) until the batch's next repack, which drops
// it.  A batch repacks when a request failed, when no request is left
// running, when frozen particles exceed a quarter of the batch, or when the
// joining requests bring at least a quarter of the running particles or one
// of them has waited JOIN_WAIT_ROUNDS rounds: joins and leaves then share
// repacks.  A batch's repack runs on its own host
// thread just before its steps, so it overlaps the other batches' steps;
// the server's contexts draw device memory from one stream-ordered pool
// that keeps freed memory, so a repack maps no new memory and waits on no
// other stream, and a new context is built on a highest-priority stream so
// its setup kernels are not queued behind the other batches' sweeps.
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

#include <cuda_runtime.h>

#include "../../include/grasph_cuda.h"

namespace gc {
bool ctx_same_structure(gc_ctx* a, int ia, gc_ctx* b, int ib);
bool ctx_finalized(gc_ctx* c);
int ctx_ninst(gc_ctx* c);
int ctx_set_cfl(gc_ctx* c, int inst, double cfl);
int ctx_set_priority(gc_ctx* c, bool highest);
int64_t ctx_particles(gc_ctx* c, int inst);
int64_t ctx_moving_particles(gc_ctx* c, int inst);
int64_t ctx_estimate_bytes(gc_ctx* m, int inst);
int ctx_model_copy(gc_ctx* m, int inst, gc_ctx** out);
struct PackJob;
PackJob* ctx_pack_plan(int precision, const std::vector<std::pair<gc_ctx*, int>>& src);
int ctx_pack_build(PackJob* J, int device, cudaMemPool_t pool, gc_ctx** out, std::string* err);
int ctx_pack_fill(PackJob* J, gc_ctx* ctx, std::string* err);
void ctx_pack_free(PackJob* J);
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
    int waited = 0;  // rounds spent admitted but not yet packed
    bool solo = false;  // runs in a batch of its own (a retry after a batch failure)
    std::vector<Result> result;
    bool result_ready = false;  // result copied to the host by its batch's thread
    std::string err;
};

constexpr int JOIN_WAIT_ROUNDS = 2;

struct Batch {
    gc_ctx* proto = nullptr;  // the structure (model copy, no state)
    gc_ctx* ctx = nullptr;    // packed running context
    std::vector<int64_t> live;     // request ids, instance order of ctx
    std::vector<int64_t> joining;  // admitted, packed at the next repack
    bool dirty = false;            // a request failed: repack at the next round
    bool fresh = false;            // ctx is new: its first round runs on a highest-priority stream
    bool solo = false;             // holds one retried request, no other joins
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
    cudaMemPool_t pool = nullptr;  // device memory of every batch context
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
int find_batch(gc_server* s, gc_ctx* model, int64_t est, bool solo) {
    for (size_t b = 0; b < s->batches.size(); ++b) {
        Batch& B = s->batches[b];
        if (B.solo != solo || !gc::ctx_same_structure(B.proto, 0, model, 0)) continue;
        const bool empty = !B.ctx && B.live.empty() && B.joining.empty();
        if (solo ? empty : (B.est == 0 || (size_t)(B.est + est) <= s->max_batch)) return (int)b;
    }
    Batch nb;
    nb.solo = solo;
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
        const int b = find_batch(s, r.model, r.est, r.solo);
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

// One batch's work in a round: the repack (when requests joined or left)
// and the steps.  The plan is made on the server's thread; `run` touches
// only the batch's contexts, so batches run it concurrently.  A batch that
// is stepping repacks in a pipeline: its current context steps the round
// while the new one is built and the joiners' fields uploaded on another
// thread; after the round the staying requests' state is copied over and
// the new context takes over (the joiners step from the next round on).
struct Job {
    Batch* B = nullptr;
    bool repack = false;
    bool pipelined = false;          // the current context steps while the new one is built
    gc::PackJob* plan = nullptr;
    std::vector<int64_t> ids;        // the batch's requests in the new context
    std::vector<int64_t> joiners;    // of those, the ones not yet in a context
    std::vector<int64_t> stepping;   // the requests of the context that steps this round, in its instance order
    std::vector<double> cfl;
    int steps = 0;                   // this round's steps
    double cfl0 = 0;
    gc_ctx* nc = nullptr;            // the new context
    int pack_status = GC_OK;
    std::string pack_err;
    double repack_s = 0;
};

// A request of B's list still runs in B (a retried one was listed by the
// batch whose step failed and may run elsewhere now).
bool runs_in(gc_server* s, const Batch& B, const Request& r) {
    return r.state == RQ_RUNNING && r.batch == (int)(&B - s->batches.data());
}

Job plan_round(gc_server* s, Batch& B) {
    Job J;
    J.B = &B;
    int64_t live_p = 0, dead_p = 0, join_p = 0;
    int nlive = 0, waited = 0;
    int64_t left = s->round_steps;  // steps of this round over the current context's running requests
    for (int64_t id : B.live) {
        const Request& r = s->reqs[id];
        if (runs_in(s, B, r)) {
            live_p += r.moving;
            if (nlive == 0) J.cfl0 = r.cfl;
            ++nlive;
            left = std::min<int64_t>(left, r.nsteps - r.done);
        } else {
            dead_p += r.moving;
        }
    }
    for (int64_t id : B.joining) {
        join_p += s->reqs[id].moving;
        waited = std::max(waited, s->reqs[id].waited);
    }
    const bool join_now =
        !B.joining.empty() && (nlive == 0 || 4 * join_p >= live_p || waited >= JOIN_WAIT_ROUNDS);
    const bool drop_now = !B.live.empty() && (nlive == 0 || 4 * dead_p > live_p + dead_p);
    J.repack = B.dirty || join_now || drop_now;
    if (!J.repack)
        for (int64_t id : B.joining) s->reqs[id].waited += 1;
    J.pipelined = J.repack && B.ctx && nlive > 0 && !B.dirty;
    std::vector<std::pair<gc_ctx*, int>> src;
    if (!J.repack) {
        J.ids = B.live;
        J.steps = nlive > 0 ? (int)std::max<int64_t>(left, 0) : 0;
    } else {
        // the new context: the requests that still run after this round
        // (pipelined) or now, then the joiners
        if (J.pipelined) J.steps = (int)std::max<int64_t>(left, 0);
        for (size_t k = 0; k < B.live.size(); ++k) {
            const Request& r = s->reqs[B.live[k]];
            if (!runs_in(s, B, r)) continue;
            if (J.pipelined && r.nsteps - r.done <= J.steps) continue;  // finishes in this round
            src.push_back({B.ctx, (int)k});
            J.ids.push_back(B.live[k]);
        }
        for (int64_t id : B.joining) {
            src.push_back({s->reqs[id].model, 0});
            J.ids.push_back(id);
            J.joiners.push_back(id);
        }
        if (!J.pipelined) {
            // a batch that is not stepping: the new context steps this round
            left = s->round_steps;
            bool any = false;
            for (int64_t id : J.ids) {
                const Request& r = s->reqs[id];
                if (r.state != RQ_RUNNING) continue;
                left = std::min<int64_t>(left, r.nsteps - r.done);
                if (!any) J.cfl0 = r.cfl;
                any = true;
            }
            J.steps = any ? (int)std::max<int64_t>(left, 0) : 0;
        }
    }
    for (int64_t id : J.ids) J.cfl.push_back(s->reqs[id].cfl);
    if (J.repack && !src.empty()) J.plan = gc::ctx_pack_plan(s->precision, src);
    J.stepping = J.repack && !J.pipelined ? J.ids : B.live;
    return J;
}

// The results of the requests that finish in this round, copied to the
// host by the batch's own thread right after its steps (so the copies
// overlap the other batches' steps).
void collect_results(gc_server* s, Batch& B, const Job& J) {
    if (!B.ctx || B.last_status != GC_OK) return;
    for (size_t k = 0; k < J.stepping.size(); ++k) {
        Request& r = s->reqs.at(J.stepping[k]);
        if (!runs_in(s, B, r) || r.done + J.steps < r.nsteps) continue;
        std::vector<std::array<int64_t, 3>> fields;
        gc::ctx_result_fields(B.ctx, (int)k, fields);
        r.result.clear();
        r.result_ready = true;
        for (auto& f : fields) {
            Result res;
            res.handle = (int)f[0];
            res.field = (int)f[1];
            res.bytes.resize((size_t)f[2]);
            if (gc_download_field(B.ctx, (int)k, res.handle, res.field, res.bytes.data(), res.bytes.size()) !=
                GC_OK) {
                r.result_ready = false;
                r.err = gc::ctx_error(B.ctx);
                break;
            }
            r.result.push_back(std::move(res));
        }
    }
}

// Build the planned context (and, once its running sources have stopped,
// fill it with their state).
void build_new(gc_server* s, Job& J) {
    const double t0 = s->now();
    if (J.plan) {
        J.pack_status = gc::ctx_pack_build(J.plan, s->device, s->pool, &J.nc, &J.pack_err);
        if (J.pack_status == GC_OK)
            for (size_t k = 0; k < J.ids.size(); ++k) gc::ctx_set_cfl(J.nc, (int)k, J.cfl[k]);
    }
    J.repack_s += s->now() - t0;
}

void fill_new(gc_server* s, Job& J) {
    if (!J.nc || J.pack_status != GC_OK) return;
    const double t0 = s->now();
    J.pack_status = gc::ctx_pack_fill(J.plan, J.nc, &J.pack_err);
    J.repack_s += s->now() - t0;
}

void step_batch(Batch& B, const Job& J) {
    if (!B.ctx || J.steps <= 0) return;
    B.last_status = gc_step(B.ctx, J.steps, J.cfl0);
    if (B.last_status != GC_OK) B.last_err = gc_last_error(B.ctx);
    // a new context is built and takes its first (exact, capturing) steps
    // on a highest-priority stream, then steps at the normal priority
    if (B.fresh) {
        gc::ctx_set_priority(B.ctx, false);
        B.fresh = false;
    }
}

void run_round(gc_server* s, Job& J) {
    Batch& B = *J.B;
    if (J.pipelined) {
        std::thread builder([s, &J] { build_new(s, J); });
        step_batch(B, J);
        collect_results(s, B, J);
        builder.join();
        if (B.last_status == GC_OK) fill_new(s, J);
        return;  // the server thread switches contexts after the round's bookkeeping
    }
    if (J.repack) {
        build_new(s, J);
        fill_new(s, J);
        if (B.ctx) gc_ctx_destroy(B.ctx);
        B.ctx = J.pack_status == GC_OK ? J.nc : nullptr;
        B.fresh = B.ctx != nullptr;
        J.nc = nullptr;
    }
    step_batch(B, J);
    collect_results(s, B, J);
}

// The repack's bookkeeping, on the server's thread (after the round's
// results were read when the repack was pipelined).
void finish_repack(gc_server* s, Job& J, bool round_ok) {
    if (!J.repack) return;
    Batch& B = *J.B;
    // finished requests leave the batch now: their reservation ends
    for (int64_t id : B.live) {
        const Request& r = s->reqs[id];
        if (r.state != RQ_DONE) continue;
        s->used -= std::min(s->used, (size_t)r.est);
        B.est -= std::min(B.est, r.est);
    }
    B.joining.clear();
    B.dirty = false;
    if (J.pipelined) {
        if (B.ctx) gc_ctx_destroy(B.ctx);
        B.ctx = nullptr;
        if (!round_ok) {
            // the round failed (its requests with it): the joiners wait for
            // the next round's context
            if (J.nc) gc_ctx_destroy(J.nc);
            J.nc = nullptr;
            B.live.clear();
            B.joining = J.joiners;
            return;
        }
        if (J.pack_status == GC_OK) {
            B.ctx = J.nc;
            B.fresh = B.ctx != nullptr;
        } else if (J.nc) {
            gc_ctx_destroy(J.nc);
        }
        J.nc = nullptr;
    }
    if (J.pack_status != GC_OK) {
        for (int64_t id : J.ids) {
            Request& r = s->reqs[id];
            r.state = RQ_FAILED;
            r.err = "repack: " + J.pack_err;
            s->used -= std::min(s->used, (size_t)r.est);
        }
        B.est = 0;
        B.live.clear();
        serr(s, J.pack_status, "repack: " + J.pack_err);
        return;
    }
    B.live = J.ids;
    s->stats.repacks += 1;
    s->stats.repack_instances += (int64_t)J.ids.size();
    s->stats.repack_seconds += J.repack_s;
}

// After a round of `steps` steps: count them, copy finished results to the
// host and freeze their instances; a failure marks the batch for a repack.
void retire(gc_server* s, Batch& B, int steps, int* ncompleted) {
    std::vector<int64_t> retry;
    for (size_t k = 0; k < B.live.size(); ++k) {
        Request& r = s->reqs[B.live[k]];
        if (!runs_in(s, B, r)) continue;
        if (B.last_status != GC_OK) {
            if (!r.solo) {
                // another request may have caused it: again, alone
                r.solo = true;
                r.state = RQ_QUEUED;
                r.done = 0;
                r.waited = 0;
                r.batch = -1;
                r.t_admit = -1;
                r.result.clear();
                r.result_ready = false;
                retry.push_back(r.id);
                s->stats.retries += 1;
            } else {
                r.state = RQ_FAILED;
                r.err = B.last_err;
            }
        } else {
            r.done += steps;
            s->stats.particle_steps += r.moving * steps;
            if (r.done < r.nsteps) continue;
            // the batch's thread copied the result (collect_results)
            if (!r.result_ready) r.state = RQ_FAILED;
            if (r.state != RQ_FAILED) {
                r.state = RQ_DONE;
                r.t_done = s->now();
                ++*ncompleted;
                // frozen until the next repack drops it (still stepped, but
                // with dt = 0 its state does not change)
                gc::ctx_set_cfl(B.ctx, (int)k, 0.0);
                continue;
            }
        }
        s->used -= std::min(s->used, (size_t)r.est);
        B.est -= std::min(B.est, r.est);
        B.dirty = true;
    }
    // retried requests go to the front of the queue, in their order
    s->queue.insert(s->queue.begin(), retry.begin(), retry.end());
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
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
        delete s;
        return GC_ERR_CUDA;
    }
    // keep freed memory in the pool for the next repack (released when the
    // server is destroyed)
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
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
    if (s->pool) cudaMemPoolDestroy(s->pool);
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
    std::vector<Job> jobs;
    for (auto& B : s->batches)
        if (B.ctx || !B.joining.empty()) jobs.push_back(plan_round(s, B));
    // each batch repacks and steps on its own thread (one batch: this one)
    if (jobs.size() == 1) {
        run_round(s, jobs[0]);
    } else {
        std::vector<std::thread> th;
        for (auto& J : jobs) th.emplace_back([s, &J] { run_round(s, J); });
        for (auto& t : th) t.join();
    }
    for (auto& J : jobs) {
        if (J.pipelined) {
            // the round ran on the current context: its results first
            const bool ok = J.B->last_status == GC_OK;
            retire(s, *J.B, J.steps, &done);
            finish_repack(s, J, ok);
        } else {
            finish_repack(s, J, true);
            // (requests that need no steps at all finish now)
            if (J.B->ctx) retire(s, *J.B, J.steps, &done);
        }
        if (J.plan) gc::ctx_pack_free(J.plan);
    }
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
        for (int64_t id : B.live) out->running += runs_in(s, B, s->reqs[id]);
        out->running += (int64_t)B.joining.size();
    }
    out->device_bytes_reserved = (int64_t)s->used;
    return GC_OK;
}

}  // extern "C"
