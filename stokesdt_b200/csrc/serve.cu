// Served request stream: device-resident systems and a request queue.
//
// The reference has no server; a request is the reference's per-call work on
// one system -- MobSpme::MulVector (a mobility apply) or BrwnLanczos::Compute
// (a Brownian step) with k right-hand sides (src/mob/mob_spme.cc:219-263,
// src/brwn/brwn_lanczos.cc:278-304).  Systems are registered once: their
// engine (grid, tables, pair list after the positions' Update) stays on the
// device, admitted only while the estimated device memory of all registered
// systems fits the HBM budget.  Requests are queued in arrival order and
// taken by `lanes` workers (a CUDA stream, a host thread and a Lanczos
// workspace each); a system serves one request at a time, so requests on
// different systems overlap and requests on one system keep their order.
//
// Continuous batching (monodisperse systems with K <= 256, requests of at
// most 16 RHS): two batch lanes, each with a packed product state and a
// batched block Lanczos over all such systems (packed.h,
// packed_lanczos.h).  A free lane takes the oldest waiting request that has
// a partner -- another waiting request of the same kind and RHS count on
// another idle system -- with every such partner (up to max_batch), and runs
// them as one packed product or one lockstep Lanczos; requests that arrive
// meanwhile join the next batch, and the two lanes' batches overlap on the
// device.  A request without a partner goes to a per-request worker (a lone
// request runs faster there), or to a free batch lane when every worker is
// busy.  STOKESDT_SERVE_BATCH=all sends every batchable request to the batch
// lanes (one worker is kept for the rest); =0 turns batching off.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <string>

#include "serve.h"

namespace sdt {

using Clock = std::chrono::steady_clock;

static double now_ms()
{
    return std::chrono::duration<double, std::milli>(Clock::now().time_since_epoch()).count();
}

// Device bytes one system needs with up to `rhs` vectors per call (grids,
// tables, particle and segment arrays, pair list estimate).
size_t serve_system_bytes(int npos, double box, int K, double rmax, int rhs)
{
    const double xs = K / 2 + 4;
    const double grid = 3.0 * K * K * xs * 8.0 * rhs;
    const double tabs = 2.0 * K * K * xs * 4.0;
    const double rho = npos / (box * box * box);
    const double pairs = npos * rho * 4.0 / 3.0 * M_PI * rmax * rmax * rmax;
    const double part = npos * (36.0 * 12.0 + 3 * 8 * 4.0 + 200.0) + pairs * 24.0 + 7.0 * 3 * npos * 4.0 * rhs;
    return (size_t)(grid + tabs + part);
}

static int serve_error(ServeState *sv, int st, const std::string &msg)
{
    std::lock_guard<std::mutex> g(sv->mu);
    sv->last_error = msg;
    return st;
}

int serve_create(ServeState *sv, int device, size_t budget, int lanes, int max_npos, int max_iters, int max_nrhs,
                 double tol)
{
    if (lanes <= 0 || max_npos <= 0 || max_iters <= 0 || max_nrhs <= 0 || !(tol > 0.0))
        return serve_error(sv, kErrInvalid, "bad server arguments");
    sv->device = device;
    sv->budget = budget;
    sv->max_npos = max_npos;
    sv->max_nrhs = max_nrhs;
    sv->max_iters = max_iters;
    sv->tol = tol;
    const char *env = std::getenv("STOKESDT_SERVE_BATCH");
    sv->batching = !(env && env[0] == '0');
    sv->batch_all = sv->batching && env && std::string(env) == "all";
    if (cudaSetDevice(device) != cudaSuccess) return serve_error(sv, kErrCuda, "cudaSetDevice failed");
    if (sv->batching) {
        if (sv->batch_all) lanes = 1;  // the worker only serves what the batch lanes cannot take
        sv->blanes.resize(2);
        for (ServeBatchLane &bl : sv->blanes)
            if (cudaStreamCreateWithFlags(&bl.stream, cudaStreamNonBlocking) != cudaSuccess)
                return serve_error(sv, kErrCuda, "stream creation failed");
    }
    sv->workers.resize(lanes);
    for (int l = 0; l < lanes; l++) {
        ServeWorker &w = sv->workers[l];
        if (cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess)
            return serve_error(sv, kErrCuda, "stream creation failed");
        w.lz = new LanczosState;
        w.lz->device = device;
        w.lz->stream = w.stream;
        w.lz->dim = 3 * max_npos;
        w.lz->max_iters = max_iters;
        w.lz->max_nrhs = max_nrhs;
        w.lz->tol = tol;
        w.lz->reorth = true;
        const int st = lanczos_alloc(w.lz);
        if (st != kOk) return serve_error(sv, st, "Lanczos workspace: " + w.lz->last_error);
        if (cudaMalloc(&w.d_in, (size_t)max_nrhs * 3 * max_npos * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&w.d_out, (size_t)max_nrhs * 3 * max_npos * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            return serve_error(sv, kErrAlloc, "request staging allocation failed");
        }
    }
    for (int l = 0; l < lanes; l++) sv->workers[l].th = std::thread(serve_worker_loop, sv, l);
    for (size_t l = 0; l < sv->blanes.size(); l++) sv->blanes[l].th = std::thread(serve_batch_loop, sv, (int)l);
    return kOk;
}

// Whether request r may go to a batch lane (caller holds the lock).
static bool batchable(const ServeState *sv, const ServeRequest &r)
{
    return sv->batching && sv->systems[r.sys]->packable && r.nrhs <= std::min(sv->max_nrhs, kBlMaxK) &&
           (sv->pk_dirty || sv->rebuilding || sv->lanes_active > 0);
}

// Whether another waiting request could share a batch with r: same kind and
// RHS count, batchable, on another idle system (caller holds the lock).
static bool has_partner(const ServeState *sv, const ServeRequest &r)
{
    for (const ServeRequest &o : sv->queue)
        if (o.id != r.id && o.sys != r.sys && o.kind == r.kind && o.nrhs == r.nrhs &&
            !sv->systems[o.sys]->busy && batchable(sv, o))
            return true;
    return false;
}

int serve_register(ServeState *sv, int npos, const double *rdi, double box, int K, double xi, double rmax,
                   int porder, const double *pos, int *sys_id)
{
    if (npos <= 0 || npos > sv->max_npos || !rdi || !pos || !sys_id)
        return serve_error(sv, kErrInvalid, "bad system (npos must be in [1, max_npos])");
    const size_t need = serve_system_bytes(npos, box, K, rmax, sv->max_nrhs);
    {
        std::lock_guard<std::mutex> g(sv->mu);
        if (sv->used + need > sv->budget) {
            sv->last_error = "HBM budget exceeded: system not admitted";
            sv->rejected++;
            return kErrAlloc;
        }
        sv->used += need;
    }
    ServeSystem *s = new ServeSystem;
    s->bytes = need;
    SpmeEngine *e = &s->eng;
    e->device = sv->device;
    e->npos = npos;
    e->box = box;
    e->xi = xi;
    e->rmax = rmax;
    e->K = K;
    e->p = porder;
    bool mono = true;
    for (int i = 0; i < npos; i++) mono = mono && rdi[i] == 1.0;
    e->mono = mono;
    cudaSetDevice(sv->device);
    int st = spme_create(e);
    e->tc_enabled = false;  // the admission estimate holds no tensor-core operand tiles
    if (st == kOk) st = spme_set_radii(e, rdi);
    if (st == kOk && cudaMalloc(&s->d_pos, (size_t)3 * npos * sizeof(double)) != cudaSuccess) st = kErrAlloc;
    if (st == kOk &&
        cudaMemcpyAsync(s->d_pos, pos, (size_t)3 * npos * sizeof(double), cudaMemcpyHostToDevice, e->stream) !=
            cudaSuccess)
        st = kErrCuda;
    if (st == kOk) st = spme_update(e, s->d_pos);
    // the grid work space for max_nrhs vectors now (the admission estimate
    // counts it): a first request must not allocate, which would also stall
    // the other lanes' streams
    if (st == kOk) st = spme_reserve(e, std::min(sv->max_nrhs, e->rhs_chunk_max));
    if (st == kOk && cudaStreamSynchronize(e->stream) != cudaSuccess) st = kErrCuda;
    if (st == kOk && (cudaMalloc(&s->d_in, (size_t)sv->max_nrhs * 3 * npos * sizeof(double)) != cudaSuccess ||
                      cudaMalloc(&s->d_out, (size_t)sv->max_nrhs * 3 * npos * sizeof(double)) != cudaSuccess)) {
        cudaGetLastError();
        st = kErrAlloc;
    }
    if (st != kOk) {
        const std::string msg = e->last_error;
        cudaFree(s->d_in);
        cudaFree(s->d_out);
        cudaFree(s->d_pos);
        spme_free(e);
        delete s;
        std::lock_guard<std::mutex> g(sv->mu);
        sv->used -= need;
        sv->last_error = "system set-up failed: " + msg;
        return st;
    }
    // the engine runs on whichever worker takes its request
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    e->own_stream = false;
    e->stream = nullptr;
    s->packable = sv->batching && e->mono && e->K <= 256 && e->tma_enabled && e->tma_tabs && e->zfused;
    std::lock_guard<std::mutex> g(sv->mu);
    sv->systems.push_back(s);
    *sys_id = (int)sv->systems.size() - 1;
    // the batch lanes rebuild their packed state before their next batch
    if (s->packable) sv->pk_dirty = true;
    return kOk;
}

// Rebuilds every batch lane's packed product state and batched Lanczos
// workspace over the packable systems (no lane busy; lock not held).  Lanes
// whose workspace does not fit the HBM budget stay idle.
static int rebuild_lanes(ServeState *sv)
{
    cudaSetDevice(sv->device);
    std::vector<int> ids;
    std::vector<SpmeEngine *> eng;
    std::vector<int> npos;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        for (size_t i = 0; i < sv->systems.size(); i++)
            if (sv->systems[i]->packable) {
                sv->systems[i]->pk = (int)ids.size();
                ids.push_back((int)i);
                eng.push_back(&sv->systems[i]->eng);
                npos.push_back(sv->systems[i]->eng.npos);
            }
        sv->pk_sys = ids;
        sv->used -= sv->lane_bytes;
        sv->lane_bytes = 0;
    }
    int active = 0;
    const int rhs = std::min(sv->max_nrhs, kBlMaxK);
    // estimated bytes of one lane: class grids, FP32 work, Krylov bases
    size_t per_lane = 0;
    for (SpmeEngine *e : eng) {
        const size_t n3 = 3 * (size_t)e->npos, ld = (n3 + 31) / 32 * 32;
        per_lane += (size_t)rhs * 3 * e->K * e->K * e->XS * sizeof(float2) + (size_t)e->K * e->K * e->XS * 4 +
                    (size_t)e->npos * rhs * 13 * 4 + (size_t)(sv->max_iters + 1) * rhs * ld * 8;
    }
    int st = kOk;
    for (size_t l = 0; l < sv->blanes.size(); l++) {
        ServeBatchLane &bl = sv->blanes[l];
        if (bl.bl) {
            bl_free(bl.bl);
            delete bl.bl;
            bl.bl = nullptr;
        }
        if (bl.pk) {
            packed_free(bl.pk);
            delete bl.pk;
            bl.pk = nullptr;
        }
        if (eng.empty()) continue;
        {
            std::lock_guard<std::mutex> g(sv->mu);
            if (sv->used + per_lane > sv->budget) continue;
            sv->used += per_lane;
            sv->lane_bytes += per_lane;
        }
        bl.pk = new PackedBatch;
        st = packed_create(bl.pk, eng, rhs, sv->device, bl.stream);
        if (st == kOk) st = packed_refresh(bl.pk);
        if (st != kOk) {
            std::lock_guard<std::mutex> g(sv->mu);
            sv->lanes_active = 0;
            sv->last_error = "batch lane set-up: " + bl.pk->last_error;
            return st;
        }
        bl.bl = new BLState;
        st = bl_create(bl.bl, npos, sv->max_iters, rhs, sv->tol, sv->device, bl.stream);
        if (st != kOk) {
            std::lock_guard<std::mutex> g(sv->mu);
            sv->lanes_active = 0;
            sv->last_error = "batch lane Lanczos set-up: " + bl.bl->last_error;
            return st;
        }
        active++;
    }
    std::lock_guard<std::mutex> g(sv->mu);
    sv->lanes_active = active;
    return kOk;
}

int serve_submit(ServeState *sv, int sys_id, int kind, int nrhs, const double *in, double *out, long long *ticket)
{
    if (!in || !out || !ticket || nrhs <= 0 || nrhs > sv->max_nrhs || (kind != 0 && kind != 1))
        return serve_error(sv, kErrInvalid, "bad request");
    std::lock_guard<std::mutex> g(sv->mu);
    if (sys_id < 0 || sys_id >= (int)sv->systems.size() || !sv->systems[sys_id]) {
        sv->last_error = "unknown system";
        return kErrInvalid;
    }
    ServeRequest r;
    r.id = sv->next_ticket++;
    r.sys = sys_id;
    r.kind = kind;
    r.nrhs = nrhs;
    r.in = in;
    r.out = out;
    r.t_submit = now_ms();
    sv->queue.push_back(r);
    sv->status[r.id] = kPending;
    *ticket = r.id;
    sv->cv.notify_all();
    return kOk;
}

// Next request for the per-request workers whose system is idle, in arrival
// order: one the batch lanes cannot take, a batchable one without a
// partner, or any while no batch lane is free (locked by the caller).
static bool take_request(ServeState *sv, ServeRequest &r)
{
    bool lane_free = false;  // (the lanes' states are rebuilt without the lock)
    if (!sv->rebuilding)
        for (const ServeBatchLane &bl : sv->blanes) lane_free = lane_free || (bl.pk && !bl.busy);
    for (auto it = sv->queue.begin(); it != sv->queue.end(); ++it) {
        if (!sv->systems[it->sys]->busy &&
            (!batchable(sv, *it) ||
             (!sv->batch_all && (!lane_free || sv->rebuilding || !has_partner(sv, *it))))) {
            r = *it;
            sv->queue.erase(it);
            sv->systems[r.sys]->busy = true;
            sv->workers_busy++;
            return true;
        }
    }
    return false;
}

void serve_worker_loop(ServeState *sv, int lane)
{
    ServeWorker &w = sv->workers[lane];
    cudaSetDevice(sv->device);
    for (;;) {
        ServeRequest r;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv.wait(lk, [&] { return sv->stopping || take_request(sv, r); });
            if (sv->stopping && r.id < 0) return;
        }
        sv->cv.notify_all();  // a batch lane may take lone requests now that this worker is busy
        ServeSystem *s = sv->systems[r.sys];
        SpmeEngine *e = &s->eng;
        const int n3 = 3 * e->npos;
        const size_t bytes = (size_t)r.nrhs * n3 * sizeof(double);
        e->stream = w.stream;
        int st = kOk;
        if (cudaMemcpyAsync(w.d_in, r.in, bytes, cudaMemcpyHostToDevice, w.stream) != cudaSuccess) st = kErrCuda;
        if (st == kOk) {
            if (r.kind == 0) {
                st = spme_mulvec(e, 0, r.nrhs, 1.0, n3, w.d_in, 0.0, n3, w.d_out);
            } else {
                w.lz->dim = n3;
                std::vector<int> it((r.nrhs + w.lz->max_nrhs - 1) / w.lz->max_nrhs + 1, 0);
                st = lanczos_compute(w.lz, e, r.nrhs, n3, w.d_in, n3, w.d_out, it.data());
                if (st == kErrNotConverged) st = kOk;  // logged by the reference, result kept
            }
        }
        if (st == kOk && (cudaMemcpyAsync(r.out, w.d_out, bytes, cudaMemcpyDeviceToHost, w.stream) != cudaSuccess ||
                          cudaStreamSynchronize(w.stream) != cudaSuccess))
            st = kErrCuda;
        if (st == kOk) st = spme_check_device_error(e);
        e->stream = nullptr;
        const double t_done = now_ms();
        {
            std::lock_guard<std::mutex> g(sv->mu);
            s->busy = false;
            sv->workers_busy--;
            sv->status[r.id] = st == kOk ? kOk : st;
            sv->latency_ms[r.id] = t_done - r.t_submit;
            sv->completed++;
            if (st != kOk) sv->last_error = "request failed: " + e->last_error;
        }
        sv->cv.notify_all();
    }
}

// The request a batch lane starts its next batch with: the oldest batchable
// request on an idle system that has a partner, or, when every worker is
// busy, the oldest batchable request on an idle system (locked by the
// caller); queue end if none.
static std::deque<ServeRequest>::iterator batch_head(ServeState *sv)
{
    const bool workers_full = sv->batch_all || sv->workers_busy >= (int)sv->workers.size();
    auto lone = sv->queue.end();
    for (auto it = sv->queue.begin(); it != sv->queue.end(); ++it) {
        const ServeSystem *s = sv->systems[it->sys];
        if (s->busy || s->pk < 0 || !batchable(sv, *it)) continue;
        if (has_partner(sv, *it)) return it;
        if (workers_full && lone == sv->queue.end()) lone = it;
    }
    return lone;
}

// The batch head and every later request of its kind and RHS count on
// another idle system, up to max_batch (locked by the caller); their systems
// are marked busy.
static void take_batch(ServeState *sv, std::vector<ServeRequest> &batch)
{
    batch.clear();
    auto head = batch_head(sv);
    if (head == sv->queue.end()) return;
    const int kind = head->kind, nrhs = head->nrhs;
    for (auto it = head; it != sv->queue.end() && (int)batch.size() < sv->max_batch;) {
        ServeSystem *s = sv->systems[it->sys];
        if (!s->busy && s->pk >= 0 && batchable(sv, *it) && it->kind == kind && it->nrhs == nrhs) {
            s->busy = true;
            batch.push_back(*it);
            it = sv->queue.erase(it);
        } else {
            ++it;
        }
    }
}

static bool has_batch_work(ServeState *sv) { return batch_head(sv) != sv->queue.end(); }

// One batch on lane `lane`: copy the inputs in, one packed product or one
// lockstep block Lanczos over the batch's systems, copy the outputs out.
static int run_batch(ServeState *sv, ServeBatchLane &bl, const std::vector<ServeRequest> &batch)
{
    const int nb = (int)batch.size(), kind = batch[0].kind, k = batch[0].nrhs;
    std::vector<int> act(nb), ld(nb), it(nb, 0);
    std::vector<const double *> f(nb);
    std::vector<double *> v(nb);
    for (int j = 0; j < nb; j++) {
        ServeSystem *s = sv->systems[batch[j].sys];
        const size_t n3 = 3 * (size_t)s->eng.npos;
        if (cudaMemcpyAsync(s->d_in, batch[j].in, (size_t)k * n3 * sizeof(double), cudaMemcpyHostToDevice,
                            bl.stream) != cudaSuccess)
            return kErrCuda;
        act[j] = s->pk;
        ld[j] = (int)n3;
        f[j] = s->d_in;
        v[j] = s->d_out;
    }
    int st;
    if (kind == 0) {
        st = packed_mulvec(bl.pk, nb, act.data(), k, 1.0, f.data(), ld.data(), 0.0, v.data(), ld.data());
        if (st != kOk) serve_error(sv, st, "batched product: " + bl.pk->last_error);
    } else {
        st = bl_compute(bl.bl, bl.pk, act, k, f.data(), ld.data(), v.data(), ld.data(), it.data());
        if (st == kErrNotConverged) st = kOk;  // logged by the reference, result kept
        if (st != kOk) serve_error(sv, st, "batched Lanczos: " + bl.bl->last_error);
    }
    if (st != kOk) return st;
    for (int j = 0; j < nb; j++) {
        ServeSystem *s = sv->systems[batch[j].sys];
        const size_t n3 = 3 * (size_t)s->eng.npos;
        if (cudaMemcpyAsync(batch[j].out, s->d_out, (size_t)k * n3 * sizeof(double), cudaMemcpyDeviceToHost,
                            bl.stream) != cudaSuccess)
            return kErrCuda;
    }
    if (cudaStreamSynchronize(bl.stream) != cudaSuccess) return kErrCuda;
    st = packed_check_error(bl.pk);
    if (st != kOk) serve_error(sv, st, bl.pk->last_error);
    return st;
}

void serve_batch_loop(ServeState *sv, int lane)
{
    ServeBatchLane &bl = sv->blanes[lane];
    cudaSetDevice(sv->device);
    std::vector<ServeRequest> batch;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv.wait(lk, [&] {
                return sv->stopping || (!sv->rebuilding && (sv->pk_dirty || (bl.pk && has_batch_work(sv))));
            });
            if (sv->stopping) return;
            if (sv->pk_dirty) {
                bool others_busy = false;
                for (const ServeBatchLane &o : sv->blanes) others_busy = others_busy || o.busy;
                if (others_busy) {
                    sv->cv.wait(lk, [&] {
                        bool b = false;
                        for (const ServeBatchLane &o : sv->blanes) b = b || o.busy;
                        return sv->stopping || !b;
                    });
                    continue;
                }
                // a registration during the rebuild sets pk_dirty again
                sv->rebuilding = true;
                sv->pk_dirty = false;
                lk.unlock();
                const int st = rebuild_lanes(sv);
                lk.lock();
                sv->rebuilding = false;
                if (st != kOk || sv->lanes_active == 0) {
                    // no lane could be set up: the workers take everything
                    for (ServeSystem *s : sv->systems) s->packable = false;
                }
                sv->cv.notify_all();
                continue;
            }
            if (!bl.pk) continue;  // this lane's workspace did not fit the budget
            take_batch(sv, batch);
            if (batch.empty()) continue;
            bl.busy = true;
        }
        sv->cv.notify_all();  // workers may take partnered requests while no lane is free
        const int st = run_batch(sv, bl, batch);
        const double t_done = now_ms();
        {
            std::lock_guard<std::mutex> g(sv->mu);
            bl.busy = false;
            sv->batches++;
            sv->batched_requests += (long long)batch.size();
            for (const ServeRequest &r : batch) {
                sv->systems[r.sys]->busy = false;
                sv->status[r.id] = st;
                sv->latency_ms[r.id] = t_done - r.t_submit;
                sv->completed++;
            }
        }
        sv->cv.notify_all();
    }
}

int serve_wait(ServeState *sv, long long ticket, double timeout_ms, double *latency_ms)
{
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->status.find(ticket);
    if (it == sv->status.end()) return kErrInvalid;
    const bool done = sv->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), [&] {
        return sv->status[ticket] != kPending;
    });
    if (!done) return kErrState;  // still queued or running
    const int st = sv->status[ticket];
    if (latency_ms) *latency_ms = sv->latency_ms[ticket];
    sv->status.erase(ticket);
    sv->latency_ms.erase(ticket);
    return st;
}

void serve_free(ServeState *sv)
{
    {
        std::lock_guard<std::mutex> g(sv->mu);
        sv->stopping = true;
    }
    sv->cv.notify_all();
    for (ServeWorker &w : sv->workers)
        if (w.th.joinable()) w.th.join();
    for (ServeBatchLane &bl : sv->blanes)
        if (bl.th.joinable()) bl.th.join();
    cudaSetDevice(sv->device);
    for (ServeBatchLane &bl : sv->blanes) {
        if (bl.bl) {
            bl_free(bl.bl);
            delete bl.bl;
        }
        if (bl.pk) {
            packed_free(bl.pk);
            delete bl.pk;
        }
        if (bl.stream) cudaStreamDestroy(bl.stream);
    }
    sv->blanes.clear();
    for (ServeWorker &w : sv->workers) {
        if (w.stream) cudaStreamSynchronize(w.stream);
        if (w.lz) {
            w.lz->stream = nullptr;
            lanczos_free(w.lz);
            delete w.lz;
        }
        cudaFree(w.d_in);
        cudaFree(w.d_out);
        if (w.stream) cudaStreamDestroy(w.stream);
    }
    sv->workers.clear();
    for (ServeSystem *s : sv->systems) {
        if (!s) continue;
        s->eng.stream = nullptr;
        spme_free(&s->eng);
        cudaFree(s->d_pos);
        cudaFree(s->d_in);
        cudaFree(s->d_out);
        delete s;
    }
    sv->systems.clear();
}

}  // namespace sdt
