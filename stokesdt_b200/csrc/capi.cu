// C ABI (include/stokesdt_b200.h): handles, argument checks, host<->device
// staging.  The compute entry points are in spme.cu, real_space.cu and
// lanczos.cu; nothing here falls back to a CPU path.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/stokesdt_b200.h"
#include "handles.h"

namespace {

// Records msg as the engine's last error (any engine with a last_error).
template <typename Engine>
int fail(Engine *e, int st, const std::string &msg)
{
    e->last_error = msg;
    return st;
}

#define CAPI_CUDA(eng, call)                                                              \
    do {                                                                                  \
        cudaError_t err_ = (call);                                                        \
        if (err_ != cudaSuccess)                                                          \
            return fail(eng, SDT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

int ensure_host_staging(sdt::SpmeEngine *e, int nrhs)
{
    if (nrhs <= e->host_cap) return SDT_OK;
    cudaFree(e->d_fin);
    cudaFree(e->d_vout);
    e->d_fin = e->d_vout = nullptr;
    e->host_cap = 0;
    const size_t bytes = (size_t)nrhs * 3 * e->npos * sizeof(double);
    if (cudaMalloc(&e->d_fin, bytes) != cudaSuccess || cudaMalloc(&e->d_vout, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(e, SDT_ERR_ALLOC, "device allocation of host staging buffers failed");
    }
    e->host_cap = nrhs;
    return SDT_OK;
}

}  // namespace

extern "C" {

int sdt_batch_create(int nsys, const int *npos, const double *rdi, const double *box, const int *dim,
                     const double *xi, const double *rmax, int porder, int max_iters, int max_nrhs,
                     double tol, int reorth, int lanes, int device, sdt_batch **out)
{
    if (!out) return SDT_ERR_INVALID;
    *out = nullptr;
    sdt_batch *h = new (std::nothrow) sdt_batch;
    if (!h) return SDT_ERR_ALLOC;
    h->b.reorth = reorth != 0;
    const int st = sdt::batch_create(&h->b, nsys, npos, rdi, box, dim, xi, rmax, porder, max_iters,
                                     max_nrhs, tol, lanes, device);
    if (st != SDT_OK) {
        sdt::batch_free(&h->b);
        delete h;
        return st;
    }
    *out = h;
    return SDT_OK;
}

int sdt_batch_update_device(sdt_batch *h, const double *d_pos)
{
    if (!h || !d_pos) return SDT_ERR_INVALID;
    return sdt::batch_update(&h->b, d_pos);
}

int sdt_batch_mulvec_device(sdt_batch *h, int nrhs, double alpha, const double *d_f, double beta,
                            double *d_v)
{
    if (!h || !d_f || !d_v || nrhs < 0) return SDT_ERR_INVALID;
    if (nrhs == 0) return SDT_OK;
    return sdt::batch_mulvec(&h->b, nrhs, alpha, d_f, beta, d_v);
}

int sdt_batch_lanczos_device(sdt_batch *h, int nrhs, const double *d_z, double *d_y, int *iters)
{
    if (!h || !d_z || !d_y || nrhs <= 0) return SDT_ERR_INVALID;
    return sdt::batch_lanczos(&h->b, nrhs, d_z, d_y, iters);
}

namespace {
// device staging of `count` doubles for the host-pointer batch calls
double *batch_stage(sdt::BatchState *b, size_t count)
{
    if (count > b->stage_cap) {
        cudaFree(b->d_stage);
        b->d_stage = nullptr;
        b->stage_cap = 0;
        if (cudaMalloc(&b->d_stage, count * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        b->stage_cap = count;
    }
    return b->d_stage;
}
}  // namespace

int sdt_batch_update(sdt_batch *h, const double *pos)
{
    if (!h || !pos) return SDT_ERR_INVALID;
    sdt::BatchState *b = &h->b;
    const size_t n = (size_t)b->pos_off[b->nsys];
    if (cudaSetDevice(b->device) != cudaSuccess) return SDT_ERR_CUDA;
    double *d = batch_stage(b, n);
    if (!d) return SDT_ERR_ALLOC;
    if (cudaMemcpy(d, pos, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return SDT_ERR_CUDA;
    int st = sdt::batch_update(b, d);
    if (st == SDT_OK) st = sdt::batch_synchronize(b);
    return st;
}

int sdt_batch_mulvec(sdt_batch *h, int nrhs, double alpha, const double *f, double beta, double *v)
{
    if (!h || !f || !v || nrhs < 0) return SDT_ERR_INVALID;
    if (nrhs == 0) return SDT_OK;
    sdt::BatchState *b = &h->b;
    const size_t n = (size_t)nrhs * b->pos_off[b->nsys];
    if (cudaSetDevice(b->device) != cudaSuccess) return SDT_ERR_CUDA;
    double *d = batch_stage(b, 2 * n);
    if (!d) return SDT_ERR_ALLOC;
    if (cudaMemcpy(d, f, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        (beta != 0.0 && cudaMemcpy(d + n, v, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess))
        return SDT_ERR_CUDA;
    int st = sdt::batch_mulvec(b, nrhs, alpha, d, beta, d + n);
    if (st == SDT_OK) st = sdt::batch_synchronize(b);
    if (st == SDT_OK && cudaMemcpy(v, d + n, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = SDT_ERR_CUDA;
    return st;
}

int sdt_batch_lanczos(sdt_batch *h, int nrhs, const double *z, double *y, int *iters)
{
    if (!h || !z || !y || nrhs <= 0) return SDT_ERR_INVALID;
    sdt::BatchState *b = &h->b;
    const size_t n = (size_t)nrhs * b->pos_off[b->nsys];
    if (cudaSetDevice(b->device) != cudaSuccess) return SDT_ERR_CUDA;
    double *d = batch_stage(b, 2 * n);
    if (!d) return SDT_ERR_ALLOC;
    if (cudaMemcpy(d, z, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return SDT_ERR_CUDA;
    int st = sdt::batch_lanczos(b, nrhs, d, d + n, iters);
    if (st == SDT_OK || st == SDT_ERR_NOT_CONVERGED) {
        const int st2 = sdt::batch_synchronize(b);
        if (st2 != SDT_OK) return st2;
        if (cudaMemcpy(y, d + n, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return SDT_ERR_CUDA;
    }
    return st;
}

int sdt_batch_info(const sdt_batch *h, long long *total3n, int *lanes)
{
    if (!h) return SDT_ERR_INVALID;
    if (total3n) *total3n = h->b.pos_off.empty() ? 0 : h->b.pos_off[h->b.nsys];
    if (lanes) *lanes = (int)h->b.lanes.size();
    return SDT_OK;
}

int sdt_batch_set_packed(sdt_batch *h, int enable)
{
    if (!h) return SDT_ERR_INVALID;
    return sdt::batch_set_packed(&h->b, enable != 0);
}

int sdt_batch_get_packed(const sdt_batch *h)
{
    if (!h) return SDT_ERR_INVALID;
    return h->b.packed ? 1 : 0;
}

int sdt_batch_synchronize(sdt_batch *h)
{
    if (!h) return SDT_ERR_INVALID;
    return sdt::batch_synchronize(&h->b);
}

const char *sdt_batch_last_error(const sdt_batch *h) { return h ? h->b.last_error.c_str() : ""; }

void sdt_batch_destroy(sdt_batch *h)
{
    if (!h) return;
    sdt::batch_free(&h->b);
    delete h;
}

int sdt_serve_create(int device, double hbm_budget_bytes, int lanes, int max_npos, int max_iters,
                     int max_nrhs, double tol, sdt_serve **out)
{
    if (!out || !(hbm_budget_bytes > 0.0)) return SDT_ERR_INVALID;
    *out = nullptr;
    sdt_serve *h = new (std::nothrow) sdt_serve;
    if (!h) return SDT_ERR_ALLOC;
    const int st = sdt::serve_create(&h->s, device, (size_t)hbm_budget_bytes, lanes, max_npos, max_iters,
                                     max_nrhs, tol);
    if (st != SDT_OK) {
        sdt::serve_free(&h->s);
        delete h;
        return st;
    }
    *out = h;
    return SDT_OK;
}

int sdt_serve_register(sdt_serve *h, int npos, const double *rdi, double box, int dim, double xi,
                       double rmax, int porder, const double *pos, int *sys_id)
{
    if (!h) return SDT_ERR_INVALID;
    return sdt::serve_register(&h->s, npos, rdi, box, dim, xi, rmax, porder, pos, sys_id);
}

int sdt_serve_submit(sdt_serve *h, int sys_id, int kind, int nrhs, const double *in, double *out,
                     long long *ticket)
{
    if (!h) return SDT_ERR_INVALID;
    return sdt::serve_submit(&h->s, sys_id, kind, nrhs, in, out, ticket);
}

int sdt_serve_wait(sdt_serve *h, long long ticket, double timeout_ms, double *latency_ms)
{
    if (!h) return SDT_ERR_INVALID;
    return sdt::serve_wait(&h->s, ticket, timeout_ms, latency_ms);
}

int sdt_serve_stats(sdt_serve *h, long long *completed, long long *rejected, double *used_bytes)
{
    if (!h) return SDT_ERR_INVALID;
    std::lock_guard<std::mutex> g(h->s.mu);
    if (completed) *completed = h->s.completed;
    if (rejected) *rejected = h->s.rejected;
    if (used_bytes) *used_bytes = (double)h->s.used;
    return SDT_OK;
}

int sdt_serve_batch_stats(sdt_serve *h, long long *batches, long long *batched_requests, int *lanes_active)
{
    if (!h) return SDT_ERR_INVALID;
    std::lock_guard<std::mutex> g(h->s.mu);
    if (batches) *batches = h->s.batches;
    if (batched_requests) *batched_requests = h->s.batched_requests;
    if (lanes_active) *lanes_active = h->s.lanes_active;
    return SDT_OK;
}

const char *sdt_serve_last_error(sdt_serve *h)
{
    if (!h) return "";
    std::lock_guard<std::mutex> g(h->s.mu);
    thread_local std::string copy;
    copy = h->s.last_error;
    return copy.c_str();
}

void sdt_serve_destroy(sdt_serve *h)
{
    if (!h) return;
    sdt::serve_free(&h->s);
    delete h;
}

int sdt_steric_create(int npos, const double *rdi, double box_size, double r0, double k0, int device,
                      sdt_steric **out)
{
    if (!out) return SDT_ERR_INVALID;
    *out = nullptr;
    sdt_steric *h = new (std::nothrow) sdt_steric;
    if (!h) return SDT_ERR_ALLOC;
    h->e.npos = npos;
    h->e.box = box_size;
    h->e.r0 = r0;
    h->e.k0 = k0;
    h->e.device = device;
    const int st = sdt::steric_create(&h->e, rdi);
    if (st != SDT_OK) {
        sdt::steric_free(&h->e);
        delete h;
        return st;
    }
    *out = h;
    return SDT_OK;
}

int sdt_steric_accumulate_device(sdt_steric *h, const double *d_pos, double *d_f)
{
    if (!h) return SDT_ERR_INVALID;
    if (!d_pos || !d_f) {
        h->e.last_error = "null pointer";
        return SDT_ERR_INVALID;
    }
    if (cudaSetDevice(h->e.device) != cudaSuccess) {
        h->e.last_error = "cudaSetDevice failed";
        return SDT_ERR_CUDA;
    }
    return sdt::steric_accumulate(&h->e, d_pos, d_f);
}

int sdt_steric_accumulate(sdt_steric *h, const double *pos, double *f)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::StericEngine *e = &h->e;
    if (!pos || !f) {
        e->last_error = "null pointer";
        return SDT_ERR_INVALID;
    }
    const size_t bytes = (size_t)3 * e->npos * sizeof(double);
    cudaError_t err = cudaSetDevice(e->device);
    if (err == cudaSuccess && !e->d_hpos) err = cudaMalloc(&e->d_hpos, bytes);
    if (err == cudaSuccess && !e->d_hf) err = cudaMalloc(&e->d_hf, bytes);
    if (err == cudaSuccess) err = cudaMemcpyAsync(e->d_hpos, pos, bytes, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(e->d_hf, f, bytes, cudaMemcpyHostToDevice, e->stream);
    if (err != cudaSuccess) {
        cudaGetLastError();
        e->last_error = std::string("steric staging: ") + cudaGetErrorString(err);
        return SDT_ERR_CUDA;
    }
    const int st = sdt::steric_accumulate(e, e->d_hpos, e->d_hf);
    if (st != SDT_OK) return st;
    err = cudaMemcpyAsync(f, e->d_hf, bytes, cudaMemcpyDeviceToHost, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) {
        e->last_error = std::string("steric result: ") + cudaGetErrorString(err);
        return SDT_ERR_CUDA;
    }
    return SDT_OK;
}

int sdt_steric_set_stream(sdt_steric *h, void *stream)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::StericEngine *e = &h->e;
    if (cudaSetDevice(e->device) != cudaSuccess) return SDT_ERR_CUDA;
    if (e->own_stream && e->stream) {
        cudaStreamSynchronize(e->stream);
        cudaStreamDestroy(e->stream);
        e->own_stream = false;
        e->stream = nullptr;
    }
    if (stream) {
        e->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) return SDT_ERR_CUDA;
        e->own_stream = true;
    }
    return SDT_OK;
}

const char *sdt_steric_last_error(const sdt_steric *h) { return h ? h->e.last_error.c_str() : ""; }

void sdt_steric_destroy(sdt_steric *h)
{
    if (!h) return;
    sdt::steric_free(&h->e);
    delete h;
}

int sdt_bd_create(sdt_spme *mob, sdt_lanczos *brwn, sdt_steric *steric, double dt, int mob_interval,
                  unsigned long long seed, sdt_bd **out)
{
    if (!out) return SDT_ERR_INVALID;
    *out = nullptr;
    sdt_bd *h = new (std::nothrow) sdt_bd;
    if (!h) return SDT_ERR_ALLOC;
    h->s.mob = mob ? &mob->e : nullptr;
    h->s.lz = brwn ? &brwn->s : nullptr;
    h->s.steric = steric ? &steric->e : nullptr;
    h->s.dt = dt;
    h->s.interval = mob_interval;
    h->s.seed = seed;
    const int st = sdt::bd_create(&h->s);
    if (st != SDT_OK) {
        sdt::bd_free(&h->s);
        delete h;
        return st;
    }
    *out = h;
    return SDT_OK;
}

int sdt_bd_create_ewald(sdt_ewald *mob, sdt_lanczos *brwn, sdt_steric *steric, double dt, int mob_interval,
                        unsigned long long seed, sdt_bd **out)
{
    if (!out) return SDT_ERR_INVALID;
    *out = nullptr;
    sdt_bd *h = new (std::nothrow) sdt_bd;
    if (!h) return SDT_ERR_ALLOC;
    h->s.ew = mob ? &mob->e : nullptr;
    h->s.lz = brwn ? &brwn->s : nullptr;
    h->s.steric = steric ? &steric->e : nullptr;
    h->s.dt = dt;
    h->s.interval = mob_interval;
    h->s.seed = seed;
    const int st = sdt::bd_create(&h->s);
    if (st != SDT_OK) {
        sdt::bd_free(&h->s);
        delete h;
        return st;
    }
    *out = h;
    return SDT_OK;
}

int sdt_bd_set_positions(sdt_bd *h, const double *pos)
{
    if (!h || !pos) return SDT_ERR_INVALID;
    sdt::BdState *b = &h->s;
    if (cudaSetDevice(b->device) != cudaSuccess ||
        cudaMemcpyAsync(b->d_pos, pos, (size_t)3 * b->npos * sizeof(double), cudaMemcpyHostToDevice,
                        b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess) {
        b->last_error = "copying positions to the device failed";
        return SDT_ERR_CUDA;
    }
    return SDT_OK;
}

int sdt_bd_get_positions(sdt_bd *h, double *pos)
{
    if (!h || !pos) return SDT_ERR_INVALID;
    sdt::BdState *b = &h->s;
    if (cudaSetDevice(b->device) != cudaSuccess ||
        cudaMemcpyAsync(pos, b->d_pos, (size_t)3 * b->npos * sizeof(double), cudaMemcpyDeviceToHost,
                        b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess) {
        b->last_error = "copying positions from the device failed";
        return SDT_ERR_CUDA;
    }
    // the dense Ewald kernels have no device error word (no bounded waits)
    return h->s.mob ? sdt::spme_check_device_error(h->s.mob) : SDT_OK;
}

int sdt_bd_set_step(sdt_bd *h, long long istep)
{
    if (!h || istep < 0) return SDT_ERR_INVALID;
    h->s.istep = istep;
    return SDT_OK;
}

int sdt_bd_advance(sdt_bd *h, int nsteps)
{
    if (!h) return SDT_ERR_INVALID;
    return sdt::bd_advance(&h->s, nsteps);
}

int sdt_bd_info(sdt_bd *h, long long *istep, long long *not_converged, int *last_iters)
{
    if (!h) return SDT_ERR_INVALID;
    if (istep) *istep = h->s.istep;
    if (not_converged) *not_converged = h->s.not_converged;
    if (last_iters) *last_iters = h->s.iters.empty() ? 0 : h->s.iters[0];
    return SDT_OK;
}

int sdt_bd_draw_gaussian(sdt_bd *h, long long step, int nvec, int ld, double *z)
{
    if (!h || !z || nvec <= 0 || step < 0) return SDT_ERR_INVALID;
    sdt::BdState *b = &h->s;
    const int n3 = 3 * b->npos;
    if (ld < n3) return SDT_ERR_INVALID;
    const size_t bytes = (size_t)nvec * ld * sizeof(double);
    double *d = nullptr;
    if (cudaSetDevice(b->device) != cudaSuccess || cudaMalloc(&d, bytes) != cudaSuccess) {
        cudaGetLastError();
        b->last_error = "device allocation for the random vectors failed";
        return SDT_ERR_ALLOC;
    }
    int st = sdt::bd_gaussian(b->stream, nvec, n3, ld, b->seed, (unsigned long long)step, d);
    if (st == SDT_OK &&
        (cudaMemcpyAsync(z, d, bytes, cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
         cudaStreamSynchronize(b->stream) != cudaSuccess))
        st = SDT_ERR_CUDA;
    cudaFree(d);
    if (st != SDT_OK) b->last_error = "drawing the random vectors failed";
    return st;
}

int sdt_bd_set_stream(sdt_bd *h, void *stream)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::BdState *b = &h->s;
    if (cudaSetDevice(b->device) != cudaSuccess) return SDT_ERR_CUDA;
    if (b->own_stream && b->stream) {
        cudaStreamSynchronize(b->stream);
        cudaStreamDestroy(b->stream);
        b->own_stream = false;
        b->stream = nullptr;
    }
    if (stream) {
        b->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return SDT_ERR_CUDA;
        b->own_stream = true;
    }
    return SDT_OK;
}

int sdt_bd_synchronize(sdt_bd *h)
{
    if (!h) return SDT_ERR_INVALID;
    if (cudaSetDevice(h->s.device) != cudaSuccess || cudaStreamSynchronize(h->s.stream) != cudaSuccess) {
        h->s.last_error = "synchronize failed";
        return SDT_ERR_CUDA;
    }
    // the dense Ewald kernels have no device error word (no bounded waits)
    return h->s.mob ? sdt::spme_check_device_error(h->s.mob) : SDT_OK;
}

const char *sdt_bd_last_error(const sdt_bd *h) { return h ? h->s.last_error.c_str() : ""; }

void sdt_bd_destroy(sdt_bd *h)
{
    if (!h) return;
    sdt::bd_free(&h->s);
    delete h;
}

const char *sdt_version(void) { return "stokesdt_b200 0.1.0 (sm_100a)"; }

int sdt_spme_create(int npos, const double *rdi, double box_size, double xi, double rmax, int dim,
                    int porder, int device, sdt_spme **out)
{
    if (!out) return SDT_ERR_INVALID;
    *out = nullptr;
    if (npos <= 0 || !rdi) return SDT_ERR_INVALID;
    sdt_spme *h = new (std::nothrow) sdt_spme();
    if (!h) return SDT_ERR_ALLOC;
    sdt::SpmeEngine *e = &h->e;
    e->device = device;
    e->npos = npos;
    e->box = box_size;
    e->xi = xi;
    e->rmax = rmax;
    e->K = dim;
    e->p = porder;
    double amin = rdi[0], amax = rdi[0];
    for (int i = 1; i < npos; i++) {
        amin = std::min(amin, rdi[i]);
        amax = std::max(amax, rdi[i]);
    }
    if (!(amin > 0.0)) {
        delete h;
        return SDT_ERR_INVALID;
    }
    e->mono = (amin == 1.0 && amax == 1.0);
    int st = sdt::spme_create(e);
    if (st == SDT_OK) st = sdt::spme_set_radii(e, rdi);
    if (st != SDT_OK) {
        sdt::spme_free(e);
        delete h;
        return st;
    }
    *out = h;
    return SDT_OK;
}

int sdt_spme_update_device(sdt_spme *h, const double *d_pos)
{
    if (!h || !d_pos) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    CAPI_CUDA(e, cudaSetDevice(e->device));
    return sdt::spme_update(e, d_pos);
}

int sdt_spme_update(sdt_spme *h, const double *pos)
{
    if (!h || !pos) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    CAPI_CUDA(e, cudaSetDevice(e->device));
    int st = ensure_host_staging(e, 1);
    if (st != SDT_OK) return st;
    CAPI_CUDA(e, cudaMemcpyAsync(e->d_fin, pos, (size_t)3 * e->npos * sizeof(double), cudaMemcpyHostToDevice,
                                 e->stream));
    st = sdt::spme_update(e, e->d_fin);
    if (st != SDT_OK) return st;
    CAPI_CUDA(e, cudaStreamSynchronize(e->stream));
    return SDT_OK;
}

int sdt_spme_mulvec_device(sdt_spme *h, int mode, int nrhs, double alpha, int ldf, const double *d_f,
                           double beta, int ldv, double *d_v)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    if (nrhs > 0 && (!d_f || !d_v)) return fail(e, SDT_ERR_INVALID, "null vector pointer");
    CAPI_CUDA(e, cudaSetDevice(e->device));
    return sdt::spme_mulvec(e, mode, nrhs, alpha, ldf, d_f, beta, ldv, d_v);
}

int sdt_spme_mulvec(sdt_spme *h, int mode, int nrhs, double alpha, int ldf, const double *f, double beta,
                    int ldv, double *v)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    if (nrhs < 0) return fail(e, SDT_ERR_INVALID, "nrhs < 0");
    if (nrhs == 0) return SDT_OK;
    if (!f || !v) return fail(e, SDT_ERR_INVALID, "null vector pointer");
    const int n3 = 3 * e->npos;
    if (ldf < n3 || ldv < n3) return fail(e, SDT_ERR_INVALID, "leading dimensions must be >= 3*npos");
    CAPI_CUDA(e, cudaSetDevice(e->device));
    int st = ensure_host_staging(e, nrhs);
    if (st != SDT_OK) return st;
    const size_t row = (size_t)n3 * sizeof(double);
    CAPI_CUDA(e, cudaMemcpy2DAsync(e->d_fin, row, f, (size_t)ldf * sizeof(double), row, nrhs,
                                   cudaMemcpyHostToDevice, e->stream));
    if (beta != 0.0)
        CAPI_CUDA(e, cudaMemcpy2DAsync(e->d_vout, row, v, (size_t)ldv * sizeof(double), row, nrhs,
                                       cudaMemcpyHostToDevice, e->stream));
    st = sdt::spme_mulvec(e, mode, nrhs, alpha, n3, e->d_fin, beta, n3, e->d_vout);
    if (st != SDT_OK) return st;
    CAPI_CUDA(e, cudaMemcpy2DAsync(v, (size_t)ldv * sizeof(double), e->d_vout, row, row, nrhs,
                                   cudaMemcpyDeviceToHost, e->stream));
    CAPI_CUDA(e, cudaStreamSynchronize(e->stream));
    return sdt::spme_check_device_error(e);
}

int sdt_spme_dim(const sdt_spme *h) { return h ? 3 * h->e.npos : 0; }

int sdt_spme_set_stream(sdt_spme *h, void *stream)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    CAPI_CUDA(e, cudaSetDevice(e->device));
    if (e->own_stream && e->stream) {
        CAPI_CUDA(e, cudaStreamSynchronize(e->stream));
        cudaStreamDestroy(e->stream);
        e->own_stream = false;
        e->stream = nullptr;
    }
    if (stream) {
        e->stream = (cudaStream_t)stream;
    } else {
        CAPI_CUDA(e, cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->own_stream = true;
    }
    return SDT_OK;
}

int sdt_spme_set_pairlist(sdt_spme *h, int enable)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    e->pl_enabled = enable != 0;
    if (!e->pl_enabled) e->pl_ready = false;
    return SDT_OK;
}

int sdt_spme_pairlist_size(const sdt_spme *h, long long *pairs)
{
    if (!h || !pairs) return SDT_ERR_INVALID;
    *pairs = h->e.pl_ready ? h->e.pl_pairs : -1;
    return SDT_OK;
}

int sdt_spme_synchronize(sdt_spme *h)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    CAPI_CUDA(e, cudaSetDevice(e->device));
    CAPI_CUDA(e, cudaStreamSynchronize(e->stream));
    return sdt::spme_check_device_error(e);
}

int sdt_spme_profile_mulvec(sdt_spme *h, int nrhs, int reps, double *stage_ms, int max_stages)
{
    if (!h || !stage_ms || max_stages < sdt::kNumStages) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    CAPI_CUDA(e, cudaSetDevice(e->device));
    const int st = sdt::spme_profile(e, nrhs, reps, stage_ms);
    return st == SDT_OK ? sdt::kNumStages : st;
}

int sdt_spme_spectrum_device(sdt_spme *h, int nrhs, int ldf, const double *d_f, float *d_spec)
{
    if (!h || !d_f || !d_spec) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    CAPI_CUDA(e, cudaSetDevice(e->device));
    return sdt::spme_spectrum(e, nrhs, ldf, d_f, d_spec);
}

const char *sdt_profile_stage_name(int stage)
{
    static const char *names[sdt::kNumStages] = {"gather_forces", "real_space", "spread_x", "yfft_fwd",
                                                 "zfft_influence", "yfft_inv", "xinv_interp", "combine"};
    return (stage >= 0 && stage < sdt::kNumStages) ? names[stage] : "";
}

unsigned long long sdt_kernel_launches(void) { return sdt::g_kernel_launches.load(); }

const char *sdt_spme_last_error(const sdt_spme *h) { return h ? h->e.last_error.c_str() : "null handle"; }

void sdt_spme_destroy(sdt_spme *h)
{
    if (!h) return;
    sdt::spme_free(&h->e);
    delete h;
}

int sdt_lanczos_create(int dim, int max_iters, int max_nrhs, double tol, int device, sdt_lanczos **out)
{
    if (!out) return SDT_ERR_INVALID;
    *out = nullptr;
    if (dim <= 0 || max_iters <= 0 || max_nrhs <= 0 || !(tol > 0.0)) return SDT_ERR_INVALID;
    if (max_nrhs > dim / 3) max_nrhs = std::max(1, dim / 3);  // BrwnLanczos::Init clamp
    if (max_nrhs > 32) return SDT_ERR_UNSUPPORTED;
    sdt_lanczos *h = new (std::nothrow) sdt_lanczos();
    if (!h) return SDT_ERR_ALLOC;
    h->s.device = device;
    h->s.dim = dim;
    h->s.max_iters = max_iters;
    h->s.max_nrhs = max_nrhs;
    h->s.tol = tol;
    const int st = sdt::lanczos_alloc(&h->s);
    if (st != SDT_OK) {
        sdt::lanczos_free(&h->s);
        delete h;
        return st;
    }
    *out = h;
    return SDT_OK;
}

int sdt_lanczos_set_stream(sdt_lanczos *h, void *stream)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::LanczosState *lz = &h->s;
    if (cudaSetDevice(lz->device) != cudaSuccess) return SDT_ERR_CUDA;
    if (lz->own_stream && lz->stream) {
        cudaStreamSynchronize(lz->stream);
        cudaStreamDestroy(lz->stream);
        lz->own_stream = false;
        lz->stream = nullptr;
    }
    if (stream) {
        lz->stream = (cudaStream_t)stream;
    } else if (cudaStreamCreateWithFlags(&lz->stream, cudaStreamNonBlocking) == cudaSuccess) {
        lz->own_stream = true;
    } else {
        return SDT_ERR_CUDA;
    }
    return SDT_OK;
}

int sdt_lanczos_set_reorth(sdt_lanczos *h, int enable)
{
    if (!h) return SDT_ERR_INVALID;
    h->s.reorth = enable != 0;
    return SDT_OK;
}

int sdt_lanczos_compute_device(sdt_lanczos *h, sdt_spme *mob, int nrhs, int ldz, const double *d_z, int ldy,
                               double *d_y, int *iters)
{
    if (!h || !mob) return SDT_ERR_INVALID;
    if (cudaSetDevice(h->s.device) != cudaSuccess) return SDT_ERR_CUDA;
    const int st = sdt::lanczos_compute(&h->s, &mob->e, nrhs, ldz, d_z, ldy, d_y, iters);
    if (st != SDT_OK && st != SDT_ERR_NOT_CONVERGED) return st;
    if (cudaStreamSynchronize(h->s.stream) != cudaSuccess) {
        h->s.last_error = "stream synchronize failed";
        return SDT_ERR_CUDA;
    }
    return st;
}

// ---- dense Ewald (MobEwald) ----

int sdt_ewald_create(int npos, const double *rdi, double box_size, double tol, double xi, int device,
                     sdt_ewald **out)
{
    if (!out || !rdi) return SDT_ERR_INVALID;
    *out = nullptr;
    sdt_ewald *h = new (std::nothrow) sdt_ewald;
    if (!h) return SDT_ERR_ALLOC;
    sdt::EwaldEngine *e = &h->e;
    e->device = device;
    e->npos = npos;
    e->box = box_size;
    e->tol = tol;
    e->xi = xi;
    const int st = sdt::ewald_create(e, rdi);
    if (st != SDT_OK) {
        sdt::ewald_free(e);
        delete h;
        return st;
    }
    *out = h;
    return SDT_OK;
}

int sdt_ewald_update_device(sdt_ewald *h, const double *d_pos)
{
    if (!h || !d_pos) return SDT_ERR_INVALID;
    CAPI_CUDA(&h->e, cudaSetDevice(h->e.device));
    return sdt::ewald_update(&h->e, d_pos);
}

int sdt_ewald_update(sdt_ewald *h, const double *pos)
{
    if (!h || !pos) return SDT_ERR_INVALID;
    sdt::EwaldEngine *e = &h->e;
    CAPI_CUDA(e, cudaSetDevice(e->device));
    CAPI_CUDA(e, cudaMemcpyAsync(e->d_pos, pos, (size_t)e->n3 * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    const int st = sdt::ewald_update(e, e->d_pos);
    if (st != SDT_OK) return st;
    CAPI_CUDA(e, cudaStreamSynchronize(e->stream));
    return SDT_OK;
}

int sdt_ewald_mulvec_device(sdt_ewald *h, int nrhs, double alpha, int ldf, const double *d_f, double beta, int ldv,
                            double *d_v)
{
    if (!h || !d_f || !d_v) return SDT_ERR_INVALID;
    CAPI_CUDA(&h->e, cudaSetDevice(h->e.device));
    return sdt::ewald_mulvec(&h->e, nrhs, alpha, ldf, d_f, beta, ldv, d_v);
}

int sdt_ewald_mulvec(sdt_ewald *h, int nrhs, double alpha, int ldf, const double *f, double beta, int ldv, double *v)
{
    if (!h || !f || !v || nrhs < 0) return SDT_ERR_INVALID;
    sdt::EwaldEngine *e = &h->e;
    if (ldf < e->n3 || ldv < e->n3) {
        e->last_error = "leading dimensions must be >= 3*npos";
        return SDT_ERR_INVALID;
    }
    if (nrhs == 0) return SDT_OK;
    CAPI_CUDA(e, cudaSetDevice(e->device));
    if (nrhs > e->host_cap) {
        cudaFree(e->d_fin);
        cudaFree(e->d_vout);
        e->d_fin = e->d_vout = nullptr;
        e->host_cap = 0;
        const size_t bytes = (size_t)nrhs * e->n3 * sizeof(double);
        if (cudaMalloc(&e->d_fin, bytes) != cudaSuccess || cudaMalloc(&e->d_vout, bytes) != cudaSuccess) {
            cudaGetLastError();
            e->last_error = "device allocation of the staging buffers failed";
            return SDT_ERR_ALLOC;
        }
        e->host_cap = nrhs;
    }
    const size_t row = (size_t)e->n3 * sizeof(double);
    CAPI_CUDA(e, cudaMemcpy2DAsync(e->d_fin, row, f, (size_t)ldf * sizeof(double), row, nrhs, cudaMemcpyHostToDevice,
                                   e->stream));
    if (beta != 0.0)
        CAPI_CUDA(e, cudaMemcpy2DAsync(e->d_vout, row, v, (size_t)ldv * sizeof(double), row, nrhs,
                                       cudaMemcpyHostToDevice, e->stream));
    const int st = sdt::ewald_mulvec(e, nrhs, alpha, e->n3, e->d_fin, beta, e->n3, e->d_vout);
    if (st != SDT_OK) return st;
    CAPI_CUDA(e, cudaMemcpy2DAsync(v, (size_t)ldv * sizeof(double), e->d_vout, row, row, nrhs, cudaMemcpyDeviceToHost,
                                   e->stream));
    CAPI_CUDA(e, cudaStreamSynchronize(e->stream));
    return SDT_OK;
}

int sdt_ewald_get_matrix(sdt_ewald *h, int ldm, double *mat)
{
    if (!h || !mat) return SDT_ERR_INVALID;
    sdt::EwaldEngine *e = &h->e;
    if (ldm < e->n3) {
        e->last_error = "ldm must be >= 3*npos";
        return SDT_ERR_INVALID;
    }
    if (!e->updated) {
        e->last_error = "Update() must be called first";
        return SDT_ERR_STATE;
    }
    CAPI_CUDA(e, cudaSetDevice(e->device));
    CAPI_CUDA(e, cudaMemcpy2DAsync(mat, (size_t)ldm * sizeof(double), e->d_mat, (size_t)e->ldm * sizeof(double),
                                   (size_t)e->n3 * sizeof(double), e->n3, cudaMemcpyDeviceToHost, e->stream));
    CAPI_CUDA(e, cudaStreamSynchronize(e->stream));
    return SDT_OK;
}

int sdt_ewald_info(const sdt_ewald *h, double *xi, double *rmax, double *kmax, int *nimages, int *nkvectors)
{
    if (!h) return SDT_ERR_INVALID;
    if (xi) *xi = h->e.xi;
    if (rmax) *rmax = h->e.rmax;
    if (kmax) *kmax = h->e.kmax;
    if (nimages) *nimages = h->e.nr;
    if (nkvectors) *nkvectors = h->e.nk;
    return SDT_OK;
}

int sdt_ewald_dim(const sdt_ewald *h) { return h ? h->e.n3 : SDT_ERR_INVALID; }

int sdt_ewald_set_stream(sdt_ewald *h, void *stream)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::EwaldEngine *e = &h->e;
    CAPI_CUDA(e, cudaStreamSynchronize(e->stream));
    if (e->own_stream) cudaStreamDestroy(e->stream);
    e->own_stream = false;
    e->stream = static_cast<cudaStream_t>(stream);
    if (!e->stream) {
        CAPI_CUDA(e, cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->own_stream = true;
    }
    return SDT_OK;
}

const char *sdt_ewald_last_error(const sdt_ewald *h) { return h ? h->e.last_error.c_str() : "null handle"; }

void sdt_ewald_destroy(sdt_ewald *h)
{
    if (!h) return;
    sdt::ewald_free(&h->e);
    delete h;
}


int sdt_lanczos_compute_ewald_device(sdt_lanczos *h, sdt_ewald *mob, int nrhs, int ldz, const double *d_z, int ldy,
                                     double *d_y, int *iters)
{
    if (!h || !mob || !d_z || !d_y) return SDT_ERR_INVALID;
    sdt::LanczosState *lz = &h->s;
    if (cudaSetDevice(lz->device) != cudaSuccess) return SDT_ERR_CUDA;
    // the matrix is built on the engine stream: the solver's stream waits for it
    if (cudaStreamSynchronize(mob->e.stream) != cudaSuccess) return SDT_ERR_CUDA;
    const int st = sdt::lanczos_compute_op(lz, sdt::ewald_mob_op(&mob->e), nrhs, ldz, d_z, ldy, d_y, iters);
    if (cudaStreamSynchronize(lz->stream) != cudaSuccess) return SDT_ERR_CUDA;
    return st;
}

int sdt_lanczos_compute_ewald(sdt_lanczos *h, sdt_ewald *mob, int nrhs, int ldz, const double *z, int ldy,
                              double *y, int *iters)
{
    if (!h || !mob || !z || !y) return SDT_ERR_INVALID;
    sdt::LanczosState *lz = &h->s;
    if (nrhs < 0 || ldz < lz->dim || ldy < lz->dim) {
        lz->last_error = "bad nrhs or leading dimension";
        return SDT_ERR_INVALID;
    }
    if (nrhs == 0) return SDT_OK;
    if (cudaSetDevice(lz->device) != cudaSuccess) return SDT_ERR_CUDA;
    const int n = lz->dim;
    if (nrhs > lz->host_cap) {
        cudaFree(lz->d_zin);
        cudaFree(lz->d_yout);
        lz->d_zin = lz->d_yout = nullptr;
        lz->host_cap = 0;
        const size_t bytes = (size_t)nrhs * n * sizeof(double);
        if (cudaMalloc(&lz->d_zin, bytes) != cudaSuccess || cudaMalloc(&lz->d_yout, bytes) != cudaSuccess) {
            cudaGetLastError();
            lz->last_error = "device allocation of staging buffers failed";
            return SDT_ERR_ALLOC;
        }
        lz->host_cap = nrhs;
    }
    const size_t row = (size_t)n * sizeof(double);
    if (cudaMemcpy2DAsync(lz->d_zin, row, z, (size_t)ldz * sizeof(double), row, nrhs, cudaMemcpyHostToDevice,
                          lz->stream) != cudaSuccess) {
        lz->last_error = "copy of z failed";
        return SDT_ERR_CUDA;
    }
    if (cudaStreamSynchronize(mob->e.stream) != cudaSuccess) return SDT_ERR_CUDA;
    const int st = sdt::lanczos_compute_op(lz, sdt::ewald_mob_op(&mob->e), nrhs, n, lz->d_zin, n, lz->d_yout, iters);
    if (st != SDT_OK && st != SDT_ERR_NOT_CONVERGED) return st;
    if (cudaMemcpy2DAsync(y, (size_t)ldy * sizeof(double), lz->d_yout, row, row, nrhs, cudaMemcpyDeviceToHost,
                          lz->stream) != cudaSuccess ||
        cudaStreamSynchronize(lz->stream) != cudaSuccess) {
        lz->last_error = "copy of y failed";
        return SDT_ERR_CUDA;
    }
    return st;
}

int sdt_lanczos_compute(sdt_lanczos *h, sdt_spme *mob, int nrhs, int ldz, const double *z, int ldy, double *y,
                        int *iters)
{
    if (!h || !mob) return SDT_ERR_INVALID;
    sdt::LanczosState *lz = &h->s;
    if (nrhs < 0 || ldz < lz->dim || ldy < lz->dim) {
        lz->last_error = "bad nrhs or leading dimension";
        return SDT_ERR_INVALID;
    }
    if (nrhs == 0) return SDT_OK;
    if (cudaSetDevice(lz->device) != cudaSuccess) return SDT_ERR_CUDA;
    const int n = lz->dim;
    if (nrhs > lz->host_cap) {
        cudaFree(lz->d_zin);
        cudaFree(lz->d_yout);
        lz->d_zin = lz->d_yout = nullptr;
        lz->host_cap = 0;
        const size_t bytes = (size_t)nrhs * n * sizeof(double);
        if (cudaMalloc(&lz->d_zin, bytes) != cudaSuccess || cudaMalloc(&lz->d_yout, bytes) != cudaSuccess) {
            cudaGetLastError();
            lz->last_error = "device allocation of staging buffers failed";
            return SDT_ERR_ALLOC;
        }
        lz->host_cap = nrhs;
    }
    const size_t row = (size_t)n * sizeof(double);
    if (cudaMemcpy2DAsync(lz->d_zin, row, z, (size_t)ldz * sizeof(double), row, nrhs, cudaMemcpyHostToDevice,
                          lz->stream) != cudaSuccess) {
        lz->last_error = "copy of z failed";
        return SDT_ERR_CUDA;
    }
    const int st = sdt::lanczos_compute(lz, &mob->e, nrhs, n, lz->d_zin, n, lz->d_yout, iters);
    if (st != SDT_OK && st != SDT_ERR_NOT_CONVERGED) return st;
    if (cudaMemcpy2DAsync(y, (size_t)ldy * sizeof(double), lz->d_yout, row, row, nrhs, cudaMemcpyDeviceToHost,
                          lz->stream) != cudaSuccess ||
        cudaStreamSynchronize(lz->stream) != cudaSuccess) {
        lz->last_error = "copy of y failed";
        return SDT_ERR_CUDA;
    }
    return st;
}

int sdt_lanczos_history(const sdt_lanczos *h, double *out, int max_entries)
{
    if (!h || (max_entries > 0 && !out)) return SDT_ERR_INVALID;
    const std::vector<double> &hist = h->s.history;
    const int n = (int)hist.size();
    for (int i = 0; i < n && i < max_entries; i++) out[i] = hist[i];
    return n;
}

int sdt_lanczos_products(const sdt_lanczos *h, long long *out)
{
    if (!h || !out) return SDT_ERR_INVALID;
    *out = h->s.products;
    return SDT_OK;
}

const char *sdt_lanczos_last_error(const sdt_lanczos *h) { return h ? h->s.last_error.c_str() : "null handle"; }

void sdt_lanczos_destroy(sdt_lanczos *h)
{
    if (!h) return;
    sdt::lanczos_free(&h->s);
    delete h;
}

}  // extern "C"
