// Batched independent systems (many small suspensions processed together).
//
// There is no batched entry point in the reference; the unit of work is the
// reference's per-system sequence MobSpme::Update -> MobSpme::MulVector ->
// BrwnLanczos::Compute (src/mob/mob_spme.cc:205-263,
// src/brwn/brwn_lanczos.cc:278-304), repeated for every system.  Here every
// system keeps its own SPME engine (grid size, Ewald split and pair list of
// its own), and the systems are spread over `lanes`: a lane is a CUDA stream,
// a host thread and one Lanczos workspace sized for the largest system it
// owns.  Lanes run concurrently, so small systems that cannot fill the GPU
// alone overlap; systems go to lanes largest-first onto the least-loaded lane
// (estimated cost N * log N + K^3).
//
// Vectors of all systems are concatenated: system s owns nrhs blocks of
// 3*npos[s] doubles starting at offset nrhs * 3 * (npos[0] + ... + npos[s-1]).
//
// Packed mode (the default when every system is monodisperse with K <= 256
// and reorthogonalisation is on): after the per-system updates, every
// product is one packed launch sequence over all systems and the block
// Lanczos runs all systems in lockstep (packed.h, packed_lanczos.h), so a
// batch step takes tens of launches per Lanczos iteration instead of tens per
// system and iteration.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"

namespace sdt {

static int batch_error(BatchState *b, int st, const std::string &msg)
{
    b->last_error = msg;
    return st;
}

int batch_create(BatchState *b, int nsys, const int *npos, const double *rdi_all, const double *box,
                 const int *dim, const double *xi, const double *rmax, int porder, int max_iters,
                 int max_nrhs, double tol, int lanes, int device)
{
    if (nsys <= 0 || !npos || !rdi_all || !box || !dim || !xi || !rmax)
        return batch_error(b, kErrInvalid, "bad batch arguments");
    if (max_iters <= 0 || max_nrhs <= 0 || !(tol > 0.0))
        return batch_error(b, kErrInvalid, "bad Lanczos parameters");
    b->device = device;
    b->nsys = nsys;
    b->sys.resize(nsys);
    b->pos_off.assign(nsys + 1, 0);
    for (int s = 0; s < nsys; s++) {
        if (npos[s] <= 0) return batch_error(b, kErrInvalid, "every system needs npos > 0");
        b->pos_off[s + 1] = b->pos_off[s] + 3LL * npos[s];
    }
    if (cudaSetDevice(device) != cudaSuccess) return batch_error(b, kErrCuda, "cudaSetDevice failed");
    // engines
    long long roff = 0;
    for (int s = 0; s < nsys; s++) {
        SpmeEngine *e = new SpmeEngine;
        b->sys[s].mob = e;
        e->device = device;
        e->npos = npos[s];
        e->box = box[s];
        e->xi = xi[s];
        e->rmax = rmax[s];
        e->K = dim[s];
        e->p = porder;
        std::vector<double> r(rdi_all + roff, rdi_all + roff + npos[s]);
        roff += npos[s];
        for (double a : r)
            if (!(a > 0.0)) return batch_error(b, kErrInvalid, "particle radii must be > 0");
        e->mono = std::all_of(r.begin(), r.end(), [](double a) { return a == 1.0; });
        int st = spme_create(e);
        if (st == kOk) st = spme_set_radii(e, r.data());
        if (st != kOk) return batch_error(b, st, "system " + std::to_string(s) + ": " + e->last_error);
        // the engine runs on its lane's stream (assigned below), not its own
        if (e->own_stream && e->stream) {
            cudaStreamSynchronize(e->stream);
            cudaStreamDestroy(e->stream);
        }
        e->own_stream = false;
        e->stream = nullptr;
        e->overlap = false;    // the lanes already overlap systems
        e->tc_enabled = false;  // no tensor-core operand tiles per system
        b->sys[s].cost = (double)npos[s] * std::log2((double)npos[s] + 2.0) + std::pow((double)dim[s], 3.0);
    }
    // lanes: largest first onto the least-loaded lane
    lanes = std::max(1, std::min(lanes, nsys));
    b->lanes.resize(lanes);
    std::vector<int> order(nsys);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int c) { return b->sys[a].cost > b->sys[c].cost; });
    std::vector<double> load(lanes, 0.0);
    for (int s : order) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[l] += b->sys[s].cost;
        b->lanes[l].systems.push_back(s);
    }
    for (int l = 0; l < lanes; l++) {
        Lane &ln = b->lanes[l];
        if (cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking) != cudaSuccess)
            return batch_error(b, kErrCuda, "stream creation failed");
        int nmax = 0;
        for (int s : ln.systems) nmax = std::max(nmax, npos[s]);
        if (nmax == 0) continue;
        ln.lz = new LanczosState;
        ln.lz->device = device;
        ln.lz->stream = ln.stream;
        ln.lz->dim = 3 * nmax;
        ln.lz->max_iters = max_iters;
        ln.lz->max_nrhs = std::min(max_nrhs, nmax);
        ln.lz->tol = tol;
        ln.lz->reorth = b->reorth;
        const int st = lanczos_alloc(ln.lz);
        if (st != kOk) return batch_error(b, st, "Lanczos workspace: " + ln.lz->last_error);
        for (int s : ln.systems) b->sys[s].mob->stream = ln.stream;
    }
    b->max_iters = max_iters;
    b->max_nrhs = max_nrhs;
    b->tol = tol;
    b->packed_ok = b->reorth && max_nrhs <= kBlMaxK;
    for (int s = 0; s < nsys && b->packed_ok; s++) {
        const SpmeEngine *e = b->sys[s].mob;
        if (!e->mono || e->K > 256 || !e->tma_tabs || !e->tma_enabled || !e->zfused) b->packed_ok = false;
    }
    const char *env = std::getenv("STOKESDT_BATCH_PACKED");
    if (b->packed_ok && !(env && env[0] == '0')) return batch_set_packed(b, true);
    return kOk;
}

int batch_set_packed(BatchState *b, bool packed)
{
    if (!packed) {
        b->packed = false;
        return kOk;
    }
    if (!b->packed_ok)
        return batch_error(b, kErrUnsupported,
                           "packed mode needs monodisperse systems with K <= 256, reorthogonalisation and "
                           "at most 16 RHS per Lanczos group");
    if (!b->pk) {
        if (cudaSetDevice(b->device) != cudaSuccess) return batch_error(b, kErrCuda, "cudaSetDevice failed");
        if (!b->pstream && cudaStreamCreateWithFlags(&b->pstream, cudaStreamNonBlocking) != cudaSuccess)
            return batch_error(b, kErrCuda, "stream creation failed");
        std::vector<SpmeEngine *> eng;
        std::vector<int> npos;
        for (SystemSlot &sl : b->sys) {
            eng.push_back(sl.mob);
            npos.push_back(sl.mob->npos);
        }
        b->pk = new PackedBatch;
        int st = packed_create(b->pk, eng, std::max(1, b->max_nrhs), b->device, b->pstream);
        if (st != kOk) {
            const std::string msg = b->pk->last_error;
            packed_free(b->pk);
            delete b->pk;
            b->pk = nullptr;
            return batch_error(b, st, "packed set-up: " + msg);
        }
        b->bl = new BLState;
        st = bl_create(b->bl, npos, b->max_iters, std::max(1, b->max_nrhs), b->tol, b->device, b->pstream);
        if (st != kOk) {
            const std::string msg = b->bl->last_error;
            bl_free(b->bl);
            delete b->bl;
            b->bl = nullptr;
            return batch_error(b, st, "batched Lanczos set-up: " + msg);
        }
    }
    b->packed = true;
    // the packed descriptors follow the engines' current positions
    bool updated = true;
    for (SystemSlot &sl : b->sys) updated = updated && sl.mob->updated;
    if (updated) {
        const int st = packed_refresh(b->pk);
        if (st != kOk) return batch_error(b, st, b->pk->last_error);
    }
    return kOk;
}

// Run fn(system, lane) for every system, lanes in parallel host threads.
template <typename Fn>
static int for_each_system(BatchState *b, Fn &&fn)
{
    std::vector<int> status(b->lanes.size(), kOk);
    std::vector<std::string> msg(b->lanes.size());
    auto run_lane = [&](int l) {
        cudaSetDevice(b->device);
        for (int s : b->lanes[l].systems) {
            const int st = fn(s, b->lanes[l]);
            if (st != kOk && st != kErrNotConverged) {
                status[l] = st;
                msg[l] = "system " + std::to_string(s) + ": " + b->sys[s].mob->last_error +
                         (b->lanes[l].lz ? " " + b->lanes[l].lz->last_error : std::string());
                return;
            }
            if (st == kErrNotConverged && status[l] == kOk) status[l] = kErrNotConverged;
        }
    };
    std::vector<std::thread> th;
    for (size_t l = 1; l < b->lanes.size(); l++) th.emplace_back(run_lane, (int)l);
    run_lane(0);
    for (std::thread &t : th) t.join();
    int out = kOk;
    for (size_t l = 0; l < b->lanes.size(); l++) {
        if (status[l] != kOk && status[l] != kErrNotConverged) return batch_error(b, status[l], msg[l]);
        if (status[l] == kErrNotConverged) out = kErrNotConverged;
    }
    return out;
}

int batch_update(BatchState *b, const double *d_pos_all)
{
    if (b->packed) {
        // the positions may come from work queued on the packed stream
        if (cudaStreamSynchronize(b->pstream) != cudaSuccess)
            return batch_error(b, kErrCuda, "packed stream synchronize failed");
    }
    int st = for_each_system(b, [&](int s, Lane &) {
        return spme_update(b->sys[s].mob, d_pos_all + b->pos_off[s]);
    });
    if (st != kOk || !b->packed) return st;
    for (Lane &ln : b->lanes)
        if (ln.stream && cudaStreamSynchronize(ln.stream) != cudaSuccess)
            return batch_error(b, kErrCuda, "stream synchronize failed");
    st = packed_refresh(b->pk);
    if (st != kOk) return batch_error(b, st, b->pk->last_error);
    return kOk;
}

int batch_mulvec(BatchState *b, int nrhs, double alpha, const double *d_f_all, double beta, double *d_v_all)
{
    if (b->packed) {
        std::vector<int> act(b->nsys);
        std::vector<const double *> f(b->nsys);
        std::vector<double *> v(b->nsys);
        std::vector<int> ld(b->nsys);
        for (int r0 = 0; r0 < nrhs; r0 += b->pk->rhs_cap) {
            const int nr = std::min(b->pk->rhs_cap, nrhs - r0);
            for (int s = 0; s < b->nsys; s++) {
                const long long n3 = 3LL * b->sys[s].mob->npos;
                act[s] = s;
                f[s] = d_f_all + (long long)nrhs * b->pos_off[s] + r0 * n3;
                v[s] = d_v_all + (long long)nrhs * b->pos_off[s] + r0 * n3;
                ld[s] = (int)n3;
            }
            const int st = packed_mulvec(b->pk, b->nsys, act.data(), nr, alpha, f.data(), ld.data(), beta, v.data(),
                                         ld.data());
            if (st != kOk) return batch_error(b, st, b->pk->last_error);
        }
        return kOk;
    }
    return for_each_system(b, [&](int s, Lane &) {
        SpmeEngine *e = b->sys[s].mob;
        const long long off = (long long)nrhs * b->pos_off[s];
        const int n3 = 3 * e->npos;
        return spme_mulvec(e, 0, nrhs, alpha, n3, d_f_all + off, beta, n3, d_v_all + off);
    });
}

int batch_lanczos(BatchState *b, int nrhs, const double *d_z_all, double *d_y_all, int *iters)
{
    if (b->packed) {
        std::vector<int> sel(b->nsys), ld(b->nsys), it(b->nsys, 0);
        std::vector<const double *> z(b->nsys);
        std::vector<double *> y(b->nsys);
        int out = kOk;
        // groups of max_nrhs RHS, as BrwnLanczos::Compute; iters[] reports the first
        for (int r0 = 0; r0 < nrhs; r0 += b->max_nrhs) {
            const int k = std::min(b->max_nrhs, nrhs - r0);
            for (int s = 0; s < b->nsys; s++) {
                const long long n3 = 3LL * b->sys[s].mob->npos;
                sel[s] = s;
                z[s] = d_z_all + (long long)nrhs * b->pos_off[s] + r0 * n3;
                y[s] = d_y_all + (long long)nrhs * b->pos_off[s] + r0 * n3;
                ld[s] = (int)n3;
            }
            const int st = bl_compute(b->bl, b->pk, sel, k, z.data(), ld.data(), y.data(), ld.data(), it.data());
            if (st != kOk && st != kErrNotConverged) return batch_error(b, st, b->bl->last_error);
            if (st == kErrNotConverged) out = kErrNotConverged;
            if (r0 == 0 && iters)
                for (int s = 0; s < b->nsys; s++) iters[s] = it[s];
        }
        return out;
    }
    return for_each_system(b, [&](int s, Lane &ln) {
        SpmeEngine *e = b->sys[s].mob;
        const long long off = (long long)nrhs * b->pos_off[s];
        const int n3 = 3 * e->npos;
        // the lane's workspace serves every system it owns: size it to this one
        ln.lz->dim = n3;
        const int ng = (nrhs + ln.lz->max_nrhs - 1) / ln.lz->max_nrhs;
        std::vector<int> it(std::max(1, ng), 0);
        const int st = lanczos_compute(ln.lz, e, nrhs, n3, d_z_all + off, n3, d_y_all + off, it.data());
        if (iters) iters[s] = it[0];
        return st;
    });
}

int batch_synchronize(BatchState *b)
{
    if (cudaSetDevice(b->device) != cudaSuccess) return batch_error(b, kErrCuda, "cudaSetDevice failed");
    if (b->pk) {
        const int st = packed_check_error(b->pk);
        if (st != kOk) return batch_error(b, st, b->pk->last_error);
    }
    for (Lane &ln : b->lanes)
        if (ln.stream && cudaStreamSynchronize(ln.stream) != cudaSuccess)
            return batch_error(b, kErrCuda, "stream synchronize failed");
    for (SystemSlot &sl : b->sys) {
        const int st = spme_check_device_error(sl.mob);
        if (st != kOk) return batch_error(b, st, sl.mob->last_error);
    }
    return kOk;
}

void batch_free(BatchState *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->bl) {
        bl_free(b->bl);
        delete b->bl;
        b->bl = nullptr;
    }
    if (b->pk) {
        packed_free(b->pk);
        delete b->pk;
        b->pk = nullptr;
    }
    if (b->pstream) cudaStreamDestroy(b->pstream);
    b->pstream = nullptr;
    for (Lane &ln : b->lanes)
        if (ln.stream) cudaStreamSynchronize(ln.stream);
    for (SystemSlot &sl : b->sys) {
        if (sl.mob) {
            sl.mob->stream = nullptr;  // the lane owns the stream
            spme_free(sl.mob);
            delete sl.mob;
            sl.mob = nullptr;
        }
    }
    for (Lane &ln : b->lanes) {
        if (ln.lz) {
            ln.lz->stream = nullptr;
            lanczos_free(ln.lz);
            delete ln.lz;
            ln.lz = nullptr;
        }
        if (ln.stream) cudaStreamDestroy(ln.stream);
        ln.stream = nullptr;
    }
    b->lanes.clear();
    b->sys.clear();
    cudaFree(b->d_stage);
    b->d_stage = nullptr;
    b->stage_cap = 0;
}

}  // namespace sdt
