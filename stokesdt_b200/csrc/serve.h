// Served request stream state (device-resident systems + request queue).
#pragma once
#include <cuda_runtime.h>

#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "lanczos.h"
#include "packed.h"
#include "packed_lanczos.h"

namespace sdt {

constexpr int kPending = 1;  // request status while queued or running

struct ServeSystem {
    SpmeEngine eng;
    double *d_pos = nullptr;
    double *d_in = nullptr, *d_out = nullptr;  // request vectors (max_nrhs x 3 npos each)
    size_t bytes = 0;   // admitted device-memory estimate
    bool busy = false;  // a worker or a batch lane is running a request on it
    bool packable = false;  // monodisperse with K <= 256: served by the batch lanes
    int pk = -1;            // index in the batch lanes' packed set (-1 until built)
};

struct ServeRequest {
    long long id = -1;
    int sys = -1;
    int kind = 0;  // 0 mobility apply (M in), 1 Brownian (sqrt(M) in)
    int nrhs = 1;
    const double *in = nullptr;
    double *out = nullptr;
    double t_submit = 0.0;
};

struct ServeWorker {
    cudaStream_t stream = nullptr;
    LanczosState *lz = nullptr;
    double *d_in = nullptr, *d_out = nullptr;
    std::thread th;
};

// A batch lane: runs batches of requests (one kind, one RHS count, distinct
// systems) as one packed product or one lockstep block Lanczos over their
// systems, on its own stream with its own packed state.
struct ServeBatchLane {
    cudaStream_t stream = nullptr;
    PackedBatch *pk = nullptr;
    BLState *bl = nullptr;
    std::thread th;
    bool busy = false;
};

struct ServeState {
    int device = 0;
    size_t budget = 0, used = 0;
    int max_npos = 0, max_nrhs = 0;
    long long next_ticket = 0, completed = 0, rejected = 0;
    bool stopping = false;
    std::vector<ServeSystem *> systems;
    std::vector<ServeWorker> workers;
    // continuous batching (monodisperse systems with K <= 256)
    bool batching = true;            // cleared by STOKESDT_SERVE_BATCH=0
    bool batch_all = false;          // STOKESDT_SERVE_BATCH=all: lone requests to the batch lanes too
    int max_iters = 0, max_batch = 32;
    double tol = 0.0;
    std::vector<ServeBatchLane> blanes;
    std::vector<int> pk_sys;         // packed index -> system id
    bool pk_dirty = false, rebuilding = false;
    size_t lane_bytes = 0;           // device memory of the batch lanes' workspaces
    int lanes_active = 0;            // batch lanes whose workspace fits the budget
    int workers_busy = 0;            // per-request workers running a request
    long long batches = 0, batched_requests = 0;
    std::deque<ServeRequest> queue;
    std::map<long long, int> status;
    std::map<long long, double> latency_ms;
    std::mutex mu;
    std::condition_variable cv;
    std::string last_error;
};

size_t serve_system_bytes(int npos, double box, int K, double rmax, int rhs);
int serve_create(ServeState *sv, int device, size_t budget, int lanes, int max_npos, int max_iters, int max_nrhs,
                 double tol);
int serve_register(ServeState *sv, int npos, const double *rdi, double box, int K, double xi, double rmax,
                   int porder, const double *pos, int *sys_id);
int serve_submit(ServeState *sv, int sys_id, int kind, int nrhs, const double *in, double *out, long long *ticket);
int serve_wait(ServeState *sv, long long ticket, double timeout_ms, double *latency_ms);
void serve_worker_loop(ServeState *sv, int lane);
void serve_batch_loop(ServeState *sv, int lane);
void serve_free(ServeState *sv);

}  // namespace sdt
