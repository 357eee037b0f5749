// Batched independent systems: one SPME engine per system, systems spread
// over concurrent lanes (stream + host thread + Lanczos workspace).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "engine.h"
#include "lanczos.h"
#include "packed.h"
#include "packed_lanczos.h"

namespace sdt {

struct SystemSlot {
    SpmeEngine *mob = nullptr;
    double cost = 0.0;  // estimated work (N log N + K^3), for lane balancing
};

struct Lane {
    cudaStream_t stream = nullptr;
    LanczosState *lz = nullptr;  // sized for the largest system of the lane
    std::vector<int> systems;
};

struct BatchState {
    int device = 0;
    int nsys = 0;
    bool reorth = true;
    std::vector<SystemSlot> sys;
    std::vector<Lane> lanes;
    std::vector<long long> pos_off;  // [nsys + 1] offsets of 3N blocks
    double *d_stage = nullptr;       // host-API staging (grown on demand)
    size_t stage_cap = 0;
    // packed mode (default when every system qualifies): products and block
    // Lanczos of all systems as packed launches on one stream (packed.h);
    // lanes mode: every system's own launches, systems spread over the lanes
    bool packed_ok = false;          // the systems allow the packed mode
    bool packed = false;             // packed mode selected
    int max_iters = 0, max_nrhs = 0;
    double tol = 0.0;
    cudaStream_t pstream = nullptr;
    PackedBatch *pk = nullptr;
    BLState *bl = nullptr;
    std::string last_error;
};

// 1: packed launches (needs monodisperse systems with K <= 256), 0: lanes.
int batch_set_packed(BatchState *b, bool packed);

int batch_create(BatchState *b, int nsys, const int *npos, const double *rdi_all, const double *box,
                 const int *dim, const double *xi, const double *rmax, int porder, int max_iters,
                 int max_nrhs, double tol, int lanes, int device);
int batch_update(BatchState *b, const double *d_pos_all);
int batch_mulvec(BatchState *b, int nrhs, double alpha, const double *d_f_all, double beta, double *d_v_all);
int batch_lanczos(BatchState *b, int nrhs, const double *d_z_all, double *d_y_all, int *iters);
int batch_synchronize(BatchState *b);
void batch_free(BatchState *b);

}  // namespace sdt
