// Batched block Lanczos over the systems of a packed batch (packed_lanczos.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "packed.h"

namespace sdt {

constexpr int kBlMaxK = 16;  // largest block size of the batched solver

// One system, device copy.
struct BLSys {
    double *V = nullptr;        // Krylov basis [(max_iters + 1) k][ld]
    int n = 0, ld = 0;          // 3 npos, leading dimension
    double *coef = nullptr;     // [(max_iters + 1) k][k]: reorthogonalisation C, final D
    double *small = nullptr;    // [k][k] Gram scratch
    double *qr = nullptr;       // [3][k][k]: R^-1, running R, B^T
    double *hist = nullptr;     // [max_iters + 1][hs]: A_i | B_i | breakdown flag
    const double *z = nullptr;  // per call: input block, output block
    double *y = nullptr;
    int ldz = 0, ldy = 0;
    int mfin = 0;               // rows of the final coefficient block
};

struct BLState {
    int device = 0;
    cudaStream_t stream = nullptr;
    int nsys = 0, max_iters = 0, max_k = 0, hs = 0;
    double tol = 0.0;
    std::vector<BLSys> h_sys;
    BLSys *d_sys = nullptr;
    double *d_V = nullptr;
    double *d_mats = nullptr;      // per system [coef | small | qr | hist]
    size_t mats_stride = 0;        // doubles between two systems' blocks in d_mats
    size_t hist_pitch = 0;         // doubles of one system's history
    double *h_hist = nullptr;      // pinned [nsys][max_iters + 1][hs]
    double *h_small = nullptr;     // pinned [nsys][small | qr]
    int *d_act = nullptr, *d_first = nullptr;
    int *h_stage = nullptr;        // pinned: first[] and the active list
    int2 *d_map = nullptr, *h_map = nullptr;
    size_t map_cap = 0;
    double *d_part = nullptr;
    size_t part_cap = 0;
    int ngram = 0, ngemm = 0, nact = 0;
    std::vector<cudaEvent_t> ev;   // per iteration: its coefficients reached the host
    cudaEvent_t ev_map = nullptr;  // the last map upload has run
    int last_iters = 0;
    std::string last_error;
};

// Workspace for systems of npos[] particles, blocks of up to max_k vectors.
int bl_create(BLState *bl, const std::vector<int> &npos, int max_iters, int max_k, double tol, int device,
              cudaStream_t stream);
// y_j ~ sqrt(M_j) z_j for the systems sel[j] (global ids of `pb`, whose
// engines hold the current positions), k vectors each; iters[j] = iteration
// count (-1 if tol was not reached: kErrNotConverged, y holds the last
// iterate).
int bl_compute(BLState *bl, PackedBatch *pb, const std::vector<int> &sel, int k, const double *const *z,
               const int *ldz, double *const *y, const int *ldy, int *iters);
void bl_free(BLState *bl);

}  // namespace sdt
