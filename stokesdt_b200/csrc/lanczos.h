// Internal state of one block-Lanczos solver (BrwnLanczos) on one GPU.
#pragma once
#include <cuda_runtime.h>
#include <functional>
#include <string>
#include <vector>

#include "engine.h"

namespace sdt {

struct LanczosState {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int dim = 0, max_iters = 0, max_nrhs = 0;
    double tol = 0.0;
    bool reorth = false;        // the reference does not reorthogonalise
    int lookahead = 4;          // most eigensolves in flight with reorthogonalisation
    int ldv = 0;
    double *d_V = nullptr;      // Krylov basis [(max_iters+1) * k][ldv]
    double *d_part = nullptr;   // Gram partial sums
    unsigned *d_arrive = nullptr;  // CTAs done with a small Gram (the last one sums the parts)
    size_t part_cap = 0;
    int vec_grid = 0;                  // CTAs of the fused single-vector iteration (0: not available)
    unsigned long long vec_launches = 0;  // its launches so far (their parity picks the barrier counter)
    unsigned vec_barrier_skew = 0;     // arrivals added to its first barrier's target (failure tests only)
    unsigned *h_err = nullptr;         // pinned copy of its barrier-timeout flag
    int gram_chunks = 0;
    int num_sms = 148;
    double *d_small = nullptr;  // k x k scratch
    double *d_coef = nullptr;   // (max_iters+1)k x k coefficients
    double *d_dY = nullptr;     // k x ldv difference block
    // per-iteration [A_i | B_i | breakdown flag] blocks (stride hist_stride),
    // written on the device and copied to pinned host memory asynchronously;
    // ev[i] completes when block i has arrived
    int hist_stride = 0;
    double *d_hist = nullptr;
    double *h_hist = nullptr;
    std::vector<cudaEvent_t> ev;
    double *d_qr = nullptr;     // Cholesky-QR scratch: R^-1, running R, B^T
    long long products = 0;     // block products issued by the last compute call
    double *d_zin = nullptr;    // host-API staging
    double *d_yout = nullptr;
    int host_cap = 0;
    long long nonspd_count = 0;  // iterations whose T had negative eigenvalues
    std::vector<double> history; // ||Y_i - Y_{i-1}||_F / ||Z||_F of the last group
    // host-side timing of the last compute call (milliseconds)
    double t_sync_ms = 0.0, t_eigen_ms = 0.0, t_wait_ms = 0.0;
    std::string last_error;
};

// A mobility operator the solver applies: v := alpha M f + beta v for nrhs
// device vectors, queued on stream s (the SPME engine or the dense Ewald).
struct MobOp {
    int dim = 0;
    std::function<int(int nrhs, double alpha, int ldf, const double *f, double beta, int ldv, double *v,
                      cudaStream_t s)>
        mulvec;
    std::function<std::string()> error;
};

int lanczos_alloc(LanczosState *lz);
void lanczos_free(LanczosState *lz);
int lanczos_compute(LanczosState *lz, SpmeEngine *mob, int nrhs, int ldz, const double *d_z, int ldy,
                    double *d_y, int *iters);
// The same on any mobility operator.
int lanczos_compute_op(LanczosState *lz, const MobOp &mob, int nrhs, int ldz, const double *d_z, int ldy,
                       double *d_y, int *iters);

}  // namespace sdt
