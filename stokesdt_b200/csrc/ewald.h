// Dense Ewald-summed RPY mobility matrix on one GPU (MobEwald,
// src/mob/mob_ewald.cc:21-165; EwaldKernel src/mob/ewald.cc:86-330, tables
// src/mob/ewald.cc:643-797 of the reference).  FP64 throughout.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "engine.h"
#include "lanczos.h"

namespace sdt {

struct EwaldEngine {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int npos = 0, n3 = 0, ldm = 0;  // matrix dimension 3 npos, leading dimension
    double box = 0.0, tol = 0.0, xi = 0.0, rmax = 0.0, kmax = 0.0;
    int nr = 0, nk = 0;             // real-space images, reciprocal vectors
    double *d_rdi = nullptr;        // [npos]
    double *d_img = nullptr;        // [nr][3] image shifts
    double *d_kv = nullptr;         // [nk][8]: k1 k2 k3, 6 kexp, k^2 kexp, 0...
    double *d_pos = nullptr;        // [3 npos] positions of the last update
    double *d_cs = nullptr;         // [2][nk][npos] cos / sin(k . r_i)
    double *d_mat = nullptr;        // [n3][ldm] the mobility matrix (both triangles)
    double *d_fin = nullptr, *d_vout = nullptr;  // host-API staging
    int host_cap = 0;
    bool updated = false;
    std::string last_error;
};

// Validation as MobEwald::Init (src/mob/mob_ewald.cc:56-108): npos > 0,
// box > 0, tol > 0, xi > 0 (xi <= 0 on entry selects the reference's
// default 10^(1/6) sqrt(pi) / L, src/mob/mob_ewald.cc:50-52).  rdi is copied.
int ewald_create(EwaldEngine *e, const double *rdi);
int ewald_update(EwaldEngine *e, const double *d_pos);
int ewald_mulvec(EwaldEngine *e, int nrhs, double alpha, int ldf, const double *d_f, double beta, int ldv,
                 double *d_v);
void ewald_free(EwaldEngine *e);
// The engine as a mobility operator for the block Lanczos (products queued on
// the stream the solver passes).
MobOp ewald_mob_op(EwaldEngine *e);

}  // namespace sdt
