// Device-resident BD integrator state (BDSimBox::Advance of the reference).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "engine.h"
#include "ewald.h"
#include "lanczos.h"
#include "steric.h"

namespace sdt {

struct BdState {
    SpmeEngine *mob = nullptr;       // the mobility: SPME, or
    EwaldEngine *ew = nullptr;       // the dense Ewald matrix (exactly one of the two)
    LanczosState *lz = nullptr;
    StericEngine *steric = nullptr;  // optional
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int npos = 0, ld = 0;
    int interval = 1;                // steps per mobility interval (RHS per Lanczos call)
    double dt = 0.0;
    unsigned long long seed = 0;
    long long istep = 0;
    long long not_converged = 0;     // Lanczos calls that did not reach tol
    std::vector<int> iters;          // iteration counts of the last Lanczos call
    double *d_pos = nullptr;         // [3N] positions (not wrapped, like the reference)
    double *d_f = nullptr;           // [3N] forces
    double *d_z = nullptr;           // [interval][ld] random vectors
    double *d_disp = nullptr;        // [interval][ld] displacements
    std::string last_error;
};

int bd_create(BdState *b);
int bd_advance(BdState *b, int nsteps);
void bd_free(BdState *b);
// out[v*ld + e] ~ N(0,1), v < nvec, e < dim (counter = pair index, step).
int bd_gaussian(cudaStream_t s, long long nvec, int dim, int ld, unsigned long long seed,
                unsigned long long step, double *d_out);

}  // namespace sdt
