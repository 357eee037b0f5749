// Device building blocks shared by the single-system and the batched block
// Lanczos (lanczos.cu, packed_lanczos.cu).
#pragma once
#include <cuda_runtime.h>

namespace sdt {

// One Cholesky-QR step on the device for a k x k Gram matrix G (row-major,
// k <= KMAX), one warp: R1 = chol(G) (upper, G = R1^T R1), Ri = R1^-1,
// and the running factor Racc <- R1 Racc (Racc = R1 when `first`).  Lane 0
// forms each pivot, the lanes take the columns right of it; the operation
// order per entry is that of a column-by-column Cholesky and back
// substitution.  A pivot that is not positive (rank-deficient block: Lanczos
// breakdown) sets *flag = 1 and Ri = 0, so the block becomes zero and stays
// finite.  When Bout is given, Racc is also written to Bout and its transpose
// to Btout.
template <int KMAX>
__device__ __forceinline__ void chol_qr_step_warp(int k, const double *__restrict__ G, double *__restrict__ Ri,
                                                  double *__restrict__ Racc, int first, double *__restrict__ Bout,
                                                  double *__restrict__ Btout, double *__restrict__ flag)
{
    __shared__ double sR[KMAX * KMAX];
    __shared__ double sI[KMAX * KMAX];
    __shared__ double sA[KMAX * KMAX];
    __shared__ double sG[KMAX * KMAX];
    const int lane = threadIdx.x & 31;
    for (int t = lane; t < k * k; t += 32) {
        sR[t] = 0.0;
        sI[t] = 0.0;
        sA[t] = first ? 0.0 : Racc[t];
        sG[t] = G[t];
    }
    __syncwarp();
    bool bad = false;
    for (int j = 0; j < k; j++) {
        double d = 0.0;
        if (lane == 0) {
            d = sG[j * k + j];
            for (int t = 0; t < j; t++) d -= sR[t * k + j] * sR[t * k + j];
        }
        d = __shfl_sync(0xffffffffu, d, 0);
        if (!(d > 0.0)) {
            bad = true;
            break;
        }
        const double rjj = sqrt(d);
        if (lane == 0) sR[j * k + j] = rjj;
        const int c = j + 1 + lane;
        if (c < k) {
            double a = sG[j * k + c];
            for (int t = 0; t < j; t++) a -= sR[t * k + j] * sR[t * k + c];
            sR[j * k + c] = a / rjj;
        }
        __syncwarp();
    }
    if (bad) {
        for (int t = lane; t < k * k; t += 32) Ri[t] = 0.0;
        if (lane == 0) *flag = 1.0;
        return;
    }
    if (first && lane == 0) *flag = 0.0;
    if (lane < k) {
        const int c = lane;
        for (int r = k - 1; r >= 0; r--) {
            double v = (r == c) ? 1.0 : 0.0;
            for (int t = r + 1; t < k; t++) v -= sR[r * k + t] * sI[t * k + c];
            sI[r * k + c] = v / sR[r * k + r];
        }
    }
    __syncwarp();
    for (int t = lane; t < k * k; t += 32) {
        const int i = t / k, j = t % k;
        Ri[t] = sI[t];
        double v;
        if (first) {
            v = sR[t];
        } else {
            v = 0.0;
            for (int q = 0; q < k; q++) v += sR[i * k + q] * sA[q * k + j];
        }
        Racc[t] = v;
        if (Bout) {
            Bout[t] = v;
            Btout[j * k + i] = v;
        }
    }
}

}  // namespace sdt
