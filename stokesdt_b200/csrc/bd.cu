// Device-resident Brownian-dynamics integrator: the step loop of
// BDSimBox::Advance (src/simbox/simbox_bd.cc:296-366) with every array on the
// GPU and the random vectors drawn on the GPU.
//
// Per step (istep, irhs = istep % interval):
//   irhs == 0:  Z <- N(0,1) [interval x 3N];  mob.Update(pos);
//               Y <- sqrt(M) Z (block Lanczos, groups of max_nrhs)
//   f <- 0; f += steric(pos)                           (forces, optional)
//   Y[irhs] <- dt * M f + sqrt(2 dt) * Y[irhs]         (mob.MulVector)
//   pos += Y[irhs]
// with M the SPME operator (MobSpme) or the dense Ewald matrix (MobEwald,
// the reference driver's default mob-method).
//
// Random vectors: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC11) with key = seed and counter =
// (pair index, interval start step); each call gives two 53-bit uniforms
// and Box-Muller turns them into two N(0,1) samples.  The reference draws
// from MKL VSL (rnd_stream.cc), whose stream is not reproduced.
#include <cmath>
#include <string>

#include "bd.h"

namespace sdt {

__device__ __forceinline__ void philox_round(uint32_t &c0, uint32_t &c1, uint32_t &c2, uint32_t &c3,
                                             uint32_t k0, uint32_t k1)
{
    const uint32_t m0 = 0xD2511F53u, m1 = 0xCD9E8D57u;
    const uint32_t lo0 = m0 * c0, hi0 = __umulhi(m0, c0);
    const uint32_t lo1 = m1 * c2, hi1 = __umulhi(m1, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
}

// Philox4x32 with 10 rounds; the key advances by the Weyl constants between rounds.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
    uint32_t c0 = c.x, c1 = c.y, c2 = c.z, c3 = c.w, k0 = k.x, k1 = k.y;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        philox_round(c0, c1, c2, c3, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return make_uint4(c0, c1, c2, c3);
}

// out[v * ld + e] ~ N(0,1) for v < nvec, e < dim; element q = v * dim + e is
// the (q & 1) output of pair q >> 1.
__global__ void k_bd_gaussian(long long nelem, int dim, int ld, unsigned long long seed,
                              unsigned long long step, double *__restrict__ out)
{
    const long long pair = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long q0 = 2 * pair;
    if (q0 >= nelem) return;
    const uint4 ctr = make_uint4((uint32_t)pair, (uint32_t)(pair >> 32), (uint32_t)step,
                                 (uint32_t)(step >> 32));
    const uint4 r = philox4x32_10(ctr, make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const unsigned long long a = ((unsigned long long)r.x << 32) | r.y;
    const unsigned long long b = ((unsigned long long)r.z << 32) | r.w;
    const double u1 = ((double)(a >> 11) + 0.5) * 0x1.0p-53;  // (0, 1)
    const double u2 = ((double)(b >> 11) + 0.5) * 0x1.0p-53;
    const double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    for (int t = 0; t < 2; t++) {
        const long long q = q0 + t;
        if (q >= nelem) break;
        const long long v = q / dim, e = q - v * dim;
        out[v * ld + e] = rad * (t == 0 ? c : s);
    }
}

__global__ void k_bd_axpy(int n, const double *__restrict__ x, double *__restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

static int bd_error(BdState *b, int st, const std::string &msg)
{
    b->last_error = msg;
    return st;
}

#define BD_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t err_ = (call);                                                            \
        if (err_ != cudaSuccess)                                                              \
            return bd_error(b, kErrCuda, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

#define BD_LAUNCH()                                                                           \
    do {                                                                                      \
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                            \
        cudaError_t err_ = cudaGetLastError();                                                \
        if (err_ != cudaSuccess)                                                              \
            return bd_error(b, kErrCuda, std::string("bd kernel: ") + cudaGetErrorString(err_)); \
    } while (0)

int bd_gaussian(cudaStream_t s, long long nvec, int dim, int ld, unsigned long long seed,
                unsigned long long step, double *d_out)
{
    const long long nelem = nvec * dim;
    const long long pairs = (nelem + 1) / 2;
    if (pairs <= 0) return kOk;
    k_bd_gaussian<<<(unsigned)((pairs + 255) / 256), 256, 0, s>>>(nelem, dim, ld, seed, step, d_out);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrCuda;
}

int bd_create(BdState *b)
{
    if ((!b->mob == !b->ew) || !b->lz)
        return bd_error(b, kErrInvalid, "one mobility handle (SPME or Ewald) and a Lanczos handle are required");
    if (!(b->dt > 0.0)) return bd_error(b, kErrInvalid, "dt must be > 0");
    if (b->interval <= 0) return bd_error(b, kErrInvalid, "mob_interval must be > 0");
    const int npos = b->mob ? b->mob->npos : b->ew->npos;
    const int device = b->mob ? b->mob->device : b->ew->device;
    if (b->lz->dim != 3 * npos) return bd_error(b, kErrInvalid, "Lanczos dimension != 3*npos");
    if (b->steric && b->steric->npos != npos)
        return bd_error(b, kErrInvalid, "steric force has a different particle count");
    if (b->lz->device != device || (b->steric && b->steric->device != device))
        return bd_error(b, kErrInvalid, "all handles must be on one device");
    b->device = device;
    b->npos = npos;
    b->ld = (3 * b->npos + 31) / 32 * 32;
    BD_CUDA(cudaSetDevice(b->device));
    BD_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
    const size_t ld = b->ld;
    BD_CUDA(cudaMalloc(&b->d_pos, ld * sizeof(double)));
    BD_CUDA(cudaMalloc(&b->d_f, ld * sizeof(double)));
    BD_CUDA(cudaMalloc(&b->d_z, (size_t)b->interval * ld * sizeof(double)));
    BD_CUDA(cudaMalloc(&b->d_disp, (size_t)b->interval * ld * sizeof(double)));
    BD_CUDA(cudaMemsetAsync(b->d_pos, 0, ld * sizeof(double), b->stream));
    return kOk;
}

int bd_advance(BdState *b, int nsteps)
{
    if (nsteps < 0) return bd_error(b, kErrInvalid, "nsteps < 0");
    BD_CUDA(cudaSetDevice(b->device));
    const int n3 = 3 * b->npos;
    const double sq = std::sqrt(2.0 * b->dt);
    // every engine runs on the integrator's stream while it advances
    cudaStream_t &mob_stream = b->mob ? b->mob->stream : b->ew->stream;
    cudaStream_t s_mob = mob_stream, s_lz = b->lz->stream;
    cudaStream_t s_st = b->steric ? b->steric->stream : nullptr;
    mob_stream = b->stream;
    const std::string &mob_error = b->mob ? b->mob->last_error : b->ew->last_error;
    b->lz->stream = b->stream;
    if (b->steric) b->steric->stream = b->stream;
    int st = kOk;
    for (int k = 0; k < nsteps && st == kOk; k++) {
        const int irhs = (int)(b->istep % b->interval);
        if (irhs == 0) {
            st = bd_gaussian(b->stream, b->interval, n3, b->ld, b->seed, (unsigned long long)b->istep, b->d_z);
            if (st != kOk) {
                bd_error(b, st, "random vectors: launch failed");
                break;
            }
            st = b->mob ? spme_update(b->mob, b->d_pos) : ewald_update(b->ew, b->d_pos);
            if (st != kOk) {
                bd_error(b, st, "Update: " + mob_error);
                break;
            }
            const int ngroups = (b->interval + b->lz->max_nrhs - 1) / b->lz->max_nrhs;
            b->iters.assign(ngroups, 0);
            st = b->mob ? lanczos_compute(b->lz, b->mob, b->interval, b->ld, b->d_z, b->ld, b->d_disp,
                                          b->iters.data())
                        : lanczos_compute_op(b->lz, ewald_mob_op(b->ew), b->interval, b->ld, b->d_z, b->ld,
                                             b->d_disp, b->iters.data());
            if (st == kErrNotConverged) {
                // BrwnLanczos only logs non-convergence; keep the last iterate
                b->not_converged++;
                st = kOk;
            } else if (st != kOk) {
                bd_error(b, st, "Brownian displacements: " + b->lz->last_error);
                break;
            }
        }
        double *disp = b->d_disp + (size_t)irhs * b->ld;
        if (cudaMemsetAsync(b->d_f, 0, (size_t)n3 * sizeof(double), b->stream) != cudaSuccess) {
            st = bd_error(b, kErrCuda, "clearing the force vector failed");
            break;
        }
        if (b->steric) {
            st = steric_accumulate(b->steric, b->d_pos, b->d_f);
            if (st != kOk) {
                bd_error(b, st, "steric force: " + b->steric->last_error);
                break;
            }
        }
        st = b->mob ? spme_mulvec(b->mob, 0, 1, b->dt, b->ld, b->d_f, sq, b->ld, disp)
                    : ewald_mulvec(b->ew, 1, b->dt, b->ld, b->d_f, sq, b->ld, disp);
        if (st != kOk) {
            bd_error(b, st, "MulVector: " + mob_error);
            break;
        }
        k_bd_axpy<<<(n3 + 255) / 256, 256, 0, b->stream>>>(n3, disp, b->d_pos);
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
        if (cudaGetLastError() != cudaSuccess) {
            st = bd_error(b, kErrCuda, "position update launch failed");
            break;
        }
        b->istep++;
    }
    mob_stream = s_mob;
    b->lz->stream = s_lz;
    if (b->steric) b->steric->stream = s_st;
    return st;
}

void bd_free(BdState *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    void *ptrs[] = {b->d_pos, b->d_f, b->d_z, b->d_disp};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    b->stream = nullptr;
}

}  // namespace sdt
