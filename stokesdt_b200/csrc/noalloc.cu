// Real-space mobility product that allocates no device memory.
//
// Who needs this: code that runs where cudaMalloc is off limits -- for
// example a caller inside a host callback or a memory-pool-managed runtime
// that forbids the library from growing its own allocations after start-up,
// or an integration that must keep the device footprint fixed once the
// engine exists.  sdt_spme_mulvec_device() allocates its work buffers the
// first time it sees a larger RHS count; this entry point never does: its two
// FP32 work arrays (forces in cell order and per-particle partial sums) live
// in the fixed array below, which every GPU that loads the library holds
// until the process exits.
//
// Limits and sharing rules:
//   - npos * nrhs <= kNoAllocMaxVectors (2^18 = 262,144 particle-vectors, 6 MiB
//     of scratch); larger requests are rejected with SDT_ERR_INVALID;
//   - all calls on one GPU share the array, and it keeps whatever the last call
//     left in it.  Calls whose work overlaps on the GPU (different streams,
//     different engines on the same device) race on it and must be ordered by
//     the caller;
//   - nothing in the array needs to start at zero: each call writes every
//     element it later reads (all forces, and one partial sum per particle,
//     RHS and component) before reading it;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress, once per device with that device current; make
//     that first call before any stream capture.  The address is kept with
//     the CUDA context it belongs to: after cudaDeviceReset (a new primary
//     context) the next call looks it up again, so that call too must come
//     before any stream capture;
//   - the product always walks the cell list on the fly, also when the engine
//     holds a stored real-space pair list (the stored-list product needs a
//     larger force layout than the fixed array is sized for), so it runs
//     slower than sdt_spme_mulvec_device(SDT_MOB_REAL) on such an engine;
//   - d_f == d_v (in place) is allowed when ldf == ldv.
#include <cuda.h>

#include <mutex>

#include "../../include/stokesdt_b200.h"
#include "handles.h"

namespace sdt {

constexpr long long kNoAllocMaxVectors = 1LL << 18;
constexpr size_t kNoAllocFloats = (size_t)2 * 3 * kNoAllocMaxVectors;
constexpr int kNoAllocMaxDevices = 64;

// In host code this name is only a stand-in for the device array: never pass
// it to a kernel; use the address from cudaGetSymbolAddress instead.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

static std::mutex g_noalloc_mutex;
static float *g_noalloc_ptr[kNoAllocMaxDevices] = {};
static CUcontext g_noalloc_ctx[kNoAllocMaxDevices] = {};

// The CUDA context current on this thread (driver entry point, so the library
// needs no link-time dependency on libcuda).
static CUcontext current_context()
{
    using Fn = CUresult (*)(CUcontext *);
    static Fn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<Fn>(p);
        cudaGetLastError();
        return static_cast<Fn>(nullptr);
    }();
    CUcontext ctx = nullptr;
    if (fn && fn(&ctx) != CUDA_SUCCESS) ctx = nullptr;
    return ctx;
}

// Device address of the scratch array on `device` (current device), looked
// up again when the context has changed since the last lookup.
static int noalloc_scratch(int device, float **out)
{
    if (device < 0 || device >= kNoAllocMaxDevices) return kErrInvalid;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    const CUcontext ctx = current_context();
    if (!g_noalloc_ptr[device] || !ctx || ctx != g_noalloc_ctx[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            g_noalloc_ptr[device] = nullptr;
            return kErrCuda;
        }
        g_noalloc_ptr[device] = static_cast<float *>(p);
        g_noalloc_ctx[device] = ctx;
    }
    *out = g_noalloc_ptr[device];
    return kOk;
}

// FP64 caller forces -> FP32 [s][r][c] in real-space cell order.
__global__ void k_noalloc_gather(int n, int nr, const double *__restrict__ f, int ldf,
                                 const int *__restrict__ rs_perm, float *__restrict__ fs)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)n * nr) return;
    const int s = (int)(idx % n);
    const int r = (int)(idx / n);
    const int q = rs_perm[s];
    for (int c = 0; c < 3; c++)
        fs[((size_t)s * nr + r) * 3 + c] = (float)f[(size_t)r * ldf + 3 * q + c];
}

// v := alpha * (real + self * f) + beta * v in FP64 (beta == 0 ignores v).
// f and v may be the same array (ldf == ldv): each element is read and then
// written by one thread only, so they are not declared __restrict__.
__global__ void k_noalloc_combine(int n3, int nr, double alpha, double beta, const double *f, int ldf,
                                  const double *__restrict__ self, const float *__restrict__ vreal,
                                  double *v, int ldv)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)n3 * nr) return;
    const int e = (int)(idx % n3);
    const int r = (int)(idx / n3);
    const double acc = (double)vreal[(size_t)r * n3 + e] + self[e / 3] * f[(size_t)r * ldf + e];
    double *out = v + (size_t)r * ldv + e;
    *out = (beta == 0.0 ? 0.0 : beta * *out) + alpha * acc;
}

}  // namespace sdt

extern "C" int sdt_spme_real_mulvec_noalloc(sdt_spme *h, int nrhs, double alpha, int ldf,
                                            const double *d_f, double beta, int ldv, double *d_v)
{
    if (!h) return SDT_ERR_INVALID;
    sdt::SpmeEngine *e = &h->e;
    if (!e->updated) {
        e->last_error = "Update() must be called before the product";
        return SDT_ERR_STATE;
    }
    if (nrhs < 0) {
        e->last_error = "nrhs < 0";
        return SDT_ERR_INVALID;
    }
    if (nrhs == 0) return SDT_OK;
    const int n = e->npos, n3 = 3 * n;
    if (!d_f || !d_v || ldf < n3 || ldv < n3) {
        e->last_error = "null vector pointer or leading dimension < 3*npos";
        return SDT_ERR_INVALID;
    }
    if ((long long)n * nrhs > sdt::kNoAllocMaxVectors) {
        e->last_error = "npos * nrhs exceeds the 262144 particle-vectors of the fixed scratch array";
        return SDT_ERR_INVALID;
    }
    if (cudaSetDevice(e->device) != cudaSuccess) {
        cudaGetLastError();
        e->last_error = "cudaSetDevice failed";
        return SDT_ERR_CUDA;
    }
    float *scratch = nullptr;
    if (sdt::noalloc_scratch(e->device, &scratch) != sdt::kOk) {
        e->last_error = "cudaGetSymbolAddress of the scratch array failed";
        return SDT_ERR_CUDA;
    }
    float *fs = scratch;                                   // [n][nrhs][3]
    float *vreal = scratch + (size_t)3 * sdt::kNoAllocMaxVectors;  // [nrhs][3n]
    const int bs = 256;
    const long long work = (long long)n * nrhs;
    sdt::k_noalloc_gather<<<(int)((work + bs - 1) / bs), bs, 0, e->stream>>>(n, nrhs, d_f, ldf,
                                                                              e->d_rs_perm, fs);
    sdt::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) {
        e->last_error = "gather launch failed";
        return SDT_ERR_CUDA;
    }
    int st = sdt::real_space_launch_into(e, nrhs, fs, vreal);
    if (st != sdt::kOk) return st;
    const long long work3 = (long long)n3 * nrhs;
    sdt::k_noalloc_combine<<<(int)((work3 + bs - 1) / bs), bs, 0, e->stream>>>(
        n3, nrhs, alpha, beta, d_f, ldf, e->d_self, vreal, d_v, ldv);
    sdt::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) {
        e->last_error = "combine launch failed";
        return SDT_ERR_CUDA;
    }
    return SDT_OK;
}
