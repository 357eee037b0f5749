// Batched block Lanczos sqrt(M_s) Z_s over many systems in lockstep (the
// packed path of packed.h), FP64.
//
// Per system s the recurrence is that of lanczos.cu (BrwnLanczos::BlockLanczos,
// src/brwn/brwn_lanczos.cc:85-201, with full reorthogonalisation):
//   W = M V_i - V_{i-1} B_{i-1}^T ; A_i = V_i^T W ; W -= V_i A_i ;
//   W -= V_{0..i} (V_{0..i}^T W) ; W = V_{i+1} B_i (Cholesky QR, twice) ;
//   D_i = sqrt(T_i)[:, :k] R_0 on the host ; converged when
//   ||D_i - [D_{i-1}; 0]||_F / ||Z||_F < tol ; Y = V_{0..i} D_i at the end.
// Every step is one launch over all active systems: the products through
// packed_mulvec, the dense steps through the kernels below, whose CTAs find
// their system through a per-CTA (slot, row block) map.  One copy per
// iteration brings every system's [A_i | B_i | flag] to the host, where the
// checks of iteration i - 1 run on worker threads while the GPU runs
// iteration i; a system whose check passes leaves the active set.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "lanczos_dev.cuh"
#include "packed.h"
#include "packed_lanczos.h"

namespace sdt {

int sqrt_first_cols(int m, int k, const double *T, double *S, int *neg, const std::atomic<bool> *cancel);
int sqrt_first_cols_quad(int m, int k, const double *T, double *S, int nthreads);

namespace {

constexpr int kBlGramRows = 2048;  // rows per CTA of the Gram kernel
constexpr int kBlGemmRows = 256;   // rows per CTA of the GEMM kernel (one per thread)
constexpr int kBlCChunk = 64;      // rows of the coefficient matrix staged at a time

enum BlMat { kBlHistA = 0, kBlCoef = 1, kBlRi = 2, kBlBt = 3, kBlSmall = 4 };

__device__ __forceinline__ double *bl_mat(const BLSys &S, int kind, int it, int k, int hs)
{
    switch (kind) {
        case kBlHistA: return S.hist + (size_t)it * hs;
        case kBlCoef: return S.coef;
        case kBlRi: return S.qr;
        case kBlBt: return S.qr + 2 * k * k;
        default: return S.small;
    }
}

// part[cta][a][b] = sum over the CTA's rows e of A[a][e] B[b][e], with
// A = V + acol * ld (ma columns) and B = V + bcol * ld (mb columns) of the
// CTA's system; a in [16 blockIdx.y, +16), b in [16 blockIdx.z, +16).
__global__ void __launch_bounds__(256)
k_bl_gram_part(const BLSys *__restrict__ sys, const int *__restrict__ act, const int2 *__restrict__ map,
               int acol, int ma, int bcol, int mb, double *__restrict__ part)
{
    __shared__ double sa[16][33];
    __shared__ double sb[16][33];
    const int2 m = map[blockIdx.x];
    const BLSys &S = sys[act[m.x]];
    const int a0 = blockIdx.y * 16, b0 = blockIdx.z * 16;
    const int ta = threadIdx.x / 16, tb = threadIdx.x % 16;
    const int e0 = m.y * kBlGramRows, e1 = min(S.n, e0 + kBlGramRows);
    const double *A = S.V + (size_t)acol * S.ld, *B = S.V + (size_t)bcol * S.ld;
    double acc = 0.0;
    for (int eb = e0; eb < e1; eb += 32) {
        for (int t = threadIdx.x; t < 16 * 32; t += 256) {
            const int r = t / 32, c = t % 32;
            const int e = eb + c;
            sa[r][c] = (a0 + r < ma && e < e1) ? A[(size_t)(a0 + r) * S.ld + e] : 0.0;
            sb[r][c] = (b0 + r < mb && e < e1) ? B[(size_t)(b0 + r) * S.ld + e] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int c = 0; c < 32; c++) acc = fma(sa[ta][c], sb[tb][c], acc);
        __syncthreads();
    }
    if (a0 + ta < ma && b0 + tb < mb) part[((size_t)blockIdx.x * ma + a0 + ta) * mb + b0 + tb] = acc;
}

// Sum of the parts of slot blockIdx.y (CTAs first[j] .. first[j+1]) into the
// system's matrix `kind`: 32 outputs per CTA, parts split over 8 warps and
// added in a fixed order.
__global__ void __launch_bounds__(256)
k_bl_reduce(const BLSys *__restrict__ sys, const int *__restrict__ act, const int *__restrict__ first, int count,
            const double *__restrict__ part, int kind, int it, int k, int hs)
{
    __shared__ double red[8][33];
    const int j = blockIdx.y;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = blockIdx.x * 32 + lane;
    const int q0 = first[j], q1 = first[j + 1];
    double acc = 0.0;
    if (x < count)
        for (int q = q0 + w; q < q1; q += 8) acc += part[(size_t)q * count + x];
    red[w][lane] = acc;
    __syncthreads();
    if (w == 0 && x < count) {
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < 8; i++) t += red[i][lane];
        bl_mat(sys[act[j]], kind, it, k, hs)[x] = t;
    }
}

// Out[b][e] = beta Out[b][e] + alpha sum_a A[a][e] C[a][b], b < mb, with
// A = V + acol * ld (ma columns; ma < 0: the system's mfin), C the system's
// matrix `kind` (row-major ma x mb), Out = V + ocol * ld (ocol >= 0) or the
// system's output y (ocol < 0).  One thread per row e; each thread reads all
// its A values before it writes, so A == Out is allowed.
__global__ void __launch_bounds__(kBlGemmRows)
k_bl_gemm(const BLSys *__restrict__ sys, const int *__restrict__ act, const int2 *__restrict__ map, int acol,
          int ma_u, int kind, int it, int k, int hs, int mb, double alpha, double beta, int ocol)
{
    __shared__ double sc[kBlCChunk * kBlMaxK];
    const int2 m = map[blockIdx.x];
    const BLSys &S = sys[act[m.x]];
    const int ma = ma_u >= 0 ? ma_u : S.mfin;
    const double *C = bl_mat(S, kind, it, k, hs);
    const int e = m.y * kBlGemmRows + threadIdx.x;
    const bool live = e < S.n;
    const double *A = S.V + (size_t)acol * S.ld;
    double acc[kBlMaxK];
#pragma unroll
    for (int b = 0; b < kBlMaxK; b++) acc[b] = 0.0;
    for (int a0 = 0; a0 < ma; a0 += kBlCChunk) {
        const int na = min(kBlCChunk, ma - a0);
        __syncthreads();
        for (int t = threadIdx.x; t < na * mb; t += kBlGemmRows) sc[t] = C[(size_t)a0 * mb + t];
        __syncthreads();
        if (live) {
            for (int a = 0; a < na; a++) {
                const double x = A[(size_t)(a0 + a) * S.ld + e];
#pragma unroll
                for (int b = 0; b < kBlMaxK; b++)
                    if (b < mb) acc[b] = fma(x, sc[a * mb + b], acc[b]);
            }
        }
    }
    if (!live) return;
    double *out = ocol >= 0 ? S.V + (size_t)ocol * S.ld : S.y;
    const int ldo = ocol >= 0 ? S.ld : S.ldy;
#pragma unroll
    for (int b = 0; b < kBlMaxK; b++) {
        if (b < mb) {
            double *o = out + (size_t)b * ldo + e;
            *o = (beta == 0.0 ? 0.0 : beta * *o) + alpha * acc[b];
        }
    }
}

// One Cholesky-QR step of every active system's Gram matrix (the system's
// small scratch), one warp per system; B_bit and the flag go to the history
// (flag slot `fslot`), B^T to the transpose scratch when bit >= 0.
__global__ void __launch_bounds__(32)
k_bl_chol(const BLSys *__restrict__ sys, const int *__restrict__ act, int k, int hs, int first, int bit, int fslot)
{
    const BLSys &S = sys[act[blockIdx.x]];
    const int kk = k * k;
    double *Ri = S.qr, *Racc = S.qr + kk, *Bt = S.qr + 2 * kk;
    double *Bout = bit >= 0 ? S.hist + (size_t)bit * hs + kk : nullptr;
    chol_qr_step_warp<kBlMaxK>(k, S.small, Ri, Racc, first, Bout, Bout ? Bt : nullptr,
                               S.hist + (size_t)fslot * hs + 2 * kk);
}

// V block 0 := Z (k columns) per system.
__global__ void __launch_bounds__(kBlGemmRows)
k_bl_load_z(const BLSys *__restrict__ sys, const int *__restrict__ act, const int2 *__restrict__ map, int k)
{
    const int2 m = map[blockIdx.x];
    const BLSys &S = sys[act[m.x]];
    const int e = m.y * kBlGemmRows + threadIdx.x;
    if (e >= S.n) return;
    for (int c = 0; c < k; c++) S.V[(size_t)c * S.ld + e] = S.z[(size_t)c * S.ldz + e];
}

}  // namespace

static int bl_error(BLState *bl, int st, const std::string &msg)
{
    bl->last_error = msg;
    return st;
}

#define BL_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t err_ = (call);                                                        \
        if (err_ != cudaSuccess)                                                          \
            return bl_error(bl, kErrCuda, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

#define BL_LAUNCH()                                                                       \
    do {                                                                                  \
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                        \
        cudaError_t err_ = cudaGetLastError();                                            \
        if (err_ != cudaSuccess)                                                          \
            return bl_error(bl, kErrCuda, std::string("batched Lanczos kernel: ") + cudaGetErrorString(err_)); \
    } while (0)

int bl_create(BLState *bl, const std::vector<int> &npos, int max_iters, int max_k, double tol, int device,
              cudaStream_t stream)
{
    if (max_k < 1 || max_k > kBlMaxK || max_iters < 1 || !(tol > 0.0))
        return bl_error(bl, kErrInvalid, "batched Lanczos: 1 <= block <= 16, max_iters >= 1, tol > 0");
    bl->device = device;
    bl->stream = stream;
    bl->nsys = (int)npos.size();
    bl->max_iters = max_iters;
    bl->max_k = max_k;
    bl->tol = tol;
    bl->hs = 2 * max_k * max_k + 1;
    BL_CUDA(cudaSetDevice(device));
    bl->h_sys.assign(bl->nsys, BLSys());
    size_t vtot = 0;
    std::vector<size_t> voff(bl->nsys);
    for (int g = 0; g < bl->nsys; g++) {
        const int n = 3 * npos[g];
        const int ld = (n + 31) / 32 * 32;
        bl->h_sys[g].n = n;
        bl->h_sys[g].ld = ld;
        voff[g] = vtot;
        vtot += (size_t)(max_iters + 1) * max_k * ld;
    }
    const size_t mmax = (size_t)(max_iters + 1) * max_k;
    const size_t per_coef = mmax * max_k, per_small = (size_t)max_k * max_k, per_qr = 3 * per_small,
                 per_hist = (size_t)(max_iters + 1) * bl->hs;
    bl->mats_stride = per_coef + per_small + per_qr + per_hist;
    bl->hist_pitch = per_hist;
    BL_CUDA(cudaMalloc(&bl->d_V, vtot * sizeof(double)));
    BL_CUDA(cudaMalloc(&bl->d_mats, (size_t)bl->nsys * bl->mats_stride * sizeof(double)));
    BL_CUDA(cudaMemsetAsync(bl->d_mats, 0, (size_t)bl->nsys * bl->mats_stride * sizeof(double), stream));
    BL_CUDA(cudaMallocHost(&bl->h_hist, (size_t)bl->nsys * per_hist * sizeof(double)));
    BL_CUDA(cudaMallocHost(&bl->h_small, (size_t)bl->nsys * (per_small + per_qr) * sizeof(double)));
    double *m = bl->d_mats;
    for (int g = 0; g < bl->nsys; g++) {
        BLSys &S = bl->h_sys[g];
        S.V = bl->d_V + voff[g];
        S.coef = m;
        S.small = m + per_coef;
        S.qr = S.small + per_small;
        S.hist = S.qr + per_qr;
        m += bl->mats_stride;
    }
    BL_CUDA(cudaMalloc(&bl->d_sys, bl->nsys * sizeof(BLSys)));
    BL_CUDA(cudaMalloc(&bl->d_act, bl->nsys * sizeof(int)));
    BL_CUDA(cudaMalloc(&bl->d_first, (bl->nsys + 1) * sizeof(int)));
    BL_CUDA(cudaMallocHost(&bl->h_stage, (bl->nsys * 2 + 2) * sizeof(int)));
    // per-CTA maps: gram (kBlGramRows rows) and gemm (kBlGemmRows rows)
    size_t ng = 0, nm = 0;
    for (int g = 0; g < bl->nsys; g++) {
        ng += (bl->h_sys[g].n + kBlGramRows - 1) / kBlGramRows;
        nm += (bl->h_sys[g].n + kBlGemmRows - 1) / kBlGemmRows;
    }
    bl->map_cap = ng + nm;
    BL_CUDA(cudaMalloc(&bl->d_map, bl->map_cap * sizeof(int2)));
    BL_CUDA(cudaMallocHost(&bl->h_map, bl->map_cap * sizeof(int2)));
    bl->part_cap = ng * mmax * max_k;
    BL_CUDA(cudaMalloc(&bl->d_part, bl->part_cap * sizeof(double)));
    bl->ev.assign(max_iters + 1, nullptr);
    for (cudaEvent_t &e : bl->ev) BL_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    BL_CUDA(cudaEventCreateWithFlags(&bl->ev_map, cudaEventDisableTiming));
    BL_CUDA(cudaEventRecord(bl->ev_map, stream));
    BL_CUDA(cudaStreamSynchronize(stream));
    return kOk;
}

void bl_free(BLState *bl)
{
    if (!bl) return;
    cudaSetDevice(bl->device);
    if (bl->stream) cudaStreamSynchronize(bl->stream);
    cudaFree(bl->d_V);
    cudaFree(bl->d_mats);
    cudaFreeHost(bl->h_hist);
    cudaFreeHost(bl->h_small);
    cudaFree(bl->d_sys);
    cudaFree(bl->d_act);
    cudaFree(bl->d_first);
    cudaFreeHost(bl->h_stage);
    cudaFree(bl->d_map);
    cudaFreeHost(bl->h_map);
    cudaFree(bl->d_part);
    for (cudaEvent_t e : bl->ev)
        if (e) cudaEventDestroy(e);
    if (bl->ev_map) cudaEventDestroy(bl->ev_map);
    *bl = BLState();
}

// Maps for the active list `act`: gram CTAs (with per-slot prefix `first`),
// then gemm CTAs.  The pinned staging is rewritten only after the previous
// upload out of it has run.
static int bl_set_active(BLState *bl, const std::vector<int> &act)
{
    BL_CUDA(cudaEventSynchronize(bl->ev_map));
    int *first = bl->h_stage;          // [nact + 1]
    int *acth = bl->h_stage + bl->nsys + 1;
    int2 *mp = bl->h_map;
    size_t q = 0;
    first[0] = 0;
    for (size_t j = 0; j < act.size(); j++) {
        const int n = bl->h_sys[act[j]].n;
        for (int b = 0; b < (n + kBlGramRows - 1) / kBlGramRows; b++) mp[q++] = make_int2((int)j, b);
        first[j + 1] = (int)q;
        acth[j] = act[j];
    }
    bl->ngram = (int)q;
    for (size_t j = 0; j < act.size(); j++) {
        const int n = bl->h_sys[act[j]].n;
        for (int b = 0; b < (n + kBlGemmRows - 1) / kBlGemmRows; b++) mp[q++] = make_int2((int)j, b);
    }
    bl->ngemm = (int)q - bl->ngram;
    bl->nact = (int)act.size();
    if (act.empty()) return kOk;
    BL_CUDA(cudaMemcpyAsync(bl->d_map, mp, q * sizeof(int2), cudaMemcpyHostToDevice, bl->stream));
    BL_CUDA(cudaMemcpyAsync(bl->d_first, first, (act.size() + 1) * sizeof(int), cudaMemcpyHostToDevice, bl->stream));
    BL_CUDA(cudaMemcpyAsync(bl->d_act, acth, act.size() * sizeof(int), cudaMemcpyHostToDevice, bl->stream));
    BL_CUDA(cudaEventRecord(bl->ev_map, bl->stream));
    return kOk;
}

// Gram of columns [acol, acol+ma) and [bcol, bcol+mb) of every active system
// into matrix `kind` (iteration `it` for the history).
static int bl_gram(BLState *bl, int acol, int ma, int bcol, int mb, int kind, int it, int k)
{
    if (bl->nact == 0) return kOk;
    if ((size_t)bl->ngram * ma * mb > bl->part_cap) return bl_error(bl, kErrInvalid, "Gram partials exceed the space");
    k_bl_gram_part<<<dim3(bl->ngram, (ma + 15) / 16, (mb + 15) / 16), 256, 0, bl->stream>>>(
        bl->d_sys, bl->d_act, bl->d_map, acol, ma, bcol, mb, bl->d_part);
    BL_LAUNCH();
    const int count = ma * mb;
    k_bl_reduce<<<dim3((count + 31) / 32, bl->nact), 256, 0, bl->stream>>>(bl->d_sys, bl->d_act, bl->d_first, count,
                                                                           bl->d_part, kind, it, k, bl->hs);
    BL_LAUNCH();
    return kOk;
}

static int bl_gemm(BLState *bl, int acol, int ma, int kind, int it, int k, int mb, double alpha, double beta,
                   int ocol)
{
    if (bl->nact == 0) return kOk;
    k_bl_gemm<<<bl->ngemm, kBlGemmRows, 0, bl->stream>>>(bl->d_sys, bl->d_act, bl->d_map + bl->ngram, acol, ma,
                                                         kind, it, k, bl->hs, mb, alpha, beta, ocol);
    BL_LAUNCH();
    return kOk;
}

// Cholesky QR (twice) of the k columns at `col` of every active system, in
// place; the first pass uses the Gram already in `small` when have_g0.
static int bl_chol_qr(BLState *bl, int col, int k, bool have_g0, int bit, int fslot)
{
    for (int pass = 0; pass < 2; pass++) {
        if (!(pass == 0 && have_g0)) {
            const int st = bl_gram(bl, col, k, col, k, kBlSmall, 0, k);
            if (st != kOk) return st;
        }
        k_bl_chol<<<bl->nact, 32, 0, bl->stream>>>(bl->d_sys, bl->d_act, k, bl->hs, pass == 0 ? 1 : 0,
                                                   pass == 1 ? bit : -1, fslot);
        BL_LAUNCH();
        const int st = bl_gemm(bl, col, k, kBlRi, 0, k, k, 1.0, 0.0, col);
        if (st != kOk) return st;
    }
    return kOk;
}

// Host side of one system's check at iteration i: D_i = sqrt(T_i)[:, :k] R_0.
static int bl_solve(int i, int k, int hs, const double *hist, const double *R0, std::vector<double> &D,
                    bool *breakdown)
{
    const int kk = k * k, m = (i + 1) * k;
    *breakdown = hist[(size_t)i * hs + 2 * kk] != 0.0;
    std::vector<double> T((size_t)m * m, 0.0);
    for (int b = 0; b <= i; b++) {
        const double *A = hist + (size_t)b * hs, *B = A + kk;
        for (int r = 0; r < k; r++)
            for (int c = 0; c < k; c++)
                T[(size_t)(b * k + r) * m + b * k + c] = 0.5 * (A[r * k + c] + A[c * k + r]);
        if (b < i)
            for (int r = 0; r < k; r++)
                for (int c = 0; c < k; c++) {
                    const double x = B[r * k + c];
                    T[(size_t)((b + 1) * k + r) * m + b * k + c] = x;
                    T[(size_t)(b * k + c) * m + (b + 1) * k + r] = x;
                }
    }
    std::vector<double> S((size_t)m * k, 0.0);
    int st = sqrt_first_cols_quad(m, k, T.data(), S.data(), 1);
    if (st != 0) {
        int neg = 0;
        st = sqrt_first_cols(m, k, T.data(), S.data(), &neg, nullptr);
    }
    if (st != 0) return kErrNotConverged;
    D.assign((size_t)m * k, 0.0);
    for (int r = 0; r < m; r++)
        for (int c = 0; c < k; c++) {
            double acc = 0.0;
            for (int t = 0; t <= c; t++) acc += S[(size_t)r * k + t] * R0[t * k + c];
            D[(size_t)r * k + c] = acc;
        }
    return kOk;
}

template <typename Fn>
static void parallel_for(int n, Fn &&fn)
{
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min(n, std::min(8, hw)));
    if (nt <= 1) {
        for (int i = 0; i < n; i++) fn(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&] {
            for (int i = next++; i < n; i = next++) fn(i);
        });
    for (std::thread &t : th) t.join();
}

int bl_compute(BLState *bl, PackedBatch *pb, const std::vector<int> &sel, int k, const double *const *z,
               const int *ldz, double *const *y, const int *ldy, int *iters)
{
    if (k < 1 || k > bl->max_k) return bl_error(bl, kErrInvalid, "batched Lanczos: bad block size");
    if (sel.empty()) return kOk;
    const int kk = k * k, hs = bl->hs;
    for (size_t j = 0; j < sel.size(); j++) {
        BLSys &S = bl->h_sys[sel[j]];
        if (ldz[j] < S.n || ldy[j] < S.n) return bl_error(bl, kErrInvalid, "leading dimension < 3 npos");
        S.z = z[j];
        S.ldz = ldz[j];
        S.y = y[j];
        S.ldy = ldy[j];
        S.mfin = 0;
    }
    BL_CUDA(cudaMemcpyAsync(bl->d_sys, bl->h_sys.data(), bl->nsys * sizeof(BLSys), cudaMemcpyHostToDevice,
                            bl->stream));
    int st = bl_set_active(bl, sel);
    if (st != kOk) return st;
    k_bl_load_z<<<bl->ngemm, kBlGemmRows, 0, bl->stream>>>(bl->d_sys, bl->d_act, bl->d_map + bl->ngram, k);
    BL_LAUNCH();
    // ||Z_s||_F from Z^T Z, the first Gram matrix of the QR
    st = bl_gram(bl, 0, k, 0, k, kBlSmall, 0, k);
    if (st != kOk) return st;
    struct SysState {
        double normz = 0.0;
        std::vector<double> R0, D, Dprev;
        int done = -1;
        bool conv = false;
        int status = kOk;
    };
    std::vector<SysState> ss(bl->nsys);
    // every system's [small | qr] block in one strided copy
    const size_t sq = (size_t)bl->max_k * bl->max_k * 4;  // doubles of small + qr
    auto fetch_small = [&]() -> int {
        BL_CUDA(cudaMemcpy2DAsync(bl->h_small, sq * sizeof(double), bl->h_sys[0].small,
                                  bl->mats_stride * sizeof(double), sq * sizeof(double), bl->nsys,
                                  cudaMemcpyDeviceToHost, bl->stream));
        BL_CUDA(cudaStreamSynchronize(bl->stream));
        return kOk;
    };
    st = fetch_small();
    if (st != kOk) return st;
    std::vector<int> act;
    for (int g : sel) {
        const double *G = bl->h_small + (size_t)g * sq;
        double t = 0.0;
        for (int c = 0; c < k; c++) t += G[c * k + c];
        ss[g].normz = std::sqrt(t);
        if (ss[g].normz > 0.0)
            act.push_back(g);
        else
            ss[g].conv = true;  // Y = 0
    }
    if (act.size() != sel.size()) {
        st = bl_set_active(bl, act);
        if (st != kOk) return st;
    }
    // V_0 R_0 = Z (the spare history slot holds the breakdown flag); the
    // first pass uses the Gram matrices already formed
    st = bl_chol_qr(bl, 0, k, true, -1, bl->max_iters);
    if (st != kOk) return st;
    st = fetch_small();
    if (st != kOk) return st;
    for (int g : act) {
        const double *Racc = bl->h_small + (size_t)g * sq + (size_t)bl->max_k * bl->max_k + kk;
        ss[g].R0.assign(Racc, Racc + kk);
        double flag = 0.0;
        BL_CUDA(cudaMemcpy(&flag, bl->h_sys[g].hist + (size_t)bl->max_iters * hs + 2 * kk, sizeof(double),
                           cudaMemcpyDeviceToHost));
        if (flag != 0.0) return bl_error(bl, kErrInvalid, "a random block is rank deficient");
    }
    std::vector<std::vector<int>> act_at(bl->max_iters);
    std::vector<const double *> fp;
    std::vector<double *> vp;
    std::vector<int> ldp;
    // checks of iteration i for the systems that ran it
    using Clock = std::chrono::steady_clock;
    auto ms_since = [](Clock::time_point t) {
        return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
    };
    const bool trace = std::getenv("STOKESDT_LANCZOS_TRACE") != nullptr;
    const Clock::time_point t_start = Clock::now();
    double t_wait = 0.0, t_solve = 0.0;
    auto check = [&](int i) -> int {
        Clock::time_point tw = Clock::now();
        BL_CUDA(cudaEventSynchronize(bl->ev[i]));
        t_wait += ms_since(tw);
        tw = Clock::now();
        const std::vector<int> &ran = act_at[i];
        parallel_for((int)ran.size(), [&](int j) {
            const int g = ran[j];
            SysState &x = ss[g];
            if (x.conv) return;
            bool breakdown = false;
            std::vector<double> D;
            const int s2 = bl_solve(i, k, hs, bl->h_hist + (size_t)g * bl->hist_pitch, x.R0.data(), D, &breakdown);
            if (s2 != kOk) {
                x.status = s2;
                return;
            }
            x.done = i;
            if (i > 0) {
                const int m = (i + 1) * k;
                double diff2 = 0.0;
                for (int r = 0; r < m; r++)
                    for (int c = 0; c < k; c++) {
                        const double prev = (r < m - k) ? x.Dprev[(size_t)r * k + c] : 0.0;
                        const double d = D[(size_t)r * k + c] - prev;
                        diff2 += d * d;
                    }
                if (std::sqrt(diff2) / x.normz < bl->tol) x.conv = true;
            }
            if (breakdown) x.conv = true;
            x.Dprev = D;
            x.D = std::move(D);
        });
        t_solve += ms_since(tw);
        for (int g : ran)
            if (ss[g].status != kOk) return bl_error(bl, ss[g].status, "tridiagonal eigensolver did not converge");
        return kOk;
    };
    // with the trace on, CUDA events bracket the phases of every iteration
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
    auto mark = [&](int phase) -> cudaEvent_t {
        if (!trace) return nullptr;
        cudaEvent_t a = nullptr, b2 = nullptr;
        cudaEventCreate(&a);
        cudaEventCreate(&b2);
        cudaEventRecord(a, bl->stream);
        marks.push_back({phase, {a, b2}});
        return b2;
    };
    auto mark_end = [&](cudaEvent_t e) {
        if (e) cudaEventRecord(e, bl->stream);
    };
    int it = 0;
    int last_issued = -1;
    for (it = 0; it < bl->max_iters && !act.empty(); it++) {
        act_at[it] = act;
        const int ci = it * k, cw = (it + 1) * k;
        cudaEvent_t pe = mark(0);
        if (it > 0) {
            st = bl_gemm(bl, (it - 1) * k, k, kBlBt, 0, k, k, 1.0, 0.0, cw);  // W = V_{i-1} B_{i-1}^T
            if (st != kOk) return st;
        }
        fp.clear();
        vp.clear();
        ldp.clear();
        for (int g : act) {
            const BLSys &S = bl->h_sys[g];
            fp.push_back(S.V + (size_t)ci * S.ld);
            vp.push_back(S.V + (size_t)cw * S.ld);
            ldp.push_back(S.ld);
        }
        st = packed_mulvec(pb, (int)act.size(), act.data(), k, 1.0, fp.data(), ldp.data(), it > 0 ? -1.0 : 0.0,
                           vp.data(), ldp.data());
        if (st != kOk) return bl_error(bl, st, "packed product: " + pb->last_error);
        mark_end(pe);
        pe = mark(1);
        st = bl_gram(bl, ci, k, cw, k, kBlHistA, it, k);                            // A_i = V_i^T W
        if (st == kOk) st = bl_gemm(bl, ci, k, kBlHistA, it, k, k, -1.0, 1.0, cw);  // W -= V_i A_i
        mark_end(pe);
        pe = mark(2);
        if (st == kOk) st = bl_gram(bl, 0, cw, cw, k, kBlCoef, 0, k);               // C = V_{0..i}^T W
        if (st == kOk) st = bl_gemm(bl, 0, cw, kBlCoef, 0, k, k, -1.0, 1.0, cw);    // W -= V_{0..i} C
        mark_end(pe);
        pe = mark(3);
        if (st == kOk) st = bl_chol_qr(bl, cw, k, false, it, it);                   // W = V_{i+1} B_i
        mark_end(pe);
        if (st != kOk) return st;
        BL_CUDA(cudaMemcpy2DAsync(bl->h_hist + (size_t)it * hs, bl->hist_pitch * sizeof(double),
                                  bl->h_sys[0].hist + (size_t)it * hs, bl->mats_stride * sizeof(double),
                                  (2 * kk + 1) * sizeof(double), bl->nsys, cudaMemcpyDeviceToHost, bl->stream));
        BL_CUDA(cudaEventRecord(bl->ev[it], bl->stream));
        last_issued = it;
        // the checks of the previous iteration run while this one is on the GPU
        if (it >= 1) {
            st = check(it - 1);
            if (st != kOk) return st;
            std::vector<int> next;
            for (int g : act)
                if (!ss[g].conv) next.push_back(g);
            if (next.size() != act.size()) {
                act.swap(next);
                st = bl_set_active(bl, act);
                if (st != kOk) return st;
            }
        }
    }
    if (last_issued >= 0) {
        st = check(last_issued);
        if (st != kOk) return st;
    }
    // Y = V_{0..i} D_i per system
    for (int g : sel) {
        SysState &x = ss[g];
        BLSys &S = bl->h_sys[g];
        S.mfin = x.D.empty() ? 0 : (int)(x.D.size() / k);
        if (S.mfin > 0)
            BL_CUDA(cudaMemcpyAsync(S.coef, x.D.data(), x.D.size() * sizeof(double), cudaMemcpyHostToDevice,
                                    bl->stream));
    }
    BL_CUDA(cudaMemcpyAsync(bl->d_sys, bl->h_sys.data(), bl->nsys * sizeof(BLSys), cudaMemcpyHostToDevice,
                            bl->stream));
    st = bl_set_active(bl, sel);
    if (st == kOk) st = bl_gemm(bl, 0, -1, kBlCoef, 0, k, k, 1.0, 0.0, -1);
    if (st != kOk) return st;
    // the host copies of the coefficients are read by the queued uploads
    BL_CUDA(cudaStreamSynchronize(bl->stream));
    if (trace) {
        double ph[4] = {0, 0, 0, 0};
        for (auto &m : marks) {
            float t = 0.f;
            cudaEventElapsedTime(&t, m.second.first, m.second.second);
            ph[m.first] += t;
            cudaEventDestroy(m.second.first);
            cudaEventDestroy(m.second.second);
        }
        std::fprintf(stderr, "[batched lanczos] device ms: products %.1f, recurrence %.1f, reorthogonalisation %.1f, "
                     "QR %.1f\n", ph[0], ph[1], ph[2], ph[3]);
        std::fprintf(stderr, "[batched lanczos] %zu systems, k %d: %d iterations, %.1f ms total, %.1f ms waiting on the "
                     "GPU, %.1f ms in host solves; active per iteration:", sel.size(), k, it, ms_since(t_start),
                     t_wait, t_solve);
        for (int i = 0; i < it; i++) std::fprintf(stderr, " %zu", act_at[i].size());
        std::fprintf(stderr, "\n");
    }
    int out = kOk;
    for (size_t j = 0; j < sel.size(); j++) {
        const SysState &x = ss[sel[j]];
        const bool zero = x.normz == 0.0;
        iters[j] = zero ? 0 : (x.conv ? x.done : -1);
        if (!zero && !x.conv) out = kErrNotConverged;
    }
    bl->last_iters = it;
    return out;
}

}  // namespace sdt
