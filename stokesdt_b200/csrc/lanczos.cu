// Block Lanczos sqrt(M) Z on the device, FP64 (BrwnLanczos,
// src/brwn/brwn_lanczos.cc:16-304).
//
// Per iteration i (k = block size):
//   W = M V_i - V_{i-1} B_{i-1}^T            (one batched SPME product of k RHS)
//   A_i = V_i^T W ;  W -= V_i A_i
//   optional reorthogonalisation: W -= V_{0..i} (V_{0..i}^T W)
//   W = V_{i+1} B_i                           (Cholesky QR, applied twice)
//   S = sqrt(T_i)[:, :k] ;  D_i = S R         (host FP64 eigensolver)
//   converged when ||Y_i - Y_{i-1}||_F / ||Z||_F < tol with Y_i = V_{0..i} D_i
// With reorthogonalisation V_{0..i} is orthonormal, so ||Y_i - Y_{i-1}||_F =
// ||D_i - [D_{i-1}; 0]||_F and Y is formed once, at the end; without it Y_i
// is formed on the device every iteration exactly as the reference does
// (brwn_lanczos.cc:181-196).  The QR of the reference (dgeqrf/dorgqr) and the
// Cholesky QR used here differ only by column signs, which leave Y unchanged.
// A block of one vector (k = 1) runs the same recurrence as dot products and
// axpys, the whole iteration after the product in one cooperative launch
// (k_vec_iter).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <atomic>
#include <deque>
#include <future>
#include <string>
#include <vector>

#include "engine.h"
#include "lanczos.h"
#include "lanczos_dev.cuh"

namespace sdt {

int sqrt_first_cols(int m, int k, const double *T, double *S, int *neg, const std::atomic<bool> *cancel);
int sqrt_first_cols_quad(int m, int k, const double *T, double *S, int nthreads);

#define LZ_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t err_ = (call);                                                        \
        if (err_ != cudaSuccess) {                                                        \
            lz->last_error = std::string(#call) + ": " + cudaGetErrorString(err_);        \
            return kErrCuda;                                                              \
        }                                                                                 \
    } while (0)

#define LZ_LAUNCH()                                                                       \
    do {                                                                                  \
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                        \
        cudaError_t err_ = cudaGetLastError();                                            \
        if (err_ != cudaSuccess) {                                                        \
            lz->last_error = std::string("lanczos kernel: ") + cudaGetErrorString(err_);  \
            return kErrCuda;                                                              \
        }                                                                                 \
    } while (0)

constexpr int kGramRows = 32;   // rows staged per step of the Gram kernel
constexpr int kMaxBlock = 32;   // largest supported block size k

// part[chunk][a][b] = sum over the chunk's rows e of A[a][e] * B[b][e]
// for a in [a0, a0+16), b < mb (<= 16 per blockIdx.y tile).
__global__ void __launch_bounds__(256)
k_gram_partial(int n, int ma, const double *__restrict__ A, int lda, int mb,
               const double *__restrict__ B, int ldb, int rows_per_chunk, double *__restrict__ part)
{
    __shared__ double sa[16][kGramRows + 1];
    __shared__ double sb[16][kGramRows + 1];
    const int a0 = blockIdx.y * 16, b0 = blockIdx.z * 16;
    const int ta = threadIdx.x / 16, tb = threadIdx.x % 16;
    const int e0 = blockIdx.x * rows_per_chunk;
    const int e1 = min(n, e0 + rows_per_chunk);
    double acc = 0.0;
    for (int eb = e0; eb < e1; eb += kGramRows) {
        for (int t = threadIdx.x; t < 16 * kGramRows; t += 256) {
            const int r = t / kGramRows, c = t % kGramRows;
            const int e = eb + c;
            sa[r][c] = (a0 + r < ma && e < e1) ? A[(size_t)(a0 + r) * lda + e] : 0.0;
            sb[r][c] = (b0 + r < mb && e < e1) ? B[(size_t)(b0 + r) * ldb + e] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int c = 0; c < kGramRows; c++) acc = fma(sa[ta][c], sb[tb][c], acc);
        __syncthreads();
    }
    if (a0 + ta < ma && b0 + tb < mb)
        part[((size_t)blockIdx.x * ma + a0 + ta) * mb + b0 + tb] = acc;
}

// out[x] = sum over q < nparts of part[q][x]: 32 outputs per CTA (one per
// lane, coalesced), the parts split over the 8 warps and the 8 partial sums
// added in a fixed order.
__global__ void __launch_bounds__(256)
k_reduce_parts(int nparts, int count, const double *__restrict__ part, double *__restrict__ out)
{
    __shared__ double red[8][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = blockIdx.x * 32 + lane;
    double acc = 0.0;
    if (x < count) {
#pragma unroll 4
        for (int q = w; q < nparts; q += 8) acc += part[(size_t)q * count + x];
    }
    red[w][lane] = acc;
    __syncthreads();
    if (w == 0 && x < count) {
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < 8; j++) t += red[j][lane];
        out[x] = t;
    }
}

// Out[b][e] = beta * Out[b][e] + alpha * sum_{a < ma} A[a][e] * C[a][b], b < mb <= 32.
// One thread per row e; every thread reads its A values before writing, so
// A == Out (in-place right multiplication) is allowed (hence no __restrict__
// on A).
__global__ void __launch_bounds__(256)
k_block_gemm(int n, int ma, const double *A, int lda, const double *__restrict__ C,
             int mb, double alpha, double beta, double *Out, int ldo)
{
    extern __shared__ double sc[];  // [ma][mb]
    for (int t = threadIdx.x; t < ma * mb; t += blockDim.x) sc[t] = C[t];
    __syncthreads();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double acc[kMaxBlock];
#pragma unroll
    for (int b = 0; b < kMaxBlock; b++) acc[b] = 0.0;
    for (int a = 0; a < ma; a++) {
        const double x = A[(size_t)a * lda + e];
#pragma unroll
        for (int b = 0; b < kMaxBlock; b++)
            if (b < mb) acc[b] = fma(x, sc[a * mb + b], acc[b]);
    }
#pragma unroll
    for (int b = 0; b < kMaxBlock; b++) {
        if (b < mb) {
            double *o = Out + (size_t)b * ldo + e;
            *o = (beta == 0.0 ? 0.0 : beta * *o) + alpha * acc[b];
        }
    }
}

// Register-blocked Gram for tall A (ma >= 64 rows), mb <= 16:
// part[chunk][a][b] = sum over the chunk's rows e of A[a][e] * B[b][e].
// CTA = 128 rows of A x all 16 rows of B.  Stages of 32 columns e of both are
// copied to shared memory with cp.async, double-buffered so the next stage
// is in flight while the current one is used; four groups of 64 threads take
// 8 columns each.  A thread accumulates an 8 x 4 tile (rows ag + 16 i, cols
// bg + 4 j), so each column costs it 12 shared loads for 32 FMAs; the four
// groups' tiles are summed in shared memory at the end.  Row stride 34
// doubles keeps the 16-byte copies aligned and the tile reads conflict-free.
constexpr int kGramTileA = 128;
constexpr int kGramStageE = 32;
constexpr int kGramLd = kGramStageE + 2;
constexpr int kGramStageDoubles = (kGramTileA + 16) * kGramLd;
constexpr size_t kGramSmem = 2 * kGramStageDoubles * sizeof(double);

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Copy columns [eb, eb + 32) of rows [a0, a0+128) of A and [0, 16) of B into
// one stage buffer (zero outside [0, ma) x [.., e1) and [0, mb)).  Needs lda,
// ldb and eb even (16-byte pairs).
__device__ __forceinline__ void gram_stage(double *buf, const double *A, int lda, int ma, int a0,
                                           const double *B, int ldb, int mb, int eb, int e1, int tid)
{
    constexpr int PAIRS = kGramStageE / 2;
    for (int t = tid; t < (kGramTileA + 16) * PAIRS; t += 256) {
        const int rr = t / PAIRS, c2 = (t % PAIRS) * 2;
        const int e = eb + c2;
        const double *src;
        bool valid;
        if (rr < kGramTileA) {
            valid = a0 + rr < ma;
            src = A + (size_t)(a0 + rr) * lda + e;
        } else {
            valid = rr - kGramTileA < mb;
            src = B + (size_t)(rr - kGramTileA) * ldb + e;
        }
        const int left = e1 - e;
        const int bytes = (!valid || left <= 0) ? 0 : (left >= 2 ? 16 : 8);
        cp_async16(buf + rr * kGramLd + c2, bytes ? src : A, bytes);
    }
}

__global__ void __launch_bounds__(256, 2)
k_gram_tall(int n, int ma, const double *__restrict__ A, int lda, int mb,
            const double *__restrict__ B, int ldb, int rows_per_chunk, double *__restrict__ part)
{
    extern __shared__ __align__(16) double gsm[];  // 2 stages of [(128 + 16)][kGramLd]
    const int a0 = blockIdx.y * kGramTileA;
    const int tid = threadIdx.x;
    const int grp = tid >> 6, t64 = tid & 63, ag = t64 >> 2, bg = t64 & 3;
    const int e0 = blockIdx.x * rows_per_chunk;
    const int e1 = min(n, e0 + rows_per_chunk);
    double acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
    const int nst = (e1 - e0 + kGramStageE - 1) / kGramStageE;
    if (nst > 0) gram_stage(gsm, A, lda, ma, a0, B, ldb, mb, e0, e1, tid);
    cp_async_commit();
    for (int st = 0; st < nst; st++) {
        if (st + 1 < nst)
            gram_stage(gsm + ((st + 1) & 1) * kGramStageDoubles, A, lda, ma, a0, B, ldb, mb,
                       e0 + (st + 1) * kGramStageE, e1, tid);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const double *sA = gsm + (st & 1) * kGramStageDoubles;
        const double *sB = sA + kGramTileA * kGramLd;
#pragma unroll
        for (int c = 0; c < kGramStageE / 4; c++) {
            const int e = grp * (kGramStageE / 4) + c;
            double av[8], bv[4];
#pragma unroll
            for (int i = 0; i < 8; i++) av[i] = sA[(ag + 16 * i) * kGramLd + e];
#pragma unroll
            for (int j = 0; j < 4; j++) bv[j] = sB[(bg + 4 * j) * kGramLd + e];
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();
    // sum the four groups' tiles (stage buffer 0 reused as a 128 x 16 tile)
    double *red = gsm;
    for (int g = 0; g < 4; g++) {
        if (grp == g) {
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int idx = (ag + 16 * i) * 16 + bg + 4 * j;
                    red[idx] = (g == 0 ? 0.0 : red[idx]) + acc[i][j];
                }
        }
        __syncthreads();
    }
    for (int t = tid; t < kGramTileA * 16; t += 256) {
        const int r = t / 16, b = t % 16;
        if (a0 + r < ma && b < mb) part[((size_t)blockIdx.x * ma + a0 + r) * mb + b] = red[t];
    }
}

// Register-blocked Gram of two short blocks (mb <= 16; A in tiles of 16
// rows, one per blockIdx.y, so ma <= 16 * gridDim.y):
// part[chunk][a][b] = sum over the chunk's rows e of A[a][e] * B[b][e].
// Stages of 64 columns e of both blocks go to shared memory by cp.async,
// double-buffered; the 16 thread groups take 4 columns of a stage each and a
// thread accumulates a 4 x 4 tile (16 shared loads for 64 FMAs); the groups'
// tiles are summed in shared memory at the end.  Needs lda, ldb and the
// block starts 16-byte aligned.
//
// With `arrive` set (ma * mb small), the last CTA to finish also sums the
// parts into out[ma * mb], in the order k_reduce_parts uses (so the result
// is the same to the bit), and resets the counter for the next call.
constexpr int kSmallStageE = 64;
constexpr int kSmallLd = kSmallStageE + 2;

__global__ void __launch_bounds__(256)
k_gram_small(int n, int ma, const double *__restrict__ A, int lda, int mb, const double *__restrict__ B, int ldb,
             int rows_per_chunk, double *__restrict__ part, unsigned *__restrict__ arrive, double *__restrict__ out)
{
    __shared__ __align__(16) double st[2][32][kSmallLd];
    const int tid = threadIdx.x;
    const int a0 = blockIdx.y * 16;
    const int grp = tid >> 4, t16 = tid & 15, ai = (t16 >> 2) * 4, bi = (t16 & 3) * 4;
    const int e0 = blockIdx.x * rows_per_chunk;
    const int e1 = min(n, e0 + rows_per_chunk);
    auto stage = [&](int buf, int eb) {
        constexpr int PAIRS = kSmallStageE / 2;
        for (int q = tid; q < 32 * PAIRS; q += 256) {
            const int rr = q / PAIRS, c2 = (q % PAIRS) * 2;
            const int e = eb + c2;
            const bool isa = rr < 16;
            const int row = isa ? rr : rr - 16;
            const bool valid = isa ? a0 + row < ma : row < mb;
            const double *src = isa ? A + (size_t)(a0 + row) * lda + e : B + (size_t)row * ldb + e;
            const int left = e1 - e;
            const int bytes = (!valid || left <= 0) ? 0 : (left >= 2 ? 16 : 8);
            cp_async16(&st[buf][rr][c2], bytes ? src : A, bytes);
        }
    };
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
    const int nst = (e1 - e0 + kSmallStageE - 1) / kSmallStageE;
    if (nst > 0) stage(0, e0);
    cp_async_commit();
    for (int sg = 0; sg < nst; sg++) {
        if (sg + 1 < nst) stage((sg + 1) & 1, e0 + (sg + 1) * kSmallStageE);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int buf = sg & 1;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int e = grp * 4 + c;
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) av[i] = st[buf][ai + i][e];
#pragma unroll
            for (int j = 0; j < 4; j++) bv[j] = st[buf][16 + bi + j][e];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();
    // sum the 16 groups' tiles in a fixed order (the stage buffers reused)
    double *red = &st[0][0][0];  // [16 groups][256]
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) red[grp * 256 + (ai + i) * 16 + bi + j] = acc[i][j];
    __syncthreads();
    const int a = tid / 16, b = tid % 16;
    if (a0 + a < ma && b < mb) {
        double t = 0.0;
        for (int g = 0; g < 16; g++) t += red[g * 256 + tid];
        part[((size_t)blockIdx.x * ma + a0 + a) * mb + b] = t;
    }
    if (arrive == nullptr) return;
    __shared__ unsigned last;
    __threadfence();  // this CTA's parts are visible before it is counted
    __syncthreads();
    if (tid == 0) last = atomicAdd(arrive, 1u) == gridDim.x * gridDim.y - 1 ? 1u : 0u;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int count = ma * mb, nparts = gridDim.x;
    const int lane = tid & 31, w = tid >> 5;
    for (int x0 = 0; x0 < count; x0 += 32) {
        const int x = x0 + lane;
        double acc = 0.0;
        if (x < count)
            for (int q = w; q < nparts; q += 8) acc += __ldcg(&part[(size_t)q * count + x]);
        red[w * 33 + lane] = acc;
        __syncthreads();
        if (w == 0 && x < count) {
            double t = 0.0;
#pragma unroll
            for (int j = 0; j < 8; j++) t += red[j * 33 + lane];
            out[x] = t;
        }
        __syncthreads();
    }
    if (tid == 0) *arrive = 0u;
}

// Out[b][e] = beta * Out[b][e] + alpha * sum_{a < ma} A[a][e] * C[a][b] for
// mb <= 16: each thread owns two rows e (e and e + 256); C is staged in
// shared memory 64 rows at a time (zero-padded to 16 columns) and read as
// broadcast double2; the A loads of 8 rows are issued before their FMAs.
// Each thread reads its A values before it writes, so A == Out is allowed.
constexpr int kGemmChunk = 64;

__global__ void __launch_bounds__(256, 2)
k_gemm_tall(int n, int ma, const double *A, int lda, const double *__restrict__ C, int mb,
            double alpha, double beta, double *Out, int ldo)
{
    __shared__ __align__(16) double sc[kGemmChunk * 16];
    const int e0 = blockIdx.x * 512 + threadIdx.x, e1 = e0 + 256;
    const bool v0 = e0 < n, v1 = e1 < n;
    double acc0[16], acc1[16];
#pragma unroll
    for (int b = 0; b < 16; b++) acc0[b] = acc1[b] = 0.0;
    for (int c0 = 0; c0 < ma; c0 += kGemmChunk) {
        const int na = min(kGemmChunk, ma - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < kGemmChunk * 16; t += 256) {
            const int a = t / 16, b = t % 16;
            sc[t] = (a < na && b < mb) ? C[(size_t)(c0 + a) * mb + b] : 0.0;
        }
        __syncthreads();
        int a = 0;
        for (; a + 8 <= na; a += 8) {
            double x0[8], x1[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const double *row = A + (size_t)(c0 + a + u) * lda;
                x0[u] = v0 ? row[e0] : 0.0;
                x1[u] = v1 ? row[e1] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const double2 *cr = reinterpret_cast<const double2 *>(sc + (a + u) * 16);
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const double2 cc = cr[q];
                    acc0[2 * q] = fma(x0[u], cc.x, acc0[2 * q]);
                    acc0[2 * q + 1] = fma(x0[u], cc.y, acc0[2 * q + 1]);
                    acc1[2 * q] = fma(x1[u], cc.x, acc1[2 * q]);
                    acc1[2 * q + 1] = fma(x1[u], cc.y, acc1[2 * q + 1]);
                }
            }
        }
        for (; a < na; a++) {
            const double *row = A + (size_t)(c0 + a) * lda;
            const double x0 = v0 ? row[e0] : 0.0;
            const double x1 = v1 ? row[e1] : 0.0;
            const double2 *cr = reinterpret_cast<const double2 *>(sc + a * 16);
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const double2 cc = cr[q];
                acc0[2 * q] = fma(x0, cc.x, acc0[2 * q]);
                acc0[2 * q + 1] = fma(x0, cc.y, acc0[2 * q + 1]);
                acc1[2 * q] = fma(x1, cc.x, acc1[2 * q]);
                acc1[2 * q + 1] = fma(x1, cc.y, acc1[2 * q + 1]);
            }
        }
    }
#pragma unroll
    for (int b = 0; b < 16; b++) {
        if (b < mb) {
            if (v0) {
                double *o = Out + (size_t)b * ldo + e0;
                *o = (beta == 0.0 ? 0.0 : beta * *o) + alpha * acc0[b];
            }
            if (v1) {
                double *o = Out + (size_t)b * ldo + e1;
                *o = (beta == 0.0 ? 0.0 : beta * *o) + alpha * acc1[b];
            }
        }
    }
}

// Frobenius norm squared partials of an (mb x n) block (ld).
__global__ void k_sqnorm_partial(int n, int mb, const double *__restrict__ X, int ld,
                                 double *__restrict__ part)
{
    __shared__ double red[256];
    double s = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * mb;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / n), e = (int)(t % n);
        const double v = X[(size_t)b * ld + e];
        s = fma(v, v, s);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// ---------------------------------------------------------------------------
// Single-vector iteration (k = 1).  With one RHS every Gram matrix is a dot
// product, every block product an axpy and the Cholesky QR a normalisation
// (one pass: the second pass of a one-column Cholesky QR divides by
// 1 + O(eps)).  By default an iteration's work after the mobility product
// is one cooperative launch, k_vec_iter (below); the four-launch form over
// row chunks of `rows` (<= kVecMaxRows, one CTA each) is the fallback where
// a cooperative launch is not available (and STOKESDT_VEC_UNFUSED=1):
//   k_vec_dot          A_i = V_i . W
//   k_vec_axpy_dots    W -= A_i V_i ; c = V_{0..i}^T W      (reorthogonalised)
//   k_vec_axpy_norm    W -= A_i V_i ; g = W . W             (without)
//   k_vec_sub_norm     W -= V_{0..i} c ; g = W . W
//   k_vec_scale        V_{i+1} = W / sqrt(g) ; next W = B_i V_i
// Either way the block path's eleven launches per iteration are gone.
// Cross-CTA sums of the four-launch form: every CTA writes its partial sums
// and the last CTA to arrive adds them in a fixed order, so the results do
// not depend on scheduling.
constexpr int kVecThreads = 512;
constexpr int kVecWarps = kVecThreads / 32;
constexpr int kVecMaxRows = 2048;

// Sum of v over the CTA, valid in thread 0; `red` holds kVecWarps doubles
// and is free again once every thread has returned.
__device__ __forceinline__ double vec_cta_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
#pragma unroll
        for (int w = 0; w < kVecWarps; w++) t += red[w];
    return t;
}

// True in every thread of the last CTA to arrive (all CTAs' partial sums
// are visible to it then).  That CTA resets the counter when it is done.
__device__ __forceinline__ bool vec_last_cta(unsigned *arrive)
{
    __shared__ unsigned last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(arrive, 1u) == gridDim.x - 1 ? 1u : 0u;
    __syncthreads();
    if (last) __threadfence();
    return last != 0;
}

// out[j] = sum over CTAs q of part[q * ncol + j], by the whole CTA: up to
// 32 threads per column take the CTAs q = g, g + groups, .. (eight loads in
// flight each), and their sums are added in group order through `red`
// (kVecThreads doubles).  Thread j < ncol stores out[j] (thread 0 for one
// column).
__device__ __forceinline__ void vec_fold(int ncol, const double *part, double *out, double *red)
{
    const int G = gridDim.x, t = threadIdx.x;
    for (int j0 = 0; j0 < ncol; j0 += kVecThreads) {
        const int nc = min(kVecThreads, ncol - j0);
        const int groups = min(32, kVecThreads / nc);
        const int j = t % nc, g = t / nc;
        double s = 0.0;
        if (g < groups) {
#pragma unroll 8
            for (int q = g; q < G; q += groups) s += __ldcg(&part[(size_t)q * ncol + j0 + j]);
        }
        red[t] = s;
        __syncthreads();
        if (t < nc) {
            double a = 0.0;
            for (int gg = 0; gg < groups; gg++) a += red[gg * nc + t];
            out[j0 + t] = a;
        }
        __syncthreads();
    }
}

// The last CTA's normalisation factor from g = ||W||^2: B = sqrt(g) and
// 1/B; a g that is not positive is a breakdown (flag 1, and 1/B = 0 so the
// vector becomes zero and stays finite), as in chol_qr_step_warp.
__device__ __forceinline__ void vec_norm_fold(const double *part, double *B, double *ri, double *flag, double *red)
{
    double d = 0.0;
    vec_fold(1, part, &d, red);  // the sum lands in thread 0
    if (threadIdx.x != 0) return;
    if (!(d > 0.0)) {
        *ri = 0.0;
        *B = 0.0;
        *flag = 1.0;
    } else {
        const double r = sqrt(d);
        *B = r;
        *ri = 1.0 / r;
        *flag = 0.0;
    }
}

__global__ void __launch_bounds__(kVecThreads)
k_vec_dot(int n, int rows, const double *__restrict__ x, const double *__restrict__ y, double *__restrict__ part,
          unsigned *__restrict__ arrive, double *__restrict__ out)
{
    __shared__ double red[kVecThreads];
    const int e0 = blockIdx.x * rows, e1 = min(n, e0 + rows);
    double s = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += kVecThreads) s = fma(x[e], y[e], s);
    s = vec_cta_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
    if (!vec_last_cta(arrive)) return;
    vec_fold(1, part, out, red);
    if (threadIdx.x == 0) *arrive = 0u;
}

// W -= a V_i (a = *pa, V_i = V + (ma - 1) ldv); c[j] = V_j . W for j < ma.
// The CTA keeps its chunk of the new W in shared memory; warp w takes the
// columns 4w..4w+3, 4w+4 kVecWarps.. (four at a time) with the lanes over
// the rows, four rows a lane at once (sixteen loads in flight).
__global__ void __launch_bounds__(kVecThreads)
k_vec_axpy_dots(int n, int rows, int ma, const double *__restrict__ V, int ldv, const double *__restrict__ pa,
                double *__restrict__ W, double *__restrict__ part, unsigned *__restrict__ arrive,
                double *__restrict__ c)
{
    __shared__ double sw[kVecMaxRows];
    const int e0 = blockIdx.x * rows, len = min(n, e0 + rows) - e0;
    const double a = *pa;
    const double *Vi = V + (size_t)(ma - 1) * ldv + e0;
    for (int r = threadIdx.x; r < len; r += kVecThreads) {
        const double w = fma(-a, Vi[r], W[e0 + r]);
        W[e0 + r] = w;
        sw[r] = w;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    for (int j0 = 4 * wp; j0 < ma; j0 += 4 * kVecWarps) {
        double s[4] = {0.0, 0.0, 0.0, 0.0};
        const double *Vj = V + (size_t)j0 * ldv + e0;
        const int nq = min(4, ma - j0);
        int r = lane;
        for (; r + 96 < len; r += 128) {
            double w[4], v[4][4];
#pragma unroll
            for (int u = 0; u < 4; u++) w[u] = sw[r + 32 * u];
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int u = 0; u < 4; u++) v[q][u] = q < nq ? Vj[(size_t)q * ldv + r + 32 * u] : 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int u = 0; u < 4; u++) s[q] = fma(v[q][u], w[u], s[q]);
        }
        for (; r < len; r += 32) {
            const double w = sw[r];
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (q < nq) s[q] = fma(Vj[(size_t)q * ldv + r], w, s[q]);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
            if (lane == 0 && q < nq) part[(size_t)blockIdx.x * ma + j0 + q] = s[q];
        }
    }
    if (!vec_last_cta(arrive)) return;
    vec_fold(ma, part, c, sw);
    if (threadIdx.x == 0) *arrive = 0u;
}

// W -= a V_i (a = *pa); B = ||W||, 1/B and the breakdown flag.
__global__ void __launch_bounds__(kVecThreads)
k_vec_axpy_norm(int n, int rows, const double *__restrict__ Vi, const double *__restrict__ pa,
                double *__restrict__ W, double *__restrict__ part, unsigned *__restrict__ arrive,
                double *__restrict__ B, double *__restrict__ ri, double *__restrict__ flag)
{
    __shared__ double red[kVecThreads];
    const int e0 = blockIdx.x * rows, e1 = min(n, e0 + rows);
    const double a = *pa;
    double s = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += kVecThreads) {
        const double w = fma(-a, Vi[e], W[e]);
        W[e] = w;
        s = fma(w, w, s);
    }
    s = vec_cta_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
    if (!vec_last_cta(arrive)) return;
    vec_norm_fold(part, B, ri, flag, red);
    if (threadIdx.x == 0) *arrive = 0u;
}

// W -= sum_{j < ma} V_j c[j]; B = ||W||, 1/B and the breakdown flag.  A
// thread owns rows r, r + kVecThreads, .. of the chunk (at most four) and
// takes the columns eight at a time, their loads issued together.
__global__ void __launch_bounds__(kVecThreads)
k_vec_sub_norm(int n, int rows, int ma, const double *__restrict__ V, int ldv, const double *__restrict__ c,
               double *__restrict__ W, double *__restrict__ part, unsigned *__restrict__ arrive,
               double *__restrict__ B, double *__restrict__ ri, double *__restrict__ flag)
{
    constexpr int R = kVecMaxRows / kVecThreads;
    constexpr int J = 8;
    __shared__ double red[kVecThreads];
    const int e0 = blockIdx.x * rows, len = min(n, e0 + rows) - e0;
    double acc[R];
#pragma unroll
    for (int m = 0; m < R; m++) acc[m] = 0.0;
    int j = 0;
    for (; j + J <= ma; j += J) {
        double cj[J], v[J][R];
#pragma unroll
        for (int u = 0; u < J; u++) cj[u] = __ldg(&c[j + u]);
#pragma unroll
        for (int u = 0; u < J; u++)
#pragma unroll
            for (int m = 0; m < R; m++) {
                const int r = threadIdx.x + m * kVecThreads;
                v[u][m] = r < len ? V[(size_t)(j + u) * ldv + e0 + r] : 0.0;
            }
#pragma unroll
        for (int u = 0; u < J; u++)
#pragma unroll
            for (int m = 0; m < R; m++) acc[m] = fma(v[u][m], cj[u], acc[m]);
    }
    for (; j < ma; j++) {
        const double cj = __ldg(&c[j]);
#pragma unroll
        for (int m = 0; m < R; m++) {
            const int r = threadIdx.x + m * kVecThreads;
            if (r < len) acc[m] = fma(V[(size_t)j * ldv + e0 + r], cj, acc[m]);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < R; m++) {
        const int r = threadIdx.x + m * kVecThreads;
        if (r < len) {
            const double w = W[e0 + r] - acc[m];
            W[e0 + r] = w;
            s = fma(w, w, s);
        }
    }
    s = vec_cta_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
    if (!vec_last_cta(arrive)) return;
    vec_norm_fold(part, B, ri, flag, red);
    if (threadIdx.x == 0) *arrive = 0u;
}

// W *= *ri (the next basis vector); when Wn is given, Wn = *B Vi, the
// V_i B_i^T term that the next iteration's product subtracts from.
__global__ void __launch_bounds__(kVecThreads)
k_vec_scale(int n, const double *__restrict__ ri, double *__restrict__ W, const double *__restrict__ B,
            const double *__restrict__ Vi, double *__restrict__ Wn)
{
    const int e = blockIdx.x * kVecThreads + threadIdx.x;
    if (e >= n) return;
    W[e] *= *ri;
    if (Wn) Wn[e] = *B * Vi[e];
}

// ---------------------------------------------------------------------------
// The whole single-vector iteration in one cooperative launch: the four
// steps above as phases of one kernel, separated by grid barriers instead of
// kernel boundaries.  A CTA takes the row chunks blockIdx.x, blockIdx.x + G,
// .. (G = gridDim.x, all CTAs resident), writes one partial sum per phase
// and column, and after the barrier every CTA adds all G partials itself in
// the same fixed order, so every CTA holds the same A_i, c and B_i to the
// bit.  Barrier counters: bar[p] for this launch (p = launch parity), while
// CTA 0 clears bar[p ^ 1] for the next one (the launch before this one, which
// used it, has completed).  A barrier wait gives up after about a second
// (kVecSpinLimit polls), sets *err and returns; the host reports it.
constexpr int kVecMaxCols = 512;           // columns the fused kernel stages in shared memory
constexpr long long kVecSpinLimit = 1 << 21;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Arrive at the grid barrier and wait until `target` CTAs have arrived in
// total; false (in every thread) when the wait gave up.
__device__ __forceinline__ bool vec_grid_sync(unsigned *bar, unsigned target, unsigned *err)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        __threadfence();
        atomicAdd(bar, 1u);
        long long spins = 0;
        while (ld_acquire_u32(bar) < target) {
            if (++spins > kVecSpinLimit) {
                atomicOr(err, 1u);
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Sum of part[0 .. G) in a fixed order, by one warp: a lane loads q = lane,
// lane + 32, .. (all eight of a 256-block issued together) and adds them in
// order, then a fixed shuffle tree; every lane returns lane 0's sum.
__device__ __forceinline__ double vec_warp_sum_parts(const double *part, int G)
{
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int q0 = 0; q0 < G; q0 += 256) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int q = q0 + lane + 32 * u;
            v[u] = q < G ? __ldcg(&part[q]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) s += v[u];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return __shfl_sync(0xffffffffu, s, 0);
}

// part: [G] dot partials, [ma][G] reorthogonalisation partials (column-major,
// so a column's partials are contiguous for the fold), [G] norm partials.
// W = V_i + ldv is the product's output, updated in place; it is passed as
// its own pointer, never reached through the read-only V (whose loads may
// take the non-coherent path).  Wn as k_vec_scale.  dA/dB/dflag: the
// iteration's history slots (written by CTA 0).  While the first barrier is pending, the CTA's rows of
// V_0 .. V_{i-1} are prefetched into L2 (the mobility product in between
// has streamed far more than L2 holds), so the reorthogonalisation reads
// them from there.
__global__ void __launch_bounds__(kVecThreads, 1)
k_vec_iter(int n, int rows, int nchunks, int ma, int reorth, const double *__restrict__ V, int ldv,
           double *__restrict__ W, double *__restrict__ Wn, double *__restrict__ part, unsigned *__restrict__ bars,
           int parity,
           unsigned skew, unsigned *__restrict__ err, double *__restrict__ dA, double *__restrict__ dB,
           double *__restrict__ dflag)
{
    __shared__ double sw[kVecMaxRows];
    __shared__ double sc[kVecMaxCols];
    __shared__ double red[kVecWarps];
    __shared__ double sval[2];
    const int G = gridDim.x, tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    unsigned *bar = bars + parity;
    if (blockIdx.x == 0 && tid == 0) bars[parity ^ 1] = 0u;
    const double *Vi = V + (size_t)(ma - 1) * ldv;
    double *p1 = part, *p2 = part + G, *p3 = p2 + (size_t)G * ma;
    // after a wait that ran out: the iteration reads as a breakdown, so the
    // host stops issuing, and the flag in *err reports it
    auto give_up = [&]() {
        if (blockIdx.x == 0 && tid == 0) {
            *dA = 0.0;
            *dB = 0.0;
            *dflag = 1.0;
        }
    };

    // A_i = V_i . W
    double s = 0.0;
    for (int ch = blockIdx.x; ch < nchunks; ch += G) {
        const int e1 = min(n, (ch + 1) * rows);
        for (int e = ch * rows + tid; e < e1; e += kVecThreads) s = fma(Vi[e], W[e], s);
    }
    if (reorth) {
        // 128-byte lines of the chunks' rows of V_0 .. V_{i-1}
        for (int ch = blockIdx.x; ch < nchunks; ch += G) {
            const int e0 = ch * rows, e1 = min(n, e0 + rows);
            const int l0 = e0 / 16, nl = (e1 - 1) / 16 - l0 + 1;
            for (int t = tid; t < (ma - 1) * nl; t += kVecThreads) {
                const int j = t / nl, l = l0 + t % nl;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(V + (size_t)j * ldv + 16 * l));
            }
        }
    }
    s = vec_cta_sum(s, red);
    if (tid == 0) p1[blockIdx.x] = s;
    if (!vec_grid_sync(bar, G + skew, err)) return give_up();
    if (wp == 0) {
        const double a = vec_warp_sum_parts(p1, G);
        if (lane == 0) {
            sval[0] = a;
            if (blockIdx.x == 0) *dA = a;
        }
    }
    __syncthreads();
    const double a = sval[0];

    // W -= A_i V_i, then either c = V_{0..i}^T W or g = W . W
    s = 0.0;
    bool first = true;
    for (int ch = blockIdx.x; ch < nchunks; ch += G) {
        const int e0 = ch * rows, len = min(n, e0 + rows) - e0;
        __syncthreads();  // sw is free again
        for (int r = tid; r < len; r += kVecThreads) {
            const double w = fma(-a, Vi[e0 + r], W[e0 + r]);
            W[e0 + r] = w;
            if (reorth) sw[r] = w;
            else s = fma(w, w, s);
        }
        if (!reorth) continue;
        __syncthreads();
        // warp wp: columns j0 .. j0+3; a lane takes rows lane, lane + 32, ..,
        // eight of them (32 loads) at a time
        for (int j0 = 4 * wp; j0 < ma; j0 += 4 * kVecWarps) {
            double t[4] = {0.0, 0.0, 0.0, 0.0};
            const double *Vj = V + (size_t)j0 * ldv + e0;
            const int nq = min(4, ma - j0);
            for (int r0 = 0; r0 < len; r0 += 256) {
                double w[8], v[4][8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int r = r0 + lane + 32 * u;
                    w[u] = r < len ? sw[r] : 0.0;
                }
#pragma unroll
                for (int q = 0; q < 4; q++)
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        const int r = r0 + lane + 32 * u;
                        v[q][u] = (q < nq && r < len) ? Vj[(size_t)q * ldv + r] : 0.0;
                    }
#pragma unroll
                for (int q = 0; q < 4; q++)
#pragma unroll
                    for (int u = 0; u < 8; u++) t[q] = fma(v[q][u], w[u], t[q]);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                for (int o = 16; o > 0; o >>= 1) t[q] += __shfl_xor_sync(0xffffffffu, t[q], o);
                // lane 0 of the warp that owns column j0 + q accumulates this CTA's chunks
                if (lane == 0 && q < nq) {
                    double *dst = &p2[(size_t)(j0 + q) * G + blockIdx.x];
                    *dst = first ? t[q] : *dst + t[q];
                }
            }
        }
        first = false;
    }
    unsigned target = 2u * G;
    if (reorth) {
        if (first)  // a CTA without chunks contributes zeros
            for (int j = tid; j < ma; j += kVecThreads) p2[(size_t)j * G + blockIdx.x] = 0.0;
        if (!vec_grid_sync(bar, target, err)) return give_up();
        target += G;
        // c_j = sum over CTAs (warp w takes the columns j = w mod kVecWarps)
        for (int j = wp; j < ma; j += kVecWarps) {
            const double c = vec_warp_sum_parts(p2 + (size_t)j * G, G);
            if (lane == 0) sc[j] = c;
        }
        __syncthreads();
        // W -= V_{0..i} c ; g = W . W
        s = 0.0;
        for (int ch = blockIdx.x; ch < nchunks; ch += G) {
            const int e0 = ch * rows, len = min(n, e0 + rows) - e0;
            if (len <= kVecThreads) {
                // one row a thread: sixteen columns' loads at a time
                constexpr int J = 16;
                const int r = tid;
                if (r < len) {
                    const double *Vr = V + e0 + r;
                    double acc = 0.0;
                    int j = 0;
                    for (; j + J <= ma; j += J) {
                        double v[J];
#pragma unroll
                        for (int u = 0; u < J; u++) v[u] = Vr[(size_t)(j + u) * ldv];
#pragma unroll
                        for (int u = 0; u < J; u++) acc = fma(v[u], sc[j + u], acc);
                    }
                    for (; j < ma; j++) acc = fma(Vr[(size_t)j * ldv], sc[j], acc);
                    const double w = W[e0 + r] - acc;
                    W[e0 + r] = w;
                    s = fma(w, w, s);
                }
                continue;
            }
            constexpr int R = kVecMaxRows / kVecThreads;
            constexpr int J = 8;
            double acc[R];
#pragma unroll
            for (int m = 0; m < R; m++) acc[m] = 0.0;
            int j = 0;
            for (; j + J <= ma; j += J) {
                double v[J][R];
#pragma unroll
                for (int u = 0; u < J; u++)
#pragma unroll
                    for (int m = 0; m < R; m++) {
                        const int r = tid + m * kVecThreads;
                        v[u][m] = r < len ? V[(size_t)(j + u) * ldv + e0 + r] : 0.0;
                    }
#pragma unroll
                for (int u = 0; u < J; u++)
#pragma unroll
                    for (int m = 0; m < R; m++) acc[m] = fma(v[u][m], sc[j + u], acc[m]);
            }
            for (; j < ma; j++) {
#pragma unroll
                for (int m = 0; m < R; m++) {
                    const int r = tid + m * kVecThreads;
                    if (r < len) acc[m] = fma(V[(size_t)j * ldv + e0 + r], sc[j], acc[m]);
                }
            }
#pragma unroll
            for (int m = 0; m < R; m++) {
                const int r = tid + m * kVecThreads;
                if (r < len) {
                    const double w = W[e0 + r] - acc[m];
                    W[e0 + r] = w;
                    s = fma(w, w, s);
                }
            }
        }
    }
    s = vec_cta_sum(s, red);
    if (tid == 0) p3[blockIdx.x] = s;
    if (!vec_grid_sync(bar, target, err)) return give_up();
    // B_i = ||W||, as vec_norm_fold
    if (wp == 0) {
        const double d = vec_warp_sum_parts(p3, G);
        if (lane == 0) {
            const bool ok = d > 0.0;
            const double b = ok ? sqrt(d) : 0.0;
            sval[0] = b;
            sval[1] = ok ? 1.0 / b : 0.0;
            if (blockIdx.x == 0) {
                *dB = b;
                *dflag = ok ? 0.0 : 1.0;
            }
        }
    }
    __syncthreads();
    const double b = sval[0], ri = sval[1];
    // V_{i+1} = W / B_i ; next W = B_i V_i
    for (int ch = blockIdx.x; ch < nchunks; ch += G) {
        const int e1 = min(n, (ch + 1) * rows);
        for (int e = ch * rows + tid; e < e1; e += kVecThreads) {
            W[e] *= ri;
            if (Wn) Wn[e] = b * Vi[e];
        }
    }
}

// x *= s (host scalar)
__global__ void __launch_bounds__(kVecThreads) k_vec_scale_host(int n, double s, double *__restrict__ x)
{
    const int e = blockIdx.x * kVecThreads + threadIdx.x;
    if (e < n) x[e] *= s;
}

// ---------------------------------------------------------------------------

static int gram(LanczosState *lz, int ma, const double *A, int lda, int mb, const double *B, int ldb,
                double *d_out)
{
    const int n = lz->dim;
    const bool pairs_aligned = lda % 2 == 0 && ldb % 2 == 0 && ((uintptr_t)A % 16) == 0 &&
                               ((uintptr_t)B % 16) == 0;
    if (ma >= 64 && mb <= 16 && pairs_aligned) {
        // tall A: ~4 CTAs per SM over (row chunks x 128-row tiles of A)
        const int ta = (ma + kGramTileA - 1) / kGramTileA;
        int nchunks = std::max(1, 4 * lz->num_sms / ta);
        nchunks = std::min(nchunks, (n + 1023) / 1024);
        nchunks = (int)std::min<size_t>((size_t)nchunks, lz->part_cap / ((size_t)ma * mb));
        nchunks = std::max(1, nchunks);
        const int rows = ((n + nchunks - 1) / nchunks + kGramStageE - 1) / kGramStageE * kGramStageE;
        nchunks = (n + rows - 1) / rows;
        k_gram_tall<<<dim3(nchunks, ta), 256, kGramSmem, lz->stream>>>(n, ma, A, lda, mb, B, ldb, rows,
                                                                       lz->d_part);
        LZ_LAUNCH();
        const int count = ma * mb;
        k_reduce_parts<<<(count + 31) / 32, 256, 0, lz->stream>>>(nchunks, count, lz->d_part, d_out);
        LZ_LAUNCH();
        return kOk;
    }
    if (ma <= 64 && mb <= 16 && pairs_aligned) {
        // short blocks (A in 16-row tiles): up to two CTAs per SM over row chunks of >= 256
        // rows (short vectors still spread over the GPU: 3N = 6e4 gives 235)
        int nchunks = std::min(2 * lz->num_sms, (n + 255) / 256);
        nchunks = (int)std::min<size_t>((size_t)nchunks, lz->part_cap / ((size_t)ma * mb));
        nchunks = std::max(1, nchunks);
        const int rows = ((n + nchunks - 1) / nchunks + kSmallStageE - 1) / kSmallStageE * kSmallStageE;
        nchunks = (n + rows - 1) / rows;
        // up to 64 outputs: the kernel's last CTA sums the parts itself
        const int count = ma * mb;
        const bool fold = count <= 64;
        k_gram_small<<<dim3(nchunks, (ma + 15) / 16), 256, 0, lz->stream>>>(
            n, ma, A, lda, mb, B, ldb, rows, lz->d_part, fold ? lz->d_arrive : nullptr, d_out);
        LZ_LAUNCH();
        if (!fold) {
            k_reduce_parts<<<(count + 31) / 32, 256, 0, lz->stream>>>(nchunks, count, lz->d_part, d_out);
            LZ_LAUNCH();
        }
        return kOk;
    }
    const int ta = (ma + 15) / 16, tb = (mb + 15) / 16;
    int nchunks = std::min(lz->gram_chunks, (n + 255) / 256);
    nchunks = (int)std::min<size_t>((size_t)nchunks, lz->part_cap / ((size_t)ma * mb));
    nchunks = std::max(1, nchunks);
    const int rows = (n + nchunks - 1) / nchunks;
    k_gram_partial<<<dim3(nchunks, ta, tb), 256, 0, lz->stream>>>(n, ma, A, lda, mb, B, ldb, rows, lz->d_part);
    LZ_LAUNCH();
    const int count = ma * mb;
    k_reduce_parts<<<(count + 31) / 32, 256, 0, lz->stream>>>(nchunks, count, lz->d_part, d_out);
    LZ_LAUNCH();
    return kOk;
}

static int block_gemm(LanczosState *lz, int ma, const double *A, int lda, const double *d_C, int mb,
                      double beta, double *Out, int ldo, double alpha = 1.0)
{
    const int n = lz->dim;
    if (mb <= 16) {
        const int grid = (n + 511) / 512;
        k_gemm_tall<<<grid, 256, 0, lz->stream>>>(n, ma, A, lda, d_C, mb, alpha, beta, Out, ldo);
        LZ_LAUNCH();
        return kOk;
    }
    // stage C in chunks of rows so the shared copy stays small
    const int step = std::max(1, std::min(ma, 4096 / std::max(1, mb)));
    for (int a0 = 0; a0 < ma; a0 += step) {
        const int na = std::min(step, ma - a0);
        const size_t sm = (size_t)na * mb * sizeof(double);
        k_block_gemm<<<(n + 255) / 256, 256, sm, lz->stream>>>(n, na, A + (size_t)a0 * lda, lda,
                                                               d_C + (size_t)a0 * mb, mb, alpha,
                                                               a0 == 0 ? beta : 1.0, Out, ldo);
        LZ_LAUNCH();
    }
    return kOk;
}

using Clock = std::chrono::steady_clock;
static double ms_since(Clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

static int download(LanczosState *lz, double *h, const double *d, size_t count)
{
    const Clock::time_point t0 = Clock::now();
    LZ_CUDA(cudaMemcpyAsync(h, d, count * sizeof(double), cudaMemcpyDeviceToHost, lz->stream));
    LZ_CUDA(cudaStreamSynchronize(lz->stream));
    lz->t_sync_ms += ms_since(t0);
    return kOk;
}

static int upload(LanczosState *lz, double *d, const double *h, size_t count)
{
    LZ_CUDA(cudaMemcpyAsync(d, h, count * sizeof(double), cudaMemcpyHostToDevice, lz->stream));
    LZ_CUDA(cudaStreamSynchronize(lz->stream));
    return kOk;
}

// Row chunk of the single-vector kernels: about one chunk per SM, a
// multiple of 32 rows, at least 256 and at most kVecMaxRows.
static int vec_rows(int n, int num_sms)
{
    const int per = (n + num_sms - 1) / std::max(1, num_sms);
    return std::min(kVecMaxRows, std::max(256, (per + 31) / 32 * 32));
}

// One Cholesky-QR step of one k x k Gram matrix (chol_qr_step_warp), one warp.
__global__ void __launch_bounds__(32)
k_chol_qr_step(int k, const double *__restrict__ G, double *__restrict__ Ri, double *__restrict__ Racc,
               int first, double *__restrict__ Bout, double *__restrict__ Btout, double *__restrict__ flag)
{
    chol_qr_step_warp<kMaxBlock>(k, G, Ri, Racc, first, Bout, Btout, flag);
}

// In-place Cholesky QR of the k columns X (ld), applied twice, all on the
// device: X_in = X_out R with R (upper, row-major) left in the running-factor
// scratch and, when B is given, in B (and B^T in the transpose scratch).  If
// G0 is given it already holds X^T X (first pass).  *flag (device) is set to
// 1 on breakdown.
static int chol_qr_device(LanczosState *lz, double *X, int ld, int k, bool have_g0, double *B, double *flag)
{
    const int kk = kMaxBlock * kMaxBlock;
    double *Ri = lz->d_qr, *Racc = lz->d_qr + kk, *Bt = lz->d_qr + 2 * kk;
    for (int pass = 0; pass < 2; pass++) {
        if (!(pass == 0 && have_g0)) {
            const int st = gram(lz, k, X, ld, k, X, ld, lz->d_small);
            if (st != kOk) return st;
        }
        k_chol_qr_step<<<1, 32, 0, lz->stream>>>(k, lz->d_small, Ri, Racc, pass == 0, pass == 1 ? B : nullptr,
                                                  pass == 1 ? Bt : nullptr, flag);
        LZ_LAUNCH();
        const int st = block_gemm(lz, k, X, ld, Ri, k, 0.0, X, ld);
        if (st != kOk) return st;
    }
    return kOk;
}

int lanczos_alloc(LanczosState *lz)
{
    lz->ldv = (lz->dim + 31) / 32 * 32;
    const size_t nv = (size_t)(lz->max_iters + 1) * lz->max_nrhs * lz->ldv;
    LZ_CUDA(cudaSetDevice(lz->device));
    if (!lz->stream) {
        LZ_CUDA(cudaStreamCreateWithFlags(&lz->stream, cudaStreamNonBlocking));
        lz->own_stream = true;
    }
    LZ_CUDA(cudaMalloc(&lz->d_V, nv * sizeof(double)));
    const int mmax = (lz->max_iters + 1) * lz->max_nrhs;
    lz->gram_chunks = 296;
    int dev_sms = 148;
    if (cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, lz->device) != cudaSuccess) {
        cudaGetLastError();
        dev_sms = 148;
    }
    lz->num_sms = dev_sms;
    LZ_CUDA(cudaFuncSetAttribute(k_gram_tall, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGramSmem));
    lz->part_cap = std::max((size_t)lz->gram_chunks * 16 * 16, (size_t)64 * mmax * lz->max_nrhs);
    // the single-vector kernels' per-chunk partial sums of up to mmax columns
    const int vrows = vec_rows(lz->dim, lz->num_sms);
    lz->part_cap = std::max(lz->part_cap, (size_t)((lz->dim + vrows - 1) / vrows) * (mmax + 2));
    LZ_CUDA(cudaMalloc(&lz->d_part, lz->part_cap * sizeof(double)));
    // [0] last-CTA counter of the Gram folds, [1..2] grid-barrier counters of
    // the fused single-vector iteration, [3] its barrier-timeout flag
    LZ_CUDA(cudaMalloc(&lz->d_arrive, 4 * sizeof(unsigned)));
    LZ_CUDA(cudaMemset(lz->d_arrive, 0, 4 * sizeof(unsigned)));
    LZ_CUDA(cudaMallocHost(&lz->h_err, sizeof(unsigned)));
    *lz->h_err = 0u;
    // the fused single-vector iteration: one resident CTA per row chunk at most
    // (STOKESDT_VEC_UNFUSED=1 keeps the four-launch form)
    {
        int coop = 0, per_sm = 0;
        lz->vec_grid = 0;
        const char *unfused = std::getenv("STOKESDT_VEC_UNFUSED");
        // STOKESDT_VEC_BARRIER_SKEW=k raises the first barrier's target by k
        // arrivals that never come: the wait runs out, which the failure
        // tests use to check that it is reported
        const char *skew = std::getenv("STOKESDT_VEC_BARRIER_SKEW");
        lz->vec_barrier_skew = skew ? (unsigned)std::max(0, std::atoi(skew)) : 0u;
        if (!(unfused && unfused[0] == '1') &&
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, lz->device) == cudaSuccess && coop &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vec_iter, kVecThreads, 0) == cudaSuccess &&
            per_sm > 0)
            lz->vec_grid = std::min(per_sm * lz->num_sms, (lz->dim + vrows - 1) / vrows);
        cudaGetLastError();
    }
    LZ_CUDA(cudaMalloc(&lz->d_small, (size_t)mmax * std::max(lz->max_nrhs, 16) * sizeof(double)));
    LZ_CUDA(cudaMalloc(&lz->d_coef, (size_t)mmax * lz->max_nrhs * sizeof(double)));
    LZ_CUDA(cudaMalloc(&lz->d_dY, (size_t)lz->max_nrhs * lz->ldv * sizeof(double)));
    lz->hist_stride = 2 * lz->max_nrhs * lz->max_nrhs + 2;
    const size_t hist = (size_t)(lz->max_iters + 1) * lz->hist_stride;
    LZ_CUDA(cudaMalloc(&lz->d_hist, hist * sizeof(double)));
    LZ_CUDA(cudaMallocHost(&lz->h_hist, hist * sizeof(double)));
    LZ_CUDA(cudaMalloc(&lz->d_qr, (size_t)3 * kMaxBlock * kMaxBlock * sizeof(double)));
    lz->ev.assign(lz->max_iters + 1, nullptr);
    for (cudaEvent_t &e : lz->ev) LZ_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return kOk;
}

void lanczos_free(LanczosState *lz)
{
    if (!lz) return;
    cudaSetDevice(lz->device);
    if (lz->stream) cudaStreamSynchronize(lz->stream);
    void *ptrs[] = {lz->d_V, lz->d_part, lz->d_arrive, lz->d_small, lz->d_coef, lz->d_dY, lz->d_zin, lz->d_yout,
                    lz->d_hist, lz->d_qr};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (lz->h_hist) cudaFreeHost(lz->h_hist);
    lz->h_hist = nullptr;
    if (lz->h_err) cudaFreeHost(lz->h_err);
    lz->h_err = nullptr;
    for (cudaEvent_t e : lz->ev)
        if (e) cudaEventDestroy(e);
    lz->ev.clear();
    if (lz->own_stream && lz->stream) cudaStreamDestroy(lz->stream);
    lz->stream = nullptr;
}

// One group of k <= max_nrhs vectors.  z and y are device pointers.
// Device-time accounting of the Lanczos phases (only when tracing): event
// pairs on the solver stream, summed once the stream has drained.
struct PhaseTimer {
    bool on = false;
    cudaStream_t s = nullptr;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
    int open_phase = -1;
    cudaEvent_t open_ev = nullptr;
    void begin(int phase)
    {
        if (!on) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        open_phase = phase;
        open_ev = e;
    }
    void end()
    {
        if (!on || open_phase < 0) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        marks.push_back({open_phase, {open_ev, e}});
        open_phase = -1;
    }
    void report(int its)
    {
        if (!on) return;
        cudaStreamSynchronize(s);
        double ms[4] = {0, 0, 0, 0};
        for (auto &m : marks) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, m.second.first, m.second.second);
            ms[m.first] += t;
            cudaEventDestroy(m.second.first);
            cudaEventDestroy(m.second.second);
        }
        marks.clear();
        std::fprintf(stderr, "[lanczos] device ms over %d iterations: products %.1f, recurrence %.1f, "
                     "reorthogonalisation %.1f, QR %.1f\n", its, ms[0], ms[1], ms[2], ms[3]);
    }
};

// The single-vector iteration after the product W = M V_i - B_{i-1} V_{i-1}
// (V_i = V + it ldv, W = V_i + ldv): A_i -> dA, the optional
// reorthogonalisation, V_{i+1} B_i = W (B_i -> dB, breakdown -> dflag) and,
// when Wn is given, Wn = B_i V_i for the next product.
static int vec_iteration(LanczosState *lz, int it, double *V, double *Wn, double *dA, double *dB, double *dflag,
                         bool reorth, PhaseTimer &pt)
{
    const int n = lz->dim, ldv = lz->ldv;
    const int rows = vec_rows(n, lz->num_sms), grid = (n + rows - 1) / rows;
    double *Vi = V + (size_t)it * ldv, *W = Vi + ldv;
    double *ri = lz->d_qr;
    int ma = it + 1;
    if (lz->vec_grid > 0 && ma <= kVecMaxCols) {
        // one cooperative launch (all CTAs resident: they wait on one another)
        int nchunks = grid, rev = reorth ? 1 : 0, parity = (int)(lz->vec_launches & 1);
        unsigned skew = lz->vec_barrier_skew;
        double *part = lz->d_part;
        unsigned *bars = lz->d_arrive + 1, *err = lz->d_arrive + 3;
        void *args[] = {(void *)&n, (void *)&rows, (void *)&nchunks, (void *)&ma, (void *)&rev, (void *)&V,
                        (void *)&ldv, (void *)&W, (void *)&Wn, (void *)&part, (void *)&bars, (void *)&parity,
                        (void *)&skew, (void *)&err, (void *)&dA, (void *)&dB, (void *)&dflag};
        pt.begin(1);
        const cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_vec_iter, dim3(lz->vec_grid),
                                                          dim3(kVecThreads), args, 0, lz->stream);
        if (e == cudaErrorCooperativeLaunchTooLarge) {
            // fewer SMs than measured at allocation (a shared device): the
            // four-launch form from now on
            cudaGetLastError();
            lz->vec_grid = 0;
        } else {
            LZ_CUDA(e);
            LZ_LAUNCH();
            pt.end();
            lz->vec_launches++;
            return kOk;
        }
    }
    pt.begin(1);
    k_vec_dot<<<grid, kVecThreads, 0, lz->stream>>>(n, rows, Vi, W, lz->d_part, lz->d_arrive, dA);
    LZ_LAUNCH();
    if (!reorth) {
        k_vec_axpy_norm<<<grid, kVecThreads, 0, lz->stream>>>(n, rows, Vi, dA, W, lz->d_part, lz->d_arrive, dB,
                                                               ri, dflag);
        LZ_LAUNCH();
        pt.end();
    } else {
        k_vec_axpy_dots<<<grid, kVecThreads, 0, lz->stream>>>(n, rows, it + 1, V, ldv, dA, W, lz->d_part,
                                                               lz->d_arrive, lz->d_coef);
        LZ_LAUNCH();
        pt.end();
        pt.begin(2);
        k_vec_sub_norm<<<grid, kVecThreads, 0, lz->stream>>>(n, rows, it + 1, V, ldv, lz->d_coef, W, lz->d_part,
                                                              lz->d_arrive, dB, ri, dflag);
        LZ_LAUNCH();
        pt.end();
    }
    pt.begin(3);
    k_vec_scale<<<(n + kVecThreads - 1) / kVecThreads, kVecThreads, 0, lz->stream>>>(n, ri, W, dB, Vi, Wn);
    LZ_LAUNCH();
    pt.end();
    return kOk;
}

static int block_lanczos(LanczosState *lz, const MobOp &mob, int k, int ldz, const double *d_z, int ldy,
                         double *d_y, int *iters_out)
{
    const int n = lz->dim, ldv = lz->ldv, hs = lz->hist_stride, kk = k * k;
    double *V = lz->d_V;
    auto blk = [&](int i) { return V + (size_t)i * k * ldv; };
    // V_0 = Z
    LZ_CUDA(cudaMemcpy2DAsync(blk(0), ldv * sizeof(double), d_z, ldz * sizeof(double), n * sizeof(double), k,
                              cudaMemcpyDeviceToDevice, lz->stream));
    // ||Z||_F from G = Z^T Z, which is also the first Gram matrix of the QR
    std::vector<double> G(kk);
    int st = gram(lz, k, blk(0), ldv, k, blk(0), ldv, lz->d_small);
    if (st != kOk) return st;
    st = download(lz, G.data(), lz->d_small, (size_t)kk);
    if (st != kOk) return st;
    double normz2 = 0.0;
    for (int c = 0; c < k; c++) normz2 += G[c * k + c];
    const double normz = std::sqrt(normz2);
    if (!(normz > 0.0)) {
        LZ_CUDA(cudaMemset2DAsync(d_y, ldy * sizeof(double), 0, n * sizeof(double), k, lz->stream));
        *iters_out = 0;
        return kOk;
    }
    // V_0 R = Z (the spare history slot holds the breakdown flag); one
    // vector is normalised by the norm already at hand
    std::vector<double> R(kk);
    double flag0 = 0.0;
    if (k == 1) {
        R[0] = normz;
        k_vec_scale_host<<<(n + kVecThreads - 1) / kVecThreads, kVecThreads, 0, lz->stream>>>(n, 1.0 / normz,
                                                                                              blk(0));
        LZ_LAUNCH();
    } else {
        double *init_flag = lz->d_hist + (size_t)lz->max_iters * hs;
        st = chol_qr_device(lz, blk(0), ldv, k, true, nullptr, init_flag);
        if (st != kOk) return st;
        st = download(lz, R.data(), lz->d_qr + kMaxBlock * kMaxBlock, (size_t)kk);
        if (st == kOk) st = download(lz, &flag0, init_flag, 1);
        if (st != kOk) return st;
    }
    if (flag0 != 0.0) {
        lz->last_error = "random block is rank deficient";
        return kErrInvalid;
    }
    const bool reorth = lz->reorth;
    lz->history.clear();

    // D_i = sqrt(T_i)[:, :k] R on the host (FP64), run on a worker thread once
    // the iteration's A_i, B_i have reached pinned host memory.  T_i (m x m,
    // row-major) is assembled there from A_0..A_i and B_0..B_{i-1}.
    struct Solved {
        int status = 0, neg = 0;
        bool breakdown = false;
        double ms = 0.0;
        Clock::time_point ready;  // when the iteration's coefficients had arrived
        std::vector<double> D;
    };
    std::atomic<bool> cancel{false};
    auto solve = [k, kk, hs, &R, lz, &cancel](int it) {
        Solved out;
        cudaSetDevice(lz->device);
        if (cudaEventSynchronize(lz->ev[it]) != cudaSuccess) {
            out.status = -100;
            return out;
        }
        const Clock::time_point t0 = Clock::now();
        out.ready = t0;
        const int m = (it + 1) * k;
        const double *h = lz->h_hist;
        out.breakdown = h[(size_t)it * hs + 2 * kk] != 0.0;
        std::vector<double> T((size_t)m * m, 0.0);
        for (int b = 0; b <= it; b++) {
            const double *A = h + (size_t)b * hs, *B = A + kk;
            for (int r = 0; r < k; r++)
                for (int c = 0; c < k; c++)  // symmetrise A_b (symmetric up to rounding)
                    T[(size_t)(b * k + r) * m + b * k + c] = 0.5 * (A[r * k + c] + A[c * k + r]);
            if (b < it) {
                for (int r = 0; r < k; r++)
                    for (int c = 0; c < k; c++) {
                        const double x = B[r * k + c];
                        T[(size_t)((b + 1) * k + r) * m + b * k + c] = x;
                        T[(size_t)(b * k + c) * m + (b + 1) * k + r] = x;
                    }
            }
        }
        std::vector<double> S((size_t)m * k, 0.0);
        // quadrature form for SPD T (O(m k^2) per node); the eigendecomposition
        // when T is not positive definite (it also counts and clamps the
        // negative eigenvalues)
        out.status = sqrt_first_cols_quad(m, k, T.data(), S.data(), m >= 512 ? 4 : 1);
        if (out.status != 0) out.status = sqrt_first_cols(m, k, T.data(), S.data(), &out.neg, &cancel);
        out.D.assign((size_t)m * k, 0.0);
        for (int r = 0; r < m; r++)
            for (int c = 0; c < k; c++) {
                double acc = 0.0;
                for (int t = 0; t <= c; t++) acc += S[(size_t)r * k + t] * R[t * k + c];
                out.D[(size_t)r * k + c] = acc;
            }
        out.ms = ms_since(t0);
        return out;
    };

    std::vector<double> D, Dprev;
    int done_it = -1;          // last iteration whose D has been checked
    bool converged = false;
    // Check iteration i: ||Y_i - Y_{i-1}||_F / ||Z||_F < tol (brwn_lanczos.cc:188-196)
    auto check = [&](int i, Solved &&sv) -> int {
        if (sv.status == -100) {
            lz->last_error = "waiting for the Lanczos coefficients failed";
            return kErrCuda;
        }
        if (sv.status != 0) {
            lz->last_error = "tridiagonal eigensolver did not converge";
            return kErrNotConverged;
        }
        if (sv.neg > 0) lz->nonspd_count++;
        lz->t_eigen_ms += sv.ms;
        D = std::move(sv.D);
        const int m = (i + 1) * k;
        done_it = i;
        if (i > 0) {
            double diff2 = 0.0;
            if (reorth) {
                // orthonormal basis: ||V (D_i - [D_{i-1}; 0])|| = ||D_i - [D_{i-1}; 0]||
                for (int r = 0; r < m; r++)
                    for (int c = 0; c < k; c++) {
                        const double prev = (r < m - k) ? Dprev[(size_t)r * k + c] : 0.0;
                        const double d = D[(size_t)r * k + c] - prev;
                        diff2 += d * d;
                    }
            } else {
                // dY = V_{0..i} (D_i - [D_{i-1}; 0]) on the device
                std::vector<double> dD((size_t)m * k);
                for (int r = 0; r < m; r++)
                    for (int c = 0; c < k; c++)
                        dD[(size_t)r * k + c] =
                            D[(size_t)r * k + c] - ((r < m - k) ? Dprev[(size_t)r * k + c] : 0.0);
                int st2 = upload(lz, lz->d_coef, dD.data(), dD.size());
                if (st2 != kOk) return st2;
                st2 = block_gemm(lz, m, V, ldv, lz->d_coef, k, 0.0, lz->d_dY, ldv);
                if (st2 != kOk) return st2;
                k_sqnorm_partial<<<256, 256, 0, lz->stream>>>(n, k, lz->d_dY, ldv, lz->d_part);
                LZ_LAUNCH();
                std::vector<double> parts(256);
                st2 = download(lz, parts.data(), lz->d_part, 256);
                if (st2 != kOk) return st2;
                for (double x : parts) diff2 += x;
            }
            const double rel = std::sqrt(diff2) / normz;
            lz->history.push_back(rel);
            if (rel < lz->tol) converged = true;
        }
        // a rank-deficient W (breakdown) means V_{0..i} spans an invariant
        // subspace: the iterate is exact
        if (sv.breakdown) converged = true;
        Dprev = D;
        return kOk;
    };
    // The last checked errors decay geometrically; iteration j is expected to
    // pass the test when the extrapolated error is below tol.  Issuing work
    // past that point would only be discarded, so the host then waits for the
    // outstanding checks before it issues more.  The rate is the mean over
    // the last (up to six) checks: with one vector the error falls by ratios
    // anywhere from 0.3 to 1.4 from one check to the next, so the last ratio
    // alone often predicts no convergence at all.
    auto expect_converged = [&](int j) {
        const std::vector<double> &h = lz->history;
        if (h.size() < 2 || done_it < 0) return false;
        const int w = std::min<int>(6, (int)h.size() - 1);
        const double q = std::pow(h.back() / h[h.size() - 1 - w], 1.0 / w);
        if (!(q > 0.0) || q >= 1.0) return false;
        return h.back() * std::pow(q, (double)(j - done_it)) < lz->tol;
    };

    // The iterations are issued without waiting on the GPU: A_i, B_i and the
    // breakdown flag are copied to pinned memory behind each iteration and the
    // eigenproblems run on worker threads once they arrive.  Results are
    // checked strictly in iteration order, so the iteration count and the
    // returned iterate are those of a check after every iteration.  With
    // reorthogonalisation the check is host-only and up to `lookahead` solves
    // may be in flight; without it the check issues device work on the solver
    // stream, so one solve is in flight.  Work issued past the converged
    // iteration is discarded.
    //
    // Every solve in flight is an iteration that may run past convergence, so
    // only as many are kept as cover the host's solve: two, plus one per
    // GPU iteration time the last solve took (at most `lookahead`).  The GPU
    // iteration time is the gap between the arrivals of consecutive
    // iterations' coefficients.
    std::deque<std::pair<int, std::future<Solved>>> pending;
    const int lookahead_max = reorth ? std::max(1, lz->lookahead) : 1;
    int lookahead = lookahead_max;
    int it;
    int last_ready_it = -2;
    Clock::time_point last_ready;
    auto take_front = [&]() -> int {
        const Clock::time_point tw = Clock::now();
        Solved sv = pending.front().second.get();
        lz->t_wait_ms += ms_since(tw);
        const int i = pending.front().first;
        pending.pop_front();
        if (sv.status == 0 && last_ready_it == i - 1) {
            const double t_iter = std::chrono::duration<double, std::milli>(sv.ready - last_ready).count();
            if (t_iter > 0.0)
                lookahead = std::min(lookahead_max, 2 + (int)std::floor(sv.ms / t_iter));
        }
        last_ready_it = i;
        last_ready = sv.ready;
        return check(i, std::move(sv));
    };
    PhaseTimer pt;
    pt.on = std::getenv("STOKESDT_LANCZOS_TRACE") != nullptr;
    pt.s = lz->stream;
    double *Bt = lz->d_qr + 2 * kMaxBlock * kMaxBlock;
    for (it = 0; it < lz->max_iters && !converged; it++) {
        double *Vi = blk(it);
        double *W = blk(it + 1);
        double *dA = lz->d_hist + (size_t)it * hs, *dB = dA + kk, *dflag = dA + 2 * kk;
        pt.begin(0);
        if (it > 0) {
            // W = V_{i-1} B_{i-1}^T (one vector: already written by the last
            // iteration's scaling), then W = M V_i - W
            if (k > 1) {
                st = block_gemm(lz, k, blk(it - 1), ldv, Bt, k, 0.0, W, ldv);
                if (st != kOk) break;
            }
            st = mob.mulvec(k, 1.0, ldv, Vi, -1.0, ldv, W, lz->stream);
        } else {
            st = mob.mulvec(k, 1.0, ldv, Vi, 0.0, ldv, W, lz->stream);
        }
        lz->products++;
        pt.end();
        if (st != kOk) {
            lz->last_error = "mobility product failed: " + mob.error();
            break;
        }
        if (k == 1) {
            st = vec_iteration(lz, it, V, it + 1 < lz->max_iters ? blk(it + 2) : nullptr, dA, dB, dflag, reorth,
                               pt);
            if (st != kOk) break;
        } else {
            // A_i = V_i^T W ; W -= V_i A_i
            pt.begin(1);
            st = gram(lz, k, Vi, ldv, k, W, ldv, dA);
            if (st != kOk) break;
            st = block_gemm(lz, k, Vi, ldv, dA, k, 1.0, W, ldv, -1.0);
            if (st != kOk) break;
            pt.end();
            if (reorth) {
                pt.begin(2);
                const int ma = (it + 1) * k;
                st = gram(lz, ma, V, ldv, k, W, ldv, lz->d_coef);
                if (st != kOk) break;
                st = block_gemm(lz, ma, V, ldv, lz->d_coef, k, 1.0, W, ldv, -1.0);  // W -= V C
                if (st != kOk) break;
                pt.end();
            }
            // W = V_{i+1} B_i; B_i^T stays on the device for the next product
            pt.begin(3);
            st = chol_qr_device(lz, W, ldv, k, false, dB, dflag);
            pt.end();
            if (st != kOk) break;
        }
        if (cudaMemcpyAsync(lz->h_hist + (size_t)it * hs, dA, (size_t)(2 * kk + 1) * sizeof(double),
                            cudaMemcpyDeviceToHost, lz->stream) != cudaSuccess ||
            cudaEventRecord(lz->ev[it], lz->stream) != cudaSuccess) {
            lz->last_error = "queueing the coefficient copy failed";
            st = kErrCuda;
            break;
        }
        pending.emplace_back(it, std::async(std::launch::async, solve, it));
        // check every finished solve in order; block when too many are in
        // flight or when this iteration is expected to converge
        while (!pending.empty() && !converged && st == kOk &&
               ((int)pending.size() > lookahead || expect_converged(it) ||
                pending.front().second.wait_for(std::chrono::seconds(0)) == std::future_status::ready))
            st = take_front();
        if (st != kOk || converged) break;
    }
    pt.report(it);
    while (st == kOk && !converged && !pending.empty()) st = take_front();
    // solves started past the converged iteration are abandoned
    cancel.store(true);
    while (!pending.empty()) {
        pending.front().second.wait();
        pending.pop_front();
    }
    // A grid-barrier wait of the fused single-vector iteration that ran out
    // voids the result, whatever the checks made of it; its flag comes back
    // with the synchronisation of the coefficient upload (or of the stream,
    // when the iteration failed otherwise).
    if (k == 1)
        LZ_CUDA(cudaMemcpyAsync(lz->h_err, lz->d_arrive + 3, sizeof(unsigned), cudaMemcpyDeviceToHost, lz->stream));
    const int mfinal = (done_it + 1) * k;
    if (st == kOk) {
        st = upload(lz, lz->d_coef, D.data(), D.size());
    } else if (k == 1) {
        LZ_CUDA(cudaStreamSynchronize(lz->stream));
    }
    if (k == 1 && *lz->h_err != 0u) {
        *lz->h_err = 0u;
        LZ_CUDA(cudaMemsetAsync(lz->d_arrive, 0, 4 * sizeof(unsigned), lz->stream));
        lz->last_error = "single-vector iteration: a grid barrier wait timed out";
        return kErrCuda;
    }
    if (st != kOk) return st;
    // Y = V_{0..i} D_i
    st = block_gemm(lz, mfinal, V, ldv, lz->d_coef, k, 0.0, d_y, ldy);
    if (st != kOk) return st;
    *iters_out = converged ? done_it : -1;
    return kOk;
}

int lanczos_compute(LanczosState *lz, SpmeEngine *mob, int nrhs, int ldz, const double *d_z, int ldy,
                    double *d_y, int *iters)
{
    MobOp op;
    op.dim = 3 * mob->npos;
    // the mobility products run on the solver's stream, ordered after its work
    op.mulvec = [mob](int nr, double a, int ldf, const double *f, double b, int ldv, double *v, cudaStream_t s) {
        cudaStream_t saved = mob->stream;
        mob->stream = s;
        const int st = spme_mulvec(mob, 0, nr, a, ldf, f, b, ldv, v);
        mob->stream = saved;
        return st;
    };
    op.error = [mob]() { return mob->last_error; };
    return lanczos_compute_op(lz, op, nrhs, ldz, d_z, ldy, d_y, iters);
}

int lanczos_compute_op(LanczosState *lz, const MobOp &mob, int nrhs, int ldz, const double *d_z, int ldy,
                       double *d_y, int *iters)
{
    if (mob.dim != lz->dim) {
        lz->last_error = "mobility dimension does not match the Lanczos dimension";
        return kErrInvalid;
    }
    if (ldz < lz->dim || ldy < lz->dim || nrhs < 0) {
        lz->last_error = "bad nrhs or leading dimension";
        return kErrInvalid;
    }
    const Clock::time_point t_start = Clock::now();
    lz->t_sync_ms = lz->t_eigen_ms = lz->t_wait_ms = 0.0;
    lz->products = 0;
    int status = kOk;
    int g = 0;
    for (int r0 = 0; r0 < nrhs; r0 += lz->max_nrhs, g++) {
        const int k = std::min(lz->max_nrhs, nrhs - r0);
        int it = -1;
        const int st = block_lanczos(lz, mob, k, ldz, d_z + (size_t)r0 * ldz, ldy, d_y + (size_t)r0 * ldy, &it);
        if (st != kOk) return st;
        if (iters) iters[g] = it;
        if (it < 0) status = kErrNotConverged;
    }
    if (std::getenv("STOKESDT_LANCZOS_TRACE"))
        fprintf(stderr, "[lanczos] %d RHS: total %.1f ms, waiting on GPU %.1f ms, eigensolves %.1f ms "
                "(blocked on them %.1f ms), %lld block products\n", nrhs, ms_since(t_start), lz->t_sync_ms,
                lz->t_eigen_ms, lz->t_wait_ms, lz->products);
    return status;
}

}  // namespace sdt
