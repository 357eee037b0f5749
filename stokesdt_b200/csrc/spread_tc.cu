// Spread + x transform on the tensor cores (K = 256).
//
// For one row block (kTcBZ x kTcBY rows of (z, y)) and one RHS the
// spread followed by the real-to-complex x DFT is a matrix product over the
// particles p whose support reaches the block:
//   Ghat[c][row][kx] = sum_p ( f_c(p) wz_p(z) wy_p(y) ) * Bx_p(kx),
//   Bx_p(kx) = sum_j wx_p(j) exp(-2 pi i kx (x0_p + j) / K)
// (the x B-spline weights transformed once per Update).  The 256 real values
// Re Bx(0..H), Im Bx(1..H-1) of a particle form one GEMM column; with M =
// those 256 values (two 128-row MMA tiles), N = 8 RHS x 3 components x 4
// rows = 96
// and K = the block's particles in chunks of 16, tcgen05.mma (kind::tf32,
// FP32 accumulation in tensor memory) computes the block's half spectra
// directly: no shared-memory atomics and no x FFT.  FP32 accuracy comes from
// the 3-term TF32 split a*b ~ ah*bh + ah*bl + al*bh (relative error ~1e-7 on
// the spectra, like the FP32 FFT path).
//
// Per Update (tc_build): per-block particle lists padded to whole chunks,
// each entry's 4 row weights wz*wy, and each chunk's Bx operand tile (hi and
// lo TF32 parts) already in the K-major core-matrix layout of the MMA, so a
// CTA stages a chunk with two bulk copies.
#include <algorithm>

#include "engine.h"
#include "rowblock.cuh"
#include "tc.cuh"

namespace sdt {

__global__ void k_scan(int n, int *counts, int *start);

namespace {

constexpr int kTcChunk = 16;                               // particles per MMA K chunk
constexpr int kTcBY = 2, kTcBZ = 2;                        // rows of a block along y, z
constexpr int kTcRows = kTcBY * kTcBZ;                     // rows of a block (4)
constexpr int kTcRhs = kTcRhsPerCta;                       // right-hand sides per CTA
constexpr int kTcCols = kTcRhs * 3 * kTcRows;              // N of the MMA (96)
constexpr int kTcThreads = 256;

// Blocks a particle's support reaches: z pieces x y pieces.
constexpr int kTcMaxParts = 5;  // pieces of p <= 8 consecutive rows in blocks of 2
struct BlockParts {
    int ny, nz, yb[kTcMaxParts], ylo[kTcMaxParts], yhi[kTcMaxParts], zb[kTcMaxParts], zlo[kTcMaxParts],
        zhi[kTcMaxParts];
};

__device__ __forceinline__ void block_parts(int b, int p, int K, BlockParts &bp)
{
    bp.ny = axis_parts<kTcBY, kTcMaxParts>((b >> 10) & 1023, p, K, bp.yb, bp.ylo, bp.yhi);
    bp.nz = axis_parts<kTcBZ, kTcMaxParts>(b >> 20, p, K, bp.zb, bp.zlo, bp.zhi);
}

__global__ void k_tc_count(int n, int p, int K, int nby, const int *__restrict__ sp_base, int *__restrict__ cnt)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    BlockParts bp;
    block_parts(sp_base[s], p, K, bp);
    for (int a = 0; a < bp.nz; a++)
        for (int c = 0; c < bp.ny; c++) atomicAdd(&cnt[bp.zb[a] * nby + bp.yb[c]], 1);
}

__global__ void k_tc_pad(int nblk, int *__restrict__ cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nblk) cnt[i] = (cnt[i] + kTcChunk - 1) / kTcChunk * kTcChunk;
}

// Entries of particle s: slot and the 32 row weights of each block it reaches
// (the cursors start at the block starts; padding entries keep slot -1 and
// zero weights).
__global__ void k_tc_fill(int n, int p, int K, int nby, const int *__restrict__ sp_base,
                          const float *__restrict__ sp_w, int *__restrict__ cursor, int *__restrict__ slot,
                          float *__restrict__ wrow)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int b = sp_base[s];
    const int by0 = (b >> 10) & 1023, bz0 = b >> 20;
    const float *w = sp_w + (size_t)s * 3 * kMaxOrder;
    BlockParts bp;
    block_parts(b, p, K, bp);
    for (int a = 0; a < bp.nz; a++)
        for (int c = 0; c < bp.ny; c++) {
            const int idx = atomicAdd(&cursor[bp.zb[a] * nby + bp.yb[c]], 1);
            slot[idx] = s;
            float *wr = wrow + (size_t)idx * kTcRows;
            for (int row = 0; row < kTcRows; row++) {
                const int lz = row / kTcBY, ly = row % kTcBY;
                const int jz = (kTcBZ * bp.zb[a] + lz - bz0) & (K - 1);
                const int jy = (kTcBY * bp.yb[c] + ly - by0) & (K - 1);
                wr[row] = (jz < p && jy < p) ? w[2 * kMaxOrder + jz] * w[kMaxOrder + jy] : 0.0f;
            }
        }
}

// Bx operand tiles.  Row m < K of a chunk's operand: m <= H -> Re Bx(m),
// m > H -> Im Bx(m - H); rows 0..127 form MMA tile 0, rows 128..255 tile 1.
// Chunk q: [hi/lo][K][kTcChunk] floats, each 128-row tile K-major.  One
// thread per tile float, in memory order, so the stores are coalesced.
template <int K>
__global__ void k_tc_bx(long long nent, int p, const int *__restrict__ slot, const int *__restrict__ sp_base,
                        const float *__restrict__ sp_w, const float2 *__restrict__ tw, float *__restrict__ bx)
{
    constexpr int H = K / 2;
    static_assert(K == 256 && kTcChunk == 16, "two 128-row tiles, 16-entry chunks");
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nent * K) return;
    // memory order within a tile: (m / 8, k / 4, m % 8, k % 4)
    const int e4 = (int)(t & 3), m8 = (int)((t >> 2) & 7), k4 = (int)((t >> 5) & 3), mg = (int)((t >> 7) & 15);
    const int mt = (int)((t >> 11) & 1);
    const long long chunk = t >> 12;
    const int k = k4 * 4 + e4, m = mt * 128 + mg * 8 + m8;
    const int s = slot[chunk * kTcChunk + k];
    if (s < 0) return;  // padding stays zero
    const int x0 = sp_base[s] & 1023;
    const float *wx = sp_w + (size_t)s * 3 * kMaxOrder;
    const int kx = m <= H ? m : m - H;
    float re = 0.0f, im = 0.0f;
    for (int j = 0; j < p; j++) {
        const float2 w = __ldg(&tw[(kx * (x0 + j)) & (K - 1)]);  // exp(-2 pi i kx (x0 + j) / K)
        re = fmaf(wx[j], w.x, re);
        im = fmaf(wx[j], w.y, im);
    }
    const float v = m <= H ? re : im;
    const float hi = tf32_round(v), lo = tf32_round(v - hi);
    float *tile = bx + chunk * (2LL * K * kTcChunk);
    const int off = (int)(t & 4095);  // = (m / 128) * 128 * kTcChunk + tc_kmajor_offset(m % 128, k, kTcChunk) / 4
    tile[off] = hi;
    tile[K * kTcChunk + off] = lo;
}

// One CTA per (RHS, row block), two pipeline stages of one chunk each:
// while chunk c is staged and its MMAs run, the bulk copy of chunk c + 1 is
// in flight into the other stage (issued as soon as the MMAs of chunk c - 1
// have released that stage).  Per chunk: form the force x row-weight operand
// (hi/lo), issue 3 x (kTcChunk / 8) x (K / 128) MMAs, commit to the stage's
// barrier.  Then write the 96 half-spectrum rows from tensor memory.
template <int K>
__global__ void __launch_bounds__(kTcThreads, 2)
k_spread_tc(int n, int nby, const int *__restrict__ tc_start, const int *__restrict__ tc_slot,
            const float *__restrict__ tc_w, const float *__restrict__ tc_bx, const float *__restrict__ fs_sp,
            int XS, float2 *__restrict__ cgrid, int r0, int nr, int *err)
{
    static_assert(K == 256, "two 128-row tiles: Re Bx(0..127) | Re Bx(128), Im Bx(1..127)");
    constexpr int H = K / 2;
    constexpr int MT = K / 128;
    constexpr int A_FL = K * kTcChunk;        // floats of one (hi or lo) Bx tile set
    constexpr int B_FL = kTcCols * kTcChunk;  // floats of one (hi or lo) force operand
    constexpr int W_FL = kTcChunk * kTcRows;
    constexpr int F_FL = kTcRhs * 3 * kTcChunk;
    constexpr int STAGE = 2 * A_FL + 2 * B_FL + W_FL + F_FL;  // floats per stage
    constexpr uint32_t kLbo = 128, kSbo = (kTcChunk / 4) * 128;
    constexpr uint32_t kLoadBytes = (uint32_t)((2 * A_FL + W_FL) * sizeof(float));
    extern __shared__ __align__(1024) float smf[];  // 2 stages of [A hi|A lo|B hi|B lo|W|F]
    __shared__ uint64_t bar_ld[2], bar_mma[2];
    __shared__ uint32_t tmem_base;
    const int by = blockIdx.x, bz = blockIdx.y;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int blk = bz * nby + by;
    const int q0 = tc_start[blk], q1 = tc_start[blk + 1];
    const int nch = (q1 - q0) / kTcChunk;
    // the CTA takes every RHS group of its row block in turn, so each group
    // after the first reads the block's operand tiles back from L2; steps
    // s = g * nch + c run group g, chunk c through one pipeline
    const int ngrp = (nr + kTcRhs - 1) / kTcRhs;
    const int nsteps = nch * ngrp;
    if (warp == 0) tc_alloc(&tmem_base, 256);
    if (tid == 0) {
        for (int i = 0; i < 2; i++) {
            mbar_init(&bar_ld[i], 1);
            mbar_init(&bar_mma[i], 1);
        }
        fence_barrier_init();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tbase = tmem_base;
    constexpr uint32_t idesc = tc_idesc_tf32(128, kTcCols);
    auto issue_load = [&](int step) {
        float *st = smf + (step & 1) * STAGE;
        const int q = q0 + (step % nch) * kTcChunk;
        mbar_arrive_expect_tx(&bar_ld[step & 1], kLoadBytes);
        bulk_load(st, tc_bx + (size_t)(q / kTcChunk) * 2 * A_FL, (uint32_t)(2 * A_FL * sizeof(float)),
                  &bar_ld[step & 1]);
        bulk_load(st + 2 * A_FL + 2 * B_FL, tc_w + (size_t)q * kTcRows, (uint32_t)(W_FL * sizeof(float)),
                  &bar_ld[step & 1]);
    };
    if (tid == 0 && nsteps > 0) issue_load(0);
    // forces of the next step, gathered one step ahead (slot -> force is two
    // dependent loads; they overlap the current step's work); value
    // t = tid + u * kTcThreads is RHS rl, component c, entry k with
    // t = (rl * 3 + c) * kTcChunk + k
    constexpr int FPT = (F_FL + kTcThreads - 1) / kTcThreads;
    const int fk = tid % kTcChunk;
    float fnext[FPT];
    auto gather_forces = [&](int step) {
        const int rb = (step / nch) * kTcRhs;
        const int s = tc_slot[q0 + (step % nch) * kTcChunk + fk];
#pragma unroll
        for (int u = 0; u < FPT; u++) {
            const int t = tid + u * kTcThreads, fcc = t / kTcChunk, frl = fcc / 3;
            fnext[u] = (t < F_FL && rb + frl < nr && s >= 0)
                           ? fs_sp[(size_t)(3 * (r0 + rb + frl) + fcc % 3) * n + s]
                           : 0.0f;
        }
    };
#pragma unroll
    for (int u = 0; u < FPT; u++) fnext[u] = 0.0f;
    if (nsteps > 0) gather_forces(0);
    // epilogue of RHS group g: thread (warp, lane) holds kx = 32 (warp % 4) +
    // lane of tile 0 (Re) and tile 1 (Im; lane 0 of warps 0 and 4 holds
    // Re Bx(H) instead); warps w and w + 4 read the same lanes and split the
    // columns
    auto epilogue = [&](int g, bool zero) {
        const int rb = g * kTcRhs;
        const int wq = warp & 3;
        const int kx = wq * 32 + lane;
        const uint32_t trow = tbase + ((uint32_t)(wq * 32) << 16);
        constexpr int GPW = kTcCols / 16 / (kTcThreads / 128);  // column groups per warp
#pragma unroll 1
        for (int gg = (warp >> 2) * GPW; gg < ((warp >> 2) + 1) * GPW; gg++) {
            float re[16], im[16];
            if (!zero) {
                tc_ld_32x16(trow + (uint32_t)(gg * 16), re);
                tc_ld_32x16(trow + 128u + (uint32_t)(gg * 16), im);
                tc_wait_ld();
            } else {
#pragma unroll
                for (int j = 0; j < 16; j++) re[j] = im[j] = 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int col = gg * 16 + j;
                const int cc = col / kTcRows, row = col % kTcRows, rl = cc / 3;
                const int z = kTcBZ * bz + row / kTcBY, y = kTcBY * by + row % kTcBY;
                float2 *gp = cgrid + (((size_t)(3 * (r0 + rb + rl) + cc % 3) * K + z) * K + y) * XS;
                if (rb + rl < nr) {
                    gp[kx] = make_float2(re[j], kx == 0 ? 0.0f : im[j]);
                    if (kx == 0) gp[H] = make_float2(im[j], 0.0f);
                }
            }
        }
    };
    bool ok = true;
    int fail_bar = -1;  // 0..1: a load barrier, 2..3: an MMA barrier
    int fail_par = 0;
    for (int step = 0; step < nsteps; step++) {
        const int sidx = step & 1, c = step % nch;
        float *st = smf + sidx * STAGE;
        float *sA = st, *sB = st + 2 * A_FL, *sW = sB + 2 * B_FL, *sF = sW + W_FL;
        // the other stage is free once the MMAs of step - 1 are done: fetch
        // step + 1 into it now.  The fetching thread is in the last warp, so
        // the other warps go on with this step while it waits for those MMAs.
        if (tid == kTcThreads - 32 && step + 1 < nsteps) {
            if (step >= 1 && !mbar_wait(&bar_mma[sidx ^ 1], ((step - 1) >> 1) & 1)) {
                ok = false;
                fail_bar = 2 + (sidx ^ 1);
                fail_par = ((step - 1) >> 1) & 1;
            } else {
                issue_load(step + 1);
            }
        }
#pragma unroll
        for (int u = 0; u < FPT; u++)
            if (tid + u * kTcThreads < F_FL) sF[tid + u * kTcThreads] = fnext[u];
        if (step + 1 < nsteps) gather_forces(step + 1);
        if (ok && !mbar_wait(&bar_ld[sidx], (step >> 1) & 1)) {
            ok = false;
            fail_bar = sidx;
            fail_par = (step >> 1) & 1;
        }
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        // force operand: column ((rl, c), row), K index = entry k; a warp
        // writes one 8-column x 4-entry core-matrix slab (32 consecutive floats)
        for (int v = tid; v < kTcCols * kTcChunk; v += kTcThreads) {
            const int g = v >> 5, l = v & 31;
            const int k = (g % (kTcChunk / 4)) * 4 + (l & 3), col = (g / (kTcChunk / 4)) * 8 + (l >> 2);
            const int cc = col / kTcRows, row = col % kTcRows;
            const float x = sF[cc * kTcChunk + k] * sW[k * kTcRows + row];
            const float hi = tf32_round(x), lo = tf32_round(x - hi);
            const uint32_t off = tc_kmajor_offset(col, k, kTcChunk) / 4;
            sB[off] = hi;
            sB[B_FL + off] = lo;
        }
        fence_proxy_async_smem();
        tc_fence_before_sync();
        __syncthreads();
        tc_fence_after_sync();
        if (tid == 0) {
            for (int mt = 0; mt < MT; mt++) {
                const uint32_t d = tbase + (uint32_t)(mt * 128);
#pragma unroll
                for (int s = 0; s < kTcChunk / 8; s++) {
                    const float *ah = sA + mt * 128 * kTcChunk + s * 64, *al = ah + A_FL;
                    const float *bh = sB + s * 64, *bl = bh + B_FL;
                    const uint64_t dah = tc_smem_desc(ah, kLbo, kSbo), dal = tc_smem_desc(al, kLbo, kSbo);
                    const uint64_t dbh = tc_smem_desc(bh, kLbo, kSbo), dbl = tc_smem_desc(bl, kLbo, kSbo);
                    tc_mma_tf32(d, dah, dbh, idesc, !(c == 0 && s == 0));
                    tc_mma_tf32(d, dah, dbl, idesc, true);
                    tc_mma_tf32(d, dal, dbh, idesc, true);
                }
            }
            tc_commit(&bar_mma[sidx]);
        }
        if (c == nch - 1) {
            // last chunk of the group: wait for its MMAs, write the group's
            // spectra, and release the accumulators for the next group
            if (tid == 0 && !mbar_wait(&bar_mma[sidx], (step >> 1) & 1)) {
                ok = false;
                fail_bar = 2 + sidx;
                fail_par = (step >> 1) & 1;
            }
            if (!__syncthreads_and(ok)) {
                ok = false;
                break;
            }
            tc_fence_after_sync();
            epilogue(step / nch, false);
            tc_fence_before_sync();
            __syncthreads();
        }
    }
    if (!ok) {
        // a copy or MMAs did not complete in time: let them land (bounded)
        // before the tensor memory and the shared memory are given up
        if (fail_bar >= 0) {
            atomicExch(err, kTmaErrTimeout);
            mbar_wait(fail_bar < 2 ? &bar_ld[fail_bar] : &bar_mma[fail_bar - 2], fail_par);
        }
        tc_fence_before_sync();
        __syncthreads();
        if (warp == 0) tc_dealloc(tbase, 256);
        return;
    }
    if (nch == 0)
        for (int g = 0; g < ngrp; g++) epilogue(g, true);
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tc_dealloc(tbase, 256);
}

}  // namespace

void tc_free(SpmeEngine *e)
{
    cudaFree(e->d_tc_cnt);
    cudaFree(e->d_tc_start);
    cudaFree(e->d_tc_slot);
    cudaFree(e->d_tc_w);
    cudaFree(e->d_tc_bx);
    e->d_tc_cnt = e->d_tc_start = e->d_tc_slot = nullptr;
    e->d_tc_w = e->d_tc_bx = nullptr;
    e->tc_cap = 0;
    e->tc_ready = false;
}

int tc_build(SpmeEngine *e)
{
    e->tc_ready = false;
    if (!e->tc_enabled || e->K != 256) return kOk;
    const int n = e->npos, tby = e->K / kTcBY, nblk = tby * (e->K / kTcBZ);
    cudaStream_t s = e->stream;
    if (!e->d_tc_cnt) {
        SDT_CUDA(cudaMalloc(&e->d_tc_cnt, (size_t)nblk * sizeof(int)));
        SDT_CUDA(cudaMalloc(&e->d_tc_start, ((size_t)nblk + 1) * sizeof(int)));
    }
    SDT_CUDA(cudaMemsetAsync(e->d_tc_cnt, 0, (size_t)nblk * sizeof(int), s));
    k_tc_count<<<(n + 255) / 256, 256, 0, s>>>(n, e->p, e->K, tby, e->d_sp_base, e->d_tc_cnt);
    SDT_LAUNCH_CHECK();
    k_tc_pad<<<(nblk + 255) / 256, 256, 0, s>>>(nblk, e->d_tc_cnt);
    SDT_LAUNCH_CHECK();
    k_scan<<<1, 1024, 0, s>>>(nblk, e->d_tc_cnt, e->d_tc_start);
    SDT_LAUNCH_CHECK();
    int total = 0;
    SDT_CUDA(cudaMemcpyAsync(&total, e->d_tc_start + nblk, sizeof(int), cudaMemcpyDeviceToHost, s));
    SDT_CUDA(cudaStreamSynchronize(s));
    const long long nent = total;
    if (nent > e->tc_cap) {
        cudaFree(e->d_tc_slot);
        cudaFree(e->d_tc_w);
        cudaFree(e->d_tc_bx);
        e->d_tc_slot = nullptr;
        e->d_tc_w = e->d_tc_bx = nullptr;
        e->tc_cap = 0;
        const long long cap = (nent + nent / 8 + kTcChunk - 1) / kTcChunk * kTcChunk;
        if (cudaMalloc(&e->d_tc_slot, (size_t)cap * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&e->d_tc_w, (size_t)cap * kTcRows * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&e->d_tc_bx, (size_t)cap * 2 * e->K * sizeof(float)) != cudaSuccess) {
            // not enough device memory for the operand tiles: this engine
            // keeps the shared-memory spread
            cudaGetLastError();
            tc_free(e);
            e->tc_enabled = false;
            return kOk;
        }
        e->tc_cap = cap;
    }
    SDT_CUDA(cudaMemsetAsync(e->d_tc_slot, 0xff, (size_t)nent * sizeof(int), s));
    SDT_CUDA(cudaMemsetAsync(e->d_tc_w, 0, (size_t)nent * kTcRows * sizeof(float), s));
    SDT_CUDA(cudaMemsetAsync(e->d_tc_bx, 0, (size_t)nent * 2 * e->K * sizeof(float), s));
    // cursors start at the block starts (k_scan left them in the counters)
    k_tc_fill<<<(n + 255) / 256, 256, 0, s>>>(n, e->p, e->K, tby, e->d_sp_base, e->d_sp_w, e->d_tc_cnt,
                                             e->d_tc_slot, e->d_tc_w);
    SDT_LAUNCH_CHECK();
    const long long nt = nent * e->K;
    k_tc_bx<256><<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(nent, e->p, e->d_tc_slot, e->d_sp_base,
                                                             e->d_sp_w, e->d_tw_full, e->d_tc_bx);
    SDT_LAUNCH_CHECK();
    e->tc_ready = true;
    return kOk;
}

size_t spread_tc_smem(int K)
{
    return 2 * (size_t)(2 * K * kTcChunk + 2 * kTcCols * kTcChunk + kTcChunk * kTcRows + kTcRhs * 3 * kTcChunk) *
           sizeof(float);
}

int spread_tc_launch(SpmeEngine *e, int nr, int r0, cudaStream_t s)
{
    if (e->K != 256) return set_error(e, kErrUnsupported, "tensor-core spread needs K = 256");
    const size_t sm = spread_tc_smem(256);
    SDT_CUDA(cudaFuncSetAttribute(k_spread_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_spread_tc<256><<<dim3(256 / kTcBY, 256 / kTcBZ), kTcThreads, sm, s>>>(
        e->npos, 256 / kTcBY, e->d_tc_start, e->d_tc_slot, e->d_tc_w, e->d_tc_bx, e->d_fs_sp, e->XS, e->d_cgrid,
        r0, nr, e->d_err);
    SDT_LAUNCH_CHECK();
    return kOk;
}

}  // namespace sdt
