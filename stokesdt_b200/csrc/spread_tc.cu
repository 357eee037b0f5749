// Spread + x transform on the tensor cores (K = 256).
//
// For one row block (kTcBZ x kTcBY rows of (z, y)) and one RHS the
// spread followed by the real-to-complex x DFT is a matrix product over the
// particles p whose support reaches the block:
//   Ghat[c][row][kx] = sum_p ( f_c(p) wz_p(z) wy_p(y) ) * Bx_p(kx),
//   Bx_p(kx) = sum_j wx_p(j) exp(-2 pi i kx (x0_p + j) / K)
// (the x B-spline weights transformed once per Update).  The 256 real values
// Re Bx(0..H), Im Bx(1..H-1) of a particle form one GEMM column; with M =
// those 256 values (two 128-row MMA tiles), N = up to 16 RHS x 3 components
// x 4 rows = 192 and K = the block's particles in chunks of 16, tcgen05.mma
// (kind::tf32,
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

// Persistent, warp-specialised kernel: one CTA per SM walks the row blocks
// blockIdx.x, blockIdx.x + gridDim.x, ...; every block's chunks run through
// one pipeline whose stages are
//   - the copy thread (warp 0): a chunk's Bx operand tiles (hi and lo) and
//     row weights into a ring of kTcRing slots by bulk copy, as soon as the
//     MMAs have released the slot;
//   - the MMA thread (warp 1): per chunk 3 x (kTcChunk / 8) x (K / 128)
//     tcgen05 MMAs with all NRHS right-hand sides in one accumulator
//     (N = NRHS x 3 components x 4 rows), so each operand tile is read once
//     per product; commits release the slot, the force operand buffer and,
//     after a block's last chunk, the accumulator;
//   - eight builder warps: the force x row-weight operand (hi / lo) of a
//     chunk into one of two buffers (each thread builds the columns of the
//     forces it gathered one chunk ahead), and after a block's last chunk the
//     epilogue: tensor memory -> half-spectrum rows in HBM.
// mbarriers connect the stages; every wait is bounded, and a wait that gives
// up sets the error word and an abort flag that ends the other stages'
// waits, so the CTA always reaches its final barrier and frees its tensor
// memory after its copies and MMAs have landed.
constexpr int kTcRing = 3;                          // chunks whose operand tiles are in flight
constexpr int kTcBuildWarps = 8;
constexpr int kTcBuilders = 32 * kTcBuildWarps;
constexpr int kTcThreads = 64 + kTcBuilders;        // copy warp, MMA warp, builders

// Bounded wait that also gives up once another stage has aborted.
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag)
{
    for (int i = 0; i < kMbarPollLimit; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255) == 255 && *abort_flag) return false;
    }
    *abort_flag = 1;
    return false;
}

template <int K, int NRHS>
__global__ void __launch_bounds__(kTcThreads, 1)
k_spread_tc(int n, int nby, int nblk, const int *__restrict__ tc_start, const int *__restrict__ tc_slot,
            const float *__restrict__ tc_w, const float *__restrict__ tc_bx, const float *__restrict__ fs_sp,
            int XS, float2 *__restrict__ cgrid, int r0, int nr, int *err)
{
    static_assert(K == 256, "two 128-row tiles: Re Bx(0..127) | Re Bx(128), Im Bx(1..127)");
    constexpr int H = K / 2;
    constexpr int MT = K / 128;
    constexpr int NCOL = NRHS * 3 * kTcRows;      // N of the MMA
    constexpr int A_FL = K * kTcChunk;            // floats of one (hi or lo) Bx tile set
    constexpr int W_FL = kTcChunk * kTcRows;
    constexpr int SLOT = 2 * A_FL + W_FL;         // ring slot: A hi | A lo | row weights
    constexpr int B_FL = NCOL * kTcChunk;         // floats of one (hi or lo) force operand
    constexpr int NF = NRHS * 3 * kTcChunk;       // forces of one chunk
    constexpr int FPT = (NF + kTcBuilders - 1) / kTcBuilders;
    constexpr uint32_t kLbo = 128, kSbo = (kTcChunk / 4) * 128;
    constexpr uint32_t kLoadBytes = (uint32_t)(SLOT * sizeof(float));
    constexpr uint32_t kAccStride = 256;          // tensor-memory columns between the two M tiles
    constexpr uint32_t kTmemCols = 512;
    static_assert(NCOL <= (int)kAccStride && NCOL % 16 == 0, "accumulator fits its half of tensor memory");
    extern __shared__ __align__(1024) float smf[];  // [kTcRing][SLOT], then [2][B hi | B lo]
    float *const ring = smf;
    float *const opb = smf + kTcRing * SLOT;
    __shared__ uint64_t ring_full[kTcRing], ring_empty[kTcRing], op_full[2], op_empty[2], acc_full, acc_empty;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc_alloc(&tmem_base, kTmemCols);
    if (tid == 0) {
        for (int i = 0; i < kTcRing; i++) {
            mbar_init(&ring_full[i], 1);
            mbar_init(&ring_empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(&op_full[i], kTcBuildWarps);  // one arrive per builder warp
            mbar_init(&op_empty[i], 1);
        }
        mbar_init(&acc_full, 1);
        mbar_init(&acc_empty, kTcBuildWarps);
        abort_flag = 0;
        fence_barrier_init();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tbase = tmem_base;
    volatile int *abort = &abort_flag;
    auto chunks = [&](int b, int &q0) {
        q0 = tc_start[b];
        return (tc_start[b + 1] - q0) / kTcChunk;
    };

    if (warp == 0) {
        // ---- copy thread
        if (lane == 0) {
            int step = 0;
            bool ok = true;
            for (int b = blockIdx.x; b < nblk && ok; b += gridDim.x) {
                int q0;
                const int nch = chunks(b, q0);
                for (int c = 0; c < nch; c++, step++) {
                    const int s = step % kTcRing, u = step / kTcRing;
                    if (!tc_wait(&ring_empty[s], (u & 1) ^ 1, abort)) {
                        ok = false;
                        break;
                    }
                    float *dst = ring + s * SLOT;
                    const int q = q0 + c * kTcChunk;
                    mbar_arrive_expect_tx(&ring_full[s], kLoadBytes);
                    bulk_load(dst, tc_bx + (size_t)(q / kTcChunk) * 2 * A_FL, (uint32_t)(2 * A_FL * sizeof(float)),
                              &ring_full[s]);
                    bulk_load(dst + 2 * A_FL, tc_w + (size_t)q * kTcRows, (uint32_t)(W_FL * sizeof(float)),
                              &ring_full[s]);
                }
            }
            if (!ok) atomicExch(err, kTmaErrTimeout);
            // every copy issued must land before the CTA ends (the last
            // kTcRing copies are the only ones that may still be in flight)
            for (int i = step > kTcRing ? step - kTcRing : 0; i < step; i++)
                mbar_wait(&ring_full[i % kTcRing], (i / kTcRing) & 1);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---- MMA thread
        if (lane == 0) {
            constexpr uint32_t idesc = tc_idesc_tf32(128, NCOL);
            int step = 0, j = 0;
            bool ok = true;
            for (int b = blockIdx.x; b < nblk && ok; b += gridDim.x) {
                int q0;
                const int nch = chunks(b, q0);
                if (nch == 0) continue;
                if (!tc_wait(&acc_empty, (j & 1) ^ 1, abort)) {
                    ok = false;
                    break;
                }
                tc_fence_after_sync();
                for (int c = 0; c < nch; c++, step++) {
                    const int s = step % kTcRing, u = step / kTcRing, ob = step & 1, v = step >> 1;
                    if (!tc_wait(&ring_full[s], u & 1, abort) || !tc_wait(&op_full[ob], v & 1, abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after_sync();
                    const float *sA = ring + s * SLOT;
                    const float *sB = opb + ob * 2 * B_FL;
                    for (int mt = 0; mt < MT; mt++) {
                        const uint32_t d = tbase + (uint32_t)mt * kAccStride;
#pragma unroll
                        for (int ks = 0; ks < kTcChunk / 8; ks++) {
                            const float *ah = sA + mt * 128 * kTcChunk + ks * 64, *al = ah + A_FL;
                            const float *bh = sB + ks * 64, *bl = bh + B_FL;
                            const uint64_t dah = tc_smem_desc(ah, kLbo, kSbo), dal = tc_smem_desc(al, kLbo, kSbo);
                            const uint64_t dbh = tc_smem_desc(bh, kLbo, kSbo), dbl = tc_smem_desc(bl, kLbo, kSbo);
                            tc_mma_tf32(d, dah, dbh, idesc, !(c == 0 && ks == 0));
                            tc_mma_tf32(d, dah, dbl, idesc, true);
                            tc_mma_tf32(d, dal, dbh, idesc, true);
                        }
                    }
                    tc_commit(&op_empty[ob]);
                    tc_commit(&ring_empty[s]);
                }
                if (!ok) break;
                tc_commit(&acc_full);
                j++;
            }
            if (!ok) atomicExch(err, kTmaErrTimeout);
            // the MMAs issued last must complete before the CTA ends
            if (step > 0) mbar_wait(&op_empty[(step - 1) & 1], ((step - 1) >> 1) & 1);
        }
        __syncwarp();
    } else {
        // ---- builders: force operand per chunk, epilogue per block
        const int bt = tid - 64;
        const int q4 = warp & 3;                         // tensor-memory lane quarter of this warp
        const int half = (warp - 2) >> 2;                // which half of the column groups it writes
        // forces for (component column cc, entry k) = (idx / 16, idx % 16),
        // idx = bt + u * 256, in two stages a chunk apart so no load waits
        // on another inside a chunk: the entries' particle slots two chunks
        // ahead, their forces one chunk ahead
        // per-thread constants: entry k of each force, the force row in
        // fs_sp (null for columns past nr or past NF) and the operand offset
        // of its row 0 (rows 1..3 follow at +4 floats: columns 4 cc .. 4 cc
        // + 3 share one 8-row core-matrix group)
        int fk[FPT];
        const float *frow[FPT];
        uint32_t foff[FPT];
#pragma unroll
        for (int u = 0; u < FPT; u++) {
            const int idx = bt + u * kTcBuilders, cc = idx / kTcChunk;
            fk[u] = idx % kTcChunk;
            frow[u] = (idx < NF && cc / 3 < nr) ? fs_sp + (size_t)(3 * r0 + cc) * n : nullptr;
            foff[u] = idx < NF ? tc_kmajor_offset(cc * kTcRows, fk[u], kTcChunk) / 4 : 0u;
        }
        static_assert(kTcRows == 4, "a column's 4 rows are one 16-byte group of row weights");
        auto load_slots = [&](int qc, int (&sl)[FPT]) {
#pragma unroll
            for (int u = 0; u < FPT; u++) sl[u] = (qc >= 0 && frow[u]) ? tc_slot[qc + fk[u]] : -1;
        };
        auto load_forces = [&](const int (&sl)[FPT], float (&f)[FPT]) {
#pragma unroll
            for (int u = 0; u < FPT; u++) f[u] = sl[u] >= 0 ? frow[u][sl[u]] : 0.0f;
        };
        const size_t kkx = (size_t)K * K * XS;  // one (RHS, component) grid
        auto epilogue = [&](int b, bool zero) {
            const int by = b % nby, bz = b / nby;
            const int kx = q4 * 32 + lane;
            // row (z, y) = (2 bz + row / 2, 2 by + row % 2) of component grid 3 r0 + cc
            float2 *const base = cgrid + (size_t)3 * r0 * kkx + ((size_t)kTcBZ * bz * K + kTcBY * by) * XS + kx;
            const uint32_t trow = tbase + ((uint32_t)(q4 * 32) << 16);
            constexpr int NG = NCOL / 16;
#pragma unroll 1
            for (int gg = half * (NG / 2); gg < (half + 1) * (NG / 2) + (half ? NG % 2 : 0); gg++) {
                float re[16], im[16];
                if (!zero) {
                    tc_ld_32x16(trow + (uint32_t)(gg * 16), re);
                    tc_ld_32x16(trow + kAccStride + (uint32_t)(gg * 16), im);
                    tc_wait_ld();
                } else {
#pragma unroll
                    for (int jj = 0; jj < 16; jj++) re[jj] = im[jj] = 0.0f;
                }
#pragma unroll
                for (int jj = 0; jj < 16; jj++) {
                    const int cc = gg * (16 / kTcRows) + jj / kTcRows, row = jj % kTcRows;
                    float2 *gp = base + (size_t)cc * kkx + ((size_t)(row / kTcBY) * K + row % kTcBY) * XS;
                    if (cc / 3 < nr) {
                        gp[0] = make_float2(re[jj], kx == 0 ? 0.0f : im[jj]);
                        if (kx == 0) gp[H] = make_float2(im[jj], 0.0f);
                    }
                }
            }
        };
        // lookahead cursor over the walk's chunks (empty blocks skipped);
        // q = -1 past the end
        struct Cursor {
            int b, q0, nch, c;
        };
        auto advance = [&](Cursor &u) {
            if (u.b >= nblk) return;
            u.c++;
            while (u.c >= u.nch) {
                u.b += gridDim.x;
                if (u.b >= nblk) return;
                u.nch = chunks(u.b, u.q0);
                u.c = 0;
            }
        };
        auto q_of = [&](const Cursor &u) { return u.b < nblk ? u.q0 + u.c * kTcChunk : -1; };
        Cursor la{(int)blockIdx.x, 0, 0, -1};
        if (la.b < nblk) la.nch = chunks(la.b, la.q0);
        advance(la);  // step 0
        int snext[FPT];
        float fcur[FPT], fnext[FPT];
        load_slots(q_of(la), snext);
        load_forces(snext, fnext);  // step 0 (waits once, before the first chunk)
        advance(la);                // step 1
        load_slots(q_of(la), snext);
        int step = 0, j = 0;
        bool ok = true;
        for (int b = blockIdx.x; b < nblk && ok; b += gridDim.x) {
            int q0;
            const int nch = chunks(b, q0);
            if (nch == 0) {
                epilogue(b, true);
                continue;
            }
            for (int c = 0; c < nch; c++, step++) {
#pragma unroll
                for (int u = 0; u < FPT; u++) fcur[u] = fnext[u];
                load_forces(snext, fnext);  // step + 1 (slots loaded a chunk ago)
                advance(la);                // step + 2
                load_slots(q_of(la), snext);
                const int s = step % kTcRing, u = step / kTcRing, ob = step & 1, v = step >> 1;
                // every lane waits; the warp leaves together (its arrive and
                // tensor-memory loads are warp-wide)
                bool w_ok = tc_wait(&ring_full[s], u & 1, abort);
                if (w_ok) w_ok = tc_wait(&op_empty[ob], (v & 1) ^ 1, abort);
                if (!__all_sync(0xffffffffu, w_ok)) {
                    ok = false;
                    break;
                }
                const float *sW = ring + s * SLOT + 2 * A_FL;
                float *bh = opb + ob * 2 * B_FL, *bl = bh + B_FL;
#pragma unroll
                for (int uu = 0; uu < FPT; uu++) {
                    if (bt + uu * kTcBuilders < NF) {
                        const float4 w = *reinterpret_cast<const float4 *>(sW + fk[uu] * kTcRows);
                        const float x[4] = {fcur[uu] * w.x, fcur[uu] * w.y, fcur[uu] * w.z, fcur[uu] * w.w};
#pragma unroll
                        for (int row = 0; row < kTcRows; row++) {
                            const float hi = tf32_round(x[row]), lo = tf32_round(x[row] - hi);
                            bh[foff[uu] + 4 * row] = hi;
                            bl[foff[uu] + 4 * row] = lo;
                        }
                    }
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&op_full[ob]);
            }
            if (!ok) break;
            if (!__all_sync(0xffffffffu, tc_wait(&acc_full, j & 1, abort))) {
                ok = false;
                break;
            }
            tc_fence_after_sync();
            epilogue(b, false);
            tc_fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty);
            j++;
        }
        if (!ok) atomicExch(err, kTmaErrTimeout);
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tc_dealloc(tbase, kTmemCols);
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

// Dynamic shared memory of k_spread_tc<K, nrhs>: the copy ring and two force
// operand buffers.
static size_t spread_tc_smem(int K, int nrhs)
{
    const size_t ncol = (size_t)nrhs * 3 * kTcRows;
    return ((size_t)kTcRing * (2 * K * kTcChunk + kTcChunk * kTcRows) + 4 * ncol * kTcChunk) * sizeof(float);
}

template <int NRHS>
static int spread_tc_launch_n(SpmeEngine *e, int nr, int r0, int nsm, cudaStream_t s)
{
    const size_t sm = spread_tc_smem(256, NRHS);
    SDT_CUDA(cudaFuncSetAttribute(k_spread_tc<256, NRHS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int nby = 256 / kTcBY, nblk = nby * (256 / kTcBZ);
    k_spread_tc<256, NRHS><<<std::min(nsm, nblk), kTcThreads, sm, s>>>(e->npos, nby, nblk, e->d_tc_start,
                                                                        e->d_tc_slot, e->d_tc_w, e->d_tc_bx,
                                                                        e->d_fs_sp, e->XS, e->d_cgrid, r0, nr,
                                                                        e->d_err);
    SDT_LAUNCH_CHECK();
    return kOk;
}

int spread_tc_launch(SpmeEngine *e, int nr, int r0, cudaStream_t s)
{
    if (e->K != 256) return set_error(e, kErrUnsupported, "tensor-core spread needs K = 256");
    int nsm = 0;
    SDT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device));
    // up to 16 RHS per launch, all in one accumulator (N = 96 for <= 8)
    for (int g0 = 0; g0 < nr; g0 += 16) {
        const int gn = std::min(16, nr - g0);
        const int st = gn > 8 ? spread_tc_launch_n<16>(e, gn, r0 + g0, nsm, s)
                              : spread_tc_launch_n<8>(e, gn, r0 + g0, nsm, s);
        if (st != kOk) return st;
    }
    return kOk;
}

}  // namespace sdt
