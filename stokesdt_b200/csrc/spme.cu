// SPME Rotne-Prager-Yamakawa mobility on one B200: engine set-up, particle
// binning and the reciprocal-space pipeline.
//
// Reference semantics (paths relative to the StokesDT project):
//   CreateSpmeEngine_  src/mob/spme.cc:512-690   -> spme_create
//   ComputeSpline      src/mob/spme.cc:71-160    -> influence tables
//   UpdateSpmeEngine_  src/mob/spme.cc:366-509   -> spme_update (k_prep ...)
//   ComputeSpmeRecip_  src/mob/spme.cc:714-839   -> recip_chunk
//   MobSpme::MulVector src/mob/mob_spme.cc:219-236 -> spme_mulvec
//
// Grid layout in HBM: one complex half-spectrum per (RHS, component),
// cgrid[rc][z][y][kx], kx < K/2+1 padded to XS (multiple of 4 complex, so every
// row starts on a 32-byte sector).  The real-space grid never reaches HBM:
// spreading writes shared-memory rows that the x-direction real-to-complex FFT
// consumes in the same kernel, and the inverse x transform feeds the
// interpolation the same way.  Per RHS the passes move 8 x |cgrid| bytes:
//   k_spread_xfwd (write), k_ypass fwd (rw), k_zpass_influence (rw),
//   k_ypass inv (rw), k_xinv_interp (read).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "engine.h"
#include "packed.h"
#include "fft.cuh"
#include "tma.cuh"
#include "rowblock.cuh"

namespace sdt {

std::atomic<unsigned long long> g_kernel_launches{0};

void prof_mark(SpmeEngine *e, int stage)
{
    if (e->prof_on) cudaEventRecord(e->prof_ev[stage + 1], e->stream);
}

int set_error(SpmeEngine *e, int status, const std::string &msg)
{
    if (e) e->last_error = msg;
    return status;
}

// ---------------------------------------------------------------------------
// Set-up: influence tables (FP64 arithmetic, stored FP32)
// ---------------------------------------------------------------------------

// BSpline(porder, x) of spme.cc:38-68 evaluated in double precision on the
// host (order recurrence over a p-entry table seeded at floor(x)+1).
static double bspline_host(int p, double x)
{
    double s[kMaxOrder + 2] = {0};
    int first = (int)std::floor(x) + 1;
    if (first >= 0 && first < p) s[first] = 1.0;
    for (int i = 2; i <= p; i++)
        for (int j = 0; j < p + 1 - i; j++)
            s[j] = ((x - j + 1.0) * s[j] + (i - x + j - 1.0) * s[j + 1]) / (i - 1.0);
    return s[0];
}

// tab[z][y][kx] = ScalarRecip(|k|) * |b(kx) b(ky) b(kz)|^2 * factor(k^2), k=0 -> 0.
// flag 0: factor = 1 - k^2/3 (monodisperse a = 1, spme.cc:239)
// flag 1: factor = 1;  flag 2: factor = -k^2/6 (spme.cc:253-293)
__global__ void k_influence_table(int K, int XS, double xi, const double *kmap,
                                  const double *bmod2, int flag, float *tab)
{
    const int H = K / 2;
    const long long total = (long long)K * K * (H + 1);
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int kx = (int)(idx % (H + 1));
        const int y = (int)((idx / (H + 1)) % K);
        const int z = (int)(idx / ((long long)(H + 1) * K));
        const double fx = kmap[kx], fy = kmap[y], fz = kmap[z];
        const double kk = fx * fx + fy * fy + fz * fz;
        double v = 0.0;
        if (kk > 0.0) {
            const double kx2 = kk / (xi * xi);
            // ScalarRecip (spme.h:114-123)
            double m2 = 6.0 * M_PI * exp(-kx2 / 4.0) / kk * (1.0 + kx2 * (0.25 + kx2 / 8.0));
            m2 *= bmod2[kx] * bmod2[y] * bmod2[z];
            if (flag == 0) m2 *= (1.0 - kk / 3.0);
            else if (flag == 2) m2 *= (-kk / 6.0);
            v = m2;
        }
        tab[((size_t)z * K + y) * XS + kx] = (float)v;
    }
}

// ---------------------------------------------------------------------------
// Update: wrap, grid base/weights, bins and cells
// ---------------------------------------------------------------------------

// p weights M_p(x + 1 - frac), x = 0..p-1, of the cardinal B-spline of order
// p (BSpline(p, floor(c) - c + x) of spme.cc:469-473 is M_p(x - frac + 1)),
// by the order recurrence M_k(u) = (u M_{k-1}(u) + (k-u) M_{k-1}(u-1))/(k-1)
// over the p values that are nonzero on one unit interval.
__device__ __forceinline__ void spline_weights(int p, double frac, double *w)
{
    const double t = 1.0 - frac;
    w[0] = 1.0;
    for (int x = 1; x < kMaxOrder; x++) w[x] = 0.0;
    for (int k = 2; k <= p; k++) {
        for (int x = k - 1; x >= 0; x--) {
            const double cur = (x <= k - 2) ? w[x] : 0.0;
            const double left = (x >= 1) ? w[x - 1] : 0.0;
            w[x] = ((t + x) * cur + (k - t - x) * left) / (double)(k - 1);
        }
    }
}

__global__ void k_prep(int n, const double *__restrict__ pos, const double *__restrict__ rdi,
                       double L, int K, int p, int nbin, int nc, double cs,
                       int *__restrict__ key_sp, int *__restrict__ key_rs,
                       int *__restrict__ tmp_base, float *__restrict__ tmp_w,
                       double4 *__restrict__ tmp_pos, int *__restrict__ cnt_sp,
                       int *__restrict__ cnt_rs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double wpos[3];
    int base[3], cell[3];
    for (int d = 0; d < 3; d++) {
        double x = pos[3 * i + d];
        x -= L * floor(x / L);
        if (x >= L) x -= L;
        if (x < 0.0) x = 0.0;
        wpos[d] = x;
        // grid coordinate as in spme.cc:410-412
        const double u = x / L * K;
        double fl = floor(u);
        if (fl > K - 1) fl = K - 1;
        const double frac = u - fl;
        base[d] = (((int)fl - p / 2 + 1) % K + K) % K;
        double w[kMaxOrder];
        spline_weights(p, frac, w);
        for (int j = 0; j < kMaxOrder; j++)
            tmp_w[(size_t)i * 3 * kMaxOrder + d * kMaxOrder + j] = (j < p) ? (float)w[j] : 0.0f;
        int c = (int)(x / cs);
        cell[d] = c < 0 ? 0 : (c >= nc ? nc - 1 : c);
    }
    tmp_base[i] = base[0] | (base[1] << 10) | (base[2] << 20);
    const int bin = (base[2] / kRowBlock) * nbin + base[1] / kRowBlock;
    key_sp[i] = bin;
    atomicAdd(&cnt_sp[bin], 1);
    const int cidx = (cell[0] * nc + cell[1]) * nc + cell[2];
    key_rs[i] = cidx;
    atomicAdd(&cnt_rs[cidx], 1);
    tmp_pos[i] = make_double4(wpos[0], wpos[1], wpos[2], rdi ? rdi[i] : 1.0);
}

// Exclusive scan of counts[0..n) into start[0..n] by one 1024-thread block;
// counts[] is overwritten with the starts (it becomes the scatter cursor).
__global__ void __launch_bounds__(1024) k_scan(int n, int *counts, int *start)
{
    __shared__ int part[1024];
    const int tid = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int b = tid * per;
    int s = 0;
    for (int i = b; i < min(n, b + per); i++) s += counts[i];
    part[tid] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        int v = (tid >= off) ? part[tid - off] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = part[tid] - s;
    for (int i = b; i < min(n, b + per); i++) {
        const int c = counts[i];
        start[i] = run;
        counts[i] = run;
        run += c;
    }
    if (tid == 1023) start[n] = part[1023];
}

__global__ void k_scatter(int n, const int *__restrict__ key, int *__restrict__ cursor,
                          int *__restrict__ perm)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int slot = atomicAdd(&cursor[key[i]], 1);
    perm[slot] = i;
}

__global__ void k_fill_sorted(int n, const int *__restrict__ sp_perm, const int *__restrict__ rs_perm,
                              const int *__restrict__ tmp_base, const float *__restrict__ tmp_w,
                              const double4 *__restrict__ tmp_pos, const int *__restrict__ key_rs,
                              int *__restrict__ sp_base, float *__restrict__ sp_w,
                              double4 *__restrict__ rs_pos, float4 *__restrict__ rs_posf,
                              int *__restrict__ rs_cell, int *__restrict__ rs_inv)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int i = sp_perm[s];
    sp_base[s] = tmp_base[i];
    for (int j = 0; j < 3 * kMaxOrder; j++)
        sp_w[(size_t)s * 3 * kMaxOrder + j] = tmp_w[(size_t)i * 3 * kMaxOrder + j];
    const int q = rs_perm[s];
    const double4 pq = tmp_pos[q];
    rs_pos[s] = pq;
    rs_posf[s] = make_float4((float)pq.x, (float)pq.y, (float)pq.z, (float)pq.w);
    rs_cell[s] = key_rs[q];
    rs_inv[q] = s;
}

// Row segments of the x-direction kernels.  A particle with base grid index
// (bx0, by0, bz0) touches rows y = by0+jy, z = bz0+jz (jy, jz < p, mod K);
// rows are grouped in blocks of kRowBlockZ x kRowBlockY (z, y) and each
// (jz, jy) becomes one segment of its block: meta = row-in-block | x0 << 6
// (row-in-block = lz * kRowBlockY + ly), slot s, weight wz[jz]*wy[jy].  The
// segments of a particle are contiguous within each block's range.
//
__global__ void k_seg_count(int n, int p, int K, int nby, const int *__restrict__ sp_base,
                            int *__restrict__ seg_cnt)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int b = sp_base[s];
    int yb[3], ylo[3], yhi[3], zb[3], zlo[3], zhi[3];
    const int ny = axis_parts<kRowBlockY>((b >> 10) & 1023, p, K, yb, ylo, yhi);
    const int nz = axis_parts<kRowBlockZ>(b >> 20, p, K, zb, zlo, zhi);
    for (int a = 0; a < nz; a++)
        for (int c = 0; c < ny; c++)
            atomicAdd(&seg_cnt[zb[a] * nby + yb[c]], (zhi[a] - zlo[a]) * (yhi[c] - ylo[c]));
}

__global__ void k_seg_fill(int n, int p, int K, int nby, const int *__restrict__ sp_base,
                           const float *__restrict__ sp_w, const int *__restrict__ seg_start,
                           int *__restrict__ cursor, unsigned *__restrict__ seg_meta,
                           int *__restrict__ seg_slot, float *__restrict__ seg_w)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int b = sp_base[s];
    const int bx0 = b & 1023, by0 = (b >> 10) & 1023, bz0 = b >> 20;
    const float *w = sp_w + (size_t)s * 3 * kMaxOrder;
    int yb[3], ylo[3], yhi[3], zb[3], zlo[3], zhi[3];
    const int ny = axis_parts<kRowBlockY>(by0, p, K, yb, ylo, yhi);
    const int nz = axis_parts<kRowBlockZ>(bz0, p, K, zb, zlo, zhi);
    for (int a = 0; a < nz; a++)
        for (int c = 0; c < ny; c++) {
            const int blk = zb[a] * nby + yb[c];
            const int cnt = (zhi[a] - zlo[a]) * (yhi[c] - ylo[c]);
            // k_scan left cursor[blk] = seg_start[blk]: the atomic returns an
            // absolute position inside the block's range
            int q = atomicAdd(&cursor[blk], cnt);
            if (q < seg_start[blk] || q + cnt > seg_start[blk + 1]) continue;  // never true
            for (int jz = zlo[a]; jz < zhi[a]; jz++) {
                const int lz = ((bz0 + jz) & (K - 1)) - kRowBlockZ * zb[a];
                for (int jy = ylo[c]; jy < yhi[c]; jy++, q++) {
                    const int ly = ((by0 + jy) & (K - 1)) - kRowBlockY * yb[c];
                    seg_meta[q] = (unsigned)(lz * kRowBlockY + ly) | ((unsigned)bx0 << 6);
                    seg_slot[q] = s;
                    seg_w[q] = w[2 * kMaxOrder + jz] * w[kMaxOrder + jy];
                }
            }
        }
}

// ---------------------------------------------------------------------------
// Per-call kernels
//
// Occupancy: the x kernels (48 rows, 192 threads, 53 KB of rows at K=256)
// run four CTAs per SM; the y kernel (16 columns, 32 KB) four; the fused z
// kernel (3 components x 4 columns, 29 KB) six.
// ---------------------------------------------------------------------------

// FP64 caller forces -> FP32 copy in spread order, [r][c][s], optionally
// scaled per particle by `scale` (e.g. a^2).  Consecutive threads take
// consecutive slots s, so the writes are coalesced.
__global__ void k_gather_forces(int n, int nr, const double *__restrict__ f, int ldf,
                                const int *__restrict__ sp_perm, const double *__restrict__ scale,
                                float *__restrict__ fs_sp, float *__restrict__ zero)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)n * nr) return;
    const int s = (int)(idx % n);
    const int r = (int)(idx / n);
    const int i = sp_perm[s];
    const double sc = scale ? scale[i] : 1.0;
    const double *fi = f + (size_t)r * ldf + 3 * i;
    for (int c = 0; c < 3; c++) fs_sp[((size_t)r * 3 + c) * n + s] = (float)(fi[c] * sc);
    // optionally clear the [nr][3n] array the interpolation accumulates into
    if (zero)
        for (int c = 0; c < 3; c++) zero[(size_t)r * 3 * n + 3 * s + c] = 0.0f;
}

// Both force copies of a product in one launch.  Blocks [0, nb_sp) do
// k_gather_forces' work and clear the interpolation accumulator `zero`; the
// blocks after them make the FP32 copy in cell order, [s][r][4] (fourth
// float zero): one thread per particle i (coalesced reads of f), writing its
// nr float4 values contiguously at slot rs_inv[i].  A product that needs
// only one copy launches only its blocks.
__global__ void k_gather_both(int n, int nr, const double *__restrict__ f, int ldf,
                              const int *__restrict__ sp_perm, float *__restrict__ fs_sp,
                              float *__restrict__ zero, int nb_sp, const int *__restrict__ rs_inv,
                              float4 *__restrict__ fs_rs)
{
    if ((int)blockIdx.x < nb_sp) {
        const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (idx >= (long long)n * nr) return;
        const int s = (int)(idx % n);
        const int r = (int)(idx / n);
        const double *fi = f + (size_t)r * ldf + 3 * sp_perm[s];
        for (int c = 0; c < 3; c++) {
            fs_sp[((size_t)r * 3 + c) * n + s] = (float)fi[c];
            zero[(size_t)r * 3 * n + 3 * s + c] = 0.0f;
        }
        return;
    }
    const int i = (blockIdx.x - nb_sp) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 *out = fs_rs + (size_t)rs_inv[i] * nr;
    for (int r = 0; r < nr; r++) {
        const double *fi = f + (size_t)r * ldf + 3 * i;
        out[r] = make_float4((float)fi[0], (float)fi[1], (float)fi[2], 0.0f);
    }
}

template <int K>
__host__ __device__ constexpr int kXpassMinBlocks() { return K <= 256 ? 4 : 2; }
constexpr int kXThreads = 192;                             // threads of the x kernels
constexpr int kXRows = 3 * kRowBlockY * kRowBlockZ;        // rows per x-kernel CTA
// Shared-memory rows of the x kernels: row rr = (c * kRowBlockZ + lz) *
// kRowBlockY + ly (lr = rr mod 16, its place in the block) starts at
// x_row_offset = rr * (K + 16) + 2 * (lr / 2) floats.  The stride K + 16 keeps
// the two lines of a half warp in the FFT (rows 2m, 2m + 1) 16 banks apart,
// and the 2 * (lr / 2) shift gives the 16 rows of a block 16 distinct even
// bank offsets, so lanes holding one particle's segments touch the same x in
// 16 different banks (spread atomics, interpolation loads).  The inverse
// kernel stages a spectrum (H + 2 float2, whole 16-byte units) 16-byte
// aligned at x_stage_offset, 0 or 2 floats lower, and its c2r merge moves it
// into place.
template <int K>
__host__ __device__ constexpr int x_row_offset(int rr)
{
    return rr * (K + 16) + 2 * ((rr % (kRowBlockY * kRowBlockZ)) / 2);
}
template <int K>
__host__ __device__ constexpr int x_stage_offset(int rr)
{
    return rr * (K + 16) + 4 * ((rr % (kRowBlockY * kRowBlockZ)) / 4);
}
template <int K>
__host__ __device__ constexpr int x_rows_floats() { return kXRows * (K + 16); }
template <int K>
__host__ __device__ constexpr bool x_rows_fit()
{
    return x_row_offset<K>(kXRows - 1) + K <= x_rows_floats<K>() &&
           x_stage_offset<K>(kXRows - 1) + K + 4 <= x_rows_floats<K>() &&
           x_row_offset<K>(1) + K <= x_stage_offset<K>(2) && x_stage_offset<K>(1) + K + 4 <= x_row_offset<K>(2);
}
template <int K>
__host__ __device__ constexpr int kYpassMinBlocks() { return K <= 256 ? 4 : 2; }
template <int K>
__host__ __device__ constexpr int kZpassMinBlocks() { return K <= 256 ? 3 : 1; }

// X[k] of a length-2H real row from Z = FFT_H(x[2m] + i x[2m+1]):
// X[k] = (Z[k] + conj Z[H-k])/2 - i W_2H^k (Z[k] - conj Z[H-k])/2
__device__ __forceinline__ float2 r2c_split(float2 zk, float2 zm, float2 w)
{
    const float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 od = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));
    const float2 t = cmul(w, od);
    return make_float2(ev.x + t.y, ev.y - t.x);
}

// Z'[k] = (X[k] + conj X[H-k]) + i conj(W_2H^k) (X[k] - conj X[H-k]); the
// unnormalised inverse FFT_H of Z' gives x[2m] + i x[2m+1].
__device__ __forceinline__ float2 c2r_merge(float2 xk, float2 xm, float2 w)
{
    const float2 a = make_float2(xk.x + xm.x, xk.y - xm.y);
    const float2 b = make_float2(xk.x - xm.x, xk.y + xm.y);
    const float2 t = cmul(cconj(w), b);
    return make_float2(a.x - t.y, a.y + t.x);
}

// One CTA per (kRowBlockZ x kRowBlockY block of (z, y) rows, RHS): spread
// the three force components of the particles whose support reaches the
// block into kXRows shared-memory rows (component-major), FFT every row along x
// (real-to-complex) and write the half spectra.  Each row segment's index
// data and weights are loaded once for its 3 x p atomics.
// The work of one CTA: RHS r, row block (by, bz).
template <int K>
__device__ __forceinline__ void spread_xfwd_block(int n, int p, int nby, const int *__restrict__ seg_start,
                                                  const unsigned *__restrict__ seg_meta,
                                                  const int *__restrict__ seg_slot, const float *__restrict__ seg_w,
                                                  const float *__restrict__ sp_w, const float *__restrict__ fs_sp,
                                                  int XS, const float2 *__restrict__ tw_half,
                                                  const float2 *__restrict__ tw_full, float2 *__restrict__ cgrid,
                                                  int r, int by, int bz)
{
    constexpr int H = K / 2;
    constexpr int NRB = kRowBlockY * kRowBlockZ;
    static_assert(x_rows_fit<K>(), "rows fit the footprint");
    extern __shared__ __align__(128) float rows[];  // kXRows rows at x_row_offset<K>
    const int tid = threadIdx.x;
    {
        float4 *r4 = reinterpret_cast<float4 *>(rows);
        for (int i = tid; i < x_rows_floats<K>() / 4; i += kXThreads) r4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();

    // stream the block's row segments (index data of the next one in flight):
    // p contiguous shared-memory atomics per component.  Neighbouring lanes
    // usually hold segments of one particle (same x0, different rows), which
    // the row layout puts on different banks.  Two-stage software pipeline:
    // the index data of segment q + 2S and the force / x-weight gathers of
    // segment q + S are in flight while segment q's atomics run (S =
    // kXThreads).
    const float *f0 = fs_sp + (size_t)(3 * r) * n;
    const float *f1 = f0 + n, *f2 = f1 + n;
    const int blk = bz * nby + by;
    const int q1 = seg_start[blk + 1];
    static_assert(kMaxOrder == 8, "x weights are two float4");
    auto gather = [&](int sl, float w, float &a0, float &a1, float &a2, float *wr) {
        a0 = f0[sl] * w;
        a1 = f1[sl] * w;
        a2 = f2[sl] * w;
        const float4 *wx = reinterpret_cast<const float4 *>(sp_w + (size_t)sl * 3 * kMaxOrder);
        const float4 a = __ldg(wx), b = __ldg(wx + 1);
        wr[0] = a.x;
        wr[1] = a.y;
        wr[2] = a.z;
        wr[3] = a.w;
        wr[4] = b.x;
        wr[5] = b.y;
        wr[6] = b.z;
        wr[7] = b.w;
    };
    int q = seg_start[blk] + tid;
    unsigned mA = 0, mB = 0;
    int sA = 0;
    float wA = 0.0f, b0 = 0.0f, b1 = 0.0f, b2 = 0.0f, wrB[kMaxOrder];
    if (q < q1) {
        mB = seg_meta[q];
        gather(seg_slot[q], seg_w[q], b0, b1, b2, wrB);
    }
    int qn = q + kXThreads;
    if (qn < q1) {
        mA = seg_meta[qn];
        sA = seg_slot[qn];
        wA = seg_w[qn];
    }
    while (q < q1) {
        const unsigned m = mB;
        const float v0 = b0, v1 = b1, v2 = b2;
        float wc[kMaxOrder];
#pragma unroll
        for (int k = 0; k < kMaxOrder; k++) wc[k] = wrB[k];
        if (qn < q1) {
            mB = mA;
            gather(sA, wA, b0, b1, b2, wrB);
        }
        const int qnn = qn + kXThreads;
        if (qnn < q1) {
            mA = seg_meta[qnn];
            sA = seg_slot[qnn];
            wA = seg_w[qnn];
        }
        constexpr int kC = x_row_offset<K>(NRB) - x_row_offset<K>(0);  // component stride
        static_assert(x_row_offset<K>(2 * NRB) - x_row_offset<K>(NRB) == kC, "even component stride");
        float *row0 = rows + x_row_offset<K>(m & 31u);
        const int x0 = (int)(m >> 6);
        if (x0 + p <= K) {
            float *a = row0 + x0;
#pragma unroll
            for (int k = 0; k < kMaxOrder; k++) {
                if (k < p) {
                    atomicAdd(a + k, v0 * wc[k]);
                    atomicAdd(a + k + kC, v1 * wc[k]);
                    atomicAdd(a + k + 2 * kC, v2 * wc[k]);
                }
            }
        } else {  // the support wraps around x = K
#pragma unroll
            for (int k = 0; k < kMaxOrder; k++) {
                if (k < p) {
                    const int x = (x0 + k) & (K - 1);
                    atomicAdd(row0 + x, v0 * wc[k]);
                    atomicAdd(row0 + x + kC, v1 * wc[k]);
                    atomicAdd(row0 + x + 2 * kC, v2 * wc[k]);
                }
            }
        }
        q = qn;
        qn = qnn;
    }
    __syncthreads();

    // x FFT of the kXRows rows, kXThreads / N2 rows at a time
    constexpr int N2 = FftShape<H>::N2;
    constexpr int RPP = kXThreads / N2;
    static_assert(kXRows % RPP == 0, "whole row passes");
    const int t = tid % N2;
    for (int rr = tid / N2; rr < kXRows; rr += RPP)
        fft_line<H, false>(reinterpret_cast<float2 *>(rows + x_row_offset<K>(rr)), 1, t, tw_half);

    // split into the K/2+1 spectrum while writing it out, one warp per row
    // and lanes along kx: X[k] from Z[k] and Z[H-k] (X[0], X[H] from Z[0]).
    // A lane's kx (and twiddles) are the same in every row.
    {
        const int warp = tid >> 5, lane = tid & 31;
        constexpr int JW = (H + 1 + 31) / 32;
        float2 wk[JW];
#pragma unroll
        for (int j = 0; j < JW; j++) {
            const int kx = lane + 32 * j;
            wk[j] = (kx > 0 && kx < H) ? __ldg(&tw_full[kx]) : make_float2(1.0f, 0.0f);
        }
        for (int rr = warp; rr < kXRows; rr += kXThreads / 32) {
            const int c = rr / NRB, lr = rr % NRB;
            const int z = kRowBlockZ * bz + lr / kRowBlockY, y = kRowBlockY * by + lr % kRowBlockY;
            const float2 *zr = reinterpret_cast<const float2 *>(rows + x_row_offset<K>(rr));
            float2 *g = cgrid + (((size_t)(3 * r + c) * K + z) * K + y) * XS;
#pragma unroll
            for (int j = 0; j < JW; j++) {
                const int kx = lane + 32 * j;
                if (kx > H) break;
                float2 xk;
                if (kx == 0 || kx == H) {
                    const float2 z0 = zr[0];
                    xk = make_float2(kx == 0 ? z0.x + z0.y : z0.x - z0.y, 0.0f);
                } else {
                    xk = r2c_split(zr[kx], zr[H - kx], wk[j]);
                }
                g[kx] = xk;
            }
        }
    }
}

template <int K>
__global__ void __launch_bounds__(kXThreads, kXpassMinBlocks<K>())
k_spread_xfwd(int n, int p, int nby, const int *__restrict__ seg_start,
              const unsigned *__restrict__ seg_meta, const int *__restrict__ seg_slot,
              const float *__restrict__ seg_w, const float *__restrict__ sp_w,
              const float *__restrict__ fs_sp, int XS, const float2 *__restrict__ tw_half,
              const float2 *__restrict__ tw_full, float2 *__restrict__ cgrid, int r0)
{
    // the RHS index runs fastest, so the CTAs of one row block run together
    // and share its segment lists and weights through L2
    spread_xfwd_block<K>(n, p, nby, seg_start, seg_meta, seg_slot, seg_w, sp_w, fs_sp, XS, tw_half, tw_full, cgrid,
                         r0 + blockIdx.x, blockIdx.y, blockIdx.z);
}

// Packed: blockIdx.z = slot * nbz + bz; the slot's system and grid slice
// come from the class's slot table.
template <int K>
__global__ void __launch_bounds__(kXThreads, kXpassMinBlocks<K>())
k_spread_xfwd_packed(const PackedSys *__restrict__ sys, const PackedIO *__restrict__ io,
                     const int *__restrict__ slot_sys, int nbz, int XS, const float2 *__restrict__ tw_half,
                     const float2 *__restrict__ tw_full, float2 *__restrict__ grid, long long slot_stride)
{
    const int slot = blockIdx.z / nbz, bz = blockIdx.z - slot * nbz;
    const int g = slot_sys[slot];
    const PackedSys &S = sys[g];
    spread_xfwd_block<K>(S.n, S.p, S.nby, S.seg_start, S.seg_meta, S.seg_slot, S.seg_w, S.sp_w, io[g].fs_sp, XS,
                         tw_half, tw_full, grid + (size_t)slot * slot_stride, blockIdx.x, blockIdx.y, bz);
}

// Complex FFT along y of a 16-column kx tile of one z-plane, in place.
template <int K, bool INV>
__global__ void __launch_bounds__(kTileX * FftShape<K>::N2, kYpassMinBlocks<K>())
k_ypass(int XS, const float2 *__restrict__ tw, float2 *__restrict__ cgrid, int rc0)
{
    constexpr int H = K / 2;
    extern __shared__ float2 tile[];  // [K][kTileX]
    const int tx = blockIdx.x, z = blockIdx.y, rc = rc0 + blockIdx.z;
    const int tid = threadIdx.x;
    const int kx0 = tx * kTileX;
    float2 *g = cgrid + (((size_t)rc * K + z) * K) * XS;
    for (int i = tid; i < K * kTileX; i += blockDim.x) {
        const int y = i / kTileX, c = i - y * kTileX;
        tile[i] = (kx0 + c <= H) ? g[(size_t)y * XS + kx0 + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    // consecutive threads take consecutive columns (contiguous in smem)
    const int col = tid % kTileX, t = tid / kTileX;
    fft_line<K, INV>(tile + col, kTileX, t, tw);
    for (int i = tid; i < K * kTileX; i += blockDim.x) {
        const int y = i / kTileX, c = i - y * kTileX;
        if (kx0 + c <= H) g[(size_t)y * XS + kx0 + c] = tile[i];
    }
}

// Forward FFT along z, RPY influence multiply on the three components, inverse
// FFT along z: one CTA per (kx tile, ky, RHS).  B = m2 (I - k k^T / k^2) with
// m2 from `tab` (ApplyInfluence, spme.cc:201-310); the k = 0 mode is zeroed.
template <int K>
__global__ void __launch_bounds__(3 * kTileZ * FftShape<K>::N2, kZpassMinBlocks<K>())
k_zpass_influence(int XS, const float2 *__restrict__ tw, const float *__restrict__ kmap,
                  const float *__restrict__ tab, int r0, float2 *__restrict__ cgrid)
{
    constexpr int H = K / 2;
    extern __shared__ float2 sm[];  // [3][K][kTileZ]
    const int tx = blockIdx.x, y = blockIdx.y, r = r0 + blockIdx.z;
    const int tid = threadIdx.x;
    const int kx0 = tx * kTileZ;
    for (int i = tid; i < 3 * K * kTileZ; i += blockDim.x) {
        const int c = i / (K * kTileZ);
        const int rem = i - c * K * kTileZ;
        const int z = rem / kTileZ, cc = rem - z * kTileZ;
        const float2 *g = cgrid + (((size_t)(r * 3 + c) * K + z) * K + y) * XS;
        sm[i] = (kx0 + cc <= H) ? g[kx0 + cc] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    constexpr int N2 = FftShape<K>::N2;
    // consecutive threads take consecutive columns of one component
    const int col = tid % kTileZ, t = (tid / kTileZ) % N2, c = tid / (kTileZ * N2);
    float2 *base = sm + c * K * kTileZ + col;
    fft_line<K, false>(base, kTileZ, t, tw);

    const float fky = kmap[y];
    for (int i = tid; i < K * kTileZ; i += blockDim.x) {
        const int z = i / kTileZ, cc = i - z * kTileZ;
        const int kx = kx0 + cc;
        if (kx > H) continue;
        const float fkx = kmap[kx], fkz = kmap[z];
        const float m2 = tab[((size_t)z * K + y) * XS + kx];
        const float kk = fkx * fkx + fky * fky + fkz * fkz;
        float2 g0 = sm[i], g1 = sm[K * kTileZ + i], g2 = sm[2 * K * kTileZ + i];
        if (kk > 0.0f) {
            const float inv = 1.0f / kk;
            const float dr = (fkx * g0.x + fky * g1.x + fkz * g2.x) * inv;
            const float di = (fkx * g0.y + fky * g1.y + fkz * g2.y) * inv;
            g0 = make_float2(m2 * (g0.x - fkx * dr), m2 * (g0.y - fkx * di));
            g1 = make_float2(m2 * (g1.x - fky * dr), m2 * (g1.y - fky * di));
            g2 = make_float2(m2 * (g2.x - fkz * dr), m2 * (g2.y - fkz * di));
        } else {
            g0 = g1 = g2 = make_float2(0.f, 0.f);
        }
        sm[i] = g0;
        sm[K * kTileZ + i] = g1;
        sm[2 * K * kTileZ + i] = g2;
    }
    __syncthreads();
    fft_line<K, true>(base, kTileZ, t, tw);
    for (int i = tid; i < 3 * K * kTileZ; i += blockDim.x) {
        const int c2 = i / (K * kTileZ);
        const int rem = i - c2 * K * kTileZ;
        const int z = rem / kTileZ, cc = rem - z * kTileZ;
        if (kx0 + cc <= H) {
            float2 *g = cgrid + (((size_t)(r * 3 + c2) * K + z) * K + y) * XS;
            g[kx0 + cc] = sm[i];
        }
    }
}

// ---------------------------------------------------------------------------
// TMA-staged y and z passes.  Same transforms as k_ypass / k_zpass_influence;
// the tile arrives by one tiled bulk load per 256 lines (completing on an
// mbarrier) and leaves by tiled bulk stores, so each CTA has its whole tile
// in flight at once instead of one 8-byte load per thread and line.
// Tensor maps view the grid as float2 elements: y pass [plane][y][x] with
// plane = (rhs*3 + c)*K + z; z pass [rhs*3 + c][z][y][x].
// ---------------------------------------------------------------------------
constexpr int kTmaBoxLines = 256;  // largest box extent of a tiled copy

template <int K, bool INV>
__global__ void __launch_bounds__(kTileX * FftShape<K>::N2, kYpassMinBlocks<K>())
k_ypass_tma(const __grid_constant__ CUtensorMap map, const float2 *__restrict__ tw, int *err, int rc0)
{
    extern __shared__ __align__(1024) float2 tile[];  // [K][kTileX]
    __shared__ uint64_t bar;
    const int kx0 = blockIdx.x * kTileX;
    const int plane = (rc0 + blockIdx.z) * K + blockIdx.y;
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(&bar, (uint32_t)(K * kTileX * sizeof(float2)));
        for (int y0 = 0; y0 < K; y0 += kTmaBoxLines) tma_load_3d(tile + y0 * kTileX, &map, &bar, kx0, y0, plane);
    }
    const bool ok = mbar_wait(&bar, 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicExch(err, kTmaErrTimeout);
        return;
    }
    const int col = tid % kTileX, t = tid / kTileX;
    fft_line<K, INV>(tile + col, kTileX, t, tw);
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
        for (int y0 = 0; y0 < K; y0 += kTmaBoxLines) tma_store_3d(&map, tile + y0 * kTileX, kx0, y0, plane);
        bulk_commit();
        bulk_wait_read_all();
    }
}

template <int K>
__global__ void __launch_bounds__(3 * kTileZ * FftShape<K>::N2, kZpassMinBlocks<K>())
k_zpass_influence_tma(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap tabmap,
                      const float2 *__restrict__ tw, const float *__restrict__ kmap, int *err, int r0)
{
    constexpr int H = K / 2;
    extern __shared__ __align__(1024) float2 sm[];  // [3][K][kTileZ], then the table tile [K][kTileZ]
    float *tabs = reinterpret_cast<float *>(sm + 3 * K * kTileZ);
    __shared__ uint64_t bar;
    const int tx = blockIdx.x, y = blockIdx.y, r = r0 + blockIdx.z;
    const int tid = threadIdx.x;
    const int kx0 = tx * kTileZ;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(&bar, (uint32_t)(3 * K * kTileZ * sizeof(float2) + K * kTileZ * sizeof(float)));
        for (int c = 0; c < 3; c++)
            for (int z0 = 0; z0 < K; z0 += kTmaBoxLines)
                tma_load_4d(sm + (c * K + z0) * kTileZ, &map, &bar, kx0, y, z0, 3 * r + c);
        for (int z0 = 0; z0 < K; z0 += kTmaBoxLines)
            tma_load_3d(tabs + z0 * kTileZ, &tabmap, &bar, kx0, y, z0);
    }
    const bool ok = mbar_wait(&bar, 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicExch(err, kTmaErrTimeout);
        return;
    }
    constexpr int N2 = FftShape<K>::N2;
    const int col = tid % kTileZ, t = (tid / kTileZ) % N2, c = tid / (kTileZ * N2);
    float2 *base = sm + c * K * kTileZ + col;
    fft_line<K, false>(base, kTileZ, t, tw);

    const float fky = kmap[y];
    for (int i = tid; i < K * kTileZ; i += blockDim.x) {
        const int z = i / kTileZ, cc = i - z * kTileZ;
        const int kx = kx0 + cc;
        if (kx > H) continue;
        const float fkx = kmap[kx], fkz = kmap[z];
        const float m2 = tabs[i];
        const float kk = fkx * fkx + fky * fky + fkz * fkz;
        float2 g0 = sm[i], g1 = sm[K * kTileZ + i], g2 = sm[2 * K * kTileZ + i];
        if (kk > 0.0f) {
            const float inv = 1.0f / kk;
            const float dr = (fkx * g0.x + fky * g1.x + fkz * g2.x) * inv;
            const float di = (fkx * g0.y + fky * g1.y + fkz * g2.y) * inv;
            g0 = make_float2(m2 * (g0.x - fkx * dr), m2 * (g0.y - fkx * di));
            g1 = make_float2(m2 * (g1.x - fky * dr), m2 * (g1.y - fky * di));
            g2 = make_float2(m2 * (g2.x - fkz * dr), m2 * (g2.y - fkz * di));
        } else {
            g0 = g1 = g2 = make_float2(0.f, 0.f);
        }
        sm[i] = g0;
        sm[K * kTileZ + i] = g1;
        sm[2 * K * kTileZ + i] = g2;
    }
    __syncthreads();
    fft_line<K, true>(base, kTileZ, t, tw);
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
        for (int c2 = 0; c2 < 3; c2++)
            for (int z0 = 0; z0 < K; z0 += kTmaBoxLines)
                tma_store_4d(&map, sm + (c2 * K + z0) * kTileZ, kx0, y, z0, 3 * r + c2);
        bulk_commit();
        bulk_wait_read_all();
    }
}

// Inverse x FFT (complex-to-real) of the 3 x 32 rows of a 4 x 8 (z, y) row
// block followed by the B-spline interpolation of the particles whose
// support reaches the block (Interpolate, spme.cc:163-198).  Partial sums go
// to vrecip[r][3i+c] by atomicAdd (FP32); `iscale` (optional) multiplies them
// per particle.
//
// BULK: the block's kXRows spectra (bins 0..H and one more float2, a whole
// number of 16-byte units) come in by untiled bulk copies on one mbarrier,
// all in flight at once, at x_stage_offset; each FFT thread merges the
// pairs (k, H-k) of its step-1 samples in registers and the transform
// writes the row at x_row_offset.  Otherwise each warp loads its rows and
// merges them on the way into shared memory before the transform.
// The work of one CTA: RHS r, row block (by, bz).
template <int K, bool BULK>
__device__ __forceinline__ void xinv_interp_block(int n, int p, int nby, const int *__restrict__ seg_start,
                                                  const unsigned *__restrict__ seg_meta,
                                                  const int *__restrict__ seg_slot, const float *__restrict__ seg_w,
                                                  const float *__restrict__ sp_w, const int *__restrict__ sp_perm,
                                                  const double *__restrict__ iscale, int XS,
                                                  const float2 *__restrict__ tw_half,
                                                  const float2 *__restrict__ tw_full,
                                                  const float2 *__restrict__ cgrid, float *__restrict__ vrecip,
                                                  int *err, int r, int by, int bz)
{
    constexpr int H = K / 2;
    constexpr int NRB = kRowBlockY * kRowBlockZ;
    constexpr uint32_t kStageBytes = (uint32_t)((H + 2) * sizeof(float2));
    static_assert(kStageBytes % 16 == 0 && x_rows_fit<K>(), "staged rows fit the footprint");
    extern __shared__ __align__(128) float rows[];  // kXRows rows at x_row_offset<K>
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    auto spectrum_row = [&](int rr) {
        const int c = rr / NRB, lr = rr % NRB;
        const int z = kRowBlockZ * bz + lr / kRowBlockY, y = kRowBlockY * by + lr % kRowBlockY;
        return cgrid + (((size_t)(3 * r + c) * K + z) * K + y) * XS;
    };
    // Z'[k] from X[k] and X[H-k]: the half-length complex input of the
    // inverse transform (the DC and Nyquist bins of a real row have no
    // imaginary part)
    constexpr int N2 = FftShape<H>::N2;
    constexpr int RPP = kXThreads / N2;
    static_assert(kXRows % RPP == 0, "whole row passes");
    if constexpr (BULK) {
        __shared__ uint64_t bar;
        if (tid == 0) {
            mbar_init(&bar, 1);
            fence_barrier_init();
            mbar_arrive_expect_tx(&bar, (uint32_t)(kXRows * kStageBytes));
        }
        __syncthreads();
        if (lane == 0)
            for (int rr = warp; rr < kXRows; rr += kXThreads / 32)
                bulk_load(rows + x_stage_offset<K>(rr), spectrum_row(rr), kStageBytes, &bar);
        const bool ok = mbar_wait(&bar, 0);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) atomicExch(err, kTmaErrTimeout);
            return;
        }
        // Z'[k] = merge(X[k], X[H-k]) is formed on the way into the inverse
        // transform: thread t of a row takes step 1's samples k = N2 j + t
        // and reads X[k] and X[H-k] from the staged spectrum.  The
        // transform's first barrier separates these reads from its writes
        // into the row, which overlaps the staging area.
        const int t = tid % N2;
        for (int rr = tid / N2; rr < kXRows; rr += RPP) {
            const float2 *sr = reinterpret_cast<const float2 *>(rows + x_stage_offset<K>(rr));
            float2 a[FftShape<H>::N1];
#pragma unroll
            for (int j = 0; j < FftShape<H>::N1; j++) {
                const int k = N2 * j + t;
                float2 xk = sr[k], xm = sr[H - k];
                float2 w = make_float2(1.0f, 0.0f);
                if (k == 0) {
                    xk.y = 0.0f;
                    xm.y = 0.0f;
                } else {
                    w = __ldg(&tw_full[k]);
                }
                a[j] = c2r_merge(xk, xm, w);
            }
            fft_line_regs<H, true>(a, reinterpret_cast<float2 *>(rows + x_row_offset<K>(rr)), 1, t, tw_half);
        }
    } else {
        constexpr int JW = (H + 31) / 32;
        float2 wk[JW];
#pragma unroll
        for (int j = 0; j < JW; j++) {
            const int k = lane + 32 * j;
            wk[j] = (k > 0 && k < H) ? __ldg(&tw_full[k]) : make_float2(1.0f, 0.0f);
        }
        for (int rr = warp; rr < kXRows; rr += kXThreads / 32) {
            const float2 *g = spectrum_row(rr);
            float2 *zr = reinterpret_cast<float2 *>(rows + x_row_offset<K>(rr));
#pragma unroll
            for (int j = 0; j < JW; j++) {
                const int k = lane + 32 * j;
                if (k >= H) break;
                float2 xk = g[k], xm = g[H - k];
                if (k == 0) {
                    xk.y = 0.0f;
                    xm.y = 0.0f;
                }
                zr[k] = c2r_merge(xk, xm, wk[j]);
            }
        }
        __syncthreads();
        const int t = tid % N2;
        for (int rr = tid / N2; rr < kXRows; rr += RPP)
            fft_line<H, true>(reinterpret_cast<float2 *>(rows + x_row_offset<K>(rr)), 1, t, tw_half);
    }

    // stream the block's row segments: three p-point dot products each,
    // summed per particle over the warp's consecutive segments (a particle's
    // segments are contiguous) and added to vrecip once per run
    float *vout = vrecip + (size_t)r * 3 * n;
    const int blk = bz * nby + by;
    const int q0 = seg_start[blk], q1 = seg_start[blk + 1];
    // two-stage pipeline as in the spread: index data two segments ahead,
    // x weights one segment ahead (two 16-byte loads of the slot's 8)
    static_assert(kMaxOrder == 8, "x weights are two float4");
    auto gather_w = [&](int sl, float *wr) {
        const float4 *wx = reinterpret_cast<const float4 *>(sp_w + (size_t)sl * 3 * kMaxOrder);
        const float4 a = __ldg(wx), b = __ldg(wx + 1);
        wr[0] = a.x;
        wr[1] = a.y;
        wr[2] = a.z;
        wr[3] = a.w;
        wr[4] = b.x;
        wr[5] = b.y;
        wr[6] = b.z;
        wr[7] = b.w;
    };
    unsigned mA = 0, mB = 0;
    int sA = 0, sB = 0;
    float wA = 0.0f, wB = 0.0f, wrB[kMaxOrder];
    if (q0 + tid < q1) {
        mB = seg_meta[q0 + tid];
        sB = seg_slot[q0 + tid];
        wB = seg_w[q0 + tid];
        gather_w(sB, wrB);
    }
    if (q0 + kXThreads + tid < q1) {
        mA = seg_meta[q0 + kXThreads + tid];
        sA = seg_slot[q0 + kXThreads + tid];
        wA = seg_w[q0 + kXThreads + tid];
    }
    for (int qb = q0; qb < q1; qb += kXThreads) {
        const int q = qb + tid;
        const unsigned meta = mB;
        const int sl = sB;
        const float sw = wB;
        float wc[kMaxOrder];
#pragma unroll
        for (int k = 0; k < kMaxOrder; k++) wc[k] = wrB[k];
        if (q + kXThreads < q1) {
            mB = mA;
            sB = sA;
            wB = wA;
            gather_w(sB, wrB);
        }
        if (q + 2 * kXThreads < q1) {
            mA = seg_meta[q + 2 * kXThreads];
            sA = seg_slot[q + 2 * kXThreads];
            wA = seg_w[q + 2 * kXThreads];
        }
        float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f;
        int key = -1 - lane;  // unique for lanes past the end
        if (q < q1) {
            // the three components' rows of one (z, y) row are kC floats apart
            constexpr int kC = x_row_offset<K>(NRB) - x_row_offset<K>(0);
            static_assert(x_row_offset<K>(2 * NRB) - x_row_offset<K>(NRB) == kC, "even component stride");
            const float *row0 = rows + x_row_offset<K>(meta & 31u);
            const int x0 = (int)(meta >> 6);
            if (x0 + p <= K) {
                const float *a = row0 + x0;
#pragma unroll
                for (int k = 0; k < kMaxOrder; k++) {
                    if (k < p) {
                        p0 = fmaf(wc[k], a[k], p0);
                        p1 = fmaf(wc[k], a[k + kC], p1);
                        p2 = fmaf(wc[k], a[k + 2 * kC], p2);
                    }
                }
            } else {  // the support wraps around x = K
#pragma unroll
                for (int k = 0; k < kMaxOrder; k++) {
                    if (k < p) {
                        const int x = (x0 + k) & (K - 1);
                        p0 = fmaf(wc[k], row0[x], p0);
                        p1 = fmaf(wc[k], row0[x + kC], p1);
                        p2 = fmaf(wc[k], row0[x + 2 * kC], p2);
                    }
                }
            }
            p0 *= sw;
            p1 *= sw;
            p2 *= sw;
            key = sl;
        }
        // segmented inclusive scan over runs of equal keys; a particle has at
        // most one segment per row of the block, so a run spans at most NRB
        // lanes and offsets below NRB complete it
        static_assert(NRB <= 32 && (NRB & (NRB - 1)) == 0, "runs fit the warp");
#pragma unroll
        for (int o = 1; o < NRB; o <<= 1) {
            const float o0 = __shfl_up_sync(0xffffffffu, p0, o);
            const float o1 = __shfl_up_sync(0xffffffffu, p1, o);
            const float o2 = __shfl_up_sync(0xffffffffu, p2, o);
            const int ok = __shfl_up_sync(0xffffffffu, key, o);
            if (lane >= o && ok == key) {
                p0 += o0;
                p1 += o1;
                p2 += o2;
            }
        }
        const int nk = __shfl_down_sync(0xffffffffu, key, 1);
        const bool last = (lane == 31) || (nk != key);
        if (q < q1 && last) {
            const int i = sp_perm[key];
            if (iscale) {
                const float sc = (float)iscale[i];
                p0 *= sc;
                p1 *= sc;
                p2 *= sc;
            }
            atomicAdd(&vout[3 * i + 0], p0);
            atomicAdd(&vout[3 * i + 1], p1);
            atomicAdd(&vout[3 * i + 2], p2);
        }
    }
}

template <int K, bool BULK>
__global__ void __launch_bounds__(kXThreads, kXpassMinBlocks<K>())
k_xinv_interp(int n, int p, int nby, const int *__restrict__ seg_start,
              const unsigned *__restrict__ seg_meta, const int *__restrict__ seg_slot,
              const float *__restrict__ seg_w, const float *__restrict__ sp_w,
              const int *__restrict__ sp_perm, const double *__restrict__ iscale, int XS,
              const float2 *__restrict__ tw_half, const float2 *__restrict__ tw_full,
              const float2 *__restrict__ cgrid, float *__restrict__ vrecip, int r0, int *err)
{
    // the RHS index runs fastest, so the CTAs of one row block run together
    // and share its segment lists and weights through L2
    xinv_interp_block<K, BULK>(n, p, nby, seg_start, seg_meta, seg_slot, seg_w, sp_w, sp_perm, iscale, XS, tw_half,
                               tw_full, cgrid, vrecip, err, r0 + blockIdx.x, blockIdx.y, blockIdx.z);
}

// Packed: blockIdx.z = slot * nbz + bz (see k_spread_xfwd_packed).
template <int K>
__global__ void __launch_bounds__(kXThreads, kXpassMinBlocks<K>())
k_xinv_interp_packed(const PackedSys *__restrict__ sys, const PackedIO *__restrict__ io,
                     const int *__restrict__ slot_sys, int nbz, int XS, const float2 *__restrict__ tw_half,
                     const float2 *__restrict__ tw_full, const float2 *__restrict__ grid, long long slot_stride,
                     int *err)
{
    const int slot = blockIdx.z / nbz, bz = blockIdx.z - slot * nbz;
    const int g = slot_sys[slot];
    const PackedSys &S = sys[g];
    xinv_interp_block<K, true>(S.n, S.p, S.nby, S.seg_start, S.seg_meta, S.seg_slot, S.seg_w, S.sp_w, S.sp_perm,
                               nullptr, XS, tw_half, tw_full, grid + (size_t)slot * slot_stride, io[g].vrecip, err,
                               blockIdx.x, blockIdx.y, bz);
}

// v := alpha * (recip/L^3 + real + self*f) + beta * v, FP64.
__global__ void k_combine(int n3, int nr, int mode, double alpha, double beta, double invL3,
                          const double *__restrict__ f, int ldf, const double *__restrict__ self,
                          const float *__restrict__ vrecip, const float *__restrict__ vreal,
                          double *__restrict__ v, int ldv)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)n3 * nr) return;
    const int e = (int)(idx % n3);
    const int r = (int)(idx / n3);
    double acc = 0.0;
    if (mode != 1) acc += (double)vrecip[(size_t)r * n3 + e] * invL3;
    if (mode != 2) acc += (double)vreal[(size_t)r * n3 + e] + self[e / 3] * f[(size_t)r * ldf + e];
    double *out = v + (size_t)r * ldv + e;
    *out = (beta == 0.0 ? 0.0 : beta * *out) + alpha * acc;
}

// z pass with the forward transform, the influence function and the inverse
// transform fused in registers (K <= 256): one thread per (column, t) takes
// all three components.  After step 2 of the forward four-step transform the
// thread holds Ghat[kz] for kz = t (mod N2) -- exactly the samples step 1 of
// the inverse transform needs (x[N2 j + t]) -- so the spectrum goes through
// the influence function and into the inverse transform without a shared-
// memory round trip: six passes over the tile instead of ten.
template <int K>
__host__ __device__ constexpr int kZFusedThreads() { return z_fused_tile(K) * FftShape<K>::N2; }

// FWD_ONLY stops after the forward z transform and stores the spectrum (the
// forward-transform diagnostic sdt_spme_spectrum_device); the product uses
// FWD_ONLY = false.
// PACKED: blockIdx.x = slot * nr + r runs over the slots of a packed class
// grid; the slot's influence table (4D map, outermost coordinate = table
// index) and wave numbers come from slot_tab.
template <int K, bool FWD_ONLY = false, bool PACKED = false>
__global__ void __launch_bounds__(kZFusedThreads<K>(), 6)
k_zpass_fused_tma(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap tabmap,
                  const float2 *__restrict__ tw, const float *__restrict__ kmap, int *err, int r0,
                  const int *__restrict__ slot_tab = nullptr, int nr_packed = 1)
{
    constexpr int H = K / 2;
    constexpr int N1 = FftShape<K>::N1, N2 = FftShape<K>::N2, NR = N1 / N2;
    constexpr int CS = K * z_fused_tile(K);  // float2 per component
    extern __shared__ __align__(1024) float2 sm[];  // [3][K][z_fused_tile(K)], then the table tile [K][z_fused_tile(K)]
    float *tabs = reinterpret_cast<float *>(sm + 3 * CS);
    __shared__ uint64_t bar;
    // the RHS index runs fastest, so the CTAs that read one influence-table
    // tile run together and share it through L2
    const int r = r0 + blockIdx.x, tx = blockIdx.y, y = blockIdx.z;
    const int tid = threadIdx.x;
    const int kx0 = tx * z_fused_tile(K);
    int tabi = 0;
    if constexpr (PACKED) {
        tabi = slot_tab[blockIdx.x / nr_packed];
        kmap += (size_t)tabi * K;
    }
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(&bar, (uint32_t)(3 * CS * sizeof(float2) + CS * sizeof(float)));
        for (int c = 0; c < 3; c++)
            for (int z0 = 0; z0 < K; z0 += kTmaBoxLines)
                tma_load_4d(sm + c * CS + z0 * z_fused_tile(K), &map, &bar, kx0, y, z0, 3 * r + c);
        for (int z0 = 0; z0 < K; z0 += kTmaBoxLines) {
            if constexpr (PACKED)
                tma_load_4d(tabs + z0 * z_fused_tile(K), &tabmap, &bar, kx0, y, z0, tabi);
            else
                tma_load_3d(tabs + z0 * z_fused_tile(K), &tabmap, &bar, kx0, y, z0);
        }
    }
    const bool ok = mbar_wait(&bar, 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicExch(err, kTmaErrTimeout);
        return;
    }
    const int col = tid % z_fused_tile(K), t = tid / z_fused_tile(K);
    // element e of a column sits at sm[c * CS + e * z_fused_tile(K) + col]
    auto at = [&](int c, int e) -> float2 & { return sm[c * CS + e * z_fused_tile(K) + col]; };

    // forward step 1 per component: N1-point DFTs of x[N2 j + t], twiddled,
    // stored transposed in place (after every thread has read the component)
#pragma unroll 1
    for (int c = 0; c < 3; c++) {
        float2 a[N1];
#pragma unroll
        for (int j = 0; j < N1; j++) a[j] = at(c, N2 * j + t);
        __syncthreads();
        dft_reg<N1, false>(a);
        static_for<N1>([&](auto kc) {
            constexpr int k1 = decltype(kc)::value;
            float2 v = a[SlotOf<N1, k1>::value];
            if constexpr (k1 != 0) v = cmul(v, __ldg(&tw[(t * k1) & (K - 1)]));
            at(c, k1 * N2 + ((t + k1) & (N2 - 1))) = v;
        });
    }
    __syncthreads();
    // forward step 2: thread t takes k1 = t + r N2 and holds
    // Ghat[k1 + N1 k2] in b[c][r][slot(k2)]
    float2 b[3][NR][N2];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int rr = 0; rr < NR; rr++) {
            const int k1 = t + rr * N2;
#pragma unroll
            for (int j = 0; j < N2; j++) b[c][rr][j] = at(c, k1 * N2 + ((j + k1) & (N2 - 1)));
            dft_reg<N2, false>(b[c][rr]);
        }
    if constexpr (FWD_ONLY) {
        __syncthreads();  // every thread is done reading the transposed data
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int rr = 0; rr < NR; rr++)
                static_for<N2>([&](auto kc) {
                    constexpr int k2 = decltype(kc)::value;
                    at(c, t + rr * N2 + N1 * k2) = b[c][rr][SlotOf<N2, k2>::value];
                });
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            for (int c2 = 0; c2 < 3; c2++)
                for (int z0 = 0; z0 < K; z0 += kTmaBoxLines)
                    tma_store_4d(&map, sm + c2 * CS + z0 * z_fused_tile(K), kx0, y, z0, 3 * r + c2);
            bulk_commit();
            bulk_wait_read_all();
        }
        return;
    }
    // influence: Ghat <- m2(k) (I - k k^T / k^2) Ghat, zero at k = 0
    const int kx = kx0 + col;
    const float fkx = kx <= H ? __ldg(&kmap[kx]) : 0.0f;
    const float fky = __ldg(&kmap[y]);
#pragma unroll
    for (int rr = 0; rr < NR; rr++) {
        static_for<N2>([&](auto kc) {
            constexpr int k2 = decltype(kc)::value;
            constexpr int sl = SlotOf<N2, k2>::value;
            const int kz = t + rr * N2 + N1 * k2;
            const float fkz = __ldg(&kmap[kz]);
            const float m2 = tabs[kz * z_fused_tile(K) + col];
            const float kk = fkx * fkx + fky * fky + fkz * fkz;
            float2 g0 = b[0][rr][sl], g1 = b[1][rr][sl], g2 = b[2][rr][sl];
            if (kk > 0.0f && kx <= H) {
                const float inv = 1.0f / kk;
                const float dr = (fkx * g0.x + fky * g1.x + fkz * g2.x) * inv;
                const float di = (fkx * g0.y + fky * g1.y + fkz * g2.y) * inv;
                g0 = make_float2(m2 * (g0.x - fkx * dr), m2 * (g0.y - fkx * di));
                g1 = make_float2(m2 * (g1.x - fky * dr), m2 * (g1.y - fky * di));
                g2 = make_float2(m2 * (g2.x - fkz * dr), m2 * (g2.y - fkz * di));
            } else {
                g0 = g1 = g2 = make_float2(0.f, 0.f);
            }
            b[0][rr][sl] = g0;
            b[1][rr][sl] = g1;
            b[2][rr][sl] = g2;
        });
    }
    __syncthreads();  // every thread is done reading the transposed forward data
    // inverse step 1 straight from registers: x[N2 j + t] is Ghat[k1 + N1 k2]
    // with k1 = t + (j % NR) N2, k2 = j / NR
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float2 a[N1];
        static_for<N1>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            a[j] = b[c][j % NR][SlotOf<N2, j / NR>::value];
        });
        dft_reg<N1, true>(a);
        static_for<N1>([&](auto kc) {
            constexpr int k1 = decltype(kc)::value;
            float2 v = a[SlotOf<N1, k1>::value];
            if constexpr (k1 != 0) {
                float2 w = __ldg(&tw[(t * k1) & (K - 1)]);
                w.y = -w.y;
                v = cmul(v, w);
            }
            at(c, k1 * N2 + ((t + k1) & (N2 - 1))) = v;
        });
    }
    __syncthreads();
    // inverse step 2 per component, natural order
#pragma unroll 1
    for (int c = 0; c < 3; c++) {
        float2 d[NR][N2];
#pragma unroll
        for (int rr = 0; rr < NR; rr++) {
            const int k1 = t + rr * N2;
#pragma unroll
            for (int j = 0; j < N2; j++) d[rr][j] = at(c, k1 * N2 + ((j + k1) & (N2 - 1)));
        }
        __syncthreads();
#pragma unroll
        for (int rr = 0; rr < NR; rr++) {
            const int k1 = t + rr * N2;
            dft_reg<N2, true>(d[rr]);
            static_for<N2>([&](auto kc) {
                constexpr int k2 = decltype(kc)::value;
                at(c, k1 + N1 * k2) = d[rr][SlotOf<N2, k2>::value];
            });
        }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
        for (int c2 = 0; c2 < 3; c2++)
            for (int z0 = 0; z0 < K; z0 += kTmaBoxLines)
                tma_store_4d(&map, sm + c2 * CS + z0 * z_fused_tile(K), kx0, y, z0, 3 * r + c2);
        bulk_commit();
        bulk_wait_read_all();
    }
}

// ---------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------

static inline int grid1d(long long n, int bs) { return (int)((n + bs - 1) / bs); }

// fwd_only: stop after the forward transform (spread + x, y and z FFTs),
// leaving the half spectrum in d_cgrid (fused z pass only).
template <int K>
static int recip_pass(SpmeEngine *e, int nr, const float *tab, const double *iscale, int r0 = 0,
                      cudaStream_t st = nullptr, bool fwd_only = false)
{
    constexpr int H = K / 2;
    cudaStream_t s = st ? st : e->stream;
    const size_t smx = (size_t)x_rows_floats<K>() * sizeof(float);
    const size_t smy = (size_t)K * kTileX * sizeof(float2);
    const size_t smz = (size_t)3 * K * kTileZ * sizeof(float2);
    const size_t smz_tma = smz + (size_t)K * kTileZ * sizeof(float);
    constexpr int TZ = z_fused_tile(K);
    const size_t smzf_tma = (size_t)3 * K * TZ * sizeof(float2) + (size_t)K * TZ * sizeof(float);
    const int ntile = (H + 1 + kTileX - 1) / kTileX;
    const int ntilez = (H + 1 + kTileZ - 1) / kTileZ;
    const int ntilezf = (H + 1 + TZ - 1) / TZ;
    SDT_CUDA(cudaFuncSetAttribute(k_spread_xfwd<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    SDT_CUDA(cudaFuncSetAttribute(k_xinv_interp<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    SDT_CUDA(cudaFuncSetAttribute(k_xinv_interp<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
    SDT_CUDA(cudaFuncSetAttribute(k_ypass<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
    SDT_CUDA(cudaFuncSetAttribute(k_ypass<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
    SDT_CUDA(cudaFuncSetAttribute(k_zpass_influence<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
    if (e->tma_ready) {
        SDT_CUDA(cudaFuncSetAttribute(k_ypass_tma<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
        SDT_CUDA(cudaFuncSetAttribute(k_ypass_tma<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
        SDT_CUDA(cudaFuncSetAttribute(k_zpass_influence_tma<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smz_tma));
        if constexpr (K <= 256) {
            SDT_CUDA(cudaFuncSetAttribute(k_zpass_fused_tma<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smzf_tma));
            if (fwd_only)
                SDT_CUDA(cudaFuncSetAttribute(k_zpass_fused_tma<K, true>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smzf_tma));
        }
    }
    if (fwd_only && !(K <= 256 && e->tma_ready && e->zfused))
        return set_error(e, kErrUnsupported, "the forward-spectrum diagnostic needs the fused z pass (K <= 256)");
    const int ty = kTileX * FftShape<K>::N2;
    const int tz = 3 * kTileZ * FftShape<K>::N2;
    if (K == 256 && e->tc_ready && nr >= kTcMinRhs) {
        const int st = spread_tc_launch(e, nr, r0, s);
        if (st != kOk) return st;
    } else {
        k_spread_xfwd<K><<<dim3(nr, e->nby, e->nbz), kXThreads, smx, s>>>(
            e->npos, e->p, e->nby, e->d_seg_start, e->d_seg_meta, e->d_seg_slot, e->d_seg_w, e->d_sp_w,
            e->d_fs_sp, e->XS, e->d_tw_half, e->d_tw_full, e->d_cgrid, r0);
        SDT_LAUNCH_CHECK();
    }
    prof_mark(e, kStSpreadX);
    if (e->tma_ready) {
        k_ypass_tma<K, false><<<dim3(ntile, K, nr * 3), ty, smy, s>>>(e->tmap_y, e->d_tw_full, e->d_err, 3 * r0);
        SDT_LAUNCH_CHECK();
        prof_mark(e, kStYFwd);
        const CUtensorMap &tabmap = tab == e->d_tab2 ? e->tmap_tab2 : e->tmap_tab0;
        bool fused = false;
        if constexpr (K <= 256) {
            if (e->zfused) {
                const CUtensorMap &tabmapf = tab == e->d_tab2 ? e->tmap_tab2f : e->tmap_tab0f;
                if (fwd_only) {
                    k_zpass_fused_tma<K, true><<<dim3(nr, ntilezf, K), kZFusedThreads<K>(), smzf_tma, s>>>(
                        e->tmap_zf, tabmapf, e->d_tw_full, e->d_kmap, e->d_err, r0);
                    SDT_LAUNCH_CHECK();
                    return kOk;
                }
                k_zpass_fused_tma<K><<<dim3(nr, ntilezf, K), kZFusedThreads<K>(), smzf_tma, s>>>(
                    e->tmap_zf, tabmapf, e->d_tw_full, e->d_kmap, e->d_err, r0);
                fused = true;
            }
        }
        if (!fused)
            k_zpass_influence_tma<K><<<dim3(ntilez, K, nr), tz, smz_tma, s>>>(e->tmap_z, tabmap, e->d_tw_full,
                                                                          e->d_kmap, e->d_err, r0);
        SDT_LAUNCH_CHECK();
        prof_mark(e, kStZInfl);
        k_ypass_tma<K, true><<<dim3(ntile, K, nr * 3), ty, smy, s>>>(e->tmap_y, e->d_tw_full, e->d_err, 3 * r0);
        SDT_LAUNCH_CHECK();
        prof_mark(e, kStYInv);
    } else {
        k_ypass<K, false><<<dim3(ntile, K, nr * 3), ty, smy, s>>>(e->XS, e->d_tw_full, e->d_cgrid, 3 * r0);
        SDT_LAUNCH_CHECK();
        prof_mark(e, kStYFwd);
        k_zpass_influence<K><<<dim3(ntilez, K, nr), tz, smz, s>>>(e->XS, e->d_tw_full, e->d_kmap, tab, r0,
                                                                  e->d_cgrid);
        SDT_LAUNCH_CHECK();
        prof_mark(e, kStZInfl);
        k_ypass<K, true><<<dim3(ntile, K, nr * 3), ty, smy, s>>>(e->XS, e->d_tw_full, e->d_cgrid, 3 * r0);
        SDT_LAUNCH_CHECK();
        prof_mark(e, kStYInv);
    }
    auto xinv = e->tma_enabled ? k_xinv_interp<K, true> : k_xinv_interp<K, false>;
    xinv<<<dim3(nr, e->nby, e->nbz), kXThreads, smx, s>>>(
        e->npos, e->p, e->nby, e->d_seg_start, e->d_seg_meta, e->d_seg_slot, e->d_seg_w, e->d_sp_w,
        e->d_sp_perm, iscale, e->XS, e->d_tw_half, e->d_tw_full, e->d_cgrid, e->d_vrecip, r0, e->d_err);
    SDT_LAUNCH_CHECK();
    prof_mark(e, kStXInterp);
    return kOk;
}

static int recip_dispatch(SpmeEngine *e, int nr, const float *tab, const double *iscale, int r0 = 0,
                          cudaStream_t st = nullptr, bool fwd_only = false)
{
    switch (e->K) {
        case 32: return recip_pass<32>(e, nr, tab, iscale, r0, st, fwd_only);
        case 64: return recip_pass<64>(e, nr, tab, iscale, r0, st, fwd_only);
        case 128: return recip_pass<128>(e, nr, tab, iscale, r0, st, fwd_only);
        case 256: return recip_pass<256>(e, nr, tab, iscale, r0, st, fwd_only);
        case 512: return recip_pass<512>(e, nr, tab, iscale, r0, st, fwd_only);
        default: return set_error(e, kErrUnsupported, "grid dimension must be 32, 64, 128, 256 or 512");
    }
}

int spme_set_radii(SpmeEngine *e, const double *rdi)
{
    const int n = e->npos;
    std::vector<double> self(n), a2(n);
    for (int i = 0; i < n; i++) {
        const double a = rdi[i];
        // self_a = 1/a - xi/sqrt(pi) (6 - 40/3 xi^2 a^2)  (mob_spme.cc:151)
        self[i] = 1.0 / a - e->xi / std::sqrt(M_PI) * (6.0 - 40.0 / 3.0 * e->xi * e->xi * a * a);
        a2[i] = a * a;
    }
    const size_t bytes = (size_t)n * sizeof(double);
    if ((!e->d_rdi && cudaMalloc(&e->d_rdi, bytes) != cudaSuccess) ||
        (!e->d_rdi2 && cudaMalloc(&e->d_rdi2, bytes) != cudaSuccess) ||
        cudaMemcpy(e->d_rdi, rdi, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(e->d_rdi2, a2.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(e->d_self, self.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return set_error(e, kErrCuda, "uploading the particle radii failed");
    }
    return kOk;
}

// Side streams and fork/join events of the overlapped product (created on
// first use; they live as long as the engine).
static int ensure_side_streams(SpmeEngine *e)
{
    if (e->side[0]) return kOk;
    for (int q = 0; q < 3; q++) {
        SDT_CUDA(cudaStreamCreateWithFlags(&e->side[q], cudaStreamNonBlocking));
        SDT_CUDA(cudaEventCreateWithFlags(&e->ev_join[q], cudaEventDisableTiming));
    }
    SDT_CUDA(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
    return kOk;
}

int spme_check_device_error(SpmeEngine *e)
{
    if (!e->d_err) return kOk;
    int h = 0;
    SDT_CUDA(cudaMemcpyAsync(&h, e->d_err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    SDT_CUDA(cudaStreamSynchronize(e->stream));
    if (h == 0) return kOk;
    SDT_CUDA(cudaMemsetAsync(e->d_err, 0, sizeof(int), e->stream));
    return set_error(e, kErrCuda, "a grid pass timed out waiting for its tile copy (results invalid)");
}

int spme_reserve(SpmeEngine *e, int rhs)
{
    if (rhs <= e->rhs_cap) return kOk;
    const size_t n = (size_t)e->npos;
    const size_t grid = (size_t)3 * e->K * e->K * e->XS;
    cudaFree(e->d_cgrid);
    cudaFree(e->d_fs_sp);
    cudaFree(e->d_fs_rs);
    cudaFree(e->d_vrecip);
    cudaFree(e->d_vreal);
    e->d_cgrid = nullptr;
    e->d_fs_sp = e->d_fs_rs = e->d_vrecip = e->d_vreal = nullptr;
    e->rhs_cap = 0;
    if (cudaMalloc(&e->d_cgrid, grid * rhs * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&e->d_fs_sp, 3 * n * rhs * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&e->d_fs_rs, 4 * n * rhs * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&e->d_vrecip, 3 * n * rhs * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&e->d_vreal, 3 * n * rhs * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return set_error(e, kErrAlloc, "device allocation of the SPME work space failed");
    }
    // the padding columns kx > K/2 are never written by the passes: keep them zero
    SDT_CUDA(cudaMemsetAsync(e->d_cgrid, 0, grid * rhs * sizeof(float2), e->stream));
    e->rhs_cap = rhs;
    e->tma_ready = false;
    if (e->tma_enabled) {
        const unsigned long long K = e->K, XS = e->XS, el = sizeof(float2);
        const unsigned lines = (unsigned)std::min(e->K, 256);
        const unsigned long long dy[3] = {XS, K, 3ull * rhs * K};
        const unsigned long long sy[2] = {XS * el, K * XS * el};
        const unsigned by[3] = {(unsigned)kTileX, lines, 1u};
        const unsigned long long dz[4] = {XS, K, K, 3ull * rhs};
        const unsigned long long sz[3] = {XS * el, K * XS * el, K * K * XS * el};
        const unsigned bz[4] = {(unsigned)kTileZ, 1u, lines, 1u};
        const unsigned bzf[4] = {(unsigned)z_fused_tile(e->K), 1u, lines, 1u};
        e->tma_ready = e->tma_tabs && encode_tmap_f2(&e->tmap_y, e->d_cgrid, 3, dy, sy, by) &&
                       encode_tmap_f2(&e->tmap_z, e->d_cgrid, 4, dz, sz, bz) &&
                       encode_tmap_f2(&e->tmap_zf, e->d_cgrid, 4, dz, sz, bzf);
    }
    return kOk;
}

int spme_create(SpmeEngine *e)
{
    const int K = e->K, p = e->p;
    if (e->npos <= 0) return set_error(e, kErrInvalid, "npos must be > 0");
    if (!(e->box > 0.0)) return set_error(e, kErrInvalid, "box_size must be > 0");
    if (!(e->rmax > 0.0)) return set_error(e, kErrInvalid, "rmax must be > 0");
    if (!(e->xi > 0.0)) return set_error(e, kErrInvalid, "xi must be > 0");
    if (K <= 0) return set_error(e, kErrInvalid, "dim must be > 0");
    if (p <= 1) return set_error(e, kErrInvalid, "porder must be > 1");
    if (2.0 * e->rmax >= e->box) return set_error(e, kErrInvalid, "rmax must be less than box_size/2");
    if (4 * p > K) return set_error(e, kErrInvalid, "porder must be smaller than dim/4");
    if (K != 32 && K != 64 && K != 128 && K != 256 && K != 512)
        return set_error(e, kErrUnsupported, "dim must be a power of two in [32, 512]");
    if (p % 2 != 0 || p > kMaxOrder)
        return set_error(e, kErrUnsupported, "porder must be even and <= 8");

    SDT_CUDA(cudaSetDevice(e->device));
    if (!e->stream) {
        SDT_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->own_stream = true;
    }
    {
        const char *no_tma = std::getenv("STOKESDT_NO_TMA");
        e->tma_enabled = !(no_tma && no_tma[0] == '1');
        const char *ov = std::getenv("STOKESDT_OVERLAP");
        e->overlap = ov && ov[0] == '1';
        const char *nz = std::getenv("STOKESDT_NO_ZFUSE");
        e->zfused = !(nz && nz[0] == '1');
        const char *tc = std::getenv("STOKESDT_NO_TC");
        e->tc_enabled = !(tc && tc[0] == '1');
    }
    SDT_CUDA(cudaMalloc(&e->d_err, sizeof(int)));
    SDT_CUDA(cudaMemset(e->d_err, 0, sizeof(int)));
    const int H = K / 2;
    e->XS = ((H + 1) + 3) / 4 * 4;
    e->nbin = K / kRowBlock;
    e->nby = K / kRowBlockY;
    e->nbz = K / kRowBlockZ;
    e->ncnt_sp = std::max(e->nbin * e->nbin, e->nby * e->nbz);
    e->self_mono = 1.0 - e->xi / std::sqrt(M_PI) * (6.0 - 40.0 / 3.0 * e->xi * e->xi);

    // wave numbers and |b(k)|^2 (ComputeSpline, spme.cc:80-128); only the
    // modulus enters the influence table.
    std::vector<double> kmap(K), bmod2(K);
    for (int m = 0; m < K; m++) {
        const int ms = (m <= H) ? m : m - K;
        kmap[m] = ms * 2.0 * M_PI / e->box;
    }
    std::vector<double> splineval(p - 1);
    for (int i = 0; i < p - 1; i++) splineval[i] = bspline_host(p, (double)i);
    for (int m = 0; m < K; m++) {
        double re = 0.0, im = 0.0;
        for (int i = 0; i < p - 1; i++) {
            const double phi = i * kmap[m] * e->box / K;
            re += splineval[i] * std::cos(phi);
            im += splineval[i] * std::sin(phi);
        }
        bmod2[m] = 1.0 / (re * re + im * im);
    }
    std::vector<float> kmapf(K);
    for (int m = 0; m < K; m++) kmapf[m] = (float)kmap[m];
    std::vector<float2> twh(H), twf(K);
    for (int m = 0; m < H; m++) twh[m] = make_float2((float)std::cos(-2.0 * M_PI * m / H), (float)std::sin(-2.0 * M_PI * m / H));
    for (int m = 0; m < K; m++) twf[m] = make_float2((float)std::cos(-2.0 * M_PI * m / K), (float)std::sin(-2.0 * M_PI * m / K));

    double *d_kmap64 = nullptr, *d_bmod2 = nullptr;
    const size_t tabsz = (size_t)K * K * e->XS * sizeof(float);
    SDT_CUDA(cudaMalloc(&d_kmap64, K * sizeof(double)));
    SDT_CUDA(cudaMalloc(&d_bmod2, K * sizeof(double)));
    SDT_CUDA(cudaMemcpy(d_kmap64, kmap.data(), K * sizeof(double), cudaMemcpyHostToDevice));
    SDT_CUDA(cudaMemcpy(d_bmod2, bmod2.data(), K * sizeof(double), cudaMemcpyHostToDevice));
    SDT_CUDA(cudaMalloc(&e->d_tab0, tabsz));
    SDT_CUDA(cudaMemset(e->d_tab0, 0, tabsz));
    k_influence_table<<<1184, 256, 0, e->stream>>>(K, e->XS, e->xi, d_kmap64, d_bmod2, e->mono ? 0 : 1, e->d_tab0);
    SDT_LAUNCH_CHECK();
    if (!e->mono) {
        SDT_CUDA(cudaMalloc(&e->d_tab2, tabsz));
        SDT_CUDA(cudaMemset(e->d_tab2, 0, tabsz));
        k_influence_table<<<1184, 256, 0, e->stream>>>(K, e->XS, e->xi, d_kmap64, d_bmod2, 2, e->d_tab2);
        SDT_LAUNCH_CHECK();
    }
    SDT_CUDA(cudaStreamSynchronize(e->stream));
    cudaFree(d_kmap64);
    cudaFree(d_bmod2);
    SDT_CUDA(cudaMalloc(&e->d_kmap, K * sizeof(float)));
    SDT_CUDA(cudaMemcpy(e->d_kmap, kmapf.data(), K * sizeof(float), cudaMemcpyHostToDevice));
    SDT_CUDA(cudaMalloc(&e->d_tw_half, H * sizeof(float2)));
    SDT_CUDA(cudaMemcpy(e->d_tw_half, twh.data(), H * sizeof(float2), cudaMemcpyHostToDevice));
    SDT_CUDA(cudaMalloc(&e->d_tw_full, K * sizeof(float2)));
    SDT_CUDA(cudaMemcpy(e->d_tw_full, twf.data(), K * sizeof(float2), cudaMemcpyHostToDevice));
    if (e->tma_enabled) {
        // influence-table tiles of the z pass: [K z][K y][XS x] floats
        const unsigned long long KK = K, XSl = e->XS, el = sizeof(float);
        const unsigned long long dt[3] = {XSl, KK, KK};
        const unsigned long long st[2] = {XSl * el, KK * XSl * el};
        const unsigned bt[3] = {(unsigned)kTileZ, 1u, (unsigned)std::min(K, 256)};
        const unsigned btf[3] = {(unsigned)z_fused_tile(K), 1u, (unsigned)std::min(K, 256)};
        e->tma_tabs = encode_tmap(&e->tmap_tab0, e->d_tab0, 4, 3, dt, st, bt) &&
                      encode_tmap(&e->tmap_tab0f, e->d_tab0, 4, 3, dt, st, btf) &&
                      (e->mono || (encode_tmap(&e->tmap_tab2, e->d_tab2, 4, 3, dt, st, bt) &&
                                   encode_tmap(&e->tmap_tab2f, e->d_tab2, 4, 3, dt, st, btf)));
        if (e->mono) {
            e->tmap_tab2 = e->tmap_tab0;
            e->tmap_tab2f = e->tmap_tab0f;
        }
    }

    // real-space cells of edge >= rmax/2 (PairListR::NumCells, pair_r.cc:15-22)
    // and the unique neighbour offsets within two cells.
    int nc = (int)(e->box / (e->rmax / 2.0));
    nc = nc < 1 ? 1 : nc;
    e->nc = nc;
    e->cs = e->box / nc;
    std::vector<int> axis;
    for (int d = -2; d <= 2; d++) {
        const int res = ((d % nc) + nc) % nc;
        bool seen = false;
        for (int q : axis) seen |= (((q % nc) + nc) % nc) == res;
        if (!seen) axis.push_back(d);
    }
    // (dx, dy) columns of the stencil; the z neighbours of a column are one
    // or two contiguous particle ranges (cells are z-fastest)
    std::vector<int> st;
    for (int dx : axis)
        for (int dy : axis) st.push_back((dx + 8) | ((dy + 8) << 5));
    e->nstencil = (int)st.size();
    SDT_CUDA(cudaMalloc(&e->d_stencil, st.size() * sizeof(int)));
    SDT_CUDA(cudaMemcpy(e->d_stencil, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice));

    const size_t n = (size_t)e->npos;
    const size_t ncell = (size_t)nc * nc * nc;
    const size_t nbins = (size_t)e->nbin * e->nbin;
    SDT_CUDA(cudaMalloc(&e->d_sp_perm, n * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_sp_base, n * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_sp_w, n * 3 * kMaxOrder * sizeof(float)));
    SDT_CUDA(cudaMalloc(&e->d_sp_binstart, (nbins + 1) * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_seg_start, ((size_t)e->nby * e->nbz + 1) * sizeof(int)));
    const size_t nseg = n * (size_t)p * p;
    SDT_CUDA(cudaMalloc(&e->d_seg_meta, nseg * sizeof(unsigned)));
    SDT_CUDA(cudaMalloc(&e->d_seg_slot, nseg * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_seg_w, nseg * sizeof(float)));
    SDT_CUDA(cudaMalloc(&e->d_rs_perm, n * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_rs_cell, n * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_rs_pos, n * sizeof(double4)));
    SDT_CUDA(cudaMalloc(&e->d_rs_posf, n * sizeof(float4)));
    SDT_CUDA(cudaMalloc(&e->d_rs_inv, n * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_rs_cellstart, (ncell + 1) * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_counts, ((size_t)e->ncnt_sp + ncell) * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_key_sp, n * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_key_rs, n * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_tmp_base, n * sizeof(int)));
    SDT_CUDA(cudaMalloc(&e->d_tmp_w, n * 3 * kMaxOrder * sizeof(float)));
    SDT_CUDA(cudaMalloc(&e->d_tmp_pos, n * sizeof(double4)));
    SDT_CUDA(cudaMalloc(&e->d_self, n * sizeof(double)));
    return kOk;
}

int spme_update(SpmeEngine *e, const double *d_pos)
{
    e->updated = false;
    const int n = e->npos;
    const int nbins = e->nbin * e->nbin;
    const int ncell = e->nc * e->nc * e->nc;
    int *cnt_sp = e->d_counts, *cnt_rs = e->d_counts + e->ncnt_sp;
    SDT_CUDA(cudaMemsetAsync(e->d_counts, 0, (size_t)(e->ncnt_sp + ncell) * sizeof(int), e->stream));
    k_prep<<<grid1d(n, 256), 256, 0, e->stream>>>(n, d_pos, e->mono ? nullptr : e->d_rdi, e->box, e->K,
                                                  e->p, e->nbin, e->nc, e->cs, e->d_key_sp, e->d_key_rs,
                                                  e->d_tmp_base, e->d_tmp_w, e->d_tmp_pos, cnt_sp, cnt_rs);
    SDT_LAUNCH_CHECK();
    k_scan<<<1, 1024, 0, e->stream>>>(nbins, cnt_sp, e->d_sp_binstart);
    SDT_LAUNCH_CHECK();
    k_scan<<<1, 1024, 0, e->stream>>>(ncell, cnt_rs, e->d_rs_cellstart);
    SDT_LAUNCH_CHECK();
    k_scatter<<<grid1d(n, 256), 256, 0, e->stream>>>(n, e->d_key_sp, cnt_sp, e->d_sp_perm);
    SDT_LAUNCH_CHECK();
    k_scatter<<<grid1d(n, 256), 256, 0, e->stream>>>(n, e->d_key_rs, cnt_rs, e->d_rs_perm);
    SDT_LAUNCH_CHECK();
    k_fill_sorted<<<grid1d(n, 256), 256, 0, e->stream>>>(n, e->d_sp_perm, e->d_rs_perm, e->d_tmp_base,
                                                         e->d_tmp_w, e->d_tmp_pos, e->d_key_rs,
                                                         e->d_sp_base, e->d_sp_w, e->d_rs_pos, e->d_rs_posf,
                                                         e->d_rs_cell, e->d_rs_inv);
    SDT_LAUNCH_CHECK();
    // row segments of the x kernels (the spread-order counters are free again)
    const int nblk = e->nby * e->nbz;
    SDT_CUDA(cudaMemsetAsync(cnt_sp, 0, (size_t)nblk * sizeof(int), e->stream));
    k_seg_count<<<grid1d(n, 256), 256, 0, e->stream>>>(n, e->p, e->K, e->nby, e->d_sp_base, cnt_sp);
    SDT_LAUNCH_CHECK();
    k_scan<<<1, 1024, 0, e->stream>>>(nblk, cnt_sp, e->d_seg_start);
    SDT_LAUNCH_CHECK();
    k_seg_fill<<<grid1d(n, 256), 256, 0, e->stream>>>(n, e->p, e->K, e->nby, e->d_sp_base, e->d_sp_w,
                                                      e->d_seg_start, cnt_sp, e->d_seg_meta,
                                                      e->d_seg_slot, e->d_seg_w);
    SDT_LAUNCH_CHECK();
    int st = tc_build(e);
    if (st != kOk) return st;
    st = pair_list_build(e);
    if (st != kOk) return st;
    e->updated = true;
    return kOk;
}

int spme_mulvec(SpmeEngine *e, int mode, int nrhs, double alpha, int ldf, const double *d_f,
                double beta, int ldv, double *d_v)
{
    if (!e->updated) return set_error(e, kErrState, "Update() must be called before MulVector()");
    if (nrhs < 0 || mode < 0 || mode > 2) return set_error(e, kErrInvalid, "bad nrhs or mode");
    const int n = e->npos, n3 = 3 * n;
    if (nrhs == 0) return kOk;
    if (ldf < n3 || ldv < n3) return set_error(e, kErrInvalid, "leading dimensions must be >= 3*npos");
    const int chunk = std::min(nrhs, e->rhs_chunk_max);
    int st = spme_reserve(e, chunk);
    if (st != kOk) return st;
    for (int r0 = 0; r0 < nrhs; r0 += chunk) {
        const int nr = std::min(chunk, nrhs - r0);
        const double *f = d_f + (size_t)r0 * ldf;
        double *v = d_v + (size_t)r0 * ldv;
        // vrecip (interpolation atomics) is cleared by the first force gather;
        // vreal needs no clearing: the real-space kernels store every row
        {
            const int nb_sp = mode != 1 ? grid1d((long long)n * nr, 256) : 0;
            const int nb_rs = mode != 2 ? grid1d(n, 256) : 0;
            k_gather_both<<<nb_sp + nb_rs, 256, 0, e->stream>>>(n, nr, f, ldf, e->d_sp_perm, e->d_fs_sp,
                                                               e->d_vrecip, nb_sp, e->d_rs_inv,
                                                               reinterpret_cast<float4 *>(e->d_fs_rs));
            SDT_LAUNCH_CHECK();
        }
        prof_mark(e, kStGather);
        // Overlap: the real-space sum and groups of RHS of the grid chain run
        // on side streams, so compute-bound x kernels of one group share the
        // GPU with the memory-bound y/z passes of another (monodisperse, not
        // while profiling stages).
        const int groups = (e->overlap && e->mono && !e->prof_on && mode == 0 && nr >= 4) ? 2 : 1;
        if (groups > 1) {
            st = ensure_side_streams(e);
            if (st != kOk) return st;
            SDT_CUDA(cudaEventRecord(e->ev_fork, e->stream));
            for (int q = 0; q < 3; q++) SDT_CUDA(cudaStreamWaitEvent(e->side[q], e->ev_fork, 0));
            cudaStream_t main = e->stream;
            e->stream = e->side[2];
            st = real_space_launch(e, nr);
            e->stream = main;
            if (st != kOk) return st;
            const int ng = (nr + groups - 1) / groups;
            for (int g = 0; g < groups; g++) {
                const int g0 = g * ng, gn = std::min(ng, nr - g0);
                if (gn <= 0) break;
                st = recip_dispatch(e, gn, e->d_tab0, nullptr, g0, e->side[g]);
                if (st != kOk) return st;
            }
            for (int q = 0; q < 3; q++) {
                SDT_CUDA(cudaEventRecord(e->ev_join[q], e->side[q]));
                SDT_CUDA(cudaStreamWaitEvent(e->stream, e->ev_join[q], 0));
            }
            k_combine<<<grid1d((long long)n3 * nr, 256), 256, 0, e->stream>>>(
                n3, nr, mode, alpha, beta, 1.0 / (e->box * e->box * e->box), f, ldf, e->d_self, e->d_vrecip,
                e->d_vreal, v, ldv);
            SDT_LAUNCH_CHECK();
            continue;
        }
        if (mode != 2) {
            st = real_space_launch(e, nr);
            if (st != kOk) return st;
        }
        prof_mark(e, kStReal);
        if (mode != 1) {
            if (e->mono) {
                st = recip_dispatch(e, nr, e->d_tab0, nullptr);
                if (st != kOk) return st;
            } else {
                // polydisperse: M_recip = P^T [tab1 - (a_i^2 + a_j^2) k^2/6 tab1] P as
                // three passes (spme.cc:771-838): (f, tab1), (a^2 f, tab2) and
                // (f, tab2) interpolated with weight a_i^2.
                st = recip_dispatch(e, nr, e->d_tab0, nullptr);
                if (st != kOk) return st;
                k_gather_forces<<<grid1d((long long)n * nr, 256), 256, 0, e->stream>>>(
                    n, nr, f, ldf, e->d_sp_perm, e->d_rdi2, e->d_fs_sp, nullptr);
                SDT_LAUNCH_CHECK();
                st = recip_dispatch(e, nr, e->d_tab2, nullptr);
                if (st != kOk) return st;
                k_gather_forces<<<grid1d((long long)n * nr, 256), 256, 0, e->stream>>>(
                    n, nr, f, ldf, e->d_sp_perm, nullptr, e->d_fs_sp, nullptr);
                SDT_LAUNCH_CHECK();
                st = recip_dispatch(e, nr, e->d_tab2, e->d_rdi2);
                if (st != kOk) return st;
            }
        }
        k_combine<<<grid1d((long long)n3 * nr, 256), 256, 0, e->stream>>>(
            n3, nr, mode, alpha, beta, 1.0 / (e->box * e->box * e->box), f, ldf, e->d_self, e->d_vrecip,
            e->d_vreal, v, ldv);
        SDT_LAUNCH_CHECK();
        prof_mark(e, kStCombine);
    }
    return kOk;
}

// Forward transform of the spread forces of nrhs (<= 16) RHS: the half
// spectra Ghat[r][c][kz][ky][kx], kx <= K/2, as complex FP32 pairs (no
// counterpart in the reference; checks the hand-written FFT against an
// independent one).  Monodisperse engines with the fused z pass only.
int spme_spectrum(SpmeEngine *e, int nrhs, int ldf, const double *d_f, float *d_spec)
{
    if (!e->updated) return set_error(e, kErrState, "Update() must be called first");
    if (!e->mono) return set_error(e, kErrUnsupported, "spectrum diagnostic: monodisperse engines only");
    if (nrhs <= 0 || nrhs > e->rhs_chunk_max) return set_error(e, kErrInvalid, "spectrum: 1 <= nrhs <= 16");
    const int n = e->npos, K = e->K, H1 = e->K / 2 + 1;
    if (ldf < 3 * n) return set_error(e, kErrInvalid, "ldf must be >= 3*npos");
    int st = spme_reserve(e, nrhs);
    if (st != kOk) return st;
    k_gather_forces<<<grid1d((long long)n * nrhs, 256), 256, 0, e->stream>>>(n, nrhs, d_f, ldf, e->d_sp_perm,
                                                                           nullptr, e->d_fs_sp, nullptr);
    SDT_LAUNCH_CHECK();
    st = recip_dispatch(e, nrhs, e->d_tab0, nullptr, 0, nullptr, true);
    if (st != kOk) return st;
    SDT_CUDA(cudaMemcpy2DAsync(d_spec, (size_t)H1 * sizeof(float2), e->d_cgrid, (size_t)e->XS * sizeof(float2),
                               (size_t)H1 * sizeof(float2), (size_t)nrhs * 3 * K * K, cudaMemcpyDeviceToDevice,
                               e->stream));
    return kOk;
}

// Runs `reps` products of nrhs vectors (f = 1, beta = 0, internal buffers)
// with an event after every stage and returns the mean milliseconds per stage.
int spme_profile(SpmeEngine *e, int nrhs, int reps, double *stage_ms)
{
    if (!e->updated) return set_error(e, kErrState, "Update() must be called before profiling");
    if (nrhs <= 0 || nrhs > e->rhs_chunk_max || reps <= 0)
        return set_error(e, kErrInvalid, "profile: 1 <= nrhs <= 16 and reps >= 1");
    const int n3 = 3 * e->npos;
    double *d_f = nullptr, *d_v = nullptr;
    SDT_CUDA(cudaMalloc(&d_f, (size_t)nrhs * n3 * sizeof(double)));
    SDT_CUDA(cudaMalloc(&d_v, (size_t)nrhs * n3 * sizeof(double)));
    SDT_CUDA(cudaMemsetAsync(d_f, 0, (size_t)nrhs * n3 * sizeof(double), e->stream));
    for (int i = 0; i <= kNumStages; i++) SDT_CUDA(cudaEventCreate(&e->prof_ev[i]));
    double acc[kNumStages] = {0};
    int st = kOk;
    for (int r = 0; r < reps && st == kOk; r++) {
        e->prof_on = true;
        // stages that do not run (e.g. polydisperse repeats) keep the previous mark
        for (int i = 0; i <= kNumStages; i++) cudaEventRecord(e->prof_ev[i], e->stream);
        st = spme_mulvec(e, 0, nrhs, 1.0, n3, d_f, 0.0, n3, d_v);
        e->prof_on = false;
        cudaStreamSynchronize(e->stream);
        for (int i = 0; i < kNumStages && st == kOk; i++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e->prof_ev[i], e->prof_ev[i + 1]);
            acc[i] += ms;
        }
    }
    for (int i = 0; i <= kNumStages; i++) cudaEventDestroy(e->prof_ev[i]);
    cudaFree(d_f);
    cudaFree(d_v);
    for (int i = 0; i < kNumStages; i++) stage_ms[i] = acc[i] / reps;
    return st;
}

void spme_free(SpmeEngine *e)
{
    if (!e) return;
    if (e->device >= 0) cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    void *ptrs[] = {e->d_tab0, e->d_tab2, e->d_kmap, e->d_tw_half, e->d_tw_full, e->d_rdi, e->d_rdi2, e->d_self,
                    e->d_sp_perm, e->d_sp_base, e->d_sp_w, e->d_sp_binstart, e->d_seg_start, e->d_seg_meta,
                    e->d_seg_slot, e->d_seg_w, e->d_stencil, e->d_rs_perm,
                    e->d_rs_cell, e->d_rs_pos, e->d_rs_posf, e->d_rs_inv, e->d_rs_cellstart, e->d_counts, e->d_key_sp, e->d_key_rs,
                    e->d_tmp_base, e->d_tmp_w, e->d_tmp_pos, e->d_cgrid, e->d_fs_sp, e->d_fs_rs,
                    e->d_vrecip, e->d_vreal, e->d_fin, e->d_vout, e->d_err};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    tc_free(e);
    pair_list_free(e);
    for (int q = 0; q < 3; q++) {
        if (e->side[q]) {
            cudaStreamSynchronize(e->side[q]);
            cudaStreamDestroy(e->side[q]);
            e->side[q] = nullptr;
        }
        if (e->ev_join[q]) cudaEventDestroy(e->ev_join[q]);
        e->ev_join[q] = nullptr;
    }
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    e->ev_fork = nullptr;
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    e->stream = nullptr;
}

// ---------------------------------------------------------------------------
// Packed multi-system passes (packed.h): one launch per pass and grid class
// ---------------------------------------------------------------------------

#define PK_LAUNCH_CHECK()                                                                 \
    do {                                                                                  \
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                        \
        if (cudaGetLastError() != cudaSuccess) return kErrCuda;                           \
    } while (0)

static long long packed_slot_stride(const PackedClass &c, int nr)
{
    return (long long)nr * 3 * c.K * c.K * c.XS;
}

template <int K>
static int packed_x_spread_k(const PackedClass &c, const PackedSys *d_sys, const PackedIO *d_io, int nslots,
                             int nr, cudaStream_t s)
{
    const size_t smx = (size_t)x_rows_floats<K>() * sizeof(float);
    if (cudaFuncSetAttribute(k_spread_xfwd_packed<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx) !=
        cudaSuccess)
        return kErrCuda;
    k_spread_xfwd_packed<K><<<dim3(nr, c.nby, c.nbz * nslots), kXThreads, smx, s>>>(
        d_sys, d_io, c.d_slot_sys, c.nbz, c.XS, c.tw_half, c.tw_full, c.d_grid, packed_slot_stride(c, nr));
    PK_LAUNCH_CHECK();
    return kOk;
}

template <int K>
static int packed_x_interp_k(const PackedClass &c, const PackedSys *d_sys, const PackedIO *d_io, int nslots,
                             int nr, int *err, cudaStream_t s)
{
    const size_t smx = (size_t)x_rows_floats<K>() * sizeof(float);
    if (cudaFuncSetAttribute(k_xinv_interp_packed<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx) !=
        cudaSuccess)
        return kErrCuda;
    k_xinv_interp_packed<K><<<dim3(nr, c.nby, c.nbz * nslots), kXThreads, smx, s>>>(
        d_sys, d_io, c.d_slot_sys, c.nbz, c.XS, c.tw_half, c.tw_full, c.d_grid, packed_slot_stride(c, nr), err);
    PK_LAUNCH_CHECK();
    return kOk;
}

template <int K>
static int packed_y_k(const PackedClass &c, int nslots, int nr, bool inverse, int *err, cudaStream_t s)
{
    constexpr int H = K / 2;
    const size_t smy = (size_t)K * kTileX * sizeof(float2);
    const int ntile = (H + 1 + kTileX - 1) / kTileX;
    const int ty = kTileX * FftShape<K>::N2;
    auto kern = inverse ? k_ypass_tma<K, true> : k_ypass_tma<K, false>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy) != cudaSuccess)
        return kErrCuda;
    kern<<<dim3(ntile, K, nr * 3 * nslots), ty, smy, s>>>(c.tmap_y, c.tw_full, err, 0);
    PK_LAUNCH_CHECK();
    return kOk;
}

template <int K>
static int packed_z_k(const PackedClass &c, int nslots, int nr, int *err, cudaStream_t s)
{
    constexpr int H = K / 2;
    constexpr int TZ = z_fused_tile(K);
    const size_t smzf = (size_t)3 * K * TZ * sizeof(float2) + (size_t)K * TZ * sizeof(float);
    const int ntilezf = (H + 1 + TZ - 1) / TZ;
    auto kern = k_zpass_fused_tma<K, false, true>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smzf) != cudaSuccess)
        return kErrCuda;
    kern<<<dim3(nr * nslots, ntilezf, K), kZFusedThreads<K>(), smzf, s>>>(c.tmap_zf, c.tmap_tabf, c.tw_full,
                                                                         c.d_kmap, err, 0, c.d_slot_tab, nr);
    PK_LAUNCH_CHECK();
    return kOk;
}

#define PK_DISPATCH(fn, ...)                                                              \
    switch (c.K) {                                                                        \
        case 32: return fn<32>(__VA_ARGS__);                                              \
        case 64: return fn<64>(__VA_ARGS__);                                              \
        case 128: return fn<128>(__VA_ARGS__);                                            \
        case 256: return fn<256>(__VA_ARGS__);                                            \
        default: return kErrUnsupported;                                                  \
    }

int packed_x_spread(const PackedClass &c, const PackedSys *d_sys, const PackedIO *d_io, int nslots, int nr,
                    cudaStream_t s)
{
    PK_DISPATCH(packed_x_spread_k, c, d_sys, d_io, nslots, nr, s)
}

int packed_x_interp(const PackedClass &c, const PackedSys *d_sys, const PackedIO *d_io, int nslots, int nr,
                    int *err, cudaStream_t s)
{
    PK_DISPATCH(packed_x_interp_k, c, d_sys, d_io, nslots, nr, err, s)
}

int packed_y(const PackedClass &c, int nslots, int nr, bool inverse, int *err, cudaStream_t s)
{
    PK_DISPATCH(packed_y_k, c, nslots, nr, inverse, err, s)
}

int packed_z(const PackedClass &c, int nslots, int nr, int *err, cudaStream_t s)
{
    PK_DISPATCH(packed_z_k, c, nslots, nr, err, s)
}

}  // namespace sdt
