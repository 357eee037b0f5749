// Real-space Ewald RPY sum over the periodic cell list.
//
// Replaces the reference's explicit pair list + FP64 BCSR matrix
// (PairListR::FindPairs src/pairlist/pair_r.cc:95-170,
//  MobSpme::BuildSparseReal src/mob/mob_spme.cc:135-202,
//  SpMV3x3 src/util/sparse.cc:79-153): for every target particle i and every
// j != i within rmax (minimum image), the 3x3 block
//     T_ij = (xa - ya) e e^T + ya I        (e = r_ij / |r_ij|)
// with (xa, ya) = scalars_ewald_F(xi, r, a_i, a_j) (src/mob/ewald.h:55-85)
// plus the RPY overlap correction when r < a_i + a_j.  The self block is
// added in FP64 by the combine step.  Separations are formed in FP64 (minimum
// image), everything after that in FP32.
//
// Two ways to apply it, same pairs and same FP32 scalars:
//  * pair list (default): at Update, one pass counts and one pass stores, per
//    target in cell order, the pairs as (ex, ey, ez, ya) + (xa - ya, j) --
//    24 bytes a pair, the compressed form of the reference's BCSR blocks.
//    Every product then streams the list once for up to 16 right-hand sides.
//  * on the fly: every product walks the cell list again (no storage; used
//    when the list does not fit or is switched off, and by the
//    allocation-free entry point).
//
// Candidate walk (both): one warp per target (targets in cell order, so the
// warps of a CTA share most of their neighbour cells in L1).  Cells are
// stored z-fastest, so the five z neighbours of each (dx, dy) stencil column
// form one contiguous particle range (two when the column wraps): lanes sweep
// 25 such ranges with an FP32 distance prefilter, candidates are pushed to a
// per-warp queue and handed on 32 at a time with all lanes busy, where the
// exact FP64 test r <= rmax decides.
//
// Applying blocks (both): lane = (pair sub-slot, right-hand side).  With RB
// right-hand sides a step takes 32/RB pairs, and the RB lanes of one pair
// read that source's RB force vectors as one contiguous float4 row.  Partial
// sums of one right-hand side are reduced over the sub-slots with shuffles.
#include "engine.h"
#include "packed.h"

namespace sdt {

#define SDT_LAUNCH_CHECK_RS()                                                             \
    do {                                                                                  \
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                        \
        cudaError_t err_ = cudaGetLastError();                                            \
        if (err_ != cudaSuccess)                                                          \
            return set_error(e, kErrCuda, std::string("real-space launch: ") + cudaGetErrorString(err_)); \
    } while (0)

constexpr int kRsWarps = 8;
constexpr int kQueue = 64;

// (xa, ya) of scalars_ewald_F plus the overlap terms of mob_spme.cc:170-175.
__device__ __forceinline__ void rpy_scalars(float xi, float xi_spi, float r, float rinv, float aa,
                                            float ab, float &xa, float &ya)
{
    const float xir = xi * r;
    const float xir2 = xir * xir;
    const float r2inv = rinv * rinv;
    const float erfcxir = erfcf(xir);
    const float expxir2 = xi_spi * expf(-xir2);
    const float s6 = (aa * aa + ab * ab) * (1.0f / 6.0f);
    const float a0 = 2.0f * (-3.0f + xir2 * 2.0f) * expxir2 + erfcxir * rinv;
    const float b0 = 2.0f * (1.0f - xir2 * 2.0f) * expxir2 + erfcxir * rinv;
    const float a2 = 4.0f * r2inv * (1.0f + xir2 * (14.0f + xir2 * (-20.0f + xir2 * 4.0f))) * expxir2 +
                     2.0f * r2inv * rinv * erfcxir;
    const float b2 = -4.0f * r2inv * (3.0f + xir2 * (2.0f + xir2 * (-16.0f + xir2 * 4.0f))) * expxir2 -
                     6.0f * r2inv * rinv * erfcxir;
    ya = 0.75f * (a0 + a2 * s6);
    xa = 0.75f * (b0 + b2 * s6) + ya;
    if (r < aa + ab) {
        const float s2 = aa * aa + ab * ab;
        xa += -(1.5f - s2 * 0.5f * r2inv) * rinv + 2.0f / (aa + ab) - 3.0f * r / 8.0f / s2;
        ya += -(0.75f + s2 * 0.25f * r2inv) * rinv + 2.0f / (aa + ab) - 9.0f * r / 16.0f / s2;
    }
}

// Geometry shared by the kernels that walk the cell list.
struct CellWalk {
    int n, nc, ncol;
    const int *cols;          // stencil columns, packed (dx+8) | (dy+8)<<5
    const double4 *pos;       // FP64 positions + radius, cell order
    const float4 *posf;       // FP32 copy (prefilter)
    const int *cell;          // cell of each slot
    const int *cellstart;     // [nc^3 + 1]
    double box, rmax2;
    float rcand2;             // prefilter radius^2
};

// Exact inclusion test of candidate j for target s at pi: FP64 minimum-image
// separation, r <= rmax and j != i (d2 > 0).
__device__ __forceinline__ bool exact_pair(const CellWalk &w, const double4 &pi, const double4 &pj,
                                           double &ddx, double &ddy, double &ddz, double &d2)
{
    const double invbox = 1.0 / w.box;
    ddx = pj.x - pi.x;
    ddy = pj.y - pi.y;
    ddz = pj.z - pi.z;
    ddx -= w.box * rint(ddx * invbox);
    ddy -= w.box * rint(ddy * invbox);
    ddz -= w.box * rint(ddz * invbox);
    d2 = ddx * ddx + ddy * ddy + ddz * ddz;
    return d2 <= w.rmax2 && d2 > 0.0;
}

// Walk the stencil columns of target slot s: FP32-prefiltered candidates go
// to the warp's queue (64 entries) and drain(count) is called whenever 32 are
// queued and once at the end for the rest.  drain reads queue[lane] for
// lane < count and must leave the queue untouched.
template <typename Drain>
__device__ __forceinline__ void walk_candidates(const CellWalk &w, int s, int lane, int *queue,
                                                Drain &&drain)
{
    const float4 pif = w.posf[s];
    const int ci = w.cell[s];
    const int nc = w.nc;
    const int cx = ci / (nc * nc), cy = (ci / nc) % nc, cz = ci % nc;
    const float boxf = (float)w.box, invboxf = (float)(1.0 / w.box);
    int qn = 0;  // entries in the queue (uniform across the warp)

    auto scan = [&](int j0, int j1) {
        for (int jb = j0; jb < j1; jb += 32) {
            const int j = jb + lane;
            bool ok = false;
            if (j < j1 && j != s) {
                const float4 pj = w.posf[j];
                float dx = pj.x - pif.x, dy = pj.y - pif.y, dz = pj.z - pif.z;
                dx -= boxf * rintf(dx * invboxf);
                dy -= boxf * rintf(dy * invboxf);
                dz -= boxf * rintf(dz * invboxf);
                ok = dx * dx + dy * dy + dz * dz <= w.rcand2;
            }
            const unsigned mask = __ballot_sync(0xffffffffu, ok);
            const int cnt = __popc(mask);
            if (cnt == 0) continue;
            if (ok) queue[qn + __popc(mask & ((1u << lane) - 1u))] = j;
            __syncwarp();
            qn += cnt;
            if (qn >= 32) {
                drain(32);
                const int rest = qn - 32;
                int tmp = 0;
                if (lane < rest) tmp = queue[32 + lane];
                __syncwarp();
                if (lane < rest) queue[lane] = tmp;
                __syncwarp();
                qn = rest;
            }
        }
    };

    for (int k = 0; k < w.ncol; k++) {
        const int code = w.cols[k];
        const int dx = (code & 31) - 8, dy = ((code >> 5) & 31) - 8;
        const int nx = (cx + dx + 2 * nc) % nc, ny = (cy + dy + 2 * nc) % nc;
        const int base = (nx * nc + ny) * nc;
        if (nc < 5) {
            scan(w.cellstart[base], w.cellstart[base + nc]);  // every z cell of the column
        } else {
            const int lo = cz - 2, hi = cz + 2;
            if (lo >= 0 && hi < nc) {
                scan(w.cellstart[base + lo], w.cellstart[base + hi + 1]);
            } else if (lo < 0) {
                scan(w.cellstart[base + lo + nc], w.cellstart[base + nc]);
                scan(w.cellstart[base], w.cellstart[base + hi + 1]);
            } else {
                scan(w.cellstart[base + lo], w.cellstart[base + nc]);
                scan(w.cellstart[base], w.cellstart[base + hi - nc + 1]);
            }
        }
    }
    if (qn > 0) drain(qn);
}

// Block scalars of an accepted pair: e = r/|r| and (ya, xa - ya).
__device__ __forceinline__ void pair_block(double ddx, double ddy, double ddz, double d2, float ai,
                                           float aj, float xi, float xi_spi, float4 &pe, float &pc)
{
    const float d2f = (float)d2;
    const float rinv = rsqrtf(d2f);
    const float r = d2f * rinv;
    float xa, ya;
    rpy_scalars(xi, xi_spi, r, rinv, ai, aj, xa, ya);
    pe = make_float4((float)ddx * rinv, (float)ddy * rinv, (float)ddz * rinv, ya);
    pc = xa - ya;
}

// acc += T f = ya f + (xa - ya) (e . f) e
__device__ __forceinline__ void apply_block(const float4 &e, float c, float f0, float f1, float f2,
                                            float &a0, float &a1, float &a2)
{
    const float ef = c * fmaf(e.x, f0, fmaf(e.y, f1, e.z * f2));
    a0 = fmaf(ef, e.x, fmaf(e.w, f0, a0));
    a1 = fmaf(ef, e.y, fmaf(e.w, f1, a1));
    a2 = fmaf(ef, e.z, fmaf(e.w, f2, a2));
}

// Sum the partials of right-hand side lane % RB over the 32/RB sub-slots and
// store them (lanes < RB) at vreal[r0 + lane][3i .. 3i+2].
template <int RB>
__device__ __forceinline__ void store_rows(float a0, float a1, float a2, int lane, int i, int n,
                                           int r0, float *__restrict__ vreal)
{
#pragma unroll
    for (int o = 16; o >= RB; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (lane < RB) {
        float *out = vreal + (size_t)(r0 + lane) * 3 * n + 3 * i;
        out[0] = a0;
        out[1] = a1;
        out[2] = a2;
    }
}

// ---------------------------------------------------------------------------
// On-the-fly product: walk, test, evaluate and apply in one kernel.
// Forces fs: row j holds nr vectors of FC floats (FC = 4: float4 rows).
// ---------------------------------------------------------------------------
template <int RB, int FC>
__global__ void __launch_bounds__(32 * kRsWarps)
k_real_space(CellWalk w, const int *__restrict__ perm, const float *__restrict__ fs, int fstride,
             int r0, float xi, float xi_spi, float *__restrict__ vreal)
{
    static_assert(RB >= 1 && RB <= 32 && (32 % RB) == 0, "RB must divide the warp");
    static_assert(FC == 3 || FC == 4, "forces are stored as 3 or 4 floats");
    constexpr int kPairsPerStep = 32 / RB;
    __shared__ int queue[kRsWarps][kQueue];
    __shared__ float4 pair_e[kRsWarps][32];  // (ex, ey, ez, ya) of the pairs being applied
    __shared__ float2 pair_c[kRsWarps][32];  // (xa - ya, source slot as int bits)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kRsWarps + warp;
    if (s >= w.n) return;
    const double4 pi = w.pos[s];
    const int rl = lane % RB, pl = lane / RB;
    const float *frow = fs + (size_t)FC * (r0 + rl);
    float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f;

    auto drain = [&](int count) {
        float4 pe = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float pc = 0.0f;
        int pj = s;  // excluded slots keep a valid index and contribute zero
        if (lane < count) {
            const int j = queue[warp][lane];
            const double4 q = w.pos[j];
            double ddx, ddy, ddz, d2;
            if (exact_pair(w, pi, q, ddx, ddy, ddz, d2)) {
                pair_block(ddx, ddy, ddz, d2, (float)pi.w, (float)q.w, xi, xi_spi, pe, pc);
                pj = j;
            }
        }
        pair_e[warp][lane] = pe;
        pair_c[warp][lane] = make_float2(pc, __int_as_float(pj));
        __syncwarp();
        const int steps = (count + kPairsPerStep - 1) / kPairsPerStep;
        for (int t = 0; t < steps; t++) {
            const int q = t * kPairsPerStep + pl;
            const float4 e = pair_e[warp][q];
            const float2 cj = pair_c[warp][q];
            const float *fj = frow + (size_t)__float_as_int(cj.y) * fstride;
            float f0, f1, f2;
            if constexpr (FC == 4) {
                const float4 f = *reinterpret_cast<const float4 *>(fj);
                f0 = f.x; f1 = f.y; f2 = f.z;
            } else {
                f0 = fj[0]; f1 = fj[1]; f2 = fj[2];
            }
            apply_block(e, cj.x, f0, f1, f2, acc0, acc1, acc2);
        }
        __syncwarp();
    };
    walk_candidates(w, s, lane, queue[warp], drain);
    store_rows<RB>(acc0, acc1, acc2, lane, perm[s], w.n, r0, vreal);
}

// ---------------------------------------------------------------------------
// Pair list.  FILL = false: count[s] = number of pairs of target s.
// FILL = true: store them at start[s] .. start[s+1] in walk order (the same
// walk and the same FP64 test, so the counts match exactly).
// ---------------------------------------------------------------------------
template <bool FILL>
__global__ void __launch_bounds__(32 * kRsWarps)
k_pair_build(CellWalk w, float xi, float xi_spi, int *__restrict__ count,
             const long long *__restrict__ start, float4 *__restrict__ pl_e,
             float2 *__restrict__ pl_c)
{
    __shared__ int queue[kRsWarps][kQueue];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kRsWarps + warp;
    if (s >= w.n) return;
    const double4 pi = w.pos[s];
    long long out = FILL ? start[s] : 0;
    const long long end = FILL ? start[s + 1] : 0;
    int found = 0;

    auto drain = [&](int count_q) {
        bool ok = false;
        int j = 0;
        double ddx = 0.0, ddy = 0.0, ddz = 0.0, d2 = 0.0;
        double4 q = make_double4(0.0, 0.0, 0.0, 0.0);
        if (lane < count_q) {
            j = queue[warp][lane];
            q = w.pos[j];
            ok = exact_pair(w, pi, q, ddx, ddy, ddz, d2);
        }
        const unsigned mask = __ballot_sync(0xffffffffu, ok);
        if (FILL && ok) {
            const long long slot = out + __popc(mask & ((1u << lane) - 1u));
            if (slot < end) {  // the count pass found the same pairs
                float4 pe;
                float pc;
                pair_block(ddx, ddy, ddz, d2, (float)pi.w, (float)q.w, xi, xi_spi, pe, pc);
                pl_e[slot] = pe;
                pl_c[slot] = make_float2(pc, __int_as_float(j));
            }
        }
        out += __popc(mask);
        found += __popc(mask);
        __syncwarp();
    };
    walk_candidates(w, s, lane, queue[warp], drain);
    if (!FILL && lane == 0) count[s] = found;
}

// Exclusive scan of count[0..n) into start[0..n] (64-bit) by one block.
__global__ void __launch_bounds__(1024) k_scan64(int n, const int *__restrict__ count,
                                                 long long *__restrict__ start)
{
    __shared__ long long part[1024];
    const int tid = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int b = tid * per;
    const int e = min(n, b + per);
    long long s = 0;
    for (int i = b; i < e; i++) s += count[i];
    part[tid] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const long long v = (tid >= off) ? part[tid - off] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    long long run = part[tid] - s;
    for (int i = b; i < e; i++) {
        start[i] = run;
        run += count[i];
    }
    if (tid == 1023) start[n] = part[1023];
}

// Product from the stored pair list: warp per target slot s, RB right-hand
// sides r0 .. r0+RB-1 of the float4 force rows fs ([N][nr]).  The warp reads
// its row of the list in batches of 32 pairs with coalesced streaming loads,
// one batch ahead of the one it applies, and stages the current batch in
// shared memory; a batch takes RB steps of 32/RB pairs, whose force loads are
// issued kFB at a time before the math.
// The work of one CTA: targets block * kRsWarps + warp.
template <int RB>
__device__ __forceinline__ void pair_apply_block(int n, const long long *__restrict__ start,
                                                 const float4 *__restrict__ pl_e, const float2 *__restrict__ pl_c,
                                                 const int *__restrict__ perm, const float4 *__restrict__ fs,
                                                 int nr, int r0, float *__restrict__ vreal, int block)
{
    static_assert(RB >= 1 && RB <= 32 && (32 % RB) == 0, "RB must divide the warp");
    constexpr int kPairsPerStep = 32 / RB;
    constexpr int kFB = RB < 8 ? RB : 8;  // force loads in flight per lane
    // 32-pair batches of the list in flight per warp: with one RHS a pair
    // carries little work, so the stream needs more loads in flight
    constexpr int PF = RB == 1 ? 4 : 1;
    __shared__ float4 se[kRsWarps][32];
    __shared__ float2 sc[kRsWarps][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = block * kRsWarps + warp;
    if (s >= n) return;
    const int rl = lane % RB, pl = lane / RB;
    const float4 *frow = fs + r0 + rl;
    const long long b = start[s], e = start[s + 1];
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
    // slots past the row end hold a zero block on a valid source (s itself)
    const float2 pad = make_float2(0.0f, __int_as_float(s));
    float4 ne[PF];
    float2 nc[PF];
#pragma unroll
    for (int u = 0; u < PF; u++) {
        ne[u] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        nc[u] = pad;
        if (b + 32 * u + lane < e) {
            ne[u] = __ldcs(&pl_e[b + 32 * u + lane]);
            nc[u] = __ldcs(&pl_c[b + 32 * u + lane]);
        }
    }
    for (long long base0 = b; base0 < e; base0 += 32 * PF)
#pragma unroll
    for (int ub = 0; ub < PF; ub++) {
        const long long base = base0 + 32 * ub;
        if (base >= e) break;  // the same in every lane
        __syncwarp();
        se[warp][lane] = ne[ub];
        sc[warp][lane] = nc[ub];
        __syncwarp();
        const long long qn = base + 32 * PF + lane;
        ne[ub] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        nc[ub] = pad;
        if (qn < e) {
            ne[ub] = __ldcs(&pl_e[qn]);
            nc[ub] = __ldcs(&pl_c[qn]);
        }
        const int cnt = (int)min(32LL, e - base);
        const int steps = (cnt + kPairsPerStep - 1) / kPairsPerStep;
#pragma unroll
        for (int t0 = 0; t0 < RB; t0 += kFB) {
            if (t0 >= steps) break;
            float4 fv[kFB];
#pragma unroll
            for (int u = 0; u < kFB; u++) {
                const int q = (t0 + u) * kPairsPerStep + pl;
                fv[u] = frow[(size_t)__float_as_int(sc[warp][q].y) * nr];
            }
#pragma unroll
            for (int u = 0; u < kFB; u++) {
                const int q = (t0 + u) * kPairsPerStep + pl;
                apply_block(se[warp][q], sc[warp][q].x, fv[u].x, fv[u].y, fv[u].z, a0, a1, a2);
            }
        }
    }
    store_rows<RB>(a0, a1, a2, lane, perm[s], n, r0, vreal);
}

template <int RB>
__global__ void __launch_bounds__(32 * kRsWarps, 2)
k_pair_apply(int n, const long long *__restrict__ start, const float4 *__restrict__ pl_e,
             const float2 *__restrict__ pl_c, const int *__restrict__ perm,
             const float4 *__restrict__ fs, int nr, int r0, float *__restrict__ vreal)
{
    pair_apply_block<RB>(n, start, pl_e, pl_c, perm, fs, nr, r0, vreal, blockIdx.x);
}

// Packed over many systems: CTA blockIdx.x takes block map[blockIdx.x].y of
// the system in slot map[blockIdx.x].x.
template <int RB>
__global__ void __launch_bounds__(32 * kRsWarps, 2)
k_pair_apply_packed(const PackedSys *__restrict__ sys, const PackedIO *__restrict__ io,
                    const int *__restrict__ act, const int2 *__restrict__ map, int nr, int r0)
{
    const int2 m = map[blockIdx.x];
    const int g = act[m.x];
    const PackedSys &S = sys[g];
    pair_apply_block<RB>(S.n, S.pl_start, S.pl_e, S.pl_c, S.rs_perm, io[g].fs_rs, nr, r0, io[g].vreal, m.y);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

// Candidate radius of the FP32 prefilter: rmax plus a margin that covers the
// FP32 rounding of positions up to the box edge.
static float candidate_r2(const SpmeEngine *e)
{
    const double rc = e->rmax + 1e-3 + 1e-6 * e->box;
    return (float)(rc * rc);
}

static CellWalk cell_walk(const SpmeEngine *e)
{
    CellWalk w;
    w.n = e->npos;
    w.nc = e->nc;
    w.ncol = e->nstencil;
    w.cols = e->d_stencil;
    w.pos = e->d_rs_pos;
    w.posf = e->d_rs_posf;
    w.cell = e->d_rs_cell;
    w.cellstart = e->d_rs_cellstart;
    w.box = e->box;
    w.rmax2 = e->rmax * e->rmax;
    w.rcand2 = candidate_r2(e);
    return w;
}

static float xi_f(const SpmeEngine *e) { return (float)e->xi; }
static float xi_spi_f(const SpmeEngine *e) { return (float)(e->xi / sqrt(M_PI)); }

// Run L::run<RB>(r0) for RB in {16, 8, 4, 2, 1} until nr RHS are covered.
template <typename L>
static int for_rhs_blocks(int nr, const L &l)
{
    int r0 = 0;
    while (r0 < nr) {
        const int left = nr - r0;
        int st, rb;
        if (left >= 16) { rb = 16; st = l.template run<16>(r0); }
        else if (left >= 8) { rb = 8; st = l.template run<8>(r0); }
        else if (left >= 4) { rb = 4; st = l.template run<4>(r0); }
        else if (left >= 2) { rb = 2; st = l.template run<2>(r0); }
        else { rb = 1; st = l.template run<1>(r0); }
        if (st != kOk) return st;
        r0 += rb;
    }
    return kOk;
}

struct PairApplyLaunch {
    SpmeEngine *e;
    int grid, nr;
    template <int RB>
    int run(int r0) const
    {
        k_pair_apply<RB><<<grid, 32 * kRsWarps, 0, e->stream>>>(
            e->npos, e->d_pl_start, e->d_pl_e, e->d_pl_c, e->d_rs_perm,
            reinterpret_cast<const float4 *>(e->d_fs_rs), nr, r0, e->d_vreal);
        SDT_LAUNCH_CHECK_RS();
        return kOk;
    }
};

template <int FC>
struct WalkLaunch {
    SpmeEngine *e;
    CellWalk w;
    int grid, nr;
    const float *fs;
    float *vreal;
    template <int RB>
    int run(int r0) const
    {
        k_real_space<RB, FC><<<grid, 32 * kRsWarps, 0, e->stream>>>(
            w, e->d_rs_perm, fs, FC * nr, r0, xi_f(e), xi_spi_f(e), vreal);
        SDT_LAUNCH_CHECK_RS();
        return kOk;
    }
};

int real_space_launch(SpmeEngine *e, int nr)
{
    const int grid = (e->npos + kRsWarps - 1) / kRsWarps;
    if (e->pl_ready) return for_rhs_blocks(nr, PairApplyLaunch{e, grid, nr});
    return for_rhs_blocks(nr, WalkLaunch<4>{e, cell_walk(e), grid, nr, e->d_fs_rs, e->d_vreal});
}

// On-the-fly product with caller-supplied force and output buffers ([N][nr][3]
// forces in cell order, [nr][3N] output).
int real_space_launch_into(SpmeEngine *e, int nr, const float *fs, float *vreal)
{
    const int grid = (e->npos + kRsWarps - 1) / kRsWarps;
    return for_rhs_blocks(nr, WalkLaunch<3>{e, cell_walk(e), grid, nr, fs, vreal});
}

// The same with float4 force rows ([N][nr] float4, cell order) on stream s:
// the packed path's fallback for a system without a stored pair list.
int real_space_walk_into4(SpmeEngine *e, int nr, const float4 *fs, float *vreal, cudaStream_t s)
{
    const int grid = (e->npos + kRsWarps - 1) / kRsWarps;
    cudaStream_t saved = e->stream;
    e->stream = s;
    const int st =
        for_rhs_blocks(nr, WalkLaunch<4>{e, cell_walk(e), grid, nr, reinterpret_cast<const float *>(fs), vreal});
    e->stream = saved;
    return st;
}

int packed_pair_targets_per_cta() { return kRsWarps; }

struct PackedPairLaunch {
    const PackedSys *sys;
    const PackedIO *io;
    const int *act;
    const int2 *map;
    int nblocks, nr;
    cudaStream_t s;
    template <int RB>
    int run(int r0) const
    {
        k_pair_apply_packed<RB><<<nblocks, 32 * kRsWarps, 0, s>>>(sys, io, act, map, nr, r0);
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
        return cudaGetLastError() == cudaSuccess ? kOk : kErrCuda;
    }
};

int packed_pair_apply(const PackedSys *d_sys, const PackedIO *d_io, const int *d_act, const int2 *d_map,
                      int nblocks, int nr, cudaStream_t s)
{
    if (nblocks <= 0) return kOk;
    return for_rhs_blocks(nr, PackedPairLaunch{d_sys, d_io, d_act, d_map, nblocks, nr, s});
}

// Build the pair list for the current positions (after the cell sort of
// spme_update).  Grows the list storage when needed; if it cannot be had, the
// engine falls back to the on-the-fly product (pl_ready stays false).
int pair_list_build(SpmeEngine *e)
{
    e->pl_ready = false;
    if (!e->pl_enabled) return kOk;
    const int n = e->npos;
    const int grid = (n + kRsWarps - 1) / kRsWarps;
    const CellWalk w = cell_walk(e);
    if (!e->d_pl_count) {
        if (cudaMalloc(&e->d_pl_count, (size_t)n * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&e->d_pl_start, (size_t)(n + 1) * sizeof(long long)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(e, kErrAlloc, "device allocation of the pair-list index failed");
        }
    }
    k_pair_build<false><<<grid, 32 * kRsWarps, 0, e->stream>>>(w, xi_f(e), xi_spi_f(e), e->d_pl_count,
                                                               nullptr, nullptr, nullptr);
    SDT_LAUNCH_CHECK_RS();
    k_scan64<<<1, 1024, 0, e->stream>>>(n, e->d_pl_count, e->d_pl_start);
    SDT_LAUNCH_CHECK_RS();
    long long total = 0;
    if (cudaMemcpyAsync(&total, e->d_pl_start + n, sizeof(long long), cudaMemcpyDeviceToHost,
                        e->stream) != cudaSuccess ||
        cudaStreamSynchronize(e->stream) != cudaSuccess)
        return set_error(e, kErrCuda, "reading the pair count failed");
    if (total > e->pl_cap) {
        cudaFree(e->d_pl_e);
        cudaFree(e->d_pl_c);
        e->d_pl_e = nullptr;
        e->d_pl_c = nullptr;
        e->pl_cap = 0;
        const long long cap = total + total / 8 + 1024;
        const size_t bytes = (size_t)cap * (sizeof(float4) + sizeof(float2));
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || bytes > free_b / 2) {
            cudaGetLastError();
            return kOk;  // too large: products walk the cells instead
        }
        if (cudaMalloc(&e->d_pl_e, (size_t)cap * sizeof(float4)) != cudaSuccess ||
            cudaMalloc(&e->d_pl_c, (size_t)cap * sizeof(float2)) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(e->d_pl_e);
            e->d_pl_e = nullptr;
            return kOk;
        }
        e->pl_cap = cap;
    }
    e->pl_pairs = total;
    k_pair_build<true><<<grid, 32 * kRsWarps, 0, e->stream>>>(w, xi_f(e), xi_spi_f(e), nullptr,
                                                              e->d_pl_start, e->d_pl_e, e->d_pl_c);
    SDT_LAUNCH_CHECK_RS();
    e->pl_ready = true;
    return kOk;
}

void pair_list_free(SpmeEngine *e)
{
    cudaFree(e->d_pl_count);
    cudaFree(e->d_pl_start);
    cudaFree(e->d_pl_e);
    cudaFree(e->d_pl_c);
    e->d_pl_count = nullptr;
    e->d_pl_start = nullptr;
    e->d_pl_e = nullptr;
    e->d_pl_c = nullptr;
    e->pl_cap = 0;
    e->pl_ready = false;
}

}  // namespace sdt
