// Packed multi-system mobility product (packed.h): set-up, descriptors, the
// force gather and final combine kernels, and the product's orchestration.
#include <algorithm>
#include <cstring>
#include <map>

#include "packed.h"

namespace sdt {

// Work-space slices start on multiples of this many floats (256 bytes), so
// the float4 force rows are 16-byte aligned and every slice is coalesced.
constexpr size_t kWorkAlign = 64;

static inline size_t align_work(size_t nfloats) { return (nfloats + kWorkAlign - 1) / kWorkAlign * kWorkAlign; }

static int pk_error(PackedBatch *pb, int st, const std::string &msg)
{
    pb->last_error = msg;
    return st;
}

#define PK_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t err_ = (call);                                                        \
        if (err_ != cudaSuccess)                                                          \
            return pk_error(pb, kErrCuda, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

// FP64 forces of every active system -> FP32 copies in spread order
// ([r][c][n]) and cell order ([n][r] float4).  CTA blockIdx.x takes
// spread-order slots [256 * map.y, +256) of the system in slot map.x.
__global__ void __launch_bounds__(kPackedElemThreads)
k_pk_gather(const PackedSys *__restrict__ sys, const PackedIO *__restrict__ io, const int *__restrict__ act,
            const int2 *__restrict__ map, int nr)
{
    const int2 m = map[blockIdx.x];
    const int g = act[m.x];
    const PackedSys &S = sys[g];
    const PackedIO &X = io[g];
    const int s = m.y * kPackedElemThreads + threadIdx.x;
    if (s >= S.n) return;
    const int i = S.sp_perm[s];
    const int q = S.rs_inv[i];
    for (int r = 0; r < nr; r++) {
        const double *fi = X.f + (size_t)r * X.ldf + 3 * i;
        const float a = (float)fi[0], b = (float)fi[1], c = (float)fi[2];
        X.fs_sp[((size_t)r * 3 + 0) * S.n + s] = a;
        X.fs_sp[((size_t)r * 3 + 1) * S.n + s] = b;
        X.fs_sp[((size_t)r * 3 + 2) * S.n + s] = c;
        X.fs_rs[(size_t)q * nr + r] = make_float4(a, b, c, 0.0f);
    }
}

// v := alpha (recip / L^3 + real + self f) + beta v per active system, FP64
// (beta == 0 ignores v).  CTA blockIdx.x takes elements [256 * map.y, +256)
// of the flattened [r][3n] block of the system in slot map.x.
__global__ void __launch_bounds__(kPackedElemThreads)
k_pk_combine(const PackedSys *__restrict__ sys, const PackedIO *__restrict__ io, const int *__restrict__ act,
             const int2 *__restrict__ map, int nr, double alpha, double beta)
{
    const int2 m = map[blockIdx.x];
    const int g = act[m.x];
    const PackedSys &S = sys[g];
    const PackedIO &X = io[g];
    const int n3 = 3 * S.n;
    const long long idx = (long long)m.y * kPackedElemThreads + threadIdx.x;
    if (idx >= (long long)n3 * nr) return;
    const int e = (int)(idx % n3), r = (int)(idx / n3);
    const double acc = (double)X.vrecip[(size_t)r * n3 + e] * S.invL3 + (double)X.vreal[(size_t)r * n3 + e] +
                       S.self[e / 3] * X.f[(size_t)r * X.ldf + e];
    double *out = X.v + (size_t)r * X.ldv + e;
    *out = (beta == 0.0 ? 0.0 : beta * *out) + alpha * acc;
}

int packed_gather(const PackedSys *d_sys, const PackedIO *d_io, const int *d_act, const int2 *d_map, int nblocks,
                  int nr, cudaStream_t s)
{
    if (nblocks <= 0) return kOk;
    k_pk_gather<<<nblocks, kPackedElemThreads, 0, s>>>(d_sys, d_io, d_act, d_map, nr);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrCuda;
}

int packed_combine(const PackedSys *d_sys, const PackedIO *d_io, const int *d_act, const int2 *d_map,
                   int nblocks, int nr, double alpha, double beta, cudaStream_t s)
{
    if (nblocks <= 0) return kOk;
    k_pk_combine<<<nblocks, kPackedElemThreads, 0, s>>>(d_sys, d_io, d_act, d_map, nr, alpha, beta);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError() == cudaSuccess ? kOk : kErrCuda;
}

int packed_create(PackedBatch *pb, const std::vector<SpmeEngine *> &eng, int rhs_cap, int device,
                  cudaStream_t stream)
{
    if (eng.empty() || rhs_cap <= 0) return pk_error(pb, kErrInvalid, "packed batch: no systems or rhs_cap <= 0");
    pb->device = device;
    pb->stream = stream;
    pb->nsys = (int)eng.size();
    pb->rhs_cap = rhs_cap;
    pb->eng = eng;
    std::map<int, int> by_k;
    pb->sys_cls.assign(pb->nsys, -1);
    for (int g = 0; g < pb->nsys; g++) {
        const SpmeEngine *e = eng[g];
        if (!e->mono) return pk_error(pb, kErrUnsupported, "packed batch: monodisperse systems only");
        if (e->K > 256 || !e->tma_tabs || !e->tma_enabled || !e->zfused)
            return pk_error(pb, kErrUnsupported, "packed batch: grids of K <= 256 with the TMA passes");
        auto it = by_k.find(e->K);
        if (it == by_k.end()) {
            it = by_k.emplace(e->K, (int)pb->cls.size()).first;
            PackedClass c;
            c.K = e->K;
            c.XS = e->XS;
            c.nby = e->nby;
            c.nbz = e->nbz;
            c.tw_half = e->d_tw_half;
            c.tw_full = e->d_tw_full;
            pb->cls.push_back(c);
        }
        pb->sys_cls[g] = it->second;
        pb->cls[it->second].sys.push_back(g);
    }
    PK_CUDA(cudaSetDevice(device));
    for (PackedClass &c : pb->cls) {
        const size_t ns = c.sys.size();
        const size_t plane = (size_t)c.K * c.K * c.XS;
        PK_CUDA(cudaMalloc(&c.d_grid, ns * rhs_cap * 3 * plane * sizeof(float2)));
        PK_CUDA(cudaMemsetAsync(c.d_grid, 0, ns * rhs_cap * 3 * plane * sizeof(float2), stream));
        PK_CUDA(cudaMalloc(&c.d_tab, ns * plane * sizeof(float)));
        PK_CUDA(cudaMalloc(&c.d_kmap, ns * c.K * sizeof(float)));
        PK_CUDA(cudaMalloc(&c.d_slot_sys, ns * sizeof(int)));
        PK_CUDA(cudaMalloc(&c.d_slot_tab, ns * sizeof(int)));
        for (size_t t = 0; t < ns; t++) {
            const SpmeEngine *e = eng[c.sys[t]];
            PK_CUDA(cudaMemcpyAsync(c.d_tab + t * plane, e->d_tab0, plane * sizeof(float), cudaMemcpyDeviceToDevice,
                                    stream));
            PK_CUDA(cudaMemcpyAsync(c.d_kmap + t * c.K, e->d_kmap, c.K * sizeof(float), cudaMemcpyDeviceToDevice,
                                    stream));
        }
        const unsigned long long K = c.K, XS = c.XS, el = sizeof(float2), fl = sizeof(float);
        const unsigned lines = (unsigned)std::min(c.K, 256);
        const unsigned long long planes = 3ull * rhs_cap * ns;
        const unsigned long long dy[3] = {XS, K, planes * K};
        const unsigned long long sy[2] = {XS * el, K * XS * el};
        const unsigned by[3] = {(unsigned)kTileX, lines, 1u};
        const unsigned long long dz[4] = {XS, K, K, planes};
        const unsigned long long sz[3] = {XS * el, K * XS * el, K * K * XS * el};
        const unsigned bzf[4] = {(unsigned)z_fused_tile(c.K), 1u, lines, 1u};
        const unsigned long long dt[4] = {XS, K, K, (unsigned long long)ns};
        const unsigned long long st[3] = {XS * fl, K * XS * fl, K * K * XS * fl};
        const unsigned bt[4] = {(unsigned)z_fused_tile(c.K), 1u, lines, 1u};
        if (!encode_tmap_f2(&c.tmap_y, c.d_grid, 3, dy, sy, by) ||
            !encode_tmap_f2(&c.tmap_zf, c.d_grid, 4, dz, sz, bzf) ||
            !encode_tmap(&c.tmap_tabf, c.d_tab, 4, 4, dt, st, bt))
            return pk_error(pb, kErrCuda, "packed batch: tensor-map encoding failed");
    }
    pb->sys_tab.assign(pb->nsys, 0);
    for (const PackedClass &c : pb->cls)
        for (size_t t = 0; t < c.sys.size(); t++) pb->sys_tab[c.sys[t]] = (int)t;
    PK_CUDA(cudaMalloc(&pb->d_sys, pb->nsys * sizeof(PackedSys)));
    PK_CUDA(cudaMalloc(&pb->d_io, pb->nsys * sizeof(PackedIO)));
    PK_CUDA(cudaMalloc(&pb->d_act, pb->nsys * sizeof(int)));
    for (PackedStaging &sg : pb->stg) {
        PK_CUDA(cudaMallocHost(&sg.h_io, pb->nsys * sizeof(PackedIO)));
        PK_CUDA(cudaMallocHost(&sg.h_act, pb->nsys * sizeof(int)));
        PK_CUDA(cudaMallocHost(&sg.h_slots, 2 * pb->nsys * sizeof(int)));
        PK_CUDA(cudaEventCreateWithFlags(&sg.ev, cudaEventDisableTiming));
        memset(sg.h_io, 0, pb->nsys * sizeof(PackedIO));
    }
    PK_CUDA(cudaMalloc(&pb->d_err, sizeof(int)));
    PK_CUDA(cudaMemsetAsync(pb->d_err, 0, sizeof(int), stream));
    // FP32 work space: per system [nr][3][n] + [n][nr]x4 + 2 x [nr][3n]
    // floats, each slice starting on a 256-byte boundary (kWorkAlign floats)
    size_t work = 0;
    for (SpmeEngine *e : eng) work += (size_t)e->npos * rhs_cap * (3 + 4 + 3 + 3) + 4 * kWorkAlign;
    PK_CUDA(cudaMalloc(&pb->d_work, work * sizeof(float)));
    pb->work_cap = work;
    PK_CUDA(cudaStreamSynchronize(stream));
    return kOk;
}

int packed_refresh(PackedBatch *pb)
{
    std::vector<PackedSys> h(pb->nsys);
    for (int g = 0; g < pb->nsys; g++) {
        const SpmeEngine *e = pb->eng[g];
        if (!e->updated) return pk_error(pb, kErrState, "packed batch: a system has not been updated");
        PackedSys &S = h[g];
        S.n = e->npos;
        S.p = e->p;
        S.nby = e->nby;
        S.invL3 = 1.0 / (e->box * e->box * e->box);
        S.tab = pb->sys_tab[g];
        S.seg_start = e->d_seg_start;
        S.seg_meta = e->d_seg_meta;
        S.seg_slot = e->d_seg_slot;
        S.seg_w = e->d_seg_w;
        S.sp_w = e->d_sp_w;
        S.sp_perm = e->d_sp_perm;
        S.rs_inv = e->d_rs_inv;
        S.rs_perm = e->d_rs_perm;
        S.self = e->d_self;
        S.pl_start = e->pl_ready ? e->d_pl_start : nullptr;
        S.pl_e = e->pl_ready ? e->d_pl_e : nullptr;
        S.pl_c = e->pl_ready ? e->d_pl_c : nullptr;
    }
    PK_CUDA(cudaMemcpyAsync(pb->d_sys, h.data(), h.size() * sizeof(PackedSys), cudaMemcpyHostToDevice, pb->stream));
    // the copy reads a host vector: let it finish before the vector goes
    PK_CUDA(cudaStreamSynchronize(pb->stream));
    return kOk;
}

// Grows the device per-CTA map buffer to `count` entries.
static int ensure_map(PackedBatch *pb, size_t count)
{
    if (count <= pb->map_cap) return kOk;
    PK_CUDA(cudaStreamSynchronize(pb->stream));
    cudaFree(pb->d_map);
    pb->d_map = nullptr;
    pb->map_cap = 0;
    const size_t cap = count + count / 4 + 1024;
    PK_CUDA(cudaMalloc(&pb->d_map, cap * sizeof(int2)));
    pb->map_cap = cap;
    return kOk;
}

// The next staging set, once the copies out of it have run.
static int next_staging(PackedBatch *pb, size_t map_count, PackedStaging **out)
{
    PackedStaging &sg = pb->stg[pb->stg_next];
    pb->stg_next = (pb->stg_next + 1) % kPackedRing;
    if (sg.pending) {
        PK_CUDA(cudaEventSynchronize(sg.ev));
        sg.pending = false;
    }
    if (map_count > sg.map_cap) {
        cudaFreeHost(sg.h_map);
        sg.h_map = nullptr;
        sg.map_cap = 0;
        const size_t cap = map_count + map_count / 4 + 1024;
        PK_CUDA(cudaMallocHost(&sg.h_map, cap * sizeof(int2)));
        sg.map_cap = cap;
    }
    *out = &sg;
    return kOk;
}

int packed_mulvec(PackedBatch *pb, int nact, const int *act, int nr, double alpha, const double *const *f,
                  const int *ldf, double beta, double *const *v, const int *ldv)
{
    if (nact <= 0) return kOk;
    if (nr <= 0 || nr > pb->rhs_cap) return pk_error(pb, kErrInvalid, "packed product: bad RHS count");
    cudaStream_t s = pb->stream;
    const int tpc = packed_pair_targets_per_cta();
    int nb_g = 0, nb_p = 0, nb_c = 0;
    for (int j = 0; j < nact; j++) {
        const SpmeEngine *e = pb->eng[act[j]];
        const int n = e->npos;
        nb_g += (n + kPackedElemThreads - 1) / kPackedElemThreads;
        nb_c += (3 * n * nr + kPackedElemThreads - 1) / kPackedElemThreads;
        if (e->pl_ready) nb_p += (n + tpc - 1) / tpc;
    }
    const size_t nmap = (size_t)nb_g + nb_p + nb_c;
    int st = ensure_map(pb, nmap);
    if (st != kOk) return st;
    PackedStaging *sg = nullptr;
    st = next_staging(pb, nmap, &sg);
    if (st != kOk) return st;
    // per-call descriptors: vectors and compact work slices in slot order
    float *w = pb->d_work;
    std::vector<int> pl_missing;
    int2 *mg = sg->h_map, *mp = mg + nb_g, *mc = mp + nb_p;
    int ig = 0, ip = 0, ic = 0;
    for (int j = 0; j < nact; j++) {
        const int g = act[j];
        const SpmeEngine *e = pb->eng[g];
        const int n = e->npos;
        PackedIO &X = sg->h_io[g];
        X.f = f[j];
        X.v = v[j];
        X.ldf = ldf[j];
        X.ldv = ldv[j];
        X.fs_sp = w;
        w += align_work((size_t)n * nr * 3);
        X.fs_rs = reinterpret_cast<float4 *>(w);
        w += align_work((size_t)n * nr * 4);
        X.vrecip = w;
        w += align_work((size_t)n * nr * 3);
        X.vreal = w;
        w += align_work((size_t)n * nr * 3);
        sg->h_act[j] = g;
        for (int b = 0; b < (n + kPackedElemThreads - 1) / kPackedElemThreads; b++) mg[ig++] = make_int2(j, b);
        if (e->pl_ready)
            for (int b = 0; b < (n + tpc - 1) / tpc; b++) mp[ip++] = make_int2(j, b);
        else
            pl_missing.push_back(g);
        for (int b = 0; b < (3 * n * nr + kPackedElemThreads - 1) / kPackedElemThreads; b++)
            mc[ic++] = make_int2(j, b);
    }
    const size_t used = (size_t)(w - pb->d_work);
    if (used > pb->work_cap) return pk_error(pb, kErrInvalid, "packed product: work space too small");
    // per-class slot tables: slot -> system, slot -> table index
    int *hs = sg->h_slots;
    std::vector<int> cls_n(pb->cls.size(), 0), cls_off(pb->cls.size(), 0);
    for (size_t c = 1; c < pb->cls.size(); c++) cls_off[c] = cls_off[c - 1] + (int)pb->cls[c - 1].sys.size();
    for (int j = 0; j < nact; j++) {
        const int g = act[j], c = pb->sys_cls[g];
        const int k = cls_n[c]++;
        hs[cls_off[c] + k] = g;
        hs[pb->nsys + cls_off[c] + k] = pb->sys_tab[g];
    }
    PK_CUDA(cudaMemcpyAsync(pb->d_io, sg->h_io, pb->nsys * sizeof(PackedIO), cudaMemcpyHostToDevice, s));
    PK_CUDA(cudaMemcpyAsync(pb->d_act, sg->h_act, nact * sizeof(int), cudaMemcpyHostToDevice, s));
    PK_CUDA(cudaMemcpyAsync(pb->d_map, sg->h_map, nmap * sizeof(int2), cudaMemcpyHostToDevice, s));
    for (size_t c = 0; c < pb->cls.size(); c++) {
        if (cls_n[c] == 0) continue;
        PK_CUDA(cudaMemcpyAsync(pb->cls[c].d_slot_sys, hs + cls_off[c], cls_n[c] * sizeof(int),
                                cudaMemcpyHostToDevice, s));
        PK_CUDA(cudaMemcpyAsync(pb->cls[c].d_slot_tab, hs + pb->nsys + cls_off[c], cls_n[c] * sizeof(int),
                                cudaMemcpyHostToDevice, s));
    }
    PK_CUDA(cudaEventRecord(sg->ev, s));
    sg->pending = true;
    pb->calls++;
    // the interpolation adds into vrecip: start from zero
    PK_CUDA(cudaMemsetAsync(pb->d_work, 0, used * sizeof(float), s));
    const int2 *dmg = pb->d_map, *dmp = dmg + nb_g, *dmc = dmp + nb_p;
    st = packed_gather(pb->d_sys, pb->d_io, pb->d_act, dmg, nb_g, nr, s);
    if (st == kOk) st = packed_pair_apply(pb->d_sys, pb->d_io, pb->d_act, dmp, nb_p, nr, s);
    for (int g : pl_missing) {
        if (st != kOk) break;
        st = real_space_walk_into4(pb->eng[g], nr, sg->h_io[g].fs_rs, sg->h_io[g].vreal, s);
    }
    for (size_t c = 0; c < pb->cls.size() && st == kOk; c++) {
        if (cls_n[c] == 0) continue;
        const PackedClass &pc = pb->cls[c];
        st = packed_x_spread(pc, pb->d_sys, pb->d_io, cls_n[c], nr, s);
        if (st == kOk) st = packed_y(pc, cls_n[c], nr, false, pb->d_err, s);
        if (st == kOk) st = packed_z(pc, cls_n[c], nr, pb->d_err, s);
        if (st == kOk) st = packed_y(pc, cls_n[c], nr, true, pb->d_err, s);
        if (st == kOk) st = packed_x_interp(pc, pb->d_sys, pb->d_io, cls_n[c], nr, pb->d_err, s);
    }
    if (st == kOk) st = packed_combine(pb->d_sys, pb->d_io, pb->d_act, dmc, nb_c, nr, alpha, beta, s);
    if (st != kOk) return pk_error(pb, st, std::string("packed product launch failed: ") +
                                               cudaGetErrorString(cudaGetLastError()));
    return kOk;
}

int packed_check_error(PackedBatch *pb)
{
    int h = 0;
    PK_CUDA(cudaMemcpyAsync(&h, pb->d_err, sizeof(int), cudaMemcpyDeviceToHost, pb->stream));
    PK_CUDA(cudaStreamSynchronize(pb->stream));
    if (h == 0) return kOk;
    PK_CUDA(cudaMemsetAsync(pb->d_err, 0, sizeof(int), pb->stream));
    return pk_error(pb, kErrCuda, "a packed grid pass timed out waiting for its tile copy (results invalid)");
}

void packed_free(PackedBatch *pb)
{
    if (!pb) return;
    cudaSetDevice(pb->device);
    if (pb->stream) cudaStreamSynchronize(pb->stream);
    for (PackedClass &c : pb->cls) {
        cudaFree(c.d_grid);
        cudaFree(c.d_tab);
        cudaFree(c.d_kmap);
        cudaFree(c.d_slot_sys);
        cudaFree(c.d_slot_tab);
    }
    pb->cls.clear();
    cudaFree(pb->d_sys);
    cudaFree(pb->d_io);
    cudaFree(pb->d_map);
    cudaFree(pb->d_act);
    for (PackedStaging &sg : pb->stg) {
        cudaFreeHost(sg.h_io);
        cudaFreeHost(sg.h_act);
        cudaFreeHost(sg.h_slots);
        cudaFreeHost(sg.h_map);
        if (sg.ev) cudaEventDestroy(sg.ev);
        sg = PackedStaging();
    }
    cudaFree(pb->d_work);
    cudaFree(pb->d_err);
    pb->d_sys = nullptr;
    pb->d_io = nullptr;
    pb->d_map = nullptr;
    pb->d_act = nullptr;
    pb->d_work = nullptr;
    pb->d_err = nullptr;
    pb->map_cap = pb->work_cap = 0;
}

}  // namespace sdt
