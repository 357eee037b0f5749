// Internal state of one SPME RPY mobility engine on one GPU.
//
// Host code owns this struct; every pointer named d_* is device memory on
// `device`.  All kernels of the engine run on `stream`.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <string>

namespace sdt {

// Status codes shared with the C ABI (include/stokesdt_b200.h).
enum Status {
    kOk = 0,
    kErrInvalid = -1,
    kErrCuda = -2,
    kErrAlloc = -3,
    kErrState = -4,
    kErrNotConverged = -5,
    kErrUnsupported = -6,
};

// Number of kernels this library has launched since it was loaded.
extern std::atomic<unsigned long long> g_kernel_launches;

// Stages of one mobility product, in launch order (per-stage event timing).
enum Stage {
    kStGather = 0,
    kStReal,
    kStSpreadX,
    kStYFwd,
    kStZInfl,
    kStYInv,
    kStXInterp,
    kStCombine,
    kNumStages
};

constexpr int kRowBlock = 8;   // y/z extent of the bins of the spread-order sort
constexpr int kRowBlockY = 4;  // y extent of the row blocks of the x passes
constexpr int kRowBlockZ = 4;  // z extent of the row blocks of the x passes
constexpr int kMaxOrder = 8;   // largest supported B-spline order
constexpr int kTileX = 16;     // kx columns per CTA in the y pass
constexpr int kTileZ = 8;      // kx columns per CTA in the staged z pass (x 3 components)
// kx columns per CTA in the register-fused z pass: 4 at K = 256 (a 29 KB
// CTA), 8 below, so smaller grids keep the same bytes in flight per CTA
__host__ __device__ constexpr int z_fused_tile(int K) { return K <= 128 ? 8 : 4; }

struct SpmeEngine {
    // configuration
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int npos = 0;
    double box = 0.0, xi = 0.0, rmax = 0.0;
    int K = 0, p = 0;
    bool mono = true;
    int XS = 0;        // complex row length (K/2 + 1 rounded up to 4)
    int nbin = 0;      // K / kRowBlock bins per axis (spread-order sort)
    int nby = 0, nbz = 0;  // row blocks of the x passes per y / z axis
    int ncnt_sp = 0;   // counters of the spread-order sort and the segment blocks
    double self_mono = 0.0;

    // tables
    float *d_tab0 = nullptr;     // influence: lm2*(1-k^2/3) (mono) or lm2 (poly), [K][K][XS]
    float *d_tab2 = nullptr;     // poly only: lm2*(-k^2/6)
    float *d_kmap = nullptr;     // signed wave numbers 2*pi*m/L, [K]
    float2 *d_tw_half = nullptr; // W_{K/2}^m
    float2 *d_tw_full = nullptr; // W_K^m
    double *d_rdi = nullptr;     // radii [N]
    double *d_rdi2 = nullptr;    // squared radii [N] (polydisperse passes)
    double *d_self = nullptr;    // self mobility per particle [N]

    // particles in spread-bin order
    int *d_sp_perm = nullptr;      // sorted slot -> particle
    int *d_sp_base = nullptr;      // packed base grid index x | y<<10 | z<<20
    float *d_sp_w = nullptr;       // [N][3][kMaxOrder] spline weights
    int *d_sp_binstart = nullptr;  // [nbin*nbin + 1]
    // row segments of the x kernels, grouped by kRowBlockZ x kRowBlockY row block
    int *d_seg_start = nullptr;    // [nbz*nby + 1]
    unsigned *d_seg_meta = nullptr;  // row-in-block | x0 << 6
    int *d_seg_slot = nullptr;     // spread-order slot of the particle
    float *d_seg_w = nullptr;      // wz[jz] * wy[jy]
    // particles in real-space cell order
    int nc = 0;                    // cells per axis
    double cs = 0.0;               // cell edge
    int nstencil = 0;
    int *d_stencil = nullptr;      // stencil columns, packed (dx+8) | (dy+8)<<5
    int *d_rs_perm = nullptr;      // sorted slot -> particle
    int *d_rs_inv = nullptr;       // particle -> sorted slot
    int *d_rs_cell = nullptr;      // cell of each sorted slot
    double4 *d_rs_pos = nullptr;   // wrapped position + radius, sorted
    float4 *d_rs_posf = nullptr;   // the same in FP32 (candidate tests only)
    int *d_rs_cellstart = nullptr; // [nc^3 + 1]
    // real-space pair list (cell order), rebuilt at every update
    bool pl_enabled = true;        // build it at update (else walk cells per product)
    bool pl_ready = false;         // built for the current positions
    long long pl_cap = 0;          // pairs the arrays hold
    long long pl_pairs = 0;        // pairs stored
    int *d_pl_count = nullptr;     // [N] pairs per target
    long long *d_pl_start = nullptr;  // [N + 1] row starts
    float4 *d_pl_e = nullptr;      // (ex, ey, ez, ya) per pair
    float2 *d_pl_c = nullptr;      // (xa - ya, source slot as int bits) per pair

    // update scratch
    int *d_counts = nullptr;       // histogram / cursor scratch
    int *d_key_sp = nullptr, *d_key_rs = nullptr;
    int *d_tmp_base = nullptr;
    float *d_tmp_w = nullptr;
    double4 *d_tmp_pos = nullptr;

    // per-call work space (grown on demand)
    int rhs_cap = 0;               // RHS per chunk the buffers hold
    float2 *d_cgrid = nullptr;     // [rhs][3][K][K][XS] (poly: two sets)
    float *d_fs_sp = nullptr;      // [rhs][3][N] forces, spread order, FP32
    float *d_fs_rs = nullptr;      // [N][rhs][4] forces, cell order, FP32 (4th zero)
    float *d_vrecip = nullptr;     // [rhs][3N]
    float *d_vreal = nullptr;      // [rhs][3N]
    int host_cap = 0;              // RHS the host staging buffers hold
    double *d_fin = nullptr;       // host-API staging for f
    double *d_vout = nullptr;      // host-API staging for v
    int rhs_chunk_max = 16;
    // TMA staging of the y/z passes (tensor maps over d_cgrid at rhs_cap)
    bool tma_enabled = true;       // cleared by STOKESDT_NO_TMA=1 at create
    bool tma_ready = false;
    CUtensorMap tmap_y;            // [3*rhs*K planes][K y][XS x]
    CUtensorMap tmap_z;            // [3*rhs][K z][K y][XS x]
    CUtensorMap tmap_tab0;         // influence tables [K z][K y][XS x] (float)
    CUtensorMap tmap_tab2;
    CUtensorMap tmap_zf;           // the z map with z_fused_tile(K)-wide boxes (fused z pass)
    CUtensorMap tmap_tab0f, tmap_tab2f;  // table maps with z_fused_tile(K)-wide boxes
    bool tma_tabs = false;         // table maps encoded
    int *d_err = nullptr;          // device error word of the TMA passes (0 = fine)
    // overlapped product: real space and RHS groups of the grid chain on side
    // streams, joined before the combine (set by STOKESDT_OVERLAP=1; off by
    // default: at N = 1e5, K = 256, 16 RHS each kernel already fills the GPU
    // and the split product measured 2% slower)
    bool overlap = false;
    // z pass with forward FFT, influence and inverse FFT fused in registers
    // (K <= 256, TMA path; cleared by STOKESDT_NO_ZFUSE=1)
    bool zfused = true;
    // tensor-core spread (K = 256, calls of >= kTcMinRhs RHS; cleared by
    // STOKESDT_NO_TC=1, and for batch and served engines): per 2x2 row block
    // the particles whose support reaches it (padded to whole 16-particle
    // chunks), their 4 row weights wz*wy and their x-transformed weight
    // rows as TF32 hi/lo MMA operand tiles, rebuilt at every update
    bool tc_enabled = true;
    bool tc_ready = false;
    long long tc_cap = 0;          // entries the arrays hold
    int *d_tc_cnt = nullptr;       // [nblk] counts, then cursors
    int *d_tc_start = nullptr;     // [nblk + 1] entry starts (multiples of 16)
    int *d_tc_slot = nullptr;      // [entries] spread-order slot, -1 for padding
    float *d_tc_w = nullptr;       // [entries][4] row weights
    float *d_tc_bx = nullptr;      // [chunks][2][K][16] operand tiles
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[3] = {nullptr, nullptr, nullptr};

    bool updated = false;
    std::string last_error;

    // per-stage timing: when prof_on, an event is recorded after each stage
    bool prof_on = false;
    cudaEvent_t prof_ev[kNumStages + 1] = {};
    float prof_ms[kNumStages] = {};
};

// Record the end of `stage` when profiling (the start is the previous mark).
void prof_mark(SpmeEngine *e, int stage);

// spme.cu
int spme_create(SpmeEngine *e);
// Radii (npos, all > 0): self terms, a and a^2 on the device; after spme_create.
int spme_set_radii(SpmeEngine *e, const double *rdi);
int spme_update(SpmeEngine *e, const double *d_pos);
// mode: 0 full, 1 real only, 2 reciprocal only.  f, v are device pointers.
int spme_mulvec(SpmeEngine *e, int mode, int nrhs, double alpha, int ldf, const double *d_f,
                double beta, int ldv, double *d_v);
void spme_free(SpmeEngine *e);
int spme_reserve(SpmeEngine *e, int rhs);
int spme_profile(SpmeEngine *e, int nrhs, int reps, double *stage_ms);
// Forward transform of the spread forces (diagnostic; see spme.cu).
int spme_spectrum(SpmeEngine *e, int nrhs, int ldf, const double *d_f, float *d_spec);

// real_space.cu: adds the matrix-free real-space sum (without the self term)
// of `rb` RHS to d_vreal ([rb][3N], zeroed by the caller).
int real_space_launch(SpmeEngine *e, int rb);
// Same with caller-supplied buffers: fs [N][nr][3] (cell order), vreal [nr][3N].
int real_space_launch_into(SpmeEngine *e, int nr, const float *fs, float *vreal);
// Cell walk with float4 force rows fs [N][nr] (cell order) on stream s.
int real_space_walk_into4(SpmeEngine *e, int nr, const float4 *fs, float *vreal, cudaStream_t s);
// Build / release the real-space pair list (used by real_space_launch when
// pl_ready).
int pair_list_build(SpmeEngine *e);
void pair_list_free(SpmeEngine *e);

int set_error(SpmeEngine *e, int status, const std::string &msg);
// Fewest right-hand sides of a call that takes the tensor-core spread; calls
// with fewer use the shared-memory spread.
constexpr int kTcMinRhs = 8;
int tc_build(SpmeEngine *e);
void tc_free(SpmeEngine *e);
int spread_tc_launch(SpmeEngine *e, int nr, int r0, cudaStream_t s);

// Status returns inside functions that hold an engine `e`.
#define SDT_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t err_ = (call);                                                        \
        if (err_ != cudaSuccess)                                                          \
            return set_error(e, kErrCuda, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

#define SDT_LAUNCH_CHECK()                                                                \
    do {                                                                                  \
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                        \
        cudaError_t err_ = cudaGetLastError();                                            \
        if (err_ != cudaSuccess)                                                          \
            return set_error(e, kErrCuda, std::string("kernel launch: ") + cudaGetErrorString(err_)); \
    } while (0)

// Read the device error word (synchronises the engine stream); kErrCuda with
// a message if a pass gave up waiting for its tile.
int spme_check_device_error(SpmeEngine *e);

// tma.cu: tiled tensor maps of float2 / float elements (see tma.cuh)
bool encode_tmap_f2(CUtensorMap *map, const void *base, int rank, const unsigned long long *dims,
                    const unsigned long long *strides, const unsigned *box);
bool encode_tmap(CUtensorMap *map, const void *base, int elem_bytes, int rank,
                 const unsigned long long *dims, const unsigned long long *strides, const unsigned *box);

}  // namespace sdt
