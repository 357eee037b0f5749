// Packed multi-system execution: the mobility products and the block Lanczos
// of many independent suspensions run as a few launches over all of them.
//
// The reference has no batched path: each system's work is the serial
// per-system, per-RHS sequence of src/mob/spme.cc:744-770 (spread, three
// forward FFTs, influence, three backward FFTs, interpolation) inside
// MobSpme::MulVector (src/mob/mob_spme.cc:219-236), driven by
// BrwnLanczos::Compute (src/brwn/brwn_lanczos.cc:278-304).  Here every system
// keeps its own SPME engine (grid, Ewald split, pair list, tables), and:
//   - systems with the same grid edge K form a class; per call the class's
//     active systems take consecutive slots of one scratch grid, so the y and
//     z transforms are one TMA launch over all of them and the x kernels
//     (spread + x FFT, inverse x FFT + interpolation) one launch each, a CTA
//     finding its system through a slot table;
//   - force gather, real-space pair-list apply and the final combine are one
//     launch each over all systems, a CTA finding its system through a
//     per-CTA (slot, block) map;
//   - the block Lanczos iterations of all systems run in lockstep: one packed
//     product, then batched Gram, GEMM and Cholesky-QR kernels over all
//     systems, one coefficient copy to the host per iteration; systems leave
//     the active set when their check passes (packed_lanczos.h).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "engine.h"

namespace sdt {

// One system, device copy (static between updates).
struct PackedSys {
    int n = 0, p = 0, nby = 0, tab = 0;   // tab: index of the system within its K class
    double invL3 = 0.0;                   // 1 / L^3
    const int *seg_start = nullptr;
    const unsigned *seg_meta = nullptr;
    const int *seg_slot = nullptr;
    const float *seg_w = nullptr;
    const float *sp_w = nullptr;
    const int *sp_perm = nullptr;
    const int *rs_inv = nullptr;
    const int *rs_perm = nullptr;
    const double *self = nullptr;
    const long long *pl_start = nullptr;
    const float4 *pl_e = nullptr;
    const float2 *pl_c = nullptr;
};

// One system of one packed call (device copy, rebuilt per call): vectors and
// the FP32 work slices.
struct PackedIO {
    const double *f = nullptr;
    double *v = nullptr;
    int ldf = 0, ldv = 0;
    float *fs_sp = nullptr;   // [nr][3][n], spread order
    float4 *fs_rs = nullptr;  // [n][nr], cell order
    float *vrecip = nullptr;  // [nr][3n]
    float *vreal = nullptr;   // [nr][3n]
};

// Systems with one grid edge K.
struct PackedClass {
    int K = 0, XS = 0, nby = 0, nbz = 0;
    std::vector<int> sys;          // global ids of the class's systems (tab order)
    float2 *d_grid = nullptr;      // [slots][rhs][3][K][K][XS]
    float *d_tab = nullptr;        // [tab][K][K][XS] influence tables
    float *d_kmap = nullptr;       // [tab][K] wave numbers
    const float2 *tw_half = nullptr, *tw_full = nullptr;  // K-dependent twiddles (first engine's)
    CUtensorMap tmap_y, tmap_zf, tmap_tabf;
    // per call: slot -> global system id and slot -> table index
    int *d_slot_sys = nullptr, *d_slot_tab = nullptr;
};

// Pinned host staging of one packed call's descriptors.  Calls cycle
// through kPackedRing sets; a set is rewritten only after the event recorded
// behind its copies has completed, so the host can queue calls ahead.
constexpr int kPackedRing = 4;
struct PackedStaging {
    PackedIO *h_io = nullptr;      // [nsys]
    int *h_act = nullptr;          // [nsys] slot -> global system id
    int *h_slots = nullptr;        // [2 nsys] per-class slot -> system, slot -> table
    int2 *h_map = nullptr;         // per-CTA (slot, block) maps
    size_t map_cap = 0;
    cudaEvent_t ev = nullptr;
    bool pending = false;
};

struct PackedBatch {
    int device = 0;
    cudaStream_t stream = nullptr;
    int nsys = 0, rhs_cap = 0;
    std::vector<SpmeEngine *> eng;     // not owned
    std::vector<PackedClass> cls;
    std::vector<int> sys_cls;          // class of each system
    std::vector<int> sys_tab;          // index of each system within its class
    PackedSys *d_sys = nullptr;        // [nsys]
    PackedIO *d_io = nullptr;          // [nsys]
    int2 *d_map = nullptr;             // per-CTA (slot, block) maps
    size_t map_cap = 0;
    int *d_act = nullptr;              // [nsys]
    PackedStaging stg[kPackedRing];
    int stg_next = 0;
    float *d_work = nullptr;           // FP32 work space
    size_t work_cap = 0;               // floats
    int *d_err = nullptr;
    long long calls = 0;
    std::string last_error;
};

// Set up for `eng` (monodisperse engines, created; K a power of two in
// [32, 256]) with up to rhs_cap RHS per call.  The engines' streams are not
// used by packed calls.
int packed_create(PackedBatch *pb, const std::vector<SpmeEngine *> &eng, int rhs_cap, int device,
                  cudaStream_t stream);
// Refresh the device descriptors after the engines' updates.
int packed_refresh(PackedBatch *pb);
// v_s := alpha M_s f_s + beta v_s for the systems act[0..nact) (global ids),
// nr <= rhs_cap RHS each; f[j], v[j] device pointers with leading
// dimensions ldf[j], ldv[j] (j = slot).
int packed_mulvec(PackedBatch *pb, int nact, const int *act, int nr, double alpha, const double *const *f,
                  const int *ldf, double beta, double *const *v, const int *ldv);
// Reads and clears the device error word of the grid passes (synchronises).
int packed_check_error(PackedBatch *pb);
void packed_free(PackedBatch *pb);

// Launch helpers defined next to the single-system kernels.
int packed_x_spread(const PackedClass &c, const PackedSys *d_sys, const PackedIO *d_io, int nslots, int nr,
                    cudaStream_t s);
int packed_y(const PackedClass &c, int nslots, int nr, bool inverse, int *err, cudaStream_t s);
int packed_z(const PackedClass &c, int nslots, int nr, int *err, cudaStream_t s);
int packed_x_interp(const PackedClass &c, const PackedSys *d_sys, const PackedIO *d_io, int nslots, int nr,
                    int *err, cudaStream_t s);
int packed_gather(const PackedSys *d_sys, const PackedIO *d_io, const int *d_act, const int2 *d_map, int nblocks,
                  int nr, cudaStream_t s);
int packed_combine(const PackedSys *d_sys, const PackedIO *d_io, const int *d_act, const int2 *d_map,
                   int nblocks, int nr, double alpha, double beta, cudaStream_t s);
int packed_pair_apply(const PackedSys *d_sys, const PackedIO *d_io, const int *d_act, const int2 *d_map,
                      int nblocks, int nr, cudaStream_t s);
// Threads per CTA of the gather / combine kernels and targets per CTA of the
// pair-list apply (the CTA maps are built with these).
constexpr int kPackedElemThreads = 256;
int packed_pair_targets_per_cta();

}  // namespace sdt
