/*
 * stokesdt_b200.h -- C ABI of the B200 SPME/RPY mobility and block-Lanczos
 * Brownian path.  Plain C types only: opaque handles, pointers and sizes.
 *
 * Each entry point replaces a reference interface (paths relative to the
 * StokesDT project; the C++ adapters in stokesdt_b200_adapters.hpp put these
 * behind MobBase / BrwnBase / ForceBase):
 *
 *   sdt_spme_create        MobSpme::MobSpme + MobSpme::Init   src/mob/mob_spme.h:27-39,
 *                          src/mob/mob_spme.cc:19-132; engine CreateSpmeEngine
 *                          src/mob/spme.h:308-315
 *   sdt_spme_update        MobSpme::Update                    src/mob/mob_spme.cc:205-216
 *                          (UpdateSpmeEngine src/mob/spme.h:330-331)
 *   sdt_spme_mulvec        MobSpme::MulVector / RealMulVector / RecipMulVector
 *                          src/mob/mob_base.h:60-66, src/mob/mob_spme.cc:219-263
 *                          (ComputeSpmeRecip src/mob/spme.h:320-327)
 *   sdt_spme_dim           MobSpme::dim                        src/mob/mob_spme.h:94
 *   sdt_spme_destroy       MobSpme::~MobSpme / DestroySpmeEngine src/mob/mob_spme.cc:42-50
 *   sdt_lanczos_create     BrwnLanczos::BrwnLanczos + Init     src/brwn/brwn_lanczos.cc:204-275
 *   sdt_lanczos_compute    BrwnLanczos::Compute                src/brwn/brwn_lanczos.cc:278-304
 *                          (BrwnBase::Compute src/brwn/brwn_base.h:44-46)
 *   sdt_lanczos_destroy    BrwnLanczos::~BrwnLanczos           src/brwn/brwn_lanczos.cc:217-221
 *   sdt_bd_advance         BDSimBox::Advance step loop         src/simbox/simbox_bd.cc:296-366
 *   sdt_bd_create[_ewald]  BDSimBox::InitMob / InitBrwn        src/simbox/simbox_bd.cc:89-184
 *   sdt_ewald_create       MobEwald::MobEwald + MobEwald::Init src/mob/mob_ewald.cc:21-108
 *   sdt_ewald_update       MobEwald::Update (EwaldKernel)      src/mob/mob_ewald.cc:111-127,
 *                          src/mob/ewald.cc:86-330 (tables :643-797)
 *   sdt_ewald_mulvec       MobEwald::MulVector                 src/mob/mob_ewald.cc:131-152
 *   sdt_ewald_get_matrix   MobEwald::GetMatrix                 src/mob/mob_ewald.cc:155-165
 *   sdt_steric_create      StericForce::StericForce + Init     src/force/force_steric.cc:54-88
 *   sdt_steric_accumulate  StericForce::Accumulate (ForceBase)  src/force/force_steric.cc:91-104,
 *                          src/force/force_base.h:55-65 (PairListS src/pairlist/pair_s.cc:99-186)
 *
 * Conventions (as the reference):
 *   - positions and vectors are FP64, particle-major AoS: v[3*i + c];
 *   - a block of nrhs vectors is column-major: vector j starts at v + j*ld;
 *   - mulvec computes v := alpha * M * f + beta * v; beta == 0 ignores v;
 *   - mobility units: self mobility 1/a, i.e. 6*pi*eta = 1.
 * Differences from the reference, by design:
 *   - positions are wrapped into [0, L) before binning (the reference indexes
 *     out of bounds for positions outside the box, src/mob/spme.cc:404-417);
 *   - calls return a status (0 = OK, < 0 = sdt_status) instead of void, and
 *     sdt_spme_last_error() gives the message;
 *   - the grid dimension must be a power of two in [32, 512] and the spline
 *     order even and <= 8 (odd orders give non-finite output in the
 *     reference because b(k) divides by zero at the Nyquist frequency);
 *   - Lanczos honours any ldy >= 3N (the reference writes Y with its own
 *     internal leading dimension, src/brwn/brwn_lanczos.cc:184-186).
 * Threading: a handle is bound to one CUDA device and one stream; calls on one
 * handle must not overlap; different handles may run concurrently.
 */
#ifndef STOKESDT_B200_H_
#define STOKESDT_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef enum sdt_status {
    SDT_OK = 0,
    SDT_ERR_INVALID = -1,        /* bad argument (reference: Init() returns false) */
    SDT_ERR_CUDA = -2,           /* CUDA runtime error */
    SDT_ERR_ALLOC = -3,          /* device or host allocation failed */
    SDT_ERR_STATE = -4,          /* e.g. mulvec before update */
    SDT_ERR_NOT_CONVERGED = -5,  /* Lanczos hit max_iters (reference logs only) */
    SDT_ERR_UNSUPPORTED = -6     /* configuration outside the supported set */
} sdt_status;

typedef enum sdt_mulvec_mode {
    SDT_MOB_FULL = 0,   /* MobSpme::MulVector */
    SDT_MOB_REAL = 1,   /* MobSpme::RealMulVector (real space + self term) */
    SDT_MOB_RECIP = 2   /* MobSpme::RecipMulVector */
} sdt_mulvec_mode;

typedef struct sdt_spme sdt_spme;
typedef struct sdt_lanczos sdt_lanczos;

/* ---- SPME RPY mobility (MobSpme) ---- */

/* Creates and initialises an engine for npos particles with radii rdi (host,
 * copied).  All radii exactly 1.0 selects the monodisperse product, otherwise
 * the three-pass polydisperse one (src/mob/mob_spme.cc:104-118).  device is a
 * CUDA ordinal.  Validation as MobSpme::Init (src/mob/mob_spme.cc:55-93). */
int sdt_spme_create(int npos, const double *rdi, double box_size, double xi, double rmax,
                    int dim, int porder, int device, sdt_spme **out);

/* MobSpme::Update with host positions pos[3*npos] (rdi fixed at create). */
int sdt_spme_update(sdt_spme *h, const double *pos);

/* Same with a device pointer; asynchronous on the engine stream. */
int sdt_spme_update_device(sdt_spme *h, const double *d_pos);

/* v := alpha*M*f + beta*v for nrhs vectors, host pointers, synchronous.
 * mode is an sdt_mulvec_mode; ldf, ldv >= 3*npos. */
int sdt_spme_mulvec(sdt_spme *h, int mode, int nrhs, double alpha, int ldf, const double *f,
                    double beta, int ldv, double *v);

/* Same with device pointers; asynchronous on the engine stream. */
int sdt_spme_mulvec_device(sdt_spme *h, int mode, int nrhs, double alpha, int ldf,
                           const double *d_f, double beta, int ldv, double *d_v);

/* Real-space part of the mobility product (the same result as
 * sdt_spme_mulvec_device with SDT_MOB_REAL) for callers that are not allowed
 * to allocate device memory at this point, e.g. code running under a fixed
 * memory budget or inside a runtime that owns all allocations.  No
 * counterpart in the reference.  It allocates nothing: its FP32 work arrays
 * live in a fixed 6 MiB device array that every GPU loading the library holds
 * until exit, so npos * nrhs must not exceed 262144 (SDT_ERR_INVALID
 * otherwise).  Device pointers, asynchronous on the engine stream.  All calls
 * on a device share that array: calls that overlap on the GPU race.  The
 * first call on a device looks up the array's address (make it before any
 * stream capture), and so does the first call after cudaDeviceReset.  It
 * always walks the cell list, also on an engine that stores a pair list, so
 * it is slower than the allocating real-space product there.  In place
 * (d_f == d_v) is allowed with ldf == ldv. */
int sdt_spme_real_mulvec_noalloc(sdt_spme *h, int nrhs, double alpha, int ldf, const double *d_f,
                                 double beta, int ldv, double *d_v);

/* Dimension of the mobility matrix, 3*npos. */
int sdt_spme_dim(const sdt_spme *h);

/* Bind the engine to an existing cudaStream_t (NULL = the engine's own). */
int sdt_spme_set_stream(sdt_spme *h, void *stream);

/* Real-space pair list.  With enable != 0 (the default) every update stores
 * the real-space pairs of the new positions (24 bytes a pair: unit
 * separation, the two RPY scalars, the source index) and each product
 * streams them, as the reference stores its real-space BCSR matrix at
 * Update (MobSpme::Update, src/mob/mob_spme.cc:205-232).  With enable == 0,
 * or when the list does not fit in half the free device memory, each
 * product walks the cell list instead.  Takes effect at the next update. */
int sdt_spme_set_pairlist(sdt_spme *h, int enable);

/* Pairs held by the current pair list, or -1 when products walk the cells. */
int sdt_spme_pairlist_size(const sdt_spme *h, long long *pairs);

/* Block the host until all work queued on the engine stream has finished. */
int sdt_spme_synchronize(sdt_spme *h);

/* Message of the last failing call on this handle ("" if none). */
const char *sdt_spme_last_error(const sdt_spme *h);

void sdt_spme_destroy(sdt_spme *h);

/* ---- Dense Ewald RPY mobility (MobEwald) ---- */

typedef struct sdt_ewald sdt_ewald;

/* The 3N x 3N Ewald-summed RPY mobility matrix of npos particles with radii
 * rdi (copied) in a cube of edge box_size, FP64, held on the device (the
 * small-N counterpart of the SPME engine).  tol sets the real- and
 * reciprocal-space cut-offs by the reference's rules; xi <= 0 selects the
 * reference's default 10^(1/6) sqrt(pi) / L.  SDT_ERR_ALLOC when the matrix
 * (72 N^2 bytes) does not fit in half the free device memory. */
int sdt_ewald_create(int npos, const double *rdi, double box_size, double tol, double xi, int device,
                     sdt_ewald **out);
/* Builds the matrix at positions pos[3*npos] (host; synchronous) or d_pos
 * (device; asynchronous on the engine stream). */
int sdt_ewald_update(sdt_ewald *h, const double *pos);
int sdt_ewald_update_device(sdt_ewald *h, const double *d_pos);
/* v := alpha M f + beta v for nrhs vectors (beta == 0 ignores v); host
 * pointers (synchronous) or device pointers (asynchronous). */
int sdt_ewald_mulvec(sdt_ewald *h, int nrhs, double alpha, int ldf, const double *f, double beta, int ldv,
                     double *v);
int sdt_ewald_mulvec_device(sdt_ewald *h, int nrhs, double alpha, int ldf, const double *d_f, double beta,
                            int ldv, double *d_v);
/* Copies the matrix (row-major, leading dimension ldm >= 3 npos) to the host. */
int sdt_ewald_get_matrix(sdt_ewald *h, int ldm, double *mat);
/* xi, the cut-offs and the numbers of real-space images and reciprocal vectors
 * (any pointer may be NULL). */
int sdt_ewald_info(const sdt_ewald *h, double *xi, double *rmax, double *kmax, int *nimages, int *nkvectors);
int sdt_ewald_dim(const sdt_ewald *h);
int sdt_ewald_set_stream(sdt_ewald *h, void *stream);
const char *sdt_ewald_last_error(const sdt_ewald *h);
void sdt_ewald_destroy(sdt_ewald *h);

/* ---- Block Lanczos sqrt(M) z (BrwnLanczos) ---- */

/* dim = 3*npos; max_nrhs is clamped to dim/3 as in BrwnLanczos::Init
 * (src/brwn/brwn_lanczos.cc:245-249).  The Krylov recurrence, the optional
 * reorthogonalisation against all earlier blocks and the small eigenproblem
 * run in FP64. */
int sdt_lanczos_create(int dim, int max_iters, int max_nrhs, double tol, int device,
                       sdt_lanczos **out);

/* y[:, j] ~ sqrt(M) z[:, j] for nrhs vectors (host pointers), processed in
 * groups of max_nrhs like BrwnLanczos::Compute.  iters (optional, length
 * ceil(nrhs/max_nrhs)) receives the iteration count of each group, -1 if it
 * did not converge; the call then returns SDT_ERR_NOT_CONVERGED but y holds
 * the last iterate.  A group of one vector is BrwnLanczos::Lanczos
 * (src/brwn/brwn_lanczos.cc:16-82); its iterations run as one cooperative
 * launch each, and a grid-barrier wait in it that runs out (about a second)
 * makes the call return SDT_ERR_CUDA. */
int sdt_lanczos_compute(sdt_lanczos *h, sdt_spme *mob, int nrhs, int ldz, const double *z,
                        int ldy, double *y, int *iters);

/* Same with device pointers for z and y (synchronous return of iters). */
int sdt_lanczos_compute_device(sdt_lanczos *h, sdt_spme *mob, int nrhs, int ldz,
                               const double *d_z, int ldy, double *d_y, int *iters);

/* sdt_lanczos_compute / _device with the dense Ewald mobility
 * (BrwnLanczos::Compute on MobEwald, as tests/lanczos/testlanczos.cc of the
 * reference does). */
int sdt_lanczos_compute_ewald(sdt_lanczos *h, sdt_ewald *mob, int nrhs, int ldz, const double *z, int ldy,
                              double *y, int *iters);
int sdt_lanczos_compute_ewald_device(sdt_lanczos *h, sdt_ewald *mob, int nrhs, int ldz, const double *d_z,
                                     int ldy, double *d_y, int *iters);

/* Bind the solver to an existing cudaStream_t (NULL = its own).  The
 * mobility products it requests run on this stream too. */
int sdt_lanczos_set_stream(sdt_lanczos *h, void *stream);

/* 1 enables, 0 (default) disables reorthogonalisation of each new block
 * against all earlier ones.  The default follows the reference, which has
 * none, so iteration counts and iterates match BrwnLanczos; with it the basis
 * stays orthonormal and the convergence test runs on the small coefficient
 * matrix instead of on the 3N-long iterates. */
int sdt_lanczos_set_reorth(sdt_lanczos *h, int enable);

/* Convergence history of the last group of the last compute call:
 * out[i-1] = ||Y_i - Y_{i-1}||_F / ||Z||_F for iterations i = 1, 2, ...
 * (the reference only logs the final iteration count,
 * src/brwn/brwn_lanczos.cc:295-300).  Writes at most max_entries values and
 * returns the number of recorded iterations. */
int sdt_lanczos_history(const sdt_lanczos *h, double *out, int max_entries);

/* Block products M V_i issued by the last compute call, over all groups:
 * the iterations run plus any issued ahead of the convergence check and
 * discarded (the iterations are issued without waiting on the GPU). */
int sdt_lanczos_products(const sdt_lanczos *h, long long *out);

const char *sdt_lanczos_last_error(const sdt_lanczos *h);

void sdt_lanczos_destroy(sdt_lanczos *h);

/* ---- library and diagnostics (no counterpart in the reference; they play
 * the part of its rdtsc section timers, src/util/profile.h:17-72) ---- */

/* Version string of the library. */
/* ---- Batched independent systems ---- */

typedef struct sdt_batch sdt_batch;

/* nsys independent systems; system s has npos[s] particles (radii rdi,
 * concatenated), a cubic box of edge box[s], grid edge dim[s], Ewald xi[s]
 * and real-space cutoff rmax[s] (each checked as sdt_spme_create does), B-spline
 * order porder; one block-Lanczos workspace (max_iters, max_nrhs, tol,
 * reorthogonalisation when reorth != 0) per lane.  Systems are spread over
 * `lanes` concurrent CUDA streams.  The reference has no batched entry point:
 * each system follows MobSpme::Update / MulVector and BrwnLanczos::Compute.
 * Vectors of all systems are concatenated: system s owns nrhs blocks of
 * 3*npos[s] doubles at offset nrhs * 3 * (npos[0] + ... + npos[s-1]). */
int sdt_batch_create(int nsys, const int *npos, const double *rdi, const double *box, const int *dim,
                     const double *xi, const double *rmax, int porder, int max_iters, int max_nrhs,
                     double tol, int reorth, int lanes, int device, sdt_batch **out);

/* Device pointers (queued on the lanes; sdt_batch_synchronize waits). */
int sdt_batch_update_device(sdt_batch *h, const double *d_pos);
int sdt_batch_mulvec_device(sdt_batch *h, int nrhs, double alpha, const double *d_f, double beta,
                            double *d_v);
/* iters[s] (nsys entries) = iteration count of system s's first RHS group, -1
 * if it did not converge (then SDT_ERR_NOT_CONVERGED is returned). */
int sdt_batch_lanczos_device(sdt_batch *h, int nrhs, const double *d_z, double *d_y, int *iters);

/* Host pointers (staged; return when the results are on the host). */
int sdt_batch_update(sdt_batch *h, const double *pos);
int sdt_batch_mulvec(sdt_batch *h, int nrhs, double alpha, const double *f, double beta, double *v);
int sdt_batch_lanczos(sdt_batch *h, int nrhs, const double *z, double *y, int *iters);

/* Execution mode.  enable != 0 (the default when every system is
 * monodisperse with grid dimension <= 256, reorthogonalisation is on and
 * max_nrhs <= 16): every mobility product is one packed launch sequence over
 * all systems (systems of one grid dimension share each grid-pass launch) and
 * the block Lanczos iterates all systems in lockstep with batched Gram, GEMM
 * and Cholesky-QR launches; each system leaves when its check passes.
 * enable == 0: every system runs its own launches and the systems are spread
 * over the lanes.  No counterpart in the reference, which runs
 * src/mob/spme.cc:744-770 per system and per RHS.  SDT_ERR_UNSUPPORTED when
 * the systems do not allow the packed mode. */
int sdt_batch_set_packed(sdt_batch *h, int enable);
/* 1 when the packed mode is selected, 0 otherwise. */
int sdt_batch_get_packed(const sdt_batch *h);

/* Total 3*sum(npos) and the lane count. */
int sdt_batch_info(const sdt_batch *h, long long *total3n, int *lanes);
int sdt_batch_synchronize(sdt_batch *h);
const char *sdt_batch_last_error(const sdt_batch *h);
void sdt_batch_destroy(sdt_batch *h);

/* ---- Served request stream ---- */

typedef struct sdt_serve sdt_serve;

/* A server on `device` with `lanes` worker lanes (CUDA stream + host thread
 * + Lanczos workspace for up to max_npos particles and max_nrhs vectors, tol,
 * reorthogonalised) and an HBM budget (bytes) for the registered systems. */
int sdt_serve_create(int device, double hbm_budget_bytes, int lanes, int max_npos, int max_iters,
                     int max_nrhs, double tol, sdt_serve **out);

/* Register a system (as sdt_spme_create + sdt_spme_update): admitted only if
 * its estimated device memory fits the remaining budget (SDT_ERR_ALLOC
 * otherwise); its engine and pair list stay on the device. */
int sdt_serve_register(sdt_serve *h, int npos, const double *rdi, double box, int dim, double xi,
                       double rmax, int porder, const double *pos, int *sys_id);

/* Queue a request on a registered system: kind 0 = mobility apply
 * out = M in (MobSpme::MulVector), kind 1 = Brownian step out = sqrt(M) in
 * (BrwnLanczos::Compute); nrhs vectors of 3*npos doubles, host pointers that
 * must stay valid until sdt_serve_wait returns for the ticket.  Requests on
 * one system run in submission order; different systems run concurrently. */
int sdt_serve_submit(sdt_serve *h, int sys_id, int kind, int nrhs, const double *in, double *out,
                     long long *ticket);

/* Wait up to timeout_ms for a ticket: its status (SDT_ERR_STATE if still
 * pending) and its latency from submission to completion. */
int sdt_serve_wait(sdt_serve *h, long long ticket, double timeout_ms, double *latency_ms);

int sdt_serve_stats(sdt_serve *h, long long *completed, long long *rejected, double *used_bytes);

/* Continuous batching: requests on monodisperse systems with grid dimension
 * <= 256 and at most 16 RHS are served by two batch lanes.  A free lane takes
 * the oldest waiting request together with every other waiting request of the
 * same kind and RHS count on an idle system (up to 32) and runs them as one
 * packed product or one lockstep block Lanczos over their systems; requests
 * that arrive meanwhile join the next batch, and the two lanes' batches
 * overlap on the device.  A lane's workspace (grid slots and Krylov bases for
 * every such system) is charged to the HBM budget; a lane that does not fit
 * stays idle.  Set STOKESDT_SERVE_BATCH=0 at create to serve every request
 * alone.  Reports the batches run, the requests they held and the lanes in
 * use (any pointer may be NULL). */
int sdt_serve_batch_stats(sdt_serve *h, long long *batches, long long *batched_requests, int *lanes_active);
const char *sdt_serve_last_error(sdt_serve *h);
void sdt_serve_destroy(sdt_serve *h);

/* ---- Steric force (StericForce over PairListS) ---- */

typedef struct sdt_steric sdt_steric;

/* f_i += k0 (r0 (a_i + a_j)/2 - r_ij) (x_i - x_j)/r_ij over every j != i
 * with 2 r_ij / (a_i + a_j) < r0 (minimum image), FP64.  Fails (like
 * StericForce::Init) when k0 <= 0, and on npos <= 0, box_size <= 0, r0 <= 0
 * or a radius <= 0.  rdi is copied. */
int sdt_steric_create(int npos, const double *rdi, double box_size, double r0, double k0, int device,
                      sdt_steric **out);

/* f[3*npos] += steric force at pos[3*npos]; host pointers (ForceBase::Accumulate). */
int sdt_steric_accumulate(sdt_steric *h, const double *pos, double *f);

/* The same with device pointers, queued on the handle's stream. */
int sdt_steric_accumulate_device(sdt_steric *h, const double *d_pos, double *d_f);

/* Bind to an existing cudaStream_t (NULL = the handle's own). */
int sdt_steric_set_stream(sdt_steric *h, void *stream);

const char *sdt_steric_last_error(const sdt_steric *h);

void sdt_steric_destroy(sdt_steric *h);

/* ---- Device-resident BD integrator (BDSimBox::Advance) ---- */

typedef struct sdt_bd sdt_bd;

/* The step loop of BDSimBox::Advance with positions, forces, random and
 * displacement vectors on the device of `mob`:
 *   every mob_interval steps: Z ~ N(0,1) [mob_interval x 3N] drawn on the
 *   device (Philox4x32-10, key = seed, counter = (pair index, step);
 *   Box-Muller), mob Update, Y = sqrt(M) Z with `brwn`;
 *   every step: f = steric(pos) (or 0 when steric is NULL),
 *   Y[irhs] = dt M f + sqrt(2 dt) Y[irhs], pos += Y[irhs].
 * The handles must stay alive and must not be used elsewhere while the
 * integrator advances.  Non-convergence of a Lanczos call is counted (the
 * reference only logs it) and the step goes on with the last iterate. */
int sdt_bd_create(sdt_spme *mob, sdt_lanczos *brwn, sdt_steric *steric, double dt, int mob_interval,
                  unsigned long long seed, sdt_bd **out);

/* The same loop with the dense Ewald matrix as the mobility (MobEwald, the
 * reference driver's default mob-method, src/simbox/simbox_bd.cc:93-103):
 * Update rebuilds the matrix from the positions every mob_interval steps. */
int sdt_bd_create_ewald(sdt_ewald *mob, sdt_lanczos *brwn, sdt_steric *steric, double dt, int mob_interval,
                        unsigned long long seed, sdt_bd **out);

/* Positions (3*npos, host); set resets nothing else. */
int sdt_bd_set_positions(sdt_bd *h, const double *pos);
int sdt_bd_get_positions(sdt_bd *h, double *pos);

/* Step counter (BDSimBox start_step); a new interval starts when
 * istep % mob_interval == 0. */
int sdt_bd_set_step(sdt_bd *h, long long istep);

/* Advance nsteps steps (queued; sdt_bd_get_positions or sdt_bd_synchronize waits). */
int sdt_bd_advance(sdt_bd *h, int nsteps);

/* istep, Lanczos calls that missed tol, and the iteration count of the first
 * RHS group of the last Lanczos call (any pointer may be NULL). */
int sdt_bd_info(sdt_bd *h, long long *istep, long long *not_converged, int *last_iters);

/* The random vectors the integrator draws at the interval starting at
 * `step`: z[v*ld + e], v < nvec, e < 3*npos (host pointer). */
int sdt_bd_draw_gaussian(sdt_bd *h, long long step, int nvec, int ld, double *z);

/* Bind to an existing cudaStream_t (NULL = the integrator's own). */
int sdt_bd_set_stream(sdt_bd *h, void *stream);

int sdt_bd_synchronize(sdt_bd *h);
const char *sdt_bd_last_error(const sdt_bd *h);
void sdt_bd_destroy(sdt_bd *h);

/* ---- File I/O in the reference's formats (MoleculeIO, src/util/molecule_io.cc) ---- */

/* Particle count on the first line of an XYZ file.  0 on success. */
int sdt_xyz_count(const char *path, int *npos);

/* XYZ file -> pos[3*npos], rdi[npos] (radii by particle type from the
 * model file's "par" lines, 1.0 for unknown types or model == NULL),
 * box[3] = Lx Ly Lz, start step and time (MoleculeIO::ParseXYZ,
 * molecule_io.cc:141-237).  0 on success, -1 on a malformed file. */
int sdt_xyz_read(const char *path, const char *model, int npos, double *pos, double *rdi, double *box,
                 int *start_step, double *start_time);

/* One trajectory frame in MoleculeIO::WriteXYZ's layout (molecule_io.cc:384-402);
 * append != 0 appends. */
int sdt_xyz_write(const char *path, int append, int npos, const double *box, int frame, double time,
                  const double *pos);

/* Config-file value of `key` ("key value" lines, '#' comments;
 * MoleculeIO::ParseConfig, molecule_io.cc:39-88): 0 found, 1 absent, -1 error. */
int sdt_config_get(const char *path, const char *key, char *buf, int buflen);

/* "steric <r0> <k0>" line of a model file: 0 found, 1 absent, -1 error. */
int sdt_model_steric(const char *path, double *r0, double *k0);

const char *sdt_version(void);

/* Runs `reps` mobility products of nrhs (1..16) vectors on the engine's
 * current positions with a CUDA event after every stage and writes the mean
 * milliseconds of each stage to stage_ms[0..n).  Returns n (the number of
 * stages, <= max_stages) or a negative sdt_status. */
int sdt_spme_profile_mulvec(sdt_spme *h, int nrhs, int reps, double *stage_ms, int max_stages);

/* Forward transform of the spread forces, for checking the hand-written FFT
 * against an independent one: for nrhs (1..16) force vectors (device
 * pointer, leading dimension ldf >= 3*npos) writes the half spectra
 * spec[r][c][kz][ky][kx], kx = 0..K/2, of the spread grids (the grid the
 * reference spreads in src/mob/spme.cc:313-363 and transforms with its
 * forward DFTI call, src/mob/spme.cc:754-756) as interleaved FP32 (re, im)
 * pairs: nrhs * 3 * K * K * (K/2 + 1) * 2 floats.  Monodisperse engines, grid
 * dimension <= 256.  Asynchronous on the engine stream. */
int sdt_spme_spectrum_device(sdt_spme *h, int nrhs, int ldf, const double *d_f, float *d_spec);

/* Name of profile stage i ("" when out of range). */
const char *sdt_profile_stage_name(int stage);

/* Number of CUDA kernels this library has launched since it was loaded. */
unsigned long long sdt_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* STOKESDT_B200_H_ */
