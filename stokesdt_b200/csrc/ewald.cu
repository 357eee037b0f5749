// Dense Ewald-summed RPY mobility matrix on one GPU, FP64 (MobEwald /
// EwaldKernel of the reference: src/mob/mob_ewald.cc:21-165,
// src/mob/ewald.cc:86-330, tables :643-797).
//
// Block (i, j) of the 3N x 3N matrix is
//   real:  sum over lattice images d = d0 + L m with 0 < |d| <= rmax of
//          (xa - ya) e e^T + ya I, (xa, ya) the real-space RPY Ewald scalars
//          (plus the overlap correction when |d| < a_i + a_j), d0 the minimum
//          image of r_j - r_i, and the self term on the diagonal;
//   recip: sum over k != 0, |k| <= kmax of cos(k . d0) (6 - k^2 (a_i^2 +
//          a_j^2)) kexp(k) (I - k k^T / k^2).
// The reference evaluates cos(k . d0) per pair and k.  Here the reciprocal sum
// uses cos(k . d) = cos(k . r_i) cos(k . r_j) + sin(k . r_i) sin(k . r_j) with
// the per-particle factors computed once per update, so the pair sum is a
// contraction over k of products staged in shared memory (the same terms,
// rounded differently: agreement with the reference to ~1e-14 relative).
// Products v := alpha M f + beta v read the stored matrix once (one warp per
// row, every RHS of the call at once), as MobEwald::MulVector's dsymv/dsymm
// (src/mob/mob_ewald.cc:131-152).
#include <algorithm>
#include <cmath>
#include <vector>

#include "ewald.h"

namespace sdt {

namespace {

constexpr int kEwTile = 16;    // particles per tile side of the matrix kernel
constexpr int kEwKChunk = 32;  // reciprocal vectors staged at a time
constexpr int kEwMaxImg = 512;   // image shifts held in shared memory (the rest are read from global)

// EwaldReal and EwaldRecip (src/mob/ewald.cc:19-40): tail estimates that set
// the cut-offs.
double real_tail(double r, double xi)
{
    const double xir = xi * r, xir2 = xir * xir, r2 = r * r;
    return std::erfc(xir) * (0.75 + 1.5 / r2) / r +
           std::exp(-xir2) * xi / std::sqrt(M_PI) *
               (4.5 + 3.0 * xir2 + (3.0 + xir2 * (14.0 + xir2 * (4.0 + xir2))) / r2);
}

double recip_tail(double k, double xi)
{
    const double kx = k / xi, kx2 = kx * kx, k2 = k * k;
    return 6.0 * M_PI * std::exp(-kx2 / 4.0) * (1.0 + k2 / 3.0) / k2 * (1.0 + kx2 * (0.25 + kx2 / 8.0));
}

// The cut-off rules of XitoRmax / XitoKmax (src/mob/ewald.cc:43-83): shrink
// by 1 % while the tail (with a safety factor on xi) stays below tol.
double cutoff_rmax(double xi, double tol, double box)
{
    const double xi0 = xi / 1.15;
    double rmax = 10.0 * std::sqrt(-std::log(tol)) / xi;
    while (real_tail(rmax * 0.99, xi0) + 6.0 * real_tail(rmax * 0.99 + box, xi0) < tol) rmax *= 0.99;
    return rmax;
}

double cutoff_kmax(double xi, double tol, double box)
{
    const double xi0 = xi * 1.15, dk = 2.0 * M_PI / box;
    double kmax = 10.0 * std::sqrt(-std::log(tol)) * 2.0 * xi;
    while (recip_tail(kmax * 0.99, xi0) + 6.0 * recip_tail(kmax * 0.99 + dk, xi0) < tol) kmax *= 0.99;
    return kmax;
}

// cs[k][i] = cos(k . r_i), cs[nk + k][i] = sin(k . r_i).
__global__ void k_ew_factors(int n, int nk, const double *__restrict__ kv, const double *__restrict__ pos,
                             double *__restrict__ cs)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * nk) return;
    const int k = (int)(t / n), i = (int)(t % n);
    const double a = kv[4 * k] * pos[3 * i] + kv[4 * k + 1] * pos[3 * i + 1] + kv[4 * k + 2] * pos[3 * i + 2];
    double s, c;
    sincos(a, &s, &c);
    cs[(size_t)k * n + i] = c;
    cs[(size_t)(nk + k) * n + i] = s;
}

// Real-space RPY Ewald scalars xa, ya at separation r (scalars_ewald_F,
// src/mob/ewald.h:55-85), FP64.
__device__ __forceinline__ void rpy_real_scalars(double xi, double r, double a2sum, double &xa, double &ya)
{
    const double xir = xi * r, xir2 = xir * xir, r2 = r * r, r3 = r2 * r;
    const double ec = erfc(xir);
    const double ex = xi / sqrt(M_PI) * exp(-xir2);
    const double a0 = 2.0 * (-3.0 + 2.0 * xir2) * ex + ec / r;
    const double b0 = 2.0 * (1.0 - 2.0 * xir2) * ex + ec / r;
    const double a2 = 4.0 / r2 * (1.0 + xir2 * (14.0 + xir2 * (-20.0 + 4.0 * xir2))) * ex + 2.0 / r3 * ec;
    const double b2 = -4.0 / r2 * (3.0 + xir2 * (2.0 + xir2 * (-16.0 + 4.0 * xir2))) * ex - 6.0 / r3 * ec;
    ya = 0.75 * (a0 + a2 * a2sum / 6.0);
    xa = 0.75 * (b0 + b2 * a2sum / 6.0) + ya;
}

// One 3x3 block per (i <= j) pair of a kEwTile x kEwTile tile, written to
// both (i, j) and (j, i).  kw[k] = (P00, P01, P02, P11, P12, P22, 6 kexp,
// k^2 kexp) with P = I - k k^T / k^2.
__global__ void __launch_bounds__(kEwTile *kEwTile)
k_ew_matrix(int n, int nk, int nr, double box, double xi, double rmax2, const double *__restrict__ pos,
            const double *__restrict__ rdi, const double *__restrict__ img, const double *__restrict__ kw,
            const double *__restrict__ cs, double *__restrict__ mat, int ldm)
{
    __shared__ double sci[kEwKChunk][kEwTile], ssi[kEwKChunk][kEwTile];
    __shared__ double scj[kEwKChunk][kEwTile], ssj[kEwKChunk][kEwTile];
    __shared__ double skw[kEwKChunk][8];
    __shared__ double simg[kEwMaxImg * 3];
    const int i0 = blockIdx.y * kEwTile, j0 = blockIdx.x * kEwTile;
    if (i0 > j0) return;  // lower tiles are written by their transposes
    const int ti = threadIdx.x / kEwTile, tj = threadIdx.x % kEwTile;
    const int i = i0 + ti, j = j0 + tj;
    const bool live = i < n && j < n && i <= j;
    const double ai = i < n ? rdi[i] : 1.0, aj = j < n ? rdi[j] : 1.0;
    const double a2sum = ai * ai + aj * aj;
    double m[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // 00 01 02 11 12 22
    // reciprocal part
    for (int k0 = 0; k0 < nk; k0 += kEwKChunk) {
        __syncthreads();
        for (int t = threadIdx.x; t < kEwKChunk * kEwTile; t += blockDim.x) {
            const int kk = t / kEwTile, q = t % kEwTile;
            const int k = k0 + kk;
            const bool okk = k < nk;
            sci[kk][q] = (okk && i0 + q < n) ? cs[(size_t)k * n + i0 + q] : 0.0;
            ssi[kk][q] = (okk && i0 + q < n) ? cs[(size_t)(nk + k) * n + i0 + q] : 0.0;
            scj[kk][q] = (okk && j0 + q < n) ? cs[(size_t)k * n + j0 + q] : 0.0;
            ssj[kk][q] = (okk && j0 + q < n) ? cs[(size_t)(nk + k) * n + j0 + q] : 0.0;
        }
        for (int t = threadIdx.x; t < kEwKChunk * 8; t += blockDim.x) {
            const int k = k0 + t / 8;
            skw[t / 8][t % 8] = k < nk ? kw[(size_t)k0 * 8 + t] : 0.0;
        }
        __syncthreads();
        const int kn = min(kEwKChunk, nk - k0);
        for (int kk = 0; kk < kn; kk++) {
            const double c = sci[kk][ti] * scj[kk][tj] + ssi[kk][ti] * ssj[kk][tj];
            const double w = c * (skw[kk][6] - skw[kk][7] * a2sum);
#pragma unroll
            for (int q = 0; q < 6; q++) m[q] = fma(w, skw[kk][q], m[q]);
        }
    }
    // real part: lattice images of the minimum-image separation
    __syncthreads();
    const int nimg = min(nr, kEwMaxImg);
    for (int t = threadIdx.x; t < 3 * nimg; t += blockDim.x) simg[t] = img[t];
    __syncthreads();
    if (!live) return;
    double d0[3];
    for (int c = 0; c < 3; c++) {
        const double d = pos[3 * j + c] - pos[3 * i + c];
        d0[c] = d - box * rint(d / box);  // drem(d, box)
    }
    if (i == j) {
        const double self = 1.0 / ai - xi / sqrt(M_PI) * (6.0 - 40.0 / 3.0 * xi * xi * ai * ai);
        m[0] += self;
        m[3] += self;
        m[5] += self;
    }
    for (int q = 0; q < nr; q++) {
        const double *sh = q < kEwMaxImg ? &simg[3 * q] : &img[3 * q];
        const double x = d0[0] + sh[0], y = d0[1] + sh[1], z = d0[2] + sh[2];
        const double rr = x * x + y * y + z * z;
        if (rr == 0.0 || rr > rmax2) continue;
        const double r = sqrt(rr);
        double xa, ya;
        rpy_real_scalars(xi, r, a2sum, xa, ya);
        if (r < ai + aj) {  // overlapping spheres (src/mob/ewald.cc:177-185)
            xa += -(1.5 - a2sum * 0.5 / rr) / r + 2.0 / (ai + aj) - 3.0 * r / 8.0 / a2sum;
            ya += -(0.75 + a2sum * 0.25 / rr) / r + 2.0 / (ai + aj) - 9.0 * r / 16.0 / a2sum;
        }
        const double ex = x / r, ey = y / r, ez = z / r, dxy = xa - ya;
        m[0] += dxy * ex * ex + ya;
        m[1] += dxy * ex * ey;
        m[2] += dxy * ex * ez;
        m[3] += dxy * ey * ey + ya;
        m[4] += dxy * ey * ez;
        m[5] += dxy * ez * ez + ya;
    }
    const double b[3][3] = {{m[0], m[1], m[2]}, {m[1], m[3], m[4]}, {m[2], m[4], m[5]}};
    for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++) {
            mat[(size_t)(3 * i + a) * ldm + 3 * j + c] = b[a][c];
            if (i != j) mat[(size_t)(3 * j + a) * ldm + 3 * i + c] = b[a][c];
        }
}

// v[:, r] := alpha M f[:, r] + beta v[:, r] for r < nr (<= 16): one warp per
// matrix row, the row read once for every RHS.
constexpr int kEwMaxRhs = 16;
__global__ void __launch_bounds__(256)
k_ew_mulvec(int n3, int nr, double alpha, const double *__restrict__ mat, int ldm, const double *__restrict__ f,
            int ldf, double beta, double *__restrict__ v, int ldv)
{
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= n3) return;
    double acc[kEwMaxRhs];
#pragma unroll
    for (int r = 0; r < kEwMaxRhs; r++) acc[r] = 0.0;
    const double *mr = mat + (size_t)row * ldm;
    for (int c = lane; c < n3; c += 32) {
        const double x = mr[c];
#pragma unroll
        for (int r = 0; r < kEwMaxRhs; r++)
            if (r < nr) acc[r] = fma(x, f[(size_t)r * ldf + c], acc[r]);
    }
#pragma unroll
    for (int r = 0; r < kEwMaxRhs; r++) {
        if (r >= nr) break;
        double s = acc[r];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            double *o = v + (size_t)r * ldv + row;
            *o = (beta == 0.0 ? 0.0 : beta * *o) + alpha * s;
        }
    }
}

int ew_error(EwaldEngine *e, int st, const std::string &msg)
{
    e->last_error = msg;
    return st;
}

}  // namespace

#define EW_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t err_ = (call);                                                        \
        if (err_ != cudaSuccess)                                                          \
            return ew_error(e, kErrCuda, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

#define EW_LAUNCH()                                                                       \
    do {                                                                                  \
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                        \
        cudaError_t err_ = cudaGetLastError();                                            \
        if (err_ != cudaSuccess)                                                          \
            return ew_error(e, kErrCuda, std::string("ewald kernel: ") + cudaGetErrorString(err_)); \
    } while (0)

int ewald_create(EwaldEngine *e, const double *rdi)
{
    if (e->npos <= 0) return ew_error(e, kErrInvalid, "npos must be > 0");
    if (!(e->box > 0.0)) return ew_error(e, kErrInvalid, "box_size must be > 0");
    if (!(e->tol > 0.0)) return ew_error(e, kErrInvalid, "tol must be > 0");
    if (!(e->xi > 0.0)) e->xi = std::pow(10.0, 1.0 / 6.0) * std::sqrt(M_PI) / e->box;
    for (int i = 0; i < e->npos; i++)
        if (!(rdi[i] > 0.0)) return ew_error(e, kErrInvalid, "particle radii must be > 0");
    const double L = e->box, xi = e->xi;
    e->n3 = 3 * e->npos;
    e->ldm = (e->n3 + 31) / 32 * 32;
    // lattice images within rmax + the cell diagonal of the minimum image
    // (InitRealTable, src/mob/ewald.cc:643-704)
    e->rmax = cutoff_rmax(xi, e->tol, L);
    const int rmaxi = (int)(e->rmax / L) + 1;
    const double rl = std::sqrt(3.0 * L * L);
    std::vector<double> img;
    for (int m1 = -rmaxi; m1 <= rmaxi; m1++)
        for (int m2 = -rmaxi; m2 <= rmaxi; m2++)
            for (int m3 = -rmaxi; m3 <= rmaxi; m3++) {
                const int mm[3] = {m1, m2, m3};
                double q2 = 0.0;
                for (int c = 0; c < 3; c++) {
                    const double q = L * mm[c] - (mm[c] > 0 ? 0.5 * L : (mm[c] < 0 ? -0.5 * L : 0.0));
                    q2 += q * q;
                }
                if (std::sqrt(q2) <= e->rmax + rl)
                    for (int c = 0; c < 3; c++) img.push_back(L * mm[c]);
            }
    e->nr = (int)(img.size() / 3);
    // reciprocal vectors |k| <= kmax, k != 0 (InitRecipTable, :707-797)
    e->kmax = cutoff_kmax(xi, e->tol, L);
    const int kmaxi = (int)(e->kmax * L / (2.0 * M_PI));
    const double pivol = M_PI / (L * L * L);
    std::vector<double> kv, kw;
    for (int m1 = -kmaxi; m1 <= kmaxi; m1++)
        for (int m2 = -kmaxi; m2 <= kmaxi; m2++)
            for (int m3 = -kmaxi; m3 <= kmaxi; m3++) {
                if (m1 == 0 && m2 == 0 && m3 == 0) continue;
                const double k1 = 2.0 * M_PI * m1 / L, k2 = 2.0 * M_PI * m2 / L, k3 = 2.0 * M_PI * m3 / L;
                const double kk = k1 * k1 + k2 * k2 + k3 * k3, k = std::sqrt(kk);
                if (k > e->kmax) continue;
                const double k4z = kk / (4.0 * xi * xi);
                const double kexp = pivol * (1.0 + k4z * (1.0 + 2.0 * k4z)) / kk * std::exp(-k4z);
                const double ex = k1 / k, ey = k2 / k, ez = k3 / k;
                const double rec[4] = {k1, k2, k3, 0.0};
                const double w[8] = {1.0 - ex * ex, -ex * ey, -ex * ez, 1.0 - ey * ey, -ey * ez, 1.0 - ez * ez,
                                     6.0 * kexp, kk * kexp};
                kv.insert(kv.end(), rec, rec + 4);
                kw.insert(kw.end(), w, w + 8);
            }
    e->nk = (int)(kv.size() / 4);
    EW_CUDA(cudaSetDevice(e->device));
    if (!e->stream) {
        EW_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->own_stream = true;
    }
    const size_t mat_bytes = (size_t)e->n3 * e->ldm * sizeof(double);
    size_t free_b = 0, total_b = 0;
    EW_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (mat_bytes > free_b / 2)
        return ew_error(e, kErrAlloc, "the dense 3N x 3N matrix does not fit in half the free device memory");
    EW_CUDA(cudaMalloc(&e->d_mat, mat_bytes));
    EW_CUDA(cudaMalloc(&e->d_rdi, e->npos * sizeof(double)));
    EW_CUDA(cudaMalloc(&e->d_img, std::max<size_t>(1, img.size()) * sizeof(double)));
    EW_CUDA(cudaMalloc(&e->d_kv, std::max<size_t>(1, kv.size()) * sizeof(double) * 3));  // kv (4) + kw (8)
    EW_CUDA(cudaMalloc(&e->d_pos, e->n3 * sizeof(double)));
    EW_CUDA(cudaMalloc(&e->d_cs, std::max<size_t>(1, (size_t)2 * e->nk * e->npos) * sizeof(double)));
    EW_CUDA(cudaMemcpy(e->d_rdi, rdi, e->npos * sizeof(double), cudaMemcpyHostToDevice));
    if (!img.empty()) EW_CUDA(cudaMemcpy(e->d_img, img.data(), img.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (!kv.empty()) {
        EW_CUDA(cudaMemcpy(e->d_kv, kv.data(), kv.size() * sizeof(double), cudaMemcpyHostToDevice));
        EW_CUDA(cudaMemcpy(e->d_kv + kv.size(), kw.data(), kw.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    return kOk;
}

int ewald_update(EwaldEngine *e, const double *d_pos)
{
    const int n = e->npos;
    if (d_pos != e->d_pos)
        EW_CUDA(cudaMemcpyAsync(e->d_pos, d_pos, e->n3 * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    if (e->nk > 0) {
        const long long t = (long long)n * e->nk;
        k_ew_factors<<<(unsigned)((t + 255) / 256), 256, 0, e->stream>>>(n, e->nk, e->d_kv, e->d_pos, e->d_cs);
        EW_LAUNCH();
    }
    const int nt = (n + kEwTile - 1) / kEwTile;
    const double *kw = e->d_kv + (size_t)4 * e->nk;
    k_ew_matrix<<<dim3(nt, nt), kEwTile * kEwTile, 0, e->stream>>>(n, e->nk, e->nr, e->box, e->xi,
                                                                 e->rmax * e->rmax, e->d_pos, e->d_rdi, e->d_img,
                                                                 kw, e->d_cs, e->d_mat, e->ldm);
    EW_LAUNCH();
    e->updated = true;
    return kOk;
}

int ewald_mulvec(EwaldEngine *e, int nrhs, double alpha, int ldf, const double *d_f, double beta, int ldv,
                 double *d_v)
{
    if (!e->updated) return ew_error(e, kErrState, "Update() must be called before MulVector()");
    if (nrhs < 0 || ldf < e->n3 || ldv < e->n3) return ew_error(e, kErrInvalid, "bad nrhs or leading dimension");
    for (int r0 = 0; r0 < nrhs; r0 += kEwMaxRhs) {
        const int nr = std::min(kEwMaxRhs, nrhs - r0);
        k_ew_mulvec<<<(e->n3 + 7) / 8, 256, 0, e->stream>>>(e->n3, nr, alpha, e->d_mat, e->ldm,
                                                            d_f + (size_t)r0 * ldf, ldf, beta,
                                                            d_v + (size_t)r0 * ldv, ldv);
        EW_LAUNCH();
    }
    return kOk;
}

void ewald_free(EwaldEngine *e)
{
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    void *ptrs[] = {e->d_rdi, e->d_img, e->d_kv, e->d_pos, e->d_cs, e->d_mat, e->d_fin, e->d_vout};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    *e = EwaldEngine();
}

MobOp ewald_mob_op(EwaldEngine *e)
{
    MobOp op;
    op.dim = e->n3;
    op.mulvec = [e](int nr, double a, int ldf, const double *f, double b, int ldv, double *v, cudaStream_t s) {
        cudaStream_t saved = e->stream;
        e->stream = s;
        const int st = ewald_mulvec(e, nr, a, ldf, f, b, ldv, v);
        e->stream = saved;
        return st;
    };
    op.error = [e]() { return e->last_error; };
    return op;
}

}  // namespace sdt
