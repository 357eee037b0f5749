/*
 * Test infrastructure only (oracle).  Implements the subset of the MKL DFTI
 * descriptor API that the reference SPME engine calls
 * (src/mob/spme.cc:549-618 create/commit, :754-765 and :782-833 compute):
 * a 3-D double-precision real<->complex transform, in place, with explicit
 * input/output strides, conjugate-even storage "COMPLEX_COMPLEX" and a
 * backward scale factor.
 *
 * The transform is a plain row-column FFT: a real-to-complex pass along the
 * unit-stride axis (half-length complex FFT plus the standard split step),
 * then complex FFTs along the two strided axes, processed in blocks of
 * adjacent lines so the strided passes read whole cache lines.  Complex
 * line transforms are iterative radix-2 for power-of-two lengths and a
 * direct O(n^2) DFT otherwise.  Sign convention as MKL: forward uses
 * exp(-2*pi*i*j*k/n), backward exp(+2*pi*i*j*k/n), unnormalised except for
 * the configured scale.
 */
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <omp.h>
#include "mkl.h"

namespace {

struct LinePlan {
    int n = 0;
    bool pow2 = false;
    std::vector<int> rev;        // bit reversal permutation (pow2 only)
    std::vector<double> wre, wim;  // exp(-2 pi i k / n), k < n
    void init(int len)
    {
        n = len;
        pow2 = (n & (n - 1)) == 0;
        wre.resize(n);
        wim.resize(n);
        for (int k = 0; k < n; k++) {
            double a = -2.0 * M_PI * (double)k / (double)n;
            wre[k] = cos(a);
            wim[k] = sin(a);
        }
        if (pow2) {
            rev.resize(n);
            int lg = 0;
            while ((1 << lg) < n) lg++;
            for (int i = 0; i < n; i++) {
                int r = 0;
                for (int b = 0; b < lg; b++) r |= ((i >> b) & 1) << (lg - 1 - b);
                rev[i] = r;
            }
        }
    }
    // In-place complex transform of re/im arrays of length n; sign -1 forward.
    void run(double *re, double *im, int sign, double *tre, double *tim) const
    {
        if (n <= 1) return;
        if (pow2) {
            for (int i = 0; i < n; i++) {
                int r = rev[i];
                if (r > i) {
                    double t = re[i]; re[i] = re[r]; re[r] = t;
                    t = im[i]; im[i] = im[r]; im[r] = t;
                }
            }
            for (int len = 2; len <= n; len <<= 1) {
                int half = len >> 1;
                int step = n / len;
                for (int i = 0; i < n; i += len) {
                    for (int j = 0; j < half; j++) {
                        double wr = wre[j * step];
                        double wi = sign < 0 ? wim[j * step] : -wim[j * step];
                        int a = i + j, b = a + half;
                        double vr = re[b] * wr - im[b] * wi;
                        double vi = re[b] * wi + im[b] * wr;
                        re[b] = re[a] - vr;
                        im[b] = im[a] - vi;
                        re[a] += vr;
                        im[a] += vi;
                    }
                }
            }
        } else {
            for (int k = 0; k < n; k++) {
                double sr = 0.0, si = 0.0;
                for (int j = 0; j < n; j++) {
                    int idx = (int)(((long)j * k) % n);
                    double wr = wre[idx];
                    double wi = sign < 0 ? wim[idx] : -wim[idx];
                    sr += re[j] * wr - im[j] * wi;
                    si += re[j] * wi + im[j] * wr;
                }
                tre[k] = sr;
                tim[k] = si;
            }
            memcpy(re, tre, sizeof(double) * n);
            memcpy(im, tim, sizeof(double) * n);
        }
    }
};

}  // namespace

struct SdtDftiDesc {
    int dims;
    long len[3];
    long istr[4];
    long ostr[4];
    double fscale;
    double bscale;
    bool committed;
    LinePlan plan[3];
    LinePlan half_plan;   // length len[2]/2 for the real split step
    bool use_half;
};

namespace {

// Real row (length n, stride s, real units) -> n/2+1 complex (stride cs, complex units)
void RowR2C(const SdtDftiDesc *d, const double *in, long s, double *out, long cs,
            std::vector<double> &buf)
{
    const int n = (int)d->len[2];
    double *re = &buf[0], *im = re + n, *tre = im + n, *tim = tre + n;
    if (d->use_half) {
        const int h = n / 2;
        for (int m = 0; m < h; m++) {
            re[m] = in[(2 * m) * s];
            im[m] = in[(2 * m + 1) * s];
        }
        d->half_plan.run(re, im, -1, tre, tim);
        // split step: X[k] = (Z[k]+conj Z[h-k])/2 - i/2 W^k (Z[k]-conj Z[h-k])
        for (int k = 0; k <= h; k++) {
            int k1 = k % h, k2 = (h - k) % h;
            double zr = re[k1], zi = im[k1];
            double cr = re[k2], ci = -im[k2];
            double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
            double orr = 0.5 * (zr - cr), oi = 0.5 * (zi - ci);  // (Z - conj)/2
            double wr = d->plan[2].wre[k % n], wi = d->plan[2].wim[k % n];
            // -i * W * o
            double tr = wr * orr - wi * oi, ti = wr * oi + wi * orr;
            out[2 * (k * cs) + 0] = er + ti;
            out[2 * (k * cs) + 1] = ei - tr;
        }
    } else {
        for (int j = 0; j < n; j++) {
            re[j] = in[j * s];
            im[j] = 0.0;
        }
        d->plan[2].run(re, im, -1, tre, tim);
        for (int k = 0; k <= n / 2; k++) {
            out[2 * (k * cs) + 0] = re[k];
            out[2 * (k * cs) + 1] = im[k];
        }
    }
}

// n/2+1 complex (stride cs) -> real row (stride s), unnormalised backward
void RowC2R(const SdtDftiDesc *d, const double *in, long cs, double *out, long s,
            double scale, std::vector<double> &buf)
{
    const int n = (int)d->len[2];
    double *re = &buf[0], *im = re + n, *tre = im + n, *tim = tre + n;
    if (d->use_half) {
        const int h = n / 2;
        for (int k = 0; k < h; k++) {
            double xr = in[2 * (k * cs)], xi = in[2 * (k * cs) + 1];
            double yr = in[2 * ((h - k) * cs)], yi = -in[2 * ((h - k) * cs) + 1];
            if (k == 0) { xi = 0.0; yi = 0.0; }  // real DC and Nyquist bins
            double ar = xr + yr, ai = xi + yi;      // 2E
            double br = xr - yr, bi = xi - yi;      // X - conj X'
            // conj(W^k) = exp(+2 pi i k/n)
            double wr = d->plan[2].wre[k], wi = -d->plan[2].wim[k];
            double orr = br * wr - bi * wi, oi = br * wi + bi * wr;  // 2O
            re[k] = ar - oi;   // 2E + i*2O
            im[k] = ai + orr;
        }
        d->half_plan.run(re, im, +1, tre, tim);
        for (int m = 0; m < h; m++) {
            out[(2 * m) * s] = re[m] * scale;
            out[(2 * m + 1) * s] = im[m] * scale;
        }
    } else {
        for (int k = 0; k <= n / 2; k++) {
            re[k] = in[2 * (k * cs)];
            im[k] = in[2 * (k * cs) + 1];
        }
        for (int k = n / 2 + 1; k < n; k++) {
            re[k] = re[n - k];
            im[k] = -im[n - k];
        }
        d->plan[2].run(re, im, +1, tre, tim);
        for (int j = 0; j < n; j++) out[j * s] = re[j] * scale;
    }
}

// Complex FFT along axis `ax` (0 or 1) of the complex array with strides cstr
// (complex units) and extents nz x ny x nxc.  Lines are processed in blocks of
// adjacent entries of the unit-stride axis.
void AxisPass(const SdtDftiDesc *d, double *data, int ax, int sign, long nxc)
{
    const long n0 = d->len[0], n1 = d->len[1];
    const long c0 = d->ostr[1], c1 = d->ostr[2], c2 = d->ostr[3];
    const int n = (int)d->len[ax];
    const long lstride = (ax == 0) ? c0 : c1;
    const long outer = (ax == 0) ? n1 : n0;
    const long ostride = (ax == 0) ? c1 : c0;
    const int B = 8;
    const long nblk = (nxc + B - 1) / B;
    #pragma omp parallel
    {
        std::vector<double> buf((size_t)4 * n * B + 4 * n);
        #pragma omp for schedule(static)
        for (long t = 0; t < outer * nblk; t++) {
            long o = t / nblk;
            long k0 = (t % nblk) * B;
            int nb = (int)((k0 + B <= nxc) ? B : nxc - k0);
            double *re = &buf[0];
            double *im = re + (size_t)n * B;
            double *tre = im + (size_t)n * B;
            double *tim = tre + n;
            for (int j = 0; j < n; j++) {
                const double *p = data + 2 * (o * ostride + j * lstride + k0 * c2);
                for (int b = 0; b < nb; b++) {
                    re[b * n + j] = p[2 * b * c2];
                    im[b * n + j] = p[2 * b * c2 + 1];
                }
            }
            for (int b = 0; b < nb; b++) {
                d->plan[ax].run(re + b * n, im + b * n, sign, tre, tim);
            }
            for (int j = 0; j < n; j++) {
                double *p = data + 2 * (o * ostride + j * lstride + k0 * c2);
                for (int b = 0; b < nb; b++) {
                    p[2 * b * c2] = re[b * n + j];
                    p[2 * b * c2 + 1] = im[b * n + j];
                }
            }
        }
    }
}

}  // namespace

extern "C" {

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *handle, int precision, int domain,
                              MKL_LONG dimension, ...)
{
    if (precision != DFTI_DOUBLE || domain != DFTI_REAL || dimension != 3) return 1;
    va_list ap;
    va_start(ap, dimension);
    const MKL_LONG *sz = va_arg(ap, const MKL_LONG *);
    va_end(ap);
    SdtDftiDesc *d = new SdtDftiDesc();
    d->dims = 3;
    for (int i = 0; i < 3; i++) d->len[i] = sz[i];
    // default: packed row-major strides
    d->istr[0] = 0; d->istr[3] = 1; d->istr[2] = d->len[2]; d->istr[1] = d->len[1] * d->len[2];
    d->ostr[0] = 0; d->ostr[3] = 1; d->ostr[2] = d->len[2] / 2 + 1;
    d->ostr[1] = d->len[1] * (d->len[2] / 2 + 1);
    d->fscale = 1.0;
    d->bscale = 1.0;
    d->committed = false;
    d->use_half = false;
    *handle = d;
    return 0;
}

MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE d, int param, ...)
{
    va_list ap;
    va_start(ap, param);
    MKL_LONG ret = 0;
    switch (param) {
        case DFTI_INPUT_STRIDES: {
            const MKL_LONG *s = va_arg(ap, const MKL_LONG *);
            for (int i = 0; i < 4; i++) d->istr[i] = s[i];
            break;
        }
        case DFTI_OUTPUT_STRIDES: {
            const MKL_LONG *s = va_arg(ap, const MKL_LONG *);
            for (int i = 0; i < 4; i++) d->ostr[i] = s[i];
            break;
        }
        case DFTI_CONJUGATE_EVEN_STORAGE: {
            int v = va_arg(ap, int);
            ret = (v == DFTI_COMPLEX_COMPLEX) ? 0 : 1;
            break;
        }
        case DFTI_BACKWARD_SCALE:
            d->bscale = va_arg(ap, double);
            break;
        case DFTI_FORWARD_SCALE:
            d->fscale = va_arg(ap, double);
            break;
        default:
            ret = 1;
    }
    va_end(ap);
    return ret;
}

MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE d)
{
    for (int i = 0; i < 3; i++) d->plan[i].init((int)d->len[i]);
    const int n = (int)d->len[2];
    d->use_half = (n % 2 == 0) && n >= 4 && ((n / 2) & (n / 2 - 1)) == 0;
    if (d->use_half) d->half_plan.init(n / 2);
    d->committed = true;
    return 0;
}

// Forward: input real with istr, output complex with ostr, in place.  The
// backward descriptor of the reference swaps the two stride sets, so the
// real layout is always the one with the larger (real-unit) strides.
static void Forward3D(SdtDftiDesc *d, double *data)
{
    const long n0 = d->len[0], n1 = d->len[1], n2 = d->len[2];
    const long s0 = d->istr[1], s1 = d->istr[2], s2 = d->istr[3];
    const long c0 = d->ostr[1], c1 = d->ostr[2], c2 = d->ostr[3];
    #pragma omp parallel
    {
        std::vector<double> buf(4 * n2 + 8);
        #pragma omp for schedule(static)
        for (long r = 0; r < n0 * n1; r++) {
            long i0 = r / n1, i1 = r % n1;
            RowR2C(d, data + i0 * s0 + i1 * s1, s2, data + 2 * (i0 * c0 + i1 * c1), c2, buf);
        }
    }
    const long nxc = n2 / 2 + 1;
    AxisPass(d, data, 1, -1, nxc);
    AxisPass(d, data, 0, -1, nxc);
    if (d->fscale != 1.0) {
        for (long i0 = 0; i0 < n0; i0++)
            for (long i1 = 0; i1 < n1; i1++)
                for (long k = 0; k < nxc; k++) {
                    double *p = data + 2 * (i0 * c0 + i1 * c1 + k * c2);
                    p[0] *= d->fscale;
                    p[1] *= d->fscale;
                }
    }
}

static void Backward3D(SdtDftiDesc *d, double *data)
{
    // For the backward descriptor the input is complex (istr) and the
    // output is real (ostr); present them to the passes the same way.
    SdtDftiDesc v = *d;
    for (int i = 0; i < 4; i++) {
        v.ostr[i] = d->istr[i];   // complex strides
        v.istr[i] = d->ostr[i];   // real strides
    }
    const long n0 = v.len[0], n1 = v.len[1], n2 = v.len[2];
    const long nxc = n2 / 2 + 1;
    AxisPass(&v, data, 0, +1, nxc);
    AxisPass(&v, data, 1, +1, nxc);
    const long s0 = v.istr[1], s1 = v.istr[2], s2 = v.istr[3];
    const long c0 = v.ostr[1], c1 = v.ostr[2], c2 = v.ostr[3];
    #pragma omp parallel
    {
        std::vector<double> buf(4 * n2 + 8);
        #pragma omp for schedule(static)
        for (long r = 0; r < n0 * n1; r++) {
            long i0 = r / n1, i1 = r % n1;
            RowC2R(&v, data + 2 * (i0 * c0 + i1 * c1), c2, data + i0 * s0 + i1 * s1, s2,
                   d->bscale, buf);
        }
    }
}

// Wall time spent in the two compute calls since load (or the last reset),
// so a timed reference run can report the share of its time this stand-in
// FFT takes (it is not MKL).
static double g_fft_seconds = 0.0;
static long long g_fft_calls = 0;

static double now_s() { return omp_get_wtime(); }

MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE d, void *inout, ...)
{
    if (!d->committed) return 1;
    const double t0 = now_s();
    Forward3D(d, (double *)inout);
    g_fft_seconds += now_s() - t0;
    g_fft_calls++;
    return 0;
}

MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE d, void *inout, ...)
{
    if (!d->committed) return 1;
    const double t0 = now_s();
    Backward3D(d, (double *)inout);
    g_fft_seconds += now_s() - t0;
    g_fft_calls++;
    return 0;
}

// Seconds and calls of the compute calls so far; reset != 0 zeroes them.
double sdt_shim_fft_seconds(int reset, long long *calls)
{
    const double t = g_fft_seconds;
    if (calls) *calls = g_fft_calls;
    if (reset) {
        g_fft_seconds = 0.0;
        g_fft_calls = 0;
    }
    return t;
}

MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *handle)
{
    if (handle && *handle) {
        delete *handle;
        *handle = NULL;
    }
    return 0;
}

}  // extern "C"
