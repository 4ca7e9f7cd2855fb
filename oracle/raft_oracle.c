/*
 * raft_oracle.c -- CPU restatement of the ssc-raft parallel-beam hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
 * ssc-raft_b200/csrc: tests/, __graft_entry__.smoke() and the cpu_baseline leg
 * of bench.py are the only callers.  The product never links or calls it.
 *
 * Everything accumulates in FP64.  Where the reference computes an integer
 * sample index from FP32 arithmetic (nearest-truncation operators, "ref"
 * mode) the index is computed here with the same FP32 expressions, including
 * the multiply-add contraction the reference build applies (a*b - c*d is
 * evaluated as fmaf(a, b, -(c*d)) and i*d + m as fmaf(i, d, m); found by
 * comparing against the reference library's own outputs).  Two things the
 * oracle cannot restate: the GPU fast-intrinsic sin/cos (the caller may pass
 * those values as data, `tcos`/`tsin`; otherwise libm's are used) and the
 * fast approximate division (here an IEEE division), so a sample whose exact
 * position lies on a bin boundary may land in the neighbouring bin.
 *
 * Reference files followed (paths inside cnpem/ssc-raft):
 *   edge padding      cuda/src/common/padding.cu:140-178 (paddR2R)
 *   crop              cuda/src/common/padding.cu:245-268 (remove_paddR2R)
 *   filter weights    cuda/src/processing/filters/filters.cu:33-51 (tent + phase)
 *                     cuda/src/processing/filters/filters.cu:395-438 (Filter::apply)
 *   filter driver     cuda/src/processing/filters/filters.cu:163-190 (filterFBP)
 *                     cuda/src/processing/filters/filters.cu:120-161 (filterFBPpad)
 *   FBP backprojector cuda/src/geometries/parallel/reconstruction_methods/fbp.cu:8-76
 *   FBP driver        cuda/src/geometries/parallel/reconstruction_methods/fbp.cu:81-236
 *   Radon RT          cuda/src/geometries/parallel/forward_methods/radon_rt.cu:131-174
 *   EM kernels        cuda/src/geometries/parallel/reconstruction_methods/kernels/em_RT_kernel.cu:20-351
 *   tEM / eEM loops   cuda/src/geometries/parallel/reconstruction_methods/em_rt.cu:154-192,316-355
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

static const double PI_D = 3.14159265358979323846;

/* ------------------------------------------------------------------------ */
/* Mixed-radix FFT (any length; smallest-prime-factor decimation in time).   */
/* ------------------------------------------------------------------------ */
static int smallest_factor(int n)
{
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (int p = 3; p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

/* out[k] = sum_n in[n*stride] w^(n*k*(ntot/n)), w = exp(sign*2*pi*i/ntot);
 * recursive decimation in time.  `root` holds the ntot roots of unity. */
static void fft_rec(int n, const cplx *in, int stride, cplx *out, const cplx *root, int ntot,
                    cplx *scratch)
{
    if (n == 1) { out[0] = in[0]; return; }
    int p = smallest_factor(n);
    int m = n / p;
    for (int r = 0; r < p; r++)
        fft_rec(m, in + (size_t)r * stride, stride * p, out + (size_t)r * m, root, ntot, scratch);
    int step = ntot / n;      /* root index of exp(2 pi i / n) */
    int pstep = ntot / p;     /* root index of exp(2 pi i / p) */
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++)
            scratch[r] = out[(size_t)r * m + k] * root[(size_t)((long long)r * k * step % ntot)];
        for (int q = 0; q < p; q++) {
            cplx acc = 0;
            for (int r = 0; r < p; r++) acc += scratch[r] * root[(size_t)(((long long)r * q) % p) * pstep];
            scratch[p + q] = acc;
        }
        for (int q = 0; q < p; q++) out[(size_t)q * m + k] = scratch[p + q];
    }
}

static void fft(int n, const cplx *in, cplx *out, const cplx *root, cplx *scratch)
{
    fft_rec(n, in, 1, out, root, n, scratch);
}

static cplx *make_roots(int n, int sign)
{
    cplx *root = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    for (int m = 0; m < n; m++) {
        double ang = sign * 2.0 * PI_D * (double)m / (double)n;
        root[m] = cos(ang) + I * sin(ang);
    }
    return root;
}

/* ------------------------------------------------------------------------ */
/* Filter spectrum.                                                          */
/* ------------------------------------------------------------------------ */

/* Filter::apply (filters.cu:395-438).  `w` is the tent weight. */
static double ref_apply(int type, double w, double paganin, double reg)
{
    double pg = 1.0 / (1.0 + paganin * w * w);
    switch (type) {
    case 1: return w * exp(-0.693 * reg * w * w) * pg;
    case 2: return w * (1.0 / (1.0 + reg * w * w)) * pg;
    case 3: return w * cos(PI_D * 0.5 * w) * pg;
    case 4: {
        double param = fmax(w * reg * PI_D * 0.5, 1e-4);
        return w * (sin(param) / param) * pg;
    }
    case 5: return w * (0.5 + 0.5 * cos(2.0 * PI_D * w)) * pg;
    case 6: return w * (0.54 + 0.46 * cos(2.0 * PI_D * w)) * pg;
    case 7: return w * pg;
    case 8: return (w > 0) ? 1.0 / (2.0 * PI_D) : 0.0; /* SIGN(0)=0: DC weight taken as 0 */
    default: return 1.0;
    }
}

/* Linear-interpolation ("lin") mode filters: true ramp |k|/Np times a window
 * of nu = 2k/Np (nu = 1 at Nyquist).  Filter ids follow the reference enum
 * (filters.hpp:26-37) plus 9 = Shepp-Logan. */
static double lin_apply(int type, double nu, double paganin, double reg)
{
    double ramp = 0.5 * nu;
    double pg = 1.0 / (1.0 + paganin * nu * nu);
    switch (type) {
    case 1: return ramp * exp(-0.693 * reg * nu * nu) * pg;
    case 2: return ramp / (1.0 + reg * nu * nu) * pg;
    case 3: return ramp * cos(0.5 * PI_D * nu) * pg;
    case 4: {
        double param = fmax(nu * reg * PI_D * 0.5, 1e-4);
        return ramp * (sin(param) / param) * pg;
    }
    case 5: return ramp * 0.5 * (1.0 + cos(PI_D * nu)) * pg;
    case 6: return ramp * (0.54 + 0.46 * cos(PI_D * nu)) * pg;
    case 7: return ramp * pg;
    case 8: return (nu > 0) ? 1.0 / (2.0 * PI_D) : 0.0;
    case 9: {
        double a = 0.5 * PI_D * nu;
        return ramp * (a > 0 ? sin(a) / a : 1.0) * pg;
    }
    default: return 1.0;
    }
}

/* Full-length (Hermitian-extended) filter spectrum, including the
 * 1/(Np*pixel) normalisation of filters.cu:184-186.
 * mode 0 = ref (tent weight 0.5*min(k,M-k)/M, M=Np/2+1, phase denominator 2M-2),
 * mode 1 = lin (ramp |k|/Np, phase denominator Np). */
void oracle_filter_spectrum(int mode, int type, int Np, double paganin, double reg,
                            double offset, double pixel, double *hre, double *him)
{
    int M = Np / 2 + 1;
    double norm = 1.0 / ((double)Np * pixel);
    for (int k = 0; k < Np; k++) {
        int kk = (k <= Np / 2) ? k : Np - k;
        double w, phase;
        if (mode == 0) {
            double tent = 0.5 * fmin((double)kk, (double)(M - kk)) / (double)M;
            w = ref_apply(type, tent, paganin, reg);
            phase = 2.0 * PI_D / (double)(2 * M - 2) * offset * (double)kk;
        } else {
            w = lin_apply(type, 2.0 * (double)kk / (double)Np, paganin, reg);
            phase = 2.0 * PI_D * offset * (double)kk / (double)Np;
        }
        double re = w * cos(phase), im = -w * sin(phase);
        if (k > Np / 2) im = -im;                      /* conjugate half */
        if ((Np % 2 == 0) && k == Np / 2) im = 0.0;      /* C2R drops Im of the Nyquist bin */
        hre[k] = re * norm;
        him[k] = im * norm;
    }
}

/* Edge-replicating pad (padding.cu:140-178): out[i] = in[clamp(i - pad*N/2)]. */
static void pad_row(const float *in, int N, int pad, int Np, double *out)
{
    int off = (pad * N) / 2;
    for (int i = 0; i < Np; i++) {
        int ii = i - off;
        if (ii < 0) ii = 0;
        if (ii > N - 1) ii = N - 1;
        out[i] = in[ii];
    }
}

/* Filtered, padded rows q[row][0..Np) for nrows rows of length N.
 * type 0 ('none') copies the padded row unscaled, as the reference skips the
 * filter entirely for it (fbp.cu:102-103). */
void oracle_filter_rows(int mode, int type, int N, int nrows, int pad, double paganin,
                        double reg, double offset, double pixel, const float *sino, double *q)
{
    int Np = N * (1 + pad);
    double *hre = (double *)malloc(sizeof(double) * Np);
    double *him = (double *)malloc(sizeof(double) * Np);
    oracle_filter_spectrum(mode, type, Np, paganin, reg, offset, pixel, hre, him);
    cplx *rfwd = make_roots(Np, -1), *rinv = make_roots(Np, +1);
#pragma omp parallel
    {
        double *row = (double *)malloc(sizeof(double) * Np);
        cplx *a = (cplx *)malloc(sizeof(cplx) * Np);
        cplx *b = (cplx *)malloc(sizeof(cplx) * Np);
        cplx *scratch = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * Np + 8));
#pragma omp for schedule(dynamic, 4)
        for (int r = 0; r < nrows; r++) {
            pad_row(sino + (size_t)r * N, N, pad, Np, row);
            double *qr = q + (size_t)r * Np;
            if (type == 0) {
                memcpy(qr, row, sizeof(double) * Np);
                continue;
            }
            for (int i = 0; i < Np; i++) a[i] = row[i];
            fft(Np, a, b, rfwd, scratch);
            for (int k = 0; k < Np; k++) b[k] *= (hre[k] + I * him[k]);
            fft(Np, b, a, rinv, scratch);
            for (int i = 0; i < Np; i++) qr[i] = creal(a[i]);
        }
        free(row); free(a); free(b); free(scratch);
    }
    free(hre); free(him); free(rfwd); free(rinv);
}

/* Lowpass (low_pass.cu:9-29 + filterFBPpad): filter with internal padding,
 * axis offset 0, result cropped back to N (centre, offset pad*N/2). */
void oracle_lowpass(int mode, int type, int N, int nrows, int pad, double paganin, double reg,
                    double pixel, const float *sino, double *out)
{
    int Np = N * (1 + pad);
    int off = (pad * N) / 2;
    double *q = (double *)malloc(sizeof(double) * (size_t)nrows * Np);
    oracle_filter_rows(mode, type, N, nrows, pad, paganin, reg, 0.0, pixel, sino, q);
    for (int r = 0; r < nrows; r++)
        for (int i = 0; i < N; i++) out[(size_t)r * N + i] = q[(size_t)r * Np + off + i];
    free(q);
}

/* ------------------------------------------------------------------------ */
/* FBP backprojection on the central N x N window of the padded grid.       */
/* ------------------------------------------------------------------------ */
static void angle_steps(const float *angles, int A, float *dth)
{
    for (int a = 0; a < A; a++) {
        if (A == 1) { dth[a] = 1.0f; continue; }
        dth[a] = (a == A - 1) ? angles[a] - angles[a - 1] : angles[a + 1] - angles[a];
    }
}

static float angle_scale(const float *angles, int A)
{
    return (angles[A - 1] > (float)PI_D) ? (float)PI_D / angles[A - 1] : 1.0f;
}

/* mode 0: fbp.cu:38-74 truncation rule.  mode 1: linear interpolation on the
 * same sample grid (u = (t - tmin)/dt, samples at integer u, zero outside). */
#define DEFINE_BP(NAME, ACC)                                                                   \
void NAME(int mode, int N, int A, int nslices, int pad, float pixel_x, float pixel_y,           \
          const float *angles, const double *q, ACC *img, const float *tcos, const float *tsin) \
{                                                                                               \
    int Np = N * (1 + pad);                                                                     \
    int off = (pad * N) / 2;                                                                    \
    float *cs = (float *)malloc(sizeof(float) * A), *sn = (float *)malloc(sizeof(float) * A);   \
    float *dth = (float *)malloc(sizeof(float) * A);                                            \
    double *cd = (double *)malloc(sizeof(double) * A), *sd = (double *)malloc(sizeof(double) * A); \
    for (int a = 0; a < A; a++) {                                                               \
        cs[a] = tcos ? tcos[a] : cosf(angles[a]); sn[a] = tsin ? tsin[a] : sinf(angles[a]);     \
        cd[a] = cos((double)angles[a]); sd[a] = sin((double)angles[a]);                         \
    }                                                                                           \
    angle_steps(angles, A, dth);                                                                \
    float scale = angle_scale(angles, A);                                                       \
    float xmin = -pixel_x * (float)Np / 2.0f;                                                   \
    float ymin = -pixel_y * (float)Np / 2.0f;                                                   \
    float tmin = -pixel_x * (float)Np / 2.0f;                                                   \
    float dt = pixel_x;                                                                         \
    _Pragma("omp parallel for collapse(2) schedule(dynamic, 8)")                                \
    for (int k = 0; k < nslices; k++)                                                           \
        for (int jj = 0; jj < N; jj++) {                                                        \
            const double *qk = q + (size_t)k * A * Np;                                          \
            for (int ii = 0; ii < N; ii++) {                                                    \
                int i = ii + off, j = jj + off;                                                 \
                ACC sum = 0;                                                                    \
                if (mode == 0) {                                                                \
                    float x = fmaf((float)i, pixel_x, xmin);                                    \
                    float y = fmaf((float)j, pixel_y, ymin);                                    \
                    for (int a = 0; a < A; a++) {                                               \
                        float t = fmaf(x, cs[a], -(y * sn[a]));                                 \
                        int ti = (int)((t - tmin) / dt);                                        \
                        if (ti > -1 && ti < Np) sum += (ACC)qk[(size_t)a * Np + ti] * (ACC)dth[a]; \
                    }                                                                           \
                } else {                                                                        \
                    double x = ((double)i - 0.5 * Np) * pixel_x;                                \
                    double y = ((double)j - 0.5 * Np) * pixel_y;                                \
                    for (int a = 0; a < A; a++) {                                               \
                        double u = (x * cd[a] - y * sd[a]) / pixel_x + 0.5 * Np;                \
                        double fl = floor(u);                                                   \
                        int b0 = (int)fl;                                                       \
                        double f = u - fl;                                                      \
                        double v0 = (b0 >= 0 && b0 < Np) ? qk[(size_t)a * Np + b0] : 0.0;      \
                        double v1 = (b0 + 1 >= 0 && b0 + 1 < Np) ? qk[(size_t)a * Np + b0 + 1] : 0.0; \
                        sum += (ACC)(((1.0 - f) * v0 + f * v1) * (double)dth[a]);              \
                    }                                                                           \
                }                                                                               \
                img[((size_t)k * N + jj) * N + ii] = sum * (ACC)scale;                          \
            }                                                                                   \
        }                                                                                       \
    free(cs); free(sn); free(dth); free(cd); free(sd);                                           \
}

DEFINE_BP(oracle_fbp_backproject, double)
DEFINE_BP(oracle_fbp_backproject_f32, float)

/* Full FBP: filter (unless type 'none') then backproject.  img is [nslices,N,N]. */
/* tcos/tsin (may be NULL): sin/cos values to use for the nearest-sample
 * index rule instead of libm's, e.g. the GPU fast-intrinsic values the
 * reference computes (opt.cu:187-194), recorded as data in the fixtures. */
void oracle_fbp(int mode, int type, int N, int A, int nslices, int pad, double paganin,
                double reg, double offset, float pixel_x, float pixel_y, const float *angles,
                const float *sino, double *img, const float *tcos, const float *tsin)
{
    int Np = N * (1 + pad);
    double *q = (double *)malloc(sizeof(double) * (size_t)nslices * A * Np);
    oracle_filter_rows(mode, type, N, nslices * A, pad, paganin, reg, offset, pixel_x, sino, q);
    oracle_fbp_backproject(mode, N, A, nslices, pad, pixel_x, pixel_y, angles, q, img, tcos, tsin);
    free(q);
}

/* FP32-accumulating variant used as the timed CPU baseline. */
void oracle_fbp_f32(int mode, int type, int N, int A, int nslices, int pad, double paganin,
                    double reg, double offset, float pixel_x, float pixel_y, const float *angles,
                    const float *sino, float *img)
{
    int Np = N * (1 + pad);
    double *q = (double *)malloc(sizeof(double) * (size_t)nslices * A * Np);
    oracle_filter_rows(mode, type, N, nslices * A, pad, paganin, reg, offset, pixel_x, sino, q);
    oracle_fbp_backproject_f32(mode, N, A, nslices, pad, pixel_x, pixel_y, angles, q, img, NULL, NULL);
    free(q);
}

/* ------------------------------------------------------------------------ */
/* Radon RT (radon_rt.cu:131-174).  out[k][a][i]                            */
/* ------------------------------------------------------------------------ */
void oracle_radon_rt(int nx, int ny, int nrays, int A, int nslices, float ax, float ay,
                     const float *angles, const float *img, double *out, const float *tcos,
                     const float *tsin)
{
    float dx = 2.0f * ax / (float)(nx - 1);
    float dy = 2.0f * ay / (float)(ny - 1);
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = 0; k < nslices; k++)
        for (int a = 0; a < A; a++) {
            float c = tcos ? tcos[a] : cosf(angles[a]), s = tsin ? tsin[a] : sinf(angles[a]);
            for (int i = 0; i < nrays; i++) {
                float t = fmaf((float)i, dx, -ax);
                double sum = 0;
                for (int r = 0; r < ny; r++) {
                    float sr = fmaf((float)r, dy, -ay);
                    float x = fmaf(t, c, -(sr * s));
                    float y = fmaf(t, s, sr * c);
                    int ix = (int)((x + 1) / dx);
                    int iy = (int)((y + 1) / dy);
                    if (ix >= 0 && ix < nx && iy >= 0 && iy < ny)
                        sum += img[((size_t)k * ny + iy) * nx + ix];
                }
                out[((size_t)k * A + a) * nrays + i] = sum * (double)dy;
            }
        }
}

/* ------------------------------------------------------------------------ */
/* EM operators (em_RT_kernel.cu).                                           */
/* ------------------------------------------------------------------------ */

/* kernel_radon (em_RT_kernel.cu:145-185), a = 1: out[k][a][r] */
void oracle_em_forward(int N, int nrays, int A, int nslices, const float *angles,
                       const double *img, double *out, const float *tcos, const float *tsin)
{
    float a1 = 1.0f;
    float dt = (float)(2.0 * a1 / (nrays - 1));
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = 0; k < nslices; k++)
        for (int a = 0; a < A; a++) {
            float c = tcos ? tcos[a] : cosf(angles[a]), s = tsin ? tsin[a] : sinf(angles[a]);
            for (int r = 0; r < nrays; r++) {
                float t = fmaf((float)r, dt, -a1);
                double sum = 0;
                for (int m = 0; m < nrays; m++) {
                    float sm = fmaf((float)m, dt, -a1);
                    float x = fmaf(t, c, -(sm * s));
                    float y = fmaf(t, s, sm * c);
                    int X = (int)((x + 1) / dt);
                    int Y = (int)((y + 1) / dt);
                    if (X >= 0 && X < N && Y >= 0 && Y < N)
                        sum += img[((size_t)k * N + Y) * N + X];
                }
                out[((size_t)k * A + a) * nrays + r] = sum * (double)dt;
            }
        }
}

/* kernel_backprojection (em_RT_kernel.cu:92-142); sino==NULL gives the
 * back-projection of ones (kernel_backprojectionOfOnes, :303-351). */
void oracle_em_backproject(int N, int nrays, int A, int nslices, const float *angles,
                           const double *sino, double *img, const float *tcos, const float *tsin)
{
    float dxy = (float)(2.0 / (N - 1));
    float dt = (float)(2.0 / (nrays - 1));
    float *cs = (float *)malloc(sizeof(float) * A), *sn = (float *)malloc(sizeof(float) * A);
    float *dth = (float *)malloc(sizeof(float) * A);
    for (int a = 0; a < A; a++) {
        cs[a] = tcos ? tcos[a] : cosf(angles[a]);
        sn[a] = tsin ? tsin[a] : sinf(angles[a]);
    }
    angle_steps(angles, A, dth);
#pragma omp parallel for collapse(2) schedule(dynamic, 8)
    for (int k = 0; k < nslices; k++)
        for (int j = 0; j < N; j++)
            for (int i = 0; i < N; i++) {
                float x = fmaf((float)i, dxy, -1.0f);
                float y = fmaf((float)j, dxy, -1.0f);
                double sum = 0;
                for (int a = 0; a < A; a++) {
                    float t = fmaf(x, cs[a], y * sn[a]);
                    int T = (int)((t + 1.0f) / dt);
                    if (T > -1 && T < nrays)
                        sum += (sino ? sino[((size_t)k * A + a) * nrays + T] : 1.0) * (double)dth[a];
                }
                img[((size_t)k * N + j) * N + i] = sum;
            }
    free(cs); free(sn); free(dth);
}

/* tEM (em_rt.cu:154-192).  counts = exp(-data) already applied (as the
 * Python wrapper does, em_methods.py:109).  flat is [nslices][nrays]
 * (intended semantics: flat of the slice, not of the angle row). */
void oracle_tem(int N, int nrays, int A, int nslices, int niter, const float *angles,
                const float *counts, const float *flat, double *obj, const float *fcos,
                const float *fsin, const float *bcos, const float *bsin)
{
    size_t ns = (size_t)nslices * A * nrays, ni = (size_t)nslices * N * N;
    double *c = (double *)malloc(sizeof(double) * ns);
    double *p = (double *)malloc(sizeof(double) * ns);
    double *bc = (double *)malloc(sizeof(double) * ni);
    double *b = (double *)malloc(sizeof(double) * ni);
    for (size_t i = 0; i < ns; i++) c[i] = counts[i];
    oracle_em_backproject(N, nrays, A, nslices, angles, c, bc, bcos, bsin);
    for (int it = 0; it < niter; it++) {
        oracle_em_forward(N, nrays, A, nslices, angles, obj, p, fcos, fsin);
        for (int k = 0; k < nslices; k++)
            for (int a = 0; a < A; a++)
                for (int r = 0; r < nrays; r++) {
                    size_t ix = ((size_t)k * A + a) * nrays + r;
                    p[ix] = (double)flat[(size_t)k * nrays + r] * exp(-p[ix]);
                }
        oracle_em_backproject(N, nrays, A, nslices, angles, p, b, bcos, bsin);
        for (size_t i = 0; i < ni; i++) obj[i] = obj[i] * b[i] / bc[i];
    }
    free(c); free(p); free(bc); free(b);
}

/* eEM (em_rt.cu:316-355; kernel_radonWithDivision em_RT_kernel.cu:188-246). */
void oracle_eem(int N, int nrays, int A, int nslices, int niter, const float *angles,
                const float *tomo, double *obj, const float *fcos, const float *fsin,
                const float *bcos, const float *bsin)
{
    size_t ns = (size_t)nslices * A * nrays, ni = (size_t)nslices * N * N;
    double *p = (double *)malloc(sizeof(double) * ns);
    double *bo = (double *)malloc(sizeof(double) * ni);
    double *b = (double *)malloc(sizeof(double) * ni);
    oracle_em_backproject(N, nrays, A, nslices, angles, NULL, bo, bcos, bsin);
    for (int it = 0; it < niter; it++) {
        oracle_em_forward(N, nrays, A, nslices, angles, obj, p, fcos, fsin);
        for (size_t i = 0; i < ns; i++) {
            double v = p[i];
            double sg = (v > 0) ? 1.0 : ((v < 0) ? -1.0 : 0.0);
            double r = (double)tomo[i] * sg / sqrt(1e-8 + v * v);
            p[i] = r < 0 ? 0.0 : r;
        }
        oracle_em_backproject(N, nrays, A, nslices, angles, p, b, bcos, bsin);
        for (size_t i = 0; i < ni; i++) obj[i] = obj[i] * b[i] / bo[i];
    }
    free(p); free(bo); free(b);
}

/* Transmission data residual ||flat*exp(-Ax) - y|| / ||y|| and Poisson
 * negative log-likelihood sum(flat*exp(-Ax) + y*Ax), both per slice. */
void oracle_tem_metrics(int N, int nrays, int A, int nslices, const float *angles,
                        const float *counts, const float *flat, const double *obj,
                        double *residual, double *nll, const float *fcos, const float *fsin)
{
    size_t ns = (size_t)nslices * A * nrays;
    double *p = (double *)malloc(sizeof(double) * ns);
    oracle_em_forward(N, nrays, A, nslices, angles, obj, p, fcos, fsin);
    for (int k = 0; k < nslices; k++) {
        double num = 0, den = 0, l = 0;
        for (int a = 0; a < A; a++)
            for (int r = 0; r < nrays; r++) {
                size_t ix = ((size_t)k * A + a) * nrays + r;
                double m = (double)flat[(size_t)k * nrays + r] * exp(-p[ix]);
                double y = counts[ix];
                num += (m - y) * (m - y);
                den += y * y;
                l += m + y * p[ix];
            }
        residual[k] = sqrt(num) / (den > 0 ? sqrt(den) : 1.0);
        nll[k] = l;
    }
    free(p);
}

/* ------------------------------------------------------------------------ */
/* 3x3 convolution, stride 1, zero padding 1, NHWC (the warm-start U-Net's   */
/* layer; no reference counterpart).  FP64.                                  */
/* x [N][H][W][Cin], w [Cout][3][3][Cin], y [N][H][W][Cout]                  */
/* ------------------------------------------------------------------------ */
void oracle_conv3x3_fwd(const double *x, const double *w, const double *b, double *y, int N, int H, int W,
                        int Cin, int Cout, int relu)
{
#pragma omp parallel for collapse(2)
    for (int n = 0; n < N; n++)
        for (int yy = 0; yy < H; yy++)
            for (int xx = 0; xx < W; xx++)
                for (int co = 0; co < Cout; co++) {
                    double s = b ? b[co] : 0.0;
                    for (int ky = -1; ky <= 1; ky++)
                        for (int kx = -1; kx <= 1; kx++) {
                            int sy = yy + ky, sx = xx + kx;
                            if (sy < 0 || sy >= H || sx < 0 || sx >= W) continue;
                            const double *xp = x + (((size_t)n * H + sy) * W + sx) * Cin;
                            const double *wp = w + ((size_t)co * 9 + (ky + 1) * 3 + (kx + 1)) * Cin;
                            for (int ci = 0; ci < Cin; ci++) s += xp[ci] * wp[ci];
                        }
                    if (relu && s < 0) s = 0;
                    y[(((size_t)n * H + yy) * W + xx) * Cout + co] = s;
                }
}

/* dw[co][tap][ci] = sum_p dy[p][co] x[p+tap][ci] */
void oracle_conv3x3_wgrad(const double *dy, const double *x, double *dw, int N, int H, int W, int Cin, int Cout)
{
#pragma omp parallel for collapse(2)
    for (int co = 0; co < Cout; co++)
        for (int tap = 0; tap < 9; tap++) {
            int ky = tap / 3 - 1, kx = tap % 3 - 1;
            for (int ci = 0; ci < Cin; ci++) {
                double s = 0;
                for (int n = 0; n < N; n++)
                    for (int yy = 0; yy < H; yy++)
                        for (int xx = 0; xx < W; xx++) {
                            int sy = yy + ky, sx = xx + kx;
                            if (sy < 0 || sy >= H || sx < 0 || sx >= W) continue;
                            s += dy[(((size_t)n * H + yy) * W + xx) * Cout + co] *
                                 x[(((size_t)n * H + sy) * W + sx) * Cin + ci];
                        }
                dw[((size_t)co * 9 + tap) * Cin + ci] = s;
            }
        }
}

/* dx[p][ci] = sum_{co,tap} dy[p - tap][co] w[co][tap][ci] */
void oracle_conv3x3_dgrad(const double *dy, const double *w, double *dx, int N, int H, int W, int Cin, int Cout)
{
#pragma omp parallel for collapse(2)
    for (int n = 0; n < N; n++)
        for (int yy = 0; yy < H; yy++)
            for (int xx = 0; xx < W; xx++)
                for (int ci = 0; ci < Cin; ci++) {
                    double s = 0;
                    for (int tap = 0; tap < 9; tap++) {
                        int ky = tap / 3 - 1, kx = tap % 3 - 1;
                        int oy = yy - ky, ox = xx - kx;
                        if (oy < 0 || oy >= H || ox < 0 || ox >= W) continue;
                        const double *dp = dy + (((size_t)n * H + oy) * W + ox) * Cout;
                        for (int co = 0; co < Cout; co++) s += dp[co] * w[((size_t)co * 9 + tap) * Cin + ci];
                    }
                    dx[(((size_t)n * H + yy) * W + xx) * Cin + ci] = s;
                }
}

/* Flat/dark correction, BackgroundCorrection (background_correction.cu:15-47),
 * and -log, Klog (opt.cu:196-214), in FP64: per slice z, angle a, ray x
 *   flat = F[z][0][x]                                      (one flat)
 *        = F[z][0][x] (1 - a/A) + (a/A) F[z][1][x]         (two or more: first two)
 *   t    = max(D - dark, 0.5) / max(flat - dark, 0.5),  t = -log(t) if is_log. */
void oracle_background(const float *frames, const float *flat, const float *dark, int nrays, int nangles,
                       int nslices, int numflats, int is_log, double *out)
{
#pragma omp parallel for collapse(2)
    for (int z = 0; z < nslices; z++)
        for (int a = 0; a < nangles; a++)
            for (int x = 0; x < nrays; x++) {
                const double dk = dark[(size_t)z * nrays + x];
                double ft = flat[(size_t)z * numflats * nrays + x];
                if (numflats > 1) {
                    const double w = (double)a / (double)nangles;
                    ft = ft * (1.0 - w) + w * flat[((size_t)z * numflats + 1) * nrays + x];
                }
                const size_t i = ((size_t)z * nangles + a) * nrays + x;
                const double t = fmax(frames[i] - dk, 0.5) / fmax(ft - dk, 0.5);
                out[i] = is_log ? -log(t) : t;
            }
}

/* The BST operator on one slice of prepared rows [A][Np] (bst.cu:22-98):
 * half-rays of Np/2 samples split at Np/2 (the left one reversed), weighted by
 * w_half (half of it at the centre), zero-padded to L, L-point FFT times
 * 2 / (L max(min(k, L-k), 1/2)); polar -> Cartesian on an S x S grid with the
 * reference's float geometry and arc weights (t = iarc - angle on the lower
 * arc); S x S inverse transform (unnormalised); out[j][i] =
 * Re(grid[j+off][i+off]) / scale for i, j < ncrop. */
static void bst_slice(const double *rows, int A, int Np, int L, int S, int off, int ncrop, double w_half,
                      float scale, double *out, const cplx *rootsL, const cplx *rinvS)
{
    const int half = Np / 2, c = Np / 2, twoA = 2 * A;
    cplx *P = (cplx *)malloc(sizeof(cplx) * (size_t)twoA * L);
    cplx *cart = (cplx *)calloc((size_t)S * S, sizeof(cplx));
#pragma omp parallel
    {
        cplx *a = (cplx *)malloc(sizeof(cplx) * L);
        cplx *b = (cplx *)malloc(sizeof(cplx) * L);
        cplx *scratch = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * L + 8));
#pragma omp for schedule(dynamic, 4)
        for (int r = 0; r < A; r++) {
            const double *row = rows + (size_t)r * Np;
            for (int side = 0; side < 2; side++) {
                for (int idx = 0; idx < L; idx++) {
                    double v = 0.0;
                    if (idx < half) {
                        double w = idx == 0 ? 0.5 * w_half : w_half;
                        v = w * (side == 0 ? row[c - 1 - idx] : row[c + idx]);
                    }
                    a[idx] = v;
                }
                fft(L, a, b, rootsL, scratch);
                cplx *dst = P + (size_t)(side == 0 ? r : A + r) * L;
                for (int k = 0; k < L; k++) {
                    double m = (double)(k < L - k ? k : L - k);
                    dst[k] = b[k] * (2.0 / ((double)L * (m > 0.5 ? m : 0.5)));
                }
            }
        }
        free(a); free(b); free(scratch);
    }
#pragma omp parallel for schedule(dynamic, 8)
    for (int ty = 0; ty < S; ty++)
        for (int tx = 0; tx < S; tx++) {
            int posx = tx - S / 2, posy = ty - S / 2;
            float rho = (float)L * hypotf((float)posx, (float)posy) / (float)S;
            float angle = (float)twoA * (0.5f * atan2f((float)posy, (float)posx) / (float)PI_D + 0.5f);
            int irho = (int)rho;
            int iarc = (int)angle;
            cplx v = 0;
            if (irho < L / 2 - 1) {
                float pfrac = rho - (float)irho;
                float tfrac = (float)iarc - angle;
                iarc = iarc % twoA;
                int uarc = (iarc + 1) % twoA;
                const cplx *q0 = P + (size_t)iarc * L + irho, *q1 = P + (size_t)uarc * L + irho;
                cplx i0 = q0[0] * (double)(1.0f - pfrac) + q0[1] * (double)pfrac;
                cplx i1 = q1[0] * (double)(1.0f - pfrac) + q1[1] * (double)pfrac;
                v = i0 * (double)tfrac + i1 * (double)(1.0f - tfrac);
            }
            float sgn = 4.0f * ((float)(tx % 2) - 0.5f) * ((float)(ty % 2) - 0.5f);
            cart[(size_t)((ty + S / 2) % S) * S + (tx + S / 2) % S] = v * (double)sgn;
        }
#pragma omp parallel
    {
        cplx *a = (cplx *)malloc(sizeof(cplx) * S);
        cplx *b = (cplx *)malloc(sizeof(cplx) * S);
        cplx *scratch = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * S + 8));
#pragma omp for schedule(dynamic, 8)
        for (int y = 0; y < S; y++) {
            fft(S, cart + (size_t)y * S, b, rinvS, scratch);
            memcpy(cart + (size_t)y * S, b, sizeof(cplx) * S);
        }
#pragma omp for schedule(dynamic, 8)
        for (int i = 0; i < ncrop; i++) {
            for (int y = 0; y < S; y++) a[y] = cart[(size_t)y * S + off + i];
            fft(S, a, b, rinvS, scratch);
            for (int j = 0; j < ncrop; j++) out[(size_t)j * ncrop + i] = creal(b[off + j]) / (double)scale;
        }
        free(a); free(b); free(scratch);
    }
    free(P); free(cart);
}

/* FBP by the backprojection slice theorem: getBST (bst.cu:251-312) on the
 * padded tomogram of getBSTGPU (bst.cu:534-642), BSTFilter / BandFilterC2C
 * (filters.cu:295-390), sino2p / convBST / polar2cartesian_fourier
 * (bst.cu:22-98).  Transforms and accumulation in FP64; the regridding
 * geometry (radius, arc index and their fractions) in float, as the
 * reference computes it.  The half-rays are zero-padded (the reference's
 * buffer is not cleared) and all A rows are padded (the reference's padding
 * call covers N rows; identical when A == N).  csino: integer axis offset. */
void oracle_bst(const float *tomo, int N, int A, int B, int pad, int ftype, double paganin, double reg, int csino,
                float pixel, double *out)
{
    const int Np = N * (1 + pad), off = (pad * N) / 2;
    cplx *G = (cplx *)malloc(sizeof(cplx) * Np);
    for (int k = 0; k < Np; k++) {
        double w = ref_apply(ftype, (double)(k < Np - k ? k : Np - k) / (double)Np, paganin, reg);
        double ph = -2.0 * PI_D * (double)csino * (double)k / (double)Np;
        G[k] = w * (cos(ph) + I * sin(ph));
    }
    cplx *rfwd = make_roots(Np, -1), *rinv = make_roots(Np, +1);
    const float scale = (float)Np * pixel * 4.0f;
    double *rows = (double *)malloc(sizeof(double) * (size_t)A * Np);
    for (int z = 0; z < B; z++) {
#pragma omp parallel
        {
            cplx *a = (cplx *)malloc(sizeof(cplx) * Np);
            cplx *b = (cplx *)malloc(sizeof(cplx) * Np);
            cplx *scratch = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * Np + 8));
#pragma omp for schedule(dynamic, 4)
            for (int r = 0; r < A; r++) {
                double *row = rows + (size_t)r * Np;
                pad_row(tomo + ((size_t)z * A + r) * N, N, pad, Np, row);
                if (ftype != 0) {
                    for (int i = 0; i < Np; i++) a[i] = row[i];
                    fft(Np, a, b, rfwd, scratch);
                    for (int k = 0; k < Np; k++) b[k] *= G[k];
                    fft(Np, b, a, rinv, scratch);
                    for (int i = 0; i < Np; i++) row[i] = creal(a[i]);
                }
            }
            free(a); free(b); free(scratch);
        }
        bst_slice(rows, A, Np, Np, Np, off, N, 4.0, scale, out + (size_t)z * N * N, rfwd, rinv);
    }
    free(rows); free(G); free(rfwd); free(rinv);
}

/* 2-D transform in place of a [ny][nx] complex array: rows, then columns. */
static void fft2_inplace(cplx *d, int nx, int ny, int sign)
{
    cplx *rx = make_roots(nx, sign), *ry = make_roots(ny, sign);
    cplx *a = (cplx *)malloc(sizeof(cplx) * (size_t)(nx > ny ? nx : ny));
    cplx *b = (cplx *)malloc(sizeof(cplx) * (size_t)(nx > ny ? nx : ny));
    int m = nx > ny ? nx : ny;
    cplx *scratch = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * m + 8));
    for (int y = 0; y < ny; y++) {
        fft(nx, d + (size_t)y * nx, b, rx, scratch);
        memcpy(d + (size_t)y * nx, b, sizeof(cplx) * nx);
    }
    for (int x = 0; x < nx; x++) {
        for (int y = 0; y < ny; y++) a[y] = d[(size_t)y * nx + x];
        fft(ny, a, b, ry, scratch);
        for (int y = 0; y < ny; y++) d[(size_t)y * nx + x] = b[y];
    }
    free(rx); free(ry); free(a); free(b); free(scratch);
}

/* Rotation-axis offset by phase correlation: getCentersino / getCentersino_subpixel
 * (rotation_axis.cu:14-46,221-360): transforms in FP64, the correlation then
 * rounded to float and searched exactly as the reference's host loops do
 * (float |c|^2, the integer search over x = 0, 4, ... then the remainder, the
 * sub-pixel search over x = i * 0.01 with abs2InterpCubic's float weights). */
double oracle_centersino(const float *frame0, const float *frame180, const float *dark, const float *flat,
                         int sizex, int sizey, int subpixel)
{
    size_t plane = (size_t)sizex * sizey;
    cplx *F = (cplx *)malloc(sizeof(cplx) * plane), *G = (cplx *)malloc(sizeof(cplx) * plane);
    for (int y = 0; y < sizey; y++)
        for (int x = 0; x < sizex; x++) {
            size_t i = (size_t)y * sizex + x;
            double dk = dark[i], ft = flat[i], q = fmax(ft - dk, 0.5);
            F[i] = -log(fmax(frame0[i] - dk, 0.5) / q);
            G[(size_t)y * sizex + (sizex - 1 - x)] = -log(fmax(frame180[i] - dk, 0.5) / q);
        }
    fft2_inplace(F, sizex, sizey, -1);
    fft2_inplace(G, sizex, sizey, -1);
    for (int y = 0; y < sizey; y++)
        for (int x = 0; x < sizex; x++) {
            size_t i = (size_t)y * sizex + x;
            double xx = fmin((double)(sizex - x), (double)x) / sizex;
            double yy = fmin((double)(sizey - y), (double)y) / sizey;
            double gauss = exp(-20.0 * (xx * xx + yy * yy));
            cplx fg = F[i] * conj(G[i]);
            F[i] = fg * gauss / cabs(fg);
        }
    fft2_inplace(F, sizex, sizey, +1);
    float *re = (float *)malloc(sizeof(float) * plane), *im = (float *)malloc(sizeof(float) * plane);
    for (size_t i = 0; i < plane; i++) { re[i] = (float)creal(F[i]); im[i] = (float)cimag(F[i]); }
#define ABS2(i) (re[i] * re[i] + im[i] * im[i])
    float maxx = 0.0f;
    double result;
    if (!subpixel) {
        int posx = 0;
        int irange = (sizex >> 2) << 2;
        for (int j = 0; j < sizey; j++) {
            for (int i = 0; i < irange; i += 4) {
                float bbs = ABS2((size_t)j * sizex + i);
                if (bbs > maxx) { maxx = bbs; posx = i; }
            }
            for (int i = irange; i < sizex; i++) {
                float bbs = ABS2((size_t)j * sizex + i);
                if (bbs > maxx) { maxx = bbs; posx = i; }
            }
        }
        if (posx > (float)sizex / 2) posx -= sizex;
        result = (double)(-posx / 2);
    } else {
        float bestpos = 0.0f;
        const float di = 0.01f;
        for (int j = 0; j < sizey; j++)
            for (float i = 0; i < (float)sizex; i++) {
                float posx = i * di, posy = (float)j;
                int x0 = (int)floorf(posx), y0 = (int)floorf(posy);
                int x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, y1 = y0 + 1, y2 = y0 + 2, y3 = y0 + 3;
                int xs[4] = {x0, x1, x2, x3}, ys[4] = {y0, y1, y2, y3};
                float v[4][4];
                for (int a = 0; a < 4; a++)
                    for (int b = 0; b < 4; b++)
                        v[a][b] = (ys[a] >= 0 && ys[a] < sizey && xs[b] >= 0 && xs[b] < sizex)
                                      ? ABS2((size_t)ys[a] * sizex + xs[b]) : 0.0f;
                /* abs2InterpCubic (rotation_axis.cu:155-220): term order v00, v10, v20, v30, v01, ... */
                float s = 0.0f;
                int first = 1;
                for (int b = 0; b < 4; b++)
                    for (int a = 0; a < 4; a++) {
                        float num = 1.0f;
                        int den = 1;
                        int firstf = 1;
                        for (int m = 0; m < 4; m++)
                            if (m != b) {
                                float t = (float)xs[m] - posx;
                                num = firstf ? t : num * t;
                                firstf = 0;
                                den *= xs[m] - xs[b];
                            }
                        for (int m = 0; m < 4; m++)
                            if (m != a) {
                                num = num * ((float)ys[m] - posy);
                                den *= ys[m] - ys[a];
                            }
                        float term = (num / (float)den) * v[a][b];
                        s = first ? term : s + term;
                        first = 0;
                    }
                if (s > maxx) { maxx = s; bestpos = i * di; }
            }
        if (bestpos > (float)sizex / 2.0f) bestpos -= (float)sizex;
        result = (double)(-bestpos / 2.0f);
    }
#undef ABS2
    free(F); free(G); free(re); free(im);
    return result;
}

/* getRotAxisCorrection (rotation_axis.cu:455-526): rows edge-padded to Np = 3N,
 * R2C, times exp(-i 2 pi / (2M - 2) offset k) with M = Np/2 + 1 (the Nyquist bin
 * of an even Np keeps only the real part, as C2R reads it), C2R, / Np, centre crop. */
void oracle_rotaxis(const float *tomo, int nrays, int nrows, float offset, double *out)
{
    int pad = 2, Np = nrays * (1 + pad), off = (pad * nrays) / 2, M = Np / 2 + 1;
    cplx *H = (cplx *)malloc(sizeof(cplx) * Np);
    for (int k = 0; k < Np; k++) {
        int kk = k <= Np / 2 ? k : Np - k;
        double ph = 2.0 * PI_D / (double)(2 * M - 2) * (double)offset * kk;
        double re = cos(ph), im = -sin(ph);
        if (k > Np / 2) im = -im;
        if (Np % 2 == 0 && k == Np / 2) im = 0.0;
        H[k] = (re + I * im) / (double)Np;
    }
    cplx *rf = make_roots(Np, -1), *ri = make_roots(Np, +1);
#pragma omp parallel
    {
        double *row = (double *)malloc(sizeof(double) * Np);
        cplx *a = (cplx *)malloc(sizeof(cplx) * Np), *b = (cplx *)malloc(sizeof(cplx) * Np);
        cplx *scratch = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * Np + 8));
#pragma omp for
        for (int r = 0; r < nrows; r++) {
            pad_row(tomo + (size_t)r * nrays, nrays, pad, Np, row);
            for (int i = 0; i < Np; i++) a[i] = row[i];
            fft(Np, a, b, rf, scratch);
            for (int k = 0; k < Np; k++) b[k] *= H[k];
            fft(Np, b, a, ri, scratch);
            for (int i = 0; i < nrays; i++) out[(size_t)r * nrays + i] = creal(a[off + i]);
        }
        free(row); free(a); free(b); free(scratch);
    }
    free(H); free(rf); free(ri);
}


/* Fourier-slice projection of one N x N slice into counts (pst_counts_real,
 * radon_fst.cu:544-637): fftshift, corners of an L x L zero grid, 2-D FFT,
 * fftshift; per angle the polar samples (cos t, sin t) (r - L/2), nearest
 * (interp 0, round half to even) or the reference's bilinear variant (1);
 * fftshift, 1-D inverse FFT (unnormalised), fftshift, centre N, times scale;
 * counts = flat where p < 0, else flat exp(-p).  cs / sn: the cosine and sine
 * the reference computes (GPU fast intrinsics, given as data). */
static void fst_counts(const double *x, int N, int A, int L, int interp, float scale, const float *cs,
                       const float *sn, const float *flat, double *counts, const cplx *rfwdL, const cplx *rinvL)
{
    cplx *W = (cplx *)calloc((size_t)L * L, sizeof(cplx));
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            int r = j < N / 2 ? j : j + L - N, c = i < N / 2 ? i : i + L - N;
            W[(size_t)r * L + c] = x[(size_t)((j + N / 2) % N) * N + (i + N / 2) % N];
        }
    fft2_inplace(W, L, L, -1);
    const long long LL = (long long)L * L;
#define SPEC(idx) W[(size_t)(((long long)(idx) / L + L / 2) % L) * L + (size_t)((((long long)(idx) % L) + L / 2) % L)]
#pragma omp parallel
    {
        cplx *h = (cplx *)malloc(sizeof(cplx) * L), *H = (cplx *)malloc(sizeof(cplx) * L);
        cplx *scratch = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * L + 8));
#pragma omp for schedule(dynamic, 4)
        for (int a = 0; a < A; a++) {
            for (int q = 0; q < L; q++) {
                int r = (q + L / 2) % L;
                float rho = (float)((double)r - (double)L / 2.0);
                float xpos = cs[a] * rho, ypos = sn[a] * rho;
                cplx v = 0;
                if (interp == 0) {
                    long long xi = (long long)rintf(xpos) + L / 2, yi = (long long)rintf(ypos) + L / 2;
                    long long idx = yi * L + xi;
                    if (idx < LL) v = SPEC(idx);
                } else {
                    long long xd = (long long)floorf(xpos) + L / 2, xu = (long long)ceilf(xpos) + L / 2;
                    long long yd = (long long)floorf(ypos) + L / 2, yu = (long long)ceilf(ypos) + L / 2;
                    cplx fdd = SPEC(yd * L + xd), fdu = SPEC(yu * L + xd);
                    cplx fud = SPEC(yd * L + xu), fuu = SPEC(yu * L + xu);
                    float xd_pos = (float)xd - L / 2, xu_pos = (float)xu - L / 2;
                    float yd_pos = (float)yd - L / 2, yu_pos = (float)yu - L / 2;
                    if (xd == xu && yd == yu) v = fdd;
                    else if (xd == xu) v = (double)(yu_pos - ypos) * fdd + (double)(ypos - yd_pos) * fuu;
                    else if (yd == yu) v = (double)(xu_pos - xpos) * fdd + (double)(xpos - xd_pos) * fuu;
                    else
                        v = (double)(yu_pos - ypos) * ((double)(xu_pos - xpos) * fdd + (double)(xpos - xd_pos) * fud) +
                            (double)(ypos - yd_pos) * ((double)(xu_pos - xpos) * fdu + (double)(xpos - xd_pos) * fuu);
                }
                h[q] = v;
            }
            fft(L, h, H, rinvL, scratch);
            for (int i = 0; i < N; i++) {
                double p = creal(H[((L - N) / 2 + i + L / 2) % L]) * (double)scale;
                counts[(size_t)a * N + i] = p < 0 ? flat[i] : flat[i] * exp(-p);
            }
        }
        free(h); free(H); free(scratch);
    }
#undef SPEC
    free(W);
    (void)rfwdL;
}

/* tEMFQ (get_tEM_FQ, em_frequency.cu:13-87): backcounts = 1 / BST(counts);
 * niter times: model = FST(x); x <- x * (BST(model) * backcounts).  The BST
 * here is EMFQ_BST (bst.cu:100-249): no filter and no padding of the rows,
 * half-rays N/2 zero-padded to N (zpad+1)/2 with weight (zpad+1)^2, an N x N
 * grid, scale 1.  obj: initial guess in, result out ([B][N][N], FP64). */
void oracle_temfq(const float *counts, const float *flat, const float *cs, const float *sn, int N, int A, int B,
                  int zpad, int interp, int niter, float dx, double *obj)
{
    const int L = N * (1 + zpad), pad0 = zpad + 1, Lb = N * pad0 / 2;
    const float scale = dx > 0.f ? dx / (float)L : (float)(1.0 / (float)L);
    cplx *rfL = make_roots(L, -1), *riL = make_roots(L, +1);
    cplx *rfLb = make_roots(Lb, -1), *riN = make_roots(N, +1);
    double *rows = (double *)malloc(sizeof(double) * (size_t)A * N);
    double *inv = (double *)malloc(sizeof(double) * (size_t)N * N);
    double *back = (double *)malloc(sizeof(double) * (size_t)N * N);
    double *model = (double *)malloc(sizeof(double) * (size_t)A * N);
    for (int z = 0; z < B; z++) {
        double *x = obj + (size_t)z * N * N;
        const float *fl = flat + (size_t)z * N;
        for (size_t i = 0; i < (size_t)A * N; i++) rows[i] = counts[(size_t)z * A * N + i];
        bst_slice(rows, A, N, Lb, N, 0, N, (double)(pad0 * pad0), 1.0f, inv, rfLb, riN);
        for (size_t i = 0; i < (size_t)N * N; i++) inv[i] = 1.0 / inv[i];
        for (int k = 0; k < niter; k++) {
            fst_counts(x, N, A, L, interp, scale, cs, sn, fl, model, rfL, riL);
            bst_slice(model, A, N, Lb, N, 0, N, (double)(pad0 * pad0), 1.0f, back, rfLb, riN);
            for (size_t i = 0; i < (size_t)N * N; i++) x[i] *= back[i] * inv[i];
        }
    }
    free(rows); free(inv); free(back); free(model);
    free(rfL); free(riL); free(rfLb); free(riN);
}
