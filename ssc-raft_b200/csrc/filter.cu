// filter.cu -- the FBP row filter and the lowpass filter.
//
// Reference behaviour (cnpem/ssc-raft):
//   * rows are edge-replicated from N to Np = N*(1+pad) bins with a left offset
//     of pad*N/2 (cuda/src/common/padding.cu:140-178);
//   * each padded row goes through a real FFT, is multiplied by
//     w(k) * exp(-i*2*pi*offset*k/(2M-2)) with the tent weight
//     w = Filter::apply(0.5*min(k, M-k)/M), M = Np/2+1
//     (cuda/src/processing/filters/filters.cu:33-51,395-438), inverse FFT,
//     then divided by Np*pixel (filters.cu:163-190);
//   * filter type 'none' skips the filter and the scaling (fbp.cu:102-103).
//
// B200 design: one CTA filters two rows at once as the real and imaginary
// parts of a single complex sequence (the full-length filter spectrum is
// Hermitian, so the two filtered rows come back as the real and imaginary
// parts of the inverse transform).  Padding, the forward FFT, the spectral
// multiply (weight, axis-shift phase, normalisation), the inverse FFT, the
// angle-step weight and the output packing for the backprojector all happen
// in one kernel with the row held in shared memory.  The FFT is a
// self-sorting (Stockham) mixed-radix transform with radices 2,3,4,5,7,8
// whose twiddles come from an FP64-built table; lengths with a larger prime
// factor use a direct circular-convolution kernel instead.  No cuFFT.
#include "raft.hpp"
#include "profile.hpp"
#include "fft.cuh"

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

namespace raft {

// ============================================================ host: spectrum
static double ref_apply(int type, double w, double paganin, double reg)
{
    // Filter::apply, filters.cu:395-438 (input is the tent weight)
    const double pg = 1.0 / (1.0 + paganin * w * w);
    switch (type) {
    case FILTER_GAUSSIAN: return w * std::exp(-0.693 * reg * w * w) * pg;
    case FILTER_LORENTZ: return w * (1.0 / (1.0 + reg * w * w)) * pg;
    case FILTER_COSINE: return w * std::cos(M_PI * 0.5 * w) * pg;
    case FILTER_RECTANGLE: {
        double param = std::fmax(w * reg * M_PI * 0.5, 1e-4);
        return w * (std::sin(param) / param) * pg;
    }
    case FILTER_HANN: return w * (0.5 + 0.5 * std::cos(2.0 * M_PI * w)) * pg;
    case FILTER_HAMMING: return w * (0.54 + 0.46 * std::cos(2.0 * M_PI * w)) * pg;
    case FILTER_RAMP: return w * pg;
    // 1/(2*pi*SIGN(w)); the reference's SIGN(0)=0 makes the DC weight infinite,
    // here the DC weight is taken as 0.
    case FILTER_DIFFERENTIAL: return w > 0 ? 1.0 / (2.0 * M_PI) : 0.0;
    default: return w * pg;  // Shepp-Logan has no reference counterpart: tent
    }
}

double filter_apply_ref(int type, double w, double paganin, double reg)
{
    return ref_apply(type, w, paganin, reg);
}

static double lin_apply(int type, double nu, double paganin, double reg)
{
    // true ramp |k|/Np = nu/2 (nu = 1 at Nyquist) times a window of nu
    const double ramp = 0.5 * nu;
    const double pg = 1.0 / (1.0 + paganin * nu * nu);
    switch (type) {
    case FILTER_GAUSSIAN: return ramp * std::exp(-0.693 * reg * nu * nu) * pg;
    case FILTER_LORENTZ: return ramp / (1.0 + reg * nu * nu) * pg;
    case FILTER_COSINE: return ramp * std::cos(0.5 * M_PI * nu) * pg;
    case FILTER_RECTANGLE: {
        double param = std::fmax(nu * reg * M_PI * 0.5, 1e-4);
        return ramp * (std::sin(param) / param) * pg;
    }
    case FILTER_HANN: return ramp * 0.5 * (1.0 + std::cos(M_PI * nu)) * pg;
    case FILTER_HAMMING: return ramp * (0.54 + 0.46 * std::cos(M_PI * nu)) * pg;
    case FILTER_RAMP: return ramp * pg;
    case FILTER_DIFFERENTIAL: return nu > 0 ? 1.0 / (2.0 * M_PI) : 0.0;
    case FILTER_SHEPP_LOGAN: {
        double a = 0.5 * M_PI * nu;
        return ramp * (a > 0 ? std::sin(a) / a : 1.0) * pg;
    }
    default: return ramp * pg;
    }
}

void filter_spectrum_host(int geometry, int ftype, int Np, double paganin, double reg,
                          double offset, double pixel, double *hre, double *him)
{
    const int M = Np / 2 + 1;
    const double norm = 1.0 / ((double)Np * pixel);
    for (int k = 0; k < Np; k++) {
        const int kk = (k <= Np / 2) ? k : Np - k;
        double w, phase;
        if (geometry == GEOM_FBP_LIN) {
            w = lin_apply(ftype, 2.0 * kk / (double)Np, paganin, reg);
            phase = 2.0 * M_PI * offset * kk / (double)Np;
        } else if (ftype == FILTER_AXIS_SHIFT) {
            // rot_axis_correction_kernel (rotation_axis.cu:455-465): pure phase,
            // the same 2M-2 denominator; the inverse is divided by Np only
            w = pixel;
            phase = 2.0 * M_PI / (double)(2 * M - 2) * offset * kk;
        } else {
            const double tent = 0.5 * std::fmin((double)kk, (double)(M - kk)) / (double)M;
            w = ref_apply(ftype, tent, paganin, reg);
            // filters.cu:46 uses the denominator 2M-2 (= Np for even Np)
            phase = 2.0 * M_PI / (double)(2 * M - 2) * offset * kk;
        }
        double re = w * std::cos(phase), im = -w * std::sin(phase);
        if (k > Np / 2) im = -im;                  // Hermitian extension
        if (Np % 2 == 0 && k == Np / 2) im = 0.0;  // C2R ignores Im of the Nyquist bin
        hre[k] = re * norm;
        him[k] = im * norm;
    }
}

// ============================================================== host: plan
constexpr size_t kFilterSmemMax = 220 * 1024;

bool build_filter_plan(FilterPlan &plan, int geometry, int ftype, int N, int pad, double paganin,
                       double reg, double offset, double pixel, int device)
{
    (void)device;
    plan.N = N;
    plan.pad = pad;
    plan.Np = N * (1 + pad);
    plan.off = (pad * N) / 2;
    const int Np = plan.Np;
    plan.skip = (ftype == FILTER_NONE);
    if (plan.skip) return true;

    const size_t smem = 2 * (size_t)fft_span(Np) * sizeof(float2);   // ping-pong buffers
    plan.fft = factorize(Np, plan.radix, plan.nradix) && smem <= kFilterSmemMax;
    plan.threads = fft_threads(Np);
    std::vector<double> hre(Np), him(Np);
    filter_spectrum_host(geometry, ftype, Np, paganin, reg, offset, pixel, hre.data(), him.data());
    if (plan.fft) {
        std::vector<float2> H(Np), tw(Np);
        for (int k = 0; k < Np; k++) {
            H[k] = make_float2((float)hre[k], (float)him[k]);
            double a = -2.0 * M_PI * (double)k / (double)Np;
            tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        RAFT_CUDA(cudaMalloc(&plan.d_H, sizeof(float2) * Np));
        RAFT_CUDA(cudaMalloc(&plan.d_tw, sizeof(float2) * Np));
        RAFT_CUDA(cudaMemcpy(plan.d_H, H.data(), sizeof(float2) * Np, cudaMemcpyHostToDevice));
        RAFT_CUDA(cudaMemcpy(plan.d_tw, tw.data(), sizeof(float2) * Np, cudaMemcpyHostToDevice));
    } else {
        // impulse response h[m] = (1/Np) sum_k H[k] exp(+2 pi i k m / Np) (real)
        std::vector<float> h(Np);
        for (int m = 0; m < Np; m++) {
            double acc = 0.0;
            for (int k = 0; k < Np; k++) {
                double a = 2.0 * M_PI * (double)(((long long)k * m) % Np) / (double)Np;
                acc += hre[k] * std::cos(a) - him[k] * std::sin(a);
            }
            h[m] = (float)acc;  // H already carries 1/Np
        }
        RAFT_CUDA(cudaMalloc(&plan.d_h, sizeof(float) * Np));
        RAFT_CUDA(cudaMemcpy(plan.d_h, h.data(), sizeof(float) * Np, cudaMemcpyHostToDevice));
    }
    return true;
}

void release_filter_plan(FilterPlan &plan)
{
    if (plan.d_H) cudaFree(plan.d_H);
    if (plan.d_tw) cudaFree(plan.d_tw);
    if (plan.d_h) cudaFree(plan.d_h);
    plan.d_H = plan.d_tw = nullptr;
    plan.d_h = nullptr;
}

// ===================================================== device: output pack
struct PackArgs {
    void *out;
    const float *wt;
    int nangles, wlo, Wg, store, Np;
};

__device__ __forceinline__ float row_value(const float2 *z, int u, int Np, int part)
{
    if (u < 0 || u >= Np) return 0.f;
    float2 c = z[u];
    return part == 0 ? c.x : -c.y;
}

// Write window row `row` (part 0: real part, 1: negated imaginary part) of the
// filtered padded row held in z, scaled by the angle weight.
__device__ __forceinline__ void pack_row(const float2 *z, int row, int part, const PackArgs &a)
{
    const float w = a.wt ? a.wt[row % a.nangles] : 1.f;
    const size_t rb = (size_t)row * a.Wg;
    for (int e = threadIdx.x; e < a.Wg; e += blockDim.x) {
        const int u = a.wlo + e;
        const float v0 = row_value(z, u, a.Np, part) * w;
        if (a.store == STORE_F32) {
            reinterpret_cast<float *>(a.out)[rb + e] = v0;
        } else {
            const float v1 = row_value(z, u + 1, a.Np, part) * w;
            const float mid = 0.5f * (v0 + v1), dif = v1 - v0;
            if (a.store == STORE_PAIR_F32)
                reinterpret_cast<float2 *>(a.out)[rb + e] = make_float2(mid, dif);
            else
                reinterpret_cast<__nv_bfloat162 *>(a.out)[rb + e] = __floats2bfloat162_rn(mid, dif);
        }
    }
}

// ================================================== kernel: FFT filter
// two CTAs per SM (registers capped at 64: two 512-thread CTAs, or 384 + 384)
__global__ void __launch_bounds__(512, 2)
filter_fft_kernel(const float *__restrict__ sino, int N, int Np, int off, int nrows,
                  const float2 *__restrict__ H, const float2 *__restrict__ tw, RadixList rl,
                  PackArgs pk, int skip, float *lowpass_out)
{
    extern __shared__ float2 smem_fft[];
    float2 *z = smem_fft;
    float2 *zb = smem_fft + fft_span(Np);
    const int r0 = 2 * blockIdx.x, r1 = r0 + 1;
    const bool has1 = r1 < nrows;
    const float *s0 = sino + (size_t)r0 * N;
    const float *s1 = sino + (size_t)r1 * N;
    // edge-replicating pad (padding.cu:140-178) of both rows into one complex row
    for (int n = threadIdx.x; n < Np; n += blockDim.x) {
        int i = n - off;
        i = i < 0 ? 0 : (i > N - 1 ? N - 1 : i);
        z[n] = make_float2(__ldg(&s0[i]), has1 ? __ldg(&s1[i]) : 0.f);
    }
    __syncthreads();
    if (!skip) {
        z = fft_forward(z, zb, Np, rl, tw);
        // spectral multiply, then conjugate so that a second forward FFT
        // yields the conjugated inverse transform
        for (int k = threadIdx.x; k < Np; k += blockDim.x) {
            float2 g = cmul(z[k], __ldg(&H[k]));
            z[k] = make_float2(g.x, -g.y);
        }
        __syncthreads();
        zb = (z == smem_fft) ? smem_fft + fft_span(Np) : smem_fft;
        z = fft_forward(z, zb, Np, rl, tw);
    } else {
        // no transform: match the conjugation convention of pack_row
        for (int k = threadIdx.x; k < Np; k += blockDim.x) z[k].y = -z[k].y;
        __syncthreads();
    }
    if (lowpass_out) {
        // lowpass (low_pass.cu / filterFBPpad): centre crop back to N bins
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            float2 c = z[off + i];
            lowpass_out[(size_t)r0 * N + i] = c.x;
            if (has1) lowpass_out[(size_t)r1 * N + i] = -c.y;
        }
        return;
    }
    pack_row(z, r0, 0, pk);
    if (has1) pack_row(z, r1, 1, pk);
}

// ============================================ kernel: direct convolution
// Any Np (used when Np has a prime factor > 7 or does not fit shared memory).
__global__ void __launch_bounds__(256)
filter_direct_kernel(const float *__restrict__ sino, int N, int Np, int off, int nrows,
                     const float *__restrict__ h, PackArgs pk, int skip, float *lowpass_out)
{
    extern __shared__ float2 z[];   // z[u].x = padded row, then filtered value
    float *p = reinterpret_cast<float *>(z + Np);  // Np floats
    const int row = blockIdx.x;
    const float *s = sino + (size_t)row * N;
    for (int n = threadIdx.x; n < Np; n += blockDim.x) {
        int i = n - off;
        i = i < 0 ? 0 : (i > N - 1 ? N - 1 : i);
        p[n] = __ldg(&s[i]);
    }
    __syncthreads();
    for (int u = threadIdx.x; u < Np; u += blockDim.x) {
        float acc;
        if (skip) {
            acc = p[u];
        } else {
            acc = 0.f;
            int d = u;  // (u - m) mod Np for m = 0
            for (int m = 0; m < Np; m++) {
                acc = fmaf(p[m], __ldg(&h[d]), acc);
                d = (d == 0) ? Np - 1 : d - 1;
            }
        }
        z[u] = make_float2(acc, 0.f);
    }
    __syncthreads();
    if (lowpass_out) {
        for (int i = threadIdx.x; i < N; i += blockDim.x) lowpass_out[(size_t)row * N + i] = z[off + i].x;
        return;
    }
    pack_row(z, row, 0, pk);
}

void launch_filter(const FilterPlan &plan, const FilterLaunch &fl, cudaStream_t st)
{
    PackArgs pk;
    pk.out = fl.out;
    pk.wt = fl.wt;
    pk.nangles = fl.nangles;
    pk.wlo = fl.wlo;
    pk.Wg = fl.Wg;
    pk.store = fl.store;
    pk.Np = plan.Np;
    float *lp = fl.out_padded ? reinterpret_cast<float *>(fl.out) : nullptr;
    if (fl.nrows <= 0) return;
    if (plan.fft || plan.skip) {
        RadixList rl;
        rl.n = plan.skip ? 0 : plan.nradix;
        for (int i = 0; i < rl.n; i++) rl.r[i] = plan.radix[i];
        const int T = plan.skip ? 256 : plan.threads;
        const size_t smem = 2 * (size_t)fft_span(plan.Np) * sizeof(float2);
        static thread_local int configured_dev = -1;
        int dev = 0;
        cudaGetDevice(&dev);
        if (configured_dev != dev) {
            RAFT_CUDA(cudaFuncSetAttribute(filter_fft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kFilterSmemMax));
            RAFT_CUDA(cudaFuncSetAttribute(filter_fft_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
            configured_dev = dev;
        }
        ProfScope ps(PROF_FILTER, st);
        filter_fft_kernel<<<(fl.nrows + 1) / 2, T, smem, st>>>(
            fl.sino, plan.N, plan.Np, plan.off, fl.nrows, plan.d_H, plan.d_tw, rl, pk,
            plan.skip ? 1 : 0, lp);
    } else {
        const size_t smem = (size_t)plan.Np * (sizeof(float2) + sizeof(float));
        RAFT_CHECK(smem <= kFilterSmemMax, "filter: padded row too long for the direct filter");
        RAFT_CUDA(cudaFuncSetAttribute(filter_direct_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kFilterSmemMax));
        ProfScope ps(PROF_FILTER, st);
        filter_direct_kernel<<<fl.nrows, 256, smem, st>>>(fl.sino, plan.N, plan.Np, plan.off, fl.nrows,
                                                          plan.d_h, pk, 0, lp);
    }
    RAFT_CUDA(cudaGetLastError());
}

}  // namespace raft

namespace raft {

// Shape of an FFT filter plan (length, radix passes, CTA size) without
// allocating anything; returns false when the padded length needs the
// direct-convolution path.  Used by the no-allocation FBP entry point.
bool filter_plan_shape(FilterPlan &plan, int ftype, int N, int pad)
{
    plan.N = N;
    plan.pad = pad;
    plan.Np = N * (1 + pad);
    plan.off = (pad * N) / 2;
    plan.skip = (ftype == FILTER_NONE);
    plan.threads = fft_threads(plan.Np);
    plan.fft = factorize(plan.Np, plan.radix, plan.nradix) &&
               2 * (size_t)fft_span(plan.Np) * sizeof(float2) <= kFilterSmemMax;
    return plan.skip || plan.fft;
}

}  // namespace raft
