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

#include <cooperative_groups.h>

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
static int cluster_size_for(int Np, int *radix, int &nradix);

bool build_filter_plan(FilterPlan &plan, int geometry, int ftype, int N, int pad, double paganin,
                       double reg, double offset, double pixel, int device)
{
    plan.N = N;
    plan.pad = pad;
    plan.Np = N * (1 + pad);
    plan.off = (pad * N) / 2;
    const int Np = plan.Np;
    plan.skip = (ftype == FILTER_NONE);
    plan.cluster = 0;
    if (plan.skip) {
        // pad + copy only; rows beyond one CTA's shared memory go through the cluster kernel
        if (2 * (size_t)fft_span(Np) * sizeof(float2) > kFilterSmemMax)
            plan.cluster = cluster_size_for(Np, plan.radix, plan.nradix);
        return true;
    }

    const size_t smem = 2 * (size_t)fft_span(Np) * sizeof(float2);   // ping-pong buffers
    plan.fft = factorize(Np, plan.radix, plan.nradix) && smem <= kFilterSmemMax;
    plan.threads = fft_threads(Np);
    plan.bs_M = 0;
    if (!plan.fft) {
        // too long for one CTA: a cluster of CTAs, m = Np / C points each
        plan.cluster = cluster_size_for(Np, plan.radix, plan.nradix);
        plan.fft = plan.cluster > 0;
    }
    if (!plan.fft) {
        // a prime factor above 7: Bluestein's algorithm (two M-point transforms
        // per direction) when its buffers fit one CTA, else direct convolution
        const int M = fft_plan_length(Np);
        if (M > 0 && 2 * (size_t)fft_span(M) * sizeof(float2) <= kFilterSmemMax) {
            const FftTable &t = fft_table(device, Np);
            plan.bs_M = M;
            plan.bs_chirp = t.plan.chirp;
            plan.bs_B = t.plan.B;
            plan.nradix = t.plan.rl.n;
            for (int i = 0; i < plan.nradix; i++) plan.radix[i] = t.plan.rl.r[i];
            plan.threads = fft_threads(M);
            plan.fft = 1;
        }
    }
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
    int il;        // 1: rows interleaved by slice in groups of four ([group][angle][Wg][4], 4-byte elements)
};

// Rows are filtered in pairs of neighbouring angles of one slice (the real and
// imaginary parts of one complex transform); a slice with an odd number of
// angles ends with a single row.  Pairs never mix slices, so a slice's result
// does not depend on the batch it came in.  For interleaved output the four
// slices of a group are the four fastest-varying CTAs, so the stores that
// fill each 16-byte element of the output arrive together.
struct RowPair {
    int k, a0;      // slice, first angle (a0 + 1 is the second row when it exists)
};
__device__ __forceinline__ RowPair row_pair(int p, int nangles, int il)
{
    const int PA = (nangles + 1) / 2;
    RowPair rp;
    if (il) {
        const int rest = p >> 2;
        rp.k = 4 * (rest / PA) + (p & 3);
        rp.a0 = 2 * (rest % PA);
    } else {
        rp.k = p / PA;
        rp.a0 = 2 * (p % PA);
    }
    return rp;
}
// Row pairs (CTAs) one filter launch over nslices slices runs.
static inline long long row_pairs(int nslices, int nangles, int il)
{
    const long long PA = (nangles + 1) / 2;
    return il ? (long long)((nslices + 3) / 4) * 4 * PA : (long long)nslices * PA;
}

// Index of window element e of (slice k, angle a) in the output rows.
__device__ __forceinline__ size_t out_index(const PackArgs &a, int k, int ang, int e)
{
    return a.il ? (((size_t)(k >> 2) * a.nangles + ang) * a.Wg + e) * 4 + (k & 3)
                : ((size_t)k * a.nangles + ang) * a.Wg + e;
}

__device__ __forceinline__ float row_value(const float2 *z, int u, int Np, int part)
{
    if (u < 0 || u >= Np) return 0.f;
    float2 c = z[u];
    return part == 0 ? c.x : -c.y;
}

// Store window element e of (slice k, angle ang) from the filtered samples
// v0 = row[u], v1 = row[u + 1] (already weighted).
__device__ __forceinline__ void store_elem(const PackArgs &a, int k, int ang, int e, float v0, float v1)
{
    const size_t o = out_index(a, k, ang, e);
    if (a.store == STORE_F32) {
        reinterpret_cast<float *>(a.out)[o] = v0;
    } else {
        const float mid = 0.5f * (v0 + v1), dif = v1 - v0;
        if (a.store == STORE_PAIR_F32)
            reinterpret_cast<float2 *>(a.out)[o] = make_float2(mid, dif);
        else
            reinterpret_cast<__nv_bfloat162 *>(a.out)[o] = __floats2bfloat162_rn(mid, dif);
    }
}

// Write the window row of (slice k, angle ang) (part 0: real part, 1: negated
// imaginary part) of the filtered padded row held in z, scaled by the angle weight.
__device__ __forceinline__ void pack_row(const float2 *z, int k, int ang, int part, const PackArgs &a)
{
    const float w = a.wt ? a.wt[ang] : 1.f;
    for (int e = threadIdx.x; e < a.Wg; e += blockDim.x) {
        const int u = a.wlo + e;
        const float v0 = row_value(z, u, a.Np, part) * w;
        const float v1 = a.store == STORE_F32 ? 0.f : row_value(z, u + 1, a.Np, part) * w;
        store_elem(a, k, ang, e, v0, v1);
    }
}

// Zero window rows of a slice beyond the batch (interleaved output only: the
// group's 16-byte elements are read whole).
__device__ __forceinline__ void zero_rows(int k, int a0, const PackArgs &a)
{
    for (int ang = a0; ang < min(a0 + 2, a.nangles); ang++)
        for (int e = threadIdx.x; e < a.Wg; e += blockDim.x) store_elem(a, k, ang, e, 0.f, 0.f);
}

// ================================================== kernel: FFT filter
// two CTAs per SM (registers capped at 64: two 512-thread CTAs, or 384 + 384)
__global__ void __launch_bounds__(512, 2)
filter_fft_kernel(const float *__restrict__ sino, int N, int Np, int off, int nslices,
                  const float2 *__restrict__ H, FftPlan P, PackArgs pk, int skip, float *lowpass_out)
{
    extern __shared__ float2 smem_fft[];
    float2 *z = smem_fft;
    float2 *zb = smem_fft + fft_plan_span(P);
    const RowPair rp = row_pair(blockIdx.x, pk.nangles, pk.il);
    if (rp.k >= nslices) {
        zero_rows(rp.k, rp.a0, pk);
        return;
    }
    const int r0 = rp.k * pk.nangles + rp.a0, r1 = r0 + 1;
    const bool has1 = rp.a0 + 1 < pk.nangles;
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
        z = fft_run(z, zb, P);
        // spectral multiply, then conjugate so that a second forward FFT
        // yields the conjugated inverse transform
        for (int k = threadIdx.x; k < Np; k += blockDim.x) {
            float2 g = cmul(z[k], __ldg(&H[k]));
            z[k] = make_float2(g.x, -g.y);
        }
        __syncthreads();
        zb = (z == smem_fft) ? smem_fft + fft_plan_span(P) : smem_fft;
        z = fft_run(z, zb, P);
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
    pack_row(z, rp.k, rp.a0, 0, pk);
    if (has1) pack_row(z, rp.k, rp.a0 + 1, 1, pk);
}

// ====================================== kernel: FFT filter, fixed length
// The same filter for the common padded lengths, with the transform length a
// compile-time constant (cfft_passes): the first forward pass reads the two
// sinogram rows straight from global memory (edge-replicating pad included),
// the spectral multiply and conjugation sit in the last forward pass, and for
// single-float window rows the last inverse pass stores the window elements
// from registers (other row formats go through shared memory and pack_row).
// Bit for bit the results of filter_fft_kernel.
template <int NP, int R0>
struct FxRowsIn {
    const float *s0, *s1;
    int N, off;
    bool has1;
    __device__ __forceinline__ float2 operator()(int j, int it, int r) const
    {
        (void)it;
        int i = j + r * (NP / R0) - off;
        i = i < 0 ? 0 : (i > N - 1 ? N - 1 : i);
        return make_float2(__ldg(&s0[i]), has1 ? __ldg(&s1[i]) : 0.f);
    }
};
template <int R, int NS>
struct FxSpecOut {
    float2 *d;
    const float2 *H;
    __device__ __forceinline__ void operator()(int q, int k, const float2 (&v)[R]) const
    {
        (void)q;   // the last pass: NS R = NP, q = 0
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int i = k + r * NS;
            const float2 g = cmul(v[r], __ldg(&H[i]));
            d[i] = make_float2(g.x, -g.y);
        }
    }
};
struct FxSpecLast {
    float2 *d;
    const float2 *H;
    template <int R, int NS> __device__ __forceinline__ FxSpecOut<R, NS> at() const { return {d, H}; }
};
// window element e = u - wlo of both rows, from filtered sample u (registers)
struct FxWindow {
    float *out;
    size_t base0, base1;   // element 0 of the two window rows
    int stride, wlo, Wg;
    float w0, w1;
    bool has1;
};
template <int R, int NS>
struct FxWinOut {
    FxWindow w;
    __device__ __forceinline__ void operator()(int q, int k, const float2 (&v)[R]) const
    {
        (void)q;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int e = k + r * NS - w.wlo;
            if ((unsigned)e < (unsigned)w.Wg) {
                w.out[w.base0 + (size_t)e * w.stride] = v[r].x * w.w0;
                if (w.has1) w.out[w.base1 + (size_t)e * w.stride] = (-v[r].y) * w.w1;
            }
        }
    }
};
struct FxWinLast {
    FxWindow w;
    template <int R, int NS> __device__ __forceinline__ FxWinOut<R, NS> at() const { return {w}; }
};

// CTAs per SM the launch bounds ask for: as many as shared memory and the
// thread limit allow, but no fewer than 64 registers per thread.
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int fixed_filter_min_blocks(int NP)
{
    return cmin(cmin((220 * 1024) / (2 * fft_span(NP) * 8), 2048 / c_fft_threads(NP)),
                65536 / (64 * c_fft_threads(NP))) < 1
               ? 1
               : cmin(cmin((220 * 1024) / (2 * fft_span(NP) * 8), 2048 / c_fft_threads(NP)),
                      65536 / (64 * c_fft_threads(NP)));
}

template <int NP, bool IL, bool FUSED>
__global__ void __launch_bounds__(c_fft_threads(NP), fixed_filter_min_blocks(NP))
filter_fixed_kernel(const float *__restrict__ sino, int N, int off, int nslices, const float2 *__restrict__ H,
                    PackArgs pk)
{
    constexpr CRadices rl = c_factorize(NP);
    constexpr int T = c_fft_threads(NP);
    extern __shared__ float2 smem_fft[];
    float2 *A = smem_fft, *B = smem_fft + fft_span(NP);
    const RowPair rp = row_pair(blockIdx.x, pk.nangles, IL);
    if (rp.k >= nslices) {
        zero_rows(rp.k, rp.a0, pk);
        return;
    }
    const int r0 = rp.k * pk.nangles + rp.a0, r1 = r0 + 1;
    const bool has1 = rp.a0 + 1 < pk.nangles;
    // forward transform of the two edge-padded rows, times H, conjugated
    const FxRowsIn<NP, rl.r[0]> rows{sino + (size_t)r0 * N, sino + (size_t)r1 * N, N, off, has1};
    float2 *X = cfft_out_buffer<NP>() ? B : A, *Y = (X == A) ? B : A;
    cfft_passes<NP, 0, 1>(A, B, rows, FxSpecLast{X, H});
    __syncthreads();
    // inverse transform (forward transform of the conjugate; conjugated on output)
    const CSmemIn<NP, T, rl.r[0], false> spec(X);
    if constexpr (FUSED) {
        FxWindow w;
        w.out = reinterpret_cast<float *>(pk.out);
        w.stride = IL ? 4 : 1;
        w.base0 = IL ? ((size_t)(rp.k >> 2) * pk.nangles + rp.a0) * pk.Wg * 4 + (rp.k & 3)
                     : ((size_t)rp.k * pk.nangles + rp.a0) * pk.Wg;
        w.base1 = w.base0 + (size_t)pk.Wg * w.stride;
        w.wlo = pk.wlo;
        w.Wg = pk.Wg;
        w.w0 = pk.wt ? pk.wt[rp.a0] : 1.f;
        w.w1 = (pk.wt && has1) ? pk.wt[rp.a0 + 1] : 1.f;
        w.has1 = has1;
        cfft_passes<NP, 0, 1>(X, Y, spec, FxWinLast{w});
        // window elements outside the padded row
        const int lo = min(pk.Wg, max(0, -pk.wlo)), hi = max(0, NP - pk.wlo);
        for (int e = threadIdx.x; e < pk.Wg; e += T) {
            if (e >= lo && e < hi) continue;
            w.out[w.base0 + (size_t)e * w.stride] = 0.f * w.w0;
            if (has1) w.out[w.base1 + (size_t)e * w.stride] = 0.f * w.w1;
        }
    } else {
        float2 *Z = cfft_out_buffer<NP>() ? Y : X;
        cfft_passes<NP, 0, 1>(X, Y, spec, CPlainLast{Z});
        __syncthreads();
        pack_row(Z, rp.k, rp.a0, 0, pk);
        if (has1) pack_row(Z, rp.k, rp.a0 + 1, 1, pk);
    }
}

static bool g_fixed_filter = true;
bool fixed_transforms_enabled() { return g_fixed_filter; }

template <int NP, bool IL, bool FUSED>
static void launch_fixed_one(const FilterPlan &plan, const FilterLaunch &fl, const PackArgs &pk, int nsl,
                             cudaStream_t st)
{
    static thread_local int configured_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = 2 * (size_t)fft_span(NP) * sizeof(float2);
    if (configured_dev != dev) {
        RAFT_CUDA(cudaFuncSetAttribute(filter_fixed_kernel<NP, IL, FUSED>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        RAFT_CUDA(cudaFuncSetAttribute(filter_fixed_kernel<NP, IL, FUSED>,
                                       cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        configured_dev = dev;
    }
    ProfScope ps(PROF_FILTER, st);
    filter_fixed_kernel<NP, IL, FUSED><<<(unsigned)row_pairs(nsl, fl.nangles, IL), c_fft_threads(NP), smem, st>>>(
        fl.sino, plan.N, plan.off, nsl, plan.d_H, pk);
}

template <int NP>
static void launch_fixed_np(const FilterPlan &plan, const FilterLaunch &fl, const PackArgs &pk, int nsl,
                            cudaStream_t st)
{
    const bool f32 = fl.store == STORE_F32;
    if (fl.interleaved) {
        if (f32) launch_fixed_one<NP, true, true>(plan, fl, pk, nsl, st);
        else launch_fixed_one<NP, true, false>(plan, fl, pk, nsl, st);
    } else {
        if (f32) launch_fixed_one<NP, false, true>(plan, fl, pk, nsl, st);
        else launch_fixed_one<NP, false, false>(plan, fl, pk, nsl, st);
    }
}

// Runs the fixed-length filter when one is compiled for plan.Np.
static bool launch_fixed_filter(const FilterPlan &plan, const FilterLaunch &fl, const PackArgs &pk, int nsl,
                                cudaStream_t st)
{
    if (!g_fixed_filter) return false;
    switch (plan.Np) {
    case 1024: launch_fixed_np<1024>(plan, fl, pk, nsl, st); return true;
    case 1536: launch_fixed_np<1536>(plan, fl, pk, nsl, st); return true;
    case 2048: launch_fixed_np<2048>(plan, fl, pk, nsl, st); return true;
    case 3072: launch_fixed_np<3072>(plan, fl, pk, nsl, st); return true;
    case 4096: launch_fixed_np<4096>(plan, fl, pk, nsl, st); return true;
    case 6144: launch_fixed_np<6144>(plan, fl, pk, nsl, st); return true;
    case 8192: launch_fixed_np<8192>(plan, fl, pk, nsl, st); return true;
    case 12288: launch_fixed_np<12288>(plan, fl, pk, nsl, st); return true;
    default: return false;
    }
}

// ============================================ kernel: cluster FFT filter
// Padded rows too long for one CTA's shared memory (two ping-pong buffers of
// Np complex values) are filtered by a cluster of C CTAs (thread-block
// cluster, distributed shared memory), each holding m = Np / C values, with a
// four-step decomposition Np = m * C that needs only two exchanges between
// the CTAs:
//   forward  X[k1 + m k2] = sum_i2 W_C^(i2 k2) W_Np^(i2 k1) FFT_m(x[C i1 + i2])[k1]
//   inverse  (a forward transform of the conjugate, conjugated)
//            y[C i1 + i2] = FFT_m over k1 of W_Np^(i2 k1) sum_k2 W_C^(i2 k2) X'[k1 + m k2]
// CTA rank r holds the row in the strided order x[C i1 + r] (i1 < m), so the
// m-point transforms are local; the C-point transforms of the middle step run
// in registers, one k1 per thread over this CTA's block of k1, reading the C
// values from the C CTAs' shared memory; the spectral multiply (weight,
// axis-shift phase, normalisation) sits between the forward and the inverse
// C-point transforms in the same registers.  The results are bit-for-bit
// independent of which CTA computed them, but not of C: a row is filtered
// identically by every launch of the same length.
template <int C>
__device__ __forceinline__ void small_dft(float2 (&v)[C])
{
    if constexpr (C == 2 || C == 3 || C == 4 || C == 5 || C == 7 || C == 8) {
        Dft<C>::run(v);
    } else {
        float2 in[C];
#pragma unroll
        for (int r = 0; r < C; r++) in[r] = v[r];
#pragma unroll
        for (int q = 0; q < C; q++) {
            float2 acc = in[0];
#pragma unroll
            for (int r = 1; r < C; r++) {
                float sn, cs;
                sincospif(-2.0f * (float)((r * q) % C) / (float)C, &sn, &cs);
                acc = cadd(acc, cmul(in[r], make_float2(cs, sn)));
            }
            v[q] = acc;
        }
    }
}

// exp(-2 pi i e / n) for an integer exponent 0 <= e < n
__device__ __forceinline__ float2 root_of_unity(int e, int n)
{
    float sn, cs;
    sincospif(-2.0f * (float)e / (float)n, &sn, &cs);
    return make_float2(cs, sn);
}

// Elements of one of the cluster kernel's two buffers: the m-point transform's
// span, and at least the C * ceil(m / C) values of the middle step.
__host__ __device__ inline int cluster_span(int m, int C) { return max(fft_span(m), C * ((m + C - 1) / C)); }

template <int C>
__global__ void __launch_bounds__(512)
filter_fft_cluster_kernel(const float *__restrict__ sino, int N, int Np, int off, int nslices,
                          const float2 *__restrict__ H, RadixList rl, PackArgs pk, int skip, float *lowpass_out)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int m = Np / C, T = blockDim.x, tid = threadIdx.x;
    extern __shared__ float2 smem_fft[];
    float2 *bufA = smem_fft, *bufB = smem_fft + cluster_span(m, C);
    const RowPair rp = row_pair(blockIdx.x / C, pk.nangles, pk.il);
    if (rp.k >= nslices) {        // the whole cluster: no cluster barrier is reached
        if (rank == 0) zero_rows(rp.k, rp.a0, pk);
        return;
    }
    const int r0 = rp.k * pk.nangles + rp.a0, r1 = r0 + 1;
    const bool has1 = rp.a0 + 1 < pk.nangles;
    const float *s0 = sino + (size_t)r0 * N;
    const float *s1 = sino + (size_t)r1 * N;
    // edge-replicating pad (padding.cu:140-178), this CTA's strided share
    for (int i1 = tid; i1 < m; i1 += T) {
        int i = C * i1 + rank - off;
        i = i < 0 ? 0 : (i > N - 1 ? N - 1 : i);
        bufA[i1] = make_float2(__ldg(&s0[i]), has1 ? __ldg(&s1[i]) : 0.f);
    }
    __syncthreads();
    float2 *R = bufA;
    if (skip) {
        // no transform: match the conjugation convention of the output step
        for (int i1 = tid; i1 < m; i1 += T) bufA[i1].y = -bufA[i1].y;
    } else {
    float2 *Y = fft_forward(bufA, bufB, m, rl, nullptr);   // plain order, same buffer in every CTA
    float2 *Wb = (Y == bufA) ? bufB : bufA;
    cl.sync();
    // middle step for this CTA's block of k1: gather the C values, forward
    // C-point DFT (with the W_Np^(i2 k1) twiddles), spectral multiply and
    // conjugation, C-point DFT and twiddles of the inverse
    const int kb = (m + C - 1) / C, k1s = rank * kb, k1e = min(m, k1s + kb);
    for (int k1 = k1s + tid; k1 < k1e; k1 += T) {
        float2 v[C];
#pragma unroll
        for (int i2 = 0; i2 < C; i2++) {
            const float2 y = cl.map_shared_rank(Y, i2)[k1];
            v[i2] = i2 ? cmul(y, root_of_unity(i2 * k1, Np)) : y;
        }
        small_dft<C>(v);
#pragma unroll
        for (int k2 = 0; k2 < C; k2++) {
            const float2 g = cmul(v[k2], __ldg(&H[k1 + m * k2]));
            v[k2] = make_float2(g.x, -g.y);
        }
        small_dft<C>(v);
#pragma unroll
        for (int i2 = 0; i2 < C; i2++)
            Wb[(k1 - k1s) * C + i2] = i2 ? cmul(v[i2], root_of_unity(i2 * k1, Np)) : v[i2];
    }
    cl.sync();
    // this CTA's i2 = rank: its values of every k1, from the CTA owning the k1
    for (int k1 = tid; k1 < m; k1 += T) {
        const int own = k1 / kb;
        Y[k1] = cl.map_shared_rank(Wb, own)[(k1 - own * kb) * C + rank];
    }
    cl.sync();   // every CTA has read the Wb buffers before they are overwritten
    R = fft_forward(Y, Wb, m, rl, nullptr);            // conj of the filtered row, strided order
    }
    cl.sync();
    // output: element u of the filtered row sits in CTA u % C at u / C
    auto at = [&](int u) -> float2 {
        return cl.map_shared_rank(R, u % C)[u / C];
    };
    if (lowpass_out) {
        const int ib = (N + C - 1) / C;
        for (int i = rank * ib + tid; i < min(N, (rank + 1) * ib); i += T) {
            const float2 c = at(off + i);
            lowpass_out[(size_t)r0 * N + i] = c.x;
            if (has1) lowpass_out[(size_t)r1 * N + i] = -c.y;
        }
    } else {
        const int eb = (pk.Wg + C - 1) / C;
        const int e0 = rank * eb, e1 = min(pk.Wg, e0 + eb);
        for (int part = 0; part < (has1 ? 2 : 1); part++) {
            const int ang = rp.a0 + part;
            const float w = pk.wt ? pk.wt[ang] : 1.f;
            for (int e = e0 + tid; e < e1; e += T) {
                const int u = pk.wlo + e;
                auto val = [&](int v) -> float {
                    if (v < 0 || v >= Np) return 0.f;
                    const float2 c = at(v);
                    return (part == 0 ? c.x : -c.y) * w;
                };
                store_elem(pk, rp.k, ang, e, val(u), pk.store == STORE_F32 ? 0.f : val(u + 1));
            }
        }
    }
    cl.sync();   // keep this CTA's shared memory until every CTA has read it
}

// Smallest cluster size C (2..8) for which Np = m * C with m a transform
// length of the shared-memory FFT whose two buffers fit one CTA; 0 if none.
static int cluster_size_for(int Np, int *radix, int &nradix)
{
    for (int C = 2; C <= 8; C++) {
        if (Np % C) continue;
        const int m = Np / C;
        if (2 * (size_t)cluster_span(m, C) * sizeof(float2) > kFilterSmemMax) continue;
        if (factorize(m, radix, nradix)) return C;
    }
    return 0;
}

template <int C>
static void launch_cluster_filter(const FilterPlan &plan, const FilterLaunch &fl, const PackArgs &pk, float *lp,
                                  cudaStream_t st)
{
    const int m = plan.Np / C;
    const size_t smem = 2 * (size_t)cluster_span(m, C) * sizeof(float2);
    RadixList rl;
    rl.n = plan.nradix;
    for (int i = 0; i < rl.n; i++) rl.r[i] = plan.radix[i];
    RAFT_CUDA(cudaFuncSetAttribute(filter_fft_cluster_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kFilterSmemMax));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(C * row_pairs(fl.nrows / fl.nangles, fl.nangles, pk.il)));
    cfg.blockDim = dim3((unsigned)fft_threads(m));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ProfScope ps(PROF_FILTER, st);
    RAFT_CUDA(cudaLaunchKernelEx(&cfg, filter_fft_cluster_kernel<C>, fl.sino, plan.N, plan.Np, plan.off,
                                 fl.nrows / fl.nangles,
                                 (const float2 *)plan.d_H, rl, pk, plan.skip ? 1 : 0, lp));
}

// ============================================ kernel: direct convolution
// Any Np (used when Np has a prime factor > 7 or does not fit shared memory).
__global__ void __launch_bounds__(256)
filter_direct_kernel(const float *__restrict__ sino, int N, int Np, int off, int nslices,
                     const float *__restrict__ h, PackArgs pk, int skip, float *lowpass_out)
{
    extern __shared__ float2 z[];   // z[u].x = padded row, then filtered value
    float *p = reinterpret_cast<float *>(z + Np);  // Np floats
    // one row per CTA; for interleaved output the group's four slices run side by side
    int k, ang;
    if (pk.il) {
        const int rest = blockIdx.x >> 2;
        k = 4 * (rest / pk.nangles) + (blockIdx.x & 3);
        ang = rest % pk.nangles;
    } else {
        k = blockIdx.x / pk.nangles;
        ang = blockIdx.x % pk.nangles;
    }
    if (k >= nslices) {
        for (int e = threadIdx.x; e < pk.Wg; e += blockDim.x) store_elem(pk, k, ang, e, 0.f, 0.f);
        return;
    }
    const int row = k * pk.nangles + ang;
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
    pack_row(z, k, ang, 0, pk);
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
    pk.il = fl.interleaved;
    float *lp = fl.out_padded ? reinterpret_cast<float *>(fl.out) : nullptr;
    if (fl.nrows <= 0) return;
    RAFT_CHECK(fl.nangles > 0 && fl.nrows % fl.nangles == 0, "filter: rows must be whole slices of nangles rows");
    RAFT_CHECK(!fl.interleaved || (!lp && store_bytes(fl.store) == 4),
               "filter: interleaved output takes 4-byte window elements");
    const int nsl = fl.nrows / fl.nangles;
    if (plan.cluster) {
        switch (plan.cluster) {
        case 2: launch_cluster_filter<2>(plan, fl, pk, lp, st); break;
        case 3: launch_cluster_filter<3>(plan, fl, pk, lp, st); break;
        case 4: launch_cluster_filter<4>(plan, fl, pk, lp, st); break;
        case 5: launch_cluster_filter<5>(plan, fl, pk, lp, st); break;
        case 6: launch_cluster_filter<6>(plan, fl, pk, lp, st); break;
        case 7: launch_cluster_filter<7>(plan, fl, pk, lp, st); break;
        default: launch_cluster_filter<8>(plan, fl, pk, lp, st); break;
        }
        return;
    }
    if (plan.fft && !plan.skip && !lp && plan.bs_M <= 0 && launch_fixed_filter(plan, fl, pk, nsl, st)) {
        RAFT_CUDA(cudaGetLastError());
        return;
    }
    if (plan.fft || plan.skip) {
        FftPlan P;
        P.n = plan.Np;
        P.M = plan.bs_M > 0 ? plan.bs_M : plan.Np;
        P.rl.n = plan.skip ? 0 : plan.nradix;
        for (int i = 0; i < P.rl.n; i++) P.rl.r[i] = plan.radix[i];
        P.chirp = plan.bs_chirp;
        P.B = plan.bs_B;
        const int T = plan.skip ? 256 : plan.threads;
        const size_t smem = 2 * (size_t)fft_plan_span(P) * sizeof(float2);
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
        filter_fft_kernel<<<(unsigned)row_pairs(nsl, fl.nangles, pk.il), T, smem, st>>>(
            fl.sino, plan.N, plan.Np, plan.off, nsl, plan.d_H, P, pk, plan.skip ? 1 : 0, lp);
    } else {
        const size_t smem = (size_t)plan.Np * (sizeof(float2) + sizeof(float));
        RAFT_CHECK(smem <= kFilterSmemMax, "filter: padded row too long for the direct filter");
        RAFT_CUDA(cudaFuncSetAttribute(filter_direct_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kFilterSmemMax));
        ProfScope ps(PROF_FILTER, st);
        const unsigned rows = (unsigned)(pk.il ? (long long)((nsl + 3) / 4) * 4 * fl.nangles : fl.nrows);
        filter_direct_kernel<<<rows, 256, smem, st>>>(fl.sino, plan.N, plan.Np, plan.off, nsl, plan.d_h, pk, 0,
                                                      lp);
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

extern "C" {
// 1 (default): transforms of 1024, 1536, 2048, 3072, 4096, 6144, 8192 and 12288 points
// (FBP filter rows, BST) run the compile-time-length kernels; 0: every length
// runs the generic ones.
int raft_filter_set_fixed(int on)
{
    raft::g_fixed_filter = on != 0;
    return 0;
}
}
