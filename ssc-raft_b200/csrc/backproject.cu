// backproject.cu -- the backprojector for FBP and for the EM iterations.
//
// Reference kernels restated (cnpem/ssc-raft):
//   * FBP  BackProjection_SS, cuda/src/geometries/parallel/reconstruction_methods/fbp.cu:8-76
//     x = xmin + i*dx, t = x*cos - y*sin, sample = sino[(int)((t - tmin)/dt)]
//     on the padded (N*(1+pad))^2 grid, then the centre N x N is cropped
//     (padding.cu:245-268).  Here only the centre window is computed; for
//     those pixels the arithmetic is identical.
//   * EM   kernel_backprojection / kernel_backprojectionWithUpdate,
//     cuda/src/geometries/parallel/reconstruction_methods/kernels/em_RT_kernel.cu:92-142,249-300
//     x = -1 + i*2/(N-1), t = x*cos + y*sin, T = (int)((t + 1)/dt),
//     optional update x <- x * BP / den.
//   * FBP with linear interpolation (north-star operator): same pixel and
//     detector grid, the sample at fractional bin u = (t - tmin)/dt is
//     interpolated between bins floor(u) and floor(u)+1 (zero outside).
//
// B200 design.  A CTA owns a 64 x 32 pixel tile of one slice (256 threads,
// 8 pixels per thread spread so that every warp touches an 8 x 4 pixel
// block -> one shared-memory wavefront per gather).  Angles stream through a
// two-stage pipeline of 32-angle blocks: for every angle, warp 0 computes the
// detector window the tile can reach and one lane issues a 1-D bulk copy
// (cp.async.bulk, the TMA engine) of that window from the filtered rows in
// HBM/L2 into shared memory, completing on an mbarrier; while block s is
// gathered, block s+1 is in flight.  The filtered rows already carry the
// angle step, so the inner loop is: position, round, gather, interpolate,
// accumulate.  All waits are bounded and report through a device flag.
#include "raft.hpp"
#include "ptx.hpp"
#include "profile.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace raft {

struct __align__(16) AngleParam {
    float a, b, c;
    int d;
};

struct BpArgs {
    const unsigned char *filt;   // window rows [nslices*nangles][Wg] elements
    float *img;                  // [nslices][No][No]
    const float *den;            // update denominator (EM), same layout as img
    int No, nangles, nslices;
    int wlo, Wg, W, esize;
    // FBP reference arithmetic
    float xmin, ymin, dx, dy, tmin, dt;
    int offo;
    // EM reference arithmetic
    float xymin, dxy;
    // linear geometry
    double c0, ratio, u0;
    const float *cs, *sn;        // FP32 tables (fast intrinsics, as the reference)
    const double *csd, *snd;     // FP64 tables
    int *err;
    int update;                  // 0: store, 1: img = img * acc / den
    int il;                      // 1: filt holds groups of 4 slices interleaved, [group][angle][Wg][4 elements]
};

constexpr uint32_t kWaitLimit = 1u << 24;
constexpr int kParamBytes = 2 * 32 * (int)sizeof(AngleParam);   // two stages of at most 32 angles
constexpr int kWinOffset = 128 + kParamBytes;   // bytes before the windows

static_assert(kWinOffset % 128 == 0, "window area alignment");

// ------------------------------------------------------------------------
// per-angle window base (warp 0, one lane per angle)
// ------------------------------------------------------------------------
template <int GEOM>
__device__ __forceinline__ void angle_param(const BpArgs &p, int a, int x0, int y0, AngleParam &ap, int &base)
{
    const int align = 16 / p.esize;
    int lo;
    if constexpr (GEOM == GEOM_FBP_LIN) {
        const double c = p.csd[a], s = -p.snd[a] * p.ratio;
        const double v00 = ((double)x0 + p.c0) * c + ((double)y0 + p.c0) * s + p.u0;
        const double vmin = v00 + fmin(0.0, (BP_TX - 1) * c) + fmin(0.0, (BP_TY - 1) * s);
        lo = (int)floor(vmin) - 1;
        int b = lo - ((lo % align) + align) % align;
        b = max(0, min(b, p.Wg - p.W));
        base = b;
        ap.a = (float)(v00 - (double)b);
        ap.b = (float)c;
        ap.c = (float)s;
        ap.d = b;
    } else {
        const float c = p.cs[a], s = p.sn[a];
        int tmin_i = 0x7fffffff;
#pragma unroll
        for (int cy = 0; cy < 2; cy++)
#pragma unroll
            for (int cx = 0; cx < 2; cx++) {
                const int i = x0 + cx * (BP_TX - 1), j = y0 + cy * (BP_TY - 1);
                int ti;
                // the corner bins need not match bp_tile's per-pixel rounding
                // exactly: the window starts one bin below the lowest corner
                if constexpr (GEOM == GEOM_FBP_REF) {
                    const int ip = i + p.offo, jp = j + p.offo;
                    float x = p.xmin + ip * p.dx;
                    float y = p.ymin + jp * p.dy;
                    float t = x * c - y * s;
                    ti = (int)((t - p.tmin) / p.dt);
                } else {
                    float x = p.xymin + i * p.dxy;
                    float y = p.xymin + j * p.dxy;
                    float t = x * c + y * s;
                    ti = (int)((t - p.tmin) / p.dt);
                }
                tmin_i = min(tmin_i, ti);
            }
        lo = tmin_i - 1 - p.wlo;
        int b = lo - ((lo % align) + align) % align;
        b = max(0, min(b, p.Wg - p.W));
        base = b;
        ap.a = c;
        ap.b = s;
        ap.c = 0.f;
        ap.d = p.wlo + b;   // padded-bin index of window element 0
    }
}

// ------------------------------------------------------------------------
// element fetch
// ------------------------------------------------------------------------
template <int STORE>
__device__ __forceinline__ float lerp_fetch(const unsigned char *w, int k, float f)
{
    if constexpr (STORE == STORE_PAIR_F32) {
        const float2 sd = reinterpret_cast<const float2 *>(w)[k];
        return fmaf(f, sd.y, sd.x);
    } else {
        const uint32_t bits = reinterpret_cast<const uint32_t *>(w)[k];
        const float mid = __uint_as_float(bits << 16);
        const float dif = __uint_as_float(bits & 0xffff0000u);
        return fmaf(f, dif, mid);
    }
}

// ------------------------------------------------------------------------
// kernel
//
// S slices share one CTA: the per-pixel position, rounding and window index
// are computed once per (pixel, angle) and reused for every slice, whose
// windows sit side by side in shared memory ([angle][slice][W]).  With IL
// (S = 4) the rows arrive interleaved by slice ([group][angle][Wg][4
// elements], see interleave4_kernel), the staged windows are [angle][W][4]
// and one 16-byte load (two for f32 pairs) fetches the sample of all four
// slices: one bulk copy per angle instead of four, one or two shared-memory
// instructions per (pixel, angle) instead of four.  AB (angles per pipeline stage) is a launch
// parameter; S and AB are chosen by the autotuner below.
// ------------------------------------------------------------------------
// One 64 x 32 tile of S slices.  `gstage` counts the pipeline stages this
// CTA has consumed so far (a persistent CTA runs many tiles through the same
// two buffers and mbarriers); returns false if a staging wait timed out.
template <int GEOM, int STORE, int S, bool IL = false>
__device__ __forceinline__ bool bp_tile(const BpArgs &p, const int AB, const int x0, const int y0,
                                        const int slice0, unsigned char *smem, uint32_t &gstage)
{
    static_assert(!IL || S == 4, "interleaved rows: four slices per CTA");
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    AngleParam *prm = reinterpret_cast<AngleParam *>(smem + 128);
    unsigned char *win = smem + kWinOffset;
    constexpr int esize = (STORE == STORE_PAIR_F32) ? 8 : 4;
    const int W = p.W;
    const int wbytes = W * esize;                // one window
    const int stage_bytes = AB * S * wbytes;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nsl = min(S, p.nslices - slice0);  // valid slices of this CTA
    const int A = p.nangles;
    const int nst = (A + AB - 1) / AB;

    // thread -> pixels: warp covers an 8 x 4 block per (i, j)
    const int lx = lane & 7, ly = lane >> 3;
    const int wx = warp & 1, wy = warp >> 1;
    int li[4], lj[2];
#pragma unroll
    for (int i = 0; i < 4; i++) li[i] = wx * 32 + lx + 8 * i;
#pragma unroll
    for (int j = 0; j < 2; j++) lj[j] = wy * 8 + ly + 4 * j;

    const unsigned char *rows = IL ? p.filt + (size_t)(slice0 / 4) * A * p.Wg * (4 * esize)
                                   : p.filt + (size_t)slice0 * A * p.Wg * esize;
    const size_t slice_stride = (size_t)A * p.Wg * esize;

    auto issue = [&](int s, int b) {
        // warp 0 only: one window base per angle, then one bulk copy per (angle, slice)
        const int a0 = s * AB;
        const int na = min(AB, A - a0);
        if (lane < na) {
            AngleParam ap;
            int base;
            angle_param<GEOM>(p, a0 + lane, x0, y0, ap, base);
            prm[b * 32 + lane] = ap;
        }
        if (lane == 0) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&bars[b], (uint32_t)(na * (IL ? S : nsl) * wbytes));
        }
        __syncwarp();
        unsigned char *dst = win + (size_t)b * stage_bytes;
        if constexpr (IL) {
            // one copy of the four interleaved windows per angle
            for (int al = lane; al < na; al += 32) {
                const int base = prm[b * 32 + al].d - (GEOM == GEOM_FBP_LIN ? 0 : p.wlo);
                bulk_g2s(dst + (size_t)al * S * wbytes, rows + ((size_t)(a0 + al) * p.Wg + base) * (4 * esize),
                         (uint32_t)(S * wbytes), &bars[b]);
            }
        } else {
            for (int c = lane; c < na * nsl; c += 32) {
                const int al = c / nsl, sl = c - al * nsl;
                const int base = prm[b * 32 + al].d - (GEOM == GEOM_FBP_LIN ? 0 : p.wlo);
                bulk_g2s(dst + (size_t)(al * S + sl) * wbytes,
                         rows + sl * slice_stride + ((size_t)(a0 + al) * p.Wg + base) * esize, (uint32_t)wbytes,
                         &bars[b]);
            }
        }
    };

    if (warp == 0) issue(0, gstage & 1);
    __syncthreads();

    float acc[S][2][4];
#pragma unroll
    for (int q = 0; q < S; q++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int i = 0; i < 4; i++) acc[q][j][i] = 0.f;
    // Interleaved bf16 pairs: slices (0, 1) and (2, 3) accumulate as pairs
    // with the packed two-lane FP32 instructions (each lane rounds as the
    // scalar instruction does, so the sums are the same bits as acc's).  The
    // nearest f32 kernel, bound by the shared-memory pipe, measured 2 %
    // slower with them and keeps scalar adds.
    constexpr bool PK = IL && STORE == STORE_PAIR_BF16;
    float2 accp[2][2][4];
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int i = 0; i < 4; i++) accp[h][j][i] = make_float2(0.f, 0.f);

    // per-thread coordinates in the reference's float arithmetic
    float xr[4], yr[2];
    if constexpr (GEOM == GEOM_FBP_REF) {
#pragma unroll
        for (int i = 0; i < 4; i++) xr[i] = __fmaf_rn((float)(x0 + li[i] + p.offo), p.dx, p.xmin);
#pragma unroll
        for (int j = 0; j < 2; j++) yr[j] = __fmaf_rn((float)(y0 + lj[j] + p.offo), p.dy, p.ymin);
    } else if constexpr (GEOM == GEOM_EM_REF) {
#pragma unroll
        for (int i = 0; i < 4; i++) xr[i] = __fmaf_rn((float)(x0 + li[i]), p.dxy, p.xymin);
#pragma unroll
        for (int j = 0; j < 2; j++) yr[j] = __fmaf_rn((float)(y0 + lj[j]), p.dxy, p.xymin);
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++) xr[i] = (float)li[i];
#pragma unroll
        for (int j = 0; j < 2; j++) yr[j] = (float)lj[j];
    }

    bool ok = true;
    for (int s = 0; s < nst && ok; s++) {
        const uint32_t g = gstage + s;
        const int b = g & 1;
        if (s + 1 < nst && warp == 0) issue(s + 1, b ^ 1);
        // bounded wait; the CTA agrees on the outcome at the end of the stage
        const bool got = mbar_wait_bounded(&bars[b], (g >> 1) & 1, kWaitLimit);
        const int na = min(AB, A - s * AB);
        const unsigned char *wb = win + (size_t)b * stage_bytes;
        const AngleParam *pb = prm + b * 32;
        for (int al = 0; al < na; al++) {
            const AngleParam ap = pb[al];
            const unsigned char *w = wb + (size_t)al * S * wbytes;
            if constexpr (GEOM == GEOM_FBP_LIN) {
                const float MAGIC = 12582912.0f;   // 1.5 * 2^23: fadd rounds to an integer
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const float vrow = fmaf(yr[j], ap.c, ap.a);
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float v = fmaf(xr[i], ap.b, vrow);
                        const float m = __fadd_rn(v, MAGIC);
                        const unsigned k = min((unsigned)(__float_as_int(m) - 0x4B400000), (unsigned)(W - 1));
                        const float f = __fsub_rn(v, __fsub_rn(m, MAGIC));
                        if constexpr (IL && STORE == STORE_PAIR_F32) {
                            // bin k: (mid, dif) of slices 0..3 in 32 bytes
                            const float4 u0 = reinterpret_cast<const float4 *>(w)[2 * k];
                            const float4 u1 = reinterpret_cast<const float4 *>(w)[2 * k + 1];
                            acc[0][j][i] += fmaf(f, u0.y, u0.x);
                            acc[1][j][i] += fmaf(f, u0.w, u0.z);
                            acc[2][j][i] += fmaf(f, u1.y, u1.x);
                            acc[3][j][i] += fmaf(f, u1.w, u1.z);
                        } else if constexpr (IL) {
                            // bin k: bf16 (mid, dif) pairs of slices 0..3 in 16 bytes;
                            // value = mid + f dif per slice, two slices per instruction
                            const uint4 u = reinterpret_cast<const uint4 *>(w)[k];
                            const float2 ff = make_float2(f, f);
                            const float2 mid01 = make_float2(__uint_as_float(u.x << 16), __uint_as_float(u.y << 16));
                            const float2 dif01 = make_float2(__uint_as_float(u.x & 0xffff0000u),
                                                             __uint_as_float(u.y & 0xffff0000u));
                            const float2 mid23 = make_float2(__uint_as_float(u.z << 16), __uint_as_float(u.w << 16));
                            const float2 dif23 = make_float2(__uint_as_float(u.z & 0xffff0000u),
                                                             __uint_as_float(u.w & 0xffff0000u));
                            accp[0][j][i] = __fadd2_rn(accp[0][j][i], __ffma2_rn(ff, dif01, mid01));
                            accp[1][j][i] = __fadd2_rn(accp[1][j][i], __ffma2_rn(ff, dif23, mid23));
                        } else {
                            const unsigned char *wk = w + (size_t)k * esize;
#pragma unroll
                            for (int q = 0; q < S; q++)
                                acc[q][j][i] += lerp_fetch<STORE>(wk + q * wbytes, 0, f);
                        }
                    }
                }
            } else {
                const float c = ap.a, sn = ap.b;
                const int wbase = ap.d;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    // FBP: t = x*cos - y*sin, EM: t = x*cos + y*sin, each one fmaf
                    // with y*sin rounded first (the reference build's contraction)
                    const float ys = (GEOM == GEOM_FBP_REF) ? -__fmul_rn(yr[j], sn) : __fmul_rn(yr[j], sn);
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float t = __fmaf_rn(xr[i], c, ys);
                        int ti = (int)((t - p.tmin) / p.dt);
                        const unsigned k = min((unsigned)(ti - wbase), (unsigned)(W - 1));
                        if constexpr (IL) {
                            const float4 v = reinterpret_cast<const float4 *>(w)[k];
                            acc[0][j][i] += v.x;
                            acc[1][j][i] += v.y;
                            acc[2][j][i] += v.z;
                            acc[3][j][i] += v.w;
                        } else {
                            const float *wk = reinterpret_cast<const float *>(w) + k;
#pragma unroll
                            for (int q = 0; q < S; q++) acc[q][j][i] += wk[q * W];
                        }
                    }
                }
            }
        }
        if (!__syncthreads_and(got)) {
            ok = false;
            if (tid == 0 && p.err) atomicExch(p.err, 1);
            // give copies still in flight a last bounded chance to land
            mbar_wait_bounded(&bars[b], (g >> 1) & 1, kWaitLimit);
        }
    }
    gstage += nst;
    if (!ok) return false;

#pragma unroll
    for (int q = 0; q < S; q++) {
        if (q >= nsl) break;
        float *out = p.img + (size_t)(slice0 + q) * p.No * p.No;
        const float *den = p.den ? p.den + (size_t)(slice0 + q) * p.No * p.No : nullptr;
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int X = x0 + li[i], Y = y0 + lj[j];
                if (X < p.No && Y < p.No) {
                    const size_t o = (size_t)Y * p.No + X;
                    const float a = PK ? ((q & 1) ? accp[q >> 1][j][i].y : accp[q >> 1][j][i].x) : acc[q][j][i];
                    if (p.update) out[o] = out[o] * a / den[o];
                    else out[o] = a;
                }
            }
    }
    return true;
}


template <int GEOM, int STORE, int S, bool IL = false>
__device__ __forceinline__ void bp_body(const BpArgs &p, const int AB)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t gstage = 0;
    bp_tile<GEOM, STORE, S, IL>(p, AB, blockIdx.x * BP_TX, blockIdx.y * BP_TY, blockIdx.z * S, smem, gstage);
}

template <int GEOM, int STORE, int S>
__global__ void __launch_bounds__(BP_THREADS) bp_kernel(const BpArgs p, const int AB)
{
    bp_body<GEOM, STORE, S>(p, AB);
}

// The S = 4 instance, held to 80 registers so that three CTAs fit an SM
// (its shared memory allows three).
template <int GEOM, int STORE, bool IL>
__global__ void __launch_bounds__(BP_THREADS, 3) bp_kernel_s4(const BpArgs p, const int AB)
{
    bp_body<GEOM, STORE, 4, IL>(p, AB);
}

// Window rows [nslices][nangles][Wg] of 4-byte (E = uint32_t: f32, bf16 pair) or
// 8-byte (E = uint2: f32 pair) elements -> [ceil(nslices/4)][nangles][Wg][4],
// slices beyond nslices zero; a bit copy, one CTA per (group, angle) row.
template <typename E>
__global__ void interleave4_kernel(const E *__restrict__ rows, E *__restrict__ out, int nslices, int A, int Wg)
{
    const int r = blockIdx.x, g = r / A, a = r - g * A;
    const E *src[4];
#pragma unroll
    for (int q = 0; q < 4; q++) src[q] = 4 * g + q < nslices ? rows + ((size_t)(4 * g + q) * A + a) * Wg : nullptr;
    E *dst = out + (size_t)r * Wg * 4;
    E zero;
    memset(&zero, 0, sizeof(E));
    for (int e = threadIdx.x; e < Wg; e += blockDim.x) {
#pragma unroll
        for (int q = 0; q < 4; q++) dst[4 * e + q] = src[q] ? __ldcs(src[q] + e) : zero;
    }
}

// ------------------------------------------------------------------------
// Ragged persistent backprojector: many requests (different image sizes,
// angle counts, windows) in one launch.  Work items (request, tile, slice
// group) are numbered request by request; each CTA takes the next item from
// an atomic counter until none are left.  When a request's last item
// finishes, its completion time (%globaltimer, ns) is recorded.
// ------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int GEOM, int STORE, int S>
__global__ void __launch_bounds__(BP_THREADS)
bp_ragged_kernel(const BpArgs *__restrict__ reqs, const int *__restrict__ item_start, int nreq, int total,
                 const int AB, int *queue, int *remaining, unsigned long long *t_done)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    __shared__ int s_item, s_req;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t gstage = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const int it = atomicAdd(queue, 1);
            int r = 0;
            if (it < total)
                while (r + 1 < nreq && item_start[r + 1] <= it) r++;
            s_item = it;
            s_req = r;
        }
        __syncthreads();
        const int it = s_item, r = s_req;
        if (it >= total) break;
        const BpArgs &p = reqs[r];
        const int local = it - item_start[r];
        const int tx = (p.No + BP_TX - 1) / BP_TX, ty = (p.No + BP_TY - 1) / BP_TY;
        const int bx = local % tx, by = (local / tx) % ty, bz = local / (tx * ty);
        const bool ok = bp_tile<GEOM, STORE, S>(p, AB, bx * BP_TX, by * BP_TY, bz * S, smem, gstage);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicSub(&remaining[r], 1) == 1 && t_done) t_done[r] = global_ns();
        }
        if (!ok) break;   // uniform: bp_tile's outcome is agreed by the whole CTA
    }
}

// ------------------------------------------------------------------------
// Self test of the bounded staging wait: one thread waits on an mbarrier that
// is arrived on (arrive = 1) or that nothing ever arrives on (arrive = 0); a
// wait that runs out after `limit` polls sets the flag, as the staging
// pipeline does, and the kernel returns.
// ------------------------------------------------------------------------
__global__ void bounded_wait_selftest_kernel(int arrive, unsigned limit, int *err)
{
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_mbar_init();
    if (arrive) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&bar)) : "memory");
    if (!mbar_wait_bounded(&bar, 0, limit)) atomicExch(err, 1);
}

int selftest_bounded_wait(int gpu, int arrive, unsigned limit)
{
    RAFT_CUDA(cudaSetDevice(gpu));
    int *d_err = nullptr;
    RAFT_CUDA(cudaMalloc(&d_err, sizeof(int)));
    int h = -1;
    cudaError_t e = cudaMemset(d_err, 0, sizeof(int));
    if (e == cudaSuccess) {
        count_launch();
        bounded_wait_selftest_kernel<<<1, 32>>>(arrive, limit, d_err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    RAFT_CUDA(e);
    return h;
}

// ------------------------------------------------------------------------
// angle tables: the reference computes sin/cos with the fast intrinsics,
// __sinf/__cosf for FBP (opt.cu:187-194) and __sincosf for EM
// (em_RT_kernel.cu:120); angle steps as em_RT_kernel.cu:122-126 / fbp.cu:61-64.
// ------------------------------------------------------------------------
__global__ void angle_table_kernel(const float *angles, int A, float *cs, float *sn, float *wt, int em)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A) return;
    if (em) {
        float s, c;
        __sincosf(angles[k], &s, &c);
        cs[k] = c;
        sn[k] = s;
    } else {
        sn[k] = __sinf(angles[k]);
        cs[k] = __cosf(angles[k]);
    }
    if (wt) {
        float d;
        if (A == 1) d = 1.0f;
        else if (k == A - 1) d = angles[k] - angles[k - 1];
        else d = angles[k + 1] - angles[k];
        // FBP angular correction for scans beyond pi (fbp.cu:24-28); EM has none
        float scale = 1.0f;
        if (!em && angles[A - 1] > float(M_PI)) scale = float(M_PI) / angles[A - 1];
        wt[k] = d * scale;
    }
}

void launch_angle_tables(const float *d_angles, int nangles, float *d_cos, float *d_sin, float *d_wt,
                         int em_sincos, cudaStream_t st)
{
    count_launch();
    angle_table_kernel<<<(nangles + 127) / 128, 128, 0, st>>>(d_angles, nangles, d_cos, d_sin, d_wt,
                                                               em_sincos);
    RAFT_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------------
// host: window planning and launch
// ------------------------------------------------------------------------
static int floor_to(int v, int a) { return v - (((v % a) + a) % a); }
static int ceil_to(int v, int a) { return floor_to(v + a - 1, a); }

WindowLayout plan_window(const BpPlanInput &in)
{
    WindowLayout L;
    const int esize = store_bytes(in.store);
    const int align = 16 / esize;
    L.align = align;
    const int Xext = ((in.No + BP_TX - 1) / BP_TX) * BP_TX;
    const int Yext = ((in.No + BP_TY - 1) / BP_TY) * BP_TY;
    double span, lo, hi;
    if (in.geometry == GEOM_EM_REF) {
        const double dxy = in.dxy, dt = in.dt;
        const double xm = std::max(1.0, std::fabs(-1.0 + (Xext - 1) * dxy));
        const double ym = std::max(1.0, std::fabs(-1.0 + (Yext - 1) * dxy));
        const double Rt = std::sqrt(xm * xm + ym * ym);
        lo = (-Rt + 1.0) / dt;
        hi = (Rt + 1.0) / dt;
        span = std::sqrt(std::pow((BP_TX - 1) * dxy, 2) + std::pow((BP_TY - 1) * dxy, 2)) / dt;
    } else {
        // x = xmin + (i + offo) * dx for i in [0, Xext)
        const double xa = std::fabs(in.xmin + (double)in.offo * in.dx);
        const double xb = std::fabs(in.xmin + (double)(in.offo + Xext - 1) * in.dx);
        const double ya = std::fabs(in.ymin + (double)in.offo * in.dy);
        const double yb = std::fabs(in.ymin + (double)(in.offo + Yext - 1) * in.dy);
        const double xm = std::max(xa, xb), ym = std::max(ya, yb);
        const double Rt = std::sqrt(xm * xm + ym * ym);
        lo = (-Rt - in.tmin) / in.dt;
        hi = (Rt - in.tmin) / in.dt;
        span = std::sqrt(std::pow((BP_TX - 1) * in.dx, 2) + std::pow((BP_TY - 1) * in.dy, 2)) / in.dt;
    }
    // staged window: tile span, +1 inclusive, 1 bin margin each side,
    // rounding of the aligned start, 1 extra for the lin pair index rounding
    L.W = ceil_to((int)std::ceil(span) + 1 + 2 + (align - 1) + 2, align);
    L.wlo = floor_to((int)std::floor(lo) - 4 - align, align);
    const int whi = (int)std::ceil(hi) + 4 + L.W + align;
    L.Wg = ceil_to(whi - L.wlo, align);
    return L;
}

// ------------------------------------------------------------------------
// launch + autotuner
// ------------------------------------------------------------------------
constexpr size_t kBpSmemMax = 100 * 1024;

static size_t bp_smem(int S, int AB, int W, int esize)
{
    return kWinOffset + 2 * (size_t)AB * S * W * esize;
}

template <int GEOM, int STORE, int S, bool IL = false>
static void launch_bp_s(const BpArgs &a, int AB, cudaStream_t st)
{
    const int esize = (STORE == STORE_PAIR_F32) ? 8 : 4;
    const size_t smem = bp_smem(S, AB, a.W, esize);
    RAFT_CHECK(smem <= kBpSmemMax && AB >= 1 && AB <= 32, "backprojector: staged window too large");
    static thread_local int configured = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    void (*kern)(const BpArgs, const int);
    if constexpr (S == 4) kern = bp_kernel_s4<GEOM, STORE, IL>;
    else kern = bp_kernel<GEOM, STORE, S>;
    if (configured != dev) {
        RAFT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBpSmemMax));
        configured = dev;
    }
    dim3 grid((a.No + BP_TX - 1) / BP_TX, (a.No + BP_TY - 1) / BP_TY, (a.nslices + S - 1) / S);
    ProfScope ps(PROF_BACKPROJECT, st);
    kern<<<grid, BP_THREADS, smem, st>>>(a, AB);
    RAFT_CUDA(cudaGetLastError());
}

template <int GEOM, int STORE>
static void launch_bp_cfg(const BpArgs &a, BpTune t, cudaStream_t st)
{
    switch (t.S) {
    case 1: launch_bp_s<GEOM, STORE, 1>(a, t.AB, st); break;
    case 2: launch_bp_s<GEOM, STORE, 2>(a, t.AB, st); break;
    default:
        if (a.il) launch_bp_s<GEOM, STORE, 4, true>(a, t.AB, st);
        else launch_bp_s<GEOM, STORE, 4>(a, t.AB, st);
        break;
    }
}

static void launch_bp_any(const BpArgs &a, int geometry, int store, BpTune t, cudaStream_t st)
{
    switch (geometry) {
    case GEOM_FBP_REF: launch_bp_cfg<GEOM_FBP_REF, STORE_F32>(a, t, st); break;
    case GEOM_EM_REF: launch_bp_cfg<GEOM_EM_REF, STORE_F32>(a, t, st); break;
    default:
        if (store == STORE_PAIR_BF16) launch_bp_cfg<GEOM_FBP_LIN, STORE_PAIR_BF16>(a, t, st);
        else launch_bp_cfg<GEOM_FBP_LIN, STORE_PAIR_F32>(a, t, st);
        break;
    }
}

// Tuning table: (device, geometry, store, No, W, nangles) -> (S, AB).
using TuneKey = std::tuple<int, int, int, int, int, int>;
static std::mutex g_tune_mtx;
static std::map<TuneKey, BpTune> g_tune;

static const BpTune kTuneCandidates[] = {{1, 32}, {1, 16}, {2, 32}, {2, 16}, {2, 8}, {4, 16}, {4, 8}};

static bool tuning_enabled()
{
    const char *e = std::getenv("RAFT_BP_TUNE");
    return !(e && e[0] == '0');
}

// RAFT_BP_TUNE="S,AB" forces one candidate (for tests that compare every
// launch shape); returns false when unset, malformed or not a candidate.
static bool forced_tune(BpTune &t)
{
    const char *e = std::getenv("RAFT_BP_TUNE");
    int s = 0, ab = 0;
    if (!e || std::sscanf(e, "%d,%d", &s, &ab) != 2) return false;
    for (const BpTune &c : kTuneCandidates)
        if (c.S == s && c.AB == ab) {
            t = c;
            return true;
        }
    return false;
}

bool bp_forced_planar()
{
    BpTune t;
    return forced_tune(t) && t.S != 4;
}

// Pick (S, AB) for this configuration: the cached choice, else time every
// candidate that fits shared memory on 8 to 32 slices of the real data
// (store launches only -- they are idempotent), else a default.  With
// a_il (the same launch on slice-interleaved rows) the S = 4 candidates are
// timed on it; prep_il makes those rows and is called at most once.  With
// il_only the rows exist only interleaved: the S = 4 candidates alone.
template <class Prep>
static BpTune choose_tune(const BpArgs &a, const BpArgs *a_il, Prep &&prep_il, int geometry, int store,
                          cudaStream_t st, bool il_only = false)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const TuneKey key(dev, geometry, store + (a_il ? 16 : 0) + (il_only ? 32 : 0), a.No, a.W, a.nangles);
    const int esize = store_bytes(store);
    BpTune forced;
    if (forced_tune(forced) && bp_smem(forced.S, forced.AB, a.W, esize) <= kBpSmemMax && (!il_only || forced.S == 4))
        return forced;
    {
        std::lock_guard<std::mutex> lk(g_tune_mtx);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) return it->second;
    }
    BpTune best{2, 16};
    if (il_only) best = {4, 16};
    if (bp_smem(best.S, best.AB, a.W, esize) > kBpSmemMax) best = {il_only ? 4 : 1, 8};
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cap);
    const bool can_tune = tuning_enabled() && a.update == 0 && cap == cudaStreamCaptureStatusNone;
    if (can_tune) {
        // enough slices that a four-slice grid is several waves deep (a shallow
        // grid's tail would favour the smaller slice groups), 8 to 32
        BpArgs t0 = a;
        const long long tiles = (long long)((a.No + BP_TX - 1) / BP_TX) * ((a.No + BP_TY - 1) / BP_TY);
        const int want = (int)std::min<long long>(32, std::max<long long>(8, (4LL * 3 * 148 * 8 + tiles - 1) / tiles));
        if (a.nslices < std::min(want, 8)) {
            // too few slices to time the shapes fairly (a pipeline's small
            // first chunk): run the default now, tune on a later launch
            return best;
        }
        t0.nslices = std::min(a.nslices, (want + 3) / 4 * 4);
        cudaEvent_t e0, e1;
        RAFT_CUDA(cudaEventCreate(&e0));
        RAFT_CUDA(cudaEventCreate(&e1));
        float best_ms = 1e30f;
        for (const BpTune &c : kTuneCandidates) {
            if (bp_smem(c.S, c.AB, a.W, esize) > kBpSmemMax) continue;
            if (il_only && c.S != 4) continue;
            BpArgs t = t0;
            if (c.S == 4 && a_il) {
                prep_il();
                t = *a_il;
                t.nslices = t0.nslices;
            }
            launch_bp_any(t, geometry, store, c, st);   // warm
            // the fastest of three single launches (less sensitive to a stray slow one)
            float ms = 1e30f;
            for (int rep = 0; rep < 3; rep++) {
                RAFT_CUDA(cudaEventRecord(e0, st));
                launch_bp_any(t, geometry, store, c, st);
                RAFT_CUDA(cudaEventRecord(e1, st));
                RAFT_CUDA(cudaEventSynchronize(e1));
                float one = 0.f;
                RAFT_CUDA(cudaEventElapsedTime(&one, e0, e1));
                ms = std::min(ms, one);
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (can_tune || !tuning_enabled()) {
        std::lock_guard<std::mutex> lk(g_tune_mtx);
        g_tune[key] = best;
    }
    return best;
}

std::string bp_tune_table()
{
    std::lock_guard<std::mutex> lk(g_tune_mtx);
    std::string out = "[";
    for (auto &kv : g_tune) {
        char buf[160];
        snprintf(buf, sizeof buf, "%s{\"geometry\":%d,\"store\":%d,\"N\":%d,\"W\":%d,\"nangles\":%d,\"S\":%d,\"AB\":%d}",
                 out.size() > 1 ? "," : "", std::get<1>(kv.first), std::get<2>(kv.first), std::get<3>(kv.first),
                 std::get<4>(kv.first), std::get<5>(kv.first), kv.second.S, kv.second.AB);
        out += buf;
    }
    return out + "]";
}

static BpArgs to_args(const BpLaunch &bl)
{
    BpArgs a;
    a.filt = reinterpret_cast<const unsigned char *>(bl.filt);
    a.img = bl.img;
    a.den = bl.den;
    a.No = bl.No;
    a.nangles = bl.nangles;
    a.nslices = bl.nslices;
    a.wlo = bl.win.wlo;
    a.Wg = bl.win.Wg;
    a.W = bl.win.W;
    a.esize = store_bytes(bl.geometry == GEOM_FBP_LIN ? bl.store : STORE_F32);
    a.xmin = bl.geo.xmin;
    a.ymin = bl.geo.ymin;
    a.dx = bl.geo.dx;
    a.dy = bl.geo.dy;
    a.tmin = bl.geo.tmin;
    a.dt = bl.geo.dt;
    a.offo = bl.geo.offo;
    a.xymin = -1.0f;
    a.dxy = bl.geo.dxy;
    a.c0 = bl.geo.c0;
    a.ratio = bl.geo.ratio;
    a.u0 = bl.geo.u0;
    a.cs = bl.cs;
    a.sn = bl.sn;
    a.csd = bl.csd;
    a.snd = bl.snd;
    a.err = bl.err;
    a.update = bl.den ? 1 : 0;
    a.il = 0;
    return a;
}

size_t bp_il_bytes(int nslices, int nangles, int Wg, int esize)
{
    return (size_t)((nslices + 3) / 4) * nangles * Wg * 4 * esize;
}

void launch_backproject(const BpLaunch &bl, cudaStream_t st)
{
    if (bl.nslices <= 0 || bl.nangles <= 0) return;
    const BpArgs a = to_args(bl);
    const int store = bl.geometry == GEOM_FBP_LIN ? bl.store : STORE_F32;
    // four slices per CTA on slice-interleaved rows, when the caller provides the workspace
    // (4-byte elements: f32 samples and bf16 pairs; the 8-byte f32 pairs keep
    // their planar rows, whose S = 4 shape measured faster)
    const bool il_ok = bl.il_ws != nullptr && a.esize == 4;
    BpArgs a_il = a;
    a_il.filt = reinterpret_cast<const unsigned char *>(bl.il_ws);
    a_il.il = 1;
    if (bl.il_ready) {
        // the filter wrote the rows interleaved: four slices per CTA only
        RAFT_CHECK(il_ok, "backprojector: interleaved rows need the workspace and 4-byte elements");
        auto none = []() {};
        const BpTune t = choose_tune(a_il, &a_il, none, bl.geometry, store, st, true);
        launch_bp_any(a_il, bl.geometry, store, t, st);
        return;
    }
    bool il_done = false;
    auto prep_il = [&]() {
        if (il_done) return;
        count_launch();
        const unsigned grid = (unsigned)(((bl.nslices + 3) / 4) * bl.nangles);
        if (a.esize == 8)
            interleave4_kernel<uint2><<<grid, 256, 0, st>>>(reinterpret_cast<const uint2 *>(bl.filt),
                                                          reinterpret_cast<uint2 *>(bl.il_ws), bl.nslices,
                                                          bl.nangles, bl.win.Wg);
        else
            interleave4_kernel<uint32_t><<<grid, 256, 0, st>>>(reinterpret_cast<const uint32_t *>(bl.filt),
                                                             reinterpret_cast<uint32_t *>(bl.il_ws), bl.nslices,
                                                             bl.nangles, bl.win.Wg);
        RAFT_CUDA(cudaGetLastError());
        il_done = true;
    };
    const BpTune t = choose_tune(a, il_ok ? &a_il : nullptr, prep_il, bl.geometry, store, st);
    if (il_ok && t.S == 4) {
        prep_il();
        launch_bp_any(a_il, bl.geometry, store, t, st);
    } else {
        launch_bp_any(a, bl.geometry, store, t, st);
    }
}

// ------------------------------------------------------------------------
// ragged batches
// ------------------------------------------------------------------------
constexpr int kRaggedAB = 16;

static size_t al256(size_t v) { return (v + 255) & ~(size_t)255; }

// Byte offsets of the regions of a ragged descriptor workspace; the same
// function sizes the workspace and lays it out.
struct RaggedLayout {
    size_t args, item_start, counts, remaining, queue, tdone, total;
};

static RaggedLayout ragged_layout(int nreq)
{
    RaggedLayout L;
    size_t off = 0;
    L.args = off;       off = al256(off + sizeof(BpArgs) * nreq);
    L.item_start = off; off = al256(off + sizeof(int) * (nreq + 1));
    L.counts = off;     off = al256(off + sizeof(int) * nreq);
    L.remaining = off;  off = al256(off + sizeof(int) * nreq);
    L.queue = off;      off = al256(off + sizeof(int) * 4);
    L.tdone = off;      off = al256(off + sizeof(unsigned long long) * nreq);
    L.total = off;
    return L;
}

size_t ragged_bp_bytes(int nreq) { return ragged_layout(nreq).total; }

void ragged_bp_prepare(RaggedBp &rb, const BpLaunch *reqs, int nreq, int geometry, int store, void *d_ws)
{
    rb.nreq = nreq;
    rb.geometry = geometry;
    rb.store = geometry == GEOM_FBP_LIN ? store : STORE_F32;
    std::vector<BpArgs> args(nreq);
    std::vector<int> start(nreq + 1), counts(nreq);
    int total = 0, wmax = 0;
    for (int r = 0; r < nreq; r++) {
        args[r] = to_args(reqs[r]);
        const int tx = (reqs[r].No + BP_TX - 1) / BP_TX, ty = (reqs[r].No + BP_TY - 1) / BP_TY;
        counts[r] = tx * ty * reqs[r].nslices;    // one slice per CTA (S = 1)
        start[r] = total;
        total += counts[r];
        wmax = std::max(wmax, reqs[r].win.W);
    }
    start[nreq] = total;
    rb.total = total;
    rb.wmax = wmax;
    char *base = static_cast<char *>(d_ws);
    const RaggedLayout L = ragged_layout(nreq);
    rb.d_args = base + L.args;
    rb.d_item_start = (int *)(base + L.item_start);
    rb.d_counts = (int *)(base + L.counts);
    rb.d_remaining = (int *)(base + L.remaining);
    rb.d_queue = (int *)(base + L.queue);
    rb.d_tdone = (unsigned long long *)(base + L.tdone);
    RAFT_CUDA(cudaMemcpy(rb.d_args, args.data(), sizeof(BpArgs) * nreq, cudaMemcpyHostToDevice));
    RAFT_CUDA(cudaMemcpy(rb.d_item_start, start.data(), sizeof(int) * (nreq + 1), cudaMemcpyHostToDevice));
    RAFT_CUDA(cudaMemcpy(rb.d_counts, counts.data(), sizeof(int) * nreq, cudaMemcpyHostToDevice));
    RAFT_CUDA(cudaMemset(rb.d_tdone, 0, sizeof(unsigned long long) * nreq));
}

__global__ void ragged_reset_kernel(int *queue, int *remaining, const int *counts, int nreq)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) *queue = 0;
    for (int r = t; r < nreq; r += gridDim.x * blockDim.x) remaining[r] = counts[r];
}

template <int GEOM, int STORE>
static void launch_ragged_t(const RaggedBp &rb, cudaStream_t st)
{
    const int esize = (STORE == STORE_PAIR_F32) ? 8 : 4;
    const size_t smem = bp_smem(1, kRaggedAB, rb.wmax, esize);
    RAFT_CHECK(smem <= kBpSmemMax, "ragged backprojector: window too large");
    static thread_local int configured = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured != dev) {
        RAFT_CUDA(cudaFuncSetAttribute(bp_ragged_kernel<GEOM, STORE, 1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBpSmemMax));
        configured = dev;
    }
    int per_sm = 0, nsm = 0;
    RAFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_ragged_kernel<GEOM, STORE, 1>, BP_THREADS,
                                                            smem));
    RAFT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int grid = std::max(1, std::min(rb.total, std::max(1, per_sm) * nsm));
    count_launch();
    ragged_reset_kernel<<<1, 256, 0, st>>>(rb.d_queue, rb.d_remaining, rb.d_counts, rb.nreq);
    ProfScope ps(PROF_BACKPROJECT, st);
    bp_ragged_kernel<GEOM, STORE, 1><<<grid, BP_THREADS, smem, st>>>(
        reinterpret_cast<const BpArgs *>(rb.d_args), rb.d_item_start, rb.nreq, rb.total, kRaggedAB, rb.d_queue,
        rb.d_remaining, rb.d_tdone);
    RAFT_CUDA(cudaGetLastError());
}

void ragged_bp_launch(const RaggedBp &rb, cudaStream_t st)
{
    if (rb.nreq <= 0 || rb.total <= 0) return;
    switch (rb.geometry) {
    case GEOM_FBP_REF: launch_ragged_t<GEOM_FBP_REF, STORE_F32>(rb, st); break;
    case GEOM_EM_REF: launch_ragged_t<GEOM_EM_REF, STORE_F32>(rb, st); break;
    default:
        if (rb.store == STORE_PAIR_BF16) launch_ragged_t<GEOM_FBP_LIN, STORE_PAIR_BF16>(rb, st);
        else launch_ragged_t<GEOM_FBP_LIN, STORE_PAIR_F32>(rb, st);
        break;
    }
}

__global__ void stamp_kernel(unsigned long long *t)
{
    if (threadIdx.x == 0) *t = global_ns();
}

void launch_stamp(unsigned long long *d_t, cudaStream_t st)
{
    count_launch();
    stamp_kernel<<<1, 32, 0, st>>>(d_t);
    RAFT_CUDA(cudaGetLastError());
}

}  // namespace raft
