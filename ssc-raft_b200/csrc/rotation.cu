// rotation.cu -- rotation-axis estimation from the 0 and 180 degree frames.
//
// Reference: getCentersino / getCentersino_subpixel / getCentersino16,
// cuda/src/processing/rotation_axis.cu:14-46,221-360,429-451:
//   f = -log(max(frame0 - dark, 0.5) / max(flat - dark, 0.5)),
//   g = the same of frame180, mirrored in x;
//   F = FFT2(f), G = FFT2(g); F <- F conj(G) e^{-20 (xx^2 + yy^2)} / |F conj(G)|
//   with xx = min(x, sizex - x)/sizex, yy = min(y, sizey - y)/sizey;
//   f <- IFFT2(F) (unnormalised);
//   integer search: the first (row-major) maximum of |f|^2 over x = 0, 4, 8, ...
//   below sizex rounded down to a multiple of 4, then every x of the
//   remainder; posx > sizex/2 wraps to posx - sizex; result -posx/2 (int);
//   sub-pixel search: the first maximum over rows y and x = i * 0.01 for
//   i < sizex of the cubic Lagrange interpolation of |f|^2 (abs2InterpCubic,
//   :155-220; at integer y only the row y contributes), result -x/2 after the
//   same wrap.  Both searches keep the reference's candidate sets as they are.
//
// B200 design: the frames are one detector image each, so the work is a
// handful of launches: a fused correction/mirror kernel, row and column
// transforms in shared memory (fft.cuh; columns are gathered with a stride),
// the normalised cross-spectrum, and the peak search as one pass over all
// candidates with a 64-bit atomic maximum of (value bits, reversed scan
// order) -- the reference's first-strict-maximum rule -- instead of copying
// the correlation to the host.  The candidate values are computed with the
// reference's float expressions (its search runs on the host, IEEE float,
// no contraction), written with explicit round-to-nearest operations.
// Compiled with fast math like the reference's device code (the -log, the
// divisions and the Gaussian use the same intrinsics).
#include "raft.hpp"
#include "profile.hpp"
#include "fft.cuh"

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

namespace raft {

namespace {

template <typename T>
__global__ void cross_frame_kernel(float2 *f, float2 *g, const T *frame0, const T *frame1, const T *dark,
                                   const T *flat, int sizex)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= sizex) return;
    const size_t i = (size_t)y * sizex + x;
    const float dk = (float)dark[i], ft = (float)flat[i];
    const float q = fmaxf(ft - dk, 0.5f);
    f[i] = make_float2(-__logf(__fdividef(fmaxf((float)frame0[i] - dk, 0.5f), q)), 0.f);
    g[(size_t)y * sizex + (sizex - 1 - x)] = make_float2(-__logf(__fdividef(fmaxf((float)frame1[i] - dk, 0.5f), q)), 0.f);
}

// In-place transforms of `count` sequences of length n: sequence r starts at
// data + r * seq_stride, element k at + k * elem_stride.  inverse: unnormalised
// inverse (conjugate, forward, conjugate).
__global__ void __launch_bounds__(512)
fft_strided_kernel(float2 *data, int n, size_t seq_stride, size_t elem_stride, FftPlan P, int inverse)
{
    extern __shared__ float2 sm_rot[];
    float2 *base = data + (size_t)blockIdx.x * seq_stride;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const float2 v = base[(size_t)k * elem_stride];
        sm_rot[k] = inverse ? make_float2(v.x, -v.y) : v;
    }
    __syncthreads();
    const float2 *r = fft_run(sm_rot, sm_rot + fft_plan_span(P), P);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const float2 v = r[k];
        base[(size_t)k * elem_stride] = inverse ? make_float2(v.x, -v.y) : v;
    }
}

// KCrossCorrelation (rotation_axis.cu:30-45)
__global__ void cross_spectrum_kernel(float2 *F, const float2 *G, int sizex, int sizey)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= sizex) return;
    const size_t i = (size_t)y * sizex + x;
    const float xx = fminf((float)(sizex - x), (float)x) / (float)sizex;
    const float yy = fminf((float)(sizey - y), (float)y) / (float)sizey;
    const float gauss = __expf(-20.0f * (xx * xx + yy * yy));
    const float2 a = F[i], b = G[i];
    const float2 fg = make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);   // a * conj(b)
    const float m = sqrtf(fg.x * fg.x + fg.y * fg.y);
    F[i] = make_float2(__fdividef(fg.x * gauss, m), __fdividef(fg.y * gauss, m));
}

// |c|^2 as the reference's host search computes it (two rounded products, one rounded sum)
__device__ __forceinline__ float abs2_rn(float2 c) { return __fadd_rn(__fmul_rn(c.x, c.x), __fmul_rn(c.y, c.y)); }

__device__ __forceinline__ unsigned long long peak_key(float v, unsigned order)
{
    // strict maximum over v > 0 (the search starts from 0); equal values: the
    // earliest candidate, i.e. the largest reversed order
    if (!(v > 0.0f)) return 0ull;
    return ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)(0xffffffffu - order);
}

__device__ __forceinline__ void warp_max_commit(unsigned long long key, unsigned long long *best)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if ((threadIdx.x & 31) == 0 && key) atomicMax(best, key);
}

// integer search: candidates per row x = 0, 4, ..., irange - 4, then irange .. sizex - 1
__global__ void peak_int_kernel(const float2 *f, int sizex, int sizey, unsigned long long *best)
{
    const int irange = sizex & ~3;
    const int per_row = irange / 4 + (sizex - irange);
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = 0ull;
    if (c < (long long)per_row * sizey) {
        const int y = (int)(c / per_row), k = (int)(c - (long long)y * per_row);
        const int x = k < irange / 4 ? 4 * k : irange + (k - irange / 4);
        key = peak_key(abs2_rn(f[(size_t)y * sizex + x]), (unsigned)c);
    }
    warp_max_commit(key, best);
}

// sub-pixel search: rows y, x = i * 0.01f for i < sizex, cubic Lagrange in x
// (abs2InterpCubic at integer y: only the row y contributes; the weights are
// the reference's float products in its order, divided by 36, -12, 12, -36)
__global__ void peak_subpixel_kernel(const float2 *f, int sizex, int sizey, unsigned long long *best)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = 0ull;
    if (c < (long long)sizex * sizey) {
        const int y = (int)(c / sizex), i = (int)(c - (long long)y * sizex);
        const float p = __fmul_rn((float)i, 0.01f);
        const int x0 = (int)floorf(p);
        float v[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int xm = x0 + m;
            v[m] = (xm >= 0 && xm < sizex) ? abs2_rn(f[(size_t)y * sizex + xm]) : 0.0f;
        }
        const float d0 = __fsub_rn((float)x0, p), d1 = __fsub_rn((float)(x0 + 1), p);
        const float d2 = __fsub_rn((float)(x0 + 2), p), d3 = __fsub_rn((float)(x0 + 3), p);
        // y factors (y1 - y)(y2 - y)(y3 - y) = 1, 2, 3 applied in order
        auto yf = [](float t) { return __fmul_rn(__fmul_rn(__fmul_rn(t, 1.0f), 2.0f), 3.0f); };
        const float w0 = __fdiv_rn(yf(__fmul_rn(__fmul_rn(d1, d2), d3)), 36.0f);
        const float w1 = __fdiv_rn(yf(__fmul_rn(__fmul_rn(d0, d2), d3)), -12.0f);
        const float w2 = __fdiv_rn(yf(__fmul_rn(__fmul_rn(d0, d1), d3)), 12.0f);
        const float w3 = __fdiv_rn(yf(__fmul_rn(__fmul_rn(d0, d1), d2)), -36.0f);
        float s = __fmul_rn(w0, v[0]);
        s = __fadd_rn(s, __fmul_rn(w1, v[1]));
        s = __fadd_rn(s, __fmul_rn(w2, v[2]));
        s = __fadd_rn(s, __fmul_rn(w3, v[3]));
        key = peak_key(s, (unsigned)c);
    }
    warp_max_commit(key, best);
}

void fft2(int device, float2 *data, int sizex, int sizey, int inverse, cudaStream_t st)
{
    const FftTable &tx = fft_table(device, sizex), &ty = fft_table(device, sizey);
    const size_t smx = 2 * (size_t)fft_plan_span(tx.plan) * sizeof(float2),
                 smy = 2 * (size_t)fft_plan_span(ty.plan) * sizeof(float2);
    RAFT_CUDA(cudaFuncSetAttribute(fft_strided_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)std::max(smx, smy)));
    count_launch();
    fft_strided_kernel<<<sizey, fft_threads(tx.plan.M), smx, st>>>(data, sizex, sizex, 1, tx.plan, inverse);
    RAFT_CUDA(cudaGetLastError());
    count_launch();
    fft_strided_kernel<<<sizex, fft_threads(ty.plan.M), smy, st>>>(data, sizey, 1, sizex, ty.plan, inverse);
    RAFT_CUDA(cudaGetLastError());
}

}  // namespace

bool centersino_shape_ok(int sizex, int sizey)
{
    const size_t lim = 227 * 1024;
    const int Mx = fft_plan_length(sizex), My = fft_plan_length(sizey);
    return sizex >= 1 && sizey >= 1 && Mx > 0 && My > 0 && 2 * (size_t)fft_span(Mx) * sizeof(float2) <= lim &&
           2 * (size_t)fft_span(My) * sizeof(float2) <= lim && (unsigned long long)sizex * sizey < 0xffffffffull;
}

template <typename T>
double centersino_device(int device, const T *d_frame0, const T *d_frame1, const T *d_dark, const T *d_flat,
                         int sizex, int sizey, int subpixel, void *workspace, cudaStream_t st)
{
    const size_t plane = (size_t)sizex * sizey;
    float2 *F = (float2 *)workspace;
    float2 *G = F + plane;
    unsigned long long *best = (unsigned long long *)(G + plane);
    dim3 grid((sizex + 127) / 128, sizey);
    count_launch();
    cross_frame_kernel<T><<<grid, 128, 0, st>>>(F, G, d_frame0, d_frame1, d_dark, d_flat, sizex);
    RAFT_CUDA(cudaGetLastError());
    fft2(device, F, sizex, sizey, 0, st);
    fft2(device, G, sizex, sizey, 0, st);
    count_launch();
    cross_spectrum_kernel<<<grid, 128, 0, st>>>(F, G, sizex, sizey);
    RAFT_CUDA(cudaGetLastError());
    fft2(device, F, sizex, sizey, 1, st);
    RAFT_CUDA(cudaMemsetAsync(best, 0, sizeof(unsigned long long), st));
    const int irange = sizex & ~3;
    const long long ncand = subpixel ? (long long)sizex * sizey : (long long)(irange / 4 + sizex - irange) * sizey;
    count_launch();
    if (subpixel) peak_subpixel_kernel<<<(unsigned)((ncand + 255) / 256), 256, 0, st>>>(F, sizex, sizey, best);
    else peak_int_kernel<<<(unsigned)((ncand + 255) / 256), 256, 0, st>>>(F, sizex, sizey, best);
    RAFT_CUDA(cudaGetLastError());
    unsigned long long key = 0;
    RAFT_CUDA(cudaMemcpyAsync(&key, best, sizeof(key), cudaMemcpyDeviceToHost, st));
    RAFT_CUDA(cudaStreamSynchronize(st));
    const unsigned order = key ? 0xffffffffu - (unsigned)(key & 0xffffffffull) : 0u;
    if (subpixel) {
        const int i = key ? (int)(order % (unsigned)sizex) : 0;
        float bestpos = (float)i * 0.01f;
        if (bestpos > (float)sizex / 2.0f) bestpos -= (float)sizex;
        return -bestpos / 2.0f;
    }
    int posx = 0;
    if (key) {
        const int per_row = irange / 4 + (sizex - irange);
        const int k = (int)(order % (unsigned)per_row);
        posx = k < irange / 4 ? 4 * k : irange + (k - irange / 4);
    }
    if (posx > (float)sizex / 2) posx -= sizex;
    return -posx / 2;
}

size_t centersino_workspace_bytes(int sizex, int sizey)
{
    return 2 * (size_t)sizex * sizey * sizeof(float2) + 256;
}

template double centersino_device<float>(int, const float *, const float *, const float *, const float *, int, int,
                                         int, void *, cudaStream_t);
template double centersino_device<uint16_t>(int, const uint16_t *, const uint16_t *, const uint16_t *,
                                            const uint16_t *, int, int, int, void *, cudaStream_t);

}  // namespace raft
