// background.cu -- flat/dark correction of projections, optionally with -log.
//
// Reference: BackgroundCorrection, cuda/src/processing/background_correction.cu:15-47
// and Klog (getLog), cuda/src/common/opt.cu:196-214:
//     flat  = flat[z][0]                                  (one flat)
//           = flat[z][0] * (1 - a/A) + (a/A) * flat[z][1] (two or more: only the
//             first two are used, interpolated by the angle index a of A)
//     T     = max(D - dark, 0.5) / max(flat - dark, 0.5)
//     T     = -log(T)                                     (is_log)
// on frames [slices][angles][rays], flat [slices][nflats][rays], dark [slices][rays].
//
// B200: pure streaming work (one read + one write per element; the flat and
// dark rows of a slice are re-read from L1/L2 by every angle), so the kernel is
// written for the HBM roofline: 16-byte vector accesses when the row length and
// the pointers allow, a grid of whole rows, two rows per thread, streaming
// cache hints, and the fast division / log the reference's fast-math build uses
// (IEEE division and logf made the kernel instruction-bound at 57 % of HBM).
#include "raft.hpp"
#include "profile.hpp"

#include <algorithm>
#include <cstdint>

namespace raft {

// One row of V-wide vectors: flat/dark correction (+ -log) of src into dst.
template <int V>
__device__ __forceinline__ void background_row(const float *src, float *dst, const float *fb, const float *fa,
                                               const float *dk, int v, int numflats, float interp, int is_log)
{
    float d[V], f[V], s[V], r[V];
    if constexpr (V == 4) {
        const float4 d4 = __ldg(reinterpret_cast<const float4 *>(dk) + v);
        const float4 f4 = __ldg(reinterpret_cast<const float4 *>(fb) + v);
        const float4 s4 = __ldcs(reinterpret_cast<const float4 *>(src) + v);
        d[0] = d4.x; d[1] = d4.y; d[2] = d4.z; d[3] = d4.w;
        f[0] = f4.x; f[1] = f4.y; f[2] = f4.z; f[3] = f4.w;
        s[0] = s4.x; s[1] = s4.y; s[2] = s4.z; s[3] = s4.w;
        if (numflats > 1) {
            const float4 g4 = __ldg(reinterpret_cast<const float4 *>(fa) + v);
            const float g[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
            for (int e = 0; e < 4; e++) f[e] = f[e] * (1.0f - interp) + interp * g[e];
        }
    } else {
        d[0] = __ldg(dk + v);
        f[0] = __ldg(fb + v);
        s[0] = __ldcs(src + v);
        if (numflats > 1) f[0] = f[0] * (1.0f - interp) + interp * __ldg(fa + v);
    }
#pragma unroll
    for (int e = 0; e < V; e++) {
        // fast division and log, as the reference build (fast math) computes them
        const float t = __fdividef(fmaxf(s[e] - d[e], 0.5f), fmaxf(f[e] - d[e], 0.5f));
        r[e] = is_log ? -__logf(t) : t;
    }
    if constexpr (V == 4) __stcs(reinterpret_cast<float4 *>(dst) + v, make_float4(r[0], r[1], r[2], r[3]));
    else __stcs(dst + v, r[0]);
}

// Rows are taken two at a time per thread (more loads in flight); the frames
// stream through with evict-first hints so the flat and dark rows, re-read by
// every angle of a slice, stay in L2.  `in` and `out` may be the same array
// (each element is read, then written, by one thread), so they are not
// declared __restrict__.
// Row counts (slices x angles) fit 32 bits, so the slice / angle split of a
// row index is a 32-bit division (a 64-bit one is an emulated routine that
// dominated the kernel's instruction count).
template <int V>
__global__ void __launch_bounds__(256)
background_kernel(const float *in, float *out, const float *__restrict__ flat, const float *__restrict__ dark,
                  int nrays, int nangles, unsigned nrows, int numflats, int is_log)
{
    const int nv = nrays / V;                         // vectors per row
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    for (unsigned row0 = 2u * blockIdx.y; row0 < nrows; row0 += 2u * gridDim.y) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const unsigned row = row0 + h;
            if (row >= nrows) break;
            const int z = (int)(row / (unsigned)nangles);
            const int a = (int)(row - (unsigned)z * (unsigned)nangles);
            const float interp = (float)a / (float)nangles;
            const float *fb = flat + (size_t)z * numflats * nrays;
            background_row<V>(in + (size_t)row * nrays, out + (size_t)row * nrays, fb, fb + nrays,
                              dark + (size_t)z * nrays, v, numflats, interp, is_log);
        }
    }
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

void launch_background(const float *in, float *out, const float *flat, const float *dark, int nrays, int nangles,
                       int nslices, int numflats, int is_log, cudaStream_t st)
{
    const long long nrows = (long long)nslices * nangles;
    if (nrows <= 0 || nrays <= 0) return;
    RAFT_CHECK(numflats >= 1, "background correction: at least one flat is needed");
    RAFT_CHECK(nrows < (1LL << 31), "background correction: slices x angles must be below 2^31");
    const bool vec = nrays % 4 == 0 && aligned16(in) && aligned16(out) && aligned16(flat) && aligned16(dark);
    const int V = vec ? 4 : 1;
    const int nv = nrays / V;
    dim3 block(256);
    dim3 grid((nv + 255) / 256, (unsigned)std::min<long long>((nrows + 1) / 2, 65535));
    count_launch();
    if (vec) background_kernel<4><<<grid, block, 0, st>>>(in, out, flat, dark, nrays, nangles, (unsigned)nrows, numflats, is_log);
    else background_kernel<1><<<grid, block, 0, st>>>(in, out, flat, dark, nrays, nangles, (unsigned)nrows, numflats, is_log);
    RAFT_CUDA(cudaGetLastError());
}

}  // namespace raft
