// unet.cu -- tensor-core kernels of the learned warm start for EM.
//
// A small U-Net maps an FBP image to an estimate that tEM starts from
// (no reference counterpart: the reference only exposes the initial guess,
// em_methods.py:117-122 / em_rt.cu:135).  Activations are BF16 NHWC with
// channel counts that are multiples of 32; weights are BF16 [Cout][3][3][Cin]
// with FP32 master copies; every accumulation is FP32.
//
// The forward / data-gradient convolution runs on the tcgen05 tensor cores
// (unet_tc.cu) wherever its 128-pixel tile fits; the kernels here are
// implicit GEMMs on mma.sync.m16n8k16 BF16 -> FP32:
//   conv3x3_fwd    y = act(conv(x) + b); x may be the channel concatenation
//                  of two tensors (the decoder's skip connection), read
//                  in place -- no concatenated copy is materialised
//   conv3x3_dgrad  the data gradient is conv3x3_fwd of dY with the weights
//                  flipped in space and transposed in channels
//   conv3x3_wgrad  dW[co][tap][ci] = sum over pixels of dY[p][co] * x[p+tap][ci],
//                  pixels split across CTAs, FP32 atomic accumulation
// plus the memory-bound pieces: ReLU mask, 2x2 average pooling, nearest 2x
// upsampling, the 1x1 output head with the residual connection, MSE loss
// gradient and Adam.
#include "raft.hpp"
#include "profile.hpp"

#include <cuda_bf16.h>

namespace raft {

typedef __nv_bfloat16 bf16;

// ------------------------------------------------------------ mma helpers
__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3, const void *p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(smem_addr(p)));
}

__device__ __forceinline__ void ldmatrix_x4_trans(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3,
                                                  const void *p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(smem_addr(p)));
}

// D = A(16x16, row) * B(16x8, col) + D, BF16 inputs, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float *d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ------------------------------------------------------------ conv forward
// CTA: 128 threads = 4 warps; tile = 64 consecutive pixels of one image row
// (n, y, x0..x0+63) x 32 output channels.  Warp w owns pixels 16w..16w+15
// and all 32 channels (4 n8 tiles).  K = 9 taps x Cin in chunks of 32
// channels, staged through shared memory (rows padded to 40 halves so the
// ldmatrix row addresses fall in distinct banks).
constexpr int CV_PIX = 64, CV_CO = 32, CV_KC = 32, CV_LD = 40;

struct ConvArgs {
    const bf16 *x0, *x1;   // inputs [N][H][W][C0] and [N][H][W][C1] (x1 may be null, C1 = 0)
    int C0, C1;
    const bf16 *w;         // [Cout][3][3][C0+C1]
    const float *bias;     // [Cout] or null
    bf16 *y;               // [N][H][W][Cout], or channels [0, Cy0) when y1 is set
    bf16 *y1;              // optional second output: channels [Cy0, Cout) as [N][H][W][Cout-Cy0]
    int Cy0;
    int N, H, W, Cout;
    int relu;
};

__global__ void __launch_bounds__(128) conv3x3_fwd_kernel(const ConvArgs a)
{
    __shared__ __align__(128) bf16 As[CV_PIX * CV_LD];
    __shared__ __align__(128) bf16 Bs[CV_CO * CV_LD];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = (a.W + CV_PIX - 1) / CV_PIX;
    const int row = blockIdx.x / tiles_x;                // n*H + y
    const int x0 = (blockIdx.x % tiles_x) * CV_PIX;
    const int n = row / a.H, y = row % a.H;
    const int co0 = blockIdx.y * CV_CO;
    const int Cin = a.C0 + a.C1;
    float acc[4][4];
#pragma unroll
    for (int t = 0; t < 4; t++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[t][e] = 0.f;

    for (int tap = 0; tap < 9; tap++) {
        const int ky = tap / 3 - 1, kx = tap % 3 - 1;
        const int yy = y + ky;
        for (int c0 = 0; c0 < Cin; c0 += CV_KC) {
            // A: 64 pixels x 32 channels (4 x 16-byte chunks per pixel)
            const bf16 *src;
            int cs, C;
            if (c0 < a.C0) { src = a.x0; cs = c0; C = a.C0; }
            else { src = a.x1; cs = c0 - a.C0; C = a.C1; }
            for (int e = tid; e < CV_PIX * 4; e += 128) {
                const int p = e >> 2, q = e & 3;
                const int xx = x0 + p + kx;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W && x0 + p < a.W)
                    v = *reinterpret_cast<const uint4 *>(src + (((size_t)n * a.H + yy) * a.W + xx) * C + cs + q * 8);
                *reinterpret_cast<uint4 *>(&As[p * CV_LD + q * 8]) = v;
            }
            // B: 32 output channels x 32 input channels of this tap
            for (int e = tid; e < CV_CO * 4; e += 128) {
                const int o = e >> 2, q = e & 3;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (co0 + o < a.Cout)
                    v = *reinterpret_cast<const uint4 *>(a.w + ((size_t)(co0 + o) * 9 + tap) * Cin + c0 + q * 8);
                *reinterpret_cast<uint4 *>(&Bs[o * CV_LD + q * 8]) = v;
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < CV_KC; kk += 16) {
                uint32_t a0, a1, a2, a3;
                {
                    const int mi = lane >> 3, r = lane & 7;
                    const bf16 *pa = &As[(warp * 16 + (mi & 1) * 8 + r) * CV_LD + kk + (mi >> 1) * 8];
                    ldmatrix_x4(a0, a1, a2, a3, pa);
                }
#pragma unroll
                for (int nt = 0; nt < 4; nt += 2) {
                    uint32_t b0, b1, b2, b3;
                    const int mi = lane >> 3, r = lane & 7;
                    // matrices: (n 0-7,k lo) (n 0-7,k hi) (n 8-15,k lo) (n 8-15,k hi)
                    const bf16 *pb = &Bs[(nt * 8 + (mi >> 1) * 8 + r) * CV_LD + kk + (mi & 1) * 8];
                    ldmatrix_x4(b0, b1, b2, b3, pb);
                    mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
                    mma_bf16(acc[nt + 1], a0, a1, a2, a3, b2, b3);
                }
            }
            __syncthreads();
        }
    }
    // epilogue: bias, ReLU, BF16 store
    const int g = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int p = warp * 16 + g + h * 8;
            const int co = co0 + nt * 8 + tg * 2;
            if (x0 + p >= a.W || co >= a.Cout) continue;
            float v0 = acc[nt][h * 2], v1 = acc[nt][h * 2 + 1];
            if (a.bias) {
                v0 += a.bias[co];
                v1 += a.bias[co + 1];
            }
            if (a.relu) {
                v0 = fmaxf(v0, 0.f);
                v1 = fmaxf(v1, 0.f);
            }
            const size_t pix = ((size_t)n * a.H + y) * a.W + x0 + p;
            bf16 *dst;
            if (a.y1 && co >= a.Cy0) dst = a.y1 + pix * (a.Cout - a.Cy0) + (co - a.Cy0);
            else if (a.y1) dst = a.y + pix * a.Cy0 + co;
            else dst = a.y + pix * a.Cout + co;
            *reinterpret_cast<__nv_bfloat162 *>(dst) = __floats2bfloat162_rn(v0, v1);
        }
    }
}

// ------------------------------------------------------------ weight grad
// CTA tile: 32 output channels x 32 input channels of one tap; K = a slice of
// NP pixels; the partial sums are added atomically into dW (FP32).
// A = dY^T (co x pixels) and B = x_tap (pixels x ci) are both stored
// pixel-major in shared memory and read with transposing ldmatrix.
constexpr int WG_CO = 32, WG_CI = 32, WG_KP = 32, WG_LD = 40;

struct WgradArgs {
    const bf16 *dy;        // [N][H][W][Cout]
    const bf16 *x0, *x1;   // inputs as in ConvArgs
    int C0, C1;
    float *dw;             // [Cout][3][3][C0+C1], accumulated
    float *dbias;          // [Cout], accumulated (taps 0 CTAs only) or null
    int N, H, W, Cout;
    int pix_per_cta;
};

__global__ void __launch_bounds__(128) conv3x3_wgrad_kernel(const WgradArgs a)
{
    __shared__ __align__(128) bf16 Ds[WG_KP * WG_LD];   // [pixel][co]
    __shared__ __align__(128) bf16 Xs[WG_KP * WG_LD];   // [pixel][ci]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Cin = a.C0 + a.C1;
    const int nci = Cin / WG_CI, nco = (a.Cout + WG_CO - 1) / WG_CO;
    int b = blockIdx.x;
    const int cib = b % nci; b /= nci;
    const int cob = b % nco; b /= nco;
    const int tap = b % 9;
    const int pchunk = blockIdx.y;
    const int ky = tap / 3 - 1, kx = tap % 3 - 1;
    const int co0 = cob * WG_CO, ci0 = cib * WG_CI;
    const bf16 *src;
    int cs, C;
    if (ci0 < a.C0) { src = a.x0; cs = ci0; C = a.C0; }
    else { src = a.x1; cs = ci0 - a.C0; C = a.C1; }
    const long total = (long)a.N * a.H * a.W;
    const long p_begin = (long)pchunk * a.pix_per_cta;
    const long p_end = min(total, p_begin + a.pix_per_cta);
    // warp w: co rows 16*(w&1).., ci cols 16*(w>>1).. (2 n8 tiles)
    const int wm = (warp & 1) * 16, wn = (warp >> 1) * 16;
    float acc[2][4];
#pragma unroll
    for (int t = 0; t < 2; t++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[t][e] = 0.f;
    float bsum = 0.f;
    for (long p0 = p_begin; p0 < p_end; p0 += WG_KP) {
        for (int e = tid; e < WG_KP * 4; e += 128) {
            const int pp = e >> 2, q = e & 3;
            const long p = p0 + pp;
            uint4 vd = make_uint4(0, 0, 0, 0), vx = make_uint4(0, 0, 0, 0);
            if (p < p_end) {
                const int xx = (int)(p % a.W);
                const long r = p / a.W;
                const int yy = (int)(r % a.H), n = (int)(r / a.H);
                if (co0 + q * 8 < a.Cout)
                    vd = *reinterpret_cast<const uint4 *>(a.dy + p * a.Cout + co0 + q * 8);
                const int sy = yy + ky, sx = xx + kx;
                if (sy >= 0 && sy < a.H && sx >= 0 && sx < a.W)
                    vx = *reinterpret_cast<const uint4 *>(src + (((size_t)n * a.H + sy) * a.W + sx) * C + cs + q * 8);
            }
            *reinterpret_cast<uint4 *>(&Ds[pp * WG_LD + q * 8]) = vd;
            *reinterpret_cast<uint4 *>(&Xs[pp * WG_LD + q * 8]) = vx;
        }
        __syncthreads();
        if (a.dbias && tap == 4 && cib == 0 && tid < WG_CO) {
            for (int pp = 0; pp < WG_KP; pp++) bsum += __bfloat162float(Ds[pp * WG_LD + tid]);
        }
#pragma unroll
        for (int kk = 0; kk < WG_KP; kk += 16) {
            // A (16 co x 16 pixels) from Ds[pixel][co]: transposed loads
            uint32_t a0, a1, a2, a3;
            {
                const int mi = lane >> 3, r = lane & 7;
                // matrices: (co lo, k lo) (co hi, k lo) (co lo, k hi) (co hi, k hi)
                const bf16 *pa = &Ds[(kk + (mi >> 1) * 8 + r) * WG_LD + wm + (mi & 1) * 8];
                ldmatrix_x4_trans(a0, a1, a2, a3, pa);
            }
            // B (16 pixels x 16 ci) from Xs[pixel][ci]: transposed loads give [ci][k] fragments
            uint32_t b0, b1, b2, b3;
            {
                const int mi = lane >> 3, r = lane & 7;
                // matrices: (ci 0-7, k lo) (ci 0-7, k hi) (ci 8-15, k lo) (ci 8-15, k hi)
                const bf16 *pb = &Xs[(kk + (mi & 1) * 8 + r) * WG_LD + wn + (mi >> 1) * 8];
                ldmatrix_x4_trans(b0, b1, b2, b3, pb);
            }
            mma_bf16(acc[0], a0, a1, a2, a3, b0, b1);
            mma_bf16(acc[1], a0, a1, a2, a3, b2, b3);
        }
        __syncthreads();
    }
    const int g = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 2; nt++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int co = co0 + wm + g + h * 8;
            const int ci = ci0 + wn + nt * 8 + tg * 2;
            if (co >= a.Cout) continue;
            float *d = a.dw + ((size_t)co * 9 + tap) * Cin + ci;
            atomicAdd(d, acc[nt][h * 2]);
            atomicAdd(d + 1, acc[nt][h * 2 + 1]);
        }
    if (a.dbias && tap == 4 && cib == 0 && tid < WG_CO && co0 + tid < a.Cout) atomicAdd(&a.dbias[co0 + tid], bsum);
}

// --------------------------------------------------------- small kernels
// w'[ci][tap'][co] = w[co][8 - tap'][ci]  (data-gradient weights)
__global__ void flip_weights_kernel(const bf16 *w, bf16 *wt, int Cout, int Cin)
{
    const size_t n = (size_t)Cout * 9 * Cin;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int ci = (int)(e % Cin);
        const int tap = (int)((e / Cin) % 9);
        const int co = (int)(e / ((size_t)Cin * 9));
        wt[((size_t)ci * 9 + (8 - tap)) * Cout + co] = w[e];
    }
}

__global__ void relu_bwd_kernel(const bf16 *y, const bf16 *dy, bf16 *dpre, size_t n)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        dpre[e] = __bfloat162float(y[e]) > 0.f ? dy[e] : __float2bfloat16(0.f);
}

// Eight elements per thread as 16-byte vectors (n % 8 == 0, 16-byte aligned):
// the same selection, decided on the bits (y > 0 <=> sign clear and nonzero).
__global__ void relu_bwd_v8_kernel(const uint4 *y, const uint4 *dy, uint4 *dpre, size_t n8)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n8; e += (size_t)gridDim.x * blockDim.x) {
        const uint4 a = y[e], g = dy[e];
        const uint32_t av[4] = {a.x, a.y, a.z, a.w}, gv[4] = {g.x, g.y, g.z, g.w};
        uint32_t o[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int16_t lo = (int16_t)(av[q] & 0xffffu), hi = (int16_t)(av[q] >> 16);
            o[q] = (lo > 0 ? (gv[q] & 0xffffu) : 0u) | (hi > 0 ? (gv[q] & 0xffff0000u) : 0u);
        }
        dpre[e] = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

// 2x2 average pooling, NHWC
__global__ void pool_fwd_kernel(const bf16 *x, bf16 *y, int N, int H, int W, int C)
{
    const int Ho = H / 2, Wo = W / 2;
    const size_t n = (size_t)N * Ho * Wo * C;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t pix = e / C;
        const int xo = (int)(pix % Wo), yo = (int)((pix / Wo) % Ho), b = (int)(pix / ((size_t)Wo * Ho));
        const size_t base = (((size_t)b * H + 2 * yo) * W + 2 * xo) * C + c;
        const float s = __bfloat162float(x[base]) + __bfloat162float(x[base + C]) +
                        __bfloat162float(x[base + (size_t)W * C]) + __bfloat162float(x[base + (size_t)W * C + C]);
        y[e] = __float2bfloat16(0.25f * s);
    }
}

__global__ void pool_bwd_kernel(const bf16 *dy, bf16 *dx, int N, int H, int W, int C)
{
    // dx[b][y][x][c] = 0.25 * dy[b][y/2][x/2][c]
    const size_t n = (size_t)N * H * W * C;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t pix = e / C;
        const int x = (int)(pix % W), y = (int)((pix / W) % H), b = (int)(pix / ((size_t)W * H));
        dx[e] = __float2bfloat16(0.25f * __bfloat162float(dy[(((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]));
    }
}

// nearest 2x upsampling (H, W = input size)
__global__ void up_fwd_kernel(const bf16 *x, bf16 *y, int N, int H, int W, int C)
{
    const size_t n = (size_t)N * 4 * H * W * C;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t pix = e / C;
        const int X = (int)(pix % (2 * W)), Y = (int)((pix / (2 * W)) % (2 * H)), b = (int)(pix / ((size_t)4 * W * H));
        y[e] = x[(((size_t)b * H + Y / 2) * W + X / 2) * C + c];
    }
}

__global__ void up_bwd_kernel(const bf16 *dy, bf16 *dx, int N, int H, int W, int C)
{
    const size_t n = (size_t)N * H * W * C;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t pix = e / C;
        const int x = (int)(pix % W), y = (int)((pix / W) % H), b = (int)(pix / ((size_t)W * H));
        const size_t base = (((size_t)b * 2 * H + 2 * y) * 2 * W + 2 * x) * C + c;
        const size_t rs = (size_t)2 * W * C;
        dx[e] = __float2bfloat16(__bfloat162float(dy[base]) + __bfloat162float(dy[base + C]) +
                                 __bfloat162float(dy[base + rs]) + __bfloat162float(dy[base + rs + C]));
    }
}

// Vectorised forms of the pooling / upsampling passes: one thread per (pixel,
// group of 8 channels), 16-byte loads and stores, 32-bit index arithmetic
// (used when every element index fits in 31 bits; C a multiple of 8).
__device__ __forceinline__ void bf8_to_f(const uint4 v, float *f)
{
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 t = __bfloat1622float2(h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}

__device__ __forceinline__ uint4 f_to_bf8(const float *f)
{
    uint4 v;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&v);
#pragma unroll
    for (int i = 0; i < 4; i++) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    return v;
}

__global__ void pool_fwd_v8_kernel(const bf16 *x, bf16 *y, int N, int H, int W, int C)
{
    const int Ho = H / 2, Wo = W / 2, G = C / 8;
    const unsigned n = (unsigned)N * Ho * Wo * G;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const unsigned g = e % G, pix = e / G;
        const unsigned xo = pix % Wo, r = pix / Wo, yo = r % Ho, b = r / Ho;
        const bf16 *p = x + ((size_t)(b * H + 2 * yo) * W + 2 * xo) * C + 8 * g;
        float a[8], t[8];
        bf8_to_f(*reinterpret_cast<const uint4 *>(p), a);
        bf8_to_f(*reinterpret_cast<const uint4 *>(p + C), t);
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] += t[i];
        bf8_to_f(*reinterpret_cast<const uint4 *>(p + (size_t)W * C), t);
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] += t[i];
        bf8_to_f(*reinterpret_cast<const uint4 *>(p + (size_t)W * C + C), t);
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] = 0.25f * (a[i] + t[i]);
        *reinterpret_cast<uint4 *>(y + (size_t)pix * C + 8 * g) = f_to_bf8(a);
    }
}

__global__ void pool_bwd_v8_kernel(const bf16 *dy, bf16 *dx, int N, int H, int W, int C)
{
    const int G = C / 8;
    const unsigned n = (unsigned)N * H * W * G;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const unsigned g = e % G, pix = e / G;
        const unsigned xx = pix % W, r = pix / W, yy = r % H, b = r / H;
        float a[8];
        bf8_to_f(*reinterpret_cast<const uint4 *>(dy + ((size_t)(b * (H / 2) + yy / 2) * (W / 2) + xx / 2) * C + 8 * g),
                 a);
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] *= 0.25f;
        *reinterpret_cast<uint4 *>(dx + (size_t)pix * C + 8 * g) = f_to_bf8(a);
    }
}

__global__ void up_fwd_v8_kernel(const bf16 *x, bf16 *y, int N, int H, int W, int C)
{
    const int G = C / 8;
    const unsigned n = (unsigned)N * 4 * H * W * G;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const unsigned g = e % G, pix = e / G;
        const unsigned X = pix % (2 * W), r = pix / (2 * W), Y = r % (2 * H), b = r / (2 * H);
        *reinterpret_cast<uint4 *>(y + (size_t)pix * C + 8 * g) =
            *reinterpret_cast<const uint4 *>(x + ((size_t)(b * H + Y / 2) * W + X / 2) * C + 8 * g);
    }
}

__global__ void up_bwd_v8_kernel(const bf16 *dy, bf16 *dx, int N, int H, int W, int C)
{
    const int G = C / 8;
    const unsigned n = (unsigned)N * H * W * G;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const unsigned g = e % G, pix = e / G;
        const unsigned xx = pix % W, r = pix / W, yy = r % H, b = r / H;
        const bf16 *p = dy + ((size_t)(b * 2 * H + 2 * yy) * 2 * W + 2 * xx) * C + 8 * g;
        const size_t rs = (size_t)2 * W * C;
        float a[8], t[8];
        bf8_to_f(*reinterpret_cast<const uint4 *>(p), a);
        bf8_to_f(*reinterpret_cast<const uint4 *>(p + C), t);
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] += t[i];
        bf8_to_f(*reinterpret_cast<const uint4 *>(p + rs), t);
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] += t[i];
        bf8_to_f(*reinterpret_cast<const uint4 *>(p + rs + C), t);
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] += t[i];
        *reinterpret_cast<uint4 *>(dx + (size_t)pix * C + 8 * g) = f_to_bf8(a);
    }
}

// input packing, one thread per pixel: channel 0 = scaled image, the rest zero
__global__ void input_pack_v8_kernel(const float *img, const float *scale, bf16 *x, int N, int HW, int C)
{
    const unsigned n = (unsigned)N * HW;
    for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        float f[8] = {img[p] * scale[p / HW], 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        uint4 *dst = reinterpret_cast<uint4 *>(x + (size_t)p * C);
        dst[0] = f_to_bf8(f);
        for (int g = 1; g < C / 8; g++) dst[g] = make_uint4(0, 0, 0, 0);
    }
}

// The network's first layer for inference, from the image itself: the input
// has one channel (image x scale, rounded to BF16 as the packed input is),
// so the 3x3 convolution to 32 channels with bias and ReLU is nine FP32
// multiply-adds per output channel -- no 32-channel input of which 31 are
// zero, no tensor-core pass over them.  Weights [32][3][3][Cin]: channel 0 of
// each tap is used (the others multiply zero inputs).  One CTA per 32 x 8
// output pixels and image; one thread per pixel, 32 channels, 64-byte stores.
__global__ void __launch_bounds__(256) input_conv_kernel(const float *__restrict__ img,
                                                         const float *__restrict__ scale, const bf16 *__restrict__ w,
                                                         const float *__restrict__ b, bf16 *__restrict__ y, int H,
                                                         int W, int Cin)
{
    __shared__ float xs[10][34];   // input rows y0-1 .. y0+8, columns x0-1 .. x0+32
    __shared__ float ws[9][32];    // w[co][tap][0]
    __shared__ float bs[32];
    const int n = blockIdx.z, x0 = blockIdx.x * 32, y0 = blockIdx.y * 8;
    const float sc = scale[n];
    for (int i = threadIdx.x; i < 10 * 34; i += blockDim.x) {
        const int r = i / 34, c = i - r * 34, gy = y0 + r - 1, gx = x0 + c - 1;
        float v = 0.f;
        if (gy >= 0 && gy < H && gx >= 0 && gx < W)
            v = __bfloat162float(__float2bfloat16(img[((size_t)n * H + gy) * W + gx] * sc));
        xs[r][c] = v;
    }
    for (int i = threadIdx.x; i < 9 * 32; i += blockDim.x) {
        const int t = i >> 5, co = i & 31;
        ws[t][co] = __bfloat162float(w[((size_t)co * 9 + t) * Cin]);
    }
    if (threadIdx.x < 32) bs[threadIdx.x] = b[threadIdx.x];
    __syncthreads();
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    const int gx = x0 + lx, gy = y0 + ly;
    if (gx >= W || gy >= H) return;
    float xv[9];
#pragma unroll
    for (int t = 0; t < 9; t++) xv[t] = xs[ly + t / 3][lx + t % 3];
    uint4 *dst = reinterpret_cast<uint4 *>(y + (((size_t)n * H + gy) * W + gx) * 32);
#pragma unroll
    for (int g = 0; g < 4; g++) {
        float f[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int co = 8 * g + j;
            float acc = 0.f;
#pragma unroll
            for (int t = 0; t < 9; t++) acc = fmaf(xv[t], ws[t][co], acc);
            f[j] = fmaxf(acc + bs[co], 0.f);
        }
        dst[g] = f_to_bf8(f);
    }
}

// The first layer's weight and bias gradients in training, from the image
// itself: only channel 0 of its input carries data, so
//   dw[co][tap][0] = sum_p dpre[p][co] x[p + tap],   db[co] = sum_p dpre[p][co]
// with x = bf16(img x scale) (zero outside the image).  Pass 1: one CTA per
// image row, 320 threads = 288 (tap, channel) sums + 32 bias sums over the
// row's pixels, staged in shared memory; partial sums [row][320].  Pass 2:
// one CTA per output, the rows' partials summed in a fixed order, so the
// result does not depend on scheduling.
__global__ void __launch_bounds__(320) input_wgrad_rows_kernel(const float *__restrict__ img,
                                                               const float *__restrict__ scale,
                                                               const bf16 *__restrict__ dpre, float *__restrict__ part,
                                                               int H, int W)
{
    extern __shared__ __align__(16) unsigned char smem_iw[];
    bf16 *ds = reinterpret_cast<bf16 *>(smem_iw);                          // [W][32]
    float *xs = reinterpret_cast<float *>(smem_iw + (size_t)W * 64);      // [3][W + 2]
    const int y = blockIdx.x, n = blockIdx.y, W2 = W + 2;
    const float sc = scale[n];
    const uint4 *src = reinterpret_cast<const uint4 *>(dpre + ((size_t)n * H + y) * W * 32);
    uint4 *dst = reinterpret_cast<uint4 *>(ds);
    for (int i = threadIdx.x; i < W * 4; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < 3 * W2; i += blockDim.x) {
        const int r = i / W2, c = i - r * W2, gy = y + r - 1, gx = c - 1;
        float v = 0.f;
        if (gy >= 0 && gy < H && gx >= 0 && gx < W)
            v = __bfloat162float(__float2bfloat16(img[((size_t)n * H + gy) * W + gx] * sc));
        xs[i] = v;
    }
    __syncthreads();
    const int t = threadIdx.x, co = t & 31;
    float acc = 0.f;
    if (t < 288) {
        const int tap = t >> 5, ky = tap / 3, kx = tap - 3 * ky;
        const float *xr = xs + ky * W2 + kx;
        for (int px = 0; px < W; px++) acc = fmaf(__bfloat162float(ds[px * 32 + co]), xr[px], acc);
    } else {
        for (int px = 0; px < W; px++) acc += __bfloat162float(ds[px * 32 + co]);
    }
    part[((size_t)n * H + y) * 320 + t] = acc;
}

__global__ void __launch_bounds__(256) input_wgrad_reduce_kernel(const float *__restrict__ part, int nrows,
                                                                 float *__restrict__ dw, int Cin,
                                                                 float *__restrict__ db)
{
    __shared__ float red[256];
    const int t = blockIdx.x;   // output: (tap, channel) t < 288, bias t - 288
    float s = 0.f;
    for (int r = threadIdx.x; r < nrows; r += blockDim.x) s += part[(size_t)r * 320 + t];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (t < 288) dw[((size_t)(t & 31) * 9 + (t >> 5)) * Cin] = red[0];
        else db[t - 288] = red[0];
    }
}

// head, one thread per pixel with 16-byte channel loads (C <= 64, weights in shared memory)
__global__ void head_fwd_v8_kernel(const bf16 *h, const float *w, const float *b, const float *img,
                                   const float *scale, float *out, int N, int HW, int C)
{
    __shared__ float ws[64];
    for (int c = threadIdx.x; c < C; c += blockDim.x) ws[c] = w[c];
    __syncthreads();
    const unsigned n = (unsigned)N * HW;
    const float b0 = b[0];
    for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        float s = b0;
        const uint4 *src = reinterpret_cast<const uint4 *>(h + (size_t)p * C);
        for (int g = 0; g < C / 8; g++) {
            float f[8];
            bf8_to_f(src[g], f);
#pragma unroll
            for (int i = 0; i < 8; i++) s += f[i] * ws[8 * g + i];
        }
        out[p] = img[p] * scale[p / HW] + s;
    }
}

static bool fits31(size_t n) { return n < ((size_t)1 << 31); }

// input image (FP32 [N][H][W], scaled) -> BF16 NHWC with C channels, channel 0 = image
__global__ void input_pack_kernel(const float *img, const float *scale, bf16 *x, int N, int H, int W, int C)
{
    const size_t n = (size_t)N * H * W * C;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t pix = e / C;
        const int b = (int)(pix / ((size_t)H * W));
        x[e] = __float2bfloat16(c == 0 ? img[pix] * scale[b] : 0.f);
    }
}

// head: out[p] = inp[p] + sum_c h[p][c] * w[c] + b   (FP32 out; residual on the scaled input)
__global__ void head_fwd_kernel(const bf16 *h, const float *w, const float *b, const float *img, const float *scale,
                                float *out, int N, int HW, int C)
{
    const size_t n = (size_t)N * HW;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        float s = b[0];
        for (int c = 0; c < C; c++) s += __bfloat162float(h[p * C + c]) * w[c];
        out[p] = img[p] * scale[p / HW] + s;
    }
}

// MSE loss gradient on the head output: g = 2 (out - target*scale) / count; loss partial sums in FP64
__global__ void mse_grad_kernel(const float *out, const float *target, const float *scale, float *g, double *loss,
                                int N, int HW)
{
    const size_t n = (size_t)N * HW;
    double part = 0.0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const float d = out[p] - target[p] * scale[p / HW];
        g[p] = 2.f * d / (float)n;
        part += (double)d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, part / (double)n);
}

// head backward: dh[p][c] = g[p] * w[c]; dw[c] += sum_p g[p] h[p][c]; db += sum g
__global__ void head_bwd_kernel(const bf16 *h, const float *w, const float *g, bf16 *dh, float *dw, float *db, int N,
                                int HW, int C)
{
    const size_t n = (size_t)N * HW;
    float lw[64];
    for (int c = 0; c < C; c++) lw[c] = 0.f;
    float lb = 0.f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const float gp = g[p];
        lb += gp;
        for (int c = 0; c < C; c++) {
            dh[p * C + c] = __float2bfloat16(gp * w[c]);
            lw[c] += gp * __bfloat162float(h[p * C + c]);
        }
    }
    for (int c = 0; c < C; c++) {
        float v = lw[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&dw[c], v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lb += __shfl_xor_sync(0xffffffffu, lb, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(db, lb);
}

// The same with 16-byte vectors: a thread owns one 8-channel group of a pixel
// (G = C / 8 groups per pixel, G a power of two <= 8), so its weights and
// partial sums stay in registers; the grid stride is a multiple of 256 and so
// of G, which keeps each thread on one group.  Partial sums meet in shared
// memory before one atomic per channel per block.
__global__ void __launch_bounds__(256) head_bwd_v8_kernel(const uint4 *h, const float *w, const float *g, uint4 *dh,
                                                          float *dw, float *db, size_t npix, int G)
{
    __shared__ float part[8][65];
    const int lg = __ffs(G) - 1;
    const size_t e0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, n = npix << lg;
    const int c8 = threadIdx.x & (G - 1), lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float wr[8], lw[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        wr[j] = w[8 * c8 + j];
        lw[j] = 0.f;
    }
    float lb = 0.f;
    for (size_t e = e0; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const float gp = g[e >> lg];
        if (c8 == 0) lb += gp;
        const uint4 v = h[e];
        const __nv_bfloat162 *hh = reinterpret_cast<const __nv_bfloat162 *>(&v);
        uint4 o;
        __nv_bfloat162 *oo = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float2 f = __bfloat1622float2(hh[q]);
            lw[2 * q] += gp * f.x;
            lw[2 * q + 1] += gp * f.y;
            oo[q] = __floats2bfloat162_rn(gp * wr[2 * q], gp * wr[2 * q + 1]);
        }
        dh[e] = o;
    }
#pragma unroll
    for (int j = 0; j < 8; j++)
        for (int o = G; o < 32; o <<= 1) lw[j] += __shfl_xor_sync(0xffffffffu, lw[j], o);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lb += __shfl_xor_sync(0xffffffffu, lb, o);
    if (lane < G) {
#pragma unroll
        for (int j = 0; j < 8; j++) part[warp][8 * lane + j] = lw[j];
    }
    if (lane == 0) part[warp][64] = lb;
    __syncthreads();
    const int C = 8 * G, nw = blockDim.x >> 5;
    if (threadIdx.x <= C) {
        const int c = threadIdx.x < C ? threadIdx.x : 64;
        float v = 0.f;
        for (int k = 0; k < nw; k++) v += part[k][c];
        atomicAdd(threadIdx.x < C ? &dw[c] : db, v);
    }
}

// Adam on FP32 master weights; writes the BF16 compute copy (wb may be null)
__global__ void adam_kernel(float *w, float *m, float *v, const float *g, bf16 *wb, size_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[e];
        const float mi = b1 * m[e] + (1.f - b1) * gi;
        const float vi = b2 * v[e] + (1.f - b2) * gi * gi;
        m[e] = mi;
        v[e] = vi;
        const float wi = w[e] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[e] = wi;
        if (wb) wb[e] = __float2bfloat16(wi);
    }
}

__global__ void add_bf16_kernel(bf16 *y, const bf16 *x, size_t n)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        y[e] = __float2bfloat16(__bfloat162float(y[e]) + __bfloat162float(x[e]));
}

__global__ void add_bf16_v8_kernel(uint4 *y, const uint4 *x, size_t n8)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n8; e += (size_t)gridDim.x * blockDim.x) {
        uint4 a = y[e];
        const uint4 b = x[e];
        __nv_bfloat162 *pa = reinterpret_cast<__nv_bfloat162 *>(&a);
        const __nv_bfloat162 *pb = reinterpret_cast<const __nv_bfloat162 *>(&b);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float2 fa = __bfloat1622float2(pa[q]), fb = __bfloat1622float2(pb[q]);
            pa[q] = __floats2bfloat162_rn(fa.x + fb.x, fa.y + fb.y);
        }
        y[e] = a;
    }
}

__global__ void f32_to_bf16_kernel(const float *a, bf16 *b, size_t n)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        b[e] = __float2bfloat16(a[e]);
}

static int grid_for(size_t n)
{
    size_t g = (n + 255) / 256;
    return (int)(g > 148 * 32 ? 148 * 32 : (g == 0 ? 1 : g));
}

}  // namespace raft

using namespace raft;

// ------------------------------------------------------------------ C ABI
extern "C" {

// Which kernel runs the 3x3 convolution: 0 = the tcgen05/TMA kernel (unet_tc.cu)
// wherever its tile fits (W >= 128 or W dividing 128), else the mma.sync kernel;
// 1 = the mma.sync kernel only (kept for other widths and for comparison);
// 2 = the tcgen05 kernel only (a shape it does not take is an error).
static int g_conv_path = 0;

int raft_unet_set_conv_path(int path)
{
    if (path < 0 || path > 2) return 1;
    g_conv_path = path;
    return 0;
}

// Halo tiles of the tcgen05 convolution for its 32 -> 32 channel layers (1, the
// default) or the per-tap operand tiles for every layer (0).
int raft_unet_set_conv_halo(int on)
{
    conv3x3_tc_set_halo(on);
    return 0;
}

// Nine-tap CTAs of the tcgen05 weight gradient where Cout <= 128 (1, the
// default) or 128-row blocks of (tap, channel) for every layer (0).
int raft_unet_set_wgrad_nine(int on)
{
    conv3x3_wgrad_tc_set_nine(on);
    return 0;
}

// 1 if a bounded wait of the tcgen05 convolution ran out since the last call
// (the flag is cleared); synchronises the current device.
int raft_unet_conv_error(void) { return conv3x3_tc_error(); }

// y = act(conv3x3(concat(x0, x1)) + bias); C0, C1, Cout multiples of 32 (C1 may be 0).
// With y1 != NULL the output channels are split: [0, Cy0) -> y, [Cy0, Cout) -> y1
// (the data gradient of a concatenated input, back into its two parts).
int raft_unet_conv_fwd(const void *x0, int C0, const void *x1, int C1, const void *w, const float *bias, void *y,
                       void *y1, int Cy0, int N, int H, int W, int Cout, int relu, void *stream)
{
    if (C0 % 32 || C1 % 32 || Cout % 32 || N < 1 || H < 1 || W < 1) return 1;
    if (y1 && (Cy0 % 32 || Cy0 <= 0 || Cy0 >= Cout)) return 1;
    if (g_conv_path != 1) {
        const int rc = conv3x3_tc(x0, C0, x1, C1, w, bias, y, y1, Cy0, N, H, W, Cout, relu, (cudaStream_t)stream);
        if (rc != 2) return rc;
        if (g_conv_path == 2) return 1;
    }
    ConvArgs a{(const bf16 *)x0, (const bf16 *)x1, C0, C1, (const bf16 *)w, bias, (bf16 *)y, (bf16 *)y1, Cy0,
               N, H, W, Cout, relu};
    dim3 grid((unsigned)((size_t)N * H * ((W + CV_PIX - 1) / CV_PIX)), Cout / CV_CO);
    count_launch();
    conv3x3_fwd_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// dW += sum_p dY[p] x[p+tap] (FP32), dbias += sum_p dY[p] (if non-null).
int raft_unet_conv_wgrad(const void *dy, const void *x0, int C0, const void *x1, int C1, float *dw, float *dbias,
                         int N, int H, int W, int Cout, void *stream)
{
    if (C0 % 32 || C1 % 32 || Cout % 32) return 1;
    if (g_conv_path != 1) {
        const int rc = conv3x3_wgrad_tc(dy, x0, C0, x1, C1, dw, dbias, N, H, W, Cout, (cudaStream_t)stream);
        if (rc != 2) return rc;
        if (g_conv_path == 2) return 1;
    }
    const int Cin = C0 + C1;
    const long total = (long)N * H * W;
    const int ppc = 2048;
    WgradArgs a{(const bf16 *)dy, (const bf16 *)x0, (const bf16 *)x1, C0, C1, dw, dbias, N, H, W, Cout, ppc};
    dim3 grid((unsigned)(9 * (Cin / WG_CI) * (Cout / WG_CO)), (unsigned)((total + ppc - 1) / ppc));
    count_launch();
    conv3x3_wgrad_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_flip_weights(const void *w, void *wt, int Cout, int Cin, void *stream)
{
    const size_t n = (size_t)Cout * 9 * Cin;
    count_launch();
    flip_weights_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const bf16 *)w, (bf16 *)wt, Cout, Cin);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_relu_bwd(const void *y, const void *dy, void *dpre, size_t n, void *stream)
{
    count_launch();
    if (n % 8 == 0 && ((uintptr_t)y | (uintptr_t)dy | (uintptr_t)dpre) % 16 == 0)
        relu_bwd_v8_kernel<<<grid_for(n / 8), 256, 0, (cudaStream_t)stream>>>(
            (const uint4 *)y, (const uint4 *)dy, (uint4 *)dpre, n / 8);
    else
        relu_bwd_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const bf16 *)y, (const bf16 *)dy,
                                                                       (bf16 *)dpre, n);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_pool(int backward, const void *src, void *dst, int N, int H, int W, int C, void *stream)
{
    count_launch();
    if (C % 8 == 0 && fits31((size_t)N * H * W * C)) {
        if (!backward)
            pool_fwd_v8_kernel<<<grid_for((size_t)N * H * W * C / 32), 256, 0, (cudaStream_t)stream>>>(
                (const bf16 *)src, (bf16 *)dst, N, H, W, C);
        else
            pool_bwd_v8_kernel<<<grid_for((size_t)N * H * W * C / 8), 256, 0, (cudaStream_t)stream>>>(
                (const bf16 *)src, (bf16 *)dst, N, H, W, C);
        return cudaGetLastError() == cudaSuccess ? 0 : 1;
    }
    if (!backward)
        pool_fwd_kernel<<<grid_for((size_t)N * H * W * C / 4), 256, 0, (cudaStream_t)stream>>>((const bf16 *)src,
                                                                                                (bf16 *)dst, N, H, W, C);
    else
        pool_bwd_kernel<<<grid_for((size_t)N * H * W * C), 256, 0, (cudaStream_t)stream>>>((const bf16 *)src,
                                                                                            (bf16 *)dst, N, H, W, C);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// H, W: the low-resolution size
int raft_unet_upsample(int backward, const void *src, void *dst, int N, int H, int W, int C, void *stream)
{
    count_launch();
    if (C % 8 == 0 && fits31((size_t)N * 4 * H * W * C)) {
        if (!backward)
            up_fwd_v8_kernel<<<grid_for((size_t)N * 4 * H * W * C / 8), 256, 0, (cudaStream_t)stream>>>(
                (const bf16 *)src, (bf16 *)dst, N, H, W, C);
        else
            up_bwd_v8_kernel<<<grid_for((size_t)N * H * W * C / 8), 256, 0, (cudaStream_t)stream>>>(
                (const bf16 *)src, (bf16 *)dst, N, H, W, C);
        return cudaGetLastError() == cudaSuccess ? 0 : 1;
    }
    if (!backward)
        up_fwd_kernel<<<grid_for((size_t)N * 4 * H * W * C), 256, 0, (cudaStream_t)stream>>>(
            (const bf16 *)src, (bf16 *)dst, N, H, W, C);
    else
        up_bwd_kernel<<<grid_for((size_t)N * H * W * C), 256, 0, (cudaStream_t)stream>>>((const bf16 *)src,
                                                                                          (bf16 *)dst, N, H, W, C);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_input(const float *img, const float *scale, void *x, int N, int H, int W, int C, void *stream)
{
    count_launch();
    if (C % 8 == 0 && fits31((size_t)N * H * W * C)) {
        input_pack_v8_kernel<<<grid_for((size_t)N * H * W), 256, 0, (cudaStream_t)stream>>>(img, scale, (bf16 *)x, N,
                                                                                             H * W, C);
        return cudaGetLastError() == cudaSuccess ? 0 : 1;
    }
    input_pack_kernel<<<grid_for((size_t)N * H * W * C), 256, 0, (cudaStream_t)stream>>>(img, scale, (bf16 *)x, N, H,
                                                                                        W, C);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_input_conv(const float *img, const float *scale, const void *w, int Cin, const float *bias, void *y,
                         int N, int H, int W, void *stream)
{
    if (N <= 0 || H <= 0 || W <= 0 || Cin < 1 || ((uintptr_t)y % 16) != 0) return 1;
    count_launch();
    const dim3 grid((W + 31) / 32, (H + 7) / 8, N);
    input_conv_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(img, scale, (const bf16 *)w, bias, (bf16 *)y, H, W,
                                                              Cin);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_input_wgrad(const float *img, const float *scale, const void *dpre, float *dw, int Cin, float *db,
                          float *work, size_t work_floats, int N, int H, int W, void *stream)
{
    const size_t rows = (size_t)N * H, smem = (size_t)W * 64 + (size_t)3 * (W + 2) * sizeof(float);
    if (N <= 0 || H <= 0 || W <= 0 || Cin < 1 || work_floats < rows * 320 || smem > 200 * 1024 ||
        ((uintptr_t)dpre % 16) != 0)
        return 1;
    // set at every call: the size depends on W
    if (cudaFuncSetAttribute(input_wgrad_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 1;
    count_launch();
    input_wgrad_rows_kernel<<<dim3(H, N), 320, smem, (cudaStream_t)stream>>>(img, scale, (const bf16 *)dpre, work, H,
                                                                          W);
    count_launch();
    input_wgrad_reduce_kernel<<<320, 256, 0, (cudaStream_t)stream>>>(work, (int)rows, dw, Cin, db);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_head(int backward, const void *h, const float *w, const float *b, const float *img,
                   const float *scale, float *out_or_grad, void *dh, float *dw, float *db, int N, int HW, int C,
                   void *stream)
{
    if (C > 64) return 1;
    count_launch();
    if (!backward && C % 8 == 0 && fits31((size_t)N * HW * C)) {
        head_fwd_v8_kernel<<<grid_for((size_t)N * HW), 256, 0, (cudaStream_t)stream>>>((const bf16 *)h, w, b, img, scale,
                                                                                       out_or_grad, N, HW, C);
        return cudaGetLastError() == cudaSuccess ? 0 : 1;
    }
    if (!backward)
        head_fwd_kernel<<<grid_for((size_t)N * HW), 256, 0, (cudaStream_t)stream>>>((const bf16 *)h, w, b, img, scale,
                                                                                    out_or_grad, N, HW, C);
    else if (C % 8 == 0 && C <= 64 && ((C / 8) & (C / 8 - 1)) == 0 && ((uintptr_t)h | (uintptr_t)dh) % 16 == 0)
        head_bwd_v8_kernel<<<grid_for((size_t)N * HW * (C / 8)), 256, 0, (cudaStream_t)stream>>>(
            (const uint4 *)h, w, out_or_grad, (uint4 *)dh, dw, db, (size_t)N * HW, C / 8);
    else
        head_bwd_kernel<<<grid_for((size_t)N * HW), 256, 0, (cudaStream_t)stream>>>((const bf16 *)h, w, out_or_grad,
                                                                                    (bf16 *)dh, dw, db, N, HW, C);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_mse(const float *out, const float *target, const float *scale, float *grad, double *loss, int N, int HW,
                  void *stream)
{
    count_launch();
    mse_grad_kernel<<<grid_for((size_t)N * HW), 256, 0, (cudaStream_t)stream>>>(out, target, scale, grad, loss, N, HW);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_adam(float *w, float *m, float *v, const float *g, void *wb, size_t n, float lr, float b1, float b2,
                   float eps, int step, void *stream)
{
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    count_launch();
    adam_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, m, v, g, (bf16 *)wb, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_add(void *y, const void *x, size_t n, void *stream)
{
    count_launch();
    if (n % 8 == 0 && ((uintptr_t)y | (uintptr_t)x) % 16 == 0)
        add_bf16_v8_kernel<<<grid_for(n / 8), 256, 0, (cudaStream_t)stream>>>((uint4 *)y, (const uint4 *)x, n / 8);
    else
        add_bf16_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((bf16 *)y, (const bf16 *)x, n);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int raft_unet_to_bf16(const float *a, void *b, size_t n, void *stream)
{
    count_launch();
    f32_to_bf16_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(a, (bf16 *)b, n);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // extern "C"
