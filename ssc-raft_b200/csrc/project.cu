// project.cu -- the ray-driven parallel-beam projectors.
//
// Reference kernels restated (cnpem/ssc-raft):
//   * Radon_RT_version_sscRadon, cuda/src/geometries/parallel/forward_methods/radon_rt.cu:131-174
//       dx = 2ax/(nx-1), dy = 2ay/(ny-1), t = -ax + i*dx, for r < ny:
//       s = -ay + r*dy, (x, y) = (t c - s s_, t s_ + s c),
//       sum img[(int)((y+1)/dy)][(int)((x+1)/dx)], out = sum*dy
//   * kernel_radon, em_RT_kernel.cu:145-185 (EM forward; one step dt = 2/(nrays-1)
//     for rays, samples and pixels), with the EM epilogues fused:
//       tEM  kernel_flatTimesExp (em_RT_kernel.cu:20-32): q = flat * exp(-p)
//       eEM  kernel_radonWithDivision (em_RT_kernel.cu:188-246):
//            q = max(0, y * SIGN(p) / sqrt(1e-8 + p^2))
//     and the angle step folded in, written straight into the window rows
//     the EM backprojector stages.  Optional FP64 reductions (data residual,
//     Poisson log-likelihood) are accumulated per slice in the same pass.
//
// The sample positions and indices are computed with the reference's FP32
// expressions (this file is compiled with fast math, as the reference is),
// so the nearest-pixel choice is the reference's.  The multiply-adds are
// written out (t = i*d - a, x = t*c - s*sin, y = t*sin + s*c as single-rounding
// fmaf with the product s*sin / s*c rounded first -- the contraction the
// reference build produces) so that no template instance can contract them
// differently.
#include "raft.hpp"
#include "profile.hpp"

#include <cstdlib>
#include <type_traits>

namespace raft {

constexpr int PJ_WARPS = 8;   // 256 threads per block

// Thread -> (ray, angle, sample phase) shapes.  A warp covers RW neighbouring
// rays at AW = 32 / (RW PH) neighbouring angles, each ray's samples split over
// PH lanes (lane ph sums samples m = ph, ph + PH, ... in order; the PH partial
// sums are then combined by a fixed butterfly of warp shuffles, so the
// summation order depends on PH alone, not on the slice count, the layout or
// the ray/angle shape); a block covers BR rays x BA angles.  The lanes of a
// warp load their samples together.  With one angle and one phase per warp
// (RW = 32) the 32 pixels lie on a line across the ray direction, one pixel
// apart: along an image row near 0 degrees, but on ~23 different rows near 45
// degrees.  A few rays x a few consecutive samples cover a compact
// parallelogram instead (about 12 cache lines per warp load of 32-byte pixels
// against 15-17 for the line, averaged over angles).  Measured (B200, 512 x
// 1024^2 x 900): interleaved 8-slice images four rays x four phases x two
// angles, Radon 5096 GUPS against 4655 for one angle x 32 rays, tEM 176.7
// against 182.1 ms per iteration; planar single-slice projection (instruction
// issue bound) is best sequential (ragged batch 1863 GUPS) and costs 3.7 % at
// PH = 4 (eight rays x four phases, 1795 GUPS), kept so that every slice count
// sums in the same order.
template <int RW, int PH, int BRS> struct PjShape {
    static_assert(32 % (RW * PH) == 0, "a warp holds whole (ray, phase) groups");
    static constexpr int AW = 32 / (RW * PH);     // angles per warp
    static constexpr int BR = BRS;                // rays per block
    static constexpr int BA = 256 / (BR * PH);    // angles per block
    static constexpr int WR = BR / RW;            // warps along the rays
    static_assert(BR % RW == 0 && BA % AW == 0 && WR * (BA / AW) == 8, "eight warps per block");
};

// S slices per thread share every sample's position and pixel index (the
// geometry is the same for all slices).  Warps whose angle is steeper than
// 45 degrees read a transposed copy of the images (imgT[x][y]) so that the
// 32 rays of the warp touch consecutive addresses; the index arithmetic and
// therefore the chosen pixels are unchanged.  IL = 1 (S = 8) reads the
// slice-interleaved copies instead (il[g][y][x][8], ilT[g][x][y][8]): one
// sample's eight slice values are one 32-byte load (one sector).
// 256-bit read-only load of eight consecutive floats (32-byte aligned)
__device__ __forceinline__ void ldg_v8(const float *p, float (&w)[8])
{
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(w[0]), "=f"(w[1]), "=f"(w[2]), "=f"(w[3]), "=f"(w[4]), "=f"(w[5]), "=f"(w[6]), "=f"(w[7])
                 : "l"(p));
}

template <int EM, int EPI, int S, int IL, int RW, int PH, int BRS>
__device__ __forceinline__ void project_block(const ProjLaunch &p, const int bx, const int by, const int bz)
{
    static_assert(!IL || S == 8, "interleaved images hold groups of 8 slices");
    using Sh = PjShape<RW, PH, BRS>;
    const int w = threadIdx.y, lane = threadIdx.x;
    const int ph = lane / (RW * Sh::AW);                                      // sample phase
    const int i = bx * Sh::BR + (w % Sh::WR) * RW + lane % RW;                // ray
    const int j = by * Sh::BA + (w / Sh::WR) * Sh::AW + (lane / RW) % Sh::AW;  // angle
    const int k0 = bz * S;                        // first slice
    const int nsl = min(S, p.nslices - k0);
    const bool valid = (i < p.nrays) && (j < p.nangles);
    const int nx = p.nx, ny = p.ny;
    const size_t plane = (size_t)nx * ny;
    float value[S], linesum[S];
    float step = 0.f;
#pragma unroll
    for (int q = 0; q < S; q++) value[q] = linesum[q] = 0.f;
    if (valid) {
        const float ang = p.angles[j];
        const float ctheta = __cosf(ang);
        const float stheta = __sinf(ang);
        const bool steep = (IL ? p.ilT : p.imgT) && fabsf(stheta) > fabsf(ctheta);
        const float *img = IL ? (steep ? p.ilT : p.il) + (size_t)bz * plane * 8
                              : (steep ? p.imgT : p.img) + (size_t)k0 * plane;
        // address = Y*nx + X (row-major) or X*ny + Y (transposed)
        const int sy = steep ? 1 : nx, sx = steep ? ny : 1;
        // This lane's samples (m = ph, ph + PH, ...) are processed four at a
        // time: the four positions and pixel loads are issued together
        // (independent, so their latency overlaps), then added in sample order.
        auto sample_loop = [&](const float t, const float d0, const float ay0, const float ddx,
                               const float ddy, const int nsamp, const int limx, const int limy) {
            int m = ph;
            for (; m + 3 * PH < nsamp; m += 4 * PH) {
                float v[4][S];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const float s = __fmaf_rn((float)(m + u * PH), d0, -ay0);
                    const float x = __fmaf_rn(t, ctheta, -__fmul_rn(s, stheta));
                    const float y = __fmaf_rn(t, stheta, __fmul_rn(s, ctheta));
                    const int X = (int)((x + 1) / ddx);
                    const int Y = (int)((y + 1) / ddy);
                    if constexpr (IL) {
                        // one 32-byte load: the pixel's eight slice values, or
                        // eight zeros (p.il_zero) for a sample outside the image
                        const bool in = ((unsigned)X < (unsigned)limx) & ((unsigned)Y < (unsigned)limy);
                        const unsigned pix = (unsigned)Y * (unsigned)sy + (unsigned)X * (unsigned)sx;
                        float w[8];
                        ldg_v8(in ? img + (size_t)pix * 8 : p.il_zero, w);
#pragma unroll
                        for (int q = 0; q < 8; q++) v[u][q] = w[q];
                    } else {
                        // 32-bit pixel index (the launch checks nx * ny < 2^32), predicated loads
                        const bool in = ((unsigned)X < (unsigned)limx) & ((unsigned)Y < (unsigned)limy);
                        const unsigned pix = (unsigned)Y * (unsigned)sy + (unsigned)X * (unsigned)sx;
#pragma unroll
                        for (int q = 0; q < S; q++) {
                            float val = 0.f;
                            if (in && q < nsl) val = __ldg(img + q * plane + pix);
                            v[u][q] = val;
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int q = 0; q < S; q++) linesum[q] += v[u][q];
            }
            for (; m < nsamp; m += PH) {
                const float s = __fmaf_rn((float)m, d0, -ay0);
                const float x = __fmaf_rn(t, ctheta, -__fmul_rn(s, stheta));
                const float y = __fmaf_rn(t, stheta, __fmul_rn(s, ctheta));
                const int X = (int)((x + 1) / ddx);
                const int Y = (int)((y + 1) / ddy);
                if (((unsigned)X < (unsigned)limx) & ((unsigned)Y < (unsigned)limy)) {
                    const unsigned pix = (unsigned)Y * (unsigned)sy + (unsigned)X * (unsigned)sx;
                    if constexpr (IL) {
                        float w[8];
                        ldg_v8(img + (size_t)pix * 8, w);
#pragma unroll
                        for (int q = 0; q < S; q++) linesum[q] += w[q];
                    } else {
#pragma unroll
                        for (int q = 0; q < S; q++)
                            if (q < nsl) linesum[q] += __ldg(img + q * plane + pix);
                    }
                }
            }
        };
        if constexpr (EM) {
            // kernel_radon: dt = 2.0*a/(nrays-1) in double, a = 1; one step for
            // rays, samples and pixels; the image is N x N with N = nx
            const float a = p.ax;
            const float dt = (float)(2.0 * a / (p.nrays - 1));
            const float t = __fmaf_rn((float)i, dt, -a);
            sample_loop(t, dt, a, dt, dt, p.nrays, nx, nx);
            step = dt;
        } else {
            const float dx = 2.0f * p.ax / (float)(unsigned)(nx - 1);
            const float dy = 2.0f * p.ay / (float)(unsigned)(ny - 1);
            const float t = __fmaf_rn((float)i, dx, -p.ax);
            sample_loop(t, dy, p.ay, dx, dy, ny, nx, ny);
            step = dy;
        }
    }
    // combine the PH partial sums of each ray (every lane of the warp takes
    // part; the lanes of one ray share its validity, invalid rays sum zeros):
    // ((p0 + p1) + (p2 + p3)) for PH = 4, the same in every lane of the ray
#pragma unroll
    for (int o = RW * Sh::AW; o < 32; o <<= 1)
#pragma unroll
        for (int q = 0; q < S; q++) linesum[q] += __shfl_xor_sync(0xffffffffu, linesum[q], o);
#pragma unroll
    for (int q = 0; q < S; q++) value[q] = linesum[q] * step;

    // FP64 metric terms of this lane's slices q = ph + PH u (slot u = q / PH)
    constexpr int U = (S + PH - 1) / PH;
    double r2[U], y2[U], nll[U];
#pragma unroll
    for (int u = 0; u < U; u++) r2[u] = y2[u] = nll[u] = 0.0;
#pragma unroll
    for (int q = 0; q < S; q++) {
        const int k = k0 + q;
        if (!valid || q >= nsl || q % PH != ph) continue;   // phase lane ph writes slices q = ph mod PH
        const size_t vox = ((size_t)k * p.nangles + j) * p.nrays + i;
        float out = value[q];
        if constexpr (EPI == 1) {
            // tEM: model = flat * exp(-p); data = counts (kernel_flatTimesExp, em_RT_kernel.cu:20-32)
            const float fl = p.flat[(size_t)k * p.nrays + i];
            out = fl * __expf(-value[q]);
            if (p.metrics) {
                const double y = p.data[vox];
                const double m = fl * exp(-(double)value[q]);
                r2[q / PH] = (m - y) * (m - y);
                y2[q / PH] = y * y;
                nll[q / PH] = m + y * (double)value[q];
            }
        } else if constexpr (EPI == 2) {
            // eEM ratio, APPROXINVX(value, 1e-4) = SIGN/sqrtf(SQR(e)+SQR(x)) (configs.hpp:30-32)
            const float TOLZERO = 0.0001f;
            const float y = p.data[vox];
            const int sgn = (value[q] > 0) ? 1 : ((value[q] < 0) ? -1 : 0);
            out = y * (sgn / sqrtf(TOLZERO * TOLZERO + value[q] * value[q]));
            if (out < 0) out = 0.0f;
            if (p.metrics) {
                const double yd = y, m = value[q];
                r2[q / PH] = (m - yd) * (m - yd);
                y2[q / PH] = yd * yd;
                nll[q / PH] = (m > 0) ? m - yd * log(m) : 0.0;
            }
        }
        if (p.windowed) {
            const float w = p.wt ? p.wt[j] : 1.f;
            const size_t e = (size_t)(i - p.wlo);
            // 2: rows interleaved by slice in groups of four, the layout the
            // four-slice backprojector stages (the four phase lanes of a ray
            // write the four floats of one 16-byte element)
            const size_t o = p.windowed == 2 ? ((((size_t)(k >> 2) * p.nangles + j) * p.Wg + e) << 2) + (k & 3)
                                             : ((size_t)k * p.nangles + j) * p.Wg + e;
            p.out[o] = out * w;
        } else {
            p.out[vox] = out;
        }
    }
    if constexpr (EPI != 0) {
        if (p.metrics) {
            // FP64 per-slice sums: over the warp's lanes of one sample phase
            // (the lanes holding slice q), then across the block's warps
            __shared__ double red[3][S][PJ_WARPS];
            constexpr int G = RW * Sh::AW;   // lanes of one phase
#pragma unroll
            for (int u = 0; u < U; u++) {
                double a0 = r2[u], a1 = y2[u], a2 = nll[u];
#pragma unroll
                for (int o = 1; o < G; o <<= 1) {
                    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
                    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
                }
                const int q = ph + PH * u;
                if (threadIdx.x % G == 0 && q < S) {
                    red[0][q][threadIdx.y] = a0;
                    red[1][q][threadIdx.y] = a1;
                    red[2][q][threadIdx.y] = a2;
                }
            }
            __syncthreads();
            if (threadIdx.y == 0 && threadIdx.x < 3 * S) {
                const int q = threadIdx.x / 3, c = threadIdx.x - 3 * q;
                if (q < nsl) {
                    double sum = 0.0;
                    for (int w = 0; w < PJ_WARPS; w++) sum += red[c][q][w];
                    atomicAdd(&p.metrics[(size_t)(k0 + q) * 3 + c], sum);
                }
            }
        }
    }
}

template <int EM, int EPI, int S, int IL, int RW, int PH, int BRS>
__global__ void __launch_bounds__(32 * PJ_WARPS)
project_kernel(const ProjLaunch p)
{
    project_block<EM, EPI, S, IL, RW, PH, BRS>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Launch shapes (rays per warp RW, sample phases PH, rays per block BR): by
// default four rays x four phases x two angles per warp on interleaved images
// and eight rays x four phases on planar ones, 32 rays per block (blocks of
// 16, 8 or 4 rays at more angles measured 8-10 % slower on the interleaved
// images, the same on planar ones); RAFT_PJ_SEQUENTIAL=1 sums every ray in one
// lane in sample order (the reference's order; 32 rays at one angle, or four
// rays at eight angles per warp).  Read at every launch.
struct PjChoice {
    int rw, ph, br;
};
static bool pj_sequential()
{
    const char *e = getenv("RAFT_PJ_SEQUENTIAL");
    return e && atoi(e) == 1;
}
static PjChoice pj_il() { return pj_sequential() ? PjChoice{32, 1, 32} : PjChoice{4, 4, 32}; }
static PjChoice pj_pl() { return pj_sequential() ? PjChoice{4, 1, 32} : PjChoice{8, 4, 32}; }
template <class F>
static void pj_dispatch(PjChoice c, F &&f)
{
    using std::integral_constant;
    if (c.rw == 32) f(integral_constant<int, 32>{}, integral_constant<int, 1>{}, integral_constant<int, 32>{});
    else if (c.ph == 1) f(integral_constant<int, 4>{}, integral_constant<int, 1>{}, integral_constant<int, 32>{});
    else if (c.rw == 4) f(integral_constant<int, 4>{}, integral_constant<int, 4>{}, integral_constant<int, 32>{});
    else f(integral_constant<int, 8>{}, integral_constant<int, 4>{}, integral_constant<int, 32>{});
}

int project_blocks_per_slice(int nrays, int nangles)
{
    int n = 0;
    pj_dispatch(pj_pl(), [&](auto rw, auto ph, auto br) {
        using Sh = PjShape<decltype(rw)::value, decltype(ph)::value, decltype(br)::value>;
        n = ((nrays + Sh::BR - 1) / Sh::BR) * ((nangles + Sh::BA - 1) / Sh::BA);
    });
    return n;
}

// Ragged projector: one launch over many single-slice requests of different
// sizes; block b belongs to the request r with blk_start[r] <= b < blk_start[r+1].
template <int EM, int EPI, int RW, int PH, int BRS>
__global__ void __launch_bounds__(32 * PJ_WARPS)
project_ragged_kernel(const ProjLaunch *__restrict__ reqs, const int *__restrict__ blk_start, int nreq)
{
    __shared__ int s_r;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        int lo = 0, hi = nreq - 1;
        while (lo < hi) {                       // last r with blk_start[r] <= blockIdx.x
            const int mid = (lo + hi + 1) / 2;
            if (blk_start[mid] <= (int)blockIdx.x) lo = mid;
            else hi = mid - 1;
        }
        s_r = lo;
    }
    __syncthreads();
    const int r = s_r;
    const ProjLaunch &p = reqs[r];
    const int local = blockIdx.x - blk_start[r];
    const int nbx = (p.nrays + PjShape<RW, PH, BRS>::BR - 1) / PjShape<RW, PH, BRS>::BR;
    project_block<EM, EPI, 1, 0, RW, PH, BRS>(p, local % nbx, local / nbx, 0);
}

template <int RW, int PH, int BRS>
static void launch_ragged_shape(const ProjLaunch *d_reqs, const int *d_blk_start, int nreq, int total_blocks,
                                int em, int epilogue, cudaStream_t st)
{
    dim3 block(32, PJ_WARPS);
    if (!em)
        project_ragged_kernel<0, 0, RW, PH, BRS><<<total_blocks, block, 0, st>>>(d_reqs, d_blk_start, nreq);
    else if (epilogue == 1)
        project_ragged_kernel<1, 1, RW, PH, BRS><<<total_blocks, block, 0, st>>>(d_reqs, d_blk_start, nreq);
    else if (epilogue == 2)
        project_ragged_kernel<1, 2, RW, PH, BRS><<<total_blocks, block, 0, st>>>(d_reqs, d_blk_start, nreq);
    else
        project_ragged_kernel<1, 0, RW, PH, BRS><<<total_blocks, block, 0, st>>>(d_reqs, d_blk_start, nreq);
}

void launch_project_ragged(const ProjLaunch *d_reqs, const int *d_blk_start, int nreq, int total_blocks, int em,
                           int epilogue, cudaStream_t st)
{
    if (nreq <= 0 || total_blocks <= 0) return;
    ProfScope ps(PROF_PROJECT, st);
    pj_dispatch(pj_pl(), [&](auto rw, auto ph, auto br) {
        launch_ragged_shape<decltype(rw)::value, decltype(ph)::value, decltype(br)::value>(
            d_reqs, d_blk_start, nreq, total_blocks, em, epilogue, st);
    });
    RAFT_CUDA(cudaGetLastError());
}

// Tiled transpose of each slice: out[k][x][y] = in[k][y][x].
__global__ void transpose_kernel(const float *__restrict__ in, float *__restrict__ out, int nx, int ny)
{
    __shared__ float tile[32][33];
    const size_t plane = (size_t)nx * ny;
    const float *src = in + blockIdx.z * plane;
    float *dst = out + blockIdx.z * plane;
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int y = by + r, x = bx + threadIdx.x;
        if (x < nx && y < ny) tile[r][threadIdx.x] = src[(size_t)y * nx + x];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int x = bx + r, y = by + threadIdx.x;
        if (x < nx && y < ny) dst[(size_t)x * ny + y] = tile[threadIdx.x][r];
    }
}

void launch_transpose(const float *in, float *out, int nx, int ny, int nslices, cudaStream_t st)
{
    if (nslices <= 0) return;
    count_launch();
    dim3 grid((nx + 31) / 32, (ny + 31) / 32, nslices);
    transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(in, out, nx, ny);
    RAFT_CUDA(cudaGetLastError());
}

// Slice-interleaved copies of groups of 8 planes, row-major and transposed:
// il[g][y][x][s] = ilT[g][x][y][s] = in[8g + s][y][x] (zero where 8g + s is
// past the last plane), plus the eight zeros that samples outside the image
// read.  One 32 x 32 pixel tile of all 8 planes per block.
__global__ void __launch_bounds__(256)
interleave_kernel(const float *__restrict__ in, float *__restrict__ il, float *__restrict__ ilT,
                  float *__restrict__ zero8, int nx, int ny, int nslices)
{
    __shared__ float tile[8][32][33];
    const size_t plane = (size_t)nx * ny;
    const int g = blockIdx.z, tx = threadIdx.x;
    if ((blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.y) == 0 && tx < 8) zero8[tx] = 0.f;
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
#pragma unroll
    for (int s = 0; s < 8; s++) {
        const int k = g * 8 + s;
        for (int r = threadIdx.y; r < 32; r += blockDim.y) {
            const int y = by + r, x = bx + tx;
            tile[s][r][tx] = (k < nslices && x < nx && y < ny) ? in[(size_t)k * plane + (size_t)y * nx + x] : 0.f;
        }
    }
    __syncthreads();
    float *o = il + (size_t)g * plane * 8;
    float *oT = ilT + (size_t)g * plane * 8;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int y = by + r, x = bx + tx;
        if (x < nx && y < ny) {
            float4 *d = reinterpret_cast<float4 *>(o + ((size_t)y * nx + x) * 8);
            d[0] = make_float4(tile[0][r][tx], tile[1][r][tx], tile[2][r][tx], tile[3][r][tx]);
            d[1] = make_float4(tile[4][r][tx], tile[5][r][tx], tile[6][r][tx], tile[7][r][tx]);
        }
        x = bx + r;
        y = by + tx;
        if (x < nx && y < ny) {
            float4 *d = reinterpret_cast<float4 *>(oT + ((size_t)x * ny + y) * 8);
            d[0] = make_float4(tile[0][tx][r], tile[1][tx][r], tile[2][tx][r], tile[3][tx][r]);
            d[1] = make_float4(tile[4][tx][r], tile[5][tx][r], tile[6][tx][r], tile[7][tx][r]);
        }
    }
}

static bool use_interleaved(int nslices) { return nslices >= 8; }

size_t proj_scratch_bytes(int nx, int ny, int nslices)
{
    const size_t plane = (size_t)nx * ny * sizeof(float);
    if (nslices <= 0) return 16;
    if (use_interleaved(nslices)) return 2 * (size_t)((nslices + 7) / 8) * 8 * plane + 8 * sizeof(float);
    return (size_t)nslices * plane;
}

void stage_proj_images(ProjLaunch &pl, void *scratch, cudaStream_t st)
{
    if (pl.nslices <= 0) return;
    if (use_interleaved(pl.nslices)) {
        // the projector indexes a pixel of the interleaved copies in 32 bits
        RAFT_CHECK((size_t)pl.nx * pl.ny <= 0xffffffffull, "projector: image plane above 2^32 pixels");
        const int G = (pl.nslices + 7) / 8;
        float *il = (float *)scratch;
        float *ilT = il + (size_t)G * 8 * pl.nx * pl.ny;
        float *zero8 = ilT + (size_t)G * 8 * pl.nx * pl.ny;
        count_launch();
        dim3 grid((pl.nx + 31) / 32, (pl.ny + 31) / 32, G);
        interleave_kernel<<<grid, dim3(32, 8), 0, st>>>(pl.img, il, ilT, zero8, pl.nx, pl.ny, pl.nslices);
        RAFT_CUDA(cudaGetLastError());
        pl.il = il;
        pl.ilT = ilT;
        pl.il_zero = zero8;
        pl.imgT = nullptr;
    } else {
        float *t = (float *)scratch;
        launch_transpose(pl.img, t, pl.nx, pl.ny, pl.nslices, st);
        pl.imgT = t;
        pl.il = pl.ilT = pl.il_zero = nullptr;
    }
}

template <int EM, int EPI, int S, int IL, int RW, int PH, int BRS>
static void launch_project_shape(const ProjLaunch &pl, cudaStream_t st)
{
    using Sh = PjShape<RW, PH, BRS>;
    dim3 grid((pl.nrays + Sh::BR - 1) / Sh::BR, (pl.nangles + Sh::BA - 1) / Sh::BA, (pl.nslices + S - 1) / S);
    project_kernel<EM, EPI, S, IL, RW, PH, BRS><<<grid, dim3(32, PJ_WARPS), 0, st>>>(pl);
}

template <int EM, int EPI>
static void launch_project_s(const ProjLaunch &pl, int S, cudaStream_t st)
{
    ProfScope ps(PROF_PROJECT, st);
    if (S == 8) {
        pj_dispatch(pj_il(), [&](auto rw, auto ph, auto br) {
            launch_project_shape<EM, EPI, 8, 1, decltype(rw)::value, decltype(ph)::value, decltype(br)::value>(pl, st);
        });
    } else {
        pj_dispatch(pj_pl(), [&](auto rw, auto ph, auto br) {
            constexpr int RW = decltype(rw)::value, PH = decltype(ph)::value, BR = decltype(br)::value;
            if (S == 4) launch_project_shape<EM, EPI, 4, 0, RW, PH, BR>(pl, st);
            else if (S == 2) launch_project_shape<EM, EPI, 2, 0, RW, PH, BR>(pl, st);
            else launch_project_shape<EM, EPI, 1, 0, RW, PH, BR>(pl, st);
        });
    }
    RAFT_CUDA(cudaGetLastError());
}

void launch_project(const ProjLaunch &pl, cudaStream_t st)
{
    if (pl.nslices <= 0 || pl.nangles <= 0 || pl.nrays <= 0) return;
    // the projector indexes a pixel of a plane in 32 bits
    RAFT_CHECK((size_t)pl.nx * pl.ny <= 0xffffffffull, "projector: image plane above 2^32 pixels");
    RAFT_CHECK((pl.il == nullptr) == (pl.ilT == nullptr) && (pl.il == nullptr) == (pl.il_zero == nullptr),
               "projector: interleaved copies come with their transposed copy and zero pixel");
    const int S = pl.il ? 8 : (pl.nslices >= 4 ? 4 : (pl.nslices >= 2 ? 2 : 1));
    if (!pl.em) {
        launch_project_s<0, 0>(pl, S, st);
    } else {
        switch (pl.epilogue) {
        case 1: launch_project_s<1, 1>(pl, S, st); break;
        case 2: launch_project_s<1, 2>(pl, S, st); break;
        default: launch_project_s<1, 0>(pl, S, st); break;
        }
    }
}

// Plain sinogram -> weighted window rows (the rest of each row stays zero).
// sino == nullptr writes the weight itself (back-projection of ones).
__global__ void to_window_kernel(const float *__restrict__ sino, float *__restrict__ rows,
                                 const float *__restrict__ wt, int nrows, int nangles, int nrays, int wlo,
                                 int Wg)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrays) return;
    for (int r = blockIdx.y; r < nrows; r += gridDim.y) {
        const float w = wt ? wt[r % nangles] : 1.f;
        const float v = sino ? sino[(size_t)r * nrays + i] : 1.f;
        rows[(size_t)r * Wg + (i - wlo)] = v * w;
    }
}

void launch_to_window(const float *sino, float *rows, const float *wt, int nrows, int nangles, int nrays,
                      int wlo, int Wg, cudaStream_t st)
{
    if (nrows <= 0) return;
    dim3 grid((nrays + 255) / 256, nrows < 65535 ? nrows : 65535);
    count_launch();
    to_window_kernel<<<grid, 256, 0, st>>>(sino, rows, wt, nrows, nangles, nrays, wlo, Wg);
    RAFT_CUDA(cudaGetLastError());
}

}  // namespace raft
