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
// so the nearest-pixel choice is the reference's.
#include "raft.hpp"
#include "profile.hpp"

namespace raft {

constexpr int PJ_RAYS = 32;
constexpr int PJ_ANGLES = 8;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int EM, int EPI>
__global__ void __launch_bounds__(PJ_RAYS * PJ_ANGLES)
project_kernel(const ProjLaunch p)
{
    const int i = blockIdx.x * PJ_RAYS + threadIdx.x;     // ray
    const int j = blockIdx.y * PJ_ANGLES + threadIdx.y;   // angle
    const int k = blockIdx.z;                             // slice
    const bool valid = (i < p.nrays) && (j < p.nangles);
    const int nx = p.nx, ny = p.ny;
    const float *img = p.img + (size_t)k * nx * ny;
    float value = 0.f;
    if (valid) {
        if constexpr (EM) {
            // kernel_radon: dt = 2.0*a/(nrays-1) in double, a = 1
            const float a = p.ax;
            const float dt = (float)(2.0 * a / (p.nrays - 1));
            const float ctheta = __cosf(p.angles[j]);
            const float stheta = __sinf(p.angles[j]);
            const float t = -a + i * dt;
            float linesum = 0.f;
            for (int m = 0; m < p.nrays; m++) {
                const float s = -a + m * dt;
                const float x = t * ctheta - s * stheta;
                const float y = t * stheta + s * ctheta;
                const int X = (int)((x + 1) / dt);
                const int Y = (int)((y + 1) / dt);
                if ((X >= 0) & (X < nx) & (Y >= 0) & (Y < nx))
                    linesum += __ldg(&img[Y * nx + X]);
            }
            value = linesum * dt;
        } else {
            const float dx = 2.0f * p.ax / (float)(unsigned)(nx - 1);
            const float dy = 2.0f * p.ay / (float)(unsigned)(ny - 1);
            const float ctheta = __cosf(p.angles[j]);
            const float stheta = __sinf(p.angles[j]);
            const float t = -p.ax + i * dx;
            float linesum = 0.f;
            for (int r = 0; r < ny; r++) {
                const float s = -p.ay + r * dy;
                const float x = t * ctheta - s * stheta;
                const float y = t * stheta + s * ctheta;
                const int ix = (int)((x + 1) / dx);
                const int iy = (int)((y + 1) / dy);
                if ((ix >= 0) & (ix < nx) & (iy >= 0) & (iy < ny))
                    linesum += __ldg(&img[(size_t)iy * nx + ix]);
            }
            value = linesum * dy;
        }
    }

    const size_t vox = ((size_t)k * p.nangles + j) * p.nrays + i;
    float q = value;
    double r2 = 0.0, y2 = 0.0, nll = 0.0;
    if (valid) {
        if constexpr (EPI == 1) {
            // tEM: model = flat * exp(-p); data = counts
            const float fl = p.flat[(size_t)k * p.nrays + i];
            q = fl * __expf(-value);
            if (p.metrics) {
                const double y = p.data[vox];
                const double m = fl * exp(-(double)value);
                r2 = (m - y) * (m - y);
                y2 = y * y;
                nll = m + y * (double)value;
            }
        } else if constexpr (EPI == 2) {
            // eEM ratio, APPROXINVX(value, 1e-4) = SIGN/sqrtf(SQR(e)+SQR(x)) (configs.hpp:30-32)
            const float TOLZERO = 0.0001f;
            const float y = p.data[vox];
            const int sgn = (value > 0) ? 1 : ((value < 0) ? -1 : 0);
            q = y * (sgn / sqrtf(TOLZERO * TOLZERO + value * value));
            if (q < 0) q = 0.0f;
            if (p.metrics) {
                const double yd = y, m = value;
                r2 = (m - yd) * (m - yd);
                y2 = yd * yd;
                nll = (m > 0) ? m - yd * log(m) : 0.0;
            }
        }
        if (p.windowed) {
            const float w = p.wt ? p.wt[j] : 1.f;
            p.out[((size_t)k * p.nangles + j) * p.Wg + (i - p.wlo)] = q * w;
        } else {
            p.out[vox] = q;
        }
    }
    if constexpr (EPI != 0) {
        if (p.metrics) {
            __shared__ double red[3][PJ_ANGLES];
            r2 = warp_sum(r2);
            y2 = warp_sum(y2);
            nll = warp_sum(nll);
            if (threadIdx.x == 0) {
                red[0][threadIdx.y] = r2;
                red[1][threadIdx.y] = y2;
                red[2][threadIdx.y] = nll;
            }
            __syncthreads();
            if (threadIdx.y == 0 && threadIdx.x < 3) {
                double s = 0.0;
                for (int w = 0; w < PJ_ANGLES; w++) s += red[threadIdx.x][w];
                atomicAdd(&p.metrics[(size_t)k * 3 + threadIdx.x], s);
            }
        }
    }
}

void launch_project(const ProjLaunch &pl, cudaStream_t st)
{
    if (pl.nslices <= 0 || pl.nangles <= 0 || pl.nrays <= 0) return;
    ProfScope ps(PROF_PROJECT, st);
    dim3 block(PJ_RAYS, PJ_ANGLES);
    dim3 grid((pl.nrays + PJ_RAYS - 1) / PJ_RAYS, (pl.nangles + PJ_ANGLES - 1) / PJ_ANGLES, pl.nslices);
    if (!pl.em) {
        project_kernel<0, 0><<<grid, block, 0, st>>>(pl);
    } else {
        switch (pl.epilogue) {
        case 1: project_kernel<1, 1><<<grid, block, 0, st>>>(pl); break;
        case 2: project_kernel<1, 2><<<grid, block, 0, st>>>(pl); break;
        default: project_kernel<1, 0><<<grid, block, 0, st>>>(pl); break;
        }
    }
    RAFT_CUDA(cudaGetLastError());
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
