// noalloc.cu -- an FBP entry point that allocates nothing.
//
// raft_fbp_device_noalloc runs the same filter + backprojection as
// raft_fbp_device on caller-owned device buffers, but takes its working
// memory (filter spectrum and twiddles, angle tables, the error flag and the
// filtered window rows) from one file-scope device array of fixed size
// instead of cudaMalloc.  It exists for callers that cannot allocate device
// memory while reconstructing: acquisition pipelines that reserve the GPU's
// memory when a scan starts so that reconstruction can never fail for lack
// of memory halfway through, and host applications whose own allocator owns
// the device memory, where a cudaMalloc behind its back breaks the host's
// memory accounting.
//
// The array (kNoallocScratchBytes, 64 MiB) is held by every GPU that loads
// this module until the process exits.  All calls share it and it keeps the
// last call's contents; every region a call reads is written by that same
// call first, and the error flag is cleared per call.  Two calls whose work
// overlaps on the GPU (different host threads or streams, same device) race
// on the array: the entry point serialises host-side calls, but a caller
// that issues work on several streams must not let two of these calls run
// concurrently on one device.
//
// Set-up: the first call on each device (with that device current) looks up
// the array's device address with cudaGetSymbolAddress; make that first call
// before any stream capture.  The address belongs to the device's context:
// like the library's other per-device state (streams, workspaces), it does
// not survive a cudaDeviceReset by the host application.
//
// Every call ends by synchronising the stream it was given.  It always runs
// the planar backprojector: the slice-interleaved rows raft_fbp_device uses
// for four slices at a time need four slices' rows twice over (178 MB at
// 2048^2 x 1800), beyond the array.
#include "engine.hpp"

#include <cmath>
#include <mutex>

namespace raft {

constexpr size_t kNoallocScratchBytes = 64u << 20;   // 64 MiB per GPU
constexpr int kNoallocMaxNp = 14080;                   // FFT filter in shared memory
constexpr int kNoallocMaxAngles = 32768;
constexpr int kNoallocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

static std::mutex g_noalloc_mtx;
static unsigned char *g_noalloc_ptr[kNoallocMaxDevices] = {};
// host staging of the tables (static storage: nothing is allocated per call)
static double g_hre[kNoallocMaxNp], g_him[kNoallocMaxNp];
static float2 g_h2[2 * kNoallocMaxNp];
static double g_trig[2 * kNoallocMaxAngles];

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Device address of the scratch array for `gpu` (current device).
static unsigned char *scratch_for(int gpu)
{
    if (!g_noalloc_ptr[gpu]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error(std::string("raft_fbp_device_noalloc: cudaGetSymbolAddress failed: ") +
                      cudaGetErrorString(e));
            throw CudaFail();
        }
        g_noalloc_ptr[gpu] = static_cast<unsigned char *>(p);
    }
    return g_noalloc_ptr[gpu];
}

}  // namespace raft

using namespace raft;

extern "C" int raft_fbp_device_noalloc(int gpu, float *d_obj, const float *d_tomogram, const float *angles,
                                       const float *paramf, const int *parami, int geometry, int store,
                                       void *stream)
{
    clear_error();
    FbpConfig cfg;
    if (!parse_fbp_params(paramf, parami, cfg)) return 1;
    if (!check_gpu_id(gpu)) return 1;
    if (gpu >= kNoallocMaxDevices) {
        set_error("raft_fbp_device_noalloc: device id beyond the supported maximum (64)");
        return 1;
    }
    if ((geometry == GEOM_FBP_REF && store != STORE_F32) ||
        (geometry == GEOM_FBP_LIN && store != STORE_PAIR_F32 && store != STORE_PAIR_BF16) ||
        (geometry != GEOM_FBP_REF && geometry != GEOM_FBP_LIN)) {
        set_error("raft_fbp_device_noalloc: geometry/store as raft_fbp_ext (0/0, 1/1, 1/2)");
        return 1;
    }
    if (cfg.nslices == 0) return 0;
    if (!d_obj || !d_tomogram || !angles) {
        set_error("null data pointer");
        return 1;
    }
    cfg.geometry = geometry;
    cfg.store = store;
    const int N = cfg.nrays, A = cfg.nangles, No = cfg.objsize, pad = cfg.pad;
    FilterPlan plan;
    if (!filter_plan_shape(plan, cfg.filter, N, pad)) {
        set_error("raft_fbp_device_noalloc: padded length N*(1+pad) must have only the prime factors "
                  "2, 3, 5, 7 and be at most 14080");
        return 1;
    }
    if (plan.Np > kNoallocMaxNp || A > kNoallocMaxAngles) {
        set_error("raft_fbp_device_noalloc: N*(1+pad) must be <= 14080 and nangles <= 32768");
        return 1;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mtx);
    try {
        RAFT_CUDA(cudaSetDevice(gpu));
        cudaStream_t st = (cudaStream_t)stream;
        unsigned char *base = scratch_for(gpu);

        // geometry: the same FP32 expressions as prepare_fbp (fbp.cu:38-44)
        FbpPrepared fp;
        fp.cfg = cfg;
        fp.No = No;
        fp.Np = N * (1 + pad);
        fp.Npo = No * (1 + pad);
        BpGeo &g = fp.geo;
        g.xmin = -cfg.pixel_x * (float)fp.Npo / 2.0f;
        g.ymin = -cfg.pixel_y * (float)fp.Npo / 2.0f;
        g.dx = cfg.pixel_x;
        g.dy = cfg.pixel_y;
        g.tmin = -cfg.pixel_x * (float)fp.Np / 2.0f;
        g.dt = cfg.pixel_x;
        g.offo = (pad * No) / 2;
        BpPlanInput pi;
        pi.geometry = geometry;
        pi.store = store;
        pi.No = No;
        pi.xmin = g.xmin;
        pi.ymin = g.ymin;
        pi.dx = g.dx;
        pi.dy = g.dy;
        pi.tmin = g.tmin;
        pi.dt = g.dt;
        pi.offo = g.offo;
        fp.win = plan_window(pi);
        g.c0 = (double)g.offo - 0.5 * fp.Npo;
        g.ratio = (double)cfg.pixel_y / (double)cfg.pixel_x;
        g.u0 = 0.5 * fp.Np - fp.win.wlo - 0.5;

        // scratch layout
        const int Np = fp.Np;
        size_t off = 0;
        const size_t o_H = off;        off = align256(off + sizeof(float2) * Np);
        const size_t o_tw = off;       off = align256(off + sizeof(float2) * Np);
        const size_t o_trig = off;     off = align256(off + sizeof(double) * 2 * A);
        const size_t o_tab = off;      off = align256(off + sizeof(float) * 4 * A);
        const size_t o_err = off;      off = align256(off + sizeof(int));
        const size_t o_rows = off;
        const size_t row_bytes = (size_t)A * fp.win.Wg * store_bytes(store);
        if (o_rows + row_bytes > kNoallocScratchBytes) {
            set_error("raft_fbp_device_noalloc: one slice needs " + std::to_string(o_rows + row_bytes) +
                      " bytes of scratch, more than the 64 MiB maximum (reduce nangles or N)");
            return 1;
        }
        const int chunk = (int)std::min<size_t>((kNoallocScratchBytes - o_rows) / row_bytes, 32);

        // filter spectrum and twiddles (host, FP64 -> FP32), as build_filter_plan
        if (!plan.skip) {
            filter_spectrum_host(geometry, cfg.filter, Np, cfg.paganin, cfg.reg, cfg.offset, cfg.pixel_x, g_hre,
                                 g_him);
            for (int k = 0; k < Np; k++) {
                g_h2[k] = make_float2((float)g_hre[k], (float)g_him[k]);
                const double a = -2.0 * M_PI * (double)k / (double)Np;
                g_h2[Np + k] = make_float2((float)std::cos(a), (float)std::sin(a));
            }
            plan.d_H = reinterpret_cast<float2 *>(base + o_H);
            plan.d_tw = reinterpret_cast<float2 *>(base + o_tw);
            RAFT_CUDA(cudaMemcpyAsync(plan.d_H, g_h2, sizeof(float2) * Np, cudaMemcpyHostToDevice, st));
            RAFT_CUDA(cudaMemcpyAsync(plan.d_tw, g_h2 + Np, sizeof(float2) * Np, cudaMemcpyHostToDevice, st));
        }
        fp.plan = &plan;

        // angle tables
        FbpTables tb;
        tb.csd = reinterpret_cast<double *>(base + o_trig);
        tb.snd = tb.csd + A;
        float *d_ang = reinterpret_cast<float *>(base + o_tab);
        tb.cs = d_ang + A;
        tb.sn = tb.cs + A;
        tb.wt = tb.sn + A;
        tb.err = reinterpret_cast<int *>(base + o_err);
        RAFT_CUDA(cudaMemcpyAsync(d_ang, angles, sizeof(float) * A, cudaMemcpyHostToDevice, st));
        RAFT_CUDA(cudaMemsetAsync(tb.err, 0, sizeof(int), st));
        launch_angle_tables(d_ang, A, tb.cs, tb.sn, tb.wt, 0, st);
        if (geometry == GEOM_FBP_LIN) {
            for (int a = 0; a < A; a++) {
                g_trig[a] = std::cos((double)angles[a]);
                g_trig[A + a] = std::sin((double)angles[a]);
            }
            RAFT_CUDA(cudaMemcpyAsync(tb.csd, g_trig, sizeof(double) * 2 * A, cudaMemcpyHostToDevice, st));
        }

        // filter + backprojection, `chunk` slices at a time through the rows region
        DeviceState unused;
        void *rows = base + o_rows;
        const size_t tomo_ps = (size_t)A * N, obj_ps = (size_t)No * No;
        for (int s0 = 0; s0 < cfg.nslices; s0 += chunk) {
            const int ns = std::min(chunk, cfg.nslices - s0);
            fbp_chunk(unused, fp, tb, d_tomogram + tomo_ps * s0, d_obj + obj_ps * s0, ns, rows, st);
        }
        int flag = 0;
        RAFT_CUDA(cudaMemcpyAsync(&flag, tb.err, sizeof(int), cudaMemcpyDeviceToHost, st));
        RAFT_CUDA(cudaStreamSynchronize(st));
        RAFT_CHECK(flag == 0, "raft_fbp_device_noalloc: a bounded wait in the staging pipeline timed out");
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}
