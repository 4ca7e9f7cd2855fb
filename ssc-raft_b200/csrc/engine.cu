// engine.cu -- host-side execution engine.
//
// Reference drivers this replaces (cnpem/ssc-raft):
//   getFBPGPU        cuda/src/geometries/parallel/reconstruction_methods/fbp.cu:127-236
//   getFilterLowPassGPU cuda/src/processing/filters/low_pass.cu:33-82
//   getRadonRTGPU    cuda/src/geometries/parallel/forward_methods/radon_rt.cu:203-250
//   get_tEM_RT_GPU / get_tEM_RT   .../reconstruction_methods/em_rt.cu:86-192
//   get_eEM_RT_GPU / get_eEM_RT   .../reconstruction_methods/em_rt.cu:264-355
//
// The reference allocates and frees every device buffer per call (and the
// FFT buffer per slice), builds cuFFT plans per call, and copies slice
// blocks synchronously with no overlap.  Here each device keeps grow-only
// workspaces and pinned staging buffers across calls, filter plans are
// cached, and host buffers stream through a two-slot pipeline: host copy
// into pinned memory, H2D on one stream, filter + backprojection on a
// second, D2H on a third, host copy out -- so PCIe traffic and the host
// copies overlap the kernels of the neighbouring chunk.  The EM iteration
// loop is captured once as a CUDA graph and replayed as a single launch.
#include "engine.hpp"

#include <atomic>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <thread>
#include <tuple>

namespace raft {

// ----------------------------------------------------------- buffers ------
// Injected allocation refusals (raft_inject_alloc_failures): the next n
// device-buffer requests of the engine fail as an out-of-memory would
// (whether or not the buffer would have grown).
static std::atomic<int> g_alloc_failures{0};
void inject_alloc_failures(int n) { g_alloc_failures.store(n > 0 ? n : 0); }

void *DevBuf::get(size_t need)
{
    if (need == 0) need = 16;
    int left = g_alloc_failures.load();
    while (left > 0 && !g_alloc_failures.compare_exchange_weak(left, left - 1)) {
    }
    if (left > 0) {
        set_error("device allocation of " + std::to_string(need) + " bytes refused (injected failure)");
        throw CudaFail{};
    }
    if (need > bytes) {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        RAFT_CUDA(cudaMalloc(&ptr, need));
        bytes = need;
    }
    return ptr;
}
void DevBuf::release()
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}
void *PinBuf::get(size_t need)
{
    if (need == 0) need = 16;
    if (need > bytes) {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        RAFT_CUDA(cudaHostAlloc(&ptr, need, cudaHostAllocPortable));
        bytes = need;
    }
    return ptr;
}
void PinBuf::release()
{
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

void DeviceState::ensure()
{
    if (init) return;
    RAFT_CUDA(cudaStreamCreateWithFlags(&s_comp, cudaStreamNonBlocking));
    RAFT_CUDA(cudaStreamCreateWithFlags(&s_h2d, cudaStreamNonBlocking));
    RAFT_CUDA(cudaStreamCreateWithFlags(&s_d2h, cudaStreamNonBlocking));
    int lo = 0, hi = 0;
    RAFT_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    RAFT_CUDA(cudaStreamCreateWithPriority(&s_hi, cudaStreamNonBlocking, hi));
    RAFT_CUDA(cudaStreamCreateWithPriority(&s_lo, cudaStreamNonBlocking, lo));
    for (int b = 0; b < 2; b++) {
        RAFT_CUDA(cudaEventCreateWithFlags(&ev_h2d[b], cudaEventDisableTiming));
        RAFT_CUDA(cudaEventCreateWithFlags(&ev_comp[b], cudaEventDisableTiming));
        RAFT_CUDA(cudaEventCreateWithFlags(&ev_d2h[b], cudaEventDisableTiming));
    }
    RAFT_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    init = true;
}

cudaStream_t resolve_stream(DeviceState &ds, void *stream, cudaStream_t own)
{
    if (stream) return (cudaStream_t)stream;
    RAFT_CUDA(cudaEventRecord(ds.ev_join, cudaStreamLegacy));
    RAFT_CUDA(cudaStreamWaitEvent(own, ds.ev_join, 0));
    return own;
}

static std::mutex g_state_mtx;
static std::map<int, std::unique_ptr<DeviceState>> g_states;

DeviceState &device_state(int device)
{
    std::lock_guard<std::mutex> lk(g_state_mtx);
    auto &p = g_states[device];
    if (!p) {
        p.reset(new DeviceState());
        p->device = device;
    }
    return *p;
}

// ------------------------------------------------------------ plan cache --
using PlanKey = std::tuple<int, int, int, int, int, double, double, double, double>;
static std::mutex g_plan_mtx;
static std::map<PlanKey, FilterPlan> g_plans;

const FilterPlan &cached_filter_plan(int device, int geometry, int ftype, int N, int pad, double paganin,
                                     double reg, double offset, double pixel)
{
    // the spectrum depends on the geometry only through ref vs lin
    const int g = geometry == GEOM_FBP_LIN ? 1 : 0;
    PlanKey key(device, g, ftype, N, pad, paganin, reg, offset, pixel);
    std::lock_guard<std::mutex> lk(g_plan_mtx);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) return it->second;
    FilterPlan plan;
    build_filter_plan(plan, geometry, ftype, N, pad, paganin, reg, offset, pixel, device);
    if (g_plans.size() > 64) {
        for (auto &kv : g_plans) release_filter_plan(kv.second);
        g_plans.clear();
    }
    return g_plans.emplace(key, plan).first->second;
}

// ----------------------------------------------------------- host copies --
void parallel_memcpy(void *dst, const void *src, size_t bytes)
{
    const size_t kMin = 8u << 20;
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    unsigned nt = (unsigned)std::min<size_t>(std::min(8u, hw), bytes / kMin);
    if (nt <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t part = (bytes + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        const size_t o = t * part;
        if (o >= bytes) break;
        const size_t n = std::min(part, bytes - o);
        th.emplace_back([=] { std::memcpy((char *)dst + o, (const char *)src + o, n); });
    }
    for (auto &t : th) t.join();
}

// Generic two-slot staging pipeline: host_in (in_ps bytes per slice) ->
// device -> compute -> host_out (out_ps bytes per slice).
static bool is_pinned(const void *p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

template <class F>
static void run_pipeline(DeviceState &ds, int nslices, int chunk, size_t in_ps, size_t out_ps,
                         const void *host_in, void *host_out, F compute)
{
    if (nslices <= 0) return;
    // page-locked caller buffers are transferred directly; pageable ones are
    // staged through the device's pinned buffers by host threads
    const bool pin_src = is_pinned(host_in), pin_dst = is_pinned(host_out);
    void *din[2], *dout[2], *pin[2] = {nullptr, nullptr}, *pout[2] = {nullptr, nullptr};
    for (int b = 0; b < 2; b++) {
        din[b] = ds.sino[b].get(in_ps * chunk);
        dout[b] = ds.img[b].get(out_ps * chunk);
        if (!pin_src) pin[b] = ds.pin_in[b].get(in_ps * chunk);
        if (!pin_dst) pout[b] = ds.pin_out[b].get(out_ps * chunk);
    }
    // Chunk schedule: the first chunk's upload and the last chunk's download
    // overlap no compute, so with enough slices the chunks ramp up from four
    // slices (a whole group of the four-slice backprojector), doubling, to
    // full size, and ramp down the same way at the end: each upload then
    // hides behind the compute of a chunk half its size, and the exposed
    // ends are four slices' copies.
    std::vector<int> cs0, cns;
    {
        std::vector<int> ramp;
        for (int e = 4; e < chunk && 4 * e <= nslices; e *= 2) ramp.push_back(e);
        int edge_total = 0;
        for (int e : ramp) edge_total += 2 * e;
        if (chunk < 8 || nslices <= edge_total + chunk) {
            ramp.clear();
            edge_total = 0;
        }
        int s = 0;
        auto add = [&](int n) {
            cs0.push_back(s);
            cns.push_back(n);
            s += n;
        };
        for (int e : ramp) add(e);
        const int mid_end = nslices - edge_total / 2;
        while (s < mid_end) add(std::min(chunk, mid_end - s));
        for (int k = (int)ramp.size() - 1; k >= 0; --k) add(ramp[k]);
    }
    const int nch = (int)cs0.size();
    auto finalize = [&](int c) {
        const int b = c & 1, s0 = cs0[c], ns = cns[c];
        RAFT_CUDA(cudaEventSynchronize(ds.ev_d2h[b]));
        if (!pin_dst) parallel_memcpy((char *)host_out + (size_t)s0 * out_ps, pout[b], (size_t)ns * out_ps);
    };
    for (int c = 0; c < nch; c++) {
        const int b = c & 1, s0 = cs0[c], ns = cns[c];
        const void *src = (const char *)host_in + (size_t)s0 * in_ps;
        if (!pin_src) {
            if (c >= 2) RAFT_CUDA(cudaEventSynchronize(ds.ev_h2d[b]));
            parallel_memcpy(pin[b], src, (size_t)ns * in_ps);
            src = pin[b];
        }
        if (c >= 2) RAFT_CUDA(cudaStreamWaitEvent(ds.s_h2d, ds.ev_comp[b], 0));
        RAFT_CUDA(cudaMemcpyAsync(din[b], src, (size_t)ns * in_ps, cudaMemcpyHostToDevice, ds.s_h2d));
        RAFT_CUDA(cudaEventRecord(ds.ev_h2d[b], ds.s_h2d));
        RAFT_CUDA(cudaStreamWaitEvent(ds.s_comp, ds.ev_h2d[b], 0));
        if (c >= 2) RAFT_CUDA(cudaStreamWaitEvent(ds.s_comp, ds.ev_d2h[b], 0));
        compute(din[b], dout[b], ns, ds.s_comp);
        RAFT_CUDA(cudaEventRecord(ds.ev_comp[b], ds.s_comp));
        RAFT_CUDA(cudaStreamWaitEvent(ds.s_d2h, ds.ev_comp[b], 0));
        void *dst = pin_dst ? (void *)((char *)host_out + (size_t)s0 * out_ps) : pout[b];
        RAFT_CUDA(cudaMemcpyAsync(dst, dout[b], (size_t)ns * out_ps, cudaMemcpyDeviceToHost, ds.s_d2h));
        RAFT_CUDA(cudaEventRecord(ds.ev_d2h[b], ds.s_d2h));
        if (c >= 1) finalize(c - 1);
    }
    finalize(nch - 1);
    RAFT_CUDA(cudaStreamSynchronize(ds.s_comp));
    RAFT_CUDA(cudaStreamSynchronize(ds.s_h2d));
    RAFT_CUDA(cudaStreamSynchronize(ds.s_d2h));
}

// Slices per pipeline chunk: about 512 MB of input, at most 32, a multiple of
// four where possible (the backprojector's CTAs take four slices each).
static int auto_chunk(int nslices, size_t bytes_per_slice, int blocksize)
{
    if (blocksize > 0) return std::max(1, std::min(blocksize, nslices));
    const size_t target = (size_t)512 << 20;
    int c = (int)std::max<size_t>(1, target / std::max<size_t>(1, bytes_per_slice));
    c = std::min(c, 32);
    if (c >= 4) c -= c % 4;
    return std::max(1, std::min(c, nslices));
}

// ------------------------------------------------------------------ FBP --
FbpPrepared prepare_fbp(const FbpConfig &cfg, int device)
{
    FbpPrepared fp;
    fp.cfg = cfg;
    const int N = cfg.nrays, No = cfg.objsize, pad = cfg.pad;
    fp.No = No;
    fp.Np = N * (1 + pad);
    fp.Npo = No * (1 + pad);
    // fbp.cu:38-44 with obj_size = Npo, tomo_size.x = Np (padded sizes)
    BpGeo &g = fp.geo;
    g.xmin = -cfg.pixel_x * (float)fp.Npo / 2.0f;
    g.ymin = -cfg.pixel_y * (float)fp.Npo / 2.0f;
    g.dx = cfg.pixel_x;
    g.dy = cfg.pixel_y;
    g.tmin = -cfg.pixel_x * (float)fp.Np / 2.0f;
    g.dt = cfg.pixel_x;
    g.offo = (pad * No) / 2;   // remove_paddR2R offset (padding.cu:245-268)
    BpPlanInput pi;
    pi.geometry = cfg.geometry;
    pi.store = cfg.store;
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
    fp.plan = &cached_filter_plan(device, cfg.geometry, cfg.filter, N, pad, cfg.paganin, cfg.reg, cfg.offset,
                                  cfg.pixel_x);
    return fp;
}

FbpTables fbp_tables(DeviceState &ds, const FbpPrepared &fp, const float *h_angles, cudaStream_t st)
{
    const int A = fp.cfg.nangles;
    FbpTables tb;
    float *d_ang = (float *)ds.angles.get(sizeof(float) * A);
    RAFT_CUDA(cudaMemcpy(d_ang, h_angles, sizeof(float) * A, cudaMemcpyHostToDevice));
    char *base = (char *)ds.tabs.get(sizeof(double) * 2 * A + sizeof(float) * 3 * A + 64);
    tb.csd = (double *)base;
    tb.snd = tb.csd + A;
    tb.cs = (float *)(tb.snd + A);
    tb.sn = tb.cs + A;
    tb.wt = tb.sn + A;
    tb.err = (int *)ds.err.get(sizeof(int));
    RAFT_CUDA(cudaMemsetAsync(tb.err, 0, sizeof(int), st));
    launch_angle_tables(d_ang, A, tb.cs, tb.sn, tb.wt, 0, st);
    if (fp.cfg.geometry == GEOM_FBP_LIN) {
        std::vector<double> cd(2 * (size_t)A);
        for (int a = 0; a < A; a++) {
            cd[a] = std::cos((double)h_angles[a]);
            cd[A + a] = std::sin((double)h_angles[a]);
        }
        RAFT_CUDA(cudaMemcpy(tb.csd, cd.data(), sizeof(double) * 2 * A, cudaMemcpyHostToDevice));
    }
    return tb;
}

size_t fbp_rows_bytes(const FbpPrepared &fp, int nslices)
{
    return (size_t)nslices * fp.cfg.nangles * fp.win.Wg * store_bytes(fp.cfg.store);
}

bool fbp_fused_il(const FbpPrepared &fp)
{
    return fbp_il_bytes(fp, 1) > 0 && !bp_forced_planar();
}

void fbp_chunk(DeviceState &ds, const FbpPrepared &fp, const FbpTables &tb, const float *d_sino, float *d_img,
               int nslices, void *d_rows, cudaStream_t st, void *d_il)
{
    (void)ds;
    if (nslices <= 0) return;
    // with the interleave workspace and 4-byte elements the filter writes the
    // four-slice interleaved rows the backprojector stages, directly
    const bool fused = d_il && fbp_fused_il(fp);
    FilterLaunch fl;
    fl.sino = d_sino;
    fl.out = fused ? d_il : d_rows;
    fl.interleaved = fused ? 1 : 0;
    fl.wt = tb.wt;
    fl.nrows = nslices * fp.cfg.nangles;
    fl.nangles = fp.cfg.nangles;
    fl.wlo = fp.win.wlo;
    fl.Wg = fp.win.Wg;
    fl.store = fp.cfg.store;
    launch_filter(*fp.plan, fl, st);
    BpLaunch bl;
    bl.filt = fused ? nullptr : d_rows;
    bl.img = d_img;
    bl.No = fp.No;
    bl.nangles = fp.cfg.nangles;
    bl.nslices = nslices;
    bl.geometry = fp.cfg.geometry;
    bl.store = fp.cfg.store;
    bl.win = fp.win;
    bl.geo = fp.geo;
    bl.cs = tb.cs;
    bl.sn = tb.sn;
    bl.csd = tb.csd;
    bl.snd = tb.snd;
    bl.err = tb.err;
    bl.il_ws = d_il;
    bl.il_ready = fused ? 1 : 0;
    launch_backproject(bl, st);
}

size_t fbp_il_bytes(const FbpPrepared &fp, int nslices)
{
    return store_bytes(fp.cfg.store) == 4 ? bp_il_bytes(nslices, fp.cfg.nangles, fp.win.Wg, 4) : 0;
}

static void check_device_flag(const int *d_err, const char *what)
{
    int h = 0;
    RAFT_CUDA(cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    RAFT_CHECK(h == 0, std::string(what) + ": a bounded wait in the staging pipeline timed out");
}

void fbp_host_slab(const FbpConfig &cfg, int device, float *obj, const float *tomo, const float *angles,
                   int nslices)
{
    if (nslices <= 0) return;
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    FbpPrepared fp = prepare_fbp(cfg, device);
    FbpTables tb = fbp_tables(ds, fp, angles, ds.s_comp);
    const size_t in_ps = (size_t)cfg.nangles * cfg.nrays * sizeof(float);
    const size_t out_ps = (size_t)fp.No * fp.No * sizeof(float);
    const int chunk = auto_chunk(nslices, in_ps, cfg.blocksize);
    void *il = fbp_il_bytes(fp, chunk) ? ds.il.get(fbp_il_bytes(fp, chunk)) : nullptr;
    void *rows = (il && fbp_fused_il(fp)) ? nullptr : ds.rows.get(fbp_rows_bytes(fp, chunk));
    run_pipeline(ds, nslices, chunk, in_ps, out_ps, tomo, obj, [&](void *din, void *dout, int ns, cudaStream_t st) {
        fbp_chunk(ds, fp, tb, (const float *)din, (float *)dout, ns, rows, st, il);
    });
    check_device_flag(tb.err, "FBP");
}

// ------------------------------------------------------- rotation axis --
// getRotAxisCorrectionGPU (rotation_axis.cu:529-589): each row is edge-padded
// to 3N, shifted by a Fourier phase ramp and cropped back; the FBP filter's
// lowpass output path with a phase-only spectrum does exactly that.
void rotaxis_host_slab(int device, float *tomo, float axis_offset, int nrays, int nangles, int nslices,
                       int blocksize)
{
    if (nslices <= 0) return;
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    const int pad = 2;   // rotation_axis.cu:471
    // pixel 1: the spectrum's normalisation is then 1/Np, as opt::scale divides by nrays
    const FilterPlan &plan = cached_filter_plan(device, GEOM_FBP_REF, FILTER_AXIS_SHIFT, nrays, pad, 0.0, 0.0,
                                                (double)axis_offset, 1.0);
    const size_t ps = (size_t)nangles * nrays * sizeof(float);
    const int chunk = auto_chunk(nslices, ps, blocksize);
    run_pipeline(ds, nslices, chunk, ps, ps, tomo, tomo, [&](void *din, void *dout, int ns, cudaStream_t st) {
        FilterLaunch fl;
        fl.sino = (const float *)din;
        fl.out = dout;
        fl.nrows = ns * nangles;
        fl.nangles = nangles;
        fl.out_padded = 1;
        launch_filter(plan, fl, st);
    });
}

// Frames on the host -> the reference's integer or sub-pixel search result.
template <typename T>
double centersino_host(int device, const T *frame0, const T *frame1, const T *dark, const T *flat, int sizex,
                       int sizey, int subpixel)
{
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    const size_t plane = (size_t)sizex * sizey;
    T *d = (T *)ds.sino[0].get(4 * plane * sizeof(T));
    cudaStream_t st = ds.s_comp;
    const T *src[4] = {frame0, frame1, dark, flat};
    for (int k = 0; k < 4; k++)
        RAFT_CUDA(cudaMemcpyAsync(d + k * plane, src[k], plane * sizeof(T), cudaMemcpyHostToDevice, st));
    void *ws = ds.img[0].get(centersino_workspace_bytes(sizex, sizey));
    return centersino_device<T>(device, d, d + plane, d + 2 * plane, d + 3 * plane, sizex, sizey, subpixel, ws, st);
}

template double centersino_host<float>(int, const float *, const float *, const float *, const float *, int, int,
                                       int);
template double centersino_host<uint16_t>(int, const uint16_t *, const uint16_t *, const uint16_t *,
                                          const uint16_t *, int, int, int);

// ---------------------------------------------------------------- tEMFQ --
// _get_tEM_FQ_GPU (em_frequency.cu:301-331): slices in chunks; per chunk the
// counts, flat and initial guess go to the device, the EM runs there, the
// result comes back.
void temfq_host_slab(const TemfqConfig &cfg, int device, float *obj, const float *counts, const float *flat,
                     const float *angles, int nslices)
{
    if (nslices <= 0) return;
    const int N = cfg.nrays, A = cfg.nangles;
    RAFT_CHECK(temfq_shape_ok(N, A, cfg.zpad), "tEMFQ: unsupported sizes (N even; the N(1+zpad)- and "
                                               "N(1+zpad)/2-point transforms must fit shared memory: N(1+zpad) <= "
                                               "14528 with prime factors 2, 3, 5, 7, about 7000 otherwise)");
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    cudaStream_t st = ds.s_comp;
    const size_t per = temfq_workspace_bytes(N, A, cfg.zpad, 1);
    int chunk = (int)std::max<size_t>(1, ((size_t)8 << 30) / per);
    chunk = std::min(chunk, cfg.blocksize > 0 ? cfg.blocksize : 64);
    chunk = std::max(1, std::min(chunk, nslices));
    const size_t cps = (size_t)A * N, ops = (size_t)N * N;
    float *d_counts = (float *)ds.sino[0].get(cps * chunk * sizeof(float));
    float *d_obj = (float *)ds.img[0].get(ops * chunk * sizeof(float));
    float *d_flat = (float *)ds.flat.get((size_t)N * chunk * sizeof(float) + 16);
    float *d_ang = (float *)ds.angles.get(sizeof(float) * A);
    char *tb = (char *)ds.tabs.get(sizeof(float) * 3 * A + 64);
    float *cs = (float *)tb, *sn = cs + A, *wt = sn + A;
    void *ws = ds.rows.get(temfq_workspace_bytes(N, A, cfg.zpad, chunk));
    RAFT_CUDA(cudaMemcpyAsync(d_ang, angles, sizeof(float) * A, cudaMemcpyHostToDevice, st));
    launch_angle_tables(d_ang, A, cs, sn, wt, 0, st);   // __cosf / __sinf, as the reference's fast-math cosf/sinf
    for (int s0 = 0; s0 < nslices; s0 += chunk) {
        const int ns = std::min(chunk, nslices - s0);
        RAFT_CUDA(cudaMemcpyAsync(d_counts, counts + cps * s0, cps * ns * sizeof(float), cudaMemcpyHostToDevice, st));
        RAFT_CUDA(cudaMemcpyAsync(d_obj, obj + ops * s0, ops * ns * sizeof(float), cudaMemcpyHostToDevice, st));
        RAFT_CUDA(cudaMemcpyAsync(d_flat, flat + (size_t)N * s0, (size_t)N * ns * sizeof(float), cudaMemcpyHostToDevice,
                                  st));
        temfq_run(device, cfg, d_obj, d_counts, d_flat, cs, sn, ns, ws, st);
        RAFT_CUDA(cudaMemcpyAsync(obj + ops * s0, d_obj, ops * ns * sizeof(float), cudaMemcpyDeviceToHost, st));
        RAFT_CUDA(cudaStreamSynchronize(st));
    }
}

// ------------------------------------------------------------------ BST --
// getBSTGPU (bst.cu:534-642): slices stream through the two-slot pipeline;
// each chunk runs the three BST kernels (bst.cu in this library).
static int bst_chunk_slices(const BstPlanShape &sh, int nslices, int blocksize)
{
    // keep the per-chunk workspace near 4 GB (polar rows + crop columns)
    const size_t per = bst_workspace_bytes(sh, 1);
    int c = (int)std::max<size_t>(1, ((size_t)4 << 30) / std::max<size_t>(per, 1));
    c = std::min(c, 32);
    if (blocksize > 0) c = std::min(c, blocksize);
    return std::max(1, std::min(c, nslices));
}

void bst_host_slab(const FbpConfig &cfg, int device, float *obj, const float *tomo, int nslices)
{
    if (nslices <= 0) return;
    BstPlanShape sh;
    RAFT_CHECK(bst_plan_shape(sh, cfg.nrays, cfg.nangles, cfg.pad),
               "BST: the padded length N*(1+pad) is too long for the shared-memory transforms (at most 14528 with prime factors 2, 3, 5, 7; about 7000 otherwise)");
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    const size_t in_ps = (size_t)cfg.nangles * cfg.nrays * sizeof(float);
    const size_t out_ps = (size_t)cfg.nrays * cfg.nrays * sizeof(float);
    const int chunk = bst_chunk_slices(sh, nslices, cfg.blocksize);
    void *ws = ds.rows.get(bst_workspace_bytes(sh, chunk));
    run_pipeline(ds, nslices, chunk, in_ps, out_ps, tomo, obj, [&](void *din, void *dout, int ns, cudaStream_t st) {
        launch_bst(device, cfg, (const float *)din, (float *)dout, ns, ws, st);
    });
}

void bst_device(const FbpConfig &cfg, int device, float *d_obj, const float *d_tomo, int nslices, cudaStream_t st)
{
    BstPlanShape sh;
    RAFT_CHECK(bst_plan_shape(sh, cfg.nrays, cfg.nangles, cfg.pad),
               "BST: the padded length N*(1+pad) is too long for the shared-memory transforms (at most 14528 with prime factors 2, 3, 5, 7; about 7000 otherwise)");
    DeviceState &ds = device_state(device);
    const int chunk = bst_chunk_slices(sh, nslices, cfg.blocksize);
    void *ws = ds.rows.get(bst_workspace_bytes(sh, chunk));
    const size_t tps = (size_t)cfg.nangles * cfg.nrays, ops = (size_t)cfg.nrays * cfg.nrays;
    for (int s0 = 0; s0 < nslices; s0 += chunk) {
        const int ns = std::min(chunk, nslices - s0);
        launch_bst(device, cfg, d_tomo + tps * s0, d_obj + ops * s0, ns, ws, st);
    }
}

// -------------------------------------------------------------- lowpass --
void lowpass_host_slab(const FbpConfig &cfg, int device, float *tomo, int nslices)
{
    if (nslices <= 0 || cfg.filter == FILTER_NONE) return;   // low_pass.cu:24-25
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    // low_pass.cu:16: axis offset 0
    const FilterPlan &plan = cached_filter_plan(device, cfg.geometry, cfg.filter, cfg.nrays, cfg.pad, cfg.paganin,
                                                cfg.reg, 0.0, cfg.pixel_x);
    const size_t ps = (size_t)cfg.nangles * cfg.nrays * sizeof(float);
    const int chunk = auto_chunk(nslices, ps, cfg.blocksize);
    run_pipeline(ds, nslices, chunk, ps, ps, tomo, tomo, [&](void *din, void *dout, int ns, cudaStream_t st) {
        FilterLaunch fl;
        fl.sino = (const float *)din;
        fl.out = dout;
        fl.nrows = ns * cfg.nangles;
        fl.nangles = cfg.nangles;
        fl.out_padded = 1;
        launch_filter(plan, fl, st);
    });
}

// ------------------------------------------------------ flat / dark --
// getBackgroundCorrectionGPU (background_correction.cu:62-142): per device the
// slab's flats and darks are uploaded once; frames stream through the
// two-slot pipeline and come back corrected in place.
void background_host_slab(int device, float *frames, const float *flat, const float *dark, int nrays, int nangles,
                          int nslices, int numflats, int is_log, int blocksize)
{
    if (nslices <= 0) return;
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    const size_t fl_bytes = (size_t)nslices * numflats * nrays * sizeof(float);
    const size_t dk_bytes = (size_t)nslices * nrays * sizeof(float);
    const size_t dk_off = (fl_bytes + 255) & ~(size_t)255;
    char *aux = (char *)ds.flat.get(dk_off + dk_bytes);
    float *d_flat = (float *)aux, *d_dark = (float *)(aux + dk_off);
    RAFT_CUDA(cudaMemcpyAsync(d_flat, flat, fl_bytes, cudaMemcpyHostToDevice, ds.s_comp));
    RAFT_CUDA(cudaMemcpyAsync(d_dark, dark, dk_bytes, cudaMemcpyHostToDevice, ds.s_comp));
    const size_t ps = (size_t)nangles * nrays * sizeof(float);
    const int chunk = auto_chunk(nslices, ps, blocksize);
    int s0 = 0;   // first slice of the chunk being computed (chunks run in order)
    run_pipeline(ds, nslices, chunk, ps, ps, frames, frames, [&](void *din, void *dout, int ns, cudaStream_t st) {
        launch_background((const float *)din, (float *)dout, d_flat + (size_t)s0 * numflats * nrays,
                          d_dark + (size_t)s0 * nrays, nrays, nangles, ns, numflats, is_log, st);
        s0 += ns;
    });
}

// ---------------------------------------------------------------- Radon --
void radon_host_slab(int device, float *proj, const float *img, const float *angles, int nx, int ny, int nrays,
                     int nangles, int nslices, float ax, float ay)
{
    if (nslices <= 0) return;
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    float *d_ang = (float *)ds.angles.get(sizeof(float) * nangles);
    RAFT_CUDA(cudaMemcpy(d_ang, angles, sizeof(float) * nangles, cudaMemcpyHostToDevice));
    const size_t in_ps = (size_t)nx * ny * sizeof(float);
    const size_t out_ps = (size_t)nangles * nrays * sizeof(float);
    const int chunk = auto_chunk(nslices, std::max(in_ps, out_ps), 0);
    void *scratch = ds.imgT.get(proj_scratch_bytes(nx, ny, chunk));
    run_pipeline(ds, nslices, chunk, in_ps, out_ps, img, proj, [&](void *din, void *dout, int ns, cudaStream_t st) {
        ProjLaunch pl;
        pl.img = (const float *)din;
        pl.out = (float *)dout;
        pl.angles = d_ang;
        pl.nx = nx;
        pl.ny = ny;
        pl.nrays = nrays;
        pl.nangles = nangles;
        pl.nslices = ns;
        pl.ax = ax;
        pl.ay = ay;
        pl.em = 0;
        stage_proj_images(pl, scratch, st);
        launch_project(pl, st);
    });
}

// ------------------------------------------------------------------- EM --
EmPrepared prepare_em(const EmConfig &cfg)
{
    EmPrepared ep;
    ep.cfg = cfg;
    const int N = cfg.objsize, n = cfg.nrays;
    // em_RT_kernel.cu:97-102: dxy = 2.0/(N-1), dt = 2.0/(nrays-1) (double -> float), tmin = -1
    ep.geo.dxy = (float)(2.0 / (N - 1));
    ep.geo.dt = (float)(2.0 / (n - 1));
    ep.geo.tmin = -1.0f;
    BpPlanInput pi;
    pi.geometry = GEOM_EM_REF;
    pi.store = STORE_F32;
    pi.No = N;
    pi.dxy = ep.geo.dxy;
    pi.tmin = ep.geo.tmin;
    pi.dt = ep.geo.dt;
    ep.win = plan_window(pi);
    // every stored bin must be reachable by the projector's writes or stay zero
    return ep;
}

void em_chunk(DeviceState &ds, const EmPrepared &ep, int kind, const float *d_data, const float *d_flat,
              const float *h_angles, float *d_obj, int nslices, double *d_metrics, bool use_graph, cudaStream_t st)
{
    const EmConfig &c = ep.cfg;
    const int A = c.nangles, n = c.nrays, N = c.objsize;
    float *d_ang = (float *)ds.angles.get(sizeof(float) * A);
    RAFT_CUDA(cudaMemcpyAsync(d_ang, h_angles, sizeof(float) * A, cudaMemcpyHostToDevice, st));
    char *tb = (char *)ds.tabs.get(sizeof(float) * 3 * A + 64);
    float *cs = (float *)tb, *sn = cs + A, *wt = sn + A;
    int *err = (int *)ds.err.get(sizeof(int));
    RAFT_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    launch_angle_tables(d_ang, A, cs, sn, wt, 1, st);

    const WindowLayout &win = ep.win;
    const size_t rows_bytes = (size_t)nslices * A * win.Wg * sizeof(float);
    float *rows = (float *)ds.rows.get(rows_bytes);
    RAFT_CUDA(cudaMemsetAsync(rows, 0, rows_bytes, st));
    float *den = (float *)ds.den.get((size_t)nslices * N * N * sizeof(float));

    BpLaunch bl;
    bl.filt = rows;
    bl.No = N;
    bl.nangles = A;
    bl.nslices = nslices;
    bl.geometry = GEOM_EM_REF;
    bl.store = STORE_F32;
    bl.win = win;
    bl.geo = ep.geo;
    bl.cs = cs;
    bl.sn = sn;
    bl.err = err;
    bl.il_ws = ds.il.get(bp_il_bytes(nslices, A, win.Wg, 4));

    // sensitivity image: BP of the counts (tEM, em_rt.cu:178) or of ones (eEM, :343)
    launch_to_window(kind == 0 ? d_data : nullptr, rows, wt, nslices * A, A, n, win.wlo, win.Wg, st);
    bl.img = den;
    bl.den = nullptr;
    launch_backproject(bl, st);

    void *scratch = ds.imgT.get(proj_scratch_bytes(N, N, nslices));
    ProjLaunch pl;
    pl.img = d_obj;
    pl.out = rows;
    pl.angles = d_ang;
    pl.nx = N;
    pl.ny = N;
    pl.nrays = n;
    pl.nangles = A;
    pl.nslices = nslices;
    pl.ax = 1.0f;
    pl.ay = 1.0f;
    pl.em = 1;
    pl.epilogue = kind == 0 ? 1 : 2;
    pl.flat = d_flat;
    pl.data = d_data;
    pl.wt = wt;
    // the projector writes the window rows interleaved by slice, as the
    // four-slice backprojector stages them: no separate interleave pass per
    // iteration (margins and slices past the batch stay zero from this clear)
    pl.windowed = 2;
    pl.out = static_cast<float *>(bl.il_ws);
    RAFT_CUDA(cudaMemsetAsync(bl.il_ws, 0, bp_il_bytes(nslices, A, win.Wg, 4), st));
    pl.wlo = win.wlo;
    pl.Wg = win.Wg;
    bl.img = d_obj;
    bl.den = den;
    bl.il_ready = 1;
    if (d_metrics)
        RAFT_CUDA(cudaMemsetAsync(d_metrics, 0, sizeof(double) * 3 * nslices * (size_t)c.niter, st));

    auto body = [&]() {
        for (int it = 0; it < c.niter; it++) {
            pl.metrics = d_metrics ? d_metrics + (size_t)it * nslices * 3 : nullptr;
            stage_proj_images(pl, scratch, st);
            launch_project(pl, st);
            launch_backproject(bl, st);
        }
    };
    if (use_graph && c.niter > 0) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        RAFT_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            body();
        } catch (...) {
            cudaStreamEndCapture(st, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        RAFT_CUDA(cudaStreamEndCapture(st, &graph));
        RAFT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        RAFT_CUDA(cudaGraphLaunch(exec, st));
        RAFT_CUDA(cudaStreamSynchronize(st));
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
    } else {
        body();
    }
    RAFT_CUDA(cudaStreamSynchronize(st));
    check_device_flag(err, "EM");
}

void em_host_slab(const EmConfig &cfg, int kind, int device, float *obj, const float *data, const float *flat,
                  const float *angles, int nslices, bool flat_by_angle)
{
    (void)flat_by_angle;
    if (nslices <= 0) return;
    DeviceState &ds = device_state(device);
    std::lock_guard<std::mutex> lk(ds.mtx);
    RAFT_CUDA(cudaSetDevice(device));
    ds.ensure();
    EmPrepared ep = prepare_em(cfg);
    const int A = cfg.nangles, n = cfg.nrays, N = cfg.objsize;
    const size_t data_ps = (size_t)A * n * sizeof(float);
    const size_t obj_ps = (size_t)N * N * sizeof(float);
    const int chunk = auto_chunk(nslices, data_ps + obj_ps, cfg.blocksize);
    float *d_data = (float *)ds.sino[0].get(data_ps * chunk);
    float *d_obj = (float *)ds.img[0].get(obj_ps * chunk);
    float *d_flat = (float *)ds.flat.get((size_t)n * chunk * sizeof(float) + 16);
    cudaStream_t st = ds.s_comp;
    for (int s0 = 0; s0 < nslices; s0 += chunk) {
        const int ns = std::min(chunk, nslices - s0);
        RAFT_CUDA(cudaMemcpyAsync(d_data, data + (size_t)s0 * A * n, data_ps * ns, cudaMemcpyHostToDevice, st));
        RAFT_CUDA(cudaMemcpyAsync(d_obj, obj + (size_t)s0 * N * N, obj_ps * ns, cudaMemcpyHostToDevice, st));
        if (kind == 0)
            RAFT_CUDA(cudaMemcpyAsync(d_flat, flat + (size_t)s0 * n, sizeof(float) * n * ns, cudaMemcpyHostToDevice,
                                      st));
        em_chunk(ds, ep, kind, d_data, d_flat, angles, d_obj, ns, nullptr, true, st);
        RAFT_CUDA(cudaMemcpyAsync(obj + (size_t)s0 * N * N, d_obj, obj_ps * ns, cudaMemcpyDeviceToHost, st));
        RAFT_CUDA(cudaStreamSynchronize(st));
    }
}

}  // namespace raft
