// api.cpp -- the C ABI of libraft.so.
//
// The five reference entry points keep their exact names and signatures
// (void return, packed int/float parameter arrays, host pointers), so the
// ssc-raft ctypes layer binds them unchanged.  They never exit the process:
// failures are recorded and read back with raft_last_error().  Extensions
// (operator mode, sinogram storage precision, device-resident buffers, EM
// residual metrics) are separate exports; see include/raft_b200.h.
#include "engine.hpp"

#include <cmath>
#include <initializer_list>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace raft {

// --------------------------------------------------------------- status --
static thread_local std::string t_error;

void set_error(const std::string &msg)
{
    if (t_error.empty()) t_error = msg;
}
bool has_error() { return !t_error.empty(); }
std::string get_error() { return t_error; }
void clear_error() { t_error.clear(); }

// ----------------------------------------------------------- parameters --
// setFBPParameters, cuda/src/geometries/parallel/reconstruction_methods/parameters.cu:131-219
static bool parse_fbp_arrays(const float *paramf, const int *parami, FbpConfig &c, bool need_obj)
{
    if (!paramf || !parami) {
        set_error("null parameter array");
        return false;
    }
    c.nrays = parami[0];
    c.nangles = parami[1];
    c.nslices = parami[2];
    c.objsize = parami[3];
    c.pad = parami[4];
    c.filter = parami[7];
    c.blocksize = parami[9];
    c.beta_delta = paramf[0];
    c.reg = paramf[1];
    c.energy = paramf[2];
    c.z2 = paramf[3];
    c.pixel_x = paramf[4];
    c.pixel_y = paramf[5];
    c.offset = paramf[6];
    // parameters.cu:201-203 (float arithmetic; plank*vc in double as there)
    float wavelength = (c.beta_delta == 0.0f) ? 1.0f : (float)((4.135667696E-15 * 299792458) / c.energy);
    c.paganin = wavelength * c.z2 * float(M_PI) * c.beta_delta / (c.pixel_x * c.pixel_x);
    if (c.nrays < 2 || c.nangles < 1 || c.nslices < 0 || c.pad < 0 || c.pad > 64) {
        set_error("invalid sizes: need nrays >= 2, nangles >= 1, nslices >= 0, 0 <= pad <= 64");
        return false;
    }
    if (need_obj && c.objsize < 1) {
        set_error("invalid object size");
        return false;
    }
    if (c.filter < 0 || c.filter > 9) {
        set_error("invalid filter type (valid: 0..9)");
        return false;
    }
    if (!(c.pixel_x > 0.f) || !(c.pixel_y > 0.f) || !std::isfinite(c.pixel_x) || !std::isfinite(c.pixel_y)) {
        set_error("invalid pixel size");
        return false;
    }
    return true;
}

// setEMRTParameters, parameters.cu:8-59
static bool parse_em_arrays(const float *paramf, const int *parami, EmConfig &c)
{
    (void)paramf;
    if (!parami) {
        set_error("null parameter array");
        return false;
    }
    c.nrays = parami[0];
    c.nangles = parami[1];
    c.nslices = parami[2];
    c.objsize = parami[3];
    c.nflats = parami[7];
    c.niter = parami[8];
    c.blocksize = parami[9];
    if (c.nrays < 2 || c.nangles < 2 || c.nslices < 0 || c.objsize < 2 || c.niter < 0) {
        set_error("invalid EM sizes: need nrays >= 2, nangles >= 2, objsize >= 2, iterations >= 0");
        return false;
    }
    if (c.objsize != c.nrays) {
        set_error("EM requires objsize == nrays (em_methods.py:31,107)");
        return false;
    }
    return true;
}

static bool check_gpus(const int *gpus, int ngpus)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        set_error("no CUDA device available");
        return false;
    }
    if (!gpus || ngpus < 1) {
        set_error("empty GPU list");
        return false;
    }
    for (int i = 0; i < ngpus; i++)
        if (gpus[i] < 0 || gpus[i] >= count) {
            set_error("invalid device number " + std::to_string(gpus[i]));
            return false;
        }
    return true;
}

// Data pointers of a call with work to do must not be null (an empty batch
// may pass null).
static bool ptrs_ok(int nslices, std::initializer_list<const void *> ptrs, const char *name)
{
    if (nslices <= 0) return true;
    for (const void *p : ptrs)
        if (!p) {
            set_error(std::string(name) + ": null data pointer");
            return false;
        }
    return true;
}

// Operator / sinogram storage pairs of the FBP entry points: 0/0 (nearest,
// reference), 1/1 (linear, FP32 pairs), 1/2 (linear, BF16 pairs).
static bool fbp_mode_ok(int geometry, int store, const char *name)
{
    const bool ok = (geometry == GEOM_FBP_REF && store == STORE_F32) ||
                    (geometry == GEOM_FBP_LIN && (store == STORE_PAIR_F32 || store == STORE_PAIR_BF16));
    if (!ok)
        set_error(std::string(name) + ": geometry/store must be 0/0 (nearest), 1/1 (linear fp32) or 1/2 "
                                      "(linear bf16)");
    return ok;
}

// Contiguous z-slabs of ceil(nslices/ngpus) slices, the last ones shorter or
// empty (fbp.cu:267-301).
static void slab_partition(int nslices, int ngpus, int *start, int *count)
{
    const int sub = (nslices + ngpus - 1) / ngpus;
    int ptr = 0;
    for (int i = 0; i < ngpus; i++) {
        const int n = std::max(0, std::min(nslices - ptr, sub));
        start[i] = ptr;
        count[i] = n;
        ptr += n;
    }
}

// One host thread per device over its slab; errors from worker threads are
// carried back into the caller's status.
template <class F>
static void split_slabs(const int *gpus, int ngpus, int nslices, F work)
{
    if (ngpus == 1) {
        try {
            work(gpus[0], 0, nslices);
        } catch (const CudaFail &) {
        } catch (const std::exception &e) {
            set_error(e.what());
        }
        return;
    }
    std::vector<std::thread> th;
    std::vector<std::string> errs(ngpus);
    std::vector<int> starts(ngpus), counts(ngpus);
    slab_partition(nslices, ngpus, starts.data(), counts.data());
    for (int i = 0; i < ngpus; i++) {
        const int n = counts[i];
        const int start = starts[i];
        th.emplace_back([&, i, start, n] {
            try {
                work(gpus[i], start, n);
            } catch (const CudaFail &) {
            } catch (const std::exception &e) {
                set_error(e.what());
            }
            errs[i] = get_error();
        });
    }
    for (auto &t : th) t.join();
    for (auto &e : errs)
        if (!e.empty()) {
            set_error(e);
            break;
        }
}

// Non-static access for other translation units (the no-allocation entry point).
bool parse_fbp_params(const float *paramf, const int *parami, FbpConfig &cfg)
{
    return parse_fbp_arrays(paramf, parami, cfg, true);
}

bool check_gpu_id(int gpu) { return check_gpus(&gpu, 1); }

}  // namespace raft

using namespace raft;

template <typename T>
static double centersino_entry(const T *frame0, const T *frame180, const T *dark, const T *flat, int sizex, int sizey,
                               int subpixel, const char *name)
{
    clear_error();
    if (!frame0 || !frame180 || !dark || !flat) {
        set_error(std::string(name) + ": null frame pointer");
        return 0.0;
    }
    if (!centersino_shape_ok(sizex, sizey)) {
        set_error(std::string(name) + ": frame sides too long for the shared-memory transforms (at most 14528 with "
                                      "prime factors 2, 3, 5, 7, about 7000 otherwise)");
        return 0.0;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = 0;
    }
    if (!check_gpu_id(dev)) return 0.0;
    try {
        return centersino_host<T>(dev, frame0, frame180, dark, flat, sizex, sizey, subpixel);
    } catch (const CudaFail &) {
    }
    return 0.0;
}

extern "C" {

int raft_last_error(char *buf, int len)
{
    const std::string &e = t_error;
    if (buf && len > 0) {
        const int n = (int)std::min<size_t>(e.size(), (size_t)len - 1);
        std::memcpy(buf, e.data(), n);
        buf[n] = 0;
    }
    return e.empty() ? 0 : 1;
}

void raft_clear_error(void) { clear_error(); }

// Failure injection: the next n device-buffer requests of the library fail (as
// an out-of-memory would): the entry point reports the error and the library
// stays usable.  n = 0 clears it.
void raft_inject_alloc_failures(int n) { inject_alloc_failures(n); }

// Self test of the bounded device-side wait the staging pipelines use: returns
// 1 if a wait on a barrier nothing arrives on (arrive = 0) ran out after `limit`
// polls and was reported, 0 if the wait completed (arrive = 1), -1 on error.
int raft_selftest_bounded_wait(int gpu, int arrive, unsigned limit)
{
    clear_error();
    if (!check_gpus(&gpu, 1)) return -1;
    try {
        return selftest_bounded_wait(gpu, arrive, limit);
    } catch (const CudaFail &) {
    }
    return -1;
}

int raft_abi_version(void) { return 1; }

// Host-only: the slab each of `ngpus` devices receives for `nslices` slices.
int raft_slab_partition(int nslices, int ngpus, int *start, int *count)
{
    clear_error();
    if (nslices < 0 || ngpus < 1 || !start || !count) {
        set_error("raft_slab_partition: bad arguments");
        return 1;
    }
    slab_partition(nslices, ngpus, start, count);
    return 0;
}

// JSON list of the backprojector launch shapes chosen so far by the autotuner.
int raft_autotune_table(char *buf, int len)
{
    const std::string t = bp_tune_table();
    if (buf && len > 0) {
        const int n = (int)std::min<size_t>(t.size(), (size_t)len - 1);
        std::memcpy(buf, t.data(), n);
        buf[n] = 0;
    }
    return (int)t.size();
}

// --- FBP ------------------------------------------------------------------
static void fbp_common(int *gpus, int ngpus, float *obj, const float *tomogram, const float *angles,
                       const float *paramf, const int *parami, int geometry, int store)
{
    clear_error();
    FbpConfig cfg;
    if (!parse_fbp_arrays(paramf, parami, cfg, true)) return;
    if (!check_gpus(gpus, ngpus)) return;
    if (!obj || !tomogram || !angles) {
        set_error("null data pointer");
        return;
    }
    cfg.geometry = geometry;
    cfg.store = store;
    const size_t obj_ps = (size_t)cfg.objsize * cfg.objsize, tomo_ps = (size_t)cfg.nangles * cfg.nrays;
    split_slabs(gpus, ngpus, cfg.nslices, [&](int dev, int start, int n) {
        fbp_host_slab(cfg, dev, obj + obj_ps * start, tomogram + tomo_ps * start, angles, n);
    });
}

// Reference: getFBPMultiGPU, cuda/src/geometries/parallel/reconstruction_methods/fbp.cu:238-302
void getFBPMultiGPU(int *gpus, int ngpus, float *obj, float *tomogram, float *angles, float *paramf, int *parami)
{
    fbp_common(gpus, ngpus, obj, tomogram, angles, paramf, parami, GEOM_FBP_REF, STORE_F32);
}

int raft_fbp_ext(int *gpus, int ngpus, float *obj, const float *tomogram, const float *angles, const float *paramf,
                 const int *parami, int geometry, int store)
{
    if (geometry != GEOM_FBP_REF && geometry != GEOM_FBP_LIN) {
        clear_error();
        set_error("raft_fbp_ext: geometry must be 0 (nearest, reference) or 1 (linear)");
        return 1;
    }
    if (store < 0 || store > 2 || (geometry == GEOM_FBP_REF && store != STORE_F32) ||
        (geometry == GEOM_FBP_LIN && store == STORE_F32)) {
        clear_error();
        set_error("raft_fbp_ext: store must be 0 with geometry 0, 1 (fp32) or 2 (bf16) with geometry 1");
        return 1;
    }
    fbp_common(gpus, ngpus, obj, tomogram, angles, paramf, parami, geometry, store);
    return has_error() ? 1 : 0;
}

// Device-resident FBP on one GPU: d_obj / d_tomogram are device pointers on
// `gpu`, angles is host.  Runs on `stream`; 0 = after the work already queued
// on the legacy default stream, on the library's own stream, synchronised
// before returning.
int raft_fbp_device(int gpu, float *d_obj, const float *d_tomogram, const float *angles, const float *paramf,
                    const int *parami, int geometry, int store, void *stream)
{
    clear_error();
    FbpConfig cfg;
    if (!parse_fbp_arrays(paramf, parami, cfg, true)) return 1;
    if (!fbp_mode_ok(geometry, store, "raft_fbp_device")) return 1;
    if (!ptrs_ok(cfg.nslices, {d_obj, d_tomogram, angles}, "raft_fbp_device")) return 1;
    if (!check_gpus(&gpu, 1)) return 1;
    cfg.geometry = geometry;
    cfg.store = store;
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        cudaStream_t st = resolve_stream(ds, stream, ds.s_comp);
        FbpPrepared fp = prepare_fbp(cfg, gpu);
        FbpTables tb = fbp_tables(ds, fp, angles, st);
        const size_t tomo_ps = (size_t)cfg.nangles * cfg.nrays;
        const int chunk = std::max(1, std::min(cfg.nslices, cfg.blocksize > 0 ? cfg.blocksize : 32));
        void *il = fbp_il_bytes(fp, chunk) ? ds.il.get(fbp_il_bytes(fp, chunk)) : nullptr;
        void *rows = (il && fbp_fused_il(fp)) ? nullptr : ds.rows.get(fbp_rows_bytes(fp, chunk));
        for (int s0 = 0; s0 < cfg.nslices; s0 += chunk) {
            const int ns = std::min(chunk, cfg.nslices - s0);
            fbp_chunk(ds, fp, tb, d_tomogram + tomo_ps * s0, d_obj + (size_t)fp.No * fp.No * s0, ns, rows, st, il);
        }
        if (!stream) RAFT_CUDA(cudaStreamSynchronize(st));
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

// --- lowpass --------------------------------------------------------------
// Reference: getFilterLowPassMultiGPU, cuda/src/processing/filters/low_pass.cu:84-141
void getFilterLowPassMultiGPU(int *gpus, int ngpus, float *tomogram, float *paramf, int *parami)
{
    clear_error();
    FbpConfig cfg;
    if (!parse_fbp_arrays(paramf, parami, cfg, false)) return;
    if (!check_gpus(gpus, ngpus)) return;
    if (!tomogram) {
        set_error("null data pointer");
        return;
    }
    const size_t ps = (size_t)cfg.nangles * cfg.nrays;
    split_slabs(gpus, ngpus, cfg.nslices,
                [&](int dev, int start, int n) { lowpass_host_slab(cfg, dev, tomogram + ps * start, n); });
}

// --- flat / dark correction ---------------------------------------------------
// Reference: getBackgroundCorrectionMultiGPU, cuda/src/processing/background_correction.cu:144-178
static bool check_background(int nrays, int nangles, int nslices, int numflats, int is_log)
{
    if (nrays < 1 || nangles < 1 || nslices < 0 || numflats < 1 || (is_log != 0 && is_log != 1)) {
        set_error("background correction: need nrays, nangles, numflats >= 1, nslices >= 0, is_log 0 or 1");
        return false;
    }
    return true;
}

void getBackgroundCorrectionMultiGPU(int *gpus, int ngpus, float *frames, float *flat, float *dark, int nrays,
                                     int nangles, int nslices, int numflats, int is_log, int blocksize)
{
    clear_error();
    if (!check_background(nrays, nangles, nslices, numflats, is_log)) return;
    if (!check_gpus(gpus, ngpus)) return;
    if (!frames || !flat || !dark) {
        set_error("null data pointer");
        return;
    }
    const size_t ps = (size_t)nangles * nrays;
    split_slabs(gpus, ngpus, nslices, [&](int dev, int start, int n) {
        background_host_slab(dev, frames + ps * start, flat + (size_t)numflats * nrays * start,
                             dark + (size_t)nrays * start, nrays, nangles, n, numflats, is_log, blocksize);
    });
}

// Device-resident flat/dark correction on one GPU, in place on d_frames.
int raft_background_device(int gpu, float *d_frames, const float *d_flat, const float *d_dark, int nrays,
                           int nangles, int nslices, int numflats, int is_log, void *stream)
{
    clear_error();
    if (!check_background(nrays, nangles, nslices, numflats, is_log)) return 1;
    if (!ptrs_ok(nslices, {d_frames, d_flat, d_dark}, "raft_background_device")) return 1;
    if (!check_gpus(&gpu, 1)) return 1;
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        cudaStream_t st = resolve_stream(ds, stream, ds.s_comp);
        launch_background(d_frames, d_frames, d_flat, d_dark, nrays, nangles, nslices, numflats, is_log, st);
        if (!stream) RAFT_CUDA(cudaStreamSynchronize(st));
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

// --- Radon ----------------------------------------------------------------
// Reference: getRadonRTMultiGPU, cuda/src/geometries/parallel/forward_methods/radon_rt.cu:252-295
void getRadonRTMultiGPU(int *gpus, int ngpus, float *tomogram, float *phantom, float *angles, int sizex, int sizey,
                        int nrays, int nangles, int nslices, float ax, float ay)
{
    clear_error();
    if (sizex < 2 || sizey < 2 || nrays < 1 || nangles < 1 || nslices < 0) {
        set_error("invalid Radon sizes");
        return;
    }
    if (!check_gpus(gpus, ngpus)) return;
    if (!tomogram || !phantom || !angles) {
        set_error("null data pointer");
        return;
    }
    split_slabs(gpus, ngpus, nslices, [&](int dev, int start, int n) {
        radon_host_slab(dev, tomogram + (size_t)start * nrays * nangles, phantom + (size_t)start * sizex * sizey,
                        angles, sizex, sizey, nrays, nangles, n, ax, ay);
    });
}

// --- EM -------------------------------------------------------------------
static void em_common(int kind, int *gpus, int ngpus, float *obj, const float *data, const float *flat,
                      const float *angles, const float *paramf, const int *parami)
{
    clear_error();
    EmConfig cfg;
    if (!parse_em_arrays(paramf, parami, cfg)) return;
    if (!check_gpus(gpus, ngpus)) return;
    if (!obj || !data || !angles || (kind == 0 && !flat)) {
        set_error("null data pointer");
        return;
    }
    const size_t ops = (size_t)cfg.objsize * cfg.objsize, dps = (size_t)cfg.nangles * cfg.nrays;
    split_slabs(gpus, ngpus, cfg.nslices, [&](int dev, int start, int n) {
        em_host_slab(cfg, kind, dev, obj + ops * start, data + dps * start,
                     flat ? flat + (size_t)cfg.nrays * start : nullptr, angles, n, false);
    });
}

// Reference: get_tEM_RT_MultiGPU, cuda/src/geometries/parallel/reconstruction_methods/em_rt.cu:12-84
void get_tEM_RT_MultiGPU(int *gpus, int ngpus, float *obj, float *count, float *flat, float *angles, float *paramf,
                         int *parami)
{
    em_common(0, gpus, ngpus, obj, count, flat, angles, paramf, parami);
}

// Reference: get_eEM_RT_MultiGPU, em_rt.cu:201-262
void get_eEM_RT_MultiGPU(int *gpus, int ngpus, float *obj, float *tomogram, float *angles, float *paramf,
                         int *parami)
{
    em_common(1, gpus, ngpus, obj, tomogram, nullptr, angles, paramf, parami);
}

// Single-GPU EM with per-iteration FP64 metrics [niter][nslices][3]
// (sum (model-data)^2, sum data^2, negative log-likelihood) copied to the
// host buffer `metrics` (may be NULL).  kind 0 = tEM, 1 = eEM.
int raft_em_ext(int kind, int gpu, float *obj, const float *data, const float *flat, const float *angles, int nrays,
                int nangles, int nslices, int niter, double *metrics, int use_graph)
{
    clear_error();
    int parami[10] = {nrays, nangles, nslices, nrays, 0, 0, 0, 1, niter, 0};
    EmConfig cfg;
    if (!parse_em_arrays(nullptr, parami, cfg)) return 1;
    if (kind != 0 && kind != 1) {
        set_error("raft_em_ext: kind must be 0 (tEM) or 1 (eEM)");
        return 1;
    }
    if (!ptrs_ok(nslices, {obj, data, angles, kind == 0 ? flat : obj}, "raft_em_ext")) return 1;
    if (!check_gpus(&gpu, 1)) return 1;
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        EmPrepared ep = prepare_em(cfg);
        cudaStream_t st = ds.s_comp;
        const size_t dps = (size_t)nangles * nrays, ops = (size_t)nrays * nrays;
        float *d_data = (float *)ds.sino[0].get(dps * nslices * sizeof(float));
        float *d_obj = (float *)ds.img[0].get(ops * nslices * sizeof(float));
        float *d_flat = (float *)ds.flat.get((size_t)nrays * nslices * sizeof(float) + 16);
        double *d_met = metrics ? (double *)ds.metrics.get(sizeof(double) * 3 * (size_t)nslices * niter + 8) : nullptr;
        RAFT_CUDA(cudaMemcpyAsync(d_data, data, dps * nslices * sizeof(float), cudaMemcpyHostToDevice, st));
        RAFT_CUDA(cudaMemcpyAsync(d_obj, obj, ops * nslices * sizeof(float), cudaMemcpyHostToDevice, st));
        if (kind == 0)
            RAFT_CUDA(cudaMemcpyAsync(d_flat, flat, (size_t)nrays * nslices * sizeof(float), cudaMemcpyHostToDevice,
                                      st));
        em_chunk(ds, ep, kind, d_data, d_flat, angles, d_obj, nslices, d_met, use_graph != 0, st);
        RAFT_CUDA(cudaMemcpyAsync(obj, d_obj, ops * nslices * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (metrics)
            RAFT_CUDA(cudaMemcpyAsync(metrics, d_met, sizeof(double) * 3 * (size_t)nslices * niter,
                                      cudaMemcpyDeviceToHost, st));
        RAFT_CUDA(cudaStreamSynchronize(st));
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

// Device-resident EM on one GPU (all pointers device, angles host).
int raft_em_device(int kind, int gpu, float *d_obj, const float *d_data, const float *d_flat, const float *angles,
                   int nrays, int nangles, int nslices, int niter, double *d_metrics, int use_graph, void *stream)
{
    clear_error();
    int parami[10] = {nrays, nangles, nslices, nrays, 0, 0, 0, 1, niter, 0};
    EmConfig cfg;
    if (!parse_em_arrays(nullptr, parami, cfg)) return 1;
    if (kind != 0 && kind != 1) {
        set_error("raft_em_device: kind must be 0 (tEM) or 1 (eEM)");
        return 1;
    }
    if (!ptrs_ok(nslices, {d_obj, d_data, angles, kind == 0 ? d_flat : d_obj}, "raft_em_device")) return 1;
    if (!check_gpus(&gpu, 1)) return 1;
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        EmPrepared ep = prepare_em(cfg);
        cudaStream_t st = resolve_stream(ds, stream, ds.s_comp);
        em_chunk(ds, ep, kind, d_data, d_flat, angles, d_obj, nslices, d_metrics, use_graph != 0, st);
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

// Host-only: the window layout the backprojector would use (for tests of
// the bounds logic without a GPU).  geometry/store as raft_fbp_ext; for
// geometry 2 (EM) paramf/parami follow the EM packing.  out = {wlo, Wg, W, align}.
int raft_plan_window(const float *paramf, const int *parami, int geometry, int store, int *out)
{
    clear_error();
    try {
        if (geometry == GEOM_EM_REF) {
            EmConfig c;
            if (!parse_em_arrays(paramf, parami, c)) return 1;
            EmPrepared ep = prepare_em(c);
            out[0] = ep.win.wlo; out[1] = ep.win.Wg; out[2] = ep.win.W; out[3] = ep.win.align;
            return 0;
        }
        FbpConfig c;
        if (!parse_fbp_arrays(paramf, parami, c, true)) return 1;
        c.geometry = geometry;
        c.store = store;
        const int N = c.nrays, No = c.objsize, pad = c.pad;
        BpPlanInput pi;
        pi.geometry = geometry;
        pi.store = store;
        pi.No = No;
        const int Np = N * (1 + pad), Npo = No * (1 + pad);
        pi.xmin = -c.pixel_x * (float)Npo / 2.0f;
        pi.ymin = -c.pixel_y * (float)Npo / 2.0f;
        pi.dx = c.pixel_x;
        pi.dy = c.pixel_y;
        pi.tmin = -c.pixel_x * (float)Np / 2.0f;
        pi.dt = c.pixel_x;
        pi.offo = (pad * No) / 2;
        WindowLayout w = plan_window(pi);
        out[0] = w.wlo; out[1] = w.Wg; out[2] = w.W; out[3] = w.align;
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

// sin/cos of `angles` as the GPU's fast intrinsics produce them: kind 0 =
// __sinf/__cosf (FBP table, opt.cu:187-194; the projectors' fast-math
// sinf/cosf), kind 1 = __sincosf (EM backprojector, em_RT_kernel.cu:120).
int raft_fast_sincos(int gpu, const float *angles, int n, int kind, float *cos_out, float *sin_out)
{
    clear_error();
    if (!check_gpus(&gpu, 1)) return 1;
    if (n < 1 || !angles || !cos_out || !sin_out) {
        set_error("raft_fast_sincos: bad arguments");
        return 1;
    }
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        float *d = (float *)ds.angles.get(sizeof(float) * 3 * (size_t)n);
        RAFT_CUDA(cudaMemcpy(d, angles, sizeof(float) * n, cudaMemcpyHostToDevice));
        launch_angle_tables(d, n, d + n, d + 2 * n, nullptr, kind, ds.s_comp);
        RAFT_CUDA(cudaStreamSynchronize(ds.s_comp));
        RAFT_CUDA(cudaMemcpy(cos_out, d + n, sizeof(float) * n, cudaMemcpyDeviceToHost));
        RAFT_CUDA(cudaMemcpy(sin_out, d + 2 * n, sizeof(float) * n, cudaMemcpyDeviceToHost));
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

// Radon RT on device-resident buffers of one GPU (d_phantom [nslices][ny][nx],
// d_out [nslices][nangles][nrays], angles host); no Python-side scaling.
int raft_radon_device(int gpu, float *d_out, const float *d_phantom, const float *angles, int nx, int ny, int nrays,
                      int nangles, int nslices, float ax, float ay, void *stream)
{
    clear_error();
    if (nx < 2 || ny < 2 || nrays < 1 || nangles < 1 || nslices < 0) {
        set_error("invalid Radon sizes");
        return 1;
    }
    if (!ptrs_ok(nslices, {d_out, d_phantom, angles}, "raft_radon_device")) return 1;
    if (!check_gpus(&gpu, 1)) return 1;
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        cudaStream_t st = resolve_stream(ds, stream, ds.s_comp);
        float *d_ang = (float *)ds.angles.get(sizeof(float) * nangles);
        RAFT_CUDA(cudaMemcpyAsync(d_ang, angles, sizeof(float) * nangles, cudaMemcpyHostToDevice, st));
        void *scratch = ds.imgT.get(proj_scratch_bytes(nx, ny, nslices));
        ProjLaunch pl;
        pl.img = d_phantom;
        pl.out = d_out;
        pl.angles = d_ang;
        pl.nx = nx;
        pl.ny = ny;
        pl.nrays = nrays;
        pl.nangles = nangles;
        pl.nslices = nslices;
        pl.ax = ax;
        pl.ay = ay;
        stage_proj_images(pl, scratch, st);
        launch_project(pl, st);
        if (!stream) RAFT_CUDA(cudaStreamSynchronize(st));
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

// --- rotation axis --------------------------------------------------------------
// Reference: findcentersino / findcentersino_subpixel / findcentersino16,
// cuda/src/processing/rotation_axis.cu:429-451 (host frames [sizey][sizex], the
// calling thread's current device); getRotAxisCorrectionMultiGPU :591-643;
// correctRotationAxis (host shift) :396-426.
int findcentersino(float *frame0, float *frame180, float *dark, float *flat, int sizex, int sizey)
{
    return (int)centersino_entry<float>(frame0, frame180, dark, flat, sizex, sizey, 0, "findcentersino");
}

float findcentersino_subpixel(float *frame0, float *frame180, float *dark, float *flat, int sizex, int sizey)
{
    return (float)centersino_entry<float>(frame0, frame180, dark, flat, sizex, sizey, 1, "findcentersino_subpixel");
}

int findcentersino16(uint16_t *frame0, uint16_t *frame180, uint16_t *dark, uint16_t *flat, int sizex, int sizey)
{
    return (int)centersino_entry<uint16_t>(frame0, frame180, dark, flat, sizex, sizey, 0, "findcentersino16");
}

// Device-resident frames on `gpu`; *result receives the integer (subpixel = 0)
// or sub-pixel (1) offset.  Returns 0 on success.
int raft_centersino_device(int gpu, const float *d_frame0, const float *d_frame180, const float *d_dark,
                           const float *d_flat, int sizex, int sizey, int subpixel, double *result, void *stream)
{
    clear_error();
    if (!result || !centersino_shape_ok(sizex, sizey)) {
        set_error("raft_centersino_device: null result or unsupported frame size");
        return 1;
    }
    if (!ptrs_ok(1, {d_frame0, d_frame180, d_dark, d_flat}, "raft_centersino_device")) return 1;
    if (!check_gpus(&gpu, 1)) return 1;
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        cudaStream_t st = resolve_stream(ds, stream, ds.s_comp);
        void *ws = ds.img[0].get(centersino_workspace_bytes(sizex, sizey));
        *result = centersino_device<float>(gpu, d_frame0, d_frame180, d_dark, d_flat, sizex, sizey, subpixel ? 1 : 0,
                                           ws, st);
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

void getRotAxisCorrectionMultiGPU(int *gpus, int ngpus, float *tomogram, float axis_offset, int nrays, int nangles,
                                  int nslices, int blocksize)
{
    clear_error();
    if (nrays < 2 || nangles < 1 || nslices < 0) {
        set_error("getRotAxisCorrectionMultiGPU: invalid sizes");
        return;
    }
    if (!check_gpus(gpus, ngpus)) return;
    if (!tomogram) {
        set_error("null data pointer");
        return;
    }
    const size_t ps = (size_t)nangles * nrays;
    split_slabs(gpus, ngpus, nslices, [&](int dev, int start, int n) {
        rotaxis_host_slab(dev, tomogram + ps * start, axis_offset, nrays, nangles, n, blocksize);
    });
}

void correctRotationAxis(float *tomoin, float *tomoout, int sizex, int sizey, int sizez, int deviation)
{
    clear_error();
    if (!tomoin || !tomoout || sizex < 0 || sizey < 0 || sizez < 0) {
        set_error("correctRotationAxis: null pointer or negative size");
        return;
    }
    const int offset = deviation < 0 ? -deviation : deviation;
    for (size_t z = 0; z < (size_t)sizez; ++z)
        for (size_t y = 0; y < (size_t)sizey; ++y) {
            const float *in = tomoin + (z * sizey + y) * sizex;
            float *out = tomoout + (z * sizey + y) * sizex;
            if (deviation > 0) {            // shift right, zero fill (in place allowed)
                for (int x = sizex - 1; x >= offset; --x) out[x] = in[x - offset];
                for (int x = std::min(offset, sizex) - 1; x >= 0; --x) out[x] = 0.0f;
            } else if (deviation < 0) {     // shift left
                for (int x = 0; x < sizex - offset; ++x) out[x] = in[x + offset];
                for (int x = std::max(sizex - offset, 0); x < sizex; ++x) out[x] = 0.0f;
            }
        }
}

// --- BST ------------------------------------------------------------------
// Reference: getBSTMultiGPU, cuda/src/geometries/parallel/reconstruction_methods/bst.cu:674-734
// (packing as getFBPMultiGPU; the object is N x N; angles are taken as uniform
// over [0, pi) as the reference's regridding assumes, so `angles` is unused;
// nstreams only chose the reference's stream count).
static bool parse_bst(const float *paramf, const int *parami, FbpConfig &cfg)
{
    if (!parse_fbp_arrays(paramf, parami, cfg, true)) return false;
    if (cfg.objsize != cfg.nrays) {
        set_error("BST: the object size must equal nrays");
        return false;
    }
    BstPlanShape sh;
    if (!bst_plan_shape(sh, cfg.nrays, cfg.nangles, cfg.pad)) {
        set_error("BST: the padded length N*(1+pad) is too long for the shared-memory transforms (at most 14528 with prime factors 2, 3, 5, 7; about 7000 otherwise)");
        return false;
    }
    return true;
}

void getBSTMultiGPU(int *gpus, int ngpus, float *obj, float *tomogram, float *angles, float *paramf, int *parami,
                    int nstreams)
{
    (void)angles;
    (void)nstreams;
    clear_error();
    FbpConfig cfg;
    if (!parse_bst(paramf, parami, cfg)) return;
    if (!check_gpus(gpus, ngpus)) return;
    if (!obj || !tomogram) {
        set_error("null data pointer");
        return;
    }
    const size_t tps = (size_t)cfg.nangles * cfg.nrays, ops = (size_t)cfg.nrays * cfg.nrays;
    split_slabs(gpus, ngpus, cfg.nslices, [&](int dev, int start, int n) {
        bst_host_slab(cfg, dev, obj + ops * start, tomogram + tps * start, n);
    });
}

// Device-resident BST on one GPU (d_obj [nslices][N][N], d_tomogram [nslices][A][N]).
int raft_bst_device(int gpu, float *d_obj, const float *d_tomogram, const float *paramf, const int *parami,
                    void *stream)
{
    clear_error();
    FbpConfig cfg;
    if (!parse_bst(paramf, parami, cfg)) return 1;
    if (!ptrs_ok(cfg.nslices, {d_obj, d_tomogram}, "raft_bst_device")) return 1;
    if (!check_gpus(&gpu, 1)) return 1;
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        cudaStream_t st = resolve_stream(ds, stream, ds.s_comp);
        bst_device(cfg, gpu, d_obj, d_tomogram, cfg.nslices, st);
        if (!stream) RAFT_CUDA(cudaStreamSynchronize(st));
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

// --- tEMFQ -------------------------------------------------------------------
// Reference: get_tEM_FQ_MultiGPU, cuda/src/geometries/parallel/reconstruction_methods/em_frequency.cu:333-398
// (argument order count, obj, angles, flat as there); parami = [nrays, nangles,
// nslices, objsize, zpad, 0, 0, nflats, iterations, interpolation (0 nearest,
// 1 bilinear), blocksize], paramf = [detector pixel x, y, tv] (setEMFQParameters,
// parameters.cu:72-114; the total-variation weight is not used there either).
static bool parse_temfq(const float *paramf, const int *parami, TemfqConfig &c)
{
    if (!paramf || !parami) {
        set_error("null parameter array");
        return false;
    }
    c.nrays = parami[0];
    c.nangles = parami[1];
    c.nslices = parami[2];
    c.zpad = parami[4];
    c.niter = parami[8];
    c.interpolation = parami[9];
    c.blocksize = parami[10];
    c.dx = paramf[0];
    if (parami[3] != c.nrays) {
        set_error("tEMFQ: the object size must equal nrays");
        return false;
    }
    if (c.nslices < 0 || c.niter < 0 || (c.interpolation != 0 && c.interpolation != 1) ||
        !temfq_shape_ok(c.nrays, c.nangles, c.zpad)) {
        set_error("tEMFQ: unsupported sizes (N even; the N(1+zpad)- and N(1+zpad)/2-point transforms must fit "
                  "shared memory: N(1+zpad) <= 14528 with prime factors 2, 3, 5, 7, about 7000 otherwise), or "
                  "iterations < 0, or interpolation not 0/1");
        return false;
    }
    return true;
}

void get_tEM_FQ_MultiGPU(int *gpus, int ngpus, float *count, float *obj, float *angles, float *flat, float *paramf,
                         int *parami)
{
    clear_error();
    TemfqConfig cfg;
    if (!parse_temfq(paramf, parami, cfg)) return;
    if (!check_gpus(gpus, ngpus)) return;
    if (!count || !obj || !angles || !flat) {
        set_error("null data pointer");
        return;
    }
    const size_t cps = (size_t)cfg.nangles * cfg.nrays, ops = (size_t)cfg.nrays * cfg.nrays;
    split_slabs(gpus, ngpus, cfg.nslices, [&](int dev, int start, int n) {
        temfq_host_slab(cfg, dev, obj + ops * start, count + cps * start, flat + (size_t)cfg.nrays * start, angles, n);
    });
}

// Device-resident tEMFQ on one GPU: d_obj [nslices][N][N] in/out, d_counts
// [nslices][A][N] (not modified), d_flat [nslices][N], angles host.
int raft_temfq_device(int gpu, float *d_obj, const float *d_counts, const float *d_flat, const float *angles,
                      const float *paramf, const int *parami, void *stream)
{
    clear_error();
    TemfqConfig cfg;
    if (!parse_temfq(paramf, parami, cfg)) return 1;
    if (!ptrs_ok(cfg.nslices, {d_obj, d_counts, d_flat, angles}, "raft_temfq_device")) return 1;
    if (!check_gpus(&gpu, 1)) return 1;
    try {
        DeviceState &ds = device_state(gpu);
        std::lock_guard<std::mutex> lk(ds.mtx);
        RAFT_CUDA(cudaSetDevice(gpu));
        ds.ensure();
        cudaStream_t st = resolve_stream(ds, stream, ds.s_comp);
        const int A = cfg.nangles;
        float *d_ang = (float *)ds.angles.get(sizeof(float) * A);
        char *tb = (char *)ds.tabs.get(sizeof(float) * 3 * A + 64);
        float *cs = (float *)tb, *sn = cs + A, *wt = sn + A;
        RAFT_CUDA(cudaMemcpyAsync(d_ang, angles, sizeof(float) * A, cudaMemcpyHostToDevice, st));
        launch_angle_tables(d_ang, A, cs, sn, wt, 0, st);
        void *ws = ds.rows.get(temfq_workspace_bytes(cfg.nrays, A, cfg.zpad, std::max(1, cfg.nslices)));
        temfq_run(gpu, cfg, d_obj, d_counts, d_flat, cs, sn, cfg.nslices, ws, st);
        if (!stream) RAFT_CUDA(cudaStreamSynchronize(st));
    } catch (const CudaFail &) {
    }
    return has_error() ? 1 : 0;
}

}  // extern "C"
