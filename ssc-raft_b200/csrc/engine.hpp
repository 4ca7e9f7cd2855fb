// engine.hpp -- per-device execution engine: cached device workspaces,
// pinned staging, filter plans, and the chunked FBP / EM / Radon / lowpass
// pipelines behind the C-ABI.
#pragma once
#include "raft.hpp"

#include <mutex>
#include <vector>

namespace raft {

// Grow-only device buffer owned by a per-device workspace.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *get(size_t need);      // (re)allocates when too small; contents undefined
    void release();
};

struct PinBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *get(size_t need);
    void release();
};

// Everything one device keeps between calls.  Calls on the same device are
// serialised by `mtx` (the reference is not re-entrant per device either).
struct DeviceState {
    int device = 0;
    std::mutex mtx;
    cudaStream_t s_comp = nullptr, s_h2d = nullptr, s_d2h = nullptr;
    cudaStream_t s_hi = nullptr, s_lo = nullptr;   // ragged batches: FBP (high) and EM (low) priority
    DevBuf sino[2], img[2], rows, den, flat, data, angles, tabs, metrics, err, imgT, il;
    PinBuf pin_in[2], pin_out[2];
    cudaEvent_t ev_h2d[2] = {}, ev_comp[2] = {}, ev_d2h[2] = {};
    cudaEvent_t ev_join = nullptr;
    bool init = false;
    void ensure();
};

DeviceState &device_state(int device);

// The stream a device-pointer entry point runs on.  A caller stream is used
// as given.  NULL means the legacy default stream (PyTorch's default stream
// is that stream); the library does not run on it (a CUDA graph cannot be
// captured there) but on its own non-blocking stream `own`, which does not
// order itself after the legacy stream by itself -- so `own` is first made to
// wait for everything already queued there (the caller's copy that produced
// an input, say).  Entry points synchronise `own` before returning.
cudaStream_t resolve_stream(DeviceState &ds, void *stream, cudaStream_t own);

// Filter plan cache (per device, keyed by every spectrum input).
const FilterPlan &cached_filter_plan(int device, int geometry, int ftype, int N, int pad, double paganin,
                                     double reg, double offset, double pixel);

// Host memcpy with a few threads (staging to / from pinned buffers).
void parallel_memcpy(void *dst, const void *src, size_t bytes);

// --- FBP ---------------------------------------------------------------
struct FbpPrepared {
    FbpConfig cfg;
    int No = 0, Np = 0, Npo = 0;
    WindowLayout win;
    BpGeo geo;
    const FilterPlan *plan = nullptr;
};

FbpPrepared prepare_fbp(const FbpConfig &cfg, int device);

// Device-resident FBP of `nslices` slices (filter + backprojection), using
// the device workspace for the window rows; tables must be set up by
// fbp_tables().  d_sino [nslices][A][N] -> d_img [nslices][No][No].
struct FbpTables {
    float *cs = nullptr, *sn = nullptr, *wt = nullptr;
    double *csd = nullptr, *snd = nullptr;
    int *err = nullptr;
};
FbpTables fbp_tables(DeviceState &ds, const FbpPrepared &fp, const float *h_angles, cudaStream_t st);
// d_il (optional, fbp_il_bytes): workspace for the slice-interleaved rows the
// backprojector reads with four slices per CTA (4-byte elements: nearest f32,
// bf16 pairs), written by the filter directly (d_rows may then be null);
// null keeps the planar rows.
void fbp_chunk(DeviceState &ds, const FbpPrepared &fp, const FbpTables &tb, const float *d_sino, float *d_img,
               int nslices, void *d_rows, cudaStream_t st, void *d_il = nullptr);
size_t fbp_rows_bytes(const FbpPrepared &fp, int nslices);
// True when fbp_chunk, given the interleave workspace, has the filter write
// interleaved rows directly (no plain rows needed).
bool fbp_fused_il(const FbpPrepared &fp);
size_t fbp_il_bytes(const FbpPrepared &fp, int nslices);

// Host-buffer FBP of one slab on one device (the body of getFBPMultiGPU).
void fbp_host_slab(const FbpConfig &cfg, int device, float *obj, const float *tomo, const float *angles,
                   int nslices);

// --- lowpass -------------------------------------------------------------
void bst_host_slab(const FbpConfig &cfg, int device, float *obj, const float *tomo, int nslices);
// Device-resident BST on st (caller holds the device lock).
void bst_device(const FbpConfig &cfg, int device, float *d_obj, const float *d_tomo, int nslices, cudaStream_t st);
void rotaxis_host_slab(int device, float *tomo, float axis_offset, int nrays, int nangles, int nslices,
                       int blocksize);
template <typename T>
double centersino_host(int device, const T *frame0, const T *frame1, const T *dark, const T *flat, int sizex,
                       int sizey, int subpixel);
void temfq_host_slab(const TemfqConfig &cfg, int device, float *obj, const float *counts, const float *flat,
                     const float *angles, int nslices);
void lowpass_host_slab(const FbpConfig &cfg, int device, float *tomo, int nslices);
void background_host_slab(int device, float *frames, const float *flat, const float *dark, int nrays, int nangles,
                          int nslices, int numflats, int is_log, int blocksize);

// --- Radon ---------------------------------------------------------------
void radon_host_slab(int device, float *proj, const float *img, const float *angles, int nx, int ny,
                     int nrays, int nangles, int nslices, float ax, float ay);

// --- EM ------------------------------------------------------------------
struct EmPrepared {
    EmConfig cfg;
    WindowLayout win;
    BpGeo geo;
};
EmPrepared prepare_em(const EmConfig &cfg);

// Device-resident EM of one chunk.  kind 0 = tEM (data = exp(-input) counts,
// flat [nslices][nrays]), 1 = eEM.  obj is in/out.  metrics (optional) is a
// device array [niter][nslices][3] of FP64 sums, filled per iteration.
// use_graph captures the iteration loop as one CUDA graph.
void em_chunk(DeviceState &ds, const EmPrepared &ep, int kind, const float *d_data, const float *d_flat,
              const float *h_angles, float *d_obj, int nslices, double *d_metrics, bool use_graph,
              cudaStream_t st);

void em_host_slab(const EmConfig &cfg, int kind, int device, float *obj, const float *data, const float *flat,
                  const float *angles, int nslices, bool flat_by_angle);

// Parameter parsing / device check shared with the no-allocation entry point.
bool parse_fbp_params(const float *paramf, const int *parami, FbpConfig &cfg);
bool check_gpu_id(int gpu);
bool filter_plan_shape(FilterPlan &plan, int ftype, int N, int pad);

}  // namespace raft
