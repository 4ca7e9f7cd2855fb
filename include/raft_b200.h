/*
 * raft_b200.h -- C ABI of libraft.so (ssc-raft_b200/sscRaft/lib/libraft.so),
 * the B200 build of the ssc-raft parallel-beam reconstruction hot path.
 *
 * The first five functions are drop-in replacements: same names, argument
 * lists, packed-parameter meaning and (void) return as the reference
 * cnpem/ssc-raft library, so the reference's ctypes layer binds them
 * unchanged.  All data pointers are HOST pointers to C-contiguous float32
 * arrays (sinogram [slices][angles][rays], image [slices][N][N]); the
 * library allocates, copies and frees device memory itself (device
 * workspaces and pinned staging buffers are cached between calls).
 *
 * Error behaviour: the reference calls exit(-1) on any CUDA error
 * (cuda/inc/common/logerror.hpp:59-67) and assert()s on a bad device id.
 * Here no call exits the process; every failure is recorded in a
 * thread-local status read with raft_last_error().  The Python layer
 * (sscRaft) raises RuntimeError when it is set.
 *
 * Packed parameters (as built by sscRaft/geometries/parallel/fbp_methods.py:86-95
 * and em_methods.py:136-145 of the reference):
 *   FBP / lowpass  parami = {nrays, nangles, nslices, objsize, pad, 0, 0, filter, 0, blocksize}
 *                  paramf = {1/(beta/delta) or 0, regularization, energy_eV, z2_m,
 *                            pixel_x, pixel_y, rotation_axis_offset}
 *   EM             parami = {nrays, nangles, nslices, objsize(=nrays), 0, 0, 0, nflats,
 *                            iterations, blocksize}
 *   filter ids     0 none, 1 gaussian, 2 lorentz, 3 cosine, 4 rectangle, 5 hann,
 *                  6 hamming, 7 ramp, 8 differential, 9 shepp-logan (new)
 */
#ifndef RAFT_B200_H
#define RAFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* FBP (filter + nearest-sample backprojection, bit-faithful index rule).
 * Replaces getFBPMultiGPU, cuda/src/geometries/parallel/reconstruction_methods/fbp.cu:238-302
 * (ctypes prototype sscRaft/rafttypes.py:175-186).  obj [nslices][objsize][objsize] written. */
void getFBPMultiGPU(int *gpus, int ngpus, float *obj, float *tomogram, float *angles,
                    float *paramf, int *parami);

/* Filter only, in place on tomogram [nslices][nangles][nrays], axis offset 0.
 * Replaces getFilterLowPassMultiGPU, cuda/src/processing/filters/low_pass.cu:84-141
 * (rafttypes.py:188-198). */
void getFilterLowPassMultiGPU(int *gpus, int ngpus, float *tomogram, float *paramf, int *parami);

/* Ray-tracing Radon transform, tomogram_out [nslices][nangles][nrays] written.
 * Replaces getRadonRTMultiGPU, cuda/src/geometries/parallel/forward_methods/radon_rt.cu:252-295
 * (rafttypes.py:311-323). */
void getRadonRTMultiGPU(int *gpus, int ngpus, float *tomogram_out, float *phantom, float *angles,
                        int sizex, int sizey, int nrays, int nangles, int nslices, float ax, float ay);

/* Transmission EM; obj is the initial guess and the result; count = exp(-data)
 * (computed by the Python wrapper), flat [nslices][nrays] (the flat of each slice).
 * Replaces get_tEM_RT_MultiGPU, cuda/src/geometries/parallel/reconstruction_methods/em_rt.cu:12-84
 * (rafttypes.py:126-136). */
void get_tEM_RT_MultiGPU(int *gpus, int ngpus, float *obj, float *count, float *flat, float *angles,
                         float *paramf, int *parami);

/* Emission EM; obj is the initial guess and the result.
 * Replaces get_eEM_RT_MultiGPU, em_rt.cu:201-262 (rafttypes.py:138-147). */
void get_eEM_RT_MultiGPU(int *gpus, int ngpus, float *obj, float *tomogram, float *angles,
                         float *paramf, int *parami);

/* Rotation-axis offset from the 0 and 180 degree frames [sizey][sizex] (host arrays) by
 * phase correlation, the reference's integer / sub-pixel searches (their candidate sets kept
 * as they are), on the calling thread's current device.  Frame sides up to 14528 with prime
 * factors 2, 3, 5, 7, about 7000 otherwise.  Errors via raft_last_error (result 0).
 * Replace findcentersino / findcentersino_subpixel / findcentersino16,
 * cuda/src/processing/rotation_axis.cu:429-451 (rafttypes.py:201-219). */
int findcentersino(float *frame0, float *frame180, float *dark, float *flat, int sizex, int sizey);
float findcentersino_subpixel(float *frame0, float *frame180, float *dark, float *flat, int sizex, int sizey);
int findcentersino16(uint16_t *frame0, uint16_t *frame180, uint16_t *dark, uint16_t *flat, int sizex,
                     int sizey);

/* findcentersino(_subpixel) on device frames of one GPU; *result gets the offset.
 * NULL stream as raft_fbp_device.  Returns 0 on success. */
int raft_centersino_device(int gpu, const float *d_frame0, const float *d_frame180, const float *d_dark,
                           const float *d_flat, int sizex, int sizey, int subpixel, double *result, void *stream);

/* Sub-pixel rotation-axis correction in place: every row edge-padded to 3 nrays, shifted by
 * axis_offset samples with a Fourier phase ramp, cropped back.
 * Replaces getRotAxisCorrectionMultiGPU, cuda/src/processing/rotation_axis.cu:591-643
 * (rafttypes.py:233-241). */
void getRotAxisCorrectionMultiGPU(int *gpus, int ngpus, float *tomogram, float axis_offset, int nrays,
                                  int nangles, int nslices, int blocksize);

/* Integer shift of every row by `deviation` samples (right if positive) with zero fill,
 * on the host; tomoout may equal tomoin.  Replaces correctRotationAxis,
 * cuda/src/processing/rotation_axis.cu:396-426 (whose ctypes binding in rafttypes.py:222-231
 * declares one pointer too few; this library binds both). */
void correctRotationAxis(float *tomoin, float *tomoout, int sizex, int sizey, int sizez, int deviation);

/* FBP by the backprojection slice theorem (Fourier regridding), packing as getFBPMultiGPU
 * (object N x N).  Angles are taken as uniform over [0, pi), as the reference's regridding
 * assumes (the Python wrapper passes linspace(0, pi, A)); `angles` and `nstreams` are unused.
 * Requires N*(1+pad) <= 14528 with prime factors 2, 3, 5, 7 only, or about 7000 with larger
 * prime factors (transformed by Bluestein's algorithm).
 * Replaces getBSTMultiGPU, cuda/src/geometries/parallel/reconstruction_methods/bst.cu:674-734
 * (rafttypes.py:161-173). */
void getBSTMultiGPU(int *gpus, int ngpus, float *obj, float *tomogram, float *angles, float *paramf,
                    int *parami, int nstreams);

/* getBSTMultiGPU on device-resident buffers of one GPU; NULL stream as raft_fbp_device.
 * Returns 0 on success. */
int raft_bst_device(int gpu, float *d_obj, const float *d_tomogram, const float *paramf, const int *parami,
                    void *stream);

/* Transmission EM with the Fourier-slice projector and the BST back-projector (tEMFQ).
 * count [nslices][nangles][nrays] photon counts (read only), obj [nslices][N][N] initial
 * guess in / result out, angles uniform over [0, pi), flat [nslices][nrays];
 * parami = [nrays, nangles, nslices, objsize (= nrays), zpad, 0, 0, nflats, iterations,
 * interpolation (0 nearest, 1 bilinear), blocksize], paramf = [detector pixel x, y, tv (unused,
 * as in the reference)].  N even; N(1+zpad) up to 14528 with prime factors 2, 3, 5, 7, about
 * 7000 otherwise.
 * Replaces get_tEM_FQ_MultiGPU, cuda/src/geometries/parallel/reconstruction_methods/
 * em_frequency.cu:333-398 (rafttypes.py:149-159). */
void get_tEM_FQ_MultiGPU(int *gpus, int ngpus, float *count, float *obj, float *angles, float *flat,
                         float *paramf, int *parami);

/* get_tEM_FQ_MultiGPU on device-resident buffers of one GPU (angles host; d_counts is not
 * modified).  NULL stream as raft_fbp_device.  Returns 0 on success. */
int raft_temfq_device(int gpu, float *d_obj, const float *d_counts, const float *d_flat, const float *angles,
                      const float *paramf, const int *parami, void *stream);

/* Status of the last call on this thread: returns 0 if it succeeded, 1 and
 * the message (truncated to len-1 chars) otherwise.  Replaces the reference's
 * exit(-1) (cuda/inc/common/logerror.hpp:59-67). */
int raft_last_error(char *buf, int len);
void raft_clear_error(void);
int raft_abi_version(void);

/* Failure injection: the next n device-buffer requests of the library fail as
 * an out-of-memory would (the call reports the error; the library stays
 * usable); n = 0 clears it. */
void raft_inject_alloc_failures(int n);
/* Self test of the bounded device-side wait of the staging pipelines: 1 if a
 * wait on a barrier nothing arrives on (arrive = 0) ran out after `limit` polls
 * and was reported, 0 if it completed (arrive = 1), -1 on error. */
int raft_selftest_bounded_wait(int gpu, int arrive, unsigned limit);

/* FBP with a selectable operator and sinogram storage (host buffers).
 * geometry 0 = reference nearest-sample rule (store must be 0),
 * geometry 1 = linear interpolation with true ramp-family filters
 *              (store 1 = FP32 pairs, 2 = BF16 pairs; accumulation is FP32).
 * Extends getFBPMultiGPU (fbp.cu:238-302); returns 0 on success. */
int raft_fbp_ext(int *gpus, int ngpus, float *obj, const float *tomogram, const float *angles,
                 const float *paramf, const int *parami, int geometry, int store);

/* Flat/dark correction of frames [nslices][nangles][nrays] in place:
 * T = max(D - dark, 0.5) / max(flat - dark, 0.5), then T = -log(T) when is_log = 1;
 * flat [nslices][numflats][nrays] (with two or more flats the first two are
 * interpolated by angle index / nangles), dark [nslices][nrays].
 * Reference: getBackgroundCorrectionMultiGPU, cuda/src/processing/background_correction.cu:144-178
 * (kernel :15-47, -log opt.cu:196-214).  Errors via raft_last_error. */
void getBackgroundCorrectionMultiGPU(int *gpus, int ngpus, float *frames, float *flat, float *dark,
                                     int nrays, int nangles, int nslices, int numflats, int is_log,
                                     int blocksize);

/* getBackgroundCorrectionMultiGPU on device-resident buffers of one GPU (in place on
 * d_frames), NULL stream as raft_fbp_device.  Returns 0 on success. */
int raft_background_device(int gpu, float *d_frames, const float *d_flat, const float *d_dark, int nrays,
                           int nangles, int nslices, int numflats, int is_log, void *stream);

/* Streams of the device-pointer entry points below: work is issued on `stream`; NULL
 * means "ordered after everything already queued on the legacy default stream" (the
 * stream PyTorch uses by default): the library then runs on its own stream, made to
 * wait for that work, and synchronises it before returning.
 *
 * FBP on device-resident buffers of one GPU (d_obj, d_tomogram on `gpu`;
 * angles host), issued on `stream` (NULL: see above).
 * Same operator as raft_fbp_ext; getFBPGPU-level entry (fbp.cu:127-236). */
int raft_fbp_device(int gpu, float *d_obj, const float *d_tomogram, const float *angles,
                    const float *paramf, const int *parami, int geometry, int store, void *stream);

/* raft_fbp_device without any device-memory allocation (no counterpart in the reference).
 * For callers that cannot allocate GPU memory while reconstructing -- e.g. acquisition
 * pipelines that reserve the device memory when a scan starts so reconstruction can never
 * run out of memory mid-scan, or hosts whose own allocator owns the device memory.
 * Working memory comes from one fixed 64 MiB device array inside the library, held by
 * every GPU that loads it until exit; the first call on a device looks up that array's
 * address (make it before any stream capture).  Calls share the array: calls whose work
 * overlaps on one GPU (other host threads, other streams) race.  Runs the planar
 * backprojector, so large volumes take longer than through raft_fbp_device.  Limits: N*(1+pad) <= 14080 with prime factors 2,3,5,7,
 * nangles <= 32768, one slice's filtered rows + tables within 64 MiB; larger requests
 * return 1 with a message.  Synchronises `stream` before returning. */
int raft_fbp_device_noalloc(int gpu, float *d_obj, const float *d_tomogram, const float *angles,
                            const float *paramf, const int *parami, int geometry, int store,
                            void *stream);

/* One request of a ragged batch (no reference counterpart; the reference handles one
 * size per call).  All sizes may differ between requests. */
typedef struct raft_request {
    int kind;            /* 0 = FBP (getFBPMultiGPU operator), 1 = emission EM (get_eEM_RT_MultiGPU) */
    int nrays;           /* detector bins = image side N */
    int nangles;
    int pad;             /* FBP: padding factor (reference dic 'padding') */
    int filter;          /* FBP: filter id */
    int niter;           /* eEM: iterations (equal for all eEM requests of a batch) */
    float pixel;         /* FBP: detector pixel size */
    float offset;        /* FBP: rotation-axis offset */
    const float *angles; /* host, nangles radians */
    const float *d_data; /* device: sinogram [nangles][nrays] (FBP) or emission tomogram (eEM) */
    float *d_out;        /* device: FBP image [nrays][nrays]; eEM object, initial guess in / result out */
} raft_request;

/* Ragged batch on one GPU: FBP requests' backprojection runs as one persistent launch over
 * all requests' tiles (shortest request first), eEM requests' iterations as one ragged
 * projector + one persistent backprojector launch per iteration, replayed from a CUDA
 * graph; FBP and EM proceed on two streams.  geometry/store select the FBP operator as in
 * raft_fbp_ext.  latency_ms[i] (may be NULL) receives request i's completion time and
 * *total_ms the whole batch's, both measured on the device from the batch start.
 * NULL stream as raft_fbp_device.  Returns 0 on success. */
int raft_ragged_device(int gpu, const raft_request *reqs, int nreq, int geometry, int store,
                       double *latency_ms, double *total_ms, void *stream);

/* EM (kind 0 = tEM as get_tEM_RT_MultiGPU, 1 = eEM as get_eEM_RT_MultiGPU) on one GPU with
 * host buffers, the iteration loop replayed as one CUDA graph when use_graph != 0, and
 * per-iteration FP64 metrics [niter][nslices][3] = {sum (model-data)^2, sum data^2,
 * negative log-likelihood} of the iterate entering that iteration (metrics may be NULL).
 * The reference computes no residual (em_rt.cu:154-192,316-355). Returns 0 on success. */
int raft_em_ext(int kind, int gpu, float *obj, const float *data, const float *flat,
                const float *angles, int nrays, int nangles, int nslices, int niter,
                double *metrics, int use_graph);

/* getRadonRTMultiGPU's operator on device-resident buffers of one GPU (angles host),
 * issued on `stream` (NULL: after the legacy default stream's queued work, synchronised).  Returns 0 on success. */
int raft_radon_device(int gpu, float *d_out, const float *d_phantom, const float *angles, int nx, int ny,
                      int nrays, int nangles, int nslices, float ax, float ay, void *stream);

/* As raft_em_ext on device-resident buffers (metrics device pointer or NULL); NULL
 * stream as raft_fbp_device.  Synchronises before returning. */
int raft_em_device(int kind, int gpu, float *d_obj, const float *d_data, const float *d_flat,
                   const float *angles, int nrays, int nangles, int nslices, int niter,
                   double *d_metrics, int use_graph, void *stream);

/* Host-only: slab of slices each of ngpus devices gets in the *MultiGPU calls --
 * contiguous blocks of ceil(nslices/ngpus), as the reference's split
 * (fbp.cu:267-301, em_rt.cu:43-81).  Returns 0 on success. */
int raft_slab_partition(int nslices, int ngpus, int *start, int *count);

/* Host-only helper (no GPU needed, no reference counterpart): the detector-window
 * layout the backprojector stages for a configuration; out = {wlo, Wg, W, align}.
 * geometry 0/1 with FBP packing, 2 with EM packing.  Returns 0 on success. */
int raft_plan_window(const float *paramf, const int *parami, int geometry, int store, int *out);

/* sin/cos of angles[0..n) computed on `gpu` with the fast intrinsics the reference
 * uses: kind 0 = __sinf/__cosf (setSinCosTable, cuda/src/common/opt.cu:187-194),
 * kind 1 = __sincosf (kernel_backprojection, em_RT_kernel.cu:120).  Returns 0 on success. */
int raft_fast_sincos(int gpu, const float *angles, int n, int kind, float *cos_out, float *sin_out);

/* Instrumentation (no reference counterpart): total kernel launches issued by
 * this library in the process; optional CUDA-event timing of the filter (class 0),
 * backprojector (1) and projector (2) launches, summed since the last read. */
long long raft_launch_count(void);
/* JSON list of the backprojector launch shapes (slices per CTA, angles per stage) the
 * autotuner chose so far in this process; returns the string length. */
int raft_autotune_table(char *buf, int len);
void raft_profile_enable(int on);
int raft_profile_read(double *ms, long long *counts, int nclasses);
/* Transform kernel selection (no reference counterpart): 1 (default) = FBP filter
 * rows, BST and tEMFQ transforms of 1024, 1536, 2048, 3072, 4096, 6144, 8192 and
 * 12288 points run kernels compiled for that length (bit for bit the results of
 * the generic kernels); 0 = the generic kernels for all lengths. */
int raft_filter_set_fixed(int on);

/* Learned warm start: tensor-core kernels of the U-Net (no reference counterpart).
 * Device pointers; BF16 NHWC activations (channel counts multiples of 32), BF16 weights
 * [Cout][3][3][Cin], FP32 biases / gradients / master weights.  Return 0 on success. */
int raft_unet_conv_fwd(const void *x0, int C0, const void *x1, int C1, const void *w, const float *bias,
                       void *y, void *y1, int Cy0, int N, int H, int W, int Cout, int relu, void *stream);
/* Convolution kernel choice: 0 = tcgen05/TMA kernel where its 128-pixel tile fits (W >= 128
 * or W dividing 128), mma.sync kernel otherwise (default); 1 = mma.sync kernel only;
 * 2 = tcgen05 kernel only (other shapes fail). */
int raft_unet_set_conv_path(int path);
/* tcgen05 convolution of the 32 -> 32 channel layers (W >= 128): 1 = halo tiles (one input
 * box per 32-channel chunk serves all nine taps; default), 0 = one input box per tap. */
int raft_unet_set_conv_halo(int on);
/* tcgen05 weight gradient (W a multiple of 64; Cout 32, 64, 128 or 256; other shapes and
 * raft_unet_set_conv_path(1) use the mma.sync kernel): 1 = for Cout <= 128 one CTA per
 * 32-channel input chunk with all nine taps, the input staged once per 64-pixel k-block
 * (default); 0 = 128-row blocks of (tap, channel) for every layer. */
int raft_unet_set_wgrad_nine(int on);
/* 1 if a bounded pipeline wait of the tcgen05 convolution ran out since the last call
 * (the flag is then cleared); synchronises the current device. */
int raft_unet_conv_error(void);
int raft_unet_conv_wgrad(const void *dy, const void *x0, int C0, const void *x1, int C1, float *dw,
                         float *dbias, int N, int H, int W, int Cout, void *stream);
int raft_unet_flip_weights(const void *w, void *wt, int Cout, int Cin, void *stream);
int raft_unet_relu_bwd(const void *y, const void *dy, void *dpre, size_t n, void *stream);
int raft_unet_pool(int backward, const void *src, void *dst, int N, int H, int W, int C, void *stream);
int raft_unet_upsample(int backward, const void *src, void *dst, int N, int H, int W, int C, void *stream);
int raft_unet_input(const float *img, const float *scale, void *x, int N, int H, int W, int C, void *stream);
/* First layer for inference, from the one-channel input: y = ReLU(bias + 3x3 conv of
 * bf16(img x scale)) with the layer's weights [32][3][3][Cin] (channel 0 of each tap;
 * the packed input's other channels are zero), 32 BF16 output channels, NHWC. */
int raft_unet_input_conv(const float *img, const float *scale, const void *w, int Cin, const float *bias, void *y,
                         int N, int H, int W, void *stream);
/* First layer's gradients in training, from the one-channel input: dw[co][tap][0]
 * (dw is [32][3][3][Cin]; the other channels are left as they are) and db[co] from
 * dpre [N][H][W][32] BF16 (the ReLU-masked output gradient); work holds N*H*320
 * floats of per-row partial sums, reduced in a fixed order. */
int raft_unet_input_wgrad(const float *img, const float *scale, const void *dpre, float *dw, int Cin, float *db,
                          float *work, size_t work_floats, int N, int H, int W, void *stream);
int raft_unet_head(int backward, const void *h, const float *w, const float *b, const float *img,
                   const float *scale, float *out_or_grad, void *dh, float *dw, float *db, int N, int HW,
                   int C, void *stream);
int raft_unet_mse(const float *out, const float *target, const float *scale, float *grad, double *loss,
                  int N, int HW, void *stream);
int raft_unet_adam(float *w, float *m, float *v, const float *g, void *wb, size_t n, float lr, float b1,
                   float b2, float eps, int step, void *stream);
int raft_unet_add(void *y, const void *x, size_t n, void *stream);
int raft_unet_to_bf16(const float *a, void *b, size_t n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RAFT_B200_H */
