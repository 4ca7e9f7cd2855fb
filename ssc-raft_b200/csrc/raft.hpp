// raft.hpp -- shared host/device definitions of the B200 parallel-beam
// reconstruction library (libraft.so).
//
// Layouts (all C-contiguous, as in ssc-raft):
//   sinogram  [slices][angles][rays]   float32
//   image     [slices][N][N]           float32
//   window rows [slices*angles][Wg]    the detector bins that one slice's
//             image can reach, with zero margins, each element already
//             multiplied by the angle step dtheta_a (and by the >pi angular
//             rescale), stored as float32 (nearest-sample operators), as
//             (mid, diff) float2 pairs or as (mid, diff) bf16x2 pairs
//             (linear interpolation: value(u) = mid + (u - k - 1/2) * diff).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstddef>
#include <string>

namespace raft {

// ----------------------------------------------------------------- status --
// The reference library calls exit(-1) on any CUDA error
// (cuda/inc/common/logerror.hpp:59-67).  Here every failure is recorded in a
// thread-local status that raft_last_error() returns; nothing exits.
void set_error(const std::string &msg);
bool has_error();
std::string get_error();
void clear_error();

struct CudaFail {};

#define RAFT_CUDA(call)                                                         \
    do {                                                                        \
        cudaError_t _e = (call);                                                \
        if (_e != cudaSuccess) {                                                \
            ::raft::set_error(std::string(#call) + ": " + cudaGetErrorString(_e) \
                              + " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
            throw ::raft::CudaFail();                                           \
        }                                                                       \
    } while (0)

#define RAFT_CHECK(cond, msg)                                                   \
    do {                                                                        \
        if (!(cond)) {                                                          \
            ::raft::set_error(std::string(msg));                                \
            throw ::raft::CudaFail();                                           \
        }                                                                       \
    } while (0)

// ----------------------------------------------------------------- enums --
enum Geometry : int {
    GEOM_FBP_REF = 0,   // fbp.cu:38-72: nearest sample by truncation, pixel units
    GEOM_FBP_LIN = 1,   // same grid, linear interpolation (north-star operator)
    GEOM_EM_REF  = 2,   // em_RT_kernel.cu:92-142: [-1,1] grid, truncation
};

enum Store : int {
    STORE_F32       = 0,  // one float per bin (nearest-sample operators)
    STORE_PAIR_F32  = 1,  // (mid, diff) float2 per bin (linear interpolation)
    STORE_PAIR_BF16 = 2,  // (mid, diff) bf16x2 per bin (linear interpolation)
};

inline int store_bytes(int store) { return store == STORE_PAIR_F32 ? 8 : 4; }

// Filter ids: the reference enum (cuda/inc/processing/filters.hpp:26-37)
// plus 9 = Shepp-Logan for the linear-interpolation mode.
enum FilterType : int {
    FILTER_NONE = 0, FILTER_GAUSSIAN = 1, FILTER_LORENTZ = 2, FILTER_COSINE = 3,
    FILTER_RECTANGLE = 4, FILTER_HANN = 5, FILTER_HAMMING = 6, FILTER_RAMP = 7,
    FILTER_DIFFERENTIAL = 8, FILTER_SHEPP_LOGAN = 9,
    // internal: weight 1 and normalisation 1/Np only -- the rotation-axis shift
    // of getRotAxisCorrection (rotation_axis.cu:455-526)
    FILTER_AXIS_SHIFT = 100,
};

// ----------------------------------------------------------- filter plan --
struct FilterPlan {
    int N = 0, Np = 0, pad = 0, off = 0;
    int fft = 0;                 // 1: mixed-radix FFT path, 0: direct circular convolution
    int cluster = 0;             // > 1: FFT by a cluster of this many CTAs (radix = of Np / cluster)
    int bs_M = 0;                // > 0: Bluestein transforms of this length (radix = of bs_M)
    const float2 *bs_chirp = nullptr, *bs_B = nullptr;   // Bluestein tables (cached per device and length)
    int nradix = 0;
    int radix[24] = {};
    int threads = 0;             // CTA size of the FFT kernel
    float2 *d_H = nullptr;       // full Hermitian-extended spectrum incl. 1/(Np*pixel)
    float2 *d_tw = nullptr;      // exp(-2 pi i m / Np)
    float *d_h = nullptr;        // impulse response (direct path)
    bool skip = false;           // reference 'none' filter: pad + copy only
};

bool build_filter_plan(FilterPlan &plan, int geometry, int ftype, int N, int pad, double paganin,
                       double reg, double offset, double pixel, int device);
void release_filter_plan(FilterPlan &plan);
// Filter::apply of the reference (filters.cu:395-438) at weight w, in FP64.
double filter_apply_ref(int type, double w, double paganin, double reg);
void filter_spectrum_host(int geometry, int ftype, int Np, double paganin, double reg,
                          double offset, double pixel, double *hre, double *him);

struct FilterLaunch {
    const float *sino = nullptr;   // [nrows][N]
    void *out = nullptr;           // [nrows][Wg] window rows, or [nrows][N] (lowpass)
    const float *wt = nullptr;     // per-angle weight, indexed row % nangles
    int nrows = 0, nangles = 1;
    int wlo = 0, Wg = 0;
    int store = STORE_F32;
    int out_padded = 0;            // lowpass: centre N bins, unweighted float
    int interleaved = 0;           // 1: window rows interleaved by slice in groups of four
                                   //    ([ceil(slices/4)][nangles][Wg][4], 4-byte elements, absent slices 0)
};

void launch_filter(const FilterPlan &plan, const FilterLaunch &fl, cudaStream_t st);

// ------------------------------------------------------- window layout --
// Which stored bins a backprojection needs, and how a CTA tile stages them.
struct WindowLayout {
    int wlo = 0;      // padded-bin index of stored element 0
    int Wg = 0;       // stored elements per row (multiple of the 16-byte granule)
    int W = 0;        // staged elements per angle per tile
    int align = 4;    // element alignment of a staged window start
};

// Launch-time tile configuration of the backprojector.
constexpr int BP_THREADS = 256;
constexpr int BP_TX = 64;     // tile width  (pixels)
constexpr int BP_TY = 32;     // tile height (pixels)
constexpr int BP_AB = 32;     // maximum angles per pipeline stage

// Geometry constants of one backprojection, in the reference's FP32
// arithmetic (FBP: fbp.cu:38-44; EM: em_RT_kernel.cu:97-102).
struct BpGeo {
    float xmin = 0, ymin = 0, dx = 1, dy = 1, tmin = 0, dt = 1;  // FBP; EM uses tmin=-1, dt=2/(n-1)
    int offo = 0;          // padded-grid index of output pixel 0 (FBP)
    float dxy = 0;         // EM pixel step 2/(N-1)
    double c0 = 0;         // linear geometry: pixel i sits at (i + c0)*pixel_x
    double ratio = 1;      // pixel_y / pixel_x
    double u0 = 0;         // Np/2 - wlo - 0.5
};

struct BpPlanInput {
    int geometry = GEOM_FBP_REF, store = STORE_F32, No = 0;
    float xmin = 0, ymin = 0, dx = 1, dy = 1, tmin = 0, dt = 1;
    int offo = 0;
    float dxy = 0;
};

WindowLayout plan_window(const BpPlanInput &in);

struct BpLaunch {
    const void *filt = nullptr;   // window rows [nslices*nangles][Wg]
    float *img = nullptr;         // [nslices][No][No]
    const float *den = nullptr;   // EM update denominator; nullptr = plain store
    int No = 0, nangles = 0, nslices = 0;
    int geometry = GEOM_FBP_REF, store = STORE_F32;
    WindowLayout win;
    BpGeo geo;
    const float *cs = nullptr, *sn = nullptr;     // FP32 angle tables
    const double *csd = nullptr, *snd = nullptr;  // FP64 angle tables
    int *err = nullptr;                           // device error flag
    // optional workspace of bp_il_bytes(): lets launches of four slices per
    // CTA read the rows interleaved by slice (made here from filt)
    void *il_ws = nullptr;
    // 1: il_ws already holds the rows interleaved by slice (filt unused);
    //    only four-slice shapes run
    int il_ready = 0;
};

void launch_backproject(const BpLaunch &bl, cudaStream_t st);
size_t bp_il_bytes(int nslices, int nangles, int Wg, int esize);
// True when RAFT_BP_TUNE forces a shape of fewer than four slices per CTA
// (which reads plain, not interleaved, rows).
bool bp_forced_planar();

// Backprojector launch shape chosen by the autotuner: S slices per CTA
// (sharing each pixel's position arithmetic) and AB angles per pipeline stage.
struct BpTune {
    int S, AB;
};
std::string bp_tune_table();   // JSON list of the tuned configurations

// Ragged batch of backprojections (different sizes, angle counts, windows) in
// one persistent launch; descriptors live on the device so the launch can be
// replayed inside a CUDA graph.
struct RaggedBp {
    int nreq = 0, total = 0, wmax = 0, geometry = 0, store = 0;
    void *d_args = nullptr;
    int *d_item_start = nullptr, *d_counts = nullptr, *d_remaining = nullptr, *d_queue = nullptr;
    unsigned long long *d_tdone = nullptr;   // per-request completion time (ns, %globaltimer)
};
size_t ragged_bp_bytes(int nreq);
void ragged_bp_prepare(RaggedBp &rb, const BpLaunch *reqs, int nreq, int geometry, int store, void *d_ws);
void ragged_bp_launch(const RaggedBp &rb, cudaStream_t st);
void launch_stamp(unsigned long long *d_t, cudaStream_t st);   // write %globaltimer

// sin/cos with the reference's fast intrinsics (__sinf/__cosf for FBP,
// opt.cu:187-194; __sincosf for EM, em_RT_kernel.cu:120) and the per-angle
// weight dtheta_a (times pi/theta_last beyond pi for FBP).
void launch_angle_tables(const float *d_angles, int nangles, float *d_cos, float *d_sin,
                         float *d_wt, int em_sincos, cudaStream_t st);

// ------------------------------------------------------------ projector --
struct ProjLaunch {
    const float *img = nullptr;     // [nslices][ny][nx]
    const float *imgT = nullptr;    // optional transposed copy [nslices][nx][ny] for steep angles
    const float *il = nullptr;      // optional slice-interleaved copies (groups of 8 planes):
    const float *ilT = nullptr;     //   il [G][ny][nx][8], ilT [G][nx][ny][8]; used instead of img/imgT
    const float *il_zero = nullptr; //   with 8 zero floats (32-byte aligned) that outside samples read
    float *out = nullptr;           // plain [nslices][nangles][nrays] or window rows
    const float *angles = nullptr;
    int nx = 0, ny = 0, nrays = 0, nangles = 0, nslices = 0;
    float ax = 1.f, ay = 1.f;
    int em = 0;                     // 1: kernel_radon geometry, 0: Radon_RT_version_sscRadon
    int epilogue = 0;               // 0 plain, 1 tEM flat*exp(-p), 2 eEM ratio
    const float *flat = nullptr;    // tEM: [nslices][nrays]
    const float *data = nullptr;    // tEM counts / eEM tomogram [nslices][nangles][nrays]
    const float *wt = nullptr;      // per-angle weight applied when writing window rows
    int windowed = 0, wlo = 0, Wg = 0;   // windowed: 1 rows [slice][angle][Wg], 2 [slice/4][angle][Wg][4]
    double *metrics = nullptr;      // optional FP64 sums [nslices][3]
};

void launch_project(const ProjLaunch &pl, cudaStream_t st);

// Ragged projector over single-slice requests: block b runs request r with
// blk_start[r] <= b < blk_start[r+1] (device arrays).
void launch_project_ragged(const ProjLaunch *d_reqs, const int *d_blk_start, int nreq, int total_blocks, int em,
                           int epilogue, cudaStream_t st);
// Blocks the ragged projector runs for one single-slice request.
int project_blocks_per_slice(int nrays, int nangles);

// out[k][x][y] = in[k][y][x] for each of nslices planes.
void launch_transpose(const float *in, float *out, int nx, int ny, int nslices, cudaStream_t st);

// Scratch bytes the projector's re-laid-out images need for nslices planes.
size_t proj_scratch_bytes(int nx, int ny, int nslices);
// Write the re-laid-out copies of pl.img into `scratch` (proj_scratch_bytes):
// slice-interleaved groups of 8 (pl.il / pl.ilT) when there are 8 or more
// planes, else a transposed copy (pl.imgT).  Issued on st.
void stage_proj_images(ProjLaunch &pl, void *scratch, cudaStream_t st);

// Flat/dark correction (and -log when is_log) of frames [nslices][nangles][nrays]
// from flat [nslices][numflats][nrays] and dark [nslices][nrays]; out may equal in.
void launch_background(const float *in, float *out, const float *flat, const float *dark, int nrays, int nangles,
                       int nslices, int numflats, int is_log, cudaStream_t st);

// Copy a plain sinogram into weighted window rows (EM: BP of the counts).
void launch_to_window(const float *sino, float *rows, const float *wt, int nrows, int nangles,
                      int nrays, int wlo, int Wg, cudaStream_t st);

// ----------------------------------------------------------- parameters --
// FBP configuration as unpacked from the reference's packed arrays
// (setFBPParameters, cuda/src/geometries/parallel/reconstruction_methods/parameters.cu:131-219).
struct FbpConfig {
    int nrays = 0, nangles = 0, nslices = 0, objsize = 0;
    int pad = 0;
    int filter = FILTER_RAMP;
    int blocksize = 0;
    float beta_delta = 0.f, reg = 0.f, energy = 1.f, z2 = 0.f;
    float pixel_x = 1.f, pixel_y = 1.f, offset = 0.f;
    float paganin = 0.f;           // derived, parameters.cu:201-203
    int geometry = GEOM_FBP_REF;   // GEOM_FBP_REF or GEOM_FBP_LIN
    int store = STORE_F32;
};

// --- rotation axis -----------------------------------------------------------
// Shapes the phase-correlation finder supports (lengths with prime factors
// 2, 3, 5, 7 that fit the shared-memory transform).
bool centersino_shape_ok(int sizex, int sizey);
size_t centersino_workspace_bytes(int sizex, int sizey);
// Rotation-axis offset from the 0/180 degree frames (device arrays [sizey][sizex]):
// the reference's integer (subpixel = 0) or sub-pixel (1) search; synchronises st.
template <typename T>
double centersino_device(int device, const T *d_frame0, const T *d_frame1, const T *d_dark, const T *d_flat,
                         int sizex, int sizey, int subpixel, void *workspace, cudaStream_t st);

// --- BST (backprojection slice theorem) ------------------------------------
struct BstPlanShape {
    int N = 0, A = 0, Np = 0, L = 0, Lh = 0, S = 0, off = 0, threads = 0;
};
// Sizes of the BST transforms for N rays, A angles, padding pad; false when
// the padded length N*(1+pad) has a prime factor above 7 or exceeds the
// shared-memory limit of the row kernel (3 complex rows of Np).
bool bst_plan_shape(BstPlanShape &s, int N, int A, int pad);
// Device workspace bytes for nslices slices at once.
size_t bst_workspace_bytes(const BstPlanShape &s, int nslices);
// General form of the BST operator (both the FBP method and the EM back-
// projector of tEMFQ): rows of N samples edge-padded to Np (offset off) and
// optionally filtered, half-rays of Np/2 samples weighted by w_half (half of it
// at the centre) and zero-padded to L, an S x S grid, crop offset off, image
// divided by scale.
struct BstCore {
    int N = 0, A = 0, Np = 0, L = 0, Lh = 0, S = 0, off = 0, M = 0;
    bool filtered = false;
    const float2 *G = nullptr;      // filter weights [Np] when filtered
    float w_half = 4.0f, scale = 1.0f;
};
bool bst_core_ok(const BstCore &c);
// Compile-time-length transform kernels in use (raft_filter_set_fixed).
bool fixed_transforms_enabled();
size_t bst_core_workspace_bytes(const BstCore &c, int nslices);
void bst_run(int device, const BstCore &c, const float *d_tomo, float *d_obj, int nslices, void *workspace,
             cudaStream_t st);

// --- tEMFQ (transmission EM, Fourier-slice projector + BST back-projector) ----
struct TemfqConfig {
    int nrays = 0, nangles = 0, nslices = 0, zpad = 0, niter = 0, interpolation = 1, blocksize = 0;
    float dx = 0.f;
};
bool temfq_shape_ok(int N, int A, int zpad);
BstCore temfq_bst_core(int N, int A, int zpad);
size_t temfq_workspace_bytes(int N, int A, int zpad, int nslices);
// niter iterations on nslices slices: d_obj [nslices][N][N] (initial guess in,
// result out), d_counts [nslices][A][N] (read only), d_flat [nslices][N],
// d_cs / d_sn [A] = __cosf / __sinf of the angles.
void temfq_run(int device, const TemfqConfig &cfg, float *d_obj, const float *d_counts, const float *d_flat,
               const float *d_cs, const float *d_sn, int nslices, void *workspace, cudaStream_t st);
// BST reconstruction of nslices slices (d_tomo [nslices][A][N] -> d_obj
// [nslices][N][N]) on st; cfg gives N, A, pad, filter, paganin, reg, axis
// offset, pixel.
void launch_bst(int device, const FbpConfig &cfg, const float *d_tomo, float *d_obj, int nslices, void *workspace,
                cudaStream_t st);

// EM configuration (setEMRTParameters, parameters.cu:8-59).
struct EmConfig {
    int nrays = 0, nangles = 0, nslices = 0, objsize = 0;
    int niter = 0, blocksize = 0;
    int nflats = 1;
};

// Failure injection and self tests (engine.cu, backproject.cu).
void inject_alloc_failures(int n);
int selftest_bounded_wait(int gpu, int arrive, unsigned limit);

// U-Net 3x3 convolution on tcgen05 (unet_tc.cu): 0 launched, 1 launch error,
// 2 shape not handled (W must be >= 128 or divide 128; channels multiples of 32).
bool conv3x3_tc_supported(int C0, int C1, int W);
int conv3x3_tc(const void *x0, int C0, const void *x1, int C1, const void *w, const float *bias, void *y, void *y1,
               int Cy0, int N, int H, int W, int Cout, int relu, cudaStream_t st);
int conv3x3_tc_error();
// Weight (and bias) gradient of the 3x3 convolution on tcgen05 (unet_tc.cu);
// 0 = launched, 1 = launch error, 2 = shape not handled (W % 64, Cout not 32/64/128/256).
int conv3x3_wgrad_tc(const void *dy, const void *x0, int C0, const void *x1, int C1, float *dw, float *dbias, int N,
                     int H, int W, int Cout, cudaStream_t st);
void conv3x3_wgrad_tc_set_nine(int on);
void conv3x3_tc_set_halo(int on);

}  // namespace raft
