// bst.cu -- FBP by the backprojection slice theorem (BST), Fourier regridding.
//
// Reference (cnpem/ssc-raft): getBST / getBSTGPU,
// cuda/src/geometries/parallel/reconstruction_methods/bst.cu:251-312,534-642,
// BSTFilter + BandFilterC2C, cuda/src/processing/filters/filters.cu:295-390.
// Per slice, with N rays, A angles (uniform over [0, pi)), Np = N (1 + pad):
//   1. rows edge-padded to Np (padding.cu:140-178);
//   2. unless the filter is 'none': row <- Re IFFT_unnormalised( FFT(row)
//      * apply(min(k, Np-k)/Np) * exp(-2 pi i c k / Np) ), c = integer axis offset;
//   3. each row split at its centre Np/2 into two half-rays of Np/2 samples,
//      the left one reversed (the ray at theta + pi), scaled by 4 (2 at the
//      centre sample), zero-padded to L = Np (sino2p, bst.cu:22-48);
//   4. L-point FFT of each half-ray, times 2 / (L max(min(k, L-k), 1/2)) (convBST);
//   5. polar -> Cartesian on an S x S grid (S = Np): radius rho = L |p| / S,
//      arc index 2A (atan2(p) / 2 pi + 1/2), linear in rho and, with the
//      reference's weights (t = iarc - angle, w0 = t, w1 = 1 - t), across the
//      two arcs, zero beyond rho >= L/2 - 1; times (-1)^(x+y) and stored
//      fft-shifted (polar2cartesian_fourier, bst.cu:59-98);
//   6. S x S inverse FFT, real part / (Np pixel 4), centre N x N crop.
// Two deviations, both for the reference's uninitialised or mis-sized
// buffers: step 3's zero padding is explicit (the reference leaves it to
// freshly allocated memory), and all A rows are padded (the reference's
// padding call is sized by N rows; identical when A == N).
//
// B200 design, three kernels per batch of slices, all transforms in shared
// memory (fft.cuh), no cuFFT and no S x S intermediate in HBM:
//   bst_rows_kernel    two projection rows per CTA: pad, filter (the two rows
//                      as one complex sequence), split, and one complex FFT per
//                      row carrying both half-rays (separated by symmetry);
//                      writes only the L/2 radial bins step 5 can read;
//   bst_regrid_kernel  one Cartesian row per CTA: interpolates the row from
//                      the polar data straight into shared memory, inverse
//                      FFT along x, keeps the N crop columns;
//   bst_cols_kernel    one crop column per CTA: inverse FFT along y, keeps
//                      the N crop rows, scales.
// This file is compiled with fast math, as the reference is, so the regrid
// geometry (hypotf, atan2f, the divisions) follows its rounding.
#include "raft.hpp"
#include "profile.hpp"
#include "fft.cuh"

#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

namespace raft {

namespace {

struct BstArgs {
    const float *tomo;      // [B][A][N]
    float2 *polar;          // [B][2A][Lh]
    float2 *T;              // [B][S][N]: rows inverse-transformed along x, crop columns
    float *obj;             // [B][N][N]
    FftPlan pN, pL, pS;     // transforms of the filter (Np), the half-rays (L), the grid (S)
    const float2 *G;        // filter weights [Np], or null for 'none'
    int N, A, Np, L, Lh, S, off, M;   // M = max(Np, L): shared-memory buffer length of the row kernel
    float w_half;           // half-ray weight (the centre sample gets half of it)
    float scale;
};

// The transforms of the three kernels: NF > 0 is the compile-time length
// that every transform of the launch has (cfft_smem), 0 the plans' lengths.
template <int NF>
__device__ __forceinline__ float2 *bst_fft(float2 *a, float2 *b, const FftPlan &P)
{
    if constexpr (NF > 0) {
        (void)P;
        return cfft_smem<NF>(a, b);
    } else {
        return fft_run(a, b, P);
    }
}

template <int NF>
__global__ void __launch_bounds__(512) bst_rows_kernel(const BstArgs p)
{
    extern __shared__ float2 sm_bst[];
    float2 *z = sm_bst;
    const int slice = blockIdx.y;
    const int a0 = 2 * blockIdx.x, a1 = a0 + 1;
    const bool has1 = a1 < p.A;
    const float *s0 = p.tomo + ((size_t)slice * p.A + a0) * p.N;
    const float *s1 = s0 + p.N;
    for (int n = threadIdx.x; n < p.Np; n += blockDim.x) {
        const int i = min(max(n - p.off, 0), p.N - 1);
        z[n] = make_float2(__ldg(s0 + i), has1 ? __ldg(s1 + i) : 0.f);
    }
    __syncthreads();
    float sgn1 = 1.f;   // the second row is sgn1 * z.y
    if (p.G) {
        float2 *r = bst_fft<NF>(z, sm_bst + p.M, p.pN);
        for (int k = threadIdx.x; k < p.Np; k += blockDim.x) {
            const float2 g = cmul(r[k], __ldg(&p.G[k]));
            r[k] = make_float2(g.x, -g.y);
        }
        __syncthreads();
        // forward transform of the conjugate = conjugate of the inverse
        z = bst_fft<NF>(r, r == sm_bst ? sm_bst + p.M : sm_bst, p.pN);
        sgn1 = -1.f;
    }
    // two buffers of M elements: the filtered pair z, and the other one.  The
    // second row's half-rays are parked in its own (not yet written) polar row
    // while the first row is transformed, then brought back.
    float2 *fa = (z == sm_bst) ? sm_bst + p.M : sm_bst;
    float2 *fb = z;
    const int c = p.Np / 2, half = p.Np / 2;
    const size_t pb = (size_t)slice * 2 * p.A * p.Lh;
    float2 *park = p.polar + pb + (size_t)a1 * p.Lh;       // half <= Lh entries
    if (has1)
        for (int idx = threadIdx.x; idx < half; idx += blockDim.x) {
            const float w = idx == 0 ? 0.5f * p.w_half : p.w_half;
            park[idx] = make_float2(w * sgn1 * z[c - 1 - idx].y, w * sgn1 * z[c + idx].y);
        }
    for (int r = 0; r < (has1 ? 2 : 1); r++) {
        for (int idx = threadIdx.x; idx < p.L; idx += blockDim.x) {
            float2 h = make_float2(0.f, 0.f);
            if (idx < half) {
                if (r == 0) {
                    const float w = idx == 0 ? 0.5f * p.w_half : p.w_half;
                    h = make_float2(w * z[c - 1 - idx].x, w * z[c + idx].x);
                } else {
                    h = park[idx];       // written by this same thread above
                }
            }
            fa[idx] = h;
        }
        __syncthreads();
        const float2 *H = bst_fft<NF>(fa, fb, p.pL);
        float2 *frow = p.polar + pb + (size_t)(a0 + r) * p.Lh;           // left half-ray (theta + pi)
        float2 *rrow = p.polar + pb + (size_t)(p.A + a0 + r) * p.Lh;     // right half-ray (theta)
        for (int k = threadIdx.x; k < p.Lh; k += blockDim.x) {
            const float2 Zk = H[k], Zm = H[k == 0 ? 0 : p.L - k];
            const float sig = 2.f / ((float)p.L * fmaxf((float)k, 0.5f));
            // Z = FFT(f + i g): F(f) = (Z_k + conj Z_-k)/2, F(g) = (Z_k - conj Z_-k)/(2i)
            frow[k] = make_float2(0.5f * (Zk.x + Zm.x) * sig, 0.5f * (Zk.y - Zm.y) * sig);
            rrow[k] = make_float2(0.5f * (Zk.y + Zm.y) * sig, -0.5f * (Zk.x - Zm.x) * sig);
        }
        __syncthreads();
        // the next row's input goes to the buffer the result is not in
        fa = (H == fa) ? fb : fa;
        fb = (fa == sm_bst) ? sm_bst + p.M : sm_bst;
    }
}

template <int NF>
__global__ void __launch_bounds__(512) bst_regrid_kernel(const BstArgs p)
{
    extern __shared__ float2 sm_bst[];
    const int slice = blockIdx.y, Y = blockIdx.x;
    const int S = p.S, h = S / 2, twoA = 2 * p.A;
    const int ty = (Y - h + S) % S;            // array row Y holds grid row ty (stored shifted by S/2)
    const float posy = (float)(ty - h);
    const float sy = 4.f * ((float)(ty % 2) - 0.5f);
    const float2 *pol = p.polar + (size_t)slice * twoA * p.Lh;
    const int rmax = p.L / 2 - 1;
    for (int X = threadIdx.x; X < S; X += blockDim.x) {
        // (X - h + S) % S, X < S: one conditional add (integer modulos by
        // run-time values cost about twenty instructions each)
        const int tx = X - h < 0 ? X - h + S : X - h;
        const float posx = (float)(tx - h);
        const float rho = (float)p.L * hypotf(posx, posy) / (float)S;
        const float angle = (float)twoA * (0.5f * atan2f(posy, posx) / (float)M_PI + 0.5f);
        const int irho = (int)rho;
        int iarc = (int)angle;
        float2 v = make_float2(0.f, 0.f);
        if (irho < rmax) {
            const float pfrac = rho - (float)irho;
            const float tfrac = (float)iarc - angle;
            // angle lies in [0, twoA] (truncation keeps iarc >= 0): iarc % twoA
            // and (iarc + 1) % twoA as conditional subtractions
            iarc = iarc >= twoA ? iarc - twoA : iarc;
            const int uarc = iarc + 1 >= twoA ? iarc + 1 - twoA : iarc + 1;
            const float2 *q0 = pol + (size_t)iarc * p.Lh + irho;
            const float2 *q1 = pol + (size_t)uarc * p.Lh + irho;
            const float2 c00 = __ldg(q0), c01 = __ldg(q0 + 1), c10 = __ldg(q1), c11 = __ldg(q1 + 1);
            const float2 i0 = make_float2(c00.x * (1.f - pfrac) + c01.x * pfrac, c00.y * (1.f - pfrac) + c01.y * pfrac);
            const float2 i1 = make_float2(c10.x * (1.f - pfrac) + c11.x * pfrac, c10.y * (1.f - pfrac) + c11.y * pfrac);
            v = make_float2(i0.x * tfrac + i1.x * (1.f - tfrac), i0.y * tfrac + i1.y * (1.f - tfrac));
        }
        const float sgn = sy * ((float)(tx & 1) - 0.5f);
        sm_bst[X] = make_float2(v.x * sgn, -v.y * sgn);   // conjugated: see bst_cols_kernel
    }
    __syncthreads();
    const float2 *r = bst_fft<NF>(sm_bst, sm_bst + fft_plan_span(p.pS), p.pS);
    float2 *trow = p.T + ((size_t)slice * S + Y) * p.N;
    for (int i = threadIdx.x; i < p.N; i += blockDim.x) trow[i] = r[p.off + i];
}

// T holds conj(IFFT_x(grid)); its forward transform along y is the conjugate
// of the 2-D inverse transform, whose real part is the image.
template <int NF>
__global__ void __launch_bounds__(512) bst_cols_kernel(const BstArgs p)
{
    extern __shared__ float2 sm_bst[];
    const int slice = blockIdx.y, i = blockIdx.x;
    const float2 *tcol = p.T + (size_t)slice * p.S * p.N + i;
    for (int Y = threadIdx.x; Y < p.S; Y += blockDim.x) sm_bst[Y] = tcol[(size_t)Y * p.N];
    __syncthreads();
    const float2 *r = bst_fft<NF>(sm_bst, sm_bst + fft_plan_span(p.pS), p.pS);
    float *o = p.obj + (size_t)slice * p.N * p.N + i;
    for (int j = threadIdx.x; j < p.N; j += blockDim.x) o[(size_t)j * p.N] = r[p.off + j].x / p.scale;
}

// Forward DFT in FP64 of a 7-smooth length (recursive decimation in time on
// the smallest factor), for the Bluestein chirp spectrum.
void dft_rec(const std::complex<double> *in, size_t stride, int n, std::complex<double> *out)
{
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    int p = 2;
    while (n % p) p++;
    const int m = n / p;
    for (int r = 0; r < p; r++) dft_rec(in + r * stride, stride * p, m, out + (size_t)r * m);
    std::vector<std::complex<double>> tmp(n);
    for (int k = 0; k < m; k++)
        for (int q = 0; q < p; q++) {
            std::complex<double> acc = 0.0;
            for (int r = 0; r < p; r++) {
                const double a = -2.0 * M_PI * (double)(((long long)r * (k + (long long)q * m)) % n) / (double)n;
                acc += out[(size_t)r * m + k] * std::complex<double>(std::cos(a), std::sin(a));
            }
            tmp[(size_t)q * m + k] = acc;
        }
    std::copy(tmp.begin(), tmp.end(), out);
}

void dft_host(const std::vector<std::complex<double>> &in, std::vector<std::complex<double>> &out)
{
    out.assign(in.size(), 0.0);
    dft_rec(in.data(), 1, (int)in.size(), out.data());
}

using BstKey = std::tuple<int, int, int, int, double, double>;
std::mutex g_bst_mtx;
std::map<BstKey, float2 *> g_bst_filters;   // filter weights per (device, Np, type, offset, paganin, reg)

const float2 *bst_filter_weights(int device, int Np, int ftype, int c, double paganin, double reg)
{
    std::lock_guard<std::mutex> lk(g_bst_mtx);
    float2 *&slot = g_bst_filters[BstKey(device, Np, ftype, c, paganin, reg)];
    if (!slot) {
        std::vector<float2> G(Np);
        for (int k = 0; k < Np; k++) {
            const double w = filter_apply_ref(ftype, (double)std::min(k, Np - k) / Np, paganin, reg);
            const double ph = -2.0 * M_PI * (double)c * (double)k / (double)Np;
            G[k] = make_float2((float)(w * std::cos(ph)), (float)(w * std::sin(ph)));
        }
        RAFT_CUDA(cudaMalloc(&slot, sizeof(float2) * Np));
        RAFT_CUDA(cudaMemcpy(slot, G.data(), sizeof(float2) * Np, cudaMemcpyHostToDevice));
    }
    return slot;
}

std::mutex g_fft_mtx;
std::map<std::pair<int, int>, std::unique_ptr<FftTable>> g_fft_tables;

}  // namespace

int fft_plan_length(int n)
{
    int r[24], nr = 0;
    if (n < 1) return 0;
    if (factorize(n, r, nr)) return n;
    for (int M = 2 * n - 1; M <= 8 * n; M++)
        if (factorize(M, r, nr)) return M;
    return 0;
}

const FftTable &fft_table(int device, int n)
{
    std::lock_guard<std::mutex> lk(g_fft_mtx);
    auto &slot = g_fft_tables[{device, n}];
    if (!slot) {
        auto t = std::make_unique<FftTable>();
        const int M = fft_plan_length(n);
        RAFT_CHECK(M > 0, "FFT length without a transform plan");
        FftPlan &P = t->plan;
        P.n = n;
        P.M = M;
        RAFT_CHECK(factorize(M, P.rl.r, P.rl.n), "FFT plan length");
        if (M == n) {
            t->rl = P.rl;
            const std::vector<float2> h = fft_twiddles(n);
            RAFT_CUDA(cudaMalloc(&t->tw, sizeof(float2) * n));
            RAFT_CUDA(cudaMemcpy(t->tw, h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
        } else {
            // chirp w_j = exp(-i pi j^2 / n) (j^2 reduced mod 2n, exact in 64 bits)
            // and the M-point transform of c_m = conj(w_|m|), |m| < n, in FP64
            std::vector<float2> w(n);
            std::vector<std::complex<double>> c(M, 0.0), C(M);
            for (int j = 0; j < n; j++) {
                const long long q = ((long long)j * j) % (2LL * n);
                const double a = -M_PI * (double)q / (double)n;
                w[j] = make_float2((float)std::cos(a), (float)std::sin(a));
                const std::complex<double> cj(std::cos(a), -std::sin(a));
                c[j] = cj;
                if (j) c[M - j] = cj;
            }
            dft_host(c, C);
            std::vector<float2> B(M);
            for (int k = 0; k < M; k++) B[k] = make_float2((float)(C[k].real() / M), (float)(C[k].imag() / M));
            RAFT_CUDA(cudaMalloc(&t->chirp, sizeof(float2) * n));
            RAFT_CUDA(cudaMalloc(&t->B, sizeof(float2) * M));
            RAFT_CUDA(cudaMemcpy(t->chirp, w.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
            RAFT_CUDA(cudaMemcpy(t->B, B.data(), sizeof(float2) * M, cudaMemcpyHostToDevice));
            P.chirp = t->chirp;
            P.B = t->B;
        }
        slot = std::move(t);
    }
    return *slot;
}

FftTable::~FftTable()
{
    if (tw) cudaFree(tw);
    if (chirp) cudaFree(chirp);
    if (B) cudaFree(B);
}

constexpr size_t kBstSmemMax = 227 * 1024;

// Buffer span of the transform plan of n (Bluestein lengths transform M > n
// points); huge when n has no plan.
static int plan_span(int n)
{
    const int M = fft_plan_length(n);
    return M > 0 ? fft_span(M) : (1 << 28);
}

// Shared-memory buffer length of the row kernel: the padded row and both
// transforms' ping-pong buffers (fft_span is not monotonic at its padding limit).
static int bst_row_span(const BstCore &c)
{
    return std::max({c.Np, c.filtered ? plan_span(c.Np) : 0, plan_span(c.L)});
}

bool bst_core_ok(const BstCore &c)
{
    return c.N >= 2 && c.A >= 1 && c.L >= 2 && c.S >= 2 && 2 * (size_t)bst_row_span(c) * sizeof(float2) <= kBstSmemMax &&
           2 * (size_t)plan_span(c.S) * sizeof(float2) <= kBstSmemMax;
}

bool bst_plan_shape(BstPlanShape &s, int N, int A, int pad)
{
    s.N = N;
    s.A = A;
    s.Np = N * (1 + pad);
    s.L = s.Np;
    s.Lh = s.L / 2;
    s.S = s.Np;
    s.off = (pad * N) / 2;
    s.threads = fft_threads(s.Np);
    BstCore c;
    c.N = N; c.A = A; c.Np = s.Np; c.L = s.L; c.Lh = s.Lh; c.S = s.S; c.off = s.off; c.M = s.Np;
    c.filtered = true;
    return bst_core_ok(c);
}

size_t bst_workspace_bytes(const BstPlanShape &s, int nslices)
{
    const size_t polar = (size_t)nslices * 2 * s.A * s.Lh * sizeof(float2);
    const size_t T = (size_t)nslices * s.S * s.N * sizeof(float2);
    return ((polar + 255) & ~(size_t)255) + T;
}

size_t bst_core_workspace_bytes(const BstCore &c, int nslices)
{
    const size_t polar = (size_t)nslices * 2 * c.A * c.Lh * sizeof(float2);
    const size_t T = (size_t)nslices * c.S * c.N * sizeof(float2);
    return ((polar + 255) & ~(size_t)255) + T;
}

// Calls f(integral_constant<int, n>) when n is one of the compiled transform
// lengths, f(integral_constant<int, 0>) otherwise.
template <class F>
static void with_fixed_length(int n, F &&f)
{
    using std::integral_constant;
    switch (n) {
    case 1024: f(integral_constant<int, 1024>{}); break;
    case 1536: f(integral_constant<int, 1536>{}); break;
    case 2048: f(integral_constant<int, 2048>{}); break;
    case 3072: f(integral_constant<int, 3072>{}); break;
    case 4096: f(integral_constant<int, 4096>{}); break;
    case 6144: f(integral_constant<int, 6144>{}); break;
    case 8192: f(integral_constant<int, 8192>{}); break;
    case 12288: f(integral_constant<int, 12288>{}); break;
    default: f(integral_constant<int, 0>{}); break;
    }
}

template <int NF>
static void launch_bst_rows(const BstArgs &a, const BstCore &c, int nslices, int threads, size_t sm3, cudaStream_t st)
{
    static thread_local int configured = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured != dev) {
        RAFT_CUDA(cudaFuncSetAttribute(bst_rows_kernel<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kBstSmemMax));
        configured = dev;
    }
    bst_rows_kernel<NF><<<dim3((c.A + 1) / 2, nslices), threads, sm3, st>>>(a);
    RAFT_CUDA(cudaGetLastError());
}

template <int NF>
static void launch_bst_grid(const BstArgs &a, const BstCore &c, int nslices, int threads, size_t sm2, cudaStream_t st)
{
    static thread_local int configured = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (configured != dev) {
        RAFT_CUDA(cudaFuncSetAttribute(bst_regrid_kernel<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kBstSmemMax));
        RAFT_CUDA(cudaFuncSetAttribute(bst_cols_kernel<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kBstSmemMax));
        configured = dev;
    }
    bst_regrid_kernel<NF><<<dim3(c.S, nslices), threads, sm2, st>>>(a);
    RAFT_CUDA(cudaGetLastError());
    count_launch();
    bst_cols_kernel<NF><<<dim3(c.N, nslices), threads, sm2, st>>>(a);
    RAFT_CUDA(cudaGetLastError());
}

void bst_run(int device, const BstCore &c, const float *d_tomo, float *d_obj, int nslices, void *workspace,
             cudaStream_t st)
{
    RAFT_CHECK(bst_core_ok(c), "BST: unsupported transform lengths");
    if (nslices <= 0) return;
    const FftTable &tS = fft_table(device, c.S), &tL = fft_table(device, c.L);
    BstArgs a;
    a.tomo = d_tomo;
    a.polar = (float2 *)workspace;
    const size_t polar = (size_t)nslices * 2 * c.A * c.Lh * sizeof(float2);
    a.T = (float2 *)((char *)workspace + ((polar + 255) & ~(size_t)255));
    a.obj = d_obj;
    a.G = c.G;
    a.pN = c.G ? fft_table(device, c.Np).plan : FftPlan{};
    a.pL = tL.plan;
    a.pS = tS.plan;
    a.N = c.N;
    a.A = c.A;
    a.Np = c.Np;
    a.L = c.L;
    a.Lh = c.Lh;
    a.S = c.S;
    a.off = c.off;
    a.M = bst_row_span(c);
    a.w_half = c.w_half;
    a.scale = c.scale;
    const int threads = fft_threads(std::max({c.M, a.pN.M, a.pL.M, a.pS.M}));
    const size_t sm3 = 2 * (size_t)a.M * sizeof(float2), sm2 = 2 * (size_t)fft_plan_span(a.pS) * sizeof(float2);
    // compile-time lengths where the plans are direct: the rows kernel's
    // transforms (the filter's, when there is one, and the half-rays') and the
    // grid transforms of the regrid and column kernels; each kernel then runs
    // with the thread count of its length
    const bool en = fixed_transforms_enabled();
    const int nrow = (en && a.pL.n == a.pL.M && (!c.G || (a.pN.n == a.pL.n && a.pN.M == a.pN.n))) ? a.pL.n : 0;
    const int ngrid = (en && a.pS.n == a.pS.M) ? a.pS.n : 0;
    ProfScope ps(PROF_OTHER, st);   // counts the first of the three launches
    with_fixed_length(nrow, [&](auto nf) {
        constexpr int NF = decltype(nf)::value;
        launch_bst_rows<NF>(a, c, nslices, NF ? c_fft_threads(NF) : threads, sm3, st);
    });
    count_launch();
    with_fixed_length(ngrid, [&](auto nf) {
        constexpr int NF = decltype(nf)::value;
        launch_bst_grid<NF>(a, c, nslices, NF ? c_fft_threads(NF) : threads, sm2, st);
    });
}

void launch_bst(int device, const FbpConfig &cfg, const float *d_tomo, float *d_obj, int nslices, void *workspace,
                cudaStream_t st)
{
    BstPlanShape shape;
    RAFT_CHECK(bst_plan_shape(shape, cfg.nrays, cfg.nangles, cfg.pad),
               "BST: the padded length N*(1+pad) is too long for the shared-memory transforms (at most 14528 with prime factors 2, 3, 5, 7; about 7000 otherwise)");
    BstCore c;
    c.N = shape.N;
    c.A = shape.A;
    c.Np = shape.Np;
    c.L = shape.L;
    c.Lh = shape.Lh;
    c.S = shape.S;
    c.off = shape.off;
    c.M = shape.Np;
    c.filtered = cfg.filter != FILTER_NONE;
    // the reference passes the axis offset to an int (filters.cu:345-390)
    c.G = c.filtered ? bst_filter_weights(device, shape.Np, cfg.filter, (int)cfg.offset, cfg.paganin, cfg.reg)
                     : nullptr;
    c.w_half = 4.0f;   // pad0^2 with the reference's fixed pad0 = 2 (bst.cu:22-48, 561)
    c.scale = (float)shape.Np * cfg.pixel_x * 4.0f;
    bst_run(device, c, d_tomo, d_obj, nslices, workspace, st);
}

}  // namespace raft
