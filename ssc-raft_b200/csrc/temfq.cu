// temfq.cu -- transmission EM with the Fourier-slice projector (tEMFQ).
//
// Reference: get_tEM_FQ / get_tEM_FQ_GPU / get_tEM_FQ_MultiGPU,
// cuda/src/geometries/parallel/reconstruction_methods/em_frequency.cu:13-398,
// with the projector pst_counts_real (forward_methods/radon_fst.cu:544-637 and
// kernels/radon_fst_kernel.cu) and the back-projector EMFQ_BST(_ITER)
// (reconstruction_methods/bst.cu:100-249).  For N rays, A angles, L = N (1 + zpad):
//   backcounts = 1 / BST(counts)                       (BST: no filter, no crop,
//                                                       half-rays N/2 padded to
//                                                       N (zpad+1)/2, weight (zpad+1)^2)
//   repeat niter times:
//     model = FST(x): fftshift of the N x N image, placed in the corners of an
//             L x L zero grid, 2-D FFT, fftshift, polar samples at
//             (cos t, sin t) * (r - L/2) (nearest or bilinear), per angle
//             fftshift, 1-D inverse FFT, fftshift, centre N samples,
//             times dx / L (1 / L when dx <= 0), then flat * exp(-p)
//             (flat where p < 0);
//     x <- x * (BST(model) * backcounts).
// The reference's total-variation step is switched off there
// (parameters.cu:110), so it is not part of this operator.  Its element-wise
// kernels run on grids of size/1024 blocks and skip a tail when the sizes are
// not multiples of 1024; here every element is processed.
//
// B200 design: the fftshifts are index arithmetic, never passes over memory;
// the 2-D transform computes only the N non-zero rows of the padded grid
// (the other L - N rows are zero), then all L columns; one kernel per
// (slice, angle) gathers the polar samples straight into shared memory,
// inverse-transforms, crops, scales and forms the counts model; the BST
// back-projector is the library's (bst.cu) with this method's sizes.
// Compiled with fast math, as the reference's device code.
#include "raft.hpp"
#include "profile.hpp"
#include "fft.cuh"

namespace raft {

namespace {

struct FstArgs {
    const float *img;       // [B][N][N] current iterate
    float2 *rows;           // [B][N][L]: transforms of the N non-zero grid rows
    float2 *spec;           // [B][L][L]: spectrum, spec[b][x][y] (column-major)
    float *model;           // [B][A][N]: flat * exp(-projection)
    const float *flat;      // [B][N]
    const float *cs, *sn;   // [A]
    FftPlan pL;             // L-point transforms
    int N, A, L, interp;
    float scale;
};

// The L-point transforms: NL > 0 is L as a compile-time constant (cfft_smem,
// launched with c_fft_threads(NL) threads), 0 the plan's length.
template <int NL>
__device__ __forceinline__ const float2 *fst_fft(float2 *a, float2 *b, const FftPlan &P)
{
    if constexpr (NL > 0) {
        (void)P;
        return cfft_smem<NL>(a, b);
    } else {
        return fft_run(a, b, P);
    }
}

// Grid row q (q < N/2: row q; else row q + L - N) holds row q of the
// fftshifted image in its first N/2 and last N/2 columns.
template <int NL>
__global__ void __launch_bounds__(512) fst_rows_kernel(const FstArgs p)
{
    extern __shared__ float2 sm_fst[];
    const int b = blockIdx.y, q = blockIdx.x;
    const int N = p.N, L = p.L, h = N / 2;
    const float *src = p.img + ((size_t)b * N + (q + h) % N) * N;
    for (int c = threadIdx.x; c < L; c += blockDim.x) {
        float v = 0.f;
        if (c < h) v = src[(c + h) % N];
        else if (c >= L - (N - h)) v = src[(c - (L - N) + h) % N];
        sm_fst[c] = make_float2(v, 0.f);
    }
    __syncthreads();
    const float2 *r = fst_fft<NL>(sm_fst, sm_fst + fft_plan_span(p.pL), p.pL);
    float2 *dst = p.rows + ((size_t)b * N + q) * L;
    for (int c = threadIdx.x; c < L; c += blockDim.x) dst[c] = r[c];
}

template <int NL>
__global__ void __launch_bounds__(512) fst_cols_kernel(const FstArgs p)
{
    extern __shared__ float2 sm_fst[];
    const int b = blockIdx.y, c = blockIdx.x;
    const int N = p.N, L = p.L, h = N / 2;
    for (int y = threadIdx.x; y < L; y += blockDim.x) sm_fst[y] = make_float2(0.f, 0.f);
    __syncthreads();
    const float2 *col = p.rows + (size_t)b * N * L + c;
    for (int q = threadIdx.x; q < N; q += blockDim.x) sm_fst[q < h ? q : q + L - N] = col[(size_t)q * L];
    __syncthreads();
    const float2 *r = fst_fft<NL>(sm_fst, sm_fst + fft_plan_span(p.pL), p.pL);
    float2 *dst = p.spec + ((size_t)b * L + c) * L;
    for (int y = threadIdx.x; y < L; y += blockDim.x) dst[y] = r[y];
}

// Element of the fftshifted spectrum at row-major linear index idx (an index
// one past a row end reads the next row's first element, as the reference's
// flat indexing does).  Both coordinates wrap into [0, L), so every idx reads
// inside the slice's spectrum.
__device__ __forceinline__ float2 shifted_spec(const float2 *spec, int L, long long idx)
{
    long long ys = idx / L, xs = idx - ys * L;
    const int y = (int)((((ys + L / 2) % L) + L) % L), x = (int)((((xs + L / 2) % L) + L) % L);
    return spec[(size_t)x * L + y];
}

template <int NL>
__global__ void __launch_bounds__(512) fst_sino_kernel(const FstArgs p)
{
    extern __shared__ float2 sm_fst[];
    const int b = blockIdx.y, a = blockIdx.x;
    const int L = p.L, N = p.N;
    const float2 *spec = p.spec + (size_t)b * L * L;
    const float ca = p.cs[a], sa = p.sn[a];
    const long long LL = (long long)L * L;
    for (int qq = threadIdx.x; qq < L; qq += blockDim.x) {
        const int r = (qq + L / 2) % L;                    // the 1-D shift before the inverse transform
        const float rho = (float)((double)r - (double)L / 2.0);
        const float xpos = ca * rho, ypos = sa * rho;
        float2 v = make_float2(0.f, 0.f);
        if (p.interp == 0) {
            // cartesian2polar_nn (radon_fst_kernel.cu:455-478)
            const int xi = __float2int_rn(xpos) + L / 2, yi = __float2int_rn(ypos) + L / 2;
            const long long idx = (long long)yi * L + xi;
            if (idx < LL) v = shifted_spec(spec, L, idx);
        } else {
            // cartesian2polar_bi_v1 (radon_fst_kernel.cu:520-582)
            const long long xd = (long long)__float2int_rd(xpos) + L / 2, xu = (long long)__float2int_ru(xpos) + L / 2;
            const long long yd = (long long)__float2int_rd(ypos) + L / 2, yu = (long long)__float2int_ru(ypos) + L / 2;
            const float2 fdd = shifted_spec(spec, L, yd * L + xd), fdu = shifted_spec(spec, L, yu * L + xd);
            const float2 fud = shifted_spec(spec, L, yd * L + xu), fuu = shifted_spec(spec, L, yu * L + xu);
            const float xd_pos = (float)xd - L / 2, xu_pos = (float)xu - L / 2;
            const float yd_pos = (float)yd - L / 2, yu_pos = (float)yu - L / 2;
            if (xd == xu && yd == yu) {
                v = fdd;
            } else if (xd == xu) {
                v.x = (yu_pos - ypos) * fdd.x + (ypos - yd_pos) * fuu.x;
                v.y = (yu_pos - ypos) * fdd.y + (ypos - yd_pos) * fuu.y;
            } else if (yd == yu) {
                v.x = (xu_pos - xpos) * fdd.x + (xpos - xd_pos) * fuu.x;
                v.y = (xu_pos - xpos) * fdd.y + (xpos - xd_pos) * fuu.y;
            } else {
                v.x = (yu_pos - ypos) * ((xu_pos - xpos) * fdd.x + (xpos - xd_pos) * fud.x) +
                      (ypos - yd_pos) * ((xu_pos - xpos) * fdu.x + (xpos - xd_pos) * fuu.x);
                v.y = (yu_pos - ypos) * ((xu_pos - xpos) * fdd.y + (xpos - xd_pos) * fud.y) +
                      (ypos - yd_pos) * ((xu_pos - xpos) * fdu.y + (xpos - xd_pos) * fuu.y);
            }
        }
        sm_fst[qq] = make_float2(v.x, -v.y);               // conjugate: inverse = conj(forward(conj))
    }
    __syncthreads();
    const float2 *H = fst_fft<NL>(sm_fst, sm_fst + fft_plan_span(p.pL), p.pL);
    const float *fl = p.flat + (size_t)b * N;
    float *out = p.model + ((size_t)b * p.A + a) * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int m = ((L - N) / 2 + i + L / 2) % L;       // crop after the shift back
        const float proj = H[m].x * p.scale;               // real part (conjugation keeps it)
        out[i] = proj < 0.f ? fl[i] : fl[i] * __expf(-proj);
    }
}

template <int NL>
static void launch_fst(const FstArgs &f, int nslices, int threads, size_t sm, cudaStream_t st)
{
    // Set on every launch (a few microseconds per iteration): the limit belongs
    // to the kernel, shared by all host threads, and sm varies with L, so a
    // thread's memory of the last value it set can be undercut by another
    // thread setting a smaller one (the slab split runs one thread per entry).
    RAFT_CUDA(cudaFuncSetAttribute(fst_rows_kernel<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    RAFT_CUDA(cudaFuncSetAttribute(fst_cols_kernel<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    RAFT_CUDA(cudaFuncSetAttribute(fst_sino_kernel<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    fst_rows_kernel<NL><<<dim3(f.N, nslices), threads, sm, st>>>(f);
    RAFT_CUDA(cudaGetLastError());
    count_launch();
    fst_cols_kernel<NL><<<dim3(f.L, nslices), threads, sm, st>>>(f);
    RAFT_CUDA(cudaGetLastError());
    count_launch();
    fst_sino_kernel<NL><<<dim3(f.A, nslices), threads, sm, st>>>(f);
    RAFT_CUDA(cudaGetLastError());
}

// calc_reciprocal_element_wise: 1.0 / x in double, stored as float
__global__ void reciprocal_kernel(float *x, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = (float)(1.0 / (double)x[i]);
}

// back <- back * backcounts; x <- x * back (multiply_element_wise twice, in that order)
__global__ void emfq_update_kernel(float *x, float *back, const float *inv_bc, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float bk = back[i] * inv_bc[i];
        back[i] = bk;
        x[i] = x[i] * bk;
    }
}

unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32); }

}  // namespace

bool temfq_shape_ok(int N, int A, int zpad)
{
    if (N < 4 || N % 2 || A < 1 || zpad < 0) return false;
    const int L = N * (1 + zpad);
    if ((N * (zpad + 1)) % 2) return false;
    BstCore c = temfq_bst_core(N, A, zpad);
    const int M = fft_plan_length(L);
    return M > 0 && 2 * (size_t)fft_span(M) * sizeof(float2) <= 227 * 1024 && bst_core_ok(c);
}

BstCore temfq_bst_core(int N, int A, int zpad)
{
    // EMFQ_BST (bst.cu:100-203): rows of N samples, no padding, half-rays of
    // N/2 zero-padded to N (zpad+1)/2, weight (zpad+1)^2, an N x N grid, scale 1
    const int pad0 = zpad + 1;
    BstCore c;
    c.N = N;
    c.A = A;
    c.Np = N;
    c.L = N * pad0 / 2;
    c.Lh = c.L / 2;
    c.S = N;
    c.off = 0;
    c.M = std::max(c.Np, c.L);
    c.filtered = false;
    c.G = nullptr;
    c.w_half = (float)(pad0 * pad0);
    c.scale = 1.0f;
    return c;
}

size_t temfq_workspace_bytes(int N, int A, int zpad, int nslices)
{
    const size_t L = (size_t)N * (1 + zpad), B = nslices;
    const size_t img = B * N * N * sizeof(float);
    auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
    return al(B * A * N * sizeof(float))            // counts / model
         + 2 * al(img)                               // 1/backcounts, back
         + al(B * N * L * sizeof(float2))            // FST rows
         + al(B * L * L * sizeof(float2))            // FST spectrum
         + al(bst_core_workspace_bytes(temfq_bst_core(N, A, zpad), nslices))
         + al(2 * A * sizeof(float));                // cos / sin
}

void temfq_run(int device, const TemfqConfig &cfg, float *d_obj, const float *d_counts, const float *d_flat,
               const float *d_cs, const float *d_sn, int nslices, void *workspace, cudaStream_t st)
{
    const int N = cfg.nrays, A = cfg.nangles, zpad = cfg.zpad, L = N * (1 + zpad);
    RAFT_CHECK(temfq_shape_ok(N, A, zpad), "tEMFQ: unsupported sizes (N even; the N(1+zpad)- and N(1+zpad)/2-point "
                                           "transforms must fit shared memory: N(1+zpad) <= 14528 with prime factors "
                                           "2, 3, 5, 7, about 7000 otherwise)");
    if (nslices <= 0) return;
    const size_t B = nslices, n_img = B * N * N;
    auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
    char *w = (char *)workspace;
    float *sino = (float *)w;
    w += al(B * A * N * sizeof(float));
    float *inv_bc = (float *)w;
    w += al(n_img * sizeof(float));
    float *back = (float *)w;
    w += al(n_img * sizeof(float));
    float2 *rows = (float2 *)w;
    w += al(B * N * L * sizeof(float2));
    float2 *spec = (float2 *)w;
    w += al(B * L * L * sizeof(float2));
    void *bst_ws = w;
    const BstCore core = temfq_bst_core(N, A, zpad);
    RAFT_CUDA(cudaMemcpyAsync(sino, d_counts, B * A * N * sizeof(float), cudaMemcpyDeviceToDevice, st));

    // backcounts = 1 / BST(counts)
    bst_run(device, core, sino, inv_bc, nslices, bst_ws, st);
    count_launch();
    reciprocal_kernel<<<grid_for(n_img), 256, 0, st>>>(inv_bc, n_img);
    RAFT_CUDA(cudaGetLastError());

    const FftTable &t = fft_table(device, L);
    FstArgs f;
    f.img = d_obj;
    f.rows = rows;
    f.spec = spec;
    f.model = sino;
    f.flat = d_flat;
    f.cs = d_cs;
    f.sn = d_sn;
    f.pL = t.plan;
    f.N = N;
    f.A = A;
    f.L = L;
    f.interp = cfg.interpolation;
    // em_frequency.cu:166: dx / L, or 1 / L when dx <= 0 (the latter in double)
    f.scale = cfg.dx > 0.f ? cfg.dx / (float)L : (float)(1.0 / (float)L);
    const size_t sm = 2 * (size_t)fft_plan_span(f.pL) * sizeof(float2);
    const int threads = fft_threads(f.pL.M);
    // L as a compile-time length when it is one of those compiled
    const int fixedL = (f.pL.n == L && f.pL.M == L && threads == c_fft_threads(L) && fixed_transforms_enabled())
                           ? L : 0;
    for (int k = 0; k < cfg.niter; k++) {
        {
            ProfScope ps(PROF_PROJECT, st);   // counts the first of the three FST launches
            switch (fixedL) {
            case 1024: launch_fst<1024>(f, nslices, threads, sm, st); break;
            case 1536: launch_fst<1536>(f, nslices, threads, sm, st); break;
            case 2048: launch_fst<2048>(f, nslices, threads, sm, st); break;
            case 3072: launch_fst<3072>(f, nslices, threads, sm, st); break;
            case 4096: launch_fst<4096>(f, nslices, threads, sm, st); break;
            case 6144: launch_fst<6144>(f, nslices, threads, sm, st); break;
            case 8192: launch_fst<8192>(f, nslices, threads, sm, st); break;
            case 12288: launch_fst<12288>(f, nslices, threads, sm, st); break;
            default: launch_fst<0>(f, nslices, threads, sm, st); break;
            }
        }
        bst_run(device, core, sino, back, nslices, bst_ws, st);
        count_launch();
        emfq_update_kernel<<<grid_for(n_img), 256, 0, st>>>(d_obj, back, inv_bc, n_img);
        RAFT_CUDA(cudaGetLastError());
    }
}

}  // namespace raft
