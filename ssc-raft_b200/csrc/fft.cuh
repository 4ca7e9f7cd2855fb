// fft.cuh -- the self-sorting (Stockham) mixed-radix complex FFT shared by the
// filter, BST, tEMFQ and rotation-axis kernels.
//
// A CTA transforms one length-n sequence held in shared memory, ping-ponging
// between two buffers of fft_span(n) elements each; radices 2, 3, 4, 5, 7, 8
// (lengths whose other prime factors are rejected on the host).  The input is
// read from, and the result left in, plain order; intermediate passes store
// one pad element after every 16 (n <= 12288) so that the strided writes of
// the early passes spread over the shared-memory banks.  Twiddles: one value
// exp(-2 pi i k / n) per butterfly from sincospif (a table load from global
// memory was latency-bound; the host-built FP64 table stays available to the
// callers), its powers by repeated complex products.  Only the forward
// transform exists: an inverse is the forward transform of the conjugate,
// conjugated.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

namespace raft {

// ---------------------------------------------------------------- host --
// Radices of n, largest first among the powers of two; false if n has a prime
// factor above 7 or needs more than 24 passes.
static inline bool factorize(int n, int *radix, int &nradix)
{
    nradix = 0;
    int e2 = 0;
    while (n % 2 == 0) { n /= 2; e2++; }
    while (e2 >= 3) { radix[nradix++] = 8; e2 -= 3; }
    if (e2 == 2) radix[nradix++] = 4;
    if (e2 == 1) radix[nradix++] = 2;
    for (int p : {3, 5, 7})
        while (n % p == 0) { n /= p; radix[nradix++] = p; }
    return n == 1 && nradix <= 24;
}

// exp(-2 pi i k / n), k < n, rounded from FP64.
static inline std::vector<float2> fft_twiddles(int n)
{
    std::vector<float2> tw(n);
    for (int k = 0; k < n; k++) {
        const double a = -2.0 * M_PI * (double)k / (double)n;
        tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    return tw;
}

// Intermediate passes are stored padded up to this length (above it the two
// padded buffers would not fit beside each other in shared memory).
constexpr int kFftPadMax = 12288;
__host__ __device__ constexpr bool fft_padded(int n) { return n <= kFftPadMax; }
// Elements one ping-pong buffer of an n-point transform occupies.
__host__ __device__ constexpr int fft_span(int n) { return fft_padded(n) ? n + n / 16 + 1 : n; }

// Threads per CTA for one length-n transform: about 8 butterflies of the
// smallest radix per thread, 128..512 threads.
static inline int fft_threads(int n)
{
    int T = ((n / 16 + 31) / 32) * 32;
    return T < 128 ? 128 : (T > 512 ? 512 : T);
}

// -------------------------------------------------------------- device --
// Complex arithmetic with every rounding explicit (the compiler may not fuse
// or split any of it), so a transform gives the same bits in every kernel it
// is inlined into: the compile-time-length passes and fft_pass agree bit for
// bit.  (The packed two-lane FP32 instructions give the same bits; they
// measured 3 % slower in the 6144-point filter and are not used.)
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    return make_float2(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return add2(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b)
{
    return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
}
// multiply by -i
__device__ __forceinline__ float2 cmni(float2 a) { return make_float2(a.y, -a.x); }

// forward DFTs (exp(-2 pi i rq/R)) on registers
template <int R> struct Dft;

template <> struct Dft<2> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};
template <> struct Dft<4> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float2 s0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]);
        const float2 s1 = cadd(v[1], v[3]);
        // -i (v1 - v3)
        const float2 d1 = make_float2(__fsub_rn(v[1].y, v[3].y), __fsub_rn(v[3].x, v[1].x));
        v[0] = cadd(s0, s1);
        v[2] = csub(s0, s1);
        v[1] = cadd(d0, d1);
        v[3] = csub(d0, d1);
    }
};
template <> struct Dft<8> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float r = 0.70710678118654752f;
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4>::run(e);
        Dft<4>::run(o);
        // twiddles exp(-2 pi i k/8), k = 0..3:
        //   o1 w1 = r (o1.x + o1.y, o1.y - o1.x), o2 w2 = -i o2,
        //   o3 w3 = r (o3.y - o3.x, -(o3.x + o3.y))
        const float2 rr = make_float2(r, r), nr = make_float2(-r, -r);
        const float2 s1 = make_float2(__fadd_rn(o[1].x, o[1].y), __fsub_rn(o[1].y, o[1].x));
        const float2 s3 = make_float2(__fsub_rn(o[3].y, o[3].x), -__fadd_rn(o[3].x, o[3].y));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = fma2(rr, s1, e[1]);
        v[5] = fma2(nr, s1, e[1]);
        v[2] = make_float2(__fadd_rn(e[2].x, o[2].y), __fsub_rn(e[2].y, o[2].x));
        v[6] = make_float2(__fsub_rn(e[2].x, o[2].y), __fadd_rn(e[2].y, o[2].x));
        v[3] = fma2(rr, s3, e[3]);
        v[7] = fma2(nr, s3, e[3]);
    }
};
// odd radices: direct sum with constant roots cos/sin(2 pi m / R)
template <int R> struct Roots;
template <> struct Roots<3> {
    static __device__ __forceinline__ float c(int m) { return m == 0 ? 1.f : -0.5f; }
    static __device__ __forceinline__ float s(int m) { return m == 0 ? 0.f : (m == 1 ? 0.86602540378443865f : -0.86602540378443865f); }
};
template <> struct Roots<5> {
    static __device__ __forceinline__ float c(int m)
    {
        return m == 0 ? 1.f : (m == 1 || m == 4) ? 0.30901699437494745f : -0.80901699437494742f;
    }
    static __device__ __forceinline__ float s(int m)
    {
        return m == 0 ? 0.f : m == 1 ? 0.95105651629515357f : m == 2 ? 0.58778525229247314f
             : m == 3 ? -0.58778525229247314f : -0.95105651629515357f;
    }
};
template <> struct Roots<7> {
    static __device__ __forceinline__ float c(int m)
    {
        return m == 0 ? 1.f : (m == 1 || m == 6) ? 0.62348980185873353f
             : (m == 2 || m == 5) ? -0.22252093395631440f : -0.90096886790241913f;
    }
    static __device__ __forceinline__ float s(int m)
    {
        return m == 0 ? 0.f : m == 1 ? 0.78183148246802981f : m == 2 ? 0.97492791218182361f
             : m == 3 ? 0.43388373911755812f : m == 4 ? -0.43388373911755812f
             : m == 5 ? -0.97492791218182361f : -0.78183148246802981f;
    }
};
template <int R> struct DftOdd {
    static __device__ __forceinline__ void run(float2 *v)
    {
        float2 in[R], sw[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            in[r] = v[r];
            sw[r] = make_float2(v[r].y, v[r].x);
        }
#pragma unroll
        for (int q = 0; q < R; q++) {
            float2 acc = in[0];
#pragma unroll
            for (int r = 1; r < R; r++) {
                const int m = (r * q) % R;
                // in[r] exp(-2 pi i m / R) = in[r] (c(m) - i s(m)):
                // (x c + y s, y c - x s), two packed fmas
                const float c = Roots<R>::c(m), s = Roots<R>::s(m);
                acc = fma2(in[r], make_float2(c, c), acc);
                acc = fma2(sw[r], make_float2(s, -s), acc);
            }
            v[q] = acc;
        }
    }
};
template <> struct Dft<3> { static __device__ __forceinline__ void run(float2 *v) { DftOdd<3>::run(v); } };
template <> struct Dft<5> { static __device__ __forceinline__ void run(float2 *v) { DftOdd<5>::run(v); } };
template <> struct Dft<7> { static __device__ __forceinline__ void run(float2 *v) { DftOdd<7>::run(v); } };

__device__ __forceinline__ int fft_pad(int i) { return i + (i >> 4); }

// One Stockham pass of radix R from src to dst (Np complex values in shared
// memory; pin / pout: src / dst stored padded).  Butterfly j = q Ns + k; the
// thread's (q, k) advance by blockDim.x without a division per butterfly.
// The twiddle exp(-2 pi i k twstep / Np) is computed only when k changes (for
// Ns dividing the block size a thread keeps one k for the whole pass).  An SFU
// __sincosf in place of sincospif measured 0.6 % faster FBP and doubled the
// filter's error against the FP64 oracle (1.4e-5 for 14400-bin linear rows);
// not used.
template <int R>
__device__ __noinline__ void fft_pass(const float2 *__restrict__ src, float2 *__restrict__ dst, int Np,
                                      int Ns, const float2 *__restrict__ tw, int pin, int pout)
{
    (void)tw;
    const int nb = Np / R;
    const int twstep = Np / (Ns * R);
    const int T = blockDim.x;
    int q = threadIdx.x / Ns, k = threadIdx.x - q * Ns;
    const int dq = T / Ns, dk = T - dq * Ns;
    int kw = -1;
    float2 w1 = make_float2(1.f, 0.f);
    for (int j = threadIdx.x; j < nb; j += T) {
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int si = j + r * nb;
            v[r] = src[pin ? fft_pad(si) : si];
        }
        if (k > 0) {
            // w^r, r < R, from w = exp(-2 pi i k twstep / Np) by repeated products
            // (two complex registers live; relative error of w^7 a few 1e-7)
            if (k != kw) {
                // sincospif rounds to about one unit in the last place
                float sn, cs;
                sincospif(-2.0f * (float)(k * twstep) / (float)Np, &sn, &cs);
                w1 = make_float2(cs, sn);
                kw = k;
            }
            float2 w = w1;
#pragma unroll
            for (int r = 1; r < R; r++) {
                v[r] = cmul(v[r], w);
                if (r + 1 < R) w = cmul(w, w1);
            }
        }
        Dft<R>::run(v);
        const int base = q * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int di = base + r * Ns;
            dst[pout ? fft_pad(di) : di] = v[r];
        }
        q += dq;
        k += dk;
        if (k >= Ns) {
            k -= Ns;
            q++;
        }
    }
    __syncthreads();
}

struct RadixList {
    int n;
    int r[24];
};

// Forward FFT of a[0..Np) (plain order); a and b each hold fft_span(Np)
// elements; the result ends in a or b (plain order), which is returned.
__device__ __forceinline__ float2 *fft_forward(float2 *a, float2 *b, int Np, const RadixList &rl,
                                               const float2 *tw)
{
    int Ns = 1;
    const int pad = fft_padded(Np);
    for (int p = 0; p < rl.n; p++) {
        const int pin = pad && p > 0, pout = pad && p + 1 < rl.n;
        switch (rl.r[p]) {
        case 2: fft_pass<2>(a, b, Np, Ns, tw, pin, pout); break;
        case 3: fft_pass<3>(a, b, Np, Ns, tw, pin, pout); break;
        case 4: fft_pass<4>(a, b, Np, Ns, tw, pin, pout); break;
        case 5: fft_pass<5>(a, b, Np, Ns, tw, pin, pout); break;
        case 7: fft_pass<7>(a, b, Np, Ns, tw, pin, pout); break;
        default: fft_pass<8>(a, b, Np, Ns, tw, pin, pout); break;
        }
        Ns *= rl.r[p];
        float2 *t = a; a = b; b = t;
    }
    return a;
}


// ------------------------------------------------ compile-time length --
// The same transform for a length known at compile time: the passes are
// unrolled, so every shared-memory address is the thread's padded index plus
// an immediate offset, and a pass whose twiddle index k is the same in every
// iteration of a thread computes its twiddle once.  Radix order, twiddle
// expressions and butterflies are those of fft_pass, with every rounding
// explicit, so the results are bit for bit fft_forward's.  The first pass's
// loads and the last pass's
// stores are functors, so callers can read the input from global memory and
// consume the output in registers.
struct CRadices {
    int n;
    int r[24];
};
__host__ __device__ constexpr CRadices c_factorize(int n)
{
    CRadices o{};
    int e2 = 0;
    while (n % 2 == 0) { n /= 2; e2++; }
    while (e2 >= 3) { o.r[o.n++] = 8; e2 -= 3; }
    if (e2 == 2) o.r[o.n++] = 4;
    if (e2 == 1) o.r[o.n++] = 2;
    while (n % 3 == 0) { n /= 3; o.r[o.n++] = 3; }
    while (n % 5 == 0) { n /= 5; o.r[o.n++] = 5; }
    while (n % 7 == 0) { n /= 7; o.r[o.n++] = 7; }
    if (n != 1) o.n = -1;
    return o;
}
__host__ __device__ constexpr int c_fft_threads(int n)
{
    return ((n / 16 + 31) / 32) * 32 < 128 ? 128 : (((n / 16 + 31) / 32) * 32 > 512 ? 512 : ((n / 16 + 31) / 32) * 32);
}

// Shared-memory source of pass (R, NS): element j + r nb, stored padded or plain.
template <int NP, int T, int R, bool PIN>
struct CSmemIn {
    const float2 *s;
    int base;   // padded (or plain) index of threadIdx.x
    __device__ __forceinline__ CSmemIn(const float2 *s_) : s(s_), base(PIN ? fft_pad(threadIdx.x) : threadIdx.x) {}
    __device__ __forceinline__ float2 operator()(int j, int it, int r) const
    {
        constexpr int nb = NP / R;
        static_assert(!PIN || (T % 16 == 0 && nb % 16 == 0), "padded source needs 16 | T and 16 | nb");
        (void)j;
        return PIN ? s[base + it * (T + T / 16) + r * (nb + nb / 16)] : s[base + it * T + r * nb];
    }
};
// Shared-memory destination of pass (R, NS): element q NS R + k + r NS.
template <int NP, int R, int NS, bool POUT>
struct CSmemOut {
    float2 *d;
    __device__ __forceinline__ void operator()(int q, int k, const float2 (&v)[R]) const
    {
        const int b = q * NS * R + k;
        constexpr bool small = (16 % (NS * R)) == 0;
        constexpr bool split = (NS * R) % 16 == 0 && (NS % 16 == 0 || 16 % NS == 0);
        if (!POUT) {
#pragma unroll
            for (int r = 0; r < R; r++) d[b + r * NS] = v[r];
        } else if (small || split) {
            // pad(b + r NS) = pad(b) + r NS (+ r NS / 16 when 16 | NS R)
            const int pb = fft_pad(b);
#pragma unroll
            for (int r = 0; r < R; r++) d[pb + r * NS + (small ? 0 : (r * NS) / 16)] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) d[fft_pad(b + r * NS)] = v[r];
        }
    }
};

// One pass of radix R over NP points with T threads: v[r] = in(j, it, r)
// (element j + r NP/R of the pass input), twiddles, R-point DFT,
// out(q, k, v) (elements q NS R + k + r NS of the pass output).
template <int NP, int T, int R, int NS, class In, class Out>
__device__ __forceinline__ void cfft_pass(const In &in, const Out &out)
{
    constexpr int nb = NP / R;
    constexpr int twstep = NP / (NS * R);
    constexpr int ITER = (nb + T - 1) / T;
    constexpr bool kfix = T % NS == 0;   // k = threadIdx.x % NS in every iteration
    float2 wfix = make_float2(1.f, 0.f);
    if (kfix && NS > 1) {
        const int k = threadIdx.x % NS;
        if (k > 0) {
            float sn, cs;
            sincospif(-2.0f * (float)(k * twstep) / (float)NP, &sn, &cs);
            wfix = make_float2(cs, sn);
        }
    }
#pragma unroll
    for (int it = 0; it < ITER; it++) {
        const int j = threadIdx.x + it * T;
        if (nb % T != 0 && j >= nb) break;
        const int q = j / NS, k = j - q * NS;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = in(j, it, r);
        if (NS > 1 && k > 0) {
            float2 w1 = wfix;
            if (!kfix) {
                float sn, cs;
                sincospif(-2.0f * (float)(k * twstep) / (float)NP, &sn, &cs);
                w1 = make_float2(cs, sn);
            }
            float2 w = w1;
#pragma unroll
            for (int r = 1; r < R; r++) {
                v[r] = cmul(v[r], w);
                if (r + 1 < R) w = cmul(w, w1);
            }
        }
        Dft<R>::run(v);
        out(q, k, v);
    }
}

// Passes P.. of the NP-point transform from buffer a (b the other buffer);
// pass 0 reads through `first`, the last pass writes through `last`; the
// passes in between ping-pong through shared memory with a barrier after each.
// (NS: product of the radices of the passes before P.)
template <int NP, int P, int NS, class First, class Last>
__device__ __forceinline__ void cfft_passes(float2 *a, float2 *b, const First &first, const Last &last)
{
    constexpr CRadices rl = c_factorize(NP);
    constexpr int T = c_fft_threads(NP);
    static_assert(rl.n > 0 && fft_padded(NP), "compile-time transforms take 7-smooth lengths up to 12288");
    if constexpr (P < rl.n) {
        constexpr int R = rl.r[P];
        constexpr bool pout = P + 1 < rl.n;
        if constexpr (P == 0 && P + 1 == rl.n) {
            cfft_pass<NP, T, R, NS>(first, last.template at<R, NS>());
        } else if constexpr (P == 0) {
            cfft_pass<NP, T, R, NS>(first, CSmemOut<NP, R, NS, pout>{b});
        } else if constexpr (P + 1 == rl.n) {
            cfft_pass<NP, T, R, NS>(CSmemIn<NP, T, R, true>(a), last.template at<R, NS>());
        } else {
            cfft_pass<NP, T, R, NS>(CSmemIn<NP, T, R, true>(a), CSmemOut<NP, R, NS, pout>{b});
        }
        if constexpr (P + 1 < rl.n) {
            __syncthreads();
            cfft_passes<NP, P + 1, NS * R>(b, a, first, last);
        }
    }
}
// Buffer (0: a, 1: b) the last pass of an NP-point cfft_passes from a writes.
template <int NP>
__host__ __device__ constexpr int cfft_out_buffer() { return c_factorize(NP).n % 2 == 1 ? 1 : 0; }

// Plain-order shared-memory output of the last pass (NS R = NP: q = 0).
template <int R, int NS>
struct CPlainOut {
    float2 *d;
    __device__ __forceinline__ void operator()(int q, int k, const float2 (&v)[R]) const
    {
        (void)q;
#pragma unroll
        for (int r = 0; r < R; r++) d[k + r * NS] = v[r];
    }
};
struct CPlainLast {
    float2 *d;
    template <int R, int NS> __device__ __forceinline__ CPlainOut<R, NS> at() const { return {d}; }
};

// fft_forward for a compile-time length with blockDim.x == c_fft_threads(NP):
// the NP values in a (plain order) are transformed, the result (plain order)
// is left in the returned buffer, a or b, after a barrier.
template <int NP>
__device__ __forceinline__ float2 *cfft_smem(float2 *a, float2 *b)
{
    constexpr CRadices rl = c_factorize(NP);
    float2 *out = cfft_out_buffer<NP>() ? b : a;
    cfft_passes<NP, 0, 1>(a, b, CSmemIn<NP, c_fft_threads(NP), rl.r[0], false>(a), CPlainLast{out});
    __syncthreads();
    return out;
}

// ------------------------------------------------------- any length --
// A forward DFT of any length n held in shared memory: directly when n has
// only the prime factors 2, 3, 5, 7, otherwise by Bluestein's chirp-z
// algorithm (L. Bluestein, "A linear filtering approach to the computation of
// the discrete Fourier transform", 1970): with w_j = exp(-i pi j^2 / n),
//   X_k = w_k sum_j (x_j w_j) conj(w_(k-j)),
// a circular convolution of length M >= 2n - 1 (M 7-smooth) computed with two
// M-point transforms and the precomputed transform of the chirp.
struct FftPlan {
    int n = 0, M = 0;                 // M == n: direct transform
    RadixList rl{};                   // radices of M
    const float2 *chirp = nullptr;    // w_j, j < n                     (Bluestein)
    const float2 *B = nullptr;        // FFT_M(c) / M, c_m = conj(w_|m|)  (Bluestein)
};
// Elements each of the two shared-memory buffers of a transform needs.
__host__ __device__ inline int fft_plan_span(const FftPlan &P) { return fft_span(P.M); }

// Forward DFT of a[0..n) (plain order) with a, b holding fft_plan_span(P)
// elements each; returns the buffer holding the n results (plain order).
__device__ __forceinline__ float2 *fft_run(float2 *a, float2 *b, const FftPlan &P)
{
    if (P.M == P.n) return fft_forward(a, b, P.n, P.rl, nullptr);
    const int n = P.n, M = P.M;
    for (int j = threadIdx.x; j < M; j += blockDim.x)
        a[j] = j < n ? cmul(a[j], __ldg(&P.chirp[j])) : make_float2(0.f, 0.f);
    __syncthreads();
    float2 *r = fft_forward(a, b, M, P.rl, nullptr);
    for (int k = threadIdx.x; k < M; k += blockDim.x) {
        const float2 g = cmul(r[k], __ldg(&P.B[k]));
        r[k] = make_float2(g.x, -g.y);
    }
    __syncthreads();
    // FFT(conj(FFT(a) B)) = conj of the circular convolution (B carries 1/M)
    float2 *o = (r == a) ? b : a;
    float2 *r2 = fft_forward(r, o, M, P.rl, nullptr);
    for (int k = threadIdx.x; k < n; k += blockDim.x)
        r2[k] = cmul(make_float2(r2[k].x, -r2[k].y), __ldg(&P.chirp[k]));
    __syncthreads();
    return r2;
}

// Device twiddles and radix list of one length, cached per (device, n) for
// the life of the process (defined in bst.cu); lengths with a prime factor
// above 7 carry the Bluestein tables.
struct FftTable {
    RadixList rl;                     // radices of n (direct lengths)
    float2 *tw = nullptr;
    FftPlan plan;                     // any length
    float2 *chirp = nullptr, *B = nullptr;
    ~FftTable();
};
const FftTable &fft_table(int device, int n);
// Transform length the plan of n runs (n, or Bluestein's M); 0 if none fits 24 passes.
int fft_plan_length(int n);

}  // namespace raft
