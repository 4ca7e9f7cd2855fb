// unet_tc.cu -- the U-Net's 3x3 convolution on the 5th-generation tensor
// cores (tcgen05.mma, accumulators in tensor memory), operands staged by TMA.
//
// Implicit GEMM: D[pixel][co] = sum over (tap, ci) of X[pixel + tap][ci] * W[co][tap][ci].
// One tile = MT x 128 output pixels (BW consecutive pixels of BH image rows,
// BW = 256 / 128 / W) x BN output channels.  Per k-block (one tap, KC input
// channels) the producer issues two TMA loads into a pipeline stage:
//   A: box (KC channels, BW pixels, BH rows) of the NHWC input at
//      (c0, x0 + kx, y0 + ky, n) -- the 3x3 halo outside the image arrives as
//      zeros from the TMA unit's out-of-bounds fill, no padded copy exists;
//   B: box (KC, BN) of the weights viewed as [Cout][9 Cin].
// Both land 128-byte (KC = 64) or 64-byte (KC = 32) swizzled, the K-major
// layout the MMA's shared-memory descriptors describe.  One thread issues
// MT x KC/16 tcgen05.mma (M = 128, N = BN, K = 16, BF16 x BF16 -> FP32) per
// k-block into MT TMEM accumulators and commits the stage back to the producer
// (MT > 1 spreads the fixed cost of a pipeline step -- the barrier handoffs
// and issue of one k-block, about 0.3 us -- over more tensor-core work);
// the accumulator is double-buffered in TMEM so the epilogue of one tile
// (tcgen05.ld, bias, ReLU, BF16, NHWC store, optional split of the output
// channels into two tensors) overlaps the MMAs of the next.  CTAs are
// persistent over the tiles.
//
// Warp roles (192 threads): warp 0 = TMA producer, warp 1 = TMEM owner and
// MMA issuer, warps 2-5 = epilogue (warp w reads TMEM lanes 32 (w mod 4) ..).
// Every mbarrier wait is bounded; a wait that runs out sets the CTA's abort
// flag and the library's error flag, every role then leaves its loop, the
// MMA issuer drains its outstanding MMAs (bounded) and TMEM is released.
// No cluster launch and no multicast: every TMA load reads this GPU's memory
// into this CTA's shared memory.
#include "raft.hpp"
#include "profile.hpp"
#include "ptx.hpp"

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

namespace raft {

namespace {

typedef __nv_bfloat16 bf16;

constexpr int TC_M = 128;                 // output pixels per tile (MMA M)
constexpr int TC_THREADS = 192;
constexpr uint32_t TC_WAIT_LIMIT = 1u << 20;   // polls of try_wait (at least ~0.1 s)

struct TcArgs {
    bf16 *y, *y1;          // outputs (see raft_unet_conv_fwd)
    int Cy0;
    const float *bias;     // [Cout] or null
    int N, H, W, Cout, C0, C1;
    int BW, BH, n_xb, n_yb, n_co, tiles;
    int relu;
    int *err;              // library error flag (set on a wait that runs out)
};

// --------------------------------------------------------------- tcgen05
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// arrive on `bar` once every tcgen05.mma issued so far by this thread has completed
__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// D[tmem] (+)= A[smem desc] * B[smem desc]^T, kind::f16 (BF16 in, FP32 accumulate)
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// 32 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor, K-major, swizzled rows: start address,
// leading offset 16 B (unused for swizzled K-major), stride offset = one
// 8-row swizzle atom, descriptor version 1, layout (2 = 128 B, 4 = 64 B swizzle).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t sbo_bytes, uint32_t layout)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)layout << 61);
}

// Halo tiles (the level-0 layers: 32 channels in, 32 out, W >= 128): one tile =
// 4 rows x 128 pixels (MT = 4 MMA blocks); a k-block is one 32-channel chunk
// with all nine taps.  The input arrives once per k-block as one (4+2) x 136
// pixel halo box (64-byte swizzled rows), so a tap's 128-row operand starts
// at row (mt + ky + 1) * 136 + kx + 1 of it: a descriptor offset, no reload.
// The MMA applies the swizzle to absolute shared-memory addresses, as the TMA
// unit does (base offset 0 at any row; checked against the oracle).
constexpr int HB_W = 136, HB_H = 6, HB_ROWS = HB_W * HB_H;

// ------------------------------------------------------------------- TMA
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait that also gives up when another role has aborted.
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *err)
{
    for (uint32_t it = 0; it < TC_WAIT_LIMIT; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255) == 255 && *abort_flag) return false;
    }
    *abort_flag = 1;
    if (err) atomicExch(err, 1);
    return false;
}

struct TileCoord {
    int n, y0, x0, co0;
};

__device__ __forceinline__ TileCoord tile_coord(const TcArgs &a, int t, int BN)
{
    TileCoord c;
    const int cot = t % a.n_co;
    int r = t / a.n_co;
    const int xb = r % a.n_xb;
    r /= a.n_xb;
    const int yb = r % a.n_yb;
    c.n = r / a.n_yb;
    c.y0 = yb * a.BH;
    c.x0 = xb * a.BW;
    c.co0 = cot * BN;
    return c;
}

template <int BN, int KC, int MT, int ST, bool HALO = false>
__global__ void __launch_bounds__(TC_THREADS, 1)
    conv3x3_tc_kernel(const __grid_constant__ CUtensorMap mx0, const __grid_constant__ CUtensorMap mx1,
                      const __grid_constant__ CUtensorMap mw, const TcArgs a)
{
    static_assert(!HALO || (BN == 32 && KC == 32 && MT == 4), "halo tiles: 32 -> 32 channels, 4 MMA blocks");
    constexpr int A_PART = TC_M * KC * 2;                  // one 128-row MMA operand
    constexpr int B_TAP = BN * KC * 2;                     // one tap's weights
    constexpr int A_BYTES = HALO ? HB_ROWS * KC * 2 : MT * A_PART;
    // halo tiles keep every tap's weights resident (loaded once per CTA); the
    // stages carry the input boxes only
    constexpr int B_BYTES = HALO ? 0 : B_TAP, STAGE = A_BYTES + B_BYTES;
    constexpr uint32_t SBO = 8 * KC * 2;                   // one 8-row swizzle atom
    constexpr uint32_t LAYOUT = KC == 64 ? 2u : 4u;        // 128-byte / 64-byte swizzle
    constexpr uint32_t ACC = MT * BN;                      // TMEM columns of one accumulator buffer
    constexpr uint32_t TMEM_COLS = 2 * ACC < 32 ? 32 : 2 * ACC;
    static_assert(2 * ACC <= 512, "two accumulator buffers must fit in TMEM");
    // lanes of the MMA warp that issue: halo tiles issue their MT blocks from MT
    // lanes at once (one warp instruction, MT MMAs); each issuing lane commits
    constexpr int NISSUE = HALO ? MT : 1;
    static_assert(STAGE % 1024 == 0, "stages must keep 1024-byte alignment");
    static_assert(BN % 32 == 0 && BN <= 256 && (KC == 32 || KC == 64), "tile shape");
    // instruction descriptor: D F32, A/B BF16, both K-major, N = BN, M = 128
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(TC_M >> 4) << 24);

    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int wres_bytes = HALO ? 9 * ((a.C0 + a.C1) / KC) * B_TAP : 0;   // resident weights (halo tiles)
    uint8_t *wres = base + ST * STAGE;
    uint64_t *full = reinterpret_cast<uint64_t *>(wres + wres_bytes);
    uint64_t *empty = full + ST;
    uint64_t *accf = empty + ST;
    uint64_t *acce = accf + 2;
    uint64_t *drain = acce + 2;
    uint64_t *wbar = drain + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(wbar + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NISSUE);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], NISSUE);
            mbar_init(&acce[b], 128);
        }
        mbar_init(drain, NISSUE);
        mbar_init(wbar, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int Cin = a.C0 + a.C1;
    const int kb_per_tile = HALO ? Cin / KC : 9 * (Cin / KC);

    if (warp == 0) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            uint32_t g = 0;                      // k-blocks issued so far
            bool ok = true;
            if constexpr (HALO) {
                // every chunk's nine taps of weights, once per CTA
                mbar_arrive_expect_tx(wbar, (uint32_t)wres_bytes);
#pragma unroll 1
                for (int ck = 0; ck < Cin / KC; ++ck)
#pragma unroll 1
                    for (int tap = 0; tap < 9; ++tap)
                        tma_load_2d(wres + (ck * 9 + tap) * B_TAP, &mw, tap * Cin + ck * KC, 0, wbar);
            }
            for (int t = blockIdx.x; t < a.tiles && ok; t += gridDim.x) {
                const TileCoord c = tile_coord(a, t, BN);
                for (int kb = 0; kb < kb_per_tile && ok; ++kb, ++g) {
                    const int s = (int)(g % ST);
                    const uint32_t u = g / ST;
                    if (u >= 1 && !(ok = tc_wait(&empty[s], (u - 1) & 1, abort_flag, a.err))) break;
                    uint8_t *st = base + s * STAGE;
                    mbar_arrive_expect_tx(&full[s], STAGE);
                    if constexpr (HALO) {
                        // the halo box of one 32-channel chunk
                        const int cc = kb * KC;
                        const CUtensorMap *mx = cc < a.C0 ? &mx0 : &mx1;
                        const int ch = cc < a.C0 ? cc : cc - a.C0;
                        tma_load_4d(st, mx, ch, c.x0 - 1, c.y0 - 1, c.n, &full[s]);
                    } else {
                        const int tap = kb / (Cin / KC), cc = (kb % (Cin / KC)) * KC;
                        const int ky = tap / 3 - 1, kx = tap % 3 - 1;
                        if (cc < a.C0) tma_load_4d(st, &mx0, cc, c.x0 + kx, c.y0 + ky, c.n, &full[s]);
                        else tma_load_4d(st, &mx1, cc - a.C0, c.x0 + kx, c.y0 + ky, c.n, &full[s]);
                        tma_load_2d(st + A_BYTES, &mw, tap * Cin + cc, c.co0, &full[s]);
                    }
                }
            }
            // every issued load lands before the CTA may exit: the last use of
            // stage s was k-block s + ST * ((g - 1 - s) / ST)
            for (uint32_t s = 0; s < (uint32_t)ST && s < g; ++s)
                mbar_wait_bounded(&full[s], ((g - 1 - s) / ST) & 1, TC_WAIT_LIMIT);
            if (HALO) mbar_wait_bounded(wbar, 0, TC_WAIT_LIMIT);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------------- MMA issuer
        if (lane < NISSUE) {
            uint32_t g = 0;
            bool ok = !HALO || tc_wait(wbar, 0, abort_flag, a.err);
            int i = 0;
            for (int t = blockIdx.x; t < a.tiles && ok; t += gridDim.x, ++i) {
                const int buf = i & 1, v = i >> 1;
                if (v >= 1 && !(ok = tc_wait(&acce[buf], (v - 1) & 1, abort_flag, a.err))) break;
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)buf * ACC;
                for (int kb = 0; kb < kb_per_tile; ++kb, ++g) {
                    const int s = (int)(g % ST);
                    const uint32_t u = g / ST;
                    if (!(ok = tc_wait(&full[s], u & 1, abort_flag, a.err))) break;
                    tc_fence_after();
                    const uint32_t sa = smem_u32(base + s * STAGE);
                    if constexpr (HALO) {
                        // this lane's MMA block: output row mt = lane of the tile
                        const int mt = lane;
                        const uint64_t bd0 = umma_desc(smem_u32(wres) + (uint32_t)(kb * 9 * B_TAP), SBO, LAYOUT);
                        const uint64_t ad0 = umma_desc(sa + (uint32_t)(mt * HB_W) * (KC * 2), SBO, LAYOUT);
#pragma unroll
                        for (int tap = 0; tap < 9; ++tap) {
                            const int ky = tap / 3, kx = tap % 3;          // offsets + 1
                            // descriptor start fields count 16-byte units
                            const uint64_t bd = bd0 + (uint64_t)(tap * B_TAP / 16);
                            const uint64_t ad = ad0 + (uint64_t)((ky * HB_W + kx) * (KC * 2) / 16);
#pragma unroll
                            for (int j = 0; j < KC / 16; ++j)
                                tc_mma(d + mt * BN, ad + (uint64_t)(2 * j), bd + (uint64_t)(2 * j), IDESC,
                                       (kb | tap | j) != 0);
                        }
                    } else {
                        const uint64_t bd = umma_desc(sa + A_BYTES, SBO, LAYOUT);
#pragma unroll
                        for (int mt = 0; mt < MT; ++mt) {
                            const uint64_t ad = umma_desc(sa + mt * A_PART, SBO, LAYOUT);
#pragma unroll
                            for (int j = 0; j < KC / 16; ++j)   // K = 16 per MMA: 32 bytes further along the swizzled row
                                tc_mma(d + mt * BN, ad + (uint64_t)(2 * j), bd + (uint64_t)(2 * j), IDESC,
                                       (kb | j) != 0);
                        }
                    }
                    tc_commit(&empty[s]);
                }
                if (ok) tc_commit(&accf[buf]);
            }
            // all MMAs issued by the issuing lanes complete before TMEM is released
            tc_commit(drain);
            mbar_wait_bounded(drain, 0, TC_WAIT_LIMIT);
        }
        __syncwarp();
    } else {
        // --------------------------------------------------------- epilogue
        const int q = warp & 3;                 // TMEM lane quarter of this warp
        int i = 0;
        for (int t = blockIdx.x; t < a.tiles; t += gridDim.x, ++i) {
            const int buf = i & 1, v = i >> 1;
            if (!tc_wait(&accf[buf], v & 1, abort_flag, a.err)) break;
            tc_fence_after();
            const TileCoord c = tile_coord(a, t, BN);
#pragma unroll 1
            for (int part = 0; part < MT * (BN / 32); ++part) {
                const int mt = part / (BN / 32), ch = part % (BN / 32);
                const int m = TC_M * mt + 32 * q + lane;        // tile pixel of this thread
                const int yy = c.y0 + m / a.BW, xx = c.x0 + m % a.BW;
                const bool valid = yy < a.H && xx < a.W;
                const size_t pix = ((size_t)c.n * a.H + yy) * a.W + xx;
                uint32_t r[32];
                tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)buf * ACC + (uint32_t)(mt * BN + 32 * ch), r);
                const int co = c.co0 + 32 * ch;
                if (!valid) continue;
                float f[32];
#pragma unroll
                for (int e = 0; e < 32; ++e) f[e] = __uint_as_float(r[e]);
                if (a.bias) {
#pragma unroll
                    for (int e = 0; e < 32; ++e) f[e] += __ldg(a.bias + co + e);
                }
                if (a.relu) {
#pragma unroll
                    for (int e = 0; e < 32; ++e) f[e] = fmaxf(f[e], 0.f);
                }
                bf16 *dst;
                if (a.y1 && co >= a.Cy0) dst = a.y1 + pix * (a.Cout - a.Cy0) + (co - a.Cy0);
                else if (a.y1) dst = a.y + pix * a.Cy0 + co;
                else dst = a.y + pix * a.Cout + co;
#pragma unroll
                for (int e = 0; e < 32; e += 8) {
                    __nv_bfloat162 h0 = __floats2bfloat162_rn(f[e], f[e + 1]);
                    __nv_bfloat162 h1 = __floats2bfloat162_rn(f[e + 2], f[e + 3]);
                    __nv_bfloat162 h2 = __floats2bfloat162_rn(f[e + 4], f[e + 5]);
                    __nv_bfloat162 h3 = __floats2bfloat162_rn(f[e + 6], f[e + 7]);
                    uint4 pk;
                    pk.x = *reinterpret_cast<uint32_t *>(&h0);
                    pk.y = *reinterpret_cast<uint32_t *>(&h1);
                    pk.z = *reinterpret_cast<uint32_t *>(&h2);
                    pk.w = *reinterpret_cast<uint32_t *>(&h3);
                    *reinterpret_cast<uint4 *>(dst + e) = pk;
                }
            }
            tc_fence_before();
            mbar_arrive(&acce[buf]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

// ------------------------------------------------------------------ host
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

int *tc_err_flag(int device)
{
    static std::mutex mu;
    static int *flags[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64) return nullptr;
    if (!flags[device]) {
        if (cudaMalloc(&flags[device], sizeof(int)) != cudaSuccess) return nullptr;
        cudaMemset(flags[device], 0, sizeof(int));
    }
    return flags[device];
}

// pipeline depth: as many stages as fit in 196 KB, at most 16 (the loads in
// flight are what hides the L2 latency of the per-tap operand tiles)
// 128-pixel MMA blocks per tile: two accumulator buffers of MT x BN columns
// within TMEM's 512, an A operand of at most 32 KB
template <int BN, int KC>
constexpr int tc_mt()
{
    return (256 / BN < 4 ? 256 / BN : 4) < 32768 / (TC_M * KC * 2) ? (256 / BN < 4 ? 256 / BN : 4)
                                                                   : 32768 / (TC_M * KC * 2);
}

template <int BN, int KC>
constexpr int tc_stage_bytes()
{
    return tc_mt<BN, KC>() * TC_M * KC * 2 + BN * KC * 2;
}

template <int BN, int KC>
constexpr int tc_stages()
{
    return (196 * 1024) / tc_stage_bytes<BN, KC>() > 16 ? 16 : (196 * 1024) / tc_stage_bytes<BN, KC>();
}

template <int BN, int KC>
int launch_tc(const CUtensorMap &m0, const CUtensorMap &m1, const CUtensorMap &mw, const TcArgs &a,
              cudaStream_t st)
{
    constexpr int MT = tc_mt<BN, KC>(), ST = tc_stages<BN, KC>();
    constexpr size_t SMEM = (size_t)ST * tc_stage_bytes<BN, KC>() + 1024 + 256;
    auto kern = conv3x3_tc_kernel<BN, KC, MT, ST>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM) != cudaSuccess) return 1;
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, TC_THREADS, SMEM) != cudaSuccess || occ < 1)
        occ = 1;
    const int grid = std::max(1, std::min(a.tiles, sms * occ));
    count_launch();
    kern<<<grid, TC_THREADS, SMEM, st>>>(m0, m1, mw, a);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

bool encode_act(CUtensorMap *m, const void *ptr, int C, int N, int H, int W, int KC, int BW, int BH)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {(cuuint32_t)KC, (cuuint32_t)BW, (cuuint32_t)BH, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(ptr), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, KC == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// halo-tile instance: 32 -> 32 channels, two stages of one halo box and nine weight boxes
int launch_tc_halo(const CUtensorMap &m0, const CUtensorMap &m1, const CUtensorMap &mw, const TcArgs &a,
                   cudaStream_t st)
{
    constexpr int STAGE = HB_ROWS * 32 * 2, ST = 3;
    static_assert(STAGE % 1024 == 0, "stage alignment");
    const size_t SMEM = (size_t)ST * STAGE + (size_t)9 * ((a.C0 + a.C1) / 32) * 32 * 32 * 2 + 1024 + 256;
    auto kern = conv3x3_tc_kernel<32, 32, 4, ST, true>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM) != cudaSuccess) return 1;
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, TC_THREADS, SMEM) != cudaSuccess || occ < 1)
        occ = 1;
    const int grid = std::max(1, std::min(a.tiles, sms * occ));
    count_launch();
    kern<<<grid, TC_THREADS, SMEM, st>>>(m0, m1, mw, a);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

bool encode_w(CUtensorMap *m, const void *ptr, int Cout, int Cin, int KC, int BN)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)9 * Cin, (cuuint64_t)Cout};
    cuuint64_t strides[1] = {(cuuint64_t)9 * Cin * 2};
    cuuint32_t box[2] = {(cuuint32_t)KC, (cuuint32_t)BN};
    cuuint32_t es[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, KC == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool g_halo = true;   // halo tiles for the 32 -> 32 channel layers (raft_unet_set_conv_halo)
bool g_wgrad_nine = true;   // nine-tap weight-gradient CTAs where Cout <= 128 (raft_unet_set_wgrad_nine)

// =========================================================== weight gradient
// dW[co][tap][ci] = sum over pixels p of dY[p][co] * X[p + tap][ci] as a GEMM
// D[(tap, ci)][co] with K = pixels, on tcgen05 (M = 128 rows of (tap, ci),
// N = Cout, K = 16, BF16 x BF16 -> FP32 in TMEM).  Both operands are NHWC
// tensors whose contiguous dimension is the channel, while the MMA wants K
// (the pixels) contiguous, so each k-block of 64 pixels (one image row
// segment) is transposed in shared memory:
//   * TMA lands four 32-channel input boxes (one (tap, channel chunk) each,
//     the 3x3 shift and the border from the box coordinates and the TMA
//     zero fill) and the dY box, with 64- or 128-byte swizzled rows;
//   * four warps move them into the K-major 128-byte-swizzled operand
//     layout with ldmatrix.trans (8x8 blocks out of the swizzled staging,
//     conflict-free) and stmatrix (rows into the operand's swizzled chunks),
//     then fence the generic-proxy writes for the tensor cores;
//   * one thread issues four MMAs per k-block into one TMEM accumulator.
// A CTA owns one 128-row block of D and a contiguous range of k-blocks; its
// accumulator goes to a per-CTA partial, and a second kernel adds the
// partials in a fixed order (deterministic; no atomics).  Warp roles as the
// forward kernel: 0 TMA, 1 TMEM/MMA, 2-5 transpose, then epilogue.  Every
// wait is bounded.
constexpr int WG_KB = 64;       // pixels per k-block
constexpr int WG_THREADS = 192;

struct WgTcArgs {
    int N, H, W, C0, C1, Cout;
    int nchunks;                // 9 * Cin / 32 rows blocks of 32
    int mtiles, splits;
    long long kblocks, kper;    // N * H * (W / 64) k-blocks, per split
    float *part;                // [splits][mtiles * 128][Cout]
    int *err;
};

__device__ __forceinline__ void ldsm_x4_trans(uint32_t addr, uint32_t (&r)[4])
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr)
                 : "memory");
}

__device__ __forceinline__ void stsm_x4(uint32_t addr, const uint32_t (&r)[4])
{
    asm volatile("stmatrix.sync.aligned.m8n8.x4.shared.b16 [%0], {%1,%2,%3,%4};" ::"r"(addr), "r"(r[0]), "r"(r[1]),
                 "r"(r[2]), "r"(r[3])
                 : "memory");
}

template <int BN, int ST>
__global__ void __launch_bounds__(WG_THREADS, 1)
    wgrad_tc_kernel(const __grid_constant__ CUtensorMap mx0, const __grid_constant__ CUtensorMap mx1,
                    const __grid_constant__ CUtensorMap mdy, const WgTcArgs a)
{
    constexpr int STG_A = 4 * WG_KB * 64;           // four [64 px][32 ch] boxes, 64-byte rows
    constexpr int STG_B = WG_KB * BN * 2;           // [64 px][BN ch]: one 64-byte-row box (BN 32) or
                                                    // BN/64 boxes of 128-byte rows
    constexpr int OP_A = 128 * 128, OP_B = BN * 128;
    constexpr int STAGE = STG_A + STG_B + OP_A + OP_B;
    static_assert(STAGE % 1024 == 0 && (BN == 32 || BN % 64 == 0) && BN <= 256, "stage layout");
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(TC_M >> 4) << 24);
    constexpr uint32_t TMEM_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;

    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + ST * STAGE);
    uint64_t *stg_empty = full + ST;
    uint64_t *opfull = stg_empty + ST;
    uint64_t *op_empty = opfull + ST;
    uint64_t *accf = op_empty + ST;
    uint64_t *drain = accf + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&stg_empty[s], 4);
            mbar_init(&opfull[s], 4);
            mbar_init(&op_empty[s], 1);
        }
        mbar_init(accf, 1);
        mbar_init(drain, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int mtile = (int)(blockIdx.x % (unsigned)a.mtiles), split = (int)(blockIdx.x / (unsigned)a.mtiles);
    const long long kb0 = (long long)split * a.kper;
    const long long kb1 = kb0 + a.kper < a.kblocks ? kb0 + a.kper : a.kblocks;
    const int nk = kb1 > kb0 ? (int)(kb1 - kb0) : 0;
    const int cpt = (a.C0 + a.C1) / 32;            // channel chunks per tap
    const int xbl = a.W / WG_KB;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA
        if (lane == 0) {
            int nvalid = 0;
            for (int c = 0; c < 4; ++c) nvalid += (mtile * 4 + c < a.nchunks) ? 1 : 0;
            const uint32_t bytes = (uint32_t)(nvalid * WG_KB * 64 + STG_B);
            bool ok = true;
            int g = 0;
            for (; g < nk && ok; ++g) {
                const int s = g % ST;
                const uint32_t u = (uint32_t)(g / ST);
                if (u >= 1 && !(ok = tc_wait(&stg_empty[s], (u - 1) & 1, abort_flag, a.err))) break;
                const long long kb = kb0 + g;
                const int xb = (int)(kb % xbl);
                const long long r = kb / xbl;
                const int y = (int)(r % a.H), n = (int)(r / a.H), x0 = xb * WG_KB;
                uint8_t *st = base + s * STAGE;
                mbar_arrive_expect_tx(&full[s], bytes);
                for (int c = 0; c < 4; ++c) {
                    const int q = mtile * 4 + c;
                    if (q >= a.nchunks) break;
                    const int tap = q / cpt, ch = (q % cpt) * 32;
                    const int ky = tap / 3 - 1, kx = tap % 3 - 1;
                    if (ch < a.C0) tma_load_4d(st + c * WG_KB * 64, &mx0, ch, x0 + kx, y + ky, n, &full[s]);
                    else tma_load_4d(st + c * WG_KB * 64, &mx1, ch - a.C0, x0 + kx, y + ky, n, &full[s]);
                }
                if (BN == 32) {
                    tma_load_4d(st + STG_A, &mdy, 0, x0, y, n, &full[s]);
                } else {
                    for (int b = 0; b < BN / 64; ++b)
                        tma_load_4d(st + STG_A + b * WG_KB * 128, &mdy, 64 * b, x0, y, n, &full[s]);
                }
            }
            // every issued load lands before the CTA may exit
            for (int s = 0; s < ST && s < g; ++s)
                mbar_wait_bounded(&full[s], (uint32_t)((g - 1 - s) / ST) & 1, TC_WAIT_LIMIT);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA
        if (lane == 0) {
            bool ok = true;
            for (int g = 0; g < nk && ok; ++g) {
                const int s = g % ST;
                const uint32_t u = (uint32_t)(g / ST);
                if (!(ok = tc_wait(&opfull[s], u & 1, abort_flag, a.err))) break;
                tc_fence_after();
                const uint32_t sa = smem_u32(base + s * STAGE + STG_A + STG_B);
                const uint64_t ad = umma_desc(sa, 1024, 2), bd = umma_desc(sa + OP_A, 1024, 2);
#pragma unroll
                for (int j = 0; j < WG_KB / 16; ++j)
                    tc_mma(tmem, ad + (uint64_t)(2 * j), bd + (uint64_t)(2 * j), IDESC, (g | j) != 0);
                tc_commit(&op_empty[s]);
            }
            if (ok) tc_commit(accf);
            tc_commit(drain);
            mbar_wait_bounded(drain, 0, TC_WAIT_LIMIT);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------- transpose, epilogue
        const int tw = warp - 2, j = lane >> 3, i = lane & 7;
        bool ok = true;
        for (int g = 0; g < nk && ok; ++g) {
            const int s = g % ST;
            const uint32_t u = (uint32_t)(g / ST);
            if (!(ok = tc_wait(&full[s], u & 1, abort_flag, a.err))) break;
            if (u >= 1 && !(ok = tc_wait(&op_empty[s], (u - 1) & 1, abort_flag, a.err))) break;
            uint8_t *st = base + s * STAGE;
            const uint32_t stgA = smem_u32(st), stgB = stgA + STG_A, opA = stgB + STG_B, opB = opA + OP_A;
            uint32_t r[4];
            // A: this warp's chunk (tw); its [64 px][32 ch] box has 64-byte rows,
            // 16-byte chunk k of row p at (k ^ ((p >> 1) & 3)).  Op k: pixels
            // 8k..8k+7, channel blocks 0..3 (matrix j = channel block j).
            if (mtile * 4 + tw < a.nchunks) {
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int px = 8 * k + i;
                    ldsm_x4_trans(stgA + tw * WG_KB * 64 + px * 64 + ((j ^ ((px >> 1) & 3)) << 4), r);
                    const int row = 32 * tw + 8 * j + i;       // (tap, ci) row of this matrix row
                    stsm_x4(opA + row * 128 + ((k ^ (row & 7)) << 4), r);
                }
            }
            // B: BN rows (output channels) x 64 px; op o: pixel block o % 8,
            // channel blocks 4 (o / 8) .. + 3
#pragma unroll 1
            for (int o = tw; o < BN / 4; o += 4) {
                const int pb = o & 7, cb = 4 * (o >> 3) + j, px = 8 * pb + i;
                uint32_t src;
                if (BN == 32) src = stgB + px * 64 + ((cb ^ ((px >> 1) & 3)) << 4);
                else src = stgB + (cb >> 3) * (WG_KB * 128) + px * 128 + (((cb & 7) ^ (px & 7)) << 4);
                ldsm_x4_trans(src, r);
                const int row = 8 * cb + i;
                stsm_x4(opB + row * 128 + ((pb ^ (row & 7)) << 4), r);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&stg_empty[s]);
                mbar_arrive(&opfull[s]);
            }
        }
        // epilogue: this warp's 32 TMEM lanes = 32 rows of the block
        if (ok && nk > 0 && tc_wait(accf, 0, abort_flag, a.err)) {
            tc_fence_after();
            const int q = warp & 3;
            const int row = mtile * 128 + 32 * q + lane;
            float *dst = a.part + ((size_t)split * a.mtiles * 128 + row) * BN;
            const bool valid = row < a.nchunks * 32;
#pragma unroll 1
            for (int c = 0; c < BN / 32; ++c) {
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * c), v);
                if (valid) {
#pragma unroll
                    for (int e = 0; e < 32; e += 4)
                        *reinterpret_cast<float4 *>(dst + 32 * c + e) =
                            make_float4(__uint_as_float(v[e]), __uint_as_float(v[e + 1]), __uint_as_float(v[e + 2]),
                                        __uint_as_float(v[e + 3]));
                }
            }
        } else if (nk == 0) {
            // an empty range still contributes its (zero) partial
            const int q = warp & 3;
            const int row = mtile * 128 + 32 * q + lane;
            float *dst = a.part + ((size_t)split * a.mtiles * 128 + row) * BN;
            if (row < a.nchunks * 32)
                for (int e = 0; e < BN; ++e) dst[e] = 0.f;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

// All nine taps per CTA (Cout <= 128): the CTA owns one 32-channel input chunk
// and all 288 (tap, channel) rows -- three M = 128 blocks, the third a quarter
// full -- so a k-block stages the input once as three 66-pixel row boxes
// (rows y-1..y+1, columns x0-1..x0+64, the TMA zero fill outside the image)
// and every tap's operand rows are transposed out of them at a column offset.
// The staging ring is deeper than the operand ring: the loads of several
// k-blocks are in flight while the tensor cores work through the operands.
constexpr int WG9_BOX = 66;                   // pixels per row box (64 + the two neighbours)
constexpr int WG9_BOXB = 4608;                // one box's slot: 66 x 64 bytes, 512-byte aligned

template <int BN>
__host__ __device__ constexpr int wg9_stg_bytes()
{
    return (3 * WG9_BOXB + WG_KB * BN * 2 + 1023) / 1024 * 1024;
}
template <int BN>
__host__ __device__ constexpr int wg9_op_bytes()
{
    return BN * 128 + 288 * 128;             // [opB | opA]; the third block reads 96 rows past opA
}
constexpr int WG9_SLACK = 96 * 128;

template <int BN, int STS, int STO>
__global__ void __launch_bounds__(WG_THREADS, 1)
    wgrad_tc9_kernel(const __grid_constant__ CUtensorMap mx0, const __grid_constant__ CUtensorMap mx1,
                     const __grid_constant__ CUtensorMap mdy, const WgTcArgs a)
{
    constexpr int STG = wg9_stg_bytes<BN>(), OPS = wg9_op_bytes<BN>();
    static_assert(OPS % 1024 == 0 && (BN == 32 || BN == 64 || BN == 128), "layout");
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(TC_M >> 4) << 24);
    constexpr uint32_t TMEM_COLS = 3 * BN <= 128 ? 128 : 3 * BN <= 256 ? 256 : 512;
    constexpr uint32_t TX = 3 * WG9_BOX * 64 + WG_KB * BN * 2;

    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint8_t *stg = base;                                   // STS staging slots
    uint8_t *ops = base + STS * STG;                       // STO operand slots (+ slack)
    uint64_t *full = reinterpret_cast<uint64_t *>(ops + STO * OPS + WG9_SLACK);
    uint64_t *sfree = full + STS;
    uint64_t *opfull = sfree + STS;
    uint64_t *opfree = opfull + STO;
    uint64_t *accf = opfree + STO;
    uint64_t *drain = accf + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&sfree[s], 4);
        }
        for (int s = 0; s < STO; ++s) {
            mbar_init(&opfull[s], 4);
            mbar_init(&opfree[s], 1);
        }
        mbar_init(accf, 1);
        mbar_init(drain, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int cchunks = (a.C0 + a.C1) / 32, Cin = a.C0 + a.C1;
    const int cc = (int)(blockIdx.x % (unsigned)cchunks), split = (int)(blockIdx.x / (unsigned)cchunks);
    const long long kb0 = (long long)split * a.kper;
    const long long kb1 = kb0 + a.kper < a.kblocks ? kb0 + a.kper : a.kblocks;
    const int nk = kb1 > kb0 ? (int)(kb1 - kb0) : 0;
    const int xbl = a.W / WG_KB;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA
        if (lane == 0) {
            const int ch = cc * 32;
            const CUtensorMap *mx = ch < a.C0 ? &mx0 : &mx1;
            const int chx = ch < a.C0 ? ch : ch - a.C0;
            bool ok = true;
            int g = 0;
            for (; g < nk && ok; ++g) {
                const int s = g % STS;
                const uint32_t u = (uint32_t)(g / STS);
                if (u >= 1 && !(ok = tc_wait(&sfree[s], (u - 1) & 1, abort_flag, a.err))) break;
                const long long kb = kb0 + g;
                const int xb = (int)(kb % xbl);
                const long long r = kb / xbl;
                const int y = (int)(r % a.H), n = (int)(r / a.H), x0 = xb * WG_KB;
                // slot: the dY box(es) first (1024-byte aligned, as the 128-byte
                // swizzle needs), then the three input row boxes (512-byte aligned)
                uint8_t *st = stg + s * STG;
                mbar_arrive_expect_tx(&full[s], TX);
                if (BN == 32) {
                    tma_load_4d(st, &mdy, 0, x0, y, n, &full[s]);
                } else {
                    for (int b = 0; b < BN / 64; ++b)
                        tma_load_4d(st + b * WG_KB * 128, &mdy, 64 * b, x0, y, n, &full[s]);
                }
                for (int ky = 0; ky < 3; ++ky)
                    tma_load_4d(st + WG_KB * BN * 2 + ky * WG9_BOXB, mx, chx, x0 - 1, y + ky - 1, n, &full[s]);
            }
            for (int s = 0; s < STS && s < g; ++s)
                mbar_wait_bounded(&full[s], (uint32_t)((g - 1 - s) / STS) & 1, TC_WAIT_LIMIT);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA
        if (lane == 0) {
            bool ok = true;
            for (int g = 0; g < nk && ok; ++g) {
                const int s = g % STO;
                const uint32_t u = (uint32_t)(g / STO);
                if (!(ok = tc_wait(&opfull[s], u & 1, abort_flag, a.err))) break;
                tc_fence_after();
                const uint32_t sb = smem_u32(ops + s * OPS), sa = sb + BN * 128;
                const uint64_t bd = umma_desc(sb, 1024, 2);
#pragma unroll
                for (int mb = 0; mb < 3; ++mb) {
                    const uint64_t ad = umma_desc(sa + (uint32_t)(mb * 128 * 128), 1024, 2);
#pragma unroll
                    for (int j = 0; j < WG_KB / 16; ++j)
                        tc_mma(tmem + (uint32_t)(mb * BN), ad + (uint64_t)(2 * j), bd + (uint64_t)(2 * j), IDESC,
                               (g | j) != 0);
                }
                tc_commit(&opfree[s]);
            }
            if (ok) tc_commit(accf);
            tc_commit(drain);
            mbar_wait_bounded(drain, 0, TC_WAIT_LIMIT);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------- transpose, epilogue
        const int tw = warp - 2, j = lane >> 3, i = lane & 7;
        bool ok = true;
        for (int g = 0; g < nk && ok; ++g) {
            const int ss = g % STS, so = g % STO;
            if (!(ok = tc_wait(&full[ss], (uint32_t)(g / STS) & 1, abort_flag, a.err))) break;
            if (g >= STO && !(ok = tc_wait(&opfree[so], (uint32_t)(g / STO - 1) & 1, abort_flag, a.err))) break;
            const uint32_t sy = smem_u32(stg + ss * STG), sx = sy + WG_KB * BN * 2;
            const uint32_t opB = smem_u32(ops + so * OPS), opA = opB + BN * 128;
            uint32_t r[4];
            // A: op o -> tap o / 8, pixels 8 (o % 8) ..; tap (ky, kx) reads box ky at
            // pixel offset kx (the box starts one pixel left of x0); 64-byte rows,
            // 16-byte chunk k of row p at (k ^ ((p >> 1) & 3))
#pragma unroll 2
            for (int o = tw; o < 72; o += 4) {
                const int tap = o >> 3, k = o & 7, ky = tap / 3, kx = tap - 3 * ky;
                const int p = 8 * k + i + kx;
                ldsm_x4_trans(sx + ky * WG9_BOXB + p * 64 + ((j ^ ((p >> 1) & 3)) << 4), r);
                const int row = 32 * tap + 8 * j + i;
                stsm_x4(opA + row * 128 + ((k ^ (row & 7)) << 4), r);
            }
#pragma unroll 1
            for (int o = tw; o < BN / 4; o += 4) {
                const int pb = o & 7, cb = 4 * (o >> 3) + j, px = 8 * pb + i;
                uint32_t src;
                if (BN == 32) src = sy + px * 64 + ((cb ^ ((px >> 1) & 3)) << 4);
                else src = sy + (cb >> 3) * (WG_KB * 128) + px * 128 + (((cb & 7) ^ (px & 7)) << 4);
                ldsm_x4_trans(src, r);
                const int row = 8 * cb + i;
                stsm_x4(opB + row * 128 + ((pb ^ (row & 7)) << 4), r);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&sfree[ss]);
                mbar_arrive(&opfull[so]);
            }
        }
        if (ok && nk > 0 && tc_wait(accf, 0, abort_flag, a.err)) {
            tc_fence_after();
            const int q = warp & 3;
#pragma unroll 1
            for (int mb = 0; mb < 3; ++mb) {
                const int row = mb * 128 + 32 * q + lane;      // tap * 32 + channel of the chunk
                const bool valid = row < 288;
                const int rg = (row >> 5) * Cin + cc * 32 + (row & 31);
                float *dst = a.part + ((size_t)split * 9 * Cin + (valid ? rg : 0)) * BN;
#pragma unroll 1
                for (int c = 0; c < BN / 32; ++c) {
                    uint32_t v[32];
                    tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(mb * BN + 32 * c), v);
                    if (valid) {
#pragma unroll
                        for (int e = 0; e < 32; e += 4)
                            *reinterpret_cast<float4 *>(dst + 32 * c + e) =
                                make_float4(__uint_as_float(v[e]), __uint_as_float(v[e + 1]),
                                            __uint_as_float(v[e + 2]), __uint_as_float(v[e + 3]));
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

template <int BN>
constexpr int wg9_stages_stg()
{
    return (int)((224 * 1024 - 2 * wg9_op_bytes<BN>() - WG9_SLACK - 1280) / wg9_stg_bytes<BN>()) > 8
               ? 8
               : (int)((224 * 1024 - 2 * wg9_op_bytes<BN>() - WG9_SLACK - 1280) / wg9_stg_bytes<BN>());
}

template <int BN>
int launch_wgrad_tc9(const CUtensorMap &m0, const CUtensorMap &m1, const CUtensorMap &mdy, const WgTcArgs &a,
                     int ctas, cudaStream_t st)
{
    constexpr int STO = 2, STS = wg9_stages_stg<BN>();
    static_assert(STS >= 2, "staging ring");
    constexpr size_t SMEM = (size_t)STS * wg9_stg_bytes<BN>() + (size_t)STO * wg9_op_bytes<BN>() + WG9_SLACK +
                            1024 + 256;
    static_assert(SMEM <= 227 * 1024, "shared memory");
    auto kern = wgrad_tc9_kernel<BN, STS, STO>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM) != cudaSuccess) return 1;
    count_launch();
    kern<<<ctas, WG_THREADS, SMEM, st>>>(m0, m1, mdy, a);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// dw[co][r] += sum over splits of part[split][r][co], r = tap * Cin + ci < rows
__global__ void wgrad_reduce_kernel(const float *__restrict__ part, float *__restrict__ dw, int splits, int rows,
                                    int prow, int Cout)
{
    const size_t n = (size_t)rows * Cout;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int co = (int)(e % Cout);
        const int r = (int)(e / Cout);
        float acc = 0.f;
        for (int sp = 0; sp < splits; ++sp) acc += part[((size_t)sp * prow + r) * Cout + co];
        dw[(size_t)co * rows + r] += acc;
    }
}

// dbias[co] += sum over pixels of dy[p][co], in a fixed order: per block a
// pixel range, each thread eight channels of one pixel lane (16-byte loads,
// lanes = 256 / (Cout / 8)), lanes summed in shared memory; then one block per
// channel sums the blocks' partials (a strided per-thread sum and a tree).
__global__ void __launch_bounds__(256)
bias_partial_kernel(const bf16 *__restrict__ dy, float *__restrict__ part, long long P, int Cout, long long per)
{
    __shared__ float red[256 * 8];
    const int g8 = Cout / 8, L = 256 / g8, c8 = threadIdx.x % g8, pl = threadIdx.x / g8;
    const long long p0 = (long long)blockIdx.x * per, p1 = p0 + per < P ? p0 + per : P;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (pl < L) {
        for (long long p = p0 + pl; p < p1; p += L) {
            const uint4 v = *reinterpret_cast<const uint4 *>(dy + p * Cout + 8 * c8);
            const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float2 f = __bfloat1622float2(h[q]);
                acc[2 * q] += f.x;
                acc[2 * q + 1] += f.y;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 8; q++) red[threadIdx.x * 8 + q] = acc[q];
    __syncthreads();
    if (threadIdx.x < Cout) {
        const int co = threadIdx.x, c = co / 8, q = co % 8;
        float sum = 0.f;
        for (int l = 0; l < L; ++l) sum += red[(l * g8 + c) * 8 + q];
        part[(size_t)blockIdx.x * Cout + co] = sum;
    }
}

__global__ void __launch_bounds__(256) bias_reduce_kernel(const float *__restrict__ part, float *__restrict__ dbias,
                                                          int nblk, int Cout)
{
    __shared__ float red[256];
    const int co = blockIdx.x;
    float acc = 0.f;
    for (int b = threadIdx.x; b < nblk; b += 256) acc += part[(size_t)b * Cout + co];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) dbias[co] += red[0];
}

template <int BN>
constexpr int wg_stages()
{
    return (196 * 1024) / (4 * WG_KB * 64 + WG_KB * BN * 2 + 128 * 128 + BN * 128) > 4
               ? 4
               : (196 * 1024) / (4 * WG_KB * 64 + WG_KB * BN * 2 + 128 * 128 + BN * 128);
}

template <int BN>
int launch_wgrad_tc(const CUtensorMap &m0, const CUtensorMap &m1, const CUtensorMap &mdy, const WgTcArgs &a,
                    cudaStream_t st)
{
    constexpr int ST = wg_stages<BN>();
    constexpr size_t SMEM =
        (size_t)ST * (4 * WG_KB * 64 + WG_KB * BN * 2 + 128 * 128 + BN * 128) + 1024 + 256;
    auto kern = wgrad_tc_kernel<BN, ST>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM) != cudaSuccess) return 1;
    count_launch();
    kern<<<a.mtiles * a.splits, WG_THREADS, SMEM, st>>>(m0, m1, mdy, a);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Tensor map of an NHWC activation for the weight gradient: boxes of
// (bc channels, 64 pixels, 1 row, 1 image), 64-byte (bc 32) or 128-byte (bc 64) swizzled rows.
bool encode_wg(CUtensorMap *m, const void *ptr, int C, int N, int H, int W, int bc, int bw = WG_KB)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    cuuint32_t box[4] = {(cuuint32_t)bc, (cuuint32_t)bw, 1, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(ptr), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, bc == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Grow-only per-device workspace of the weight gradient's partial sums.
float *wgrad_workspace(int device, size_t floats)
{
    static std::mutex mu;
    static float *buf[64] = {};
    static size_t cap[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64) return nullptr;
    if (cap[device] < floats) {
        if (buf[device]) cudaFree(buf[device]);
        buf[device] = nullptr;
        cap[device] = 0;
        if (cudaMalloc(&buf[device], floats * sizeof(float)) != cudaSuccess) return nullptr;
        cap[device] = floats;
    }
    return buf[device];
}

}  // namespace

void conv3x3_tc_set_halo(int on) { g_halo = on != 0; }
void conv3x3_wgrad_tc_set_nine(int on) { g_wgrad_nine = on != 0; }

bool conv3x3_tc_supported(int C0, int C1, int W)
{
    if (C0 % 32 || C1 % 32 || C0 <= 0) return false;
    if (W >= TC_M) return true;
    return W > 0 && TC_M % W == 0;
}

// 0 = launched, 1 = launch error, 2 = shape not handled here (caller uses the mma.sync kernel)
int conv3x3_tc(const void *x0, int C0, const void *x1, int C1, const void *w, const float *bias, void *y, void *y1,
               int Cy0, int N, int H, int W, int Cout, int relu, cudaStream_t st)
{
    if (!conv3x3_tc_supported(C0, C1, W) || Cout % 32 || Cout <= 0) return 2;
    const int KC = (C0 % 64 == 0 && C1 % 64 == 0) ? 64 : 32;
    const int BN = Cout % 256 == 0 ? 256 : Cout % 128 == 0 ? 128 : Cout % 64 == 0 ? 64 : 32;
    int MT = 1;
    switch (BN * 100 + KC) {
    case 25664: MT = tc_mt<256, 64>(); break;
    case 25632: MT = tc_mt<256, 32>(); break;
    case 12864: MT = tc_mt<128, 64>(); break;
    case 12832: MT = tc_mt<128, 32>(); break;
    case 6464: MT = tc_mt<64, 64>(); break;
    case 6432: MT = tc_mt<64, 32>(); break;
    case 3264: MT = tc_mt<32, 64>(); break;
    default: MT = tc_mt<32, 32>(); break;
    }
    TcArgs a;
    a.y = (bf16 *)y;
    a.y1 = (bf16 *)y1;
    a.Cy0 = Cy0;
    a.bias = bias;
    a.N = N;
    a.H = H;
    a.W = W;
    a.Cout = Cout;
    a.C0 = C0;
    a.C1 = C1;
    // box of MT x 128 pixels: 256-pixel row segments where the image is that
    // wide, else 128-pixel segments, else whole rows
    a.BW = (W >= 2 * TC_M && MT >= 2) ? 2 * TC_M : (W >= TC_M ? TC_M : W);
    a.BH = MT * TC_M / a.BW;
    a.n_xb = (W + a.BW - 1) / a.BW;
    a.n_yb = (H + a.BH - 1) / a.BH;
    a.n_co = Cout / BN;
    const long long tiles = (long long)N * a.n_yb * a.n_xb * a.n_co;
    if (tiles <= 0 || tiles > (1LL << 30)) return 2;
    a.tiles = (int)tiles;
    a.relu = relu;
    int dev = 0;
    cudaGetDevice(&dev);
    a.err = tc_err_flag(dev);
    CUtensorMap m0, m1, mw;
    if (g_halo && Cout == 32 && KC == 32 && W >= TC_M && C0 + C1 <= 96) {
        // halo tiles: 4 rows x 128 pixels, the taps served from one box per channel chunk
        TcArgs h = a;
        h.BW = TC_M;
        h.BH = 4;
        h.n_xb = (W + TC_M - 1) / TC_M;
        h.n_yb = (H + 3) / 4;
        h.n_co = 1;
        const long long ht = (long long)N * h.n_yb * h.n_xb;
        if (ht > 0 && ht <= (1LL << 30) && encode_act(&m0, x0, C0, N, H, W, 32, HB_W, HB_H) &&
            (C1 == 0 || encode_act(&m1, x1, C1, N, H, W, 32, HB_W, HB_H)) &&
            encode_w(&mw, w, Cout, C0 + C1, 32, 32)) {
            if (C1 == 0) m1 = m0;
            h.tiles = (int)ht;
            return launch_tc_halo(m0, m1, mw, h, st);
        }
    }
    if (!encode_act(&m0, x0, C0, N, H, W, KC, a.BW, a.BH)) return 2;
    if (C1 > 0) {
        if (!encode_act(&m1, x1, C1, N, H, W, KC, a.BW, a.BH)) return 2;
    } else {
        m1 = m0;
    }
    if (!encode_w(&mw, w, Cout, C0 + C1, KC, BN)) return 2;
    switch (BN * 100 + KC) {
    case 25664: return launch_tc<256, 64>(m0, m1, mw, a, st);
    case 25632: return launch_tc<256, 32>(m0, m1, mw, a, st);
    case 12864: return launch_tc<128, 64>(m0, m1, mw, a, st);
    case 12832: return launch_tc<128, 32>(m0, m1, mw, a, st);
    case 6464: return launch_tc<64, 64>(m0, m1, mw, a, st);
    case 6432: return launch_tc<64, 32>(m0, m1, mw, a, st);
    case 3264: return launch_tc<32, 64>(m0, m1, mw, a, st);
    default: return launch_tc<32, 32>(m0, m1, mw, a, st);
    }
}

// 0 = launched, 1 = launch error, 2 = shape not handled here (caller uses the mma.sync kernel)
int conv3x3_wgrad_tc(const void *dy, const void *x0, int C0, const void *x1, int C1, float *dw, float *dbias, int N,
                     int H, int W, int Cout, cudaStream_t st)
{
    if (C0 % 32 || C1 % 32 || C0 <= 0 || W % WG_KB || N < 1 || H < 1) return 2;
    if (!(Cout == 32 || Cout == 64 || Cout == 128 || Cout == 256)) return 2;
    const int Cin = C0 + C1;
    // Cout <= 128: all nine taps per CTA (one 32-channel input chunk, inputs
    // staged once per k-block); Cout = 256: 128-row blocks of (tap, channel)
    // (three accumulators of 256 columns would not fit TMEM)
    const bool nine = Cout <= 128 && g_wgrad_nine;
    WgTcArgs a;
    a.N = N;
    a.H = H;
    a.W = W;
    a.C0 = C0;
    a.C1 = C1;
    a.Cout = Cout;
    a.nchunks = 9 * Cin / 32;
    a.mtiles = (a.nchunks + 3) / 4;
    a.kblocks = (long long)N * H * (W / WG_KB);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // one CTA per SM over all work items (shared memory holds one), at least
    // 8 k-blocks each (nine-tap CTAs); two per SM for the row-block kernel
    const int items = nine ? Cin / 32 : a.mtiles;
    long long splits = std::max(1LL, ((nine ? 1LL : 2LL) * sms + items - 1) / items);
    splits = std::min(splits, std::max(1LL, a.kblocks / 8));
    a.kper = (a.kblocks + splits - 1) / splits;
    a.splits = (int)((a.kblocks + a.kper - 1) / a.kper);
    a.err = tc_err_flag(dev);
    const long long P = (long long)N * H * W;
    const int bias_blk = dbias ? (int)std::min<long long>(4 * sms, std::max(1LL, P / 256)) : 0;
    const int prow = nine ? 9 * Cin : a.mtiles * 128;
    const size_t part_floats = (size_t)a.splits * prow * Cout;
    float *ws = wgrad_workspace(dev, part_floats + (size_t)bias_blk * Cout);
    if (!ws) return 1;
    a.part = ws;
    CUtensorMap m0, m1, mdy;
    const int bw = nine ? WG9_BOX : WG_KB;
    if (!encode_wg(&m0, x0, C0, N, H, W, 32, bw)) return 2;
    if (C1 > 0) {
        if (!encode_wg(&m1, x1, C1, N, H, W, 32, bw)) return 2;
    } else {
        m1 = m0;
    }
    if (!encode_wg(&mdy, dy, Cout, N, H, W, Cout == 32 ? 32 : 64)) return 2;
    int rc;
    if (nine) {
        const int ctas = items * a.splits;
        switch (Cout) {
        case 32: rc = launch_wgrad_tc9<32>(m0, m1, mdy, a, ctas, st); break;
        case 64: rc = launch_wgrad_tc9<64>(m0, m1, mdy, a, ctas, st); break;
        default: rc = launch_wgrad_tc9<128>(m0, m1, mdy, a, ctas, st); break;
        }
    } else {
        switch (Cout) {
        case 32: rc = launch_wgrad_tc<32>(m0, m1, mdy, a, st); break;
        case 64: rc = launch_wgrad_tc<64>(m0, m1, mdy, a, st); break;
        case 128: rc = launch_wgrad_tc<128>(m0, m1, mdy, a, st); break;
        default: rc = launch_wgrad_tc<256>(m0, m1, mdy, a, st); break;
        }
    }
    if (rc) return rc;
    const int rows = 9 * Cin;
    count_launch();
    wgrad_reduce_kernel<<<(unsigned)std::min<size_t>(((size_t)rows * Cout + 255) / 256, 148 * 16), 256, 0, st>>>(
        a.part, dw, a.splits, rows, prow, Cout);
    if (cudaGetLastError() != cudaSuccess) return 1;
    if (dbias) {
        float *bp = ws + part_floats;
        const long long per = (P + bias_blk - 1) / bias_blk;
        count_launch();
        bias_partial_kernel<<<bias_blk, 256, 0, st>>>((const bf16 *)dy, bp, P, Cout, per);
        count_launch();
        bias_reduce_kernel<<<Cout, 256, 0, st>>>(bp, dbias, bias_blk, Cout);
        if (cudaGetLastError() != cudaSuccess) return 1;
    }
    return 0;
}

// Reads and clears the tensor-core convolution's error flag of the current device
// (1 = a bounded wait ran out).  Synchronises the device.
int conv3x3_tc_error()
{
    int dev = 0;
    cudaGetDevice(&dev);
    int *f = tc_err_flag(dev);
    if (!f) return 0;
    int h = 0;
    if (cudaMemcpy(&h, f, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    if (h) cudaMemset(f, 0, sizeof(int));
    return h;
}

}  // namespace raft
