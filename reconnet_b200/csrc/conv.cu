// BF16 3x3 convolutions of the learned prior on the 5th-generation tensor
// cores (tcgen05.mma, FP32 accumulators in tensor memory), with the input
// tiles brought in by TMA tensor copies from this GPU's own memory.
//
// The prior is a small residual CNN (5 layers of 3x3 convolutions, 32
// channels, ReLU; in 1 channel, out 1 channel plus the input).  It has no
// counterpart among the reference's kernels: the reference's learned use of
// the projectors goes through TensorFlow (python/ReconNet.py:773-830, the
// projector pair as differentiable ops) and its prior solvers are dictionary
// and low-rank methods (PriorFunctionSolver/omp.cu, NuclearNormSoftThresh.cu).
//
// Activation layout ("blocked"): bf16 [N][C/8][H][W][8] -- 16 bytes per pixel
// and channel chunk.  A TMA box of 3 image rows x (128 + 2) pixels x C/8
// chunks lands in shared memory as [chunk][row][pixel][8 channels]: 16-byte
// runs of 8 channels, consecutive pixels 16 bytes apart.  That is a canonical
// no-swizzle operand layout for the tensor core as it stands:
//   forward / input gradient, D[pixel][co] = sum_k A[pixel][k] B[co][k], A
//   K-major: for tap (dy, dx) and chunk c the 128 pixels of the tile are 128
//   consecutive 16-byte rows starting at pixel dx of row dy -- the im2col
//   matrix is read in place, with no copy;
//   weight gradient, D[co][(tap, ci)] = sum_p dY[p][co] X[p + tap][ci], both
//   operands MN-major: 8 pixels x 8 channels per 128-byte core matrix.
// Zero padding at the image border is the TMA's out-of-bounds fill.
//
// Descriptor bit layouts (instruction descriptor of kind::f16, shared-memory
// matrix descriptor version 1 for sm_100) follow the PTX ISA for tcgen05.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <type_traits>
#include <string>

#include "rn_device.cuh"
#include "rn_internal.h"

namespace rn {

constexpr int kConvThreads = 128;     // one warpgroup: the 128 accumulator lanes
constexpr int kConvTile = 128;        // output pixels per tile (MMA M)
constexpr int kBoxW = kConvTile + 2;  // pixels per box row (halo of one on each side)
constexpr int kZeroBytes = 2048;      // zero rows standing in for the tenth tap of an 8-channel layer

// ---- tcgen05 / TMA primitives ------------------------------------------------
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);   // version 1, no swizzle
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 D, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc(int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 32 consecutive FP32 columns: thread t of the warp gets lane (base lane + t).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint4 pack_bf16x8(const float* v) {
    uint4 o;
    uint32_t* w = reinterpret_cast<uint32_t*>(&o);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        w[i] = *reinterpret_cast<uint32_t*>(&h);
    }
    return o;
}
__device__ __forceinline__ void unpack_bf16x8(uint4 u, float* v) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
        float2 f = __bfloat1622float2(h);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

// Offset (bytes) in a box [CH][3][boxw][16 B] of tap t's first chunk for
// output pixel 0; tap 9 (the padding of an 8-channel layer) is the zero rows.
__device__ __forceinline__ uint32_t tap_off(int t, int ch, int boxw = kBoxW) {
    if (t >= 9) return (uint32_t)(ch * 3 * boxw * 16);
    return (uint32_t)(((t / 3) * boxw + (t % 3)) * 16);
}

// ---- forward / input-gradient convolution --------------------------------------
// mode 0: out bf16 blocked = relu(conv + bias); mode 1: out fp32 [N][H][W] =
// conv[0] + bias[0] + aux (the residual); mode 2: out bf16 blocked = conv *
// (aux > 0), aux the bf16 blocked activation (ReLU mask of the input
// gradient); mode 3: out fp32 [N][cout][H][W] = conv + bias (tests).
struct ConvArgs {
    void* out;
    const uint4* wpack;   // B operand image: [kchunks][NPAD][16 B]
    const float* bias;    // [cout] or null
    const void* aux;
    int N, H, W;
    int cout;             // real output channels (1 or multiple of 8)
    int mode;
    int* err;
};

// Warp-specialised pipeline.  Warp 4 (one elected lane) is the producer: it
// keeps kConvStages - 1 TMA boxes in flight ahead of the tile whose MMAs it
// issues, and commits each tile's MMA group twice, to the box's "empty"
// barrier (the box may be refilled) and to the accumulator's "full" barrier.
// Warps 0-3 are the epilogue: thread t reads TMEM lane t (output pixel w0 + t
// of the tile's row) from one of two accumulators of 32 columns, releases the
// accumulator (one arrival per warp on its "empty" barrier) and stores.  So
// the TMA copies, the MMAs of tile i and the epilogue of tile i - 1 overlap.
//
// Boxes: the tensor map views each image row as groups of PIX pixels (16 PIX
// bytes; PIX = 8 when the width allows, else 2, else 1), so a TMA row is a
// whole 128-byte line rather than half a 32-byte sector.  A box then starts
// PIX - 1 pixels before the halo pixel w0 - 1 (128 + 2 PIX pixels) and the
// operands start 16 (PIX - 1) bytes into each box row.
constexpr int kConvStages = 3;
constexpr int kConvWsThreads = kConvThreads + 32;

template <int CH, int NPAD, int PIX>
__global__ void __launch_bounds__(kConvWsThreads) conv3x3_kernel(const __grid_constant__ CUtensorMap tm_in, ConvArgs a) {
    constexpr int KSTEPS = CH == 4 ? 18 : 5;
    constexpr int KCH = 2 * KSTEPS;                              // B chunks (the last one of an 8-channel layer is zero)
    constexpr int BOXW = kConvTile + 2 * PIX;                    // pixels per box row
    constexpr uint32_t A0 = 16 * (PIX - 1);                      // the operands' first pixel within a box row
    constexpr uint32_t BOX_BYTES = CH * 3 * BOXW * 16;
    constexpr uint32_t BOX_ALLOC = (BOX_BYTES + kZeroBytes + 1023) & ~1023u;
    constexpr uint32_t B_BYTES = KCH * NPAD * 16;
    constexpr int S = kConvStages;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // TMA destinations on a 1024-byte boundary (the allocation has 1 KB of slack)
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    unsigned char* bsm = smem + S * BOX_ALLOC;
    __shared__ __align__(8) uint64_t bar_full[S], bar_empty[S], bar_accf[2], bar_acce[2];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int s_fail;
    __shared__ float s_bias[NPAD];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_w = (a.W + kConvTile - 1) / kConvTile;
    const long long ntiles = (long long)a.N * a.H * tiles_w;
    const long long nmine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    // zero rows, weights (B operand image), barriers, accumulator columns
    for (int s = 0; s < S; s++)
        for (int i = tid; i < kZeroBytes / 16; i += kConvWsThreads)
            reinterpret_cast<uint4*>(smem + s * BOX_ALLOC + BOX_BYTES)[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < (int)(B_BYTES / 16); i += kConvWsThreads) reinterpret_cast<uint4*>(bsm)[i] = a.wpack[i];
    if (tid < NPAD) s_bias[tid] = (a.bias && tid < a.cout) ? a.bias[tid] : 0.f;
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&bar_full[s], 1);
            mbar_init(&bar_empty[s], 1);
        }
        for (int k = 0; k < 2; k++) {
            mbar_init(&bar_accf[k], 1);
            mbar_init(&bar_acce[k], kConvThreads / 32);
        }
        fence_mbar_init();
        s_fail = 0;
    }
    if (warp == 0) tmem_alloc(&tmem_slot, 64);
    fence_proxy_async();   // generic-proxy writes (zero rows, weights) before tensor-core reads
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    auto tile_coords = [&](long long i, int& n, int& h, int& w0) {
        const long long t = blockIdx.x + i * gridDim.x;
        const int tw = (int)(t % tiles_w);
        const long long r = t / tiles_w;
        h = (int)(r % a.H);
        n = (int)(r / a.H);
        w0 = tw * kConvTile;
    };

    if (warp == kConvThreads / 32) {
        if (lane == 0) {
            // ---- producer ----
            long long tma_next = 0, full_seen = 0, mma_done = 0;   // TMA issued / consumed; MMA groups issued
            bool ok = true;
            auto issue_tma = [&](long long i) -> bool {
                const int s = (int)(i % S);
                if (i >= S && !mbar_wait(&bar_empty[s], (uint32_t)((i / S - 1) & 1))) return false;
                int n, h, w0;
                tile_coords(i, n, h, w0);
                mbar_arrive_expect_tx(&bar_full[s], BOX_BYTES);
                tma_load_5d(smem + s * BOX_ALLOC, &tm_in, 0, w0 / PIX - 1, h - 1, 0, n, &bar_full[s]);
                return true;
            };
            while (tma_next < nmine && tma_next < S - 1) issue_tma(tma_next++);
            const uint32_t idesc = umma_idesc(NPAD, false, false), bbase = smem_u32(bsm);
            for (long long j = 0; j < nmine; j++) {
                const int s = (int)(j % S), acc = (int)(j & 1);
                if (!mbar_wait(&bar_full[s], (uint32_t)((j / S) & 1))) { ok = false; break; }
                full_seen = j + 1;
                if (j >= 2 && !mbar_wait(&bar_acce[acc], (uint32_t)(((j >> 1) - 1) & 1))) { ok = false; break; }
                tc_fence_after();
                const uint32_t abase = smem_u32(smem + s * BOX_ALLOC) + A0;
#pragma unroll
                for (int k = 0; k < KSTEPS; k++) {
                    uint32_t aoff, lbo;
                    if (CH == 4) {
                        const int tap = k >> 1, c0 = (k & 1) * 2;
                        aoff = tap_off(tap, CH, BOXW) + (uint32_t)(c0 * 3 * BOXW * 16);
                        lbo = 3 * BOXW * 16;
                    } else {
                        // tap 9 is the zero rows after the box (from the
                        // operands' shifted start: the same offset minus A0)
                        aoff = tap_off(2 * k, CH, BOXW) - (2 * k >= 9 ? A0 : 0);
                        lbo = tap_off(2 * k + 1, CH, BOXW) - (2 * k + 1 >= 9 ? A0 : 0) - aoff;
                    }
                    const uint64_t da = umma_desc(abase + aoff, lbo, 128);
                    const uint64_t db = umma_desc(bbase + (uint32_t)(2 * k * NPAD * 16), NPAD * 16, 128);
                    umma_bf16(tmem + (uint32_t)(acc * 32), da, db, idesc, k > 0 ? 1u : 0u);
                }
                umma_commit(&bar_empty[s]);
                umma_commit(&bar_accf[acc]);
                mma_done = j + 1;
                // the box after the ones in flight goes into the stage that
                // tile j - 1's group is releasing
                if (tma_next < nmine) {
                    if (!issue_tma(tma_next)) { ok = false; break; }
                    tma_next++;
                }
            }
            if (!ok) {
                s_fail = 1;
                // before the shared memory and the accumulator columns are
                // released: the copies issued and not yet seen, and the last
                // MMA group (its barrier completes after every earlier group)
                for (long long i = full_seen; i < tma_next; i++)
                    mbar_wait(&bar_full[i % S], (uint32_t)((i / S) & 1));
                if (mma_done > 0)
                    mbar_wait(&bar_empty[(mma_done - 1) % S], (uint32_t)(((mma_done - 1) / S) & 1));
            }
        }
    } else {
        // ---- epilogue: thread tid owns output pixel w0 + tid ----
        for (long long j = 0; j < nmine; j++) {
            const int acc = (int)(j & 1);
            if (!mbar_wait(&bar_accf[acc], (uint32_t)((j >> 1) & 1))) {
                s_fail = 1;
                break;
            }
            tc_fence_after();
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(acc * 32), v);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar_acce[acc]);
            int n, h, w0;
            tile_coords(j, n, h, w0);
            const int w = w0 + tid;
            if (w < a.W) {
                const long long pix = ((long long)n * a.H + h) * a.W + w;   // pixel index within one channel plane
                const long long plane = (long long)a.H * a.W;
                if (a.mode == 0 || a.mode == 2) {
                    uint4* o = reinterpret_cast<uint4*>(a.out);
                    const uint4* act = reinterpret_cast<const uint4*>(a.aux);
                    const int cho = a.cout / 8;
#pragma unroll
                    for (int c = 0; c < NPAD / 8; c++) {
                        if (c >= cho) break;
                        float q[8];
#pragma unroll
                        for (int i = 0; i < 8; i++) q[i] = v[c * 8 + i];
                        const long long idx = ((long long)n * cho + c) * plane + (long long)h * a.W + w;
                        if (a.mode == 0) {
#pragma unroll
                            for (int i = 0; i < 8; i++) q[i] = fmaxf(q[i] + s_bias[c * 8 + i], 0.f);
                        } else {
                            float m[8];
                            unpack_bf16x8(act[idx], m);
#pragma unroll
                            for (int i = 0; i < 8; i++) q[i] = m[i] > 0.f ? q[i] : 0.f;
                        }
                        o[idx] = pack_bf16x8(q);
                    }
                } else if (a.mode == 1) {
                    const float* res = reinterpret_cast<const float*>(a.aux);
                    reinterpret_cast<float*>(a.out)[pix] = v[0] + s_bias[0] + res[pix];
                } else {
                    float* o = reinterpret_cast<float*>(a.out);
                    for (int c = 0; c < a.cout; c++)
                        o[((long long)n * a.cout + c) * plane + (long long)h * a.W + w] = v[c] + s_bias[c];
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (tid == 0 && s_fail) atomicExch(a.err, RN_ERR_TIMEOUT);
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, 64);
}

// ---- weight gradient -------------------------------------------------------------
// D[co][col] accumulates over the CTA's tiles; col = tap * 32 + ci (32-channel
// input) or pair * 16 + (tap & 1) * 8 + ci (8-channel input, taps in pairs),
// then 16 columns of sum_p dY[p][co] (the bias gradient).  Each CTA writes its
// partial [32][ncols] to `partial`; conv_wgrad_reduce sums them.
struct WgradArgs {
    float* partial;       // [gridDim.x][32][ncols]
    int N, H, W;
    int ncols;
    int* err;
};

// kWgStages - 1 tiles' loads (a dY box and an X box each) stay in flight
// ahead of the tile whose MMAs are issued; each tile's MMA groups commit to
// its stage's "empty" barriers, which the load kWgStages - 1 tiles later
// waits for.  Boxes take PIX pixels per TMA row as in the forward kernel.
// The A operand (dY, M = 128 output-channel rows of which the first 8 CHO are
// real) spans 16 groups of 8 rows 2048 bytes apart: groups past the dY box
// read whatever shared memory follows it (more boxes), which only feeds
// accumulator rows that are never read.
constexpr int kWgStages = 4;
constexpr int kWgIssuers = 2;   // MMA-issuing threads (lane 0 of warps 0 and 1)

template <int CH, int CHO, int PIX>
__global__ void __launch_bounds__(kConvThreads) conv3x3_wgrad_kernel(const __grid_constant__ CUtensorMap tm_x,
                                                                    const __grid_constant__ CUtensorMap tm_dy,
                                                                    WgradArgs a) {
    constexpr int S = kWgStages;
    constexpr int BOXW = kConvTile + 2 * PIX;
    constexpr uint32_t A0 = 16 * (PIX - 1);
    constexpr uint32_t XBOX = CH * 3 * BOXW * 16;
    constexpr uint32_t DYBOX = CHO * kConvTile * 16;
    constexpr uint32_t DY_ALLOC = (DYBOX + 1023) & ~1023u;
    constexpr uint32_t X_ALLOC = (XBOX + kZeroBytes + 1023) & ~1023u;
    constexpr int NCOLS_TMEM = CH == 4 ? 512 : 128;
    constexpr int BIAS_COL = CH == 4 ? 288 : 80;
    static_assert(DY_ALLOC + S * X_ALLOC >= 16 * 2048, "the A operand's 16 row groups must stay in shared memory");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    unsigned char* xbox0 = smem + S * DY_ALLOC;
    unsigned char* ones = xbox0 + S * X_ALLOC;   // 512 B of bf16 ones: the bias-gradient B operand
    __shared__ __align__(8) uint64_t bar_full[S], bar_empty[kWgIssuers][S];
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tiles_w = (a.W + kConvTile - 1) / kConvTile;
    const long long ntiles = (long long)a.N * a.H * tiles_w;
    const long long nmine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    for (int i = tid; i < (int)(S * DY_ALLOC / 16); i += kConvThreads) reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
    for (int s = 0; s < S; s++)
        for (int i = tid; i < kZeroBytes / 16; i += kConvThreads)
            reinterpret_cast<uint4*>(xbox0 + s * X_ALLOC + XBOX)[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < 512 / 4; i += kConvThreads) reinterpret_cast<uint32_t*>(ones)[i] = 0x3F803F80u;   // bf16 1.0 pairs
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&bar_full[s], 1);
            for (int q = 0; q < kWgIssuers; q++) mbar_init(&bar_empty[q][s], 1);
        }
        fence_mbar_init();
        s_fail = 0;
    }
    if (warp == 0) tmem_alloc(&tmem_slot, NCOLS_TMEM);
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    auto tile_coords = [&](long long i, int& n, int& h, int& w0) {
        const long long t = blockIdx.x + i * gridDim.x;
        const int tw = (int)(t % tiles_w);
        const long long r = t / tiles_w;
        h = (int)(r % a.H);
        n = (int)(r / a.H);
        w0 = tw * kConvTile;
    };
    // kWgIssuers issuers, lane 0 of warps 0, 1, .. (warp 0's also issues the
    // loads), split each K step's MMA slots (k < 9: tap k with 32 channels;
    // CH = 1: k < 5 a pair of taps; the last slot the bias columns) into
    // contiguous runs, one per issuer.  Each commits to its own "empty"
    // barrier of the stage; a stage is refilled once every issuer's group has
    // read it.  (Two issuers: 0.59 ms per 32-channel layer against 0.77 for
    // one; four, dealing slots round-robin, 0.71.)
    if ((tid & 31) == 0 && warp < kWgIssuers) {
        const int q = warp;
        long long tma_next = 0, full_seen = 0, mma_done = 0;
        bool ok = true;
        auto issue_loads = [&](long long i) -> bool {
            const int s = (int)(i % S);
            if (i >= S)
                for (int r = 0; r < kWgIssuers; r++)
                    if (!mbar_wait(&bar_empty[r][s], (uint32_t)((i / S - 1) & 1))) return false;
            int n, h, w0;
            tile_coords(i, n, h, w0);
            mbar_arrive_expect_tx(&bar_full[s], XBOX + DYBOX);
            tma_load_5d(smem + s * DY_ALLOC, &tm_dy, 0, w0 / PIX, h, 0, n, &bar_full[s]);
            tma_load_5d(xbox0 + s * X_ALLOC, &tm_x, 0, w0 / PIX - 1, h - 1, 0, n, &bar_full[s]);
            return true;
        };
        if (q == 0)
            while (tma_next < nmine && tma_next < S - 1) issue_loads(tma_next++);
        const uint32_t ob = smem_u32(ones);
        uint32_t accum = 0;
        for (long long j = 0; j < nmine; j++) {
            const int s = (int)(j % S);
            if (!mbar_wait(&bar_full[s], (uint32_t)((j / S) & 1))) { ok = false; break; }
            full_seen = j + 1;
            tc_fence_after();
            const uint32_t dyb = smem_u32(smem + s * DY_ALLOC), xb = smem_u32(xbox0 + s * X_ALLOC) + A0;
            for (int k0 = 0; k0 < kConvTile; k0 += 16) {
                const uint64_t da = umma_desc(dyb + (uint32_t)(k0 * 16), 128, kConvTile * 16);
                constexpr int NSLOT = CH == 4 ? 10 : 6;   // taps (or tap pairs), then the bias
#pragma unroll
                for (int k = 0; k < NSLOT; k++) {
                    constexpr int PER = (NSLOT + kWgIssuers - 1) / kWgIssuers;
                    if (k / PER != q) continue;
                    if (k == NSLOT - 1) {
                        const uint64_t dbo = umma_desc(ob, 128, 256);
                        umma_bf16(tmem + (uint32_t)BIAS_COL, da, dbo, umma_idesc(16, true, true), accum);
                    } else if (CH == 4) {
                        const uint64_t db = umma_desc(xb + tap_off(k, CH, BOXW) + (uint32_t)(k0 * 16), 128, 3 * BOXW * 16);
                        umma_bf16(tmem + (uint32_t)(k * 32), da, db, umma_idesc(32, true, true), accum);
                    } else {
                        // tap 9 is the zero rows after the box (the offset
                        // from the shifted start is the plain one minus A0)
                        const uint32_t o0 = tap_off(2 * k, CH, BOXW) - (2 * k >= 9 ? A0 : 0);
                        const uint32_t o1 = tap_off(2 * k + 1, CH, BOXW) - (2 * k + 1 >= 9 ? A0 : 0);
                        const uint64_t db = umma_desc(xb + o0 + (uint32_t)(k0 * 16), 128, o1 - o0);
                        umma_bf16(tmem + (uint32_t)(k * 16), da, db, umma_idesc(16, true, true), accum);
                    }
                }
                accum = 1;
            }
            umma_commit(&bar_empty[q][s]);
            mma_done = j + 1;
            if (q == 0 && tma_next < nmine) {
                if (!issue_loads(tma_next)) { ok = false; break; }
                tma_next++;
            }
        }
        // the last group of this issuer completes after every earlier one
        if (ok && mma_done > 0)
            ok = mbar_wait(&bar_empty[q][(mma_done - 1) % S], (uint32_t)(((mma_done - 1) / S) & 1));
        if (!ok) {
            s_fail = 1;
            // give what is in flight its own bounded wait before the shared
            // memory and the accumulator columns are released
            if (q == 0)
                for (long long i = full_seen; i < tma_next; i++) mbar_wait(&bar_full[i % S], (uint32_t)((i / S) & 1));
            if (mma_done > 0) mbar_wait(&bar_empty[q][(mma_done - 1) % S], (uint32_t)(((mma_done - 1) / S) & 1));
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (!s_fail && warp == 0) {
        // lanes 0..31 hold output channels 0..31; columns in blocks of 32
        float* dst = a.partial + (long long)blockIdx.x * 32 * a.ncols;
        const bool any = nmine > 0;
        for (int cb = 0; cb < a.ncols; cb += 32) {
            float v[32];
            tmem_ld32(tmem + (uint32_t)cb, v);
            for (int i = 0; i < 32 && cb + i < a.ncols; i++) dst[(long long)tid * a.ncols + cb + i] = any ? v[i] : 0.f;
        }
    }
    if (s_fail && tid == 0) atomicExch(a.err, RN_ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, NCOLS_TMEM);
}

__global__ void conv_wgrad_reduce(float* __restrict__ out, const float* __restrict__ partial, int nparts, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0;
    for (int p = 0; p < nparts; p++) s += partial[(long long)p * n + i];
    out[i] = (float)s;
}

// FP32 image [N][H][W] -> bf16 blocked with 8 channels (channel 0 = image).
__global__ void conv_pack_image(uint4* __restrict__ out, const float* __restrict__ img, const float* __restrict__ sub,
                                float scale, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float q[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    q[0] = (img[i] - (sub ? sub[i] : 0.f)) * scale;
    out[i] = pack_bf16x8(q);
}

// ---- host side -----------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Tensor map over a blocked activation [N][ch][H][W][8] bf16 with the pixels
// taken in groups of `pix` (W a multiple of pix): a box of (8 pix, box_w /
// pix, box_h, ch, 1), each of its rows 16 pix bytes.
static int make_act_map(CUtensorMap* m, const void* base, int N, int ch, int H, int W, int box_w, int box_h,
                        int pix = 1) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return set_error(RN_ERR_CUDA, "conv: cuTensorMapEncodeTiled unavailable");
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return set_error(RN_ERR_ARG, "conv: activations must be 16-byte aligned");
    const int p = pix;
    cuuint64_t dims[5] = {(cuuint64_t)(8 * p), (cuuint64_t)(W / p), (cuuint64_t)H, (cuuint64_t)ch, (cuuint64_t)N};
    cuuint64_t strides[4] = {(cuuint64_t)(16 * p), (cuuint64_t)W * 16, (cuuint64_t)H * W * 16, (cuuint64_t)ch * H * W * 16};
    cuuint32_t box[5] = {(cuuint32_t)(8 * p), (cuuint32_t)(box_w / p), (cuuint32_t)box_h, (cuuint32_t)ch, 1};
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(RN_ERR_ARG, "conv: tensor map encoding failed (" + std::to_string((int)r) + ")");
    return RN_OK;
}

static int sm_count() {
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

template <int CH, int NPAD, int PIX>
static int launch_conv(const CUtensorMap& m, const ConvArgs& a, cudaStream_t st) {
    constexpr int KSTEPS = CH == 4 ? 18 : 5;
    constexpr uint32_t BOX_BYTES = CH * 3 * (kConvTile + 2 * PIX) * 16;
    constexpr uint32_t BOX_ALLOC = (BOX_BYTES + kZeroBytes + 1023) & ~1023u;
    const size_t smem = kConvStages * BOX_ALLOC + 2 * KSTEPS * NPAD * 16 + 1024;
    auto kern = conv3x3_kernel<CH, NPAD, PIX>;
    RN_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    RN_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
    const long long ntiles = (long long)a.N * a.H * ((a.W + kConvTile - 1) / kConvTile);
    // as many CTAs per SM as shared memory allows (64 of the SM's 512 TMEM
    // columns each), at most four
    int per_sm = 0, dev = 0, smem_sm = 0;
    RN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kConvWsThreads, smem));
    RN_CUDA_TRY(cudaGetDevice(&dev));
    RN_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    // (the per-CTA reservation and the static barriers: 2 KB)
    per_sm = std::max(1, std::min(std::max(per_sm, smem_sm / (int)(smem + 2048)), 4));
    const int grid = (int)std::min<long long>(ntiles, (long long)per_sm * sm_count());
    kern<<<grid, kConvWsThreads, smem, st>>>(m, a);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

}  // namespace rn

using namespace rn;

extern "C" int rn_conv3x3(void* d_out, const void* d_in, const void* d_wpack, const float* d_bias, const void* d_aux,
                          int N, int H, int W, int cin, int cout, int mode, int* d_err, void* stream) {
    clear_error();
    if (!d_out || !d_in || !d_wpack || !d_err) return set_error(RN_ERR_ARG, "conv: null argument");
    if (N <= 0 || H <= 0 || W <= 0) return set_error(RN_ERR_ARG, "conv: sizes must be positive");
    if (cin != 8 && cin != 32) return set_error(RN_ERR_ARG, "conv: input channels must be 8 or 32");
    if (mode < 0 || mode > 3) return set_error(RN_ERR_ARG, "conv: bad mode");
    if ((mode == 0 || mode == 2) && cout != 32) return set_error(RN_ERR_ARG, "conv: blocked outputs have 32 channels");
    if (mode == 1 && cout != 1) return set_error(RN_ERR_ARG, "conv: the residual output has one channel");
    if (mode == 3 && cout != 1 && cout != 32) return set_error(RN_ERR_ARG, "conv: cout must be 1 or 32");
    if ((mode == 0 || mode == 1) && !d_bias) return set_error(RN_ERR_ARG, "conv: bias required");
    if ((mode == 1 || mode == 2) && !d_aux) return set_error(RN_ERR_ARG, "conv: aux input required");
    CUtensorMap m;
    ConvArgs a{d_out, reinterpret_cast<const uint4*>(d_wpack), d_bias, d_aux, N, H, W, cout, mode, d_err};
    cudaStream_t st = (cudaStream_t)stream;
    auto run = [&](auto pix) {
        constexpr int P = decltype(pix)::value;
        RN_TRY(make_act_map(&m, d_in, N, cin / 8, H, W, kConvTile + 2 * P, 3, P));
        if (cin == 32) return cout == 32 ? launch_conv<4, 32, P>(m, a, st) : launch_conv<4, 16, P>(m, a, st);
        return cout == 32 ? launch_conv<1, 32, P>(m, a, st) : launch_conv<1, 16, P>(m, a, st);
    };
    if (W % 8 == 0) return run(std::integral_constant<int, 8>{});
    if (W % 2 == 0) return run(std::integral_constant<int, 2>{});
    return run(std::integral_constant<int, 1>{});
}

extern "C" int rn_conv3x3_wgrad_cols(int cin) { return cin == 32 ? 288 + 16 : 80 + 16; }

extern "C" int rn_conv3x3_wgrad(float* d_dw, float* d_partial, size_t partial_bytes, const void* d_x, const void* d_dy,
                                int N, int H, int W, int cin, int cout, int* d_err, void* stream) {
    clear_error();
    if (!d_dw || !d_partial || !d_x || !d_dy || !d_err) return set_error(RN_ERR_ARG, "conv wgrad: null argument");
    if (N <= 0 || H <= 0 || W <= 0) return set_error(RN_ERR_ARG, "conv wgrad: sizes must be positive");
    if ((cin != 8 && cin != 32) || (cout != 8 && cout != 32)) return set_error(RN_ERR_ARG, "conv wgrad: channels 8 or 32");
    const int ncols = rn_conv3x3_wgrad_cols(cin);
    const long long ntiles = (long long)N * H * ((W + kConvTile - 1) / kConvTile);
    const int grid = (int)std::min<long long>(ntiles, (long long)sm_count());
    if (partial_bytes < (size_t)grid * 32 * ncols * sizeof(float))
        return set_error(RN_ERR_ARG, "conv wgrad: partial buffer too small (" + std::to_string((size_t)grid * 32 * ncols * 4) +
                                         " bytes needed)");
    WgradArgs a{d_partial, N, H, W, ncols, d_err};
    cudaStream_t st = (cudaStream_t)stream;
    auto run = [&](auto pix) -> int {
        constexpr int P = decltype(pix)::value;
        CUtensorMap mx, mdy;
        RN_TRY(make_act_map(&mx, d_x, N, cin / 8, H, W, kConvTile + 2 * P, 3, P));
        RN_TRY(make_act_map(&mdy, d_dy, N, cout / 8, H, W, kConvTile, 1, P));
        const uint32_t xbox = (cin / 8) * 3 * (kConvTile + 2 * P) * 16;
        const uint32_t dyb = (cout / 8) * kConvTile * 16;
        const size_t smem = kWgStages * (((dyb + 1023) & ~1023u) + ((xbox + kZeroBytes + 1023) & ~1023u)) + 512 + 1024;
        auto launch = [&](auto kern) -> int {
            RN_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            kern<<<grid, kConvThreads, smem, st>>>(mx, mdy, a);
            return RN_OK;
        };
        if (cin == 32 && cout == 32) return launch(conv3x3_wgrad_kernel<4, 4, P>);
        if (cin == 32 && cout == 8) return launch(conv3x3_wgrad_kernel<4, 1, P>);
        if (cin == 8 && cout == 32) return launch(conv3x3_wgrad_kernel<1, 4, P>);
        return set_error(RN_ERR_ARG, "conv wgrad: unsupported channel pair");
    };
    if (W % 8 == 0) RN_TRY(run(std::integral_constant<int, 8>{}));
    else if (W % 2 == 0) RN_TRY(run(std::integral_constant<int, 2>{}));
    else RN_TRY(run(std::integral_constant<int, 1>{}));
    RN_CUDA_TRY(cudaGetLastError());
    const int n = 32 * ncols;
    conv_wgrad_reduce<<<(n + 255) / 256, 256, 0, st>>>(d_dw, d_partial, grid, n);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

extern "C" int rn_conv_pack_image(void* d_out, const float* d_img, const float* d_sub, float scale, int N, int H, int W,
                                  void* stream) {
    clear_error();
    if (!d_out || !d_img) return set_error(RN_ERR_ARG, "conv pack: null argument");
    const long long n = (long long)N * H * W;
    if (n <= 0) return set_error(RN_ERR_ARG, "conv pack: sizes must be positive");
    conv_pack_image<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<uint4*>(d_out), d_img,
                                                                                    d_sub, scale, n);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}
