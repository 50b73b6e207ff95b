// Learned seam blend: tcgen05 (5th-generation tensor core) implicit-GEMM 3x3
// convolutions, forward and backward, the U-Net-lite built from them, its
// loss and Adam, all on the GPU.  No reference counterpart (the reference
// blends overlaps with SeamBlend.cpp:549-587 only); the network's shape is in
// include/image360_b200_blendnet.h.
//
// Convolution as GEMM, per CTA tile of R image rows x 128 pixels:
//   D[pixel][cout] += A[pixel][(tap, cin)] * B[cout][(tap, cin)]
// with M = 128 pixels of one row, N = cout, K = 9 * cin in steps of 16.
// The input halo ((R+2) rows x 130 pixels x cin) sits in shared memory as
// 8-channel chunks, each a [pixel][8 channels] array of 16-byte rows; any
// 8 consecutive pixels of it are one 8x16-byte "core matrix" of the K-major
// no-swizzle layout, so the A operand of tap (dy, dx) is the same buffer with
// the descriptor's start address moved by (dy * 130 + dx) * 16 bytes - no
// im2col copy.  Weights are K-major [k/8][cout][8].  fp32 accumulators live in
// TMEM, two slots so the epilogue of one tile overlaps the MMAs of the next,
// and halos are double-buffered with cp.async so the next load overlaps both.
//
// Weight gradient: D[(tap, cin)][cout] += X[pixel + tap][cin] * G[pixel][cout]
// summed over pixels (K), with both operands MN-major (the 8 channels of a
// pixel are the contiguous 16 bytes); each CTA owns a 128-row chunk of
// (tap, cin) and a slice of the pixels, and writes an fp32 partial that a
// small kernel reduces.
#include "common.cuh"
#include "render_plan.hpp"
#include "tc_common.cuh"
#include "../../include/image360_b200_blendnet.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

namespace i360b
{
namespace
{
using bf16 = __nv_bfloat16;

constexpr int kTileX = 128;                // pixels per weight-gradient tile (one row)
constexpr long long kWaitSpins = 1ll << 26;  // bounded mbarrier waits
constexpr int kSlots = 4;
constexpr float kInScale = 1.0f / 32768.0f;

enum
{
    LD_PLAIN = 0,
    LD_CONCAT = 1
};
enum
{
    EP_RELU = I360B_CONV_BIAS_RELU,
    EP_LOGITS = I360B_CONV_LOGITS,
    EP_MASK = I360B_CONV_MASK,
    EP_RAW = I360B_CONV_RAW,
    EP_COMPOSITE = 4
};

struct ConvArgs
{
    const bf16* x;  // [n][h][w][cin], or the skip [n][h][w][cs] for LD_CONCAT
    const bf16* u;  // LD_CONCAT: [n][h/2][w/2][cin - cs]
    int cs;
    int n, h, w;
    const bf16* wt;     // [npad][9 * cin], k = tap * cin + c
    const float* bias;  // [npad]
    void* out;
    const bf16* act;  // EP_MASK: [n][h][w][npad]
    const i360b_blend_job* jobs;  // EP_COMPOSITE: one per image
    int* error;
};

// Tile geometry of the 3x3 convolution: TW x TH output pixels per tile, split
// into M blocks of 8 columns x 16 rows; the input halo of (TW+2) x (TH+2)
// pixels is kept per 8-channel chunk with row pitch kP = TW+2 pixels.
template <int CIN, int NPAD, int TW, int TH, int STAGES, int LD, int EW = 4>
struct ConvShape
{
    // Roles by warp: [0, EW) epilogue, EW producer, EW + 1 MMA, then (for a
    // concatenated input) 4 upsampling warps.
    static constexpr int kEpiWarps = EW;
    static constexpr int kProducerWarp = EW, kMmaWarp = EW + 1, kExpandWarp = EW + 2;
    static constexpr int kC8 = CIN / 8;
    static constexpr int kP = TW + 2;
    static constexpr int kHaloPx = (TW + 2) * (TH + 2);
    static constexpr uint32_t kBox = kHaloPx * 16;                  // bytes of one chunk box
    static constexpr uint32_t kChunk = (kBox + 127) / 128 * 128;    // TMA destinations 128-byte aligned
    static constexpr uint32_t kStage = kC8 * kChunk;
    static constexpr uint32_t kW = 9u * CIN * NPAD * 2;
    static constexpr int kBX = TW / 8, kBY = TH / 16, kMB = kBX * kBY;
    static constexpr uint32_t kSlotCols = kMB * NPAD;
    static constexpr uint32_t kTmem = tc::tmem_cols(2 * kSlotCols);
    static constexpr int kKSteps = 9 * CIN / 16;
    static constexpr int kThreads = 32 * (EW + 2) + (LD == LD_CONCAT ? 128 : 0);
    // Concatenated input: the half-resolution box behind a tile's halo,
    // (TW/2+2) x (TH/2+2) pixels per 8-channel chunk, per ring stage.
    static constexpr int kPh = TW / 2 + 2;
    static constexpr int kHalfPx = (TW / 2 + 2) * (TH / 2 + 2);
    static constexpr uint32_t kHalfBox = kHalfPx * 16;
    static constexpr uint32_t kHalfChunk = (kHalfBox + 127) / 128 * 128;
    static constexpr uint32_t kHalfStage = LD == LD_CONCAT ? kC8 * kHalfChunk : 0;  // upper bound on chunks
    static constexpr uint32_t kBars = (3 * STAGES + 4) * 8 + 16;
    static constexpr uint32_t kBias = NPAD * 4;
    static constexpr uint32_t kSmem = 128 + kW + STAGES * (kStage + kHalfStage) + kBars + kBias;
    static_assert(CIN % 16 == 0 && NPAD % 16 == 0 && NPAD >= 16 && NPAD <= 256, "MMA shape");
    static_assert(TW % 8 == 0 && TH % 16 == 0 && TW + 2 <= 256 && TH + 2 <= 256, "tile shape");
    static_assert(2 * kSlotCols <= 512, "TMEM capacity");
    static_assert(kW % 128 == 0, "ring alignment");
    static_assert(kChunk / 16 < (1u << 14) && kP < (1 << 14), "descriptor offset range");
    static_assert(kSmem <= 227u * 1024u, "shared memory");
    static_assert(EW == 4 || (EW == 8 && kMB % 2 == 0), "epilogue warps split the M blocks in two");
};

__device__ __forceinline__ uint4 pack8_bf16(const float* v)
{
    uint4 r;
    __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]);
    __nv_bfloat162 p1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]);
    __nv_bfloat162 p3 = __floats2bfloat162_rn(v[6], v[7]);
    r.x = *reinterpret_cast<uint32_t*>(&p0);
    r.y = *reinterpret_cast<uint32_t*>(&p1);
    r.z = *reinterpret_cast<uint32_t*>(&p2);
    r.w = *reinterpret_cast<uint32_t*>(&p3);
    return r;
}

__device__ __forceinline__ void unpack8_bf16(uint4 q, float* v)
{
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        __nv_bfloat162 p = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
        float2 f = __bfloat1622float2(p);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

// Source of one 16-byte (8-channel) chunk of the convolution input at (img,
// yy, xx); yy, xx inside the image.
template <int CIN, int LD>
__device__ __forceinline__ const bf16* input_chunk(const bf16* x, const bf16* u, int cs, int h, int w, int img, int yy,
                                                   int xx, int c8)
{
    if (LD == LD_PLAIN) return x + ((((size_t)img * h + yy) * w + xx) * CIN + c8 * 8);
    const int sc8 = cs >> 3;
    if (c8 < sc8) return x + ((((size_t)img * h + yy) * w + xx) * cs + c8 * 8);
    return u + ((((size_t)img * (h >> 1) + (yy >> 1)) * (w >> 1) + (xx >> 1)) * (CIN - cs) + (c8 - sc8) * 8);
}

// Softmax-weighted composite of a pixel's covered layers (the network head).
// The pixel's layer values (0 where a slot is absent).
__device__ __forceinline__ void load_slots(const i360b_blend_job& J, int y, int x, float (*v)[3])
{
#pragma unroll
    for (int i = 0; i < kSlots; ++i)
    {
        v[i][0] = v[i][1] = v[i][2] = 0.0f;
        if (J.slot[i])
        {
            const unsigned short* p = J.slot[i] + (long long)y * J.rowStride + (long long)x * J.pixStride;
            v[i][0] = __ldg(p);
            v[i][1] = __ldg(p + 1);
            v[i][2] = __ldg(p + 2);
        }
    }
}

// Softmax over the covered layers (value not (0,0,0)) of the logits, and the
// weighted sum of the layers; v from load_slots.
__device__ __forceinline__ void blend_slots(const float* l, const float (*v)[3], float* outDN, float* wts, bool* cov,
                                            int& nCov)
{
    float m = -INFINITY;
    nCov = 0;
#pragma unroll
    for (int i = 0; i < kSlots; ++i)
    {
        cov[i] = v[i][0] != 0.0f || v[i][1] != 0.0f || v[i][2] != 0.0f;
        if (cov[i])
        {
            m = fmaxf(m, l[i]);
            ++nCov;
        }
    }
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < kSlots; ++i)
    {
        wts[i] = cov[i] ? __expf(l[i] - m) : 0.0f;
        sum += wts[i];
    }
    const float inv = nCov ? 1.0f / sum : 0.0f;
    outDN[0] = outDN[1] = outDN[2] = 0.0f;
#pragma unroll
    for (int i = 0; i < kSlots; ++i)
    {
        wts[i] *= inv;
        outDN[0] += wts[i] * v[i][0];
        outDN[1] += wts[i] * v[i][1];
        outDN[2] += wts[i] * v[i][2];
    }
}

__device__ __forceinline__ void composite_pixel(const i360b_blend_job& J, int y, int x, const float* l, float* outDN,
                                                float* wts, float (*v)[3], bool* cov, int& nCov)
{
    load_slots(J, y, x, v);
    blend_slots(l, v, outDN, wts, cov, nCov);
}

// ---------------------------------------------------------------------------
// 3x3 convolution (forward, or backward-data with flipped transposed weights),
// persistent and warp-specialised; CTA b handles tiles b, b + gridDim.x, ...
//
// The A operand of tap (dy, dx) for M block (bx, by) is the halo chunk with
// the descriptor start moved by ((16 by + dy) kP + 8 bx + dx) * 16 bytes: the
// 8 pixels of a block row are one core matrix (8 rows of 16 bytes) and the 16
// block rows are core-matrix groups kP * 16 bytes apart (SBO); the two
// 8-channel halves of a K step are one chunk apart (LBO).
//
// Roles:
//   warp EW lane 0 TMA producer: one 4-D box (8 channels x (TW+2) x (TH+2))
//                  per chunk into a STAGES-deep ring, zero fill outside the
//                  image;
//   warps EW+2..   (concatenated input only) expand the TMA-loaded
//                  half-resolution box into the nearest-upsampled channels
//                  of the halo (shared memory to shared memory);
//   warp EW+1 lane 0 MMA issuer: MB x 9 CIN/16 tcgen05.mma per tile into one of
//                  two TMEM accumulators; commits free the ring stage and
//                  publish the accumulator;
//   warps 0..EW-1  epilogue (EW = 4 or 8): TMEM lanes 32q..32q+31, q = w % 4
//                  (rows 4q..4q+3 of each M block) -> bias/ReLU, mask, raw or
//                  blend head -> global.
// Every wait is bounded; a timeout sets the error flag and the CTA winds
// down after its loads have landed.
// ---------------------------------------------------------------------------
template <int CIN, int NPAD, int TW, int TH, int STAGES, int LD, int EP, int EW>
__global__ void __launch_bounds__(ConvShape<CIN, NPAD, TW, TH, STAGES, LD, EW>::kThreads, 1)
    k_conv3x3(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap tmapHalf, ConvArgs a)
{
    using S = ConvShape<CIN, NPAD, TW, TH, STAGES, LD, EW>;
    extern __shared__ unsigned char smemRaw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smemRaw) + 127) & ~uintptr_t(127));
    unsigned char* wsm = smem;
    unsigned char* ring = smem + S::kW;
    unsigned char* halfRing = ring + STAGES * S::kStage;
    uint64_t* full = reinterpret_cast<uint64_t*>(halfRing + STAGES * S::kHalfStage);
    uint64_t* empty = full + STAGES;
    uint64_t* halfFull = empty + STAGES;
    uint64_t* accFull = halfFull + STAGES;
    uint64_t* accEmpty = accFull + 2;
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(accEmpty + 2);
    float* sBias = reinterpret_cast<float*>(tmemSlot + 4);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tilesX = (a.w + TW - 1) / TW, tilesY = (a.h + TH - 1) / TH;
    const long long nTiles = (long long)a.n * tilesX * tilesY;
    if ((long long)blockIdx.x >= nTiles) return;
    const int myTiles = (int)((nTiles - 1 - blockIdx.x) / gridDim.x) + 1;
    auto coord = [&](int i, int& img, int& y0, int& x0) {
        const long long t = blockIdx.x + (long long)i * gridDim.x;
        x0 = (int)(t % tilesX) * TW;
        const long long r = t / tilesX;
        y0 = (int)(r % tilesY) * TH;
        img = (int)(r / tilesY);
    };
    const int tmaChunks = LD == LD_CONCAT ? (a.cs >> 3) : S::kC8;

    if (warp == 0) tc::tmem_alloc(tmemSlot, S::kTmem);
    if (tid == 0)
    {
        for (int s = 0; s < STAGES; ++s)
        {
            tc::mbar_init(&full[s], LD == LD_CONCAT ? 1 + 128 : 1);
            tc::mbar_init(&empty[s], 1);
            tc::mbar_init(&halfFull[s], 1);
        }
        for (int k = 0; k < 2; ++k)
        {
            tc::mbar_init(&accFull[k], 1);
            tc::mbar_init(&accEmpty[k], EW);
        }
        tc::fence_mbar_init();
    }
    {
        constexpr int kK8 = 9 * S::kC8;
        for (int q = tid; q < NPAD * kK8; q += blockDim.x)
        {
            const int n = q / kK8, k8 = q % kK8;
            tc::cp_async16(wsm + k8 * (NPAD * 16) + n * 16, a.wt + (size_t)n * 9 * CIN + k8 * 8, 16);
        }
        tc::cp_async_commit();
        for (int c = tid; c < NPAD; c += blockDim.x) sBias[c] = a.bias ? a.bias[c] : 0.0f;
        tc::cp_async_wait<0>();
        tc::fence_proxy_async();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmemSlot;
    bool ok = true;

    if (warp == S::kProducerWarp)
    {
        if (lane == 0)
        {
            int issued = 0;
            for (int i = 0; i < myTiles; ++i)
            {
                const int s = i % STAGES;
                if (!tc::mbar_wait(&empty[s], ((i / STAGES) & 1) ^ 1, kWaitSpins))
                {
                    ok = false;
                    break;
                }
                int img, y0, x0;
                coord(i, img, y0, x0);
                unsigned char* st = ring + s * S::kStage;
                if (LD == LD_CONCAT)
                {
                    // half-resolution rows/columns y0/2 - 1 .. (y0 + TH)/2 (x0, y0 even)
                    unsigned char* hs = halfRing + s * S::kHalfStage;
                    const int nu8 = S::kC8 - tmaChunks;
                    tc::mbar_arrive_expect_tx(&halfFull[s], (uint32_t)nu8 * S::kHalfBox);
                    for (int c = 0; c < nu8; ++c)
                        tc::tma_load_4d(hs + c * S::kHalfChunk, &tmapHalf, c * 8, (x0 >> 1) - 1, (y0 >> 1) - 1, img,
                                        &halfFull[s]);
                }
                tc::mbar_arrive_expect_tx(&full[s], (uint32_t)tmaChunks * S::kBox);
                for (int c = 0; c < tmaChunks; ++c)
                    tc::tma_load_4d(st + c * S::kChunk, &tmap, c * 8, x0 - 1, y0 - 1, img, &full[s]);
                issued = i + 1;
            }
            // The last loads must land before the CTA may exit.
            for (int j = max(0, issued - STAGES); j < issued; ++j)
            {
                if (!tc::mbar_wait(&full[j % STAGES], (j / STAGES) & 1, kWaitSpins)) ok = false;
                if (LD == LD_CONCAT && !tc::mbar_wait(&halfFull[j % STAGES], (j / STAGES) & 1, kWaitSpins)) ok = false;
            }
        }
    }
    else if (LD == LD_CONCAT && warp >= S::kExpandWarp)
    {
        // Nearest 2x upsample of the half-resolution box into the halo chunks
        // after the skip channels: halo pixel (hx, hy) reads box pixel
        // ((hx - 1) >> 1) + 1, ((hy - 1) >> 1) + 1 (tile origin even).
        const int ptid = tid - 32 * S::kExpandWarp;
        const int sc8 = a.cs >> 3, nu8 = S::kC8 - sc8;
        for (int i = 0; i < myTiles; ++i)
        {
            const int s = i % STAGES;
            bool got = tc::mbar_wait(&halfFull[s], (i / STAGES) & 1, kWaitSpins);
            if (!got)
            {
                ok = false;
                break;
            }
            const unsigned char* hs = halfRing + s * S::kHalfStage;
            unsigned char* st = ring + s * S::kStage;
            const int nq = nu8 * S::kHaloPx;
            for (int q = ptid; q < nq; q += 128)
            {
                const int cu = q / S::kHaloPx, px = q - cu * S::kHaloPx;
                const int hy = px / S::kP, hx = px - hy * S::kP;
                const int ly = ((hy - 1) >> 1) + 1, lx = ((hx - 1) >> 1) + 1;
                *reinterpret_cast<uint4*>(st + (sc8 + cu) * S::kChunk + px * 16) =
                    *reinterpret_cast<const uint4*>(hs + cu * S::kHalfChunk + (ly * S::kPh + lx) * 16);
            }
            tc::fence_proxy_async();  // generic smem writes -> tensor core
            tc::mbar_arrive(&full[s]);
        }
    }
    else if (warp == S::kMmaWarp)
    {
        if (lane == 0)
        {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(128, NPAD);
            const uint64_t bBase = tc::smem_desc(tc::smem_u32(wsm), NPAD * 16, 128);
            for (int i = 0; i < myTiles; ++i)
            {
                const int s = i % STAGES, acc = i & 1;
                if (!tc::mbar_wait(&full[s], (i / STAGES) & 1, kWaitSpins) ||
                    !tc::mbar_wait(&accEmpty[acc], ((i >> 1) & 1) ^ 1, kWaitSpins))
                {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                // Descriptors differ only in their start-address field: add
                // the (compile-time) offset in 16-byte units to a base.
                const uint64_t aBase = tc::smem_desc(tc::smem_u32(ring + s * S::kStage), S::kChunk, S::kP * 16);
#pragma unroll
                for (int b = 0; b < S::kMB; ++b)
                {
                    const int bx = b % S::kBX, by = b / S::kBX;
                    const uint32_t d = tmem + acc * S::kSlotCols + b * NPAD;
#pragma unroll
                    for (int ks = 0; ks < S::kKSteps; ++ks)
                    {
                        const int k0 = ks * 16, tap = k0 / CIN, c8 = (k0 % CIN) >> 3;
                        const int dy = tap / 3, dx = tap % 3;
                        const uint32_t aOff = (c8 * S::kChunk + ((by * 16 + dy) * S::kP + bx * 8 + dx) * 16) >> 4;
                        const uint32_t bOff = (2 * ks * (NPAD * 16)) >> 4;
                        tc::mma_bf16(d, aBase + aOff, bBase + bOff, idesc, ks > 0 ? 1u : 0u);
                    }
                }
                tc::mma_commit(&empty[s]);
                tc::mma_commit(&accFull[acc]);
            }
        }
    }
    else if (warp < EW)
    {
        // Warp w reads TMEM lane quadrant w % 4; with 8 epilogue warps the
        // two warps of a quadrant take alternate M blocks.
        const int quad = warp & 3, half = warp >> 2;
        for (int i = 0; i < myTiles; ++i)
        {
            const int acc = i & 1;
            bool done = tc::mbar_wait(&accFull[acc], (i >> 1) & 1, kWaitSpins);
            done = __all_sync(0xffffffffu, done);
            if (!done)
            {
                ok = false;
                break;
            }
            tc::fence_after_sync();
            int img, y0, x0;
            coord(i, img, y0, x0);
            const uint32_t base = tmem + ((uint32_t)(quad * 32) << 16) + acc * S::kSlotCols;
            for (int b = (EW == 8 ? half : 0); b < S::kMB; b += EW / 4)
            {
                const int bx = b % S::kBX, by = b / S::kBX;
                const int y = y0 + by * 16 + quad * 4 + (lane >> 3);
                const int x = x0 + bx * 8 + (lane & 7);
                const bool valid = y < a.h && x < a.w;
                const size_t pix = ((size_t)img * a.h + y) * a.w + x;
                // Global inputs of the epilogue first, so their latency
                // overlaps the TMEM loads.
                float vv[4][3];
                bool inJob = false;
                if (EP == EP_COMPOSITE)
                {
                    const i360b_blend_job& J = a.jobs[img];
                    inJob = valid && x < J.width && y < J.height;
                    if (inJob) load_slots(J, y, x, vv);
                }
                uint4 mk[EP == EP_MASK ? NPAD / 8 : 1];
                if (EP == EP_MASK && valid)
                {
                    const uint4* ap = reinterpret_cast<const uint4*>(a.act + pix * NPAD);
#pragma unroll
                    for (int q = 0; q < NPAD / 8; ++q) mk[q] = ap[q];
                }
                constexpr int kCols = (EP == EP_LOGITS || EP == EP_COMPOSITE) ? 16 : NPAD;
                uint32_t r[kCols];
#pragma unroll
                for (int cb = 0; cb < kCols / 16; ++cb) tc::tmem_ld16_nowait(base + b * NPAD + cb * 16, r + cb * 16);
                tc::tmem_wait_ld();
#pragma unroll
                for (int cb = 0; cb < kCols / 16; ++cb) tc::tmem_reg_fence16(r + cb * 16);
                if (!valid) continue;
                if (EP == EP_LOGITS || EP == EP_COMPOSITE)
                {
                    float l[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) l[j] = __uint_as_float(r[j]) + sBias[j];
                    if (EP == EP_LOGITS)
                    {
                        reinterpret_cast<float4*>(a.out)[pix] = make_float4(l[0], l[1], l[2], l[3]);
                    }
                    else if (inJob)
                    {
                        const i360b_blend_job& J = a.jobs[img];
                        float o[3], wts[4];
                        bool cov[4];
                        int nCov;
                        blend_slots(l, vv, o, wts, cov, nCov);
                        unsigned short* q = J.out + (long long)y * J.outRowStride + (long long)x * 3;
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                            q[c] = (unsigned short)__float2uint_rn(fminf(fmaxf(o[c], 0.0f), 65535.0f));
                    }
                }
                else
                {
#pragma unroll
                    for (int cb = 0; cb < NPAD / 16; ++cb)
                    {
                        float v[16];
#pragma unroll
                        for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[cb * 16 + j]);
                        if (EP == EP_RELU)
                        {
#pragma unroll
                            for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j] + sBias[cb * 16 + j], 0.0f);
                        }
                        if (EP == EP_MASK)
                        {
                            float m[16];
                            unpack8_bf16(mk[2 * cb], m);
                            unpack8_bf16(mk[2 * cb + 1], m + 8);
#pragma unroll
                            for (int j = 0; j < 16; ++j) v[j] = m[j] > 0.0f ? v[j] : 0.0f;
                        }
                        uint4* op = reinterpret_cast<uint4*>(static_cast<bf16*>(a.out) + pix * NPAD + cb * 16);
                        op[0] = pack8_bf16(v);
                        op[1] = pack8_bf16(v + 8);
                    }
                }
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&accEmpty[acc]);
        }
    }
    if (!ok) atomicOr(a.error, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0)
    {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, S::kTmem);
    }
}

// ---------------------------------------------------------------------------
// Weight gradient.  grid = (slices, chunks); CTA (s, c) accumulates rows
// c*128 .. c*128+127 of (tap, cin) over pixel tiles s, s + slices, ... (one
// tile = 128 pixels of one row) and writes partial[s][row][cout].
// ---------------------------------------------------------------------------
struct WgradArgs
{
    const bf16* x;
    const bf16* u;
    int cs;
    const bf16* g;  // [n][h][w][COUT]
    int n, h, w;
    float* partial;  // [gridDim.x][gridDim.y * 128][COUT]
    int* error;
};

template <int CIN, int COUT>
struct WgradShape
{
    static constexpr int kC8 = CIN / 8;
    static constexpr int kRows8 = 9 * kC8;
    static constexpr int kChunks = (kRows8 + 15) / 16;
    static constexpr uint32_t kA = 16 * 2048;
    static constexpr uint32_t kB = (COUT / 8) * 2048;
    static constexpr uint32_t kStage = kA + kB;
    static constexpr uint32_t kSmem = 2 * kStage + 64;
    static constexpr uint32_t kTmem = tc::tmem_cols(COUT);
    static_assert(COUT % 16 == 0 && COUT >= 16 && COUT <= 256, "MMA shape");
};

template <int CIN, int COUT, int LD>
__global__ void __launch_bounds__(128, 1) k_conv3x3_wgrad(WgradArgs a)
{
    using S = WgradShape<CIN, COUT>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 2 * S::kStage);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(mbar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int chunk = blockIdx.y;
    const int tilesX = a.w / kTileX;
    const long long nTiles = (long long)a.n * a.h * tilesX;
    const int myTiles = (long long)blockIdx.x < nTiles ? (int)((nTiles - 1 - blockIdx.x) / gridDim.x) + 1 : 0;
    float* part = a.partial + ((size_t)blockIdx.x * (gridDim.y * 128) + (size_t)chunk * 128) * COUT;
    if (myTiles == 0)
    {
        for (int q = tid; q < 128 * COUT; q += 128) part[q] = 0.0f;
        return;
    }

    auto load = [&](long long t, unsigned char* buf) {
        const int x0 = (int)(t % tilesX) * kTileX;
        const long long r = t / tilesX;
        const int y = (int)(r % a.h), img = (int)(r / a.h);
        for (int q = tid; q < 16 * kTileX; q += 128)
        {
            const int lg = q & 15, px = q >> 4;
            const int r8 = chunk * 16 + lg;
            const int tap = r8 / S::kC8, c8 = r8 % S::kC8;
            const int yy = y + tap / 3 - 1, xx = x0 + px + tap % 3 - 1;
            const bool ok = r8 < S::kRows8 && yy >= 0 && yy < a.h && xx >= 0 && xx < a.w;
            const bf16* src = ok ? input_chunk<CIN, LD>(a.x, a.u, a.cs, a.h, a.w, img, yy, xx, c8) : a.x;
            tc::cp_async16(buf + lg * 2048 + px * 16, src, ok ? 16 : 0);
        }
        constexpr int kG8 = COUT / 8;
        for (int q = tid; q < kG8 * kTileX; q += 128)
        {
            const int c8 = q % kG8, px = q / kG8;
            const bf16* src = a.g + ((((size_t)img * a.h + y) * a.w + x0 + px) * COUT + c8 * 8);
            tc::cp_async16(buf + S::kA + c8 * 2048 + px * 16, src, 16);
        }
    };

    if (warp == 0) tc::tmem_alloc(tmemSlot, S::kTmem);
    if (tid == 0)
    {
        tc::mbar_init(&mbar[0], 1);
        tc::mbar_init(&mbar[1], 1);
        tc::fence_mbar_init();
    }
    load(blockIdx.x, smem);
    tc::cp_async_commit();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmemSlot;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, COUT) | (1u << 15) | (1u << 16);  // A, B MN-major

    bool ok = true;
    for (int i = 0; i < myTiles; ++i)
    {
        const int s = i & 1;
        const long long t = blockIdx.x + (long long)i * gridDim.x;
        if (i + 1 < myTiles)
        {
            if (i >= 1 && !tc::mbar_wait(&mbar[s ^ 1], ((i - 1) >> 1) & 1, kWaitSpins)) ok = false;
            if (ok) load(t + gridDim.x, smem + (s ^ 1) * S::kStage);
            tc::cp_async_commit();
            tc::cp_async_wait<1>();
        }
        else
        {
            tc::cp_async_wait<0>();
        }
        tc::fence_proxy_async();
        if (__syncthreads_or(!ok))
        {
            ok = false;
            break;
        }
        if (tid == 0)
        {
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_u32(smem + s * S::kStage), b0 = a0 + S::kA;
#pragma unroll
            for (int j = 0; j < kTileX / 16; ++j)
                tc::mma_bf16(tmem, tc::smem_desc(a0 + j * 256, 128, 2048), tc::smem_desc(b0 + j * 256, 128, 2048),
                             idesc, (i > 0 || j > 0) ? 1u : 0u);
            tc::mma_commit(&mbar[s]);
        }
    }
    if (ok)
    {
        const int last = myTiles - 1;
        bool done = tc::mbar_wait(&mbar[last & 1], (last >> 1) & 1, kWaitSpins);
        done = __all_sync(0xffffffffu, done);
        if (!done) ok = false;
        else
        {
            tc::fence_after_sync();
            float* row = part + (size_t)(warp * 32 + lane) * COUT;
#pragma unroll 1
            for (int cb = 0; cb < COUT / 16; ++cb)
            {
                float v[16];
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + cb * 16, v);
                float4* o = reinterpret_cast<float4*>(row + cb * 16);
                o[0] = make_float4(v[0], v[1], v[2], v[3]);
                o[1] = make_float4(v[4], v[5], v[6], v[7]);
                o[2] = make_float4(v[8], v[9], v[10], v[11]);
                o[3] = make_float4(v[12], v[13], v[14], v[15]);
            }
            tc::fence_before_sync();
        }
    }
    if (!ok && lane == 0) atomicOr(a.error, 1);
    tc::cp_async_wait<0>();
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0)
    {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, S::kTmem);
    }
}

// dW[co][k] = sum over slices of partial[slice][k][co] (k = tap * cin + ci).
__global__ void k_wgrad_reduce(const float* __restrict__ partial, int slices, int rowsTotal, int coutStride, int cin,
                               int cout, float* __restrict__ dw)
{
    const int K = 9 * cin;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= K * cout) return;
    const int co = idx / K, k = idx % K;
    float s = 0.0f;
    for (int g = 0; g < slices; ++g) s += partial[((size_t)g * rowsTotal + k) * coutStride + co];
    dw[(size_t)co * K + k] = s;
}

// ---------------------------------------------------------------------------
// Glue: input packing, pooling, loss, gradient routing, bias gradients, Adam.
// ---------------------------------------------------------------------------
// The mask channel of a covered pixel: 0.25 + 0.75 min(1, d / kFeather) with
// d the distance from (x, y) to the nearest of the slot's boundary segments
// (1 when it has none).
constexpr float kFeather = 2048.0f;

__device__ __forceinline__ float feathered_mask(const float* e, float x, float y)
{
    float d2 = INFINITY;
#pragma unroll
    for (int s = 0; s < 4; ++s)
    {
        const float ax = e[4 * s], ay = e[4 * s + 1];
        if (ax != ax) continue;  // absent segment
        const float dx = e[4 * s + 2] - ax, dy = e[4 * s + 3] - ay;
        const float l2 = dx * dx + dy * dy;
        float t = l2 > 0.0f ? ((x - ax) * dx + (y - ay) * dy) / l2 : 0.0f;
        t = fminf(fmaxf(t, 0.0f), 1.0f);
        const float qx = ax + t * dx - x, qy = ay + t * dy - y;
        d2 = fminf(d2, qx * qx + qy * qy);
    }
    return 0.25f + 0.75f * fminf(1.0f, sqrtf(d2) / kFeather);
}

__global__ void k_pack_input(const i360b_blend_job* __restrict__ jobs, int n, int h, int w, bf16* __restrict__ x0)
{
    const long long total = (long long)n * h * w;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
    {
        const int img = (int)(idx / ((long long)h * w));
        const int rem = (int)(idx % ((long long)h * w));
        const int y = rem / w, x = rem % w;
        const i360b_blend_job& J = jobs[img];
        float ch[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) ch[i] = 0.0f;
        if (x < J.width && y < J.height)
        {
#pragma unroll
            for (int i = 0; i < kSlots; ++i)
            {
                if (!J.slot[i]) continue;
                const unsigned short* p = J.slot[i] + (long long)y * J.rowStride + (long long)x * J.pixStride;
                const unsigned short r = p[0], g = p[1], b = p[2];
                if ((r | g | b) == 0) continue;
                ch[4 * i] = r * kInScale;
                ch[4 * i + 1] = g * kInScale;
                ch[4 * i + 2] = b * kInScale;
                ch[4 * i + 3] = feathered_mask(J.edges[i], (float)x, (float)y);
            }
        }
        uint4* o = reinterpret_cast<uint4*>(x0 + idx * 16);
        o[0] = pack8_bf16(ch);
        o[1] = pack8_bf16(ch + 8);
    }
}

// 2x2 average pool of [n][h][w][C] (C = 8 * c8n) into [n][h/2][w/2][C].
__global__ void k_pool2(const bf16* __restrict__ in, int n, int h, int w, int c8n, bf16* __restrict__ out)
{
    const int hh = h >> 1, wh = w >> 1;
    const long long total = (long long)n * hh * wh * c8n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
    {
        const int c8 = (int)(idx % c8n);
        long long r = idx / c8n;
        const int xh = (int)(r % wh);
        r /= wh;
        const int yh = (int)(r % hh), img = (int)(r / hh);
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx)
            {
                float v[8];
                const size_t p = ((size_t)img * h + 2 * yh + dy) * w + 2 * xh + dx;
                unpack8_bf16(reinterpret_cast<const uint4*>(in + p * c8n * 8)[c8], v);
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[j] += v[j];
            }
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] *= 0.25f;
        reinterpret_cast<uint4*>(out + idx * 8)[0] = pack8_bf16(acc);
    }
}

// Gradient of the upsampled half of the concatenation: g5 = (sum over the 2x2
// children of du[..., skip: skip+C]) * (a5 > 0), at half resolution.
__global__ void k_upsample_grad(const bf16* __restrict__ du, int duC, int skip, const bf16* __restrict__ act, int n,
                                int h, int w, int c8n, bf16* __restrict__ g)
{
    const int hh = h >> 1, wh = w >> 1;
    const long long total = (long long)n * hh * wh * c8n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
    {
        const int c8 = (int)(idx % c8n);
        long long r = idx / c8n;
        const int xh = (int)(r % wh);
        r /= wh;
        const int yh = (int)(r % hh), img = (int)(r / hh);
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx)
            {
                float v[8];
                const size_t p = ((size_t)img * h + 2 * yh + dy) * w + 2 * xh + dx;
                unpack8_bf16(*reinterpret_cast<const uint4*>(du + p * duC + skip + c8 * 8), v);
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[j] += v[j];
            }
        float m[8];
        unpack8_bf16(reinterpret_cast<const uint4*>(act)[idx], m);
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = m[j] > 0.0f ? acc[j] : 0.0f;
        reinterpret_cast<uint4*>(g)[idx] = pack8_bf16(acc);
    }
}

// Gradient of the skip activation: g2 = (du[..., 0:C] + dpool / 4 upsampled)
// * (a2 > 0), at full resolution (C = 8 * c8n channels).
__global__ void k_skip_grad(const bf16* __restrict__ du, int duC, const bf16* __restrict__ dpool,
                            const bf16* __restrict__ act, int n, int h, int w, int c8n, bf16* __restrict__ g)
{
    const long long total = (long long)n * h * w * c8n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
    {
        const int c8 = (int)(idx % c8n);
        long long r = idx / c8n;
        const int x = (int)(r % w);
        r /= w;
        const int y = (int)(r % h), img = (int)(r / h);
        float a[8], b[8], m[8];
        unpack8_bf16(*reinterpret_cast<const uint4*>(du + (size_t)(idx / c8n) * duC + c8 * 8), a);
        const size_t ph = ((size_t)img * (h >> 1) + (y >> 1)) * (w >> 1) + (x >> 1);
        unpack8_bf16(reinterpret_cast<const uint4*>(dpool + ph * c8n * 8)[c8], b);
        unpack8_bf16(reinterpret_cast<const uint4*>(act)[idx], m);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = m[j] > 0.0f ? a[j] + 0.25f * b[j] : 0.0f;
        reinterpret_cast<uint4*>(g)[idx] = pack8_bf16(a);
    }
}

// Loss of the blend head and its gradient with respect to the 4 logits
// (written as 16-channel bf16, channels 4..15 zero, the layout the last
// layer's backward consumes).
__global__ void k_loss(const i360b_blend_job* __restrict__ jobs, int n, int h, int w, const float4* __restrict__ logits,
                       float invCount, bf16* __restrict__ g8, double* __restrict__ lossAcc)
{
    __shared__ float red[32];
    const long long total = (long long)n * h * w;
    float lsum = 0.0f;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
    {
        const int img = (int)(idx / ((long long)h * w));
        const int rem = (int)(idx % ((long long)h * w));
        const int y = rem / w, x = rem % w;
        const i360b_blend_job& J = jobs[img];
        float dl[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) dl[j] = 0.0f;
        if (x < J.width && y < J.height)
        {
            const float4 lv = logits[idx];
            const float l[4] = {lv.x, lv.y, lv.z, lv.w};
            float o[3], wts[4], v[4][3];
            bool cov[4];
            int nCov;
            composite_pixel(J, y, x, l, o, wts, v, cov, nCov);
            const unsigned short* tp = J.target + (long long)y * J.targetRowStride + (long long)x * 3;
            float d[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
                const float e = (o[c] - (float)tp[c]) * kInScale;
                lsum += e * e;
                d[c] = 2.0f * e * invCount;
            }
#pragma unroll
            for (int i = 0; i < kSlots; ++i)
            {
                if (!cov[i]) continue;
                float s = 0.0f;
#pragma unroll
                for (int c = 0; c < 3; ++c) s += d[c] * (v[i][c] - o[c]) * kInScale;
                dl[i] = wts[i] * s;
            }
        }
        uint4* q = reinterpret_cast<uint4*>(g8 + idx * 16);
        q[0] = pack8_bf16(dl);
        q[1] = pack8_bf16(dl + 8);
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lsum;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) atomicAdd(lossAcc, (double)v * invCount);
    }
}

// db[c] += sum over pixels of g[p][c], c < cout (g has C = 8 * c8n channels).
__global__ void k_bias_grad(const bf16* __restrict__ g, long long pixels, int c8n, int cout, float* __restrict__ db)
{
    __shared__ float red[256 * 8];
    const int lanes = blockDim.x / c8n;
    const int c8 = threadIdx.x % c8n, lane = threadIdx.x / c8n;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (lane < lanes)
        for (long long p = (long long)blockIdx.x * lanes + lane; p < pixels; p += (long long)gridDim.x * lanes)
        {
            float v[8];
            unpack8_bf16(reinterpret_cast<const uint4*>(g + p * c8n * 8)[c8], v);
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j] += v[j];
        }
#pragma unroll
    for (int j = 0; j < 8; ++j) red[threadIdx.x * 8 + j] = lane < lanes ? acc[j] : 0.0f;
    __syncthreads();
    const int C = c8n * 8;
    if ((int)threadIdx.x < C && (int)threadIdx.x < cout)
    {
        const int cc8 = threadIdx.x >> 3, j = threadIdx.x & 7;
        float s = 0.0f;
        for (int l = 0; l < lanes; ++l) s += red[(l * c8n + cc8) * 8 + j];
        atomicAdd(&db[threadIdx.x], s);
    }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int count, float lr, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
}

// Network layer table.
struct LayerDef
{
    int cin, cout;
};
constexpr LayerDef kNet[8] = {{16, 32}, {32, 32}, {32, 64}, {64, 64}, {64, 64}, {96, 32}, {32, 32}, {32, 4}};
constexpr int kNumLayers = 8;

__host__ __device__ constexpr int pad16(int c) { return (c + 15) / 16 * 16; }

struct PackArgs
{
    const float* params;
    int cin[kNumLayers], cout[kNumLayers];
    long long wOff[kNumLayers], bOff[kNumLayers];
    bf16* fwd[kNumLayers];    // [pad16(cout)][9 * cin]
    bf16* dgrad[kNumLayers];  // [cin][9 * pad16(cout)] flipped, transposed
    float* bias[kNumLayers];  // [pad16(cout)]
};

// Packs the fp32 master parameters into the bf16 operands of the forward and
// backward-data convolutions (blockIdx.y = layer).
__global__ void k_pack_weights(PackArgs a)
{
    const int l = blockIdx.y;
    const int cin = a.cin[l], cout = a.cout[l], np = pad16(cout);
    const int K = 9 * cin, Kd = 9 * np;
    const float* W = a.params + a.wOff[l];
    const int nf = np * K, nd = cin * Kd;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf + nd + np; i += gridDim.x * blockDim.x)
    {
        if (i < nf)
        {
            const int n = i / K, k = i % K;
            a.fwd[l][i] = __float2bfloat16_rn(n < cout ? W[(size_t)n * K + k] : 0.0f);
        }
        else if (i < nf + nd)
        {
            const int j = i - nf, ci = j / Kd, kd = j % Kd, tap = kd / np, co = kd % np;
            a.dgrad[l][j] = __float2bfloat16_rn(co < cout ? W[(size_t)co * K + (8 - tap) * cin + ci] : 0.0f);
        }
        else
        {
            const int c = i - nf - nd;
            a.bias[l][c] = c < cout ? a.params[a.bOff[l] + c] : 0.0f;
        }
    }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
int grid_for(long long work, int perSm)
{
    const long long cap = (long long)sm_count() * perSm;
    return (int)std::max<long long>(1, std::min<long long>(work, cap));
}

int elementwise_grid(long long n, int block = 256)
{
    return (int)std::max<long long>(1, std::min<long long>((n + block - 1) / block, (long long)sm_count() * 16));
}

// Tensor map of an NHWC bf16 tensor as (C, W, H, N) with a box of 8
// channels x boxW x boxH x 1 (zero fill outside).  The encoder comes from the
// driver through the runtime (no link against the driver library).
int make_input_map(CUtensorMap* m, const bf16* base, int c, int n, int h, int w, int boxW, int boxH)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        err = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", reinterpret_cast<void**>(&encode), 12000,
                                               cudaEnableDefault, &q);
        if (err == cudaSuccess && q != cudaDriverEntryPointSuccess) err = cudaErrorSymbolNotFound;
    });
    if (err != cudaSuccess || !encode) return cuda_fail(err, "cuTensorMapEncodeTiled entry point");
    if ((reinterpret_cast<uintptr_t>(base) & 15) || c % 8)
        return fail(I360B_INVALID_PARAM, "conv3x3 input must be 16-byte aligned with channels a multiple of 8");
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)w * c * 2, (cuuint64_t)h * w * c * 2};
    const cuuint32_t box[4] = {8, (cuuint32_t)boxW, (cuuint32_t)boxH, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(I360B_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return I360B_SUCCESS;
}

template <int CIN, int NPAD, int TW, int TH, int STAGES, int LD, int EP, int EW>
int run_conv(const ConvArgs& a, cudaStream_t s)
{
    using S = ConvShape<CIN, NPAD, TW, TH, STAGES, LD, EW>;
    static std::once_flag once;
    static int perSm = 1;
    static cudaError_t attrErr = cudaSuccess;
    std::call_once(once, [] {
        auto* k = k_conv3x3<CIN, NPAD, TW, TH, STAGES, LD, EP, EW>;
        attrErr = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmem);
        int occ = 1;
        if (attrErr == cudaSuccess)
            attrErr = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, S::kThreads, S::kSmem);
        perSm = std::max(1, std::min<int>(occ, 512 / (int)S::kTmem));
    });
    if (attrErr != cudaSuccess) return cuda_fail(attrErr, "conv3x3 attributes");
    const long long tiles = (long long)a.n * ((a.h + TH - 1) / TH) * ((a.w + TW - 1) / TW);
    if (tiles == 0) return I360B_SUCCESS;
    CUtensorMap tm, th;
    I360B_TRY(make_input_map(&tm, a.x, LD == LD_CONCAT ? a.cs : CIN, a.n, a.h, a.w, TW + 2, TH + 2));
    if (LD == LD_CONCAT)
    {
        if (a.cs % 8 || a.h % 2 || a.w % 2 || CIN - a.cs > 8 * S::kC8)
            return fail(I360B_INVALID_PARAM, "concatenated conv3x3 input: even sizes and 8-channel groups");
        I360B_TRY(make_input_map(&th, a.u, CIN - a.cs, a.n, a.h / 2, a.w / 2, TW / 2 + 2, TH / 2 + 2));
    }
    else
        th = tm;
    k_conv3x3<CIN, NPAD, TW, TH, STAGES, LD, EP, EW><<<grid_for(tiles, perSm), S::kThreads, S::kSmem, s>>>(tm, th, a);
    return check_launch("conv3x3 kernel");
}

// The (cin, npad) shapes the network uses, forward and backward, with their
// tile shape and ring depth.
int dispatch_conv(int cin, int npad, int loader, int ep, const ConvArgs& a, cudaStream_t s)
{
#define I360B_CONV(CI, NP, TW, TH, ST, LD, EP_, EW)             \
    if (cin == CI && npad == NP && loader == LD && ep == EP_) \
        return run_conv<CI, NP, TW, TH, ST, LD, EP_, EW>(a, s);
    // forward
    I360B_CONV(16, 32, 32, 32, 3, LD_PLAIN, EP_RELU, 8)
    I360B_CONV(32, 32, 16, 32, 3, LD_PLAIN, EP_RELU, 8)
    I360B_CONV(32, 64, 16, 32, 3, LD_PLAIN, EP_RELU, 8)
    I360B_CONV(64, 64, 16, 16, 3, LD_PLAIN, EP_RELU, 8)
    I360B_CONV(96, 32, 16, 16, 2, LD_CONCAT, EP_RELU, 8)
    I360B_CONV(32, 16, 32, 32, 2, LD_PLAIN, EP_LOGITS, 8)
    I360B_CONV(32, 16, 32, 32, 2, LD_PLAIN, EP_COMPOSITE, 8)
    // backward data
    I360B_CONV(16, 32, 32, 32, 3, LD_PLAIN, EP_MASK, 8)
    I360B_CONV(32, 32, 16, 32, 3, LD_PLAIN, EP_MASK, 8)
    I360B_CONV(32, 96, 16, 16, 3, LD_PLAIN, EP_RAW, 8)
    I360B_CONV(64, 64, 16, 16, 3, LD_PLAIN, EP_MASK, 8)
    I360B_CONV(64, 32, 16, 16, 3, LD_PLAIN, EP_RAW, 8)
#undef I360B_CONV
    return fail(I360B_NOT_SUPPORTED, "conv3x3: no kernel for cin=%d cout=%d loader=%d epilogue=%d", cin, npad, loader,
                ep);
}

template <int CIN, int COUT, int LD>
int run_wgrad(const WgradArgs& base, float* dw, int cout, void* scratch, size_t scratchBytes, cudaStream_t s)
{
    using S = WgradShape<CIN, COUT>;
    static std::once_flag once;
    static int perSm = 1;
    static cudaError_t attrErr = cudaSuccess;
    std::call_once(once, [] {
        attrErr = cudaFuncSetAttribute(k_conv3x3_wgrad<CIN, COUT, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)S::kSmem);
        int occ = 1;
        if (attrErr == cudaSuccess)
            attrErr = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_conv3x3_wgrad<CIN, COUT, LD>, 128, S::kSmem);
        perSm = std::max(1, std::min<int>(std::min(occ, 2), 512 / (int)S::kTmem));
    });
    if (attrErr != cudaSuccess) return cuda_fail(attrErr, "wgrad attributes");
    const long long tiles = (long long)base.n * base.h * (base.w / kTileX);
    const int slices = (int)std::max<long long>(
        1, std::min<long long>(tiles, (long long)sm_count() * perSm / S::kChunks));
    const size_t need = (size_t)slices * S::kChunks * 128 * COUT * sizeof(float);
    if (need > scratchBytes) return fail(I360B_OUT_OF_MEMORY, "wgrad scratch too small (%zu > %zu)", need, scratchBytes);
    WgradArgs a = base;
    a.partial = static_cast<float*>(scratch);
    k_conv3x3_wgrad<CIN, COUT, LD><<<dim3(slices, S::kChunks), 128, S::kSmem, s>>>(a);
    I360B_TRY(check_launch("wgrad kernel"));
    const int total = 9 * CIN * cout;
    k_wgrad_reduce<<<(total + 255) / 256, 256, 0, s>>>(a.partial, slices, S::kChunks * 128, COUT, CIN, cout, dw);
    return check_launch("wgrad reduce kernel");
}

size_t wgrad_scratch_bytes()
{
    // Upper bound over the supported shapes: slices <= 2 * SMs / chunks.
    size_t mx = 0;
    const int sms = sm_count();
    auto f = [&](int cin, int cout) {
        const int chunks = (9 * cin / 8 + 15) / 16;
        const size_t slices = std::max(1, 2 * sms / chunks);
        mx = std::max(mx, slices * chunks * 128 * cout * sizeof(float));
    };
    f(16, 32), f(32, 32), f(32, 64), f(64, 64), f(96, 32), f(32, 16);
    return mx;
}

int dispatch_wgrad(int cin, int cout, int loader, const WgradArgs& a, float* dw, int coutReal, void* scratch,
                   size_t bytes, cudaStream_t s)
{
#define I360B_WG(CI, CO, LD) \
    if (cin == CI && cout == CO && loader == LD) return run_wgrad<CI, CO, LD>(a, dw, coutReal, scratch, bytes, s);
    I360B_WG(16, 32, LD_PLAIN)
    I360B_WG(32, 32, LD_PLAIN)
    I360B_WG(32, 64, LD_PLAIN)
    I360B_WG(64, 64, LD_PLAIN)
    I360B_WG(96, 32, LD_CONCAT)
    I360B_WG(32, 16, LD_PLAIN)
#undef I360B_WG
    return fail(I360B_NOT_SUPPORTED, "conv3x3 wgrad: no kernel for cin=%d cout=%d loader=%d", cin, cout, loader);
}

int check_window(int n, int w, int h)
{
    if (n <= 0 || w <= 0 || h <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    if (w % 256 != 0 || h % 2 != 0)
        return fail(I360B_INVALID_PARAM, "blend network windows need width %% 256 == 0 and even height (got %dx%d)", w,
                    h);
    return I360B_SUCCESS;
}
}  // namespace

// ---------------------------------------------------------------------------
// The network object
// ---------------------------------------------------------------------------
struct BlendNet
{
    int device = 0;
    long long wOff[kNumLayers], bOff[kNumLayers];
    int nParams = 0;
    float* params = nullptr;
    float* grads = nullptr;
    float* adamM = nullptr;
    float* adamV = nullptr;
    bf16* packed = nullptr;  // forward and backward-data weights of all layers
    float* biasPacked = nullptr;
    bf16* fwdW[kNumLayers];
    bf16* dgW[kNumLayers];
    float* bias[kNumLayers];
    int step = 0;
    // Per-batch buffers (grown on demand).
    size_t capPix = 0;
    bool capTraining = false;
    char* act = nullptr;
    bf16 *x0 = nullptr, *a1 = nullptr, *a2 = nullptr, *p2 = nullptr, *a3 = nullptr, *a4 = nullptr, *a5 = nullptr,
         *a6 = nullptr, *a7 = nullptr;
    float* logits = nullptr;
    bf16 *g8 = nullptr, *gA = nullptr, *gB = nullptr, *du = nullptr, *gh1 = nullptr, *gh2 = nullptr, *dp = nullptr;
    void* wgScratch = nullptr;
    size_t wgBytes = 0;
    double* dLoss = nullptr;
    int* dError = nullptr;
    i360b_blend_job* dJobs = nullptr;
    i360b_blend_job* hJobs = nullptr;  // pinned staging
    int jobCap = 0;
    cudaEvent_t jobsUploaded = nullptr;
    // Recorded at the end of every call on the caller's stream; the next call
    // (possibly on another stream) waits for it, because all calls share the
    // activation buffers and the job table.
    cudaEvent_t lastUse = nullptr;
    std::mutex mu;

    int begin(cudaStream_t s)
    {
        I360B_CUDA(cudaStreamWaitEvent(s, lastUse, 0), "blend network ordering");
        return I360B_SUCCESS;
    }
    int end(cudaStream_t s, int rc)
    {
        cudaEventRecord(lastUse, s);
        return rc;
    }

    ~BlendNet()
    {
        cudaFree(params);
        cudaFree(grads);
        cudaFree(adamM);
        cudaFree(adamV);
        cudaFree(packed);
        cudaFree(biasPacked);
        cudaFree(act);
        cudaFree(wgScratch);
        cudaFree(dLoss);
        cudaFree(dError);
        cudaFree(dJobs);
        if (hJobs) cudaFreeHost(hJobs);
        if (jobsUploaded) cudaEventDestroy(jobsUploaded);
        if (lastUse) cudaEventDestroy(lastUse);
    }

    int init(unsigned long long seed)
    {
        long long off = 0;
        for (int l = 0; l < kNumLayers; ++l)
        {
            wOff[l] = off;
            off += 9LL * kNet[l].cin * kNet[l].cout;
            bOff[l] = off;
            off += kNet[l].cout;
        }
        nParams = (int)off;
        const size_t pb = (size_t)nParams * sizeof(float);
        I360B_CUDA(cudaMalloc(&params, pb), "blendnet params");
        I360B_CUDA(cudaMalloc(&grads, pb), "blendnet grads");
        I360B_CUDA(cudaMalloc(&adamM, pb), "blendnet adam");
        I360B_CUDA(cudaMalloc(&adamV, pb), "blendnet adam");
        I360B_CUDA(cudaMemset(adamM, 0, pb), "blendnet adam");
        I360B_CUDA(cudaMemset(adamV, 0, pb), "blendnet adam");
        size_t pk = 0, bk = 0;
        for (int l = 0; l < kNumLayers; ++l)
        {
            pk += (size_t)pad16(kNet[l].cout) * 9 * kNet[l].cin + (size_t)kNet[l].cin * 9 * pad16(kNet[l].cout);
            bk += pad16(kNet[l].cout);
        }
        I360B_CUDA(cudaMalloc(&packed, pk * sizeof(bf16)), "blendnet packed weights");
        I360B_CUDA(cudaMalloc(&biasPacked, bk * sizeof(float)), "blendnet packed bias");
        size_t o = 0, ob = 0;
        for (int l = 0; l < kNumLayers; ++l)
        {
            fwdW[l] = packed + o;
            o += (size_t)pad16(kNet[l].cout) * 9 * kNet[l].cin;
            dgW[l] = packed + o;
            o += (size_t)kNet[l].cin * 9 * pad16(kNet[l].cout);
            bias[l] = biasPacked + ob;
            ob += pad16(kNet[l].cout);
        }
        wgBytes = wgrad_scratch_bytes();
        I360B_CUDA(cudaMalloc(&wgScratch, wgBytes), "blendnet wgrad scratch");
        I360B_CUDA(cudaMalloc(&dLoss, sizeof(double)), "blendnet loss");
        I360B_CUDA(cudaMalloc(&dError, sizeof(int)), "blendnet error flag");
        I360B_CUDA(cudaMemset(dError, 0, sizeof(int)), "blendnet error flag");
        I360B_CUDA(cudaEventCreateWithFlags(&jobsUploaded, cudaEventDisableTiming), "blendnet event");
        I360B_CUDA(cudaEventCreateWithFlags(&lastUse, cudaEventDisableTiming), "blendnet event");
        I360B_CUDA(cudaEventRecord(lastUse, nullptr), "blendnet event");
        // He-normal weights, zero biases, zero last layer (the untrained head
        // is then the coverage-weighted mean of the layers).
        std::vector<float> h(nParams, 0.0f);
        std::mt19937_64 rng(seed);
        std::normal_distribution<float> nd(0.0f, 1.0f);
        for (int l = 0; l < kNumLayers - 1; ++l)
        {
            const float sd = std::sqrt(2.0f / (9.0f * kNet[l].cin));
            for (long long i = 0; i < 9LL * kNet[l].cin * kNet[l].cout; ++i) h[wOff[l] + i] = nd(rng) * sd;
        }
        return upload(h.data());
    }

    int upload(const float* host)
    {
        I360B_CUDA(cudaMemcpy(params, host, (size_t)nParams * sizeof(float), cudaMemcpyHostToDevice), "param upload");
        return pack(nullptr);
    }

    int pack(cudaStream_t s)
    {
        PackArgs a;
        a.params = params;
        for (int l = 0; l < kNumLayers; ++l)
        {
            a.cin[l] = kNet[l].cin;
            a.cout[l] = kNet[l].cout;
            a.wOff[l] = wOff[l];
            a.bOff[l] = bOff[l];
            a.fwd[l] = fwdW[l];
            a.dgrad[l] = dgW[l];
            a.bias[l] = bias[l];
        }
        k_pack_weights<<<dim3(64, kNumLayers), 256, 0, s>>>(a);
        return check_launch("weight pack kernel");
    }

    // Activation buffers for n windows of w x h; the backward buffers only
    // when training.
    int reserve(int n, int w, int h, bool training)
    {
        const size_t pix = (size_t)n * w * h;
        if (pix <= capPix && (!training || capTraining)) return I360B_SUCCESS;
        cudaDeviceSynchronize();
        cudaFree(act);
        act = nullptr;
        capPix = 0;
        const size_t half = pix / 4;
        const size_t tr = training ? 1 : 0;
        // bf16 element counts of every buffer, then the fp32 logits.
        const size_t counts[] = {pix * 16,       pix * 32,       pix * 32,       half * 32,      half * 64,
                                 half * 64,      half * 64,      pix * 32,       pix * 32,       tr * pix * 16,
                                 tr * pix * 32,  tr * pix * 32,  tr * pix * 96,  tr * half * 64, tr * half * 64,
                                 tr * half * 32};
        size_t total = 0;
        for (size_t c : counts) total += (c * sizeof(bf16) + 255) / 256 * 256;
        total += pix * 4 * sizeof(float);
        cudaError_t e = cudaMalloc(&act, total);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            act = nullptr;
            return fail(I360B_OUT_OF_MEMORY, "blend network: %zu bytes of activations for %d windows of %dx%d", total,
                        n, w, h);
        }
        bf16** slots[] = {&x0, &a1, &a2, &p2, &a3, &a4, &a5, &a6, &a7, &g8, &gA, &gB, &du, &gh1, &gh2, &dp};
        size_t o = 0;
        for (size_t i = 0; i < sizeof(counts) / sizeof(counts[0]); ++i)
        {
            *slots[i] = reinterpret_cast<bf16*>(act + o);
            o += (counts[i] * sizeof(bf16) + 255) / 256 * 256;
        }
        logits = reinterpret_cast<float*>(act + o);
        capPix = pix;
        capTraining = training;
        return I360B_SUCCESS;
    }

    int upload_jobs(const i360b_blend_job* jobs, int n, cudaStream_t s)
    {
        if (!jobs) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
        if (n > jobCap)
        {
            cudaDeviceSynchronize();
            cudaFree(dJobs);
            if (hJobs) cudaFreeHost(hJobs);
            dJobs = nullptr;
            hJobs = nullptr;
            jobCap = 0;
            I360B_CUDA(cudaMalloc(&dJobs, (size_t)n * sizeof(i360b_blend_job)), "blend jobs");
            I360B_CUDA(cudaMallocHost(&hJobs, (size_t)n * sizeof(i360b_blend_job)), "blend jobs");
            jobCap = n;
        }
        else
        {
            I360B_CUDA(cudaEventSynchronize(jobsUploaded), "blend jobs");
        }
        std::memcpy(hJobs, jobs, (size_t)n * sizeof(i360b_blend_job));
        I360B_CUDA(cudaMemcpyAsync(dJobs, hJobs, (size_t)n * sizeof(i360b_blend_job), cudaMemcpyHostToDevice, s),
                   "blend jobs");
        I360B_CUDA(cudaEventRecord(jobsUploaded, s), "blend jobs");
        return I360B_SUCCESS;
    }

    ConvArgs conv(const bf16* x, int n, int w, int h, int l, void* out, const i360b_blend_job* jobs) const
    {
        ConvArgs a{};
        a.x = x;
        a.n = n;
        a.h = h;
        a.w = w;
        a.wt = fwdW[l];
        a.bias = bias[l];
        a.out = out;
        a.jobs = jobs;
        a.error = dError;
        return a;
    }

    // Forward pass over the windows jobs[0..n); the last layer writes logits
    // (training) or the blended output (composite).  With `ev` non-null,
    // records ev[i] before kernel i and ev[kForwardKernels] after the last.
    static constexpr int kForwardKernels = 10;
    int forward(const i360b_blend_job* jobs, int n, int w, int h, bool composite, cudaStream_t s,
                cudaEvent_t* ev = nullptr)
    {
        const int hw = w / 2, hh = h / 2;
        auto mark = [&](int i) {
            if (ev) cudaEventRecord(ev[i], s);
        };
        mark(0);
        k_pack_input<<<elementwise_grid((long long)n * w * h), 256, 0, s>>>(jobs, n, h, w, x0);
        I360B_TRY(check_launch("input pack kernel"));
        mark(1);
        I360B_TRY(dispatch_conv(16, 32, LD_PLAIN, EP_RELU, conv(x0, n, w, h, 0, a1, jobs), s));
        mark(2);
        I360B_TRY(dispatch_conv(32, 32, LD_PLAIN, EP_RELU, conv(a1, n, w, h, 1, a2, jobs), s));
        mark(3);
        k_pool2<<<elementwise_grid((long long)n * hw * hh * 4), 256, 0, s>>>(a2, n, h, w, 4, p2);
        I360B_TRY(check_launch("pool kernel"));
        mark(4);
        I360B_TRY(dispatch_conv(32, 64, LD_PLAIN, EP_RELU, conv(p2, n, hw, hh, 2, a3, jobs), s));
        mark(5);
        I360B_TRY(dispatch_conv(64, 64, LD_PLAIN, EP_RELU, conv(a3, n, hw, hh, 3, a4, jobs), s));
        mark(6);
        I360B_TRY(dispatch_conv(64, 64, LD_PLAIN, EP_RELU, conv(a4, n, hw, hh, 4, a5, jobs), s));
        mark(7);
        ConvArgs c6 = conv(a2, n, w, h, 5, a6, jobs);
        c6.u = a5;
        c6.cs = 32;
        I360B_TRY(dispatch_conv(96, 32, LD_CONCAT, EP_RELU, c6, s));
        mark(8);
        I360B_TRY(dispatch_conv(32, 32, LD_PLAIN, EP_RELU, conv(a6, n, w, h, 6, a7, jobs), s));
        mark(9);
        if (composite) I360B_TRY(dispatch_conv(32, 16, LD_PLAIN, EP_COMPOSITE, conv(a7, n, w, h, 7, nullptr, jobs), s));
        else I360B_TRY(dispatch_conv(32, 16, LD_PLAIN, EP_LOGITS, conv(a7, n, w, h, 7, logits, jobs), s));
        mark(10);
        return I360B_SUCCESS;
    }

    // Backward data through layer l (flipped, transposed weights).
    int dgrad(int l, const bf16* g, int n, int w, int h, const bf16* actMask, void* out, int ep, cudaStream_t s)
    {
        ConvArgs a{};
        a.x = g;
        a.n = n;
        a.h = h;
        a.w = w;
        a.wt = dgW[l];
        a.out = out;
        a.act = actMask;
        a.error = dError;
        return dispatch_conv(pad16(kNet[l].cout), kNet[l].cin, LD_PLAIN, ep, a, s);
    }

    int wgrad(int l, const bf16* x, const bf16* u, int cs, const bf16* g, int n, int w, int h, cudaStream_t s)
    {
        WgradArgs a{};
        a.x = x;
        a.u = u;
        a.cs = cs;
        a.g = g;
        a.n = n;
        a.h = h;
        a.w = w;
        a.error = dError;
        I360B_TRY(dispatch_wgrad(kNet[l].cin, pad16(kNet[l].cout), cs ? LD_CONCAT : LD_PLAIN, a, grads + wOff[l],
                                 kNet[l].cout, wgScratch, wgBytes, s));
        const long long pixels = (long long)n * w * h;
        const int c8n = pad16(kNet[l].cout) / 8;
        k_bias_grad<<<std::min<long long>(sm_count() * 4, (pixels + 255) / 256), 256, 0, s>>>(g, pixels, c8n,
                                                                                              kNet[l].cout,
                                                                                              grads + bOff[l]);
        return check_launch("bias gradient kernel");
    }

    // Loss, then every parameter gradient into `grads`.
    int backward(int n, int w, int h, cudaStream_t s)
    {
        const int hw = w / 2, hh = h / 2;
        const long long pix = (long long)n * w * h;
        I360B_CUDA(cudaMemsetAsync(dLoss, 0, sizeof(double), s), "loss reset");
        I360B_CUDA(cudaMemsetAsync(grads, 0, (size_t)nParams * sizeof(float), s), "grad reset");
        k_loss<<<elementwise_grid(pix), 256, 0, s>>>(dJobs, n, h, w, reinterpret_cast<const float4*>(logits),
                                                   (float)(1.0 / (3.0 * (double)pix)), g8, dLoss);
        I360B_TRY(check_launch("loss kernel"));
        // layer 8 (32 -> 4): input a7
        I360B_TRY(wgrad(7, a7, nullptr, 0, g8, n, w, h, s));
        I360B_TRY(dgrad(7, g8, n, w, h, a7, gA, EP_MASK, s));  // gA = g7
        // layer 7 (32 -> 32): input a6
        I360B_TRY(wgrad(6, a6, nullptr, 0, gA, n, w, h, s));
        I360B_TRY(dgrad(6, gA, n, w, h, a6, gB, EP_MASK, s));  // gB = g6
        // layer 6 (96 -> 32): input concat(a2, up(a5))
        I360B_TRY(wgrad(5, a2, a5, 32, gB, n, w, h, s));
        I360B_TRY(dgrad(5, gB, n, w, h, nullptr, du, EP_RAW, s));
        k_upsample_grad<<<elementwise_grid((long long)n * hw * hh * 8), 256, 0, s>>>(du, 96, 32, a5, n, h, w, 8, gh1);
        I360B_TRY(check_launch("upsample gradient kernel"));  // gh1 = g5
        // layer 5 (64 -> 64): input a4
        I360B_TRY(wgrad(4, a4, nullptr, 0, gh1, n, hw, hh, s));
        I360B_TRY(dgrad(4, gh1, n, hw, hh, a4, gh2, EP_MASK, s));  // gh2 = g4
        // layer 4 (64 -> 64): input a3
        I360B_TRY(wgrad(3, a3, nullptr, 0, gh2, n, hw, hh, s));
        I360B_TRY(dgrad(3, gh2, n, hw, hh, a3, gh1, EP_MASK, s));  // gh1 = g3
        // layer 3 (32 -> 64): input p2
        I360B_TRY(wgrad(2, p2, nullptr, 0, gh1, n, hw, hh, s));
        I360B_TRY(dgrad(2, gh1, n, hw, hh, nullptr, dp, EP_RAW, s));  // dp = d(pool)
        k_skip_grad<<<elementwise_grid(pix * 4), 256, 0, s>>>(du, 96, dp, a2, n, h, w, 4, gA);
        I360B_TRY(check_launch("skip gradient kernel"));  // gA = g2
        // layer 2 (32 -> 32): input a1
        I360B_TRY(wgrad(1, a1, nullptr, 0, gA, n, w, h, s));
        I360B_TRY(dgrad(1, gA, n, w, h, a1, gB, EP_MASK, s));  // gB = g1
        // layer 1 (16 -> 32): input x0
        return wgrad(0, x0, nullptr, 0, gB, n, w, h, s);
    }

    int adam(float lr, cudaStream_t s)
    {
        ++step;
        const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, step)));
        const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, step)));
        k_adam<<<(nParams + 255) / 256, 256, 0, s>>>(params, grads, adamM, adamV, nParams, lr, c1, c2);
        I360B_TRY(check_launch("adam kernel"));
        return pack(s);
    }

    int check_error(cudaStream_t s)
    {
        int e = 0;
        I360B_CUDA(cudaMemcpyAsync(&e, dError, sizeof(int), cudaMemcpyDeviceToHost, s), "error flag");
        I360B_CUDA(cudaStreamSynchronize(s), "blend network");
        if (e)
        {
            cudaMemsetAsync(dError, 0, sizeof(int), s);
            return fail(I360B_KERNEL_LAUNCH_FAILED, "a tensor-core convolution gave up waiting for its MMAs");
        }
        return I360B_SUCCESS;
    }
};
}  // namespace i360b

struct i360b_blendnet
{
    i360b::BlendNet net;
};

using namespace i360b;

namespace
{
int net_prologue(i360b_blendnet* net)
{
    clear_error();
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    if (!net) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    return I360B_SUCCESS;
}
}  // namespace

extern "C" int i360b_blendnet_param_count(void)
{
    int n = 0;
    for (int l = 0; l < kNumLayers; ++l) n += 9 * kNet[l].cin * kNet[l].cout + kNet[l].cout;
    return n;
}

extern "C" int i360b_blendnet_create(unsigned long long seed, i360b_blendnet** outNet)
{
    clear_error();
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    if (!outNet) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    *outNet = nullptr;
    auto* p = new (std::nothrow) i360b_blendnet;
    if (!p) return fail(I360B_OUT_OF_MEMORY, "blend network: host allocation failed");
    int rc = p->net.init(seed);
    if (rc != I360B_SUCCESS)
    {
        delete p;
        return rc;
    }
    I360B_CUDA(cudaDeviceSynchronize(), "blend network init");
    *outNet = p;
    return I360B_SUCCESS;
}

extern "C" void i360b_blendnet_destroy(i360b_blendnet* net)
{
    if (!net) return;
    cudaDeviceSynchronize();
    delete net;
}

extern "C" int i360b_blendnet_get_params(i360b_blendnet* net, float* hostParams, int count)
{
    I360B_TRY(net_prologue(net));
    if (!hostParams || count != net->net.nParams) return fail(I360B_INVALID_PARAM, "parameter count mismatch");
    I360B_CUDA(cudaDeviceSynchronize(), "blend network");
    I360B_CUDA(cudaMemcpy(hostParams, net->net.params, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost),
               "param download");
    return I360B_SUCCESS;
}

extern "C" int i360b_blendnet_set_params(i360b_blendnet* net, const float* hostParams, int count)
{
    I360B_TRY(net_prologue(net));
    if (!hostParams || count != net->net.nParams) return fail(I360B_INVALID_PARAM, "parameter count mismatch");
    I360B_CUDA(cudaDeviceSynchronize(), "blend network");
    I360B_TRY(net->net.upload(hostParams));
    I360B_CUDA(cudaDeviceSynchronize(), "blend network");
    return I360B_SUCCESS;
}

extern "C" int i360b_blendnet_get_adam(i360b_blendnet* net, float* hostM, float* hostV, int count, int* step)
{
    I360B_TRY(net_prologue(net));
    if (!hostM || !hostV || !step || count != net->net.nParams)
        return fail(I360B_INVALID_PARAM, "parameter count mismatch");
    BlendNet& N = net->net;
    std::lock_guard<std::mutex> lk(N.mu);
    I360B_CUDA(cudaDeviceSynchronize(), "blend network");
    I360B_CUDA(cudaMemcpy(hostM, N.adamM, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost), "adam download");
    I360B_CUDA(cudaMemcpy(hostV, N.adamV, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost), "adam download");
    *step = N.step;
    return I360B_SUCCESS;
}

extern "C" int i360b_blendnet_set_adam(i360b_blendnet* net, const float* hostM, const float* hostV, int count,
                                       int step)
{
    I360B_TRY(net_prologue(net));
    if (!hostM || !hostV || count != net->net.nParams || step < 0)
        return fail(I360B_INVALID_PARAM, "parameter count mismatch or negative step");
    BlendNet& N = net->net;
    std::lock_guard<std::mutex> lk(N.mu);
    I360B_CUDA(cudaDeviceSynchronize(), "blend network");
    I360B_CUDA(cudaMemcpy(N.adamM, hostM, (size_t)count * sizeof(float), cudaMemcpyHostToDevice), "adam upload");
    I360B_CUDA(cudaMemcpy(N.adamV, hostV, (size_t)count * sizeof(float), cudaMemcpyHostToDevice), "adam upload");
    N.step = step;
    return I360B_SUCCESS;
}

extern "C" int i360b_blendnet_logits(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                     float* dLogits)
{
    I360B_TRY(net_prologue(net));
    I360B_TRY(check_window(n, w, h));
    if (!dLogits) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    BlendNet& N = net->net;
    std::lock_guard<std::mutex> lk(N.mu);
    cudaStream_t s = thread_stream();
    I360B_TRY(N.begin(s));
    int rc = [&]() -> int {
        I360B_TRY(N.reserve(n, w, h, false));
        I360B_TRY(N.upload_jobs(jobs, n, s));
        I360B_TRY(N.forward(N.dJobs, n, w, h, false, s));
        I360B_CUDA(cudaMemcpyAsync(dLogits, N.logits, (size_t)n * w * h * 4 * sizeof(float), cudaMemcpyDeviceToDevice,
                                   s),
                   "logits copy");
        return N.check_error(s);
    }();
    return N.end(s, rc);
}

extern "C" int i360b_blendnet_gradients(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                        float* hostGrad, double* hostLoss)
{
    I360B_TRY(net_prologue(net));
    I360B_TRY(check_window(n, w, h));
    BlendNet& N = net->net;
    std::lock_guard<std::mutex> lk(N.mu);
    cudaStream_t s = thread_stream();
    I360B_TRY(N.begin(s));
    int rc = [&]() -> int {
        I360B_TRY(N.reserve(n, w, h, true));
        I360B_TRY(N.upload_jobs(jobs, n, s));
        I360B_TRY(N.forward(N.dJobs, n, w, h, false, s));
        I360B_TRY(N.backward(n, w, h, s));
        I360B_TRY(N.check_error(s));
        if (hostGrad)
            I360B_CUDA(cudaMemcpy(hostGrad, N.grads, (size_t)N.nParams * sizeof(float), cudaMemcpyDeviceToHost),
                       "grad download");
        if (hostLoss)
            I360B_CUDA(cudaMemcpy(hostLoss, N.dLoss, sizeof(double), cudaMemcpyDeviceToHost), "loss download");
        return I360B_SUCCESS;
    }();
    return N.end(s, rc);
}

extern "C" int i360b_blendnet_train_step(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                         float lr, double* hostLoss, void* stream)
{
    I360B_TRY(net_prologue(net));
    I360B_TRY(check_window(n, w, h));
    BlendNet& N = net->net;
    std::lock_guard<std::mutex> lk(N.mu);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    I360B_TRY(N.begin(s));
    int rc = [&]() -> int {
        I360B_TRY(N.reserve(n, w, h, true));
        I360B_TRY(N.upload_jobs(jobs, n, s));
        I360B_TRY(N.forward(N.dJobs, n, w, h, false, s));
        I360B_TRY(N.backward(n, w, h, s));
        I360B_TRY(N.adam(lr, s));
        if (hostLoss)
        {
            I360B_CUDA(cudaMemcpyAsync(hostLoss, N.dLoss, sizeof(double), cudaMemcpyDeviceToHost, s), "loss download");
            return N.check_error(s);
        }
        return I360B_SUCCESS;
    }();
    return N.end(s, rc);
}

extern "C" int i360b_blendnet_infer(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                    void* stream)
{
    I360B_TRY(net_prologue(net));
    I360B_TRY(check_window(n, w, h));
    BlendNet& N = net->net;
    std::lock_guard<std::mutex> lk(N.mu);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    I360B_TRY(N.begin(s));
    int rc = [&]() -> int {
        I360B_TRY(N.reserve(n, w, h, false));
        I360B_TRY(N.upload_jobs(jobs, n, s));
        return N.forward(N.dJobs, n, w, h, true, s);
    }();
    return N.end(s, rc);
}

extern "C" int i360b_blendnet_profile(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                      float* kernelMs, int maxKernels)
{
    I360B_TRY(net_prologue(net));
    I360B_TRY(check_window(n, w, h));
    if (!kernelMs) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    BlendNet& N = net->net;
    std::lock_guard<std::mutex> lk(N.mu);
    cudaStream_t s = thread_stream();
    I360B_TRY(N.begin(s));
    cudaEvent_t ev[BlendNet::kForwardKernels + 1] = {};
    int rc = [&]() -> int {
        for (auto& e : ev) I360B_CUDA(cudaEventCreate(&e), "profile events");
        I360B_TRY(N.reserve(n, w, h, false));
        I360B_TRY(N.upload_jobs(jobs, n, s));
        I360B_TRY(N.forward(N.dJobs, n, w, h, true, s, ev));
        I360B_CUDA(cudaEventSynchronize(ev[BlendNet::kForwardKernels]), "profile");
        for (int i = 0; i < BlendNet::kForwardKernels && i < maxKernels; ++i)
            cudaEventElapsedTime(&kernelMs[i], ev[i], ev[i + 1]);
        return N.check_error(s);
    }();
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    return N.end(s, rc);
}

extern "C" const char* i360b_blendnet_kernel_name(int i)
{
    static const char* const names[] = {"pack_input", "conv1_16_32",  "conv2_32_32", "pool",        "conv3_32_64",
                                        "conv4_64_64", "conv5_64_64", "conv6_96_32", "conv7_32_32", "conv8_32_4_blend"};
    return i >= 0 && i < 10 ? names[i] : nullptr;
}

extern "C" int i360b_conv3x3_forward(const void* dX, const void* dU, int skipChannels, int n, int h, int w, int cin,
                                     int cout, const void* dWeights, const float* dBias, int epilogue,
                                     const void* dAct, void* dOut, void* stream)
{
    clear_error();
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    if (!dX || !dWeights || !dOut || (skipChannels > 0 && !dU)) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (n <= 0 || h <= 0 || w <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    if ((epilogue == EP_RELU || epilogue == EP_LOGITS) && !dBias) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (epilogue == EP_MASK && !dAct) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (epilogue < EP_RELU || epilogue > EP_RAW) return fail(I360B_INVALID_PARAM, "unknown epilogue %d", epilogue);
    if (skipChannels > 0 && (h % 2 || w % 256 || skipChannels % 8 || skipChannels >= cin))
        return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    static int* dErr = nullptr;
    if (!dErr) I360B_CUDA(cudaMalloc(&dErr, sizeof(int)), "error flag");
    ConvArgs a{};
    a.x = static_cast<const bf16*>(dX);
    a.u = static_cast<const bf16*>(dU);
    a.cs = skipChannels;
    a.n = n;
    a.h = h;
    a.w = w;
    a.wt = static_cast<const bf16*>(dWeights);
    a.bias = dBias;
    a.out = dOut;
    a.act = static_cast<const bf16*>(dAct);
    a.error = dErr;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    I360B_CUDA(cudaMemsetAsync(dErr, 0, sizeof(int), s), "error flag");
    I360B_TRY(dispatch_conv(cin, cout, skipChannels > 0 ? LD_CONCAT : LD_PLAIN, epilogue, a, s));
    int e = 0;
    I360B_CUDA(cudaMemcpyAsync(&e, dErr, sizeof(int), cudaMemcpyDeviceToHost, s), "error flag");
    I360B_CUDA(cudaStreamSynchronize(s), "conv3x3");
    if (e) return fail(I360B_KERNEL_LAUNCH_FAILED, "conv3x3 gave up waiting for its MMAs");
    return I360B_SUCCESS;
}

extern "C" int i360b_conv3x3_wgrad(const void* dX, const void* dU, int skipChannels, const void* dGrad, int n, int h,
                                   int w, int cin, int cout, float* dGradW, void* stream)
{
    clear_error();
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    if (!dX || !dGrad || !dGradW || (skipChannels > 0 && !dU)) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (n <= 0 || h <= 0 || w <= 0 || w % kTileX != 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    if (skipChannels > 0 && (h % 2 || w % 256 || skipChannels % 8 || skipChannels >= cin))
        return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static int* dErr = nullptr;
    if (!dErr) I360B_CUDA(cudaMalloc(&dErr, sizeof(int)), "error flag");
    const size_t bytes = wgrad_scratch_bytes();
    void* scratch = nullptr;
    I360B_TRY(dev_alloc(&scratch, bytes, s, "wgrad scratch"));
    WgradArgs a{};
    a.x = static_cast<const bf16*>(dX);
    a.u = static_cast<const bf16*>(dU);
    a.cs = skipChannels;
    a.g = static_cast<const bf16*>(dGrad);
    a.n = n;
    a.h = h;
    a.w = w;
    a.error = dErr;
    I360B_CUDA(cudaMemsetAsync(dErr, 0, sizeof(int), s), "error flag");
    int rc = dispatch_wgrad(cin, cout, skipChannels > 0 ? LD_CONCAT : LD_PLAIN, a, dGradW, cout, scratch, bytes, s);
    int e = 0;
    cudaMemcpyAsync(&e, dErr, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    dev_free(scratch, s);
    if (rc != I360B_SUCCESS) return rc;
    if (e) return fail(I360B_KERNEL_LAUNCH_FAILED, "conv3x3 wgrad gave up waiting for its MMAs");
    return I360B_SUCCESS;
}

// ---------------------------------------------------------------------------
// Learned render of a plan's output tiles
// ---------------------------------------------------------------------------
namespace i360b
{
namespace
{
constexpr int kSub = 256;  // learned-blend window side

// Copy (src non-null) or clear a w x h RGB48 rectangle; strides in elements.
struct Region
{
    const unsigned short* src;
    unsigned short* dst;
    int w, h;
    long long srcRow, dstRow;
};

__global__ void k_regions(const Region* __restrict__ regs, int n)
{
    for (int r = blockIdx.y; r < n; r += gridDim.y)
    {
        const Region R = regs[r];
        const int vals = R.w * 3;
        for (int y = blockIdx.x; y < R.h; y += gridDim.x)
        {
            unsigned short* d = R.dst + y * R.dstRow;
            if (R.src)
            {
                const unsigned short* src = R.src + y * R.srcRow;
                for (int i = threadIdx.x; i < vals; i += blockDim.x) d[i] = src[i];
            }
            else
                for (int i = threadIdx.x; i < vals; i += blockDim.x) d[i] = 0;
        }
    }
}

// Per region: sum of squared differences and largest absolute difference
// between two RGB48 rectangles (src = learned, dst = plain).
__global__ void k_judge(const Region* __restrict__ regs, int n, double* __restrict__ sse, int* __restrict__ maxErr)
{
    __shared__ double rs[8];
    __shared__ int rm[8];
    for (int r = blockIdx.x; r < n; r += gridDim.x)
    {
        const Region R = regs[r];
        const int vals = R.w * 3;
        double acc = 0.0;
        int mx = 0;
        for (int y = 0; y < R.h; ++y)
        {
            const unsigned short* a = R.src + y * R.srcRow;
            const unsigned short* b = R.dst + y * R.dstRow;
            for (int i = threadIdx.x; i < vals; i += blockDim.x)
            {
                const int d = (int)a[i] - (int)b[i];
                acc += (double)d * d;
                mx = max(mx, abs(d));
            }
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            acc += __shfl_xor_sync(0xffffffffu, acc, o);
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if ((threadIdx.x & 31) == 0)
        {
            rs[threadIdx.x >> 5] = acc;
            rm[threadIdx.x >> 5] = mx;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double t = 0.0;
            int m = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            {
                t += rs[w];
                m = max(m, rm[w]);
            }
            sse[r] = t;
            maxErr[r] = m;
        }
        __syncthreads();
    }
}

int launch_regions(const std::vector<Region>& regs, Region* dRegs, cudaStream_t s)
{
    if (regs.empty()) return I360B_SUCCESS;
    I360B_CUDA(cudaMemcpyAsync(dRegs, regs.data(), regs.size() * sizeof(Region), cudaMemcpyHostToDevice, s),
               "region upload");
    k_regions<<<dim3(16, (unsigned)std::min<size_t>(regs.size(), 65535)), 256, 0, s>>>(dRegs, (int)regs.size());
    return check_launch("region copy kernel");
}

// Footprint box of an item intersects a rectangle (inclusive box ends).
bool box_hits(const ItemDev& it, int x0, int y0, int w, int h)
{
    return it.vx0 < x0 + w && it.vx1 >= x0 && it.vy0 < y0 + h && it.vy1 >= y0;
}

long long box_overlap(const ItemDev& it, int x0, int y0, int w, int h)
{
    const long long ix = std::max(0, std::min(it.vx1 + 1, x0 + w) - std::max(it.vx0, x0));
    const long long iy = std::max(0, std::min(it.vy1 + 1, y0 + h) - std::max(it.vy0, y0));
    return ix * iy;
}

void build_subtiles(Plan& P)
{
    if (!P.subTiles.empty()) return;
    for (int t = 0; t < P.nTiles; ++t)
    {
        const TileDev& T = P.tiles[t];
        for (int oy = 0; oy < T.h; oy += kSub)
            for (int ox = 0; ox < T.w; ox += kSub)
            {
                SubTile st{};
                st.tile = t;
                st.ox = ox;
                st.oy = oy;
                st.w = std::min(kSub, T.w - ox);
                st.h = std::min(kSub, T.h - oy);
                std::vector<std::pair<long long, int>> hits;
                for (int k = 0; k < T.numItems; ++k)
                {
                    const ItemDev& it = P.items[T.firstItem + k];
                    if (box_hits(it, ox, oy, st.w, st.h)) hits.push_back({box_overlap(it, ox, oy, st.w, st.h), k});
                }
                if (hits.size() > 4)
                {
                    st.overflow = 1;
                    std::stable_sort(hits.begin(), hits.end(),
                                     [](const auto& a, const auto& b) { return a.first > b.first; });
                    hits.resize(4);
                    std::sort(hits.begin(), hits.end(), [](const auto& a, const auto& b) { return a.second < b.second; });
                }
                for (int i = 0; i < 4; ++i) st.item[i] = i < (int)hits.size() ? T.firstItem + hits[i].second : -1;
                st.kind = hits.empty() ? 0 : hits.size() == 1 ? 1 : 2;
                P.subTiles.push_back(st);
            }
    }
}

// Device scratch of the learned render, per (plan, thread of use).
struct LearnedScratch
{
    i360b_blend_job* dJobs = nullptr;
    size_t jobCap = 0;
    Region* dRegs = nullptr;
    size_t regCap = 0;
    double* dSse = nullptr;
    int* dMax = nullptr;
    size_t judgeCap = 0;
    ~LearnedScratch()
    {
        cudaFree(dJobs);
        cudaFree(dRegs);
        cudaFree(dSse);
        cudaFree(dMax);
    }
    int jobs(size_t n)
    {
        if (n <= jobCap) return I360B_SUCCESS;
        cudaFree(dJobs);
        dJobs = nullptr;
        jobCap = 0;
        I360B_CUDA(cudaMalloc(&dJobs, std::max<size_t>(n, 1) * sizeof(i360b_blend_job)), "learned jobs");
        jobCap = n;
        return I360B_SUCCESS;
    }
    int regs(size_t n)
    {
        if (n <= regCap) return I360B_SUCCESS;
        cudaFree(dRegs);
        dRegs = nullptr;
        regCap = 0;
        I360B_CUDA(cudaMalloc(&dRegs, std::max<size_t>(n, 1) * sizeof(Region)), "learned regions");
        regCap = n;
        return I360B_SUCCESS;
    }
    int judge(size_t n)
    {
        if (n <= judgeCap) return I360B_SUCCESS;
        cudaFree(dSse);
        cudaFree(dMax);
        dSse = nullptr;
        dMax = nullptr;
        judgeCap = 0;
        I360B_CUDA(cudaMalloc(&dSse, std::max<size_t>(n, 1) * sizeof(double)), "judge");
        I360B_CUDA(cudaMalloc(&dMax, std::max<size_t>(n, 1) * sizeof(int)), "judge");
        judgeCap = n;
        return I360B_SUCCESS;
    }
};

std::mutex g_scratchMu;
std::vector<std::pair<const Plan*, LearnedScratch*>> g_scratch;

LearnedScratch& scratch_for(const Plan* p)
{
    std::lock_guard<std::mutex> lk(g_scratchMu);
    for (auto& e : g_scratch)
        if (e.first == p) return *e.second;
    g_scratch.push_back({p, new LearnedScratch});
    return *g_scratch.back().second;
}
}  // namespace

void release_learned_scratch(const Plan* p)
{
    std::lock_guard<std::mutex> lk(g_scratchMu);
    for (size_t i = 0; i < g_scratch.size(); ++i)
        if (g_scratch[i].first == p)
        {
            delete g_scratch[i].second;
            g_scratch.erase(g_scratch.begin() + i);
            return;
        }
}

int learned_render(Plan& P, BlendNet& N, unsigned short* const* tileOut, int maxBatch, cudaStream_t s, float* stageMs)
{
    if (!P.render) return fail(I360B_INVALID_PARAM, "learned render needs a render plan");
    build_subtiles(P);
    LearnedScratch& S = scratch_for(&P);
    auto outOf = [&](int t) { return tileOut ? tileOut[t] : P.tiles[t].out; };
    std::vector<i360b_blend_job> jobs;
    std::vector<Region> regs;
    for (const SubTile& st : P.subTiles)
    {
        const TileDev& T = P.tiles[st.tile];
        unsigned short* out = outOf(st.tile);
        if (!out) return fail(I360B_INVALID_PARAM, "Tile %d has a null learned output.", st.tile);
        const size_t off = ((size_t)st.oy * T.w + st.ox) * 3;
        if (st.kind == 2)
        {
            i360b_blend_job j{};
            for (int i = 0; i < 4; ++i) j.slot[i] = st.item[i] >= 0 ? P.items[st.item[i]].img + off : nullptr;
            for (int i = 0; i < 4; ++i)
                for (int e = 0; e < 4; ++e)
                {
                    const float* src = st.item[i] >= 0 ? &P.itemEdges[(size_t)st.item[i] * 16 + 4 * e] : nullptr;
                    float* d = &j.edges[i][4 * e];
                    if (!src)
                    {
                        d[0] = NAN;
                        d[1] = d[2] = d[3] = 0.0f;
                        continue;
                    }
                    d[0] = src[0] - st.ox;  // NaN stays NaN
                    d[1] = src[1] - st.oy;
                    d[2] = src[2] - st.ox;
                    d[3] = src[3] - st.oy;
                }
            j.pixStride = 3;
            j.rowStride = 3LL * T.w;
            j.width = st.w;
            j.height = st.h;
            j.out = out + off;
            j.outRowStride = 3LL * T.w;
            jobs.push_back(j);
        }
        else
        {
            regs.push_back(Region{st.kind == 1 ? P.items[st.item[0]].img + off : nullptr, out + off, st.w, st.h,
                                  3LL * T.w, 3LL * T.w});
        }
    }
    I360B_TRY(S.jobs(jobs.size()));
    I360B_TRY(S.regs(regs.size()));
    cudaEvent_t ev[4] = {};
    if (stageMs)
        for (auto& e : ev) I360B_CUDA(cudaEventCreate(&e), "stage events");
    auto mark = [&](int i) {
        if (stageMs) cudaEventRecord(ev[i], s);
    };
    mark(0);
    I360B_TRY(P.enqueue_warp(s));
    mark(1);
    I360B_TRY(launch_regions(regs, S.dRegs, s));
    mark(2);
    if (!jobs.empty())
    {
        I360B_CUDA(cudaMemcpyAsync(S.dJobs, jobs.data(), jobs.size() * sizeof(i360b_blend_job), cudaMemcpyHostToDevice,
                                   s),
                   "learned jobs upload");
        const int batch = std::max(1, std::min<int>(maxBatch, (int)jobs.size()));
        I360B_TRY(N.reserve(batch, kSub, kSub, false));
        for (size_t b = 0; b < jobs.size(); b += batch)
        {
            const int n = (int)std::min<size_t>(batch, jobs.size() - b);
            I360B_TRY(N.forward(S.dJobs + b, n, kSub, kSub, true, s));
        }
    }
    mark(3);
    if (stageMs)
    {
        I360B_CUDA(cudaEventSynchronize(ev[3]), "stage events");
        for (int i = 0; i < 3; ++i) cudaEventElapsedTime(&stageMs[i], ev[i], ev[i + 1]);
        for (auto& e : ev) cudaEventDestroy(e);
    }
    // Host vectors must outlive the asynchronous uploads.
    I360B_CUDA(cudaStreamSynchronize(s), "learned render");
    return I360B_SUCCESS;
}

int learned_judge(Plan& P, unsigned short* const* tileOut, double minPsnr, double peak, i360b_learned_stats* st,
                  float* psnrOut, int maxOut, cudaStream_t s)
{
    build_subtiles(P);
    LearnedScratch& S = scratch_for(&P);
    const size_t n = P.subTiles.size();
    std::vector<Region> regs(n);
    for (size_t i = 0; i < n; ++i)
    {
        const SubTile& t = P.subTiles[i];
        const TileDev& T = P.tiles[t.tile];
        const size_t off = ((size_t)t.oy * T.w + t.ox) * 3;
        if (!tileOut[t.tile]) return fail(I360B_INVALID_PARAM, "Tile %d has a null learned output.", t.tile);
        regs[i] = Region{tileOut[t.tile] + off, P.tiles[t.tile].out + off, t.w, t.h, 3LL * T.w, 3LL * T.w};
    }
    I360B_TRY(S.regs(n));
    I360B_TRY(S.judge(n));
    if (n)
    {
        I360B_CUDA(cudaMemcpyAsync(S.dRegs, regs.data(), n * sizeof(Region), cudaMemcpyHostToDevice, s), "judge");
        k_judge<<<(unsigned)std::min<size_t>(n, 65535), 256, 0, s>>>(S.dRegs, (int)n, S.dSse, S.dMax);
        I360B_TRY(check_launch("judge kernel"));
    }
    std::vector<double> sse(n);
    std::vector<int> mx(n);
    if (n)
    {
        I360B_CUDA(cudaMemcpyAsync(sse.data(), S.dSse, n * sizeof(double), cudaMemcpyDeviceToHost, s), "judge");
        I360B_CUDA(cudaMemcpyAsync(mx.data(), S.dMax, n * sizeof(int), cudaMemcpyDeviceToHost, s), "judge");
    }
    I360B_CUDA(cudaStreamSynchronize(s), "judge");
    i360b_learned_stats r{};
    r.subTiles = (int)n;
    r.minPsnr = INFINITY;
    double psum = 0.0;
    int pcount = 0;
    std::vector<Region> fallback;
    for (size_t i = 0; i < n; ++i)
    {
        const SubTile& t = P.subTiles[i];
        r.netSubTiles += t.kind == 2;
        r.copySubTiles += t.kind == 1;
        r.emptySubTiles += t.kind == 0;
        r.overflowSubTiles += t.overflow;
        const double cnt = 3.0 * t.w * t.h;
        const double mse = sse[i] / cnt;
        const double psnr = mse > 0.0 ? 10.0 * std::log10(peak * peak / mse) : INFINITY;
        if (psnrOut && (int)i < maxOut) psnrOut[i] = (float)psnr;
        r.maxAbsError = std::max(r.maxAbsError, mx[i]);
        r.minPsnr = std::min(r.minPsnr, psnr);
        if (std::isfinite(psnr))
        {
            psum += psnr;
            ++pcount;
        }
        if (psnr < minPsnr)
        {
            ++r.fallbackSubTiles;
            // plain -> learned output
            fallback.push_back(
                Region{regs[i].dst, const_cast<unsigned short*>(regs[i].src), t.w, t.h, regs[i].dstRow, regs[i].srcRow});
        }
    }
    r.judgedSubTiles = (int)n;
    r.meanPsnr = pcount ? psum / pcount : INFINITY;
    I360B_TRY(S.regs(std::max(n, fallback.size())));
    I360B_TRY(launch_regions(fallback, S.dRegs, s));
    I360B_CUDA(cudaStreamSynchronize(s), "judge fallback");
    if (st) *st = r;
    return I360B_SUCCESS;
}
}  // namespace i360b

extern "C" int i360b_render_plan_learned(i360b_render_plan* plan, i360b_blendnet* net,
                                         unsigned short* const* dTileOut, int maxBatch, void* stream, float* stageMs)
{
    I360B_TRY(net_prologue(net));
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    if (maxBatch < 1) return fail(I360B_INVALID_PARAM, "maxBatch must be >= 1.");
    BlendNet& N = net->net;
    std::lock_guard<std::mutex> lk(N.mu);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    I360B_TRY(N.begin(s));
    int rc = learned_render(plan->plan, N, dTileOut, maxBatch, s, stageMs);
    if (rc == I360B_SUCCESS) rc = N.check_error(s);
    return N.end(s, rc);
}

extern "C" int i360b_render_plan_judge(i360b_render_plan* plan, unsigned short* const* dTileOut, double minPsnrDb,
                                       double peak, i360b_learned_stats* stats, float* hostSubTilePsnr,
                                       int maxSubTiles, void* stream)
{
    clear_error();
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    if (!plan || !dTileOut) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (!(peak > 0.0)) return fail(I360B_INVALID_PARAM, "peak must be > 0.");
    return learned_judge(plan->plan, dTileOut, minPsnrDb, peak, stats, hostSubTilePsnr, maxSubTiles,
                         static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_render_plan_windows(i360b_render_plan* plan, int maxWindows, int* info, int* numWindows)
{
    clear_error();
    if (!plan || !numWindows) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    Plan& P = plan->plan;
    if (!P.render) return fail(I360B_INVALID_PARAM, "not a render plan");
    build_subtiles(P);
    *numWindows = (int)P.subTiles.size();
    if (info)
        for (int i = 0; i < (int)P.subTiles.size() && i < maxWindows; ++i)
        {
            const SubTile& t = P.subTiles[i];
            int* o = info + 6 * i;
            o[0] = t.tile;
            o[1] = t.ox;
            o[2] = t.oy;
            o[3] = t.kind;
            o[4] = t.overflow;
            o[5] = (t.item[0] >= 0) + (t.item[1] >= 0) + (t.item[2] >= 0) + (t.item[3] >= 0);
        }
    return I360B_SUCCESS;
}

extern "C" int i360b_render_plan_tile_items(i360b_render_plan* plan, int tile, int maxItems,
                                            const unsigned short** dImages, int* boxes, float* edges, int* numItems)
{
    clear_error();
    if (!plan || !numItems) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    const Plan& P = plan->plan;
    if (tile < 0 || tile >= P.nTiles) return fail(I360B_INVALID_PARAM, "Tile %d out of range.", tile);
    if (!P.render) return fail(I360B_INVALID_PARAM, "not a render plan");
    const TileDev& T = P.tiles[tile];
    *numItems = T.numItems;
    for (int k = 0; k < T.numItems && k < maxItems; ++k)
    {
        const ItemDev& it = P.items[T.firstItem + k];
        if (dImages) dImages[k] = it.img;
        if (boxes)
        {
            boxes[4 * k] = it.vx0;
            boxes[4 * k + 1] = it.vy0;
            boxes[4 * k + 2] = it.vx1;
            boxes[4 * k + 3] = it.vy1;
        }
        if (edges)
            for (int q = 0; q < 16; ++q) edges[16 * k + q] = P.itemEdges[(size_t)(T.firstItem + k) * 16 + q];
    }
    return I360B_SUCCESS;
}
