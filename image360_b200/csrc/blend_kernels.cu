// Seam-blend kernels for a batch of tiles.  Every kernel reproduces the FP32
// arithmetic of WindowsApp.Core/SourceFiles/SeamBlend.cpp in the same order,
// so the GPU owner map and output are bit-identical to the CPU backend's.
#include "blend_kernels.cuh"

#include <cuda/atomic>
#include <cuda_fp16.h>
#include <cfloat>
#include <cstddef>

namespace i360b
{
namespace
{
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float f_inf() { return __int_as_float(0x7f800000); }

__device__ __forceinline__ bool cov_bit(const uint32_t* cov, int covWords, int x, int y)
{
    return (__ldg(cov + (size_t)y * covWords + (x >> 5)) >> (x & 31)) & 1u;
}

// ---------------------------------------------------------------------------
// Coverage (SeamBlend.cpp:564-567): covered = any channel != 0, as bits, plus
// the inclusive bounding box of covered pixels (SeamBlend.cpp:263-280).
// A CTA owns a band of a.bandRows full-width rows of one contributor; each warp
// walks its rows 32 pixels at a time, so one ballot is one coverage word.
// ---------------------------------------------------------------------------
struct BoxAcc
{
    int x0 = 0x7fffffff, y0 = 0x7fffffff, x1 = -1, y1 = -1, n = 0;
    __device__ __forceinline__ void add(bool c, int x, int y)
    {
        if (c)
        {
            ++n;
            x0 = min(x0, x);
            x1 = max(x1, x);
            y0 = min(y0, y);
            y1 = max(y1, y);
        }
    }
    // Block-wide reduction and one atomic update of the contributor's box.
    __device__ __forceinline__ void flush(int* bbox)
    {
        __shared__ int sb[5][8];
        int v0 = __reduce_min_sync(kFull, x0), v1 = __reduce_min_sync(kFull, y0);
        int v2 = __reduce_max_sync(kFull, x1), v3 = __reduce_max_sync(kFull, y1);
        int v4 = __reduce_add_sync(kFull, n);
        int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0)
        {
            sb[0][warp] = v0;
            sb[1][warp] = v1;
            sb[2][warp] = v2;
            sb[3][warp] = v3;
            sb[4][warp] = v4;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            int nw = blockDim.x >> 5;
            for (int w = 1; w < nw; ++w)
            {
                v0 = min(v0, sb[0][w]);
                v1 = min(v1, sb[1][w]);
                v2 = max(v2, sb[2][w]);
                v3 = max(v3, sb[3][w]);
                v4 += sb[4][w];
            }
            if (v2 >= 0)
            {
                atomicMin(bbox + 0, v0);
                atomicMin(bbox + 1, v1);
                atomicMax(bbox + 2, v2);
                atomicMax(bbox + 3, v3);
                atomicAdd(bbox + 4, v4);
            }
        }
    }
};

__global__ void __launch_bounds__(256) k_coverage(BlendArgs a, const Unit* __restrict__ units)
{
    const Unit u = units[blockIdx.x];
    const ItemDev& it = a.items[u.id];
    const TileDev& T = a.tiles[it.tile];
    const int W = T.w, H = T.h, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    BoxAcc box;
    const int rowsPerWarp = a.bandRows >> 3;
    for (int r = 0; r < rowsPerWarp; ++r)
    {
        const int y = u.by * a.bandRows + warp * rowsPerWarp + r;
        if (y >= H) break;
        for (int x0 = 0; x0 < W; x0 += 32)
        {
            const int x = x0 + lane;
            bool covered = false;
            if (x < W)
            {
                const unsigned short* p = it.img + ((size_t)y * W + x) * 3;
                covered = (p[0] | p[1] | p[2]) != 0;
            }
            unsigned m = __ballot_sync(kFull, covered);
            if (lane == 0) it.cov[(size_t)y * T.covWords + (x0 >> 5)] = m;
            box.add(covered, x, y);
        }
    }
    box.flush(it.bbox);
}

// ---------------------------------------------------------------------------
// Tile warp: WarpPerspective + ApplyGain of one contributor into its tile
// buffer (RenderExecutor.cpp:104-114), coverage and box emitted in the same
// pass.  Arithmetic identical to k_warp in pixel_ops.cu.
//
// A CTA makes a 128x16 block of one contributor's tile.  The source pixels
// its bilinear taps can reach - the box of the block corners' source
// positions (the corners of a projective image of a rectangle with w > 0
// bound it), widened by 2 pixels for the FP32 rounding of the per-pixel
// positions - are staged in shared memory first: rows read as 16-byte words
// (8 pixels per three words) and kept as 8-byte pixels (r | g << 16, b), so
// that a pixel's two horizontal taps are one 16-byte or two 8-byte shared
// loads.  A tap outside the staged box (never expected) is read from global
// memory instead, so the result does not depend on the margin.  Lanes take
// consecutive pixels, so one ballot is one coverage word.
// ---------------------------------------------------------------------------
constexpr int kWpW = kWarpBlockW, kWpH = kWarpBlockH;  // destination pixels per CTA
constexpr int kWpSW = 160, kWpSH = 44; // staged source box (pixels) at most

// The warp parameters of one item, read once per CTA into registers (the
// item table is in global memory, where the compiler cannot tell it apart
// from the image being written).
struct WarpItem
{
    float H[9];
    const unsigned short* src;
    int srcW, srcH;
    float gain;
    bool applyGain;
};

// The source position of destination (dX, dY) (WarpPerspective_Scalar.cpp:21-37);
// hy = {H[1] dY, H[4] dY, H[7] dY} of the row: the same rounded products,
// summed in the reference's order.  False where the pixel is (0,0,0) by the
// |w| < 1e-10 or range rule.
__device__ __forceinline__ bool warp_pos(const WarpItem& it, float dX, const float* hy, int& x0, int& y0, float& fx,
                                         float& fy)
{
    const float* H = it.H;
    float sx = fadd(fadd(fmul(H[0], dX), hy[0]), H[2]);
    float sy = fadd(fadd(fmul(H[3], dX), hy[1]), H[5]);
    const float sw1 = fadd(fadd(fmul(H[6], dX), hy[2]), H[8]);
    if (fabsf(sw1) < 1e-10f) return false;
    sx = fdiv(sx, sw1);
    sy = fdiv(sy, sw1);
    if (!(sx >= 0.0f && sx < (float)(it.srcW - 1) && sy >= 0.0f && sy < (float)(it.srcH - 1))) return false;
    x0 = (int)f2u_floor(sx);  // 0 <= sx, sy < 2^23 here
    y0 = (int)f2u_floor(sy);
    fx = fsub(sx, u2f((uint32_t)x0));
    fy = fsub(sy, u2f((uint32_t)y0));
    return true;
}

// Bilinear mix + clamp/truncate + gain of one pixel from its four taps
// (WarpPerspectiveKernels.h:16-43, GainColorOps.cpp:16-26).
__device__ __forceinline__ void warp_mix(const WarpItem& it, float fx, float fy, const unsigned short* t00,
                                         const unsigned short* t10, const unsigned short* t01,
                                         const unsigned short* t11, unsigned short o[3])
{
    const float gx = fsub(1.0f, fx), gy = fsub(1.0f, fy);
    const float w00 = fmul(gx, gy), w10 = fmul(fx, gy), w01 = fmul(gx, fy), w11 = fmul(fx, fy);
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        const float v = fadd(fadd(fadd(fmul(w00, u2f(t00[c])), fmul(w10, u2f(t10[c]))), fmul(w01, u2f(t01[c]))),
                             fmul(w11, u2f(t11[c])));
        // the warp's truncation to uint16, then the gain's (one float round trip)
        o[c] = it.applyGain ? clamp_trunc_u16(fmul(clamp_floor_u16f(v), it.gain)) : clamp_trunc_u16(v);
    }
}

__device__ __forceinline__ void px_of(uint2 v, unsigned short* t)
{
    t[0] = (unsigned short)(v.x & 0xffffu);
    t[1] = (unsigned short)(v.x >> 16);
    t[2] = (unsigned short)(v.y & 0xffffu);
}

// Zeroes n u16 elements at p (any even address), the warp's lanes together:
// at most 7 scalar stores either side of a 16-byte aligned body.
__device__ __forceinline__ void warp_zero_u16(unsigned short* p, int n, int lane)
{
    if (n <= 0) return;
    const int head = min(n, (int)(((16u - (unsigned)(reinterpret_cast<uintptr_t>(p) & 15u)) & 15u) >> 1));
    if (lane < head) p[lane] = 0;
    uint4* q = reinterpret_cast<uint4*>(p + head);
    const int nq = (n - head) >> 3;
    for (int j = lane; j < nq; j += 32) q[j] = make_uint4(0u, 0u, 0u, 0u);
    const int t0 = head + (nq << 3);
    if (lane < n - t0) p[t0 + lane] = 0;
}

// One destination pixel read straight from the source frame (the row-band
// form below): the four taps by 2-byte loads through L1.
__device__ __forceinline__ void warp_px(const WarpItem& it, float dX, const float* hy, unsigned short o[3])
{
    o[0] = o[1] = o[2] = 0;
    int x0, y0;
    float fx, fy;
    if (!warp_pos(it, dX, hy, x0, y0, fx, fy)) return;
    const unsigned short* r0 = it.src + ((size_t)y0 * it.srcW + x0) * 3;
    const unsigned short* r1 = r0 + (size_t)it.srcW * 3;
    unsigned short t00[3], t10[3], t01[3], t11[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        t00[c] = __ldg(r0 + c);
        t10[c] = __ldg(r0 + 3 + c);
        t01[c] = __ldg(r1 + c);
        t11[c] = __ldg(r1 + 3 + c);
    }
    warp_mix(it, fx, fy, t00, t10, t01, t11, o);
}

__device__ __forceinline__ WarpItem warp_item(const ItemDev& it)
{
    WarpItem wi;
#pragma unroll
    for (int q = 0; q < 9; ++q) wi.H[q] = it.H[q];
    wi.src = it.src;
    wi.srcW = it.srcW;
    wi.srcH = it.srcH;
    wi.gain = it.gain;
    wi.applyGain = !gain_is_identity(it.gain);
    return wi;
}

// Row-band form (warp shape 0): a CTA makes a.bandRows full-width rows of one
// contributor, each warp whole rows in 64-pixel segments with two pixels per
// lane in flight, gathering taps from the frame through L1; rows and segments
// outside the frame's footprint box are written as zeros without evaluating
// the mapping.  The warps take the band's rows interleaved (warp w: rows w,
// w + 8, ...), so at any time the CTA's warps walk eight neighbouring rows
// side by side and the source rows they share (a bilinear tap pair reads two
// rows, each also read by the next output row) are reused from L1 rather
// than fetched again from DRAM after the whole GPU has streamed past them.
__global__ void __launch_bounds__(256, 8) k_warp_rows(BlendArgs a, const Unit* __restrict__ units)
{
    const Unit u = units[blockIdx.x];
    const ItemDev& it = a.items[u.id];
    const TileDev& T = a.tiles[it.tile];
    const int W = T.w, H = T.h, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned short* img = const_cast<unsigned short*>(it.img);
    const WarpItem wi = warp_item(it);
    const int offX = it.offX, offY = it.offY, vx0 = it.vx0, vx1 = it.vx1, vy0 = it.vy0, vy1 = it.vy1;
    BoxAcc box;
    const int rowsPerWarp = a.bandRows >> 3;
    for (int r = 0; r < rowsPerWarp; ++r)
    {
        const int y = u.by * a.bandRows + r * 8 + warp;
        if (y >= H) break;
        const float dY = (float)(y + offY);
        const float hy[3] = {fmul(wi.H[1], dY), fmul(wi.H[4], dY), fmul(wi.H[7], dY)};
        int s0 = 0, s1 = 0;
        if (y >= vy0 && y <= vy1)
        {
            const int xs = max(vx0, 0), xe = min(vx1, W - 1);
            if (xs <= xe)
            {
                s0 = xs & ~63;
                s1 = min(W, (xe & ~63) + 64);
            }
        }
        unsigned short* row = img + (size_t)y * W * 3;
        uint32_t* covRow = it.cov + (size_t)y * T.covWords;
        warp_zero_u16(row, s0 * 3, lane);
        warp_zero_u16(row + (size_t)s1 * 3, (W - s1) * 3, lane);
        for (int j = lane; j < (s0 >> 5); j += 32) covRow[j] = 0u;
        for (int j = ((s1 + 31) >> 5) + lane; j < ((W + 31) >> 5); j += 32) covRow[j] = 0u;
        for (int x0 = s0; x0 < s1; x0 += 64)
        {
            const int xa = x0 + lane, xb = x0 + 32 + lane;
            unsigned short oa[3] = {0, 0, 0}, ob[3] = {0, 0, 0};
            if (xa < W && xa >= vx0 && xa <= vx1) warp_px(wi, (float)(xa + offX), hy, oa);
            if (xb < W && xb >= vx0 && xb <= vx1) warp_px(wi, (float)(xb + offX), hy, ob);
            const bool ca = (oa[0] | oa[1] | oa[2]) != 0, cb = (ob[0] | ob[1] | ob[2]) != 0;
            if (xa < W)
            {
                unsigned short* d = row + (size_t)xa * 3;
                d[0] = oa[0];
                d[1] = oa[1];
                d[2] = oa[2];
            }
            if (xb < W)
            {
                unsigned short* d = row + (size_t)xb * 3;
                d[0] = ob[0];
                d[1] = ob[1];
                d[2] = ob[2];
            }
            const unsigned ma = __ballot_sync(kFull, ca), mb = __ballot_sync(kFull, cb);
            if (lane == 0)
            {
                covRow[x0 >> 5] = ma;
                if (x0 + 32 < W) covRow[(x0 >> 5) + 1] = mb;
            }
            box.add(ca, xa, y);
            box.add(cb, xb, y);
        }
    }
    box.flush(it.bbox);
}

// Staged-block form (warp shape 1).
struct WarpSmem
{
    uint2 px[kWpSH][kWpSW];
    float ext[4][4];  // per corner: source x, y (FP32, rounded outward by the caller's margin), ok flag
};

__global__ void __launch_bounds__(256) k_warp_tiles(BlendArgs a, const Unit* __restrict__ units)
{
    extern __shared__ __align__(16) unsigned char warp_raw[];
    WarpSmem& S = *reinterpret_cast<WarpSmem*>(warp_raw);
    const Unit u = units[blockIdx.x];
    const ItemDev& it = a.items[u.id];
    const TileDev& T = a.tiles[it.tile];
    const int W = T.w, H = T.h, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned short* img = const_cast<unsigned short*>(it.img);
    const WarpItem wi = warp_item(it);
    const int offX = it.offX, offY = it.offY;
    const int X0 = u.bx * kWpW, Y0 = u.by * kWpH;
    const int X1 = min(X0 + kWpW, W) - 1, Y1 = min(Y0 + kWpH, H) - 1;
    // the block's part of the footprint box (tile-local; outside it the warp is (0,0,0))
    const int fx0 = max(it.vx0, X0), fx1 = min(it.vx1, X1), fy0 = max(it.vy0, Y0), fy1 = min(it.vy1, Y1);
    const bool any = fx0 <= fx1 && fy0 <= fy1;
    // The staged source box: the source positions of the corners of the
    // block's footprint part, one corner per thread of the first four.
    if (any && threadIdx.x < 4)
    {
        const int c = threadIdx.x;
        const float dx = (float)(((c & 1) ? fx1 : fx0) + offX), dy = (float)(((c & 2) ? fy1 : fy0) + offY);
        const float w = wi.H[6] * dx + wi.H[7] * dy + wi.H[8];
        const float sx = (wi.H[0] * dx + wi.H[1] * dy + wi.H[2]) / w;
        const float sy = (wi.H[3] * dx + wi.H[4] * dy + wi.H[5]) / w;
        S.ext[c][0] = sx;
        S.ext[c][1] = sy;
        S.ext[c][2] = (w > 1e-6f && fabsf(sx) < 1e8f && fabsf(sy) < 1e8f) ? 1.0f : 0.0f;
    }
    __syncthreads();
    int sbx = 0, sby = 0, sbc = 0, sbr = 0;  // staged box: x0 (8-aligned), y0, columns, rows; sbc 0 = none
    if (any && S.ext[0][2] > 0.0f && S.ext[1][2] > 0.0f && S.ext[2][2] > 0.0f && S.ext[3][2] > 0.0f)
    {
        const float mnx = fminf(fminf(S.ext[0][0], S.ext[1][0]), fminf(S.ext[2][0], S.ext[3][0]));
        const float mxx = fmaxf(fmaxf(S.ext[0][0], S.ext[1][0]), fmaxf(S.ext[2][0], S.ext[3][0]));
        const float mny = fminf(fminf(S.ext[0][1], S.ext[1][1]), fminf(S.ext[2][1], S.ext[3][1]));
        const float mxy = fmaxf(fmaxf(S.ext[0][1], S.ext[1][1]), fmaxf(S.ext[2][1], S.ext[3][1]));
        // 3 pixels of margin: the per-pixel positions are computed by the
        // reference's FP32 formula, these by a contracted one
        const int sx0 = max(0, (int)floorf(mnx) - 3), sx1 = min(wi.srcW - 1, (int)floorf(mxx) + 4);
        const int sy0 = max(0, (int)floorf(mny) - 3), sy1 = min(wi.srcH - 1, (int)floorf(mxy) + 4);
        const int xa = sx0 & ~7;
        if (sx0 <= sx1 && sy0 <= sy1 && sx1 - xa + 1 <= kWpSW && sy1 - sy0 + 1 <= kWpSH)
        {
            sbx = xa;
            sby = sy0;
            sbc = ((sx1 - xa) | 7) + 1;
            sbr = sy1 - sy0 + 1;
        }
    }
    if (sbc > 0)
    {
        // 8-pixel groups: three 16-byte words when source rows are 16-byte aligned
        const bool fast = (wi.srcW & 7) == 0 && (reinterpret_cast<uintptr_t>(wi.src) & 15) == 0;
        const int ng = sbc >> 3;
        for (int t = threadIdx.x; t < sbr * ng; t += blockDim.x)
        {
            const int r = t / ng, g = t - r * ng;
            const int gx = sbx + 8 * g;
            const unsigned short* src = wi.src + ((size_t)(sby + r) * wi.srcW + gx) * 3;
            uint2* d = &S.px[r][8 * g];
            if (fast && gx + 8 <= wi.srcW)
            {
                const uint4* s4 = reinterpret_cast<const uint4*>(src);
                const uint4 q0 = __ldg(s4), q1 = __ldg(s4 + 1), q2 = __ldg(s4 + 2);
                const uint32_t w[12] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
#pragma unroll
                for (int e = 0; e < 8; e += 2)
                {
                    // pixels e, e+1 occupy u16 3e .. 3e+5 = words 3e/2 .. 3e/2+2
                    const uint32_t a0 = w[3 * e / 2], a1 = w[3 * e / 2 + 1], a2 = w[3 * e / 2 + 2];
                    d[e] = make_uint2(a0, a1 & 0xffffu);
                    d[e + 1] = make_uint2((a1 >> 16) | (a2 << 16), a2 >> 16);
                }
            }
            else
            {
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    if (gx + e < wi.srcW)
                        d[e] = make_uint2((uint32_t)__ldg(src + 3 * e) | ((uint32_t)__ldg(src + 3 * e + 1) << 16),
                                          (uint32_t)__ldg(src + 3 * e + 2));
            }
        }
    }
    __syncthreads();
    BoxAcc box;
    for (int rr = 0; rr < kWpH / 8; ++rr)
    {
        const int y = Y0 + warp * (kWpH / 8) + rr;
        if (y > Y1) break;
        unsigned short* row = img + (size_t)y * W * 3;
        uint32_t* covRow = it.cov + (size_t)y * T.covWords;
        const bool rowIn = any && y >= fy0 && y <= fy1;
        if (!rowIn)
        {
            warp_zero_u16(row + (size_t)X0 * 3, (X1 - X0 + 1) * 3, lane);
            for (int j = (X0 >> 5) + lane; j <= (X1 >> 5); j += 32) covRow[j] = 0u;
            continue;
        }
        const float dY = (float)(y + offY);
        const float hy[3] = {fmul(wi.H[1], dY), fmul(wi.H[4], dY), fmul(wi.H[7], dY)};
#pragma unroll
        for (int i = 0; i < kWpW / 32; ++i)
        {
            const int x = X0 + 32 * i + lane;
            unsigned short o[3] = {0, 0, 0};
            int x0, y0;
            float fx, fy;
            if (x >= fx0 && x <= fx1 && warp_pos(wi, (float)(x + offX), hy, x0, y0, fx, fy))
            {
                const int cx = x0 - sbx, ry = y0 - sby;
                unsigned short t00[3], t10[3], t01[3], t11[3];
                if (cx >= 0 && cx + 1 < sbc && ry >= 0 && ry + 1 < sbr)
                {
                    px_of(S.px[ry][cx], t00);
                    px_of(S.px[ry][cx + 1], t10);
                    px_of(S.px[ry + 1][cx], t01);
                    px_of(S.px[ry + 1][cx + 1], t11);
                }
                else
                {
                    const unsigned short* r0 = wi.src + ((size_t)y0 * wi.srcW + x0) * 3;
                    const unsigned short* r1 = r0 + (size_t)wi.srcW * 3;
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                    {
                        t00[c] = __ldg(r0 + c);
                        t10[c] = __ldg(r0 + 3 + c);
                        t01[c] = __ldg(r1 + c);
                        t11[c] = __ldg(r1 + 3 + c);
                    }
                }
                warp_mix(wi, fx, fy, t00, t10, t01, t11, o);
            }
            const bool cov = (o[0] | o[1] | o[2]) != 0;
            if (x <= X1)
            {
                unsigned short* d = row + (size_t)x * 3;
                d[0] = o[0];
                d[1] = o[1];
                d[2] = o[2];
            }
            const unsigned m = __ballot_sync(kFull, cov);
            if (lane == 0 && x - lane <= X1) covRow[(x - lane) >> 5] = m;
            box.add(cov, x, y);
        }
    }
    box.flush(it.bbox);
}

// ---------------------------------------------------------------------------
// Chamfer distance (SeamBlend.cpp:206-242), exact.
//
// The raster recurrence d[p] = min(init, left+1, up+1, upleft+sqrt2,
// upright+sqrt2) is a DAG with a unique solution, so any schedule that applies
// the same rounded operations (min is exact and order-free) reproduces the CPU
// result bit for bit.  Neighbours outside the tile are skipped by the
// reference; here they are virtual cells of value +inf, which min() ignores
// (inf + c = inf), so one uniform step serves every pixel.
//
// Systolic wavefront: lane r of a warp owns row 32g + r and at step t
// computes column x = t - 2r - 2, two columns behind the lane above.  The
// value it needs from the row above at x+1 is the lane above's output of the
// previous step and arrives by one __shfl_up_sync; the values at x and x-1
// are the ones received one and two steps earlier.  Lane 0 takes its row
// above from a shared-memory ring slot written by lane 31 of the previous row
// group.  A warp runs kDtChunk steps between hand-offs: before a chunk, lane
// 0 waits (bounded) until the previous group has published every column the
// chunk reads; after it, lane 31 publishes how many columns of its row are
// final.  The initial values of a chunk (one or two coverage words, or eight
// pairs of the forward result) are loaded before its first step, and only
// chunks that touch the tile's edges test cells for being virtual.  The
// backward pass is the same code on mirrored coordinates with the forward
// result as init.
//
// Progress is published per row group (prog[g] = columns of row group g's
// last row that are final), never per ring slot: group g + nslots reuses
// group g's slot while group g + 1 may still be waiting for columns of group
// g, so a per-slot counter would let g + nslots's progress release that wait
// early.  The slot data itself is safe to reuse: a group runs a chunk only
// when the group above has finished at least 64 further steps, so when group
// g + nslots (nslots >= 2) writes column x of the slot, group g + 1 has run
// more than 64 steps past the one where it read x.
// ---------------------------------------------------------------------------
constexpr int kDtChunk = 16;  // steps between hand-offs
constexpr int kDtRing = 4;    // row-group hand-off slots
constexpr int kDtWarps = 16;  // warps per CTA
constexpr int kDtStR = 20;    // staging row stride (floats): 16 columns + pad, 16-byte rows
constexpr size_t kDtStageBytes = (size_t)kDtWarps * 32 * kDtStR * sizeof(float);
// Ring slot: columns -4 .. W of a row (index = column + 4); columns < 0 and
// column W hold +inf.
__host__ __device__ __forceinline__ int dt_ring_stride(int W) { return (W + 8) & ~3; }

template <bool BACK>
__global__ void __launch_bounds__(32 * kDtWarps, 2) k_dt(BlendArgs a, const int* __restrict__ itemList, int nslots)
{
    extern __shared__ float smem[];
    const ItemDev& it = a.items[itemList[blockIdx.x]];
    const TileDev& T = a.tiles[it.tile];
    const int Wt = T.w, Ht = T.h, covWords = T.covWords;
    // A contributor that covers none or all of its tile has d == 0 or
    // d == kInf everywhere (no seed / nothing to seed); the ownership kernel
    // substitutes those values, so the transform is skipped.
    {
        const int cnt = it.bbox[4];
        if (cnt == 0 || (long long)cnt == (long long)Wt * Ht) return;
    }
    // The transform runs on R: the covered box grown by one cell and clamped
    // to the tile, its left edge rounded down to an even column and its right
    // edge up to an odd one where the tile allows (rows of 8-byte pairs).
    // Cells outside the box are uncovered, so d == 0 there; the cells of R
    // outside the box are uncovered too and come out 0 whatever lies beyond
    // R, and every cell inside the box reads only cells of R.  So the
    // recurrence on R with +inf beyond it gives the tile transform's values
    // on R.  Nothing is written outside R: the ownership kernel, the fields'
    // only reader, takes d == 0 outside the covered box.
    const int rx0 = max(it.bbox[0] - 1, 0) & ~1, rx1 = min((it.bbox[2] + 1) | 1, Wt - 1);
    const int ry0 = max(it.bbox[1] - 1, 0), ry1 = min(it.bbox[3] + 1, Ht - 1);
    const int W = rx1 - rx0 + 1, H = ry1 - ry0 + 1;  // R's extent; the recurrence below runs on R
    const int RS = dt_ring_stride(W);
    float* ring = smem + kDtStageBytes / sizeof(float);
    int* prog = reinterpret_cast<int*>(ring + (size_t)nslots * RS);
    const float INF = f_inf();
    const int nG = (H + 31) >> 5;
    for (int i = threadIdx.x; i < nG; i += blockDim.x) prog[i] = -1;
    for (int i = threadIdx.x; i < nslots * 5; i += blockDim.x)
    {
        const int sl = i / 5, e = i - sl * 5;
        ring[(size_t)sl * RS + (e < 4 ? e : W + 4)] = INF;
    }
    __syncthreads();
    const float kInf = (float)(Wt + Ht);
    const float kDiag = 1.41421356f;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    const float* src = BACK ? it.d1 : nullptr;
    float* dst = BACK ? it.d : it.d1;
    // 8-byte pairs of columns: even row length and 8-byte aligned buffers.
    const bool pairs = (W & 1) == 0 && (Wt & 1) == 0 &&
                       ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 7) == 0;
    const int nSteps = W + 64;  // lane 31 computes column W - 1 at step W + 63

    for (int g = warp; g < nG; g += nwarps)
    {
        const int vy = g * 32 + lane;  // row in the pass's (mirrored) order
        const bool rowOk = vy < H;
        const bool fullGroup = g * 32 + 31 < H;
        const bool hasAbove = g > 0;  // lane 0's row above: the ring, else virtual
        const int ty = rowOk ? (BACK ? ry1 - vy : ry0 + vy) : ry0;  // tile row
        float* outRow = dst + (size_t)ty * Wt;
        const float* inRow = BACK ? src + (size_t)ty * Wt : nullptr;
        const uint32_t* covRow = it.cov + (size_t)ty * covWords;
        // Staging rows of this warp: a chunk's 32 x 16 values cross between
        // lanes (one row each) and 8-lane groups (one 64-byte row segment per
        // global access) here.
        float* st = smem + (size_t)warp * 32 * kDtStR;
        const int sj = lane >> 3, sp = lane & 7;  // transposed role: rows sj + 4k, pair sp
        float* ringOut = ring + (size_t)(g % nslots) * RS + 4;
        const float* ringIn = ring + (size_t)((g + nslots - 1) % nslots) * RS + 4;
        float left = INF, up0 = INF, upm1 = INF;  // own x-1; row above at x and x-1
        int seen = -1;                            // lane 0: progress of the group above already observed
        int wIdx = -4;                            // forward: coverage words wIdx .. wIdx+2 held
        uint32_t wLo = 0, wHi = 0, wNx = 0;
        // Interior chunk: every lane's row and columns lie in the tile, so no
        // cell is virtual (but lane 0's row above, in group 0).
        auto is_interior = [&](int c0) { return fullGroup && c0 - 64 >= 0 && c0 + kDtChunk - 2 <= W; };
        for (int t0 = 0; t0 < nSteps; t0 += kDtChunk)
        {
            int bad = 0;
            if (hasAbove && lane == 0)
            {
                // this chunk reads columns up to t0 + kDtChunk - 1 of the row above
                const int need = min(t0 + kDtChunk, W);
                if (seen < need)
                {
                    cuda::atomic_ref<int, cuda::thread_scope_block> pr(prog[g - 1]);
                    const long long tstart = clock64();
                    int spins = 0;
                    while ((seen = pr.load(cuda::memory_order_acquire)) < need)
                    {
                        if (++spins > 32) __nanosleep(128);
                        if (((spins & 63) == 0 || a.spinLimit == 0) &&
                            (*(volatile int*)a.error || clock64() - tstart > a.spinLimit))
                        {
                            atomicExch(a.error, 1);
                            atomicExch(a.error + 1, 1);
                            bad = 1;
                            break;
                        }
                    }
                }
            }
            if (__shfl_sync(kFull, bad, 0)) return;  // gave up waiting (error flag set)
            const int xs = t0 - 2 * lane - 2;  // this lane's column at the chunk's first step
            // Outside interior chunks cells outside the tile are +inf and never
            // stored; with an even row length a column pair is in or out as a
            // whole.  The backward pass takes its edge chunks cell by cell
            // (fewer registers in its staged path).
            const bool interior = is_interior(t0);
            if (pairs && (!BACK || interior))
            {
                // The chunk's initial values enter, and its results leave, this
                // lane's staging row in memory order (the backward pass's columns
                // reversed), four at a time.
                float* const cur = st;
                float4* myRow = reinterpret_cast<float4*>(cur + lane * kDtStR);
                uint32_t bits = 0;
                __syncwarp();  // the previous chunk's row-segment reads are done
                if (BACK)
                {
                    // Row j's 16 values sit at tile columns rx1-15-xs_j .. rx1-xs_j
                    // (mirrored); 8 lanes load each row as 8-byte pairs.
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                    {
                        const int j = 4 * k + sj;
                        const int vyj = g * 32 + j, m0 = rx1 - 15 - (t0 - 2 * j - 2) + 2 * sp;
                        *reinterpret_cast<float2*>(cur + j * kDtStR + 2 * sp) =
                            __ldg(reinterpret_cast<const float2*>(src + (size_t)(ry1 - vyj) * Wt + m0));
                    }
                    __syncwarp();
                }
                else
                {
                    // Coverage words xs>>5 and the next, held across chunks (the
                    // word after them loaded a chunk early).
                    const int xa = rx0 + xs;  // tile column of the chunk's first step
                    const int w0 = xa >> 5;
                    if (w0 != wIdx)
                    {
                        if (w0 == wIdx + 1)
                        {
                            wLo = wHi;
                            wHi = wNx;
                        }
                        else
                        {
                            wLo = w0 >= 0 && w0 < covWords ? __ldg(covRow + w0) : 0u;
                            wHi = w0 + 1 >= 0 && w0 + 1 < covWords ? __ldg(covRow + w0 + 1) : 0u;
                        }
                        wNx = w0 + 2 >= 0 && w0 + 2 < covWords ? __ldg(covRow + w0 + 2) : 0u;
                        wIdx = w0;
                    }
                    bits = __funnelshift_r(wLo, wHi, xa & 31);
                }
                // Lane 0's row above: columns t0-1 .. t0+14 (slot entries
                // t0+3 .. t0+18) as five 16-byte reads, the same for every lane.
                const float4* slot4 = reinterpret_cast<const float4*>(ringIn - 4) + (t0 >> 2);
                // The chunk's initial values, four columns at a time.
                auto chunk_in = [&](int m4, float in[4]) {
                    if (BACK)
                    {
                        const float4 v = myRow[3 - m4];  // memory columns 12-4m4 .. 15-4m4
                        in[0] = v.w;
                        in[1] = v.z;
                        in[2] = v.y;
                        in[3] = v.x;
                    }
                    else
                    {
#pragma unroll
                        for (int i = 0; i < 4; ++i) in[i] = ((bits >> (4 * m4 + i)) & 1u) ? kInf : 0.0f;
                    }
                };
                auto chunk_out = [&](int m4, const float o[4]) {
                    if (BACK) myRow[3 - m4] = make_float4(o[3], o[2], o[1], o[0]);
                    else myRow[m4] = make_float4(o[0], o[1], o[2], o[3]);
                };
                if (interior)
                {
                    // Every cell of the chunk is in the tile.  The sums with the
                    // row above are carried between steps: fadd(up0, 1) is formed
                    // one step ahead, and fadd(upm1, kDiag) is the fadd(upp1,
                    // kDiag) of two steps back (the same operands, so the same
                    // value).  min is exact in any order, so the candidates known
                    // early are combined first and a step's dependency chain is
                    // the shuffle, one add and two mins.  Lane 0 of group 0 has no
                    // row above (+inf).
                    const float4 inf4 = make_float4(INF, INF, INF, INF);
                    float prevW = hasAbove ? slot4[0].w : INF;
                    float up1 = fadd(up0, 1.0f), dg1 = fadd(up0, kDiag), dg2 = fadd(upm1, kDiag);
                    float u1 = up0, u2 = upm1;  // the row above at x and x - 1 after the chunk
#pragma unroll
                    for (int m4 = 0; m4 < kDtChunk / 4; ++m4)
                    {
                        float in[4], o[4];
                        chunk_in(m4, in);
                        const float4 blk = hasAbove ? slot4[m4 + 1] : inf4;
                        const float above[4] = {prevW, blk.x, blk.y, blk.z};
                        prevW = blk.w;
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                        {
                            const float recv = __shfl_up_sync(kFull, left, 1);
                            const float upp1 = lane == 0 ? above[i] : recv;
                            const float dg = fadd(upp1, kDiag);
                            float av = fminf(fminf(in[i], up1), dg2);
                            av = fminf(av, dg);
                            av = fminf(av, fadd(left, 1.0f));
                            up1 = fadd(upp1, 1.0f);
                            dg2 = dg1;
                            dg1 = dg;
                            u2 = u1;
                            u1 = upp1;
                            left = av;
                            o[i] = av;
                        }
                        chunk_out(m4, o);
                    }
                    up0 = u1;
                    upm1 = u2;
                }
                else
                {
#pragma unroll
                    for (int m4 = 0; m4 < kDtChunk / 4; ++m4)
                    {
                        float in[4], o[4];
                        chunk_in(m4, in);
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                        {
                            const int x = xs + 4 * m4 + i;
                            const bool ok = rowOk && x >= 0 && x < W;
                            const float recv = __shfl_up_sync(kFull, left, 1);
                            // lane 0 reads columns >= -1 of the row above (the ring
                            // holds +inf outside [0, W)); group 0 has no row above
                            float upp1 = recv;
                            if (lane == 0) upp1 = hasAbove ? ringIn[min(max(x + 1, -1), W)] : INF;
                            float av = fminf(in[i], fadd(up0, 1.0f));
                            av = fminf(av, fadd(upm1, kDiag));
                            av = fminf(av, fadd(upp1, kDiag));
                            av = fminf(av, fadd(left, 1.0f));
                            const float d = ok ? av : INF;
                            upm1 = up0;
                            up0 = upp1;
                            left = d;
                            o[i] = d;
                        }
                        chunk_out(m4, o);
                    }
                }
                // 64-byte row segments to the output.
                __syncwarp();
#pragma unroll
                for (int k = 0; k < 8; ++k)
                {
                    const int j = 4 * k + sj;
                    const int vyj = g * 32 + j, xsj = t0 - 2 * j - 2;
                    const float2 v = *reinterpret_cast<const float2*>(cur + j * kDtStR + 2 * sp);
                    if (BACK)
                    {
                        const int m0 = rx1 - 15 - xsj + 2 * sp;  // chunk columns xs_j+15-2sp, xs_j+14-2sp
                        if (interior || (vyj < H && m0 >= rx0 && m0 < rx1))
                        {
                            *reinterpret_cast<float2*>(dst + (size_t)(ry1 - vyj) * Wt + m0) = v;
                            if (j == 31) *reinterpret_cast<float2*>(ringOut + xsj + 14 - 2 * sp) = make_float2(v.y, v.x);
                        }
                    }
                    else
                    {
                        const int c0 = xsj + 2 * sp;
                        if (interior || (vyj < H && c0 >= 0 && c0 < W))
                        {
                            *reinterpret_cast<float2*>(dst + (size_t)(ry0 + vyj) * Wt + rx0 + c0) = v;
                            if (j == 31) *reinterpret_cast<float2*>(ringOut + c0) = v;
                        }
                    }
                }
            }
            else
            {
#pragma unroll
                for (int q = 0; q < kDtChunk; ++q)
                {
                    const int x = xs + q;
                    const bool ok = rowOk && x >= 0 && x < W;
                    float iv = INF;
                    if (ok)
                        iv = BACK ? __ldg(inRow + (rx1 - x))
                                  : (((__ldg(covRow + ((rx0 + x) >> 5)) >> ((rx0 + x) & 31)) & 1u) ? kInf : 0.0f);
                    const float recv = __shfl_up_sync(kFull, left, 1);
                    // lane 0 reads columns >= -1 of the row above (ring holds +inf
                    // outside [0, W)); group 0 has no row above
                    float upp1 = recv;
                    if (lane == 0) upp1 = hasAbove ? ringIn[min(max(x + 1, -1), W)] : INF;
                    float av = fminf(iv, fadd(up0, 1.0f));
                    av = fminf(av, fadd(upm1, kDiag));
                    av = fminf(av, fadd(upp1, kDiag));
                    av = fminf(av, fadd(left, 1.0f));
                    const float d = ok ? av : INF;
                    upm1 = up0;
                    up0 = upp1;
                    left = d;
                    if (ok)
                    {
                        outRow[BACK ? rx1 - x : rx0 + x] = d;
                        if (lane == 31) ringOut[x] = d;
                    }
                }
            }
            // Lane 31 publishes how many columns of its row are final.
            if (lane == 31)
            {
                const int done = min(max(t0 - 64 + kDtChunk, 0), W);
                cuda::atomic_ref<int, cuda::thread_scope_block> pr(prog[g]);
                pr.store(done, cuda::memory_order_release);
            }
        }
    }
}

// A tile's contributor descriptors staged in shared memory: the per-pixel
// loops below then index shared memory instead of chasing items[k] in global
// memory for every pixel.
constexpr int kMaxTileItems = 128;  // above the 127-contributor limit of the blend entry points

struct ItemCache
{
    const unsigned short* img[kMaxTileItems];
    const float* d[kMaxTileItems];
    const float4* nd[kMaxTileItems];
    const float* wg[kMaxTileItems];
    int cnt[kMaxTileItems];
    int4 box[kMaxTileItems];  // covered box (x0, y0, x1, y1), or its support at one level
};

// The box outside which a contributor's level-`level` pyramid values (num,
// den and weight) are exactly zero, from its covered box at level 0.  At
// level 0 the values vanish outside the covered box: num and den by
// coverage, the weight because a contributor owns only pixels inside its
// covered box (the ownership argmax needs d > 0, i.e. coverage, and the seam
// step reassigns pixels only inside two contributors' common box,
// SeamBlend.cpp:439-442, 580).  Output X of a blur + decimate step reads
// pixels 2X-2 .. 2X+2 (clamped into the level, which stays inside that
// range), so the support grows to [floor((x0-2)/2), floor((x1+2)/2)].  An
// empty box (x0 > x1) stays empty.
__device__ __forceinline__ int4 support_box(int4 b, int level)
{
    for (int l = 0; l < level; ++l)
    {
        b.x = (b.x - 2) >> 1;
        b.y = (b.y - 2) >> 1;
        b.z = (b.z + 2) >> 1;
        b.w = (b.w + 2) >> 1;
    }
    return b;
}

// The contributor's weight support at `level` (zero weight outside): its
// owned box grown as support_box does.
__device__ __forceinline__ int4 owned_support(const int* bbox, int level)
{
    return support_box(make_int4(__ldg(bbox + kOwnedBox), __ldg(bbox + kOwnedBox + 1), __ldg(bbox + kOwnedBox + 2),
                                 __ldg(bbox + kOwnedBox + 3)),
                       level);
}

// Where a contributor's num/den at `level` must be right (below the top level
// `top` of its tile): the readers take G only where the weight is non-zero -
// the band blend of the level, the Up taps of the level below (a non-zero
// weight one level down has non-zero weights at its taps) and, at level 1,
// the output's taps of owned pixels - and the down step makes level l+1 at a
// position X from level l at 2X-2 .. 2X+2.  So the box is the owned weight
// support grown by m(level) with m(top) = 0 and m(l) = 5 + 2 m(l+1) (the
// footprint of a grown box at l+1 reaches at most 5 beyond the support at l,
// support_box rounding included): m(l) = 5 (2^(top-l) - 1).  Outside it a
// pyramid step may leave num/den wrong or unwritten; the weight is right
// everywhere (level 0's is the owner mask, and each level's weight depends
// only on the weight below).
__device__ __forceinline__ int4 needed_box(const int* bbox, int level, int top)
{
    const int4 b = owned_support(bbox, level);
    const int m = 5 * ((1 << max(top - level, 0)) - 1);
    return make_int4(b.x - m, b.y - m, b.z + m, b.w + m);
}

__device__ __forceinline__ int4 covered_box(const int* bbox)
{
    return make_int4(__ldg(bbox), __ldg(bbox + 1), __ldg(bbox + 2), __ldg(bbox + 3));
}

__device__ __forceinline__ void load_item_cache(ItemCache& c, const BlendArgs& a, const TileDev& T)
{
    for (int k = threadIdx.x; k < T.numItems && k < kMaxTileItems; k += blockDim.x)
    {
        const ItemDev& it = a.items[T.firstItem + k];
        c.img[k] = it.img;
        c.d[k] = it.d;
        c.nd[k] = it.nd;
        c.wg[k] = it.wg;
        c.cnt[k] = it.bbox[4];
        c.box[k] = make_int4(it.bbox[0], it.bbox[1], it.bbox[2], it.bbox[3]);
    }
    __syncthreads();
}

// The cache's boxes as the contributors' weight supports at `level` (after
// load_item_cache): outside them a contributor's weight is zero.
__device__ __forceinline__ void level_boxes(ItemCache& c, const BlendArgs& a, const TileDev& T, int level)
{
    for (int k = threadIdx.x; k < T.numItems && k < kMaxTileItems; k += blockDim.x)
        c.box[k] = owned_support(a.items[T.firstItem + k].bbox, level);
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Ownership (SeamBlend.cpp:244-261): argmax over contributors of d > 0,
// strict '>' so ties keep the lowest index; -1 where nothing covers.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_owner(BlendArgs a, const Unit* __restrict__ units)
{
    __shared__ ItemCache C;
    __shared__ int obox[kMaxTileItems][4];  // the band's owned boxes, merged into the items' at the end
    const Unit u = units[blockIdx.x];
    const TileDev& T = a.tiles[u.id];
    for (int k = threadIdx.x; k < kMaxTileItems; k += blockDim.x)
    {
        obox[k][0] = obox[k][1] = 0x7fffffff;
        obox[k][2] = obox[k][3] = -1;
    }
    load_item_cache(C, a, T);  // (its barrier also orders the box initialisation)
    const int K = T.numItems;
    const int W = T.w;
    const long long full = (long long)W * T.h;
    const float kInf = (float)(W + T.h);
    const int row0 = u.by * a.bandRows;
    const int rows = min(a.bandRows, T.h - row0);
    // Four pixels per thread: 16-byte reads of d and one 4-byte owner store
    // when rows are 4-pixel aligned.  A contributor with no covered pixel, or
    // whose covered box misses the pixels, has d == 0 there and cannot win
    // (the argmax needs d > 0), so it is skipped.
    const bool vec = (W & 3) == 0;
    for (int r = 0; r < rows; ++r)
    {
        const int y = row0 + r;
        for (int x4 = threadIdx.x * 4; x4 < W; x4 += blockDim.x * 4)
        {
            const long long p = (long long)y * W + x4;
            const int n = min(4, W - x4);
            int best[4] = {-1, -1, -1, -1};
            float bestD[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            for (int k = 0; k < K; ++k)
            {
                const int cnt = C.cnt[k];
                if (cnt == 0) continue;
                if ((long long)cnt == full)
                {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (kInf > bestD[i])
                        {
                            bestD[i] = kInf;
                            best[i] = k;
                        }
                    continue;
                }
                const int4 B = C.box[k];
                if (y < B.y || y > B.w || x4 + 3 < B.x || x4 > B.z) continue;
                float v[4];
                if (vec)
                {
                    const float4 q = __ldg(reinterpret_cast<const float4*>(C.d[k] + p));
                    v[0] = q.x;
                    v[1] = q.y;
                    v[2] = q.z;
                    v[3] = q.w;
                }
                else
                {
#pragma unroll
                    for (int i = 0; i < 4; ++i) v[i] = i < n ? __ldg(C.d[k] + p + i) : 0.0f;
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
                {
                    const int x = x4 + i;
                    const float vi = (x >= B.x && x <= B.z) ? v[i] : 0.0f;  // d is 0 outside the covered box
                    if (vi > bestD[i])
                    {
                        bestD[i] = vi;
                        best[i] = k;
                    }
                }
            }
            if (vec)
                *reinterpret_cast<uint32_t*>(T.owner + p) = (uint32_t)(best[0] & 0xff) | ((uint32_t)(best[1] & 0xff) << 8) |
                                                            ((uint32_t)(best[2] & 0xff) << 16) |
                                                            ((uint32_t)(best[3] & 0xff) << 24);
            else
                for (int i = 0; i < n; ++i) T.owner[p + i] = (signed char)best[i];
            // owned boxes: four pixels of one owner (the common case) as one
            // key, the lanes of a key merged before one shared-memory update
            const bool one = n == 4 && best[1] == best[0] && best[2] == best[0] && best[3] == best[0];
            const int key = one ? best[0] : -2;
            const unsigned act = __activemask();
            const unsigned grp = __match_any_sync(act, key);
            const int xmin = __reduce_min_sync(grp, x4), xmax = __reduce_max_sync(grp, x4 + 3);
            if (key >= 0 && (threadIdx.x & 31) == __ffs(grp) - 1)
            {
                atomicMin(&obox[key][0], xmin);
                atomicMax(&obox[key][2], xmax);
                atomicMin(&obox[key][1], y);
                atomicMax(&obox[key][3], y);
            }
            if (!one)
                for (int i = 0; i < n; ++i)
                    if (best[i] >= 0)
                    {
                        atomicMin(&obox[best[i]][0], x4 + i);
                        atomicMax(&obox[best[i]][2], x4 + i);
                        atomicMin(&obox[best[i]][1], y);
                        atomicMax(&obox[best[i]][3], y);
                    }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < K && k < kMaxTileItems; k += blockDim.x)
        if (obox[k][2] >= 0)
        {
            int* ob = a.items[T.firstItem + k].bbox + kOwnedBox;
            atomicMin(ob, obox[k][0]);
            atomicMin(ob + 1, obox[k][1]);
            atomicMax(ob + 2, obox[k][2]);
            atomicMax(ob + 3, obox[k][3]);
        }
}

// ---------------------------------------------------------------------------
// Seam refinement (SeamBlend.cpp:293-445) for every overlapping pair of a
// tile, in the reference's (i, j) order, one 1024-thread CTA per tile.
// Lines are scanned in parallel (row lines: a warp per line with 16-byte owner
// loads; column lines: a lane per line, 16 loads in flight); the dynamic
// program over contested lines is sequential, as in the reference, and runs
// on two warps (one candidate per lane) with the per-line state in shared
// memory.
// ---------------------------------------------------------------------------
constexpr int kSeamThreads = 1024;
constexpr int kDpThreads = 512;  // 8 threads per candidate (64 candidate slots)

// First position t = tb + b (b in 0..15) of a 16-byte chunk of owner bytes,
// with 0 <= t < lineLen, whose byte equals a or b (owner indices 0..127), or
// INT_MAX: four-byte SIMD compares instead of a byte loop.
__device__ __forceinline__ int first_owner_in_chunk(uint4 v, unsigned repA, unsigned repB, int tb, int lineLen)
{
    const int b0 = max(0, -tb), b1 = min(16, lineLen - tb);
    if (b0 >= b1) return 0x7fffffff;
    const unsigned w[4] = {v.x, v.y, v.z, v.w};
    unsigned mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const unsigned m = (__vcmpeq4(w[i], repA) | __vcmpeq4(w[i], repB)) & 0x80808080u;
        mask |= (((m >> 7) & 1u) | ((m >> 14) & 2u) | ((m >> 21) & 4u) | ((m >> 28) & 8u)) << (4 * i);
    }
    mask &= ((1u << b1) - 1u) & ~((1u << b0) - 1u);
    return mask ? tb + __ffs(mask) - 1 : 0x7fffffff;
}

// Bytes of a 16-byte chunk equal to the owner index replicated in rep, as a
// 16-bit mask (bit b: byte b).
__device__ __forceinline__ unsigned chunk_byte_mask(uint4 v, unsigned rep)
{
    const unsigned w[4] = {v.x, v.y, v.z, v.w};
    unsigned mask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const unsigned m = __vcmpeq4(w[i], rep) & 0x80808080u;
        mask |= (((m >> 7) & 1u) | ((m >> 14) & 2u) | ((m >> 21) & 4u) | ((m >> 28) & 8u)) << (4 * i);
    }
    return mask;
}

// Bytes o .. o + 15 of the 32 bytes a, b (0 <= o < 16).
__device__ __forceinline__ uint4 bytes16_at(uint4 a, uint4 b, int o)
{
    const unsigned sh = (unsigned)(o & 3) * 8u;
    uint32_t w0, w1, w2, w3, w4;
    switch (o >> 2)
    {
    case 0: w0 = a.x; w1 = a.y; w2 = a.z; w3 = a.w; w4 = b.x; break;
    case 1: w0 = a.y; w1 = a.z; w2 = a.w; w3 = b.x; w4 = b.y; break;
    case 2: w0 = a.z; w1 = a.w; w2 = b.x; w3 = b.y; w4 = b.z; break;
    default: w0 = a.w; w1 = b.x; w2 = b.y; w3 = b.z; w4 = b.w; break;
    }
    return make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh), __funnelshift_r(w2, w3, sh),
                      __funnelshift_r(w3, w4, sh));
}

// Contested band of a column line (SeamBlend.cpp:347-359): the positions
// within kSeamRadius of the crossover covered by both contributors, as
// lo..hi (lo > hi: none).  The coverage bits of 8 rows are requested at once
// (both contributors' words, no short circuit).
__device__ __forceinline__ void seam_column_band(const uint32_t* covI, const uint32_t* covJ, int covWords, int x,
                                                 int oy0, int cross, int lineLen, int& outLo, int& outHi)
{
    int lo = 1, hi = 0;
    if (cross >= 0)
    {
        const int bLo = max(0, cross - kSeamRadius), bHi = min(lineLen - 1, cross + kSeamRadius);
        for (int tb = bLo; tb <= bHi; tb += 8)
        {
            bool ok[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                const int y = oy0 + min(tb + q, bHi);
                ok[q] = tb + q <= bHi && (cov_bit(covI, covWords, x, y) & cov_bit(covJ, covWords, x, y));
            }
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (ok[q])
                {
                    if (hi < lo) lo = tb + q;
                    hi = tb + q;
                }
        }
    }
    outLo = lo;
    outHi = hi;
}

// The seam DP of one pair on one warp while its values stay small integers
// (SeamBlend.cpp:362-407).  Candidate costs are sums of absolute differences
// of 16-bit values, so every value of the DP - cost, previous value, penalty
// 2|t - pt| - is an integer; while they stay below 2^23 every FP32 operation
// of the reference on them is exact (the warp form runs on lines shorter
// than 2^20 pixels, so penalties stay below 2^21, and a cost is at most
// 3 x 65535 < 2^18), and the minimum it scans for,
//   b(t) = min over kk (dp[kk] + 2 |t - pt(kk)|), lowest kk on ties,
// is an L1 distance transform: with positions in line coordinates,
//   min over pt(kk) <= t of (dp - 2 pt)[kk] + 2 t   (a prefix minimum), and
//   min over pt(kk) >= t of (dp + 2 pt)[kk] - 2 t   (a suffix minimum).
// Both are warp scans over the previous line's 49 candidates, on keys
// value * 64 + kk, so the minimum of a key is the lowest-index minimum; each
// candidate then looks its two minima up.  Lane l holds candidates l and
// l + 32.  After each line its largest value is checked against 2^23; where
// it is not below, the warp stops, leaves that line's values in dpBuf[cur ^ 1], and
// returns the line to continue from, which the general form then does with
// the reference's own FP32 operations.  Returns via the out parameters the
// first line not processed, and the last line, its width and cur.
__device__ __forceinline__ void seam_dp_warp(const int* sList, const int* sLo, const int* sHi, int* sPrev,
                                          unsigned char* sBack, const float* costs, int nC, int lineLen,
                                          float (*dpBuf)[64], int lane, int& outStart, int& outLast,
                                          int& outLastW, int& outCur)
{
    if (lineLen >= (1 << 20))
    {
        outStart = 0;  // all lines to the general form
        outLast = -1;
        outLastW = 0;
        outCur = 0;
        return;
    }
    constexpr int kPre = 4;
    constexpr int kInf = 0x7fffffff;
    const int k0 = lane, k1 = lane + 32;
    float cq0[kPre], cq1[kPre];
#pragma unroll
    for (int q = 0; q < kPre; ++q)
    {
        cq0[q] = cq1[q] = 0.0f;
        if (q < nC)
        {
            const int l = sList[q];
            const int w = sHi[l] - sLo[l] + 1;
            if (k0 < w) cq0[q] = costs[(size_t)l * kSeamBand + k0];
            if (k1 < w && k1 < kSeamBand) cq1[q] = costs[(size_t)l * kSeamBand + k1];
        }
    }
    float dp0 = 0.0f, dp1 = 0.0f;  // the previous line's values of candidates k0, k1
    int last = -1, lastLo = 0, lastW = 0, cur = 0;
    int ci2 = 0;
    for (; ci2 < nC; ++ci2)
    {
        const int line = sList[ci2];
        const int lo = sLo[line], lw = sHi[line] - lo + 1;
        const float c0 = cq0[0], c1 = cq1[0];
#pragma unroll
        for (int q = 0; q + 1 < kPre; ++q)
        {
            cq0[q] = cq0[q + 1];
            cq1[q] = cq1[q + 1];
        }
        cq0[kPre - 1] = cq1[kPre - 1] = 0.0f;
        if (ci2 + kPre < nC)
        {
            const int l = sList[ci2 + kPre];
            const int w = sHi[l] - sLo[l] + 1;
            if (k0 < w) cq0[kPre - 1] = costs[(size_t)l * kSeamBand + k0];
            if (k1 < w && k1 < kSeamBand) cq1[kPre - 1] = costs[(size_t)l * kSeamBand + k1];
        }
        float v0 = c0, v1 = c1;
        int bp0 = -1, bp1 = -1;
        if (last >= 0)
        {
            // keys of the previous candidates: slot a = kk (lane), slot b = kk + 32
            int pa = kInf, pb = kInf, sa = kInf, sb = kInf;
            if (k0 < lastW)
            {
                const int d = __float2int_rn(dp0);
                pa = (d - 2 * k0) * 64 + k0;
                sa = (d + 2 * k0) * 64 + k0;
            }
            if (k1 < lastW)
            {
                const int d = __float2int_rn(dp1);
                pb = (d - 2 * k1) * 64 + k1;
                sb = (d + 2 * k1) * 64 + k1;
            }
#pragma unroll
            for (int d = 1; d < 32; d <<= 1)
            {
                const int ta = __shfl_up_sync(kFull, pa, d), tb = __shfl_up_sync(kFull, pb, d);
                const int ua = __shfl_down_sync(kFull, sa, d), ub = __shfl_down_sync(kFull, sb, d);
                if (lane >= d)
                {
                    pa = min(pa, ta);
                    pb = min(pb, tb);
                }
                if (lane + d < 32)
                {
                    sa = min(sa, ua);
                    sb = min(sb, ub);
                }
            }
            pb = min(pb, __shfl_sync(kFull, pa, 31));  // prefixes of slot b include all of slot a
            sa = min(sa, __shfl_sync(kFull, sb, 0));   // suffixes of slot a include all of slot b
            // each candidate: b(t) at t = lo + k, position j = t - lastLo in the previous line
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int kc = h == 0 ? k0 : k1;
                const int j = lo + kc - lastLo;
                const int iF = min(max(j, 0), lastW - 1), iB = min(max(j, 0), lastW - 1);
                const int fa = __shfl_sync(kFull, pa, iF & 31), fb = __shfl_sync(kFull, pb, iF & 31);
                const int ba = __shfl_sync(kFull, sa, iB & 31), bb = __shfl_sync(kFull, sb, iB & 31);
                if (kc >= lw) continue;
                int bv = 0, bi = -1;
                if (j >= 0)
                {
                    const int key = iF < 32 ? fa : fb;
                    bv = (key >> 6) + 2 * j;
                    bi = key & 63;
                }
                if (j <= lastW - 1)
                {
                    const int key = iB < 32 ? ba : bb;
                    const int v = (key >> 6) - 2 * j, i = key & 63;
                    if (bi < 0 || v < bv || (v == bv && i < bi))
                    {
                        bv = v;
                        bi = i;
                    }
                }
                const float val = fadd(h == 0 ? c0 : c1, (float)bv);
                if (h == 0)
                {
                    v0 = val;
                    bp0 = bi;
                }
                else
                {
                    v1 = val;
                    bp1 = bi;
                }
            }
        }
        if (k0 < lw) sBack[(size_t)line * kSeamBand + k0] = (unsigned char)(bp0 < 0 ? 255 : bp0);
        if (k1 < lw) sBack[(size_t)line * kSeamBand + k1] = (unsigned char)(bp1 < 0 ? 255 : bp1);
        if (lane == 0) sPrev[line] = last;
        dp0 = v0;
        dp1 = v1;
        last = line;
        lastLo = lo;
        lastW = lw;
        cur ^= 1;
        // The next line is exact if this line's values are below 2^23 (with
        // costs below 2^18 and penalties below 2^21 its sums stay below
        // 2^24); values are non-negative, so their bits order as the values.
        const unsigned mv = __reduce_max_sync(kFull, max(k0 < lw ? __float_as_uint(v0) : 0u,
                                                         k1 < lw ? __float_as_uint(v1) : 0u));
        if (mv >= __float_as_uint(8388608.0f))
        {
            ++ci2;
            break;
        }
    }
    // the last line's values where the general form and the final choice read them
    if (k0 < lastW) dpBuf[cur ^ 1][k0] = dp0;
    if (k1 < lastW) dpBuf[cur ^ 1][k1] = dp1;
    outStart = ci2;
    outLast = last;
    outLastW = lastW;
    outCur = cur;
}

__global__ void __launch_bounds__(kSeamThreads, 1) k_seam(BlendArgs a, const int* __restrict__ tileList, int smemLines)
{
    extern __shared__ unsigned char sm_seam[];
    __shared__ float dpBuf[2][64];
    __shared__ int sLast, sBestK;
    __shared__ int sDpStart, sDpLast, sDpLastW, sDpCur;  // where the warp form of the DP stopped
    __shared__ int sBand[4];  // first and last contested line, lowest lo and highest hi of a pair
    const int tileIndex = tileList[blockIdx.x];
    const TileDev& T = a.tiles[tileIndex];
    const long long tileStart = clock64();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    constexpr int nwarps = kSeamThreads / 32;
    const int K = T.numItems;
    const int w = T.w;
    const bool inSmem = T.maxLines <= smemLines;
    int* sLo = inSmem ? reinterpret_cast<int*>(sm_seam) : T.lo;
    int* sHi = inSmem ? sLo + smemLines : T.hi;
    int* sPrev = inSmem ? sHi + smemLines : T.prevLine;
    // Contested lines in increasing order (the DP's iteration list).
    int* sList = inSmem ? sPrev + smemLines : T.list;
    unsigned char* sBack = inSmem ? reinterpret_cast<unsigned char*>(sList + smemLines) : T.back;
    __shared__ int sWarpCnt[kSeamThreads / 32 + 1];
    __shared__ int sNumContested;

    for (int i = 0; i < K; ++i)
    {
        const ItemDev& I = a.items[T.firstItem + i];
        const int bI[4] = {I.bbox[0], I.bbox[1], I.bbox[2], I.bbox[3]};
        if (bI[2] < 0) continue;
        for (int j = i + 1; j < K; ++j)
        {
            const ItemDev& J = a.items[T.firstItem + j];
            const int bJ[4] = {J.bbox[0], J.bbox[1], J.bbox[2], J.bbox[3]};
            if (bJ[2] < 0) continue;
            const int ox0 = max(bI[0], bJ[0]), oy0 = max(bI[1], bJ[1]);
            const int ox1 = min(bI[2], bJ[2]), oy1 = min(bI[3], bJ[3]);
            if (!(ox0 <= ox1 && oy0 <= oy1)) continue;
            const int bw = ox1 - ox0 + 1, bh = oy1 - oy0 + 1;
            const bool rowScan = bw >= bh;
            const float cI = rowScan ? fmul((float)(bI[0] + bI[2]), 0.5f) : fmul((float)(bI[1] + bI[3]), 0.5f);
            const float cJ = rowScan ? fmul((float)(bJ[0] + bJ[2]), 0.5f) : fmul((float)(bJ[1] + bJ[3]), 0.5f);
            const bool iLow = cI <= cJ;
            const int numLines = rowScan ? bh : bw;
            const int lineLen = rowScan ? bw : bh;
            const int ci = i, cj = j;
            auto pix = [&](int line, int t) -> size_t {
                return rowScan ? (size_t)(oy0 + line) * w + (ox0 + t) : (size_t)(oy0 + t) * w + (ox0 + line);
            };
            auto both_cov = [&](int line, int t) -> bool {
                const int x = rowScan ? ox0 + t : ox0 + line;
                const int y = rowScan ? oy0 + line : oy0 + t;
                return cov_bit(I.cov, T.covWords, x, y) && cov_bit(J.cov, T.covWords, x, y);
            };

            long long tp = clock64();
            // Phase 1: crossover of each line (SeamBlend.cpp:334-345) and its band.
            if (rowScan)
            {
                const unsigned repI = (unsigned)ci * 0x01010101u, repJ = (unsigned)cj * 0x01010101u;
                for (int line = warp; line < numLines; line += nwarps)
                {
                    const signed char* rowp = T.owner + pix(line, 0);
                    const uintptr_t base = reinterpret_cast<uintptr_t>(rowp) & ~uintptr_t(15);
                    const int off = (int)(reinterpret_cast<uintptr_t>(rowp) - base);
                    const int nChunks = (off + lineLen + 15) >> 4;
                    const uint4* src = reinterpret_cast<const uint4*>(base);
                    // pass A: first position owned by I or J, and that owner
                    int p1 = 0x7fffffff, v1 = -1;
                    for (int c0 = 0; c0 < nChunks && p1 == 0x7fffffff; c0 += 32)
                    {
                        const int c = c0 + lane;
                        int f = 0x7fffffff;
                        if (c < nChunks) f = first_owner_in_chunk(src[c], repI, repJ, c * 16 - off, lineLen);
                        p1 = __reduce_min_sync(kFull, f);
                    }
                    int cross = -1;
                    if (p1 != 0x7fffffff)
                    {
                        v1 = (int)T.owner[pix(line, p1)];
                        const unsigned repO = (v1 == ci ? (unsigned)cj : (unsigned)ci) * 0x01010101u;  // the other of I, J
                        const int cStart = (p1 + off) >> 4;
                        int f2 = 0x7fffffff;
                        for (int c0 = cStart; c0 < nChunks && f2 == 0x7fffffff; c0 += 32)
                        {
                            const int c = c0 + lane;
                            int f = 0x7fffffff;
                            if (c < nChunks) f = first_owner_in_chunk(src[c], repO, repO, c * 16 - off, lineLen);
                            if (f <= p1) f = 0x7fffffff;  // only positions after the first I/J pixel
                            f2 = __reduce_min_sync(kFull, f);
                        }
                        if (f2 != 0x7fffffff) cross = f2;
                    }
                    int lo = 1, hi = 0;
                    if (cross >= 0)
                    {
                        const int bLo = max(0, cross - kSeamRadius);
                        const int bHi = min(lineLen - 1, cross + kSeamRadius);
                        const int ta = bLo + lane, tb = bLo + 32 + lane;
                        const bool b0 = ta <= bHi && both_cov(line, ta);
                        const bool b1 = tb <= bHi && both_cov(line, tb);
                        const unsigned m0 = __ballot_sync(kFull, b0), m1 = __ballot_sync(kFull, b1);
                        if (m0 | m1)
                        {
                            lo = bLo + (m0 ? __ffs(m0) - 1 : 32 + __ffs(m1) - 1);
                            hi = bLo + (m1 ? 32 + 31 - __clz(m1) : 31 - __clz(m0));
                        }
                    }
                    if (lane == 0)
                    {
                        sLo[line] = lo;
                        sHi[line] = hi;
                    }
                }
            }
            else if ((reinterpret_cast<uintptr_t>(T.owner) & 15) == 0)
            {
                // Lines are columns.  The crossover of a column (the first
                // pixel of the other owner after its first I/J pixel) is the
                // later of the column's first I row and first J row, so both
                // are found by one parallel pass over the overlap box instead
                // of a walk down each column: 16-byte chunks of each row,
                // threads over (chunk, row segment), each segment scanned
                // top-down and its first finds merged by atomicMin into the
                // line arrays (used for the first rows here, overwritten with
                // the band below).  With a row pitch that is a multiple of 16
                // the chunks are the aligned ones (the same column offset on
                // every row); otherwise a chunk is 16 columns of the box, read
                // as the aligned chunk(s) holding them.
                int* fI = sLo;
                int* fJ = sHi;
                for (int l = tid; l < numLines; l += kSeamThreads) fI[l] = fJ[l] = 0x7fffffff;
                __syncthreads();
                const bool pitch16 = (w & 15) == 0;
                const signed char* rowp0 = T.owner + pix(0, 0);
                const int off = pitch16 ? (int)(reinterpret_cast<uintptr_t>(rowp0) & 15) : 0;
                const int nCh = (off + numLines + 15) >> 4;
                const int nSeg = max(1, kSeamThreads / nCh);
                const int segRows = (lineLen + nSeg - 1) / nSeg;
                const unsigned repI = (unsigned)ci * 0x01010101u, repJ = (unsigned)cj * 0x01010101u;
                for (int job = tid; job < nCh * nSeg; job += kSeamThreads)
                {
                    const int seg = job / nCh, c = job - seg * nCh;
                    const int tb = 16 * c - off;  // column of the chunk's byte 0
                    const int b0 = max(0, -tb), b1 = min(16, numLines - tb);
                    const unsigned valid = ((1u << b1) - 1u) & ~((1u << b0) - 1u);
                    unsigned foundI = 0, foundJ = 0;
                    const int t1 = min(lineLen, (seg + 1) * segRows);
                    for (int t = seg * segRows; t < t1 && (foundI & foundJ) != valid; ++t)
                    {
                        // byte b of v: column tb + b of row t
                        const signed char* at = rowp0 + (size_t)t * w + tb;
                        const int o = (int)(reinterpret_cast<uintptr_t>(at) & 15);
                        const uint4* ch = reinterpret_cast<const uint4*>(at - o);
                        uint4 v = ch[0];
                        if (o != 0)
                        {
                            // the second chunk only when a byte of the box lies
                            // in it (so the read stays within the map's padding)
                            const uint4 nx = o + b1 > 16 ? ch[1] : make_uint4(0u, 0u, 0u, 0u);
                            v = bytes16_at(v, nx, o);
                        }
                        const unsigned nI = chunk_byte_mask(v, repI) & valid & ~foundI;
                        const unsigned nJ = chunk_byte_mask(v, repJ) & valid & ~foundJ;
                        for (unsigned m = nI; m; m &= m - 1) atomicMin(&fI[tb + __ffs(m) - 1], t);
                        for (unsigned m = nJ; m; m &= m - 1) atomicMin(&fJ[tb + __ffs(m) - 1], t);
                        foundI |= nI;
                        foundJ |= nJ;
                    }
                }
                __syncthreads();
                for (int line = tid; line < numLines; line += kSeamThreads)
                {
                    const int a1 = fI[line], a2 = fJ[line];
                    const int cross = (a1 != 0x7fffffff && a2 != 0x7fffffff) ? max(a1, a2) : -1;
                    seam_column_band(I.cov, J.cov, T.covWords, ox0 + line, oy0, cross, lineLen, sLo[line],
                                     sHi[line]);
                }
            }
            else
            {
                for (int line = tid; line < numLines; line += kSeamThreads)
                {
                    int first = -1000, cross = -1;
                    for (int t0 = 0; t0 < lineLen && cross < 0; t0 += 16)
                    {
                        // 16 independent loads in flight, then a sequential walk.
                        int ov[16];
#pragma unroll
                        for (int q = 0; q < 16; ++q) ov[q] = (t0 + q < lineLen) ? (int)T.owner[pix(line, t0 + q)] : -2;
#pragma unroll
                        for (int q = 0; q < 16; ++q)
                        {
                            const int o = ov[q];
                            if (cross >= 0 || (o != ci && o != cj)) continue;
                            if (first == -1000) first = o;
                            else if (o != first) cross = t0 + q;
                        }
                    }
                    seam_column_band(I.cov, J.cov, T.covWords, ox0 + line, oy0, cross, lineLen, sLo[line], sHi[line]);
                }
            }
            __syncthreads();

            if (tid == 0) { long long now = clock64(); atomicAdd(a.seamCycles + 0, (unsigned long long)(now - tp)); tp = now; }
            // Phase 2: colour cost of every contested candidate
            // (SeamBlend.cpp:381-383); consecutive threads take neighbouring
            // pixels for either scan direction.
#pragma unroll 4
            for (int idx = tid; idx < numLines * kSeamBand; idx += kSeamThreads)
            {
                int line, k;
                if (rowScan) { line = idx / kSeamBand; k = idx - line * kSeamBand; }
                else { k = idx / numLines; line = idx - k * numLines; }
                if (k == 0) T.chosen[line] = -1;
                const int lo = sLo[line], hi = sHi[line];
                if (k > hi - lo) continue;
                const size_t p = pix(line, lo + k);
                const unsigned short* pa = I.img + p * 3;
                const unsigned short* pb = J.img + p * 3;
                float c = 0.0f;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) c = fadd(c, fabsf(fsub((float)pa[ch], (float)pb[ch])));
                T.cost[(size_t)line * kSeamBand + k] = c;
            }
            __syncthreads();

            if (tid == 0) { long long now = clock64(); atomicAdd(a.seamCycles + 1, (unsigned long long)(now - tp)); tp = now; }
            // Phase 3a: compact the contested lines (hi >= lo) in order.
            {
                const int per = (numLines + kSeamThreads - 1) / kSeamThreads;  // lines per thread, contiguous
                const int l0 = tid * per, l1 = min(l0 + per, numLines);
                int c = 0;
                for (int l = l0; l < l1; ++l) c += sHi[l] >= sLo[l] ? 1 : 0;
                int incl = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1)
                {
                    int v = __shfl_up_sync(kFull, incl, d);
                    if (lane >= d) incl += v;
                }
                if (lane == 31) sWarpCnt[warp] = incl;
                if (tid == 0)
                {
                    sBand[0] = sBand[2] = 0x7fffffff;
                    sBand[1] = sBand[3] = -1;
                }
                __syncthreads();
                if (tid == 0)
                {
                    int acc = 0;
                    for (int w2 = 0; w2 < nwarps; ++w2)
                    {
                        int v = sWarpCnt[w2];
                        sWarpCnt[w2] = acc;
                        acc += v;
                    }
                    sNumContested = acc;
                }
                __syncthreads();
                int pos = sWarpCnt[warp] + incl - c;
                // and the box of the contested bands (lines x positions): the
                // reassignment gives I or J pixels only inside it
                int bl0 = 0x7fffffff, bl1 = -1, bt0 = 0x7fffffff, bt1 = -1;
                for (int l = l0; l < l1; ++l)
                {
                    sPrev[l] = -1;
                    if (sHi[l] >= sLo[l])
                    {
                        sList[pos++] = l;
                        bl0 = min(bl0, l);
                        bl1 = max(bl1, l);
                        bt0 = min(bt0, sLo[l]);
                        bt1 = max(bt1, sHi[l]);
                    }
                }
                bl0 = __reduce_min_sync(kFull, bl0);
                bl1 = __reduce_max_sync(kFull, bl1);
                bt0 = __reduce_min_sync(kFull, bt0);
                bt1 = __reduce_max_sync(kFull, bt1);
                if (lane == 0 && bl1 >= 0)
                {
                    atomicMin(&sBand[0], bl0);
                    atomicMax(&sBand[1], bl1);
                    atomicMin(&sBand[2], bt0);
                    atomicMax(&sBand[3], bt1);
                }
                __syncthreads();
                if (tid == 0 && sBand[1] >= 0)
                {
                    // tile coordinates: a row line is a y and its positions x;
                    // a column line the reverse
                    const int bx0 = rowScan ? ox0 + sBand[2] : ox0 + sBand[0];
                    const int bx1 = rowScan ? ox0 + sBand[3] : ox0 + sBand[1];
                    const int by0 = rowScan ? oy0 + sBand[0] : oy0 + sBand[2];
                    const int by1 = rowScan ? oy0 + sBand[1] : oy0 + sBand[3];
                    for (int q = 0; q < 2; ++q)
                    {
                        int* ob = a.items[T.firstItem + (q == 0 ? ci : cj)].bbox + kOwnedBox;
                        atomicMin(ob, bx0);
                        atomicMin(ob + 1, by0);
                        atomicMax(ob + 2, bx1);
                        atomicMax(ob + 3, by1);
                    }
                }
            }
            // Phase 3b: dynamic program over contested lines
            // (SeamBlend.cpp:362-407).  First on one warp while its values
            // are small integers (seam_dp_warp); from the line where that
            // stops, on the first kDpThreads threads: 8 threads share a
            // candidate k, each scanning every 8th entry of the previous line
            // in index order; the parts merge to the lowest (value, index),
            // which is what the reference's strict '<' scan in index order
            // keeps.  Penalties 2|t - pt| are exact small integers formed in
            // float.  Candidate costs are fetched kPre lines ahead.
            if (warp == 0)
            {
                int st, la, lw, cu;
                seam_dp_warp(sList, sLo, sHi, sPrev, sBack, T.cost, sNumContested, lineLen, dpBuf, lane, st, la, lw,
                             cu);
                if (lane == 0)
                {
                    sDpStart = st;
                    sDpLast = la;
                    sDpLastW = lw;
                    sDpCur = cu;
                }
            }
            __syncthreads();
            if (tid < kDpThreads && sDpStart < sNumContested)
            {
                constexpr int kPre = 4;
                constexpr int kParts = 8;
                const int k = tid / kParts, part = tid % kParts;
                const int nC = sNumContested, start = sDpStart;
                float cq[kPre];
#pragma unroll
                for (int q = 0; q < kPre; ++q)
                {
                    cq[q] = 0.0f;
                    if (start + q < nC)
                    {
                        const int l = sList[start + q];
                        if (k <= sHi[l] - sLo[l]) cq[q] = T.cost[(size_t)l * kSeamBand + k];
                    }
                }
                int last = sDpLast, cur = sDpCur, lastW = sDpLastW;
                for (int ci2 = start; ci2 < nC; ++ci2)
                {
                    const int line = sList[ci2];
                    const int lo = sLo[line], lw = sHi[line] - lo + 1;
                    const float c = cq[0];
#pragma unroll
                    for (int q = 0; q + 1 < kPre; ++q) cq[q] = cq[q + 1];
                    cq[kPre - 1] = 0.0f;
                    if (ci2 + kPre < nC)
                    {
                        const int l = sList[ci2 + kPre];
                        if (k <= sHi[l] - sLo[l]) cq[kPre - 1] = T.cost[(size_t)l * kSeamBand + k];
                    }
                    float val = c;
                    int bp = -1;
                    float b = FLT_MAX;
                    if (last >= 0 && k < lw)
                    {
                        const float d0 = (float)(lo + k - sLo[last]);  // t - pt at pk = 0
#pragma unroll
                        for (int i = 0; i < (kSeamBand + kParts - 1) / kParts; ++i)
                        {
                            const int kk = part + kParts * i;
                            if (kk < lastW)
                            {
                                const float dd = fsub(d0, (float)kk);
                                const float pen = fadd(fabsf(dd), fabsf(dd));
                                const float c2 = fadd(dpBuf[cur ^ 1][kk], pen);
                                if (c2 < b)
                                {
                                    b = c2;
                                    bp = kk;
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int m = 1; m < kParts; m <<= 1)
                    {
                        const float ob = __shfl_xor_sync(0xffffffffu, b, m);
                        const int obp = __shfl_xor_sync(0xffffffffu, bp, m);
                        if (obp >= 0 && (bp < 0 || ob < b || (ob == b && obp < bp)))
                        {
                            b = ob;
                            bp = obp;
                        }
                    }
                    if (last >= 0 && k < lw) val = fadd(c, b);
                    if (part == 0 && k < lw)
                    {
                        dpBuf[cur][k] = val;
                        sBack[(size_t)line * kSeamBand + k] = (unsigned char)(bp < 0 ? 255 : bp);
                    }
                    if (tid == 0) sPrev[line] = last;
                    last = line;
                    lastW = lw;
                    cur ^= 1;
                    asm volatile("bar.sync 1, %0;" ::"r"(kDpThreads) : "memory");
                }
                if (tid == 0)
                {
                    sDpLast = last;
                    sDpLastW = lastW;
                    sDpCur = cur;
                }
            }
            __syncthreads();
            if (tid == 0)
            {
                const int last = sDpLast, lastW = sDpLastW, cur = sDpCur;
                sLast = last;
                int bestK = 0;
                if (last >= 0)
                {
                    float best = FLT_MAX;
                    for (int q = 0; q < lastW; ++q)
                        if (dpBuf[cur ^ 1][q] < best)
                        {
                            best = dpBuf[cur ^ 1][q];
                            bestK = q;
                        }
                }
                sBestK = bestK;
            }
            __syncthreads();
            if (tid == 0) { long long now = clock64(); atomicAdd(a.seamCycles + 2, (unsigned long long)(now - tp)); tp = now; }
            // Phase 4: backtrack (SeamBlend.cpp:411-428).
            if (tid == 0 && sLast >= 0)
            {
                int line = sLast, k = sBestK;
                while (line >= 0 && k >= 0)
                {
                    T.chosen[line] = sLo[line] + k;
                    const int pl = sPrev[line];
                    const int pk = sBack[(size_t)line * kSeamBand + k];
                    line = pl;
                    k = pk == 255 ? -1 : pk;
                }
            }
            __syncthreads();

            if (tid == 0) { long long now = clock64(); atomicAdd(a.seamCycles + 3, (unsigned long long)(now - tp)); tp = now; }
            // Phase 5: reassign I/J pixels inside each contested band
            // (SeamBlend.cpp:430-444).
            if (sLast >= 0)
            {
                for (int idx = tid; idx < numLines * kSeamBand; idx += kSeamThreads)
                {
                    int line, k;
                    if (rowScan) { line = idx / kSeamBand; k = idx - line * kSeamBand; }
                    else { k = idx / numLines; line = idx - k * numLines; }
                    const int ch = T.chosen[line];
                    if (ch < 0) continue;
                    const int lo = sLo[line], hi = sHi[line];
                    if (k > hi - lo) continue;
                    const int t = lo + k;
                    const size_t p = pix(line, t);
                    const signed char o = T.owner[p];
                    if (o != ci && o != cj) continue;
                    const bool onLow = t < ch;
                    T.owner[p] = (signed char)((onLow == iLow) ? ci : cj);
                }
            }
            __syncthreads();
            if (tid == 0) atomicAdd(a.seamCycles + 4, (unsigned long long)(clock64() - tp));
        }
    }
    if (tid == 0) a.seamTile[tileIndex] = (unsigned long long)(clock64() - tileStart);
}

// ---------------------------------------------------------------------------
// Pyramid (SeamBlend.cpp:15-201, 447-546).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float blur5(float a, float b, float c, float d, float e)
{
    // k0*a + k1*b + k2*c + k1*d + k0*e, left to right (SeamBlend.cpp:31-36).
    const float k0 = 1.0f / 16.0f, k1 = 4.0f / 16.0f, k2 = 6.0f / 16.0f;
    return fadd(fadd(fadd(fadd(fmul(k0, a), fmul(k1, b)), fmul(k2, c)), fmul(k1, d)), fmul(k0, e));
}

struct UpCoef
{
    int x0, x1, y0, y1;
    float wx, wy;
};

// Align-corners bilinear resize coefficients (SeamBlend.cpp:85-115); the
// scales sx, sy = (src-1)/(dst-1) are computed once per tile and level.
// Coordinates and scales are non-negative and below 2^23, so the int/float
// conversions (and the truncation, which is the floor there) are the exact
// ones of u2f / f2u_floor.
__device__ __forceinline__ void up_coef_x(float sx, int sw, int x, int& x0, float& wx)
{
    const float fx = fmul(sx, u2f((uint32_t)x));
    x0 = min((int)f2u_floor(fx), sw - 1);
    wx = fsub(fx, u2f((uint32_t)x0));
}

__device__ __forceinline__ UpCoef up_coef_s(float sx, float sy, int sw, int sh, int x, int y)
{
    UpCoef c;
    up_coef_x(sy, sh, y, c.y0, c.wy);
    c.y1 = min(c.y0 + 1, sh - 1);
    up_coef_x(sx, sw, x, c.x0, c.wx);
    c.x1 = min(c.x0 + 1, sw - 1);
    return c;
}

__device__ __forceinline__ float up_mix(float v00, float v10, float v01, float v11, float wx, float wy)
{
    float ix = fsub(1.0f, wx), iy = fsub(1.0f, wy);
    return fadd(fmul(iy, fadd(fmul(ix, v00), fmul(wx, v10))), fmul(wy, fadd(fmul(ix, v01), fmul(wx, v11))));
}

// Hole-filled Gaussian value G = num * (den > 1e-6 ? 1/den : 0)
// (SeamBlend.cpp:175-180).
__device__ __forceinline__ float3 gauss_of(float4 nd)
{
    // 1.0f / den, correctly rounded (the reference's division).
    float inv = (nd.w > 1e-6f) ? __frcp_rn(nd.w) : 0.0f;
    return make_float3(fmul(nd.x, inv), fmul(nd.y, inv), fmul(nd.z, inv));
}

// A contributor's pyramid value (num.rgb, den) and weight at index q of a
// materialised level.  Exact mode: FP32 as computed.  FP16 storage (the
// native mode): the same buffers hold half4 (num / 256, den) and a half
// weight - num is scaled by 2^-8 (exactly) so that sums of 16-bit samples
// stay inside the half range; all arithmetic stays FP32.
__device__ __forceinline__ float4 nd_at(const float4* nd, size_t q, int half)
{
    if (!half) return __ldg(nd + q);
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(nd) + q);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    return make_float4(a.x * 256.0f, a.y * 256.0f, b.x * 256.0f, b.y);
}

// The levels gmin and above of a contributor's pyramid hold, once the band
// blend of their level has run, the hole-filled Gaussian G = num * (1/den) in
// place of num: the blend of the level below, the level-0 output (level 1)
// and the fused fine kernel (level 2) read Up(G) taps, each value about
// sixteen times, and the reciprocal is then computed once per value instead
// of once per tap.  The stored G is the value gauss_of would compute, so the
// taps are bit-identical in the exact mode (with FP16 storage G / 256 is
// stored as FP16, like num / 256 before).  gmin is 1 with every level
// materialised (the level-1 blend runs before the output) and 2 with the
// fused levels (level 1 has no blend of its own).  In the exact mode G is
// stored only where the contributor's weight at that level is non-zero:
// every reader takes Up(G) taps only for a pixel of non-zero weight one level
// below (a blend term, or an owned level-0 pixel), each such tap has that
// pixel in its 5-tap footprint (align-corners: |x - 2 x0| <= 2), and the
// weight there is then a sum containing a positive product - non-zero.  A
// tap elsewhere only enters a term of weight zero, which is +-0 for any
// finite value.  (FP16 weights can round to zero, so that mode stores G
// wherever the blend passes.)
__device__ __forceinline__ bool g_stored(int level, int gmin) { return level >= gmin; }

__device__ __forceinline__ float3 g_at(const float4* nd, size_t q, int level, int gmin, int half)
{
    if (g_stored(level, gmin))
    {
        const float4 v = nd_at(nd, q, half);
        return make_float3(v.x, v.y, v.z);
    }
    return gauss_of(nd_at(nd, q, half));
}

__device__ __forceinline__ void g_store(const float4* nd, size_t q, float3 g, int half)
{
    if (!half)
    {
        const_cast<float4*>(nd)[q] = make_float4(g.x, g.y, g.z, 0.0f);
        return;
    }
    const __half2 a = __floats2half2_rn(g.x * (1.0f / 256.0f), g.y * (1.0f / 256.0f));
    const __half2 b = __floats2half2_rn(g.z * (1.0f / 256.0f), 0.0f);
    reinterpret_cast<uint2*>(const_cast<float4*>(nd))[q] =
        make_uint2(*reinterpret_cast<const uint32_t*>(&a), *reinterpret_cast<const uint32_t*>(&b));
}

__device__ __forceinline__ float wg_at(const float* wg, size_t q, int half)
{
    if (!half) return __ldg(wg + q);
    return __half2float(__ushort_as_half(__ldg(reinterpret_cast<const unsigned short*>(wg) + q)));
}

__device__ __forceinline__ void pyr_store(float4* nd, float* wg, size_t q, float4 v, float w, int half)
{
    if (!half)
    {
        nd[q] = v;
        wg[q] = w;
        return;
    }
    const __half2 a = __floats2half2_rn(v.x * (1.0f / 256.0f), v.y * (1.0f / 256.0f));
    const __half2 b = __floats2half2_rn(v.z * (1.0f / 256.0f), v.w);
    reinterpret_cast<uint2*>(nd)[q] = make_uint2(*reinterpret_cast<const uint32_t*>(&a),
                                                 *reinterpret_cast<const uint32_t*>(&b));
    reinterpret_cast<unsigned short*>(wg)[q] = __half_as_ushort(__float2half_rn(w));
}

// Blur + decimate one level (SeamBlend.cpp:60-79) for num(3), den and weight
// together.  A CTA makes a 32x8 block of level l+1 from a 68x20 footprint of
// level l staged in shared memory with replicated borders.
constexpr int kDnTW = 32, kDnTH = 16;
constexpr int kDnSW = 2 * kDnTW + 4, kDnSH = 2 * kDnTH + 4;

__global__ void __launch_bounds__(256) k_down(BlendArgs a, const Unit* __restrict__ units, int level)
{
    // Footprint staged deinterleaved (even / odd columns in separate planes)
    // so the horizontal taps of consecutive output columns are consecutive
    // shared-memory words: no bank conflicts.
    constexpr int HW = kDnSW / 2;
    extern __shared__ float dn_smem[];
    auto E = reinterpret_cast<float (*)[kDnSH][HW]>(dn_smem);
    auto O = reinterpret_cast<float (*)[kDnSH][HW]>(dn_smem + 5 * kDnSH * HW);
    auto t = reinterpret_cast<float (*)[kDnSH][kDnTW]>(dn_smem + 10 * kDnSH * HW);
    const Unit u = units[blockIdx.x];
    const ItemDev& it = a.items[u.id];
    const TileDev& T = a.tiles[it.tile];
    const int sw = T.lw[level], sh = T.lh[level];
    const int dw = T.lw[level + 1], dh = T.lh[level + 1];
    const int X0 = u.bx * kDnTW, Y0 = u.by * kDnTH;
    const int tid = threadIdx.x;
    // A footprint (rows 2Y0-2 .. 2Y0+33, columns 2X0-2 .. 2X0+65) outside
    // the contributor's support at this level reads only zeros.
    // Likewise a block outside the box where level l+1's num/den are read
    // (needed_box): its weights are zero.
    const int4 B = support_box(covered_box(it.bbox), level);
    const int4 nb = needed_box(it.bbox, level + 1, T.bands - 1);
    if (2 * X0 + 2 * kDnTW + 1 < B.x || 2 * X0 - 2 > B.z || 2 * Y0 + 2 * kDnTH + 1 < B.y || 2 * Y0 - 2 > B.w ||
        X0 + kDnTW - 1 < nb.x || X0 > nb.z || Y0 + kDnTH - 1 < nb.y || Y0 > nb.w)
    {
        for (int idx = tid; idx < kDnTW * kDnTH; idx += 256)
        {
            const int X = X0 + (idx & (kDnTW - 1)), Y = Y0 + idx / kDnTW;
            if (X >= dw || Y >= dh) continue;
            const size_t q = T.loff[level + 1] + (size_t)Y * dw + X;
            pyr_store(it.nd, it.wg, q, make_float4(0.0f, 0.0f, 0.0f, 0.0f), 0.0f, a.half);
        }
        return;
    }
    const size_t lq = T.loff[level];
    for (int idx = tid; idx < HW * kDnSH; idx += 256)
    {
        const int r = idx / HW, cp = idx - r * HW;
        const int gy = min(max(2 * Y0 - 2 + r, 0), sh - 1);
#pragma unroll
        for (int e = 0; e < 2; ++e)
        {
            const int gx = min(max(2 * X0 - 2 + 2 * cp + e, 0), sw - 1);
            const size_t p = (size_t)gy * sw + gx;
            float v[5];
            const float4 q = nd_at(it.nd, lq + p, a.half);
            v[0] = q.x;
            v[1] = q.y;
            v[2] = q.z;
            v[3] = q.w;
            v[4] = wg_at(it.wg, lq + p, a.half);
#pragma unroll
            for (int ch = 0; ch < 5; ++ch)
            {
                if (e == 0) E[ch][r][cp] = v[ch];
                else O[ch][r][cp] = v[ch];
            }
        }
    }
    __syncthreads();
    // Horizontal taps at the even columns that survive decimation:
    // output i is centred on footprint column 2i + 2.
    for (int idx = tid; idx < 5 * kDnSH * kDnTW; idx += 256)
    {
        const int ch = idx / (kDnSH * kDnTW);
        const int rem = idx - ch * kDnSH * kDnTW;
        const int r = rem / kDnTW, i = rem - r * kDnTW;
        t[ch][r][i] = blur5(E[ch][r][i], O[ch][r][i], E[ch][r][i + 1], O[ch][r][i + 1], E[ch][r][i + 2]);
    }
    __syncthreads();
    const int i = tid & 31;
    for (int j = tid >> 5; j < kDnTH; j += 8)
    {
        const int X = X0 + i, Y = Y0 + j;
        if (X >= dw || Y >= dh) continue;
        float o[5];
#pragma unroll
        for (int ch = 0; ch < 5; ++ch)
            o[ch] = blur5(t[ch][2 * j][i], t[ch][2 * j + 1][i], t[ch][2 * j + 2][i], t[ch][2 * j + 3][i],
                          t[ch][2 * j + 4][i]);
        const size_t q = T.loff[level + 1] + (size_t)Y * dw + X;
        pyr_store(it.nd, it.wg, q, make_float4(o[0], o[1], o[2], o[3]), o[4], a.half);
    }
}

// Level 0 -> 1 of a contributor's pyramids in integer arithmetic, streamed
// through registers.  At level 0 every blur input is an integer: pixel values
// (<= 65535, zero where uncovered), the 0/1 coverage and the 0/1 ownership
// mask.  With the [1,4,6,4,1]/16 kernel each product of the reference's FP32
// sequence is exact, every horizontal partial sum is a multiple of 1/16 below
// 2^16 and every vertical one a multiple of 1/256 below 2^16 (at most 24
// significant bits), so no step rounds: the level-1 value IS
// (sum_ij c_i c_j v_ij) / 256, and computing that sum in integers is
// bit-identical to the FP32 chain of SeamBlend.cpp:15-79 (blur with clamped
// borders, then decimation; num = img * coverage, den = coverage, weight =
// owner mask).  Coverage and ownership sums (<= 256 each) share one int as
// den << 16 | weight.  No shared memory: a warp
// makes one 64 x 16 block of level 1, lane i the output columns X0 + 2i and
// X0 + 2i + 1.  Each of the block's 36 footprint rows is read once - lane i's
// four level-0 pixels 2X .. 2X+3 as three 8-byte words, the halo pixels
// 2X-2, 2X-1 and 2X+4 from the neighbouring lanes by shuffle - blurred
// horizontally in registers and added into the output rows it feeds: an even
// row 2m completes output row m-2 (weight 1), adds 6x to row m-1 and starts
// row m; an odd row 2m+1 adds 4x to rows m-1 and m.  Warps whose footprint
// touches the tile's side edges (clamping) or whose rows are not 8-byte
// aligned read each footprint pixel with clamped scalar loads instead.
constexpr int kDnWarps = 8;
constexpr int kDn0W = 64;  // level-1 columns per warp

// One level-0 pixel packed for the shuffles: r | g << 16, b | coverage << 16 | owned << 17.
struct PackedPx
{
    uint32_t rg, bw;
};

__device__ __forceinline__ PackedPx pack_px(uint32_t r, uint32_t g, uint32_t b, bool owned)
{
    const uint32_t mk = (r | g | b) ? 1u : 0u;
    return PackedPx{r | (g << 16), b | (mk << 16) | ((owned ? 1u : 0u) << 17)};
}

__device__ __forceinline__ PackedPx load_px(const unsigned short* img, const signed char* own, size_t p,
                                            signed char k)
{
    const unsigned short* q = img + p * 3;
    return pack_px(__ldg(q), __ldg(q + 1), __ldg(q + 2), __ldg(own + p) == k);
}

// The four channel values r, g, b and (coverage << 16 | owned) of one pixel.
__device__ __forceinline__ void px_channels(const PackedPx& v, int* c)
{
    c[0] = (int)(v.rg & 0xffffu);
    c[1] = (int)(v.rg >> 16);
    c[2] = (int)(v.bw & 0xffffu);
    c[3] = (int)(((v.bw >> 16) & 1u) << 16 | (v.bw >> 17));
}

__device__ __forceinline__ PackedPx shfl_px(const PackedPx& v, int delta, bool up)
{
    PackedPx o;
    o.rg = up ? __shfl_up_sync(kFull, v.rg, delta) : __shfl_down_sync(kFull, v.rg, delta);
    o.bw = up ? __shfl_up_sync(kFull, v.bw, delta) : __shfl_down_sync(kFull, v.bw, delta);
    return o;
}

__global__ void __launch_bounds__(256, 4) k_down0s(BlendArgs a, const Unit* __restrict__ units, int n)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ui = blockIdx.x * kDnWarps + warp;
    if (ui >= n) return;  // uniform per warp
    const Unit u = units[ui];
    const ItemDev& it = a.items[u.id];
    const TileDev& T = a.tiles[it.tile];
    const int sw = T.lw[0], sh = T.lh[0];
    const int dw = T.lw[1], dh = T.lh[1];
    const int X0 = u.bx * kDn0W, Y0 = u.by * kDnTH;
    const int X = X0 + 2 * lane;  // this lane's first column
    const unsigned short* img = it.img;
    const signed char* own = T.owner;
    const signed char k = (signed char)it.k;
    const size_t qrow = T.loff[1];
    // A footprint (rows 2Y0-2 .. 2Y0+33, columns 2X0-2 .. 2X0+129, before
    // clamping) that misses the contributor's covered box reads only (0,0,0)
    // pixels it does not own - ownership never leaves the covered box: the
    // seam step reassigns pixels only inside two contributors' common box
    // (SeamBlend.cpp:439-442, 580) - so its outputs are exactly zero.
    {
        const int bx0 = __ldg(it.bbox), by0 = __ldg(it.bbox + 1), bx1 = __ldg(it.bbox + 2), by1 = __ldg(it.bbox + 3);
        // and a block outside the box where level 1's num/den are read (see
        // needed_box) needs only its weights, which are zero there too
        const int4 nb = needed_box(it.bbox, 1, T.bands - 1);
        if (2 * X0 + 2 * kDn0W + 1 < bx0 || 2 * X0 - 2 > bx1 || 2 * Y0 + 2 * kDnTH + 1 < by0 || 2 * Y0 - 2 > by1 ||
            X0 + kDn0W - 1 < nb.x || X0 > nb.z || Y0 + kDnTH - 1 < nb.y || Y0 > nb.w)
        {
            for (int j = 0; j < kDnTH && Y0 + j < dh; ++j)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    if (X + c < dw)
                    {
                        const size_t q = qrow + (size_t)(Y0 + j) * dw + X + c;
                        pyr_store(it.nd, it.wg, q, make_float4(0.0f, 0.0f, 0.0f, 0.0f), 0.0f, a.half);
                    }
            return;
        }
    }
    // 8-byte words need 4-pixel aligned rows on an 8-byte aligned image (a
    // caller's warped buffer may sit at any even address).
    const bool fast = (sw & 3) == 0 && ((reinterpret_cast<uintptr_t>(img) | reinterpret_cast<uintptr_t>(own)) & 7) == 0 &&
                      2 * X0 - 2 >= 0 && 2 * X0 + 2 * kDn0W <= sw - 1;
    int P[2][4], Q[2][4], R[2][4];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int ch = 0; ch < 4; ++ch) P[c][ch] = Q[c][ch] = R[c][ch] = 0;
    for (int r = 0; r < kDnSH; ++r)
    {
        const int gy = min(max(2 * Y0 - 2 + r, 0), sh - 1);
        const size_t rowp = (size_t)gy * sw;
        PackedPx px[7];  // columns 2X-2 .. 2X+4
        if (fast)
        {
            const size_t p0 = rowp + 2 * X;
            const uint2* w = reinterpret_cast<const uint2*>(img + p0 * 3);
            const uint2 w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2);
            const uint32_t ow = __ldg(reinterpret_cast<const uint32_t*>(own + p0));
            px[2] = pack_px(w0.x & 0xffffu, w0.x >> 16, w0.y & 0xffffu, (signed char)(ow & 0xffu) == k);
            px[3] = pack_px(w0.y >> 16, w1.x & 0xffffu, w1.x >> 16, (signed char)((ow >> 8) & 0xffu) == k);
            px[4] = pack_px(w1.y & 0xffffu, w1.y >> 16, w2.x & 0xffffu, (signed char)((ow >> 16) & 0xffu) == k);
            px[5] = pack_px(w2.x >> 16, w2.y & 0xffffu, w2.y >> 16, (signed char)(ow >> 24) == k);
            px[0] = shfl_px(px[4], 1, true);
            px[1] = shfl_px(px[5], 1, true);
            px[6] = shfl_px(px[2], 1, false);
            if (lane == 0)
            {
                px[0] = load_px(img, own, p0 - 2, k);
                px[1] = load_px(img, own, p0 - 1, k);
            }
            if (lane == 31) px[6] = load_px(img, own, p0 + 4, k);
        }
        else
        {
#pragma unroll
            for (int c = 0; c < 7; ++c)
                px[c] = load_px(img, own, rowp + min(max(2 * X - 2 + c, 0), sw - 1), k);
        }
        int cv[7][4];
#pragma unroll
        for (int c = 0; c < 7; ++c) px_channels(px[c], cv[c]);
        int t[2][4];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int ch = 0; ch < 4; ++ch)
                t[c][ch] = cv[2 * c][ch] + 4 * cv[2 * c + 1][ch] + 6 * cv[2 * c + 2][ch] + 4 * cv[2 * c + 3][ch] +
                           cv[2 * c + 4][ch];
        if ((r & 1) == 0)
        {
            // even row 2m: last term of output m-2, middle of m-1, first of m
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int ch = 0; ch < 4; ++ch)
                {
                    P[c][ch] += t[c][ch];
                    Q[c][ch] += 6 * t[c][ch];
                    R[c][ch] = t[c][ch];
                }
            const int j = (r >> 1) - 2;
            const int Y = Y0 + j;
            if (j >= 0 && Y < dh)
            {
                const float s256 = 1.0f / 256.0f;
#pragma unroll
                for (int c = 0; c < 2; ++c)
                {
                    if (X + c >= dw) continue;
                    const size_t q = qrow + (size_t)Y * dw + X + c;
                    pyr_store(it.nd, it.wg, q,
                              make_float4(fmul((float)P[c][0], s256), fmul((float)P[c][1], s256),
                                          fmul((float)P[c][2], s256), fmul((float)(P[c][3] >> 16), s256)),
                              fmul((float)(P[c][3] & 0xffff), s256), a.half);
                }
            }
        }
        else
        {
            // odd row 2m+1: second term of output m, fourth of m-1; then rotate
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int ch = 0; ch < 4; ++ch)
                {
                    Q[c][ch] += 4 * t[c][ch];
                    R[c][ch] += 4 * t[c][ch];
                    P[c][ch] = Q[c][ch];
                    Q[c][ch] = R[c][ch];
                }
        }
    }
}

// One pixel of a blended band (the general path).
__device__ __noinline__ void blend_pixel(const TileDev& T, const ItemCache& C, int level, int K, long long pl, int half,
                                        int gmin)
{
    const int lw = T.lw[level];
    const bool top = level == T.bands - 1;
    const int uw = T.lw[level + 1], uh = T.lh[level + 1];
    const int y = (int)(pl / lw), x = (int)(pl - (long long)y * lw);
    UpCoef c;
    if (!top) c = up_coef_s(T.usx[level], T.usy[level], uw, uh, x, y);
    const size_t p = T.loff[level] + pl;
    float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f;
    for (int k = 0; k < K; ++k)
    {
        const int4 B = C.box[k];
        if (x < B.x || x > B.z || y < B.y || y > B.w) continue;  // weight 0: the term is +-0
        float wv = wg_at(C.wg[k], p, half);
        const bool store = g_stored(level, gmin) && (half || wv != 0.0f);
        if (wv == 0.0f && !store) continue;  // the term is +-0 and no reader needs G here
        float3 g = gauss_of(nd_at(C.nd[k], p, half));
        if (store) g_store(C.nd[k], p, g, half);
        if (wv == 0.0f) continue;
        if (!top)
        {
            const size_t up = T.loff[level + 1];
            float3 a00 = g_at(C.nd[k], up + (size_t)c.y0 * uw + c.x0, level + 1, gmin, half);
            float3 a10 = g_at(C.nd[k], up + (size_t)c.y0 * uw + c.x1, level + 1, gmin, half);
            float3 a01 = g_at(C.nd[k], up + (size_t)c.y1 * uw + c.x0, level + 1, gmin, half);
            float3 a11 = g_at(C.nd[k], up + (size_t)c.y1 * uw + c.x1, level + 1, gmin, half);
            g.x = fsub(g.x, up_mix(a00.x, a10.x, a01.x, a11.x, c.wx, c.wy));
            g.y = fsub(g.y, up_mix(a00.y, a10.y, a01.y, a11.y, c.wx, c.wy));
            g.z = fsub(g.z, up_mix(a00.z, a10.z, a01.z, a11.z, c.wx, c.wy));
        }
        acc0 = fadd(acc0, fmul(wv, g.x));
        acc1 = fadd(acc1, fmul(wv, g.y));
        acc2 = fadd(acc2, fmul(wv, g.z));
    }
    float* b = T.blend + p * 3;
    b[0] = acc0;
    b[1] = acc1;
    b[2] = acc2;
}

// Four consecutive pixels of a band below the top: for each contributor the
// Up(G_l+1) taps slide along in a two-column window (the level above is half
// as wide, so x0 advances by at most one column per pixel), each column's
// texels and reciprocals computed once per contributor; every pixel's sum
// still runs over the contributors in index order with its own weights.
__device__ __forceinline__ void blend_quad(const TileDev& T, const ItemCache& C, int level, int K, long long pl,
                                           int y, int x, int half, int gmin)
{
    const int uw = T.lw[level + 1], uh = T.lh[level + 1];
    int x0[4];
    float wx[4];
    UpCoef c = up_coef_s(T.usx[level], T.usy[level], uw, uh, x, y);
    const int y0 = c.y0, y1 = c.y1;
    const float wy = c.wy;
    x0[0] = c.x0;
    wx[0] = c.wx;
#pragma unroll
    for (int i = 1; i < 4; ++i)
    {
        const UpCoef ci = up_coef_s(T.usx[level], T.usy[level], uw, uh, x + i, y);
        x0[i] = ci.x0;
        wx[i] = ci.wx;
    }
    const size_t p = T.loff[level] + pl;
    float acc[4][3];
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i][0] = acc[i][1] = acc[i][2] = 0.0f;
    const bool storeAll = g_stored(level, gmin) && half;  // FP16: G stored wherever the blend passes
    for (int k = 0; k < K; ++k)
    {
        const int4 B = C.box[k];
        if (x + 3 < B.x || x > B.z || y < B.y || y > B.w) continue;  // weight 0 on the quad: terms are +-0
        float wv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) wv[i] = wg_at(C.wg[k], p + i, half);
        if (!storeAll && wv[0] == 0.0f && wv[1] == 0.0f && wv[2] == 0.0f && wv[3] == 0.0f) continue;
        const float4* nd = C.nd[k];
        const size_t up = T.loff[level + 1];
        int cur = x0[0];
        float3 L0 = g_at(nd, up + (size_t)y0 * uw + cur, level + 1, gmin, half),
               L1 = g_at(nd, up + (size_t)y1 * uw + cur, level + 1, gmin, half);
        int nx = min(cur + 1, uw - 1);
        float3 R0 = g_at(nd, up + (size_t)y0 * uw + nx, level + 1, gmin, half),
               R1 = g_at(nd, up + (size_t)y1 * uw + nx, level + 1, gmin, half);
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            if (x0[i] != cur)
            {
                cur = x0[i];
                L0 = R0;
                L1 = R1;
                nx = min(cur + 1, uw - 1);
                R0 = g_at(nd, up + (size_t)y0 * uw + nx, level + 1, gmin, half);
                R1 = g_at(nd, up + (size_t)y1 * uw + nx, level + 1, gmin, half);
            }
            if (wv[i] == 0.0f && !storeAll) continue;
            float3 g = gauss_of(nd_at(nd, p + i, half));
            if (g_stored(level, gmin)) g_store(nd, p + i, g, half);
            if (wv[i] == 0.0f) continue;
            g.x = fsub(g.x, up_mix(L0.x, R0.x, L1.x, R1.x, wx[i], wy));
            g.y = fsub(g.y, up_mix(L0.y, R0.y, L1.y, R1.y, wx[i], wy));
            g.z = fsub(g.z, up_mix(L0.z, R0.z, L1.z, R1.z, wx[i], wy));
            acc[i][0] = fadd(acc[i][0], fmul(wv[i], g.x));
            acc[i][1] = fadd(acc[i][1], fmul(wv[i], g.y));
            acc[i][2] = fadd(acc[i][2], fmul(wv[i], g.z));
        }
    }
    float* b = T.blend + p * 3;
    if ((reinterpret_cast<uintptr_t>(b) & 15) == 0)  // the quad's 48 bytes: three 16-byte stores
    {
        float4* b4 = reinterpret_cast<float4*>(b);
        b4[0] = make_float4(acc[0][0], acc[0][1], acc[0][2], acc[1][0]);
        b4[1] = make_float4(acc[1][1], acc[1][2], acc[2][0], acc[2][1]);
        b4[2] = make_float4(acc[2][2], acc[3][0], acc[3][1], acc[3][2]);
    }
    else
    {
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            b[3 * i] = acc[i][0];
            b[3 * i + 1] = acc[i][1];
            b[3 * i + 2] = acc[i][2];
        }
    }
}

// Blended band of one level: sum over the tile's contributors, in index
// order, of weight * Laplacian (SeamBlend.cpp:501-509), where
// Laplacian = G_l - Up(G_l+1) or G_top (SeamBlend.cpp:184-201).
// Where a contributor's weight is 0 its term is exactly +-0 (the hole-filled
// Gaussian is finite), and adding +-0 to a sum that started at +0 changes
// nothing, so skipping contributors outside their weight support (the whole
// pyramid of one that owns no pixel) equals the reference's full sum.
__global__ void __launch_bounds__(256, 3) k_blend_level(BlendArgs a, const Unit* __restrict__ units, int level)
{
    __shared__ ItemCache C;
    const Unit u = units[blockIdx.x];
    const TileDev& T = a.tiles[u.id];
    load_item_cache(C, a, T);
    level_boxes(C, a, T, level);
    const int K = T.numItems;
    const int lw = T.lw[level], lh = T.lh[level];
    const bool top = level == T.bands - 1;
    const int row0 = u.by * a.bandRows;
    const int rows = min(a.bandRows, lh - row0);
    const int qpr = (lw + 3) >> 2;
    const int nq = rows * qpr;
    for (int qi = threadIdx.x; qi < nq; qi += blockDim.x)
    {
        const int r = qi / qpr;
        const int y = row0 + r, x = (qi - r * qpr) * 4;
        const long long pl = (long long)y * lw + x;
        const int cnt = min(4, lw - x);
        if (!top && cnt == 4)
        {
            blend_quad(T, C, level, K, pl, y, x, a.half, a.gmin);
            continue;
        }
        for (int i = 0; i < cnt; ++i) blend_pixel(T, C, level, K, pl + i, a.half, a.gmin);
    }
}

// Collapse one level in place: recon_l = blended_l + Up(recon_l+1)
// (SeamBlend.cpp:514-525).
__global__ void __launch_bounds__(256) k_collapse(BlendArgs a, const Unit* __restrict__ units, int level)
{
    const Unit u = units[blockIdx.x];
    const TileDev& T = a.tiles[u.id];
    const int lw = T.lw[level], lh = T.lh[level];
    const int uw = T.lw[level + 1], uh = T.lh[level + 1];
    const float* r = T.blend + T.loff[level + 1] * 3;
    const long long base = (long long)u.by * a.bandRows * lw;
    const long long n = min((long long)a.bandRows * lw, (long long)lw * lh - base);
    for (long long q = threadIdx.x; q < n; q += blockDim.x)
    {
        const long long pl = base + q;
        const int y = (int)(pl / lw), x = (int)(pl - (long long)y * lw);
        UpCoef c = up_coef_s(T.usx[level], T.usy[level], uw, uh, x, y);
        float* b = T.blend + (T.loff[level] + pl) * 3;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
        {
            float v = up_mix(r[((size_t)c.y0 * uw + c.x0) * 3 + ch], r[((size_t)c.y0 * uw + c.x1) * 3 + ch],
                             r[((size_t)c.y1 * uw + c.x0) * 3 + ch], r[((size_t)c.y1 * uw + c.x1) * 3 + ch], c.wx,
                             c.wy);
            b[ch] = fadd(b[ch], v);
        }
    }
}

// Level 0 and output (SeamBlend.cpp:514-545).  The level-0 weight of a pixel
// is 1 for its owner and 0 for every other contributor, so the blended level-0
// band is exactly the owner's Laplacian img - Up(G1); the output is
// clamp(that + Up(recon_1)) + 0.5 truncated, and 0 where nobody owns.
__device__ __forceinline__ void final_store(unsigned short* o, const float* r)
{
#pragma unroll
    for (int ch = 0; ch < 3; ++ch)
    {
        float v = r[ch];
        v = v < 65535.0f ? v : 65535.0f;
        v = 0.0f < v ? v : 0.0f;
        o[ch] = (unsigned short)f2u_floor(fadd(v, 0.5f));  // v + 0.5 in [0.5, 65535.5]
    }
}

// One output pixel (the general path).
__device__ __noinline__ void final_pixel(const TileDev& T, const ItemCache& C, const float* rc, int uw, int uh,
                                            long long p, int own, int half, int gmin)
{
    unsigned short* o = T.out + p * 3;
    if (own < 0)
    {
        o[0] = o[1] = o[2] = 0;
        return;
    }
    const int W = T.w;
    const int y = (int)(p / W), x = (int)(p - (long long)y * W);
    const unsigned short* px = C.img[own] + p * 3;
    float r[3] = {u2f(__ldg(px)), u2f(__ldg(px + 1)), u2f(__ldg(px + 2))};
    if (T.bands > 1)
    {
        const UpCoef c = up_coef_s(T.usx[0], T.usy[0], uw, uh, x, y);
        const float4* nd = C.nd[own];
        const size_t l1 = T.loff[1];
        const float3 a00 = g_at(nd, l1 + (size_t)c.y0 * uw + c.x0, 1, gmin, half);
        const float3 a10 = g_at(nd, l1 + (size_t)c.y0 * uw + c.x1, 1, gmin, half);
        const float3 a01 = g_at(nd, l1 + (size_t)c.y1 * uw + c.x0, 1, gmin, half);
        const float3 a11 = g_at(nd, l1 + (size_t)c.y1 * uw + c.x1, 1, gmin, half);
        const float lap[3] = {fsub(r[0], up_mix(a00.x, a10.x, a01.x, a11.x, c.wx, c.wy)),
                              fsub(r[1], up_mix(a00.y, a10.y, a01.y, a11.y, c.wx, c.wy)),
                              fsub(r[2], up_mix(a00.z, a10.z, a01.z, a11.z, c.wx, c.wy))};
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
        {
            const float up = up_mix(__ldg(rc + ((size_t)c.y0 * uw + c.x0) * 3 + ch),
                                    __ldg(rc + ((size_t)c.y0 * uw + c.x1) * 3 + ch),
                                    __ldg(rc + ((size_t)c.y1 * uw + c.x0) * 3 + ch),
                                    __ldg(rc + ((size_t)c.y1 * uw + c.x1) * 3 + ch), c.wx, c.wy);
            r[ch] = fadd(lap[ch], up);
        }
    }
    final_store(o, r);
}

// A level-1 texel column (rows y0 and y1) of the owner's hole-filled Gaussian
// and of the level-1 reconstruction.
struct TapColumn
{
    float3 g0, g1, u0, u1;
};

__device__ __forceinline__ TapColumn tap_column(const float4* nd, size_t l1, const float* rc, int uw, int y0, int y1,
                                                int col, int half, int gmin)
{
    const size_t q0 = (size_t)y0 * uw + col, q1 = (size_t)y1 * uw + col;
    TapColumn t;
    t.g0 = g_at(nd, l1 + q0, 1, gmin, half);
    t.g1 = g_at(nd, l1 + q1, 1, gmin, half);
    t.u0 = make_float3(__ldg(rc + q0 * 3), __ldg(rc + q0 * 3 + 1), __ldg(rc + q0 * 3 + 2));
    t.u1 = make_float3(__ldg(rc + q1 * 3), __ldg(rc + q1 * 3 + 1), __ldg(rc + q1 * 3 + 2));
    return t;
}

// Four consecutive pixels of one row with one owner share their level-1
// taps.  Level 1 is half as wide (align-corners scale <= 0.5), so from one
// pixel to the next x0 advances by at most one column: a window of two
// columns (x0 and min(x0 + 1, w - 1), which is always x1) slides along, each
// column's texels and reciprocals computed once; every pixel still combines
// its own four taps with its own weights in the reference's order.
__device__ __forceinline__ void final_quad(const TileDev& T, const ItemCache& C, const float* rc, int uw, int uh,
                                           long long p, int y, int x, int own, int half, int gmin)
{
    const float4* g1 = C.nd[own];
    const size_t l1 = T.loff[1];
    const float sx = T.usx[0];
    UpCoef c = up_coef_s(sx, T.usy[0], uw, uh, x, y);
    int cur = c.x0;
    TapColumn L = tap_column(g1, l1, rc, uw, c.y0, c.y1, cur, half, gmin);
    TapColumn R = tap_column(g1, l1, rc, uw, c.y0, c.y1, c.x1, half, gmin);
    const unsigned short* px = C.img[own] + p * 3;
    // the quad's 12 source values: three 8-byte loads when aligned
    uint32_t pw[6];
    if ((reinterpret_cast<uintptr_t>(px) & 7) == 0)
    {
        const uint2* q = reinterpret_cast<const uint2*>(px);
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            const uint2 v = __ldg(q + k);
            pw[2 * k] = v.x;
            pw[2 * k + 1] = v.y;
        }
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 6; ++k) pw[k] = (uint32_t)__ldg(px + 2 * k) | ((uint32_t)__ldg(px + 2 * k + 1) << 16);
    }
    unsigned short* o = T.out + p * 3;
    unsigned short res[12];
    const float wy = c.wy;
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        float wx = c.wx;
        if (i > 0)
        {
            int x0;
            up_coef_x(sx, uw, x + i, x0, wx);
            if (x0 != cur)  // advanced by one column
            {
                cur = x0;
                L = R;
                R = tap_column(g1, l1, rc, uw, c.y0, c.y1, min(x0 + 1, uw - 1), half, gmin);
            }
        }
        float r[3];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
        {
            const int e = 3 * i + ch;  // value index in the quad
            r[ch] = u2f((pw[e >> 1] >> (16 * (e & 1))) & 0xffffu);
        }
        const float lap[3] = {fsub(r[0], up_mix(L.g0.x, R.g0.x, L.g1.x, R.g1.x, wx, wy)),
                              fsub(r[1], up_mix(L.g0.y, R.g0.y, L.g1.y, R.g1.y, wx, wy)),
                              fsub(r[2], up_mix(L.g0.z, R.g0.z, L.g1.z, R.g1.z, wx, wy))};
        r[0] = fadd(lap[0], up_mix(L.u0.x, R.u0.x, L.u1.x, R.u1.x, wx, wy));
        r[1] = fadd(lap[1], up_mix(L.u0.y, R.u0.y, L.u1.y, R.u1.y, wx, wy));
        r[2] = fadd(lap[2], up_mix(L.u0.z, R.u0.z, L.u1.z, R.u1.z, wx, wy));
        final_store(res + 3 * i, r);
    }
    // the quad's 24 bytes: three 8-byte stores when aligned
    if ((reinterpret_cast<uintptr_t>(o) & 7) == 0)
    {
        uint2* o2 = reinterpret_cast<uint2*>(o);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            o2[k] = make_uint2((uint32_t)res[4 * k] | ((uint32_t)res[4 * k + 1] << 16),
                               (uint32_t)res[4 * k + 2] | ((uint32_t)res[4 * k + 3] << 16));
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 12; ++k) o[k] = res[k];
    }
}

__global__ void __launch_bounds__(256) k_final0(BlendArgs a, const Unit* __restrict__ units)
{
    __shared__ ItemCache C;
    const Unit u = units[blockIdx.x];
    const TileDev& T = a.tiles[u.id];
    load_item_cache(C, a, T);
    const int W = T.w, H = T.h;
    const int uw = T.lw[1], uh = T.lh[1];
    const float* rc = T.blend + T.loff[1] * 3;
    const int row0 = u.by * a.bandRows;
    const int rows = min(a.bandRows, H - row0);
    const int qpr = (W + 3) >> 2;  // quads per row
    const int nq = rows * qpr;
    const signed char* owner = T.owner;
    // a quad's four owner bytes as one word: rows of a multiple of 4 pixels
    // on a 4-byte aligned map
    const bool ownWord = (W & 3) == 0 && (reinterpret_cast<uintptr_t>(owner) & 3) == 0;
    for (int qi = threadIdx.x; qi < nq; qi += blockDim.x)
    {
        const int y = row0 + qi / qpr;
        const int x = (qi - (qi / qpr) * qpr) * 4;
        const long long p = (long long)y * W + x;
        const int cnt = min(4, W - x);
        int own[4];
        if (ownWord)
        {
            const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(owner + p));
#pragma unroll
            for (int i = 0; i < 4; ++i) own[i] = (int)(signed char)(w >> (8 * i));
        }
        else
        {
#pragma unroll
            for (int i = 0; i < 4; ++i) own[i] = i < cnt ? (int)owner[p + i] : -2;
        }
        if (cnt == 4 && T.bands > 1 && own[0] >= 0 && own[1] == own[0] && own[2] == own[0] && own[3] == own[0])
        {
            final_quad(T, C, rc, uw, uh, p, y, x, own[0], a.half, a.gmin);
            continue;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i < cnt) final_pixel(T, C, rc, uw, uh, p + i, own[i], a.half, a.gmin);
    }
}

// ---------------------------------------------------------------------------
// Fused pyramid levels 0 and 1 (SeamBlend.cpp:125-201, 447-546).
//
// Level 1 of every contributor's pyramids (num, den and weight: 20 bytes per
// level-1 pixel per contributor) and of the tile's blended bands is never
// written to memory.  Two kernels replace the level-0 and level-1 steps of
// the materialised pyramid:
//
//  k_base2  per contributor and 32x8 block of level 2: stages the level-0
//           footprint in shared memory, computes the level-1 values of the
//           block's level-1 rectangle exactly in integers (as k_down0s), then
//           blurs and decimates them to level 2 in FP32 in the reference's
//           order (as k_down).  Writes level 2 only.
//  k_fine   per tile and 64x32 block of output pixels: for every contributor
//           owning a pixel of the block's level-0 footprint, in index order,
//           recomputes its level-1 values on the block's level-1 window from
//           the staged level-0 footprint, accumulates the blended level-1 band
//           (weight x (G1 - Up(G2))) and, for the pixels it owns, the level-0
//           Laplacian img - Up(G1); then collapses level 1 with Up(recon2)
//           read from the coarse levels and writes the output.
//
// Levels 2 and above stay materialised (a sixteenth of the pixels).  The
// values are the materialised pyramid's bit for bit: the level-1 values are
// the same exact integers / 256, every FP32 operation is the same in the same
// order, and a blended-band term is skipped only where its weight is exactly
// zero (the term is then +-0, and adding +-0 to the sum, which starts at +0
// and is never -0, changes nothing).  A contributor that owns no pixel of a
// block's footprint has weight zero on the whole level-1 window.
// ---------------------------------------------------------------------------
constexpr int kB2W = 32, kB2H = 8;                  // level-2 outputs per k_base2 CTA
constexpr int kB1W = 2 * kB2W + 3, kB1H = 2 * kB2H + 3;  // its level-1 rectangle (at most)
constexpr int kB0S = 2 * kB1W + 3 + 3;              // level-0 footprint row stride: at most 137 columns from
                                                    // a 4-pixel aligned start, 35 whole groups
constexpr int kB0H = 2 * kB1H + 3;                  // level-0 footprint rows (at most)
constexpr int kRun = 4;                             // k_base2's level-1 rows per streaming task

constexpr int kFW = 64, kFH = 32;                   // output pixels per k_fine CTA
constexpr int kFRun = 2;                            // k_fine's level-1 rows per streaming task (column pairs x
                                                    // 2 rows: ~150 tasks on a ~34 x 18 window)
constexpr int kF1W = 36, kF1H = 20;                 // its level-1 window (bound; checked)
constexpr int kF0S = 2 * kF1W + 8;                  // level-0 footprint row stride: the footprint's
                                                    // at most 78 columns rounded up to whole 4-pixel groups
constexpr int kF0H = 2 * kF1H + 3;                  // level-0 footprint rows
constexpr int kF2W = 22, kF2H = 14;                 // level-2 window (bound; checked)

// Stages contributor k's level-0 pixels of tile rows [ry0, ry1] x columns
// [cx0, cx1] as packed pixels (r | g << 16, b | cov << 16 | own << 17) at
// sm[(y - rowBase) * stride + (x - colBase)] (colBase a multiple of 4, at
// most cx0), in whole groups of four pixels from cx0 & ~3 (stride must hold
// them: a multiple of 4 at least cx1 - colBase + 1).  `own` is the owner map
// of the same rows: global, or shared with row stride ownStride and the same
// bases when ownSm is set.  A group is read as three 8-byte words when the
// image rows allow it.
__device__ __forceinline__ void stage_level0(const unsigned short* img, const signed char* own, int ownStride,
                                             bool ownSm, signed char k, int W, int ry0, int ry1, int cx0, int cx1,
                                             PackedPx* sm, int stride, int rowBase, int colBase)
{
    const int cs = cx0 & ~3;
    const int ng = ((cx1 - cs) >> 2) + 1;
    const int nr = ry1 - ry0 + 1;
    const bool fast = (W & 3) == 0 && (reinterpret_cast<uintptr_t>(img) & 7) == 0;
    // (row, group) pairs without a division: threads step through the groups
    // of a row and on to later rows
    int r = threadIdx.x / ng, g = threadIdx.x - r * ng;
    const int dr = blockDim.x / ng, dg = blockDim.x - dr * ng;
    for (; r < nr; r += dr, g += dg)
    {
        if (g >= ng)
        {
            g -= ng;
            ++r;
            if (r >= nr) break;
        }
        const int c = cs + 4 * g;
        const int y = ry0 + r;
        const size_t p = (size_t)y * W + c;
        PackedPx* d = sm + (y - rowBase) * stride + (c - colBase);
        signed char o[4];
#pragma unroll
        for (int e = 0; e < 4; ++e)
            o[e] = (c + e < W) ? (ownSm ? own[(y - rowBase) * ownStride + (c + e - colBase)] : __ldg(own + p + e))
                               : (signed char)-1;
        if (fast)
        {
            const uint2* w = reinterpret_cast<const uint2*>(img + p * 3);
            const uint2 w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2);
            d[0] = pack_px(w0.x & 0xffffu, w0.x >> 16, w0.y & 0xffffu, o[0] == k);
            d[1] = pack_px(w0.y >> 16, w1.x & 0xffffu, w1.x >> 16, o[1] == k);
            d[2] = pack_px(w1.y & 0xffffu, w1.y >> 16, w2.x & 0xffffu, o[2] == k);
            d[3] = pack_px(w2.x >> 16, w2.y & 0xffffu, w2.y >> 16, o[3] == k);
        }
        else
        {
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (c + e < W)
                {
                    const unsigned short* q = img + (p + e) * 3;
                    d[e] = pack_px(__ldg(q), __ldg(q + 1), __ldg(q + 2), o[e] == k);
                }
        }
    }
}

// Exact level-1 values (num r, g, b; den; weight) of level-1 columns X1 and
// X1 + 1 and rows Y1s .. Y1s + R - 1 from a staged footprint (tile rows from
// ry0, columns from cxa), handed to emit(col, m, nr, ng, nb, den, wg) in row
// order (col 0 for X1, 1 for X1 + 1, only when `two`).  Integer sums of the
// [1,4,6,4,1] x [1,4,6,4,1] stencil over clamped level-0 coordinates,
// streamed row by row (see k_down0s for why they are exact).  The two
// columns share three of their five taps: column X1 reads clamped columns
// 2 X1 - 2 .. 2 X1 + 2 and X1 + 1 reads 2 X1 .. 2 X1 + 4, which are taps 2..6
// of the same seven (clamping commutes with the shift).  Taps past cmax
// (beyond the staged columns: only a second column that is not emitted
// reaches them) read column cmax instead.
template <typename Emit>
__device__ __forceinline__ void level1_pair(const PackedPx* sm, int stride, int ry0, int cxa, int cmax, int W, int H,
                                            int X1, bool two, int Y1s, int R, Emit emit)
{
    int col[7];
#pragma unroll
    for (int i = 0; i < 7; ++i) col[i] = min(min(max(2 * X1 - 2 + i, 0), W - 1), cmax) - cxa;
    int P[2][4] = {}, Q[2][4] = {}, Rr[2][4] = {};
    const float s256 = 1.0f / 256.0f;
    for (int r = 0; r <= 2 * R + 2; ++r)
    {
        const int gy = min(max(2 * Y1s - 2 + r, 0), H - 1);
        const PackedPx* row = sm + (gy - ry0) * stride;
        int cv[7][4];
#pragma unroll
        for (int i = 0; i < 7; ++i) px_channels(row[col[i]], cv[i]);
        int t[2][4];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int ch = 0; ch < 4; ++ch)
                t[c][ch] = cv[2 * c][ch] + 4 * cv[2 * c + 1][ch] + 6 * cv[2 * c + 2][ch] + 4 * cv[2 * c + 3][ch] +
                           cv[2 * c + 4][ch];
        if ((r & 1) == 0)
        {
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int ch = 0; ch < 4; ++ch)
                {
                    P[c][ch] += t[c][ch];
                    Q[c][ch] += 6 * t[c][ch];
                    Rr[c][ch] = t[c][ch];
                }
            const int m = (r >> 1) - 2;
            if (m >= 0)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    if (c == 0 || two)
                        emit(c, m, fmul((float)P[c][0], s256), fmul((float)P[c][1], s256), fmul((float)P[c][2], s256),
                             fmul((float)(P[c][3] >> 16), s256), fmul((float)(P[c][3] & 0xffff), s256));
        }
        else
        {
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int ch = 0; ch < 4; ++ch)
                {
                    Q[c][ch] += 4 * t[c][ch];
                    Rr[c][ch] += 4 * t[c][ch];
                    P[c][ch] = Q[c][ch];
                    Q[c][ch] = Rr[c][ch];
                }
        }
    }
}

struct Base2Smem
{
    PackedPx px[kB0H * kB0S];          // level-0 footprint; later the horizontal level-2 pass
    float l1[5][kB1H][kB1W];           // level-1 rectangle: num r, g, b, den, weight
};

__global__ void __launch_bounds__(256) k_base2(BlendArgs a, const Unit* __restrict__ units)
{
    extern __shared__ __align__(16) unsigned char base2_raw[];
    Base2Smem& S = *reinterpret_cast<Base2Smem*>(base2_raw);
    float (*t)[kB1H][kB2W] = reinterpret_cast<float (*)[kB1H][kB2W]>(S.px);  // aliases the footprint
    const Unit u = units[blockIdx.x];
    const ItemDev& it = a.items[u.id];
    const TileDev& T = a.tiles[it.tile];
    const int W = T.w, H = T.h;
    const int lw1 = T.lw[1], lh1 = T.lh[1], lw2 = T.lw[2], lh2 = T.lh[2];
    const int X2a = u.bx * kB2W, Y2a = u.by * kB2H;
    const int X2b = min(X2a + kB2W - 1, lw2 - 1), Y2b = min(Y2a + kB2H - 1, lh2 - 1);
    const int X1lo = max(0, 2 * X2a - 2), X1hi = min(lw1 - 1, 2 * X2b + 2);
    const int Y1lo = max(0, 2 * Y2a - 2), Y1hi = min(lh1 - 1, 2 * Y2b + 2);
    const int cx0 = max(0, 2 * X1lo - 2), cx1 = min(W - 1, 2 * X1hi + 2);
    const int ry0 = max(0, 2 * Y1lo - 2), ry1 = min(H - 1, 2 * Y1hi + 2);
    const size_t q2 = T.loff[2];
    // A footprint that misses the covered box reads only uncovered pixels the
    // contributor does not own: its level-2 values are exactly zero.
    const int4 cb = covered_box(it.bbox);
    if (cb.x > cb.z || cx1 < cb.x || cx0 > cb.z || ry1 < cb.y || ry0 > cb.w)
    {
        for (int idx = threadIdx.x; idx < kB2W * kB2H; idx += blockDim.x)
        {
            const int X = X2a + (idx & (kB2W - 1)), Y = Y2a + idx / kB2W;
            if (X > X2b || Y > Y2b) continue;
            const size_t q = q2 + (size_t)Y * lw2 + X;
            pyr_store(it.nd, it.wg, q, make_float4(0.0f, 0.0f, 0.0f, 0.0f), 0.0f, a.half);
        }
        return;
    }
    const int cxa = cx0 & ~3;
    stage_level0(it.img, T.owner, 0, false, (signed char)it.k, W, ry0, ry1, cx0, cx1, S.px, kB0S, ry0, cxa);
    __syncthreads();
    // level-1 rectangle: a pair of columns and a run of kRun rows per task
    const int nX1 = X1hi - X1lo + 1, nY1 = Y1hi - Y1lo + 1;
    const int nPairs = (nX1 + 1) >> 1;
    const int nRuns = (nY1 + kRun - 1) / kRun;
    for (int task = threadIdx.x; task < nPairs * nRuns; task += blockDim.x)
    {
        const int run = task / nPairs, cx = 2 * (task - run * nPairs);
        const int Y1s = Y1lo + run * kRun;
        const int R = min(kRun, Y1hi - Y1s + 1);
        level1_pair(S.px, kB0S, ry0, cxa, cx1, W, H, X1lo + cx, cx + 1 < nX1, Y1s, R,
                    [&](int c, int m, float nr, float ng, float nb, float den, float wg) {
                        const int ry = Y1s + m - Y1lo;
                        S.l1[0][ry][cx + c] = nr;
                        S.l1[1][ry][cx + c] = ng;
                        S.l1[2][ry][cx + c] = nb;
                        S.l1[3][ry][cx + c] = den;
                        S.l1[4][ry][cx + c] = wg;
                    });
    }
    __syncthreads();
    // horizontal taps at the level-2 columns (over clamped level-1 columns)
    const int nX2 = X2b - X2a + 1, nY2 = Y2b - Y2a + 1;
    for (int idx = threadIdx.x; idx < 5 * nY1 * kB2W; idx += blockDim.x)
    {
        const int ch = idx / (nY1 * kB2W);
        const int rem = idx - ch * nY1 * kB2W;
        const int r = rem / kB2W, i = rem - r * kB2W;
        if (i >= nX2) continue;
        const int X2 = X2a + i;
        float v[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) v[q] = S.l1[ch][r][min(max(2 * X2 - 2 + q, 0), lw1 - 1) - X1lo];
        t[ch][r][i] = blur5(v[0], v[1], v[2], v[3], v[4]);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nX2 * nY2; idx += blockDim.x)
    {
        const int j = idx / nX2, i = idx - j * nX2;
        const int Y2 = Y2a + j;
        int rows[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) rows[q] = min(max(2 * Y2 - 2 + q, 0), lh1 - 1) - Y1lo;
        float o[5];
#pragma unroll
        for (int ch = 0; ch < 5; ++ch)
            o[ch] = blur5(t[ch][rows[0]][i], t[ch][rows[1]][i], t[ch][rows[2]][i], t[ch][rows[3]][i], t[ch][rows[4]][i]);
        const size_t q = q2 + (size_t)Y2 * lw2 + X2a + i;
        pyr_store(it.nd, it.wg, q, make_float4(o[0], o[1], o[2], o[3]), o[4], a.half);
    }
}

struct FineSmem
{
    float g1[3][kF1H][kF1W];                   // a contributor's G1 on the level-1 window; then recon1
    float w1[kF1H][kF1W];                      // its level-1 weight
    float g2[3][kF2H][kF2W];                   // its G2 on the level-2 window
    float r2[3][kF2H][kF2W];                   // recon2 on the level-2 window
    const unsigned short* img[kMaxTileItems];
    const float4* nd[kMaxTileItems];
    const float* wg[kMaxTileItems];
    uint32_t set[kMaxTileItems / 32];          // contributors owning a footprint pixel
    int ob[kMaxTileItems][4];                  // the footprint pixels each owns: x0, y0, x1, y1 (footprint-relative)
    // Up taps, tabulated: the align-corners coefficients are separable (the x
    // part depends on x only, the y part on y only), so the block's columns
    // and rows (level 0 -> 1) and the window's (level 1 -> 2) are computed
    // once: tap indices relative to the window, and the fraction.
    short2 tx0[kFW], ty0[kFH], tx1[kF1W], ty1[kF1H];
    float fx0[kFW], fy0[kFH], fx1[kF1W], fy1[kF1H];
    // Level 1 recomputed from level 0 only (the form with level 1 in memory
    // is launched without these):
    PackedPx px[kF0H * kF0S];                  // one contributor's level-0 footprint (the part it needs)
    signed char own[kF0H * kF0S];              // the tile's owner map over the footprint
};

// Per 64x32 block of output pixels (see the section comment).  Threads own
// pixels tid + 256 j (j < 8): lanes take consecutive columns of one row, so
// shared-memory reads of neighbouring pixels and the output stores are
// contiguous across a warp.  For each contributor owning a footprint pixel,
// in index order, its level-1 values on the window come either from memory
// (L1MEM: level 1 materialised by the level-0 step; G1 read where the weight
// is non-zero, the only places they are used) or are recomputed from level 0
// in shared memory: the footprint rows and columns within 6 of the pixels it
// owns are staged (a level-1 task reads at most 6 beyond its own pixels), and
// only the level-1 tasks (pairs of columns x kFRun rows) whose level-0
// footprint holds one of those pixels are computed - elsewhere its level-1
// weight is exactly zero, so its blended-band term is +-0 (skipped) and no
// pixel it owns takes a tap there (each Up tap of a level-0 pixel has that
// pixel in its 5-tap footprint).
template <bool L1MEM>
__global__ void __launch_bounds__(256) k_fine(BlendArgs a, const Unit* __restrict__ units)
{
    extern __shared__ __align__(16) unsigned char fine_raw[];
    FineSmem& S = *reinterpret_cast<FineSmem*>(fine_raw);
    const Unit u = units[blockIdx.x];
    const TileDev& T = a.tiles[u.id];
    const int W = T.w, H = T.h, K = min(T.numItems, kMaxTileItems);
    const int X0 = u.bx * kFW, Y0 = u.by * kFH;
    const int xe = min(X0 + kFW - 1, W - 1), ye = min(Y0 + kFH - 1, H - 1);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // this thread's outputs: column ox of rows oy0 + 4 j
    const int ox = X0 + (tid & (kFW - 1)), oy0 = Y0 + (tid >> 6);
    constexpr int kPx = kFW * kFH / 256;  // 8
    int own[kPx];
#pragma unroll
    for (int j = 0; j < kPx; ++j)
    {
        const int y = oy0 + 4 * j;
        own[j] = (ox <= xe && y <= ye) ? (int)__ldg(T.owner + (size_t)y * W + ox) : -2;
    }
    for (int k = tid; k < K; k += blockDim.x)
    {
        const ItemDev& it = a.items[T.firstItem + k];
        S.img[k] = it.img;
        S.nd[k] = it.nd;
        S.wg[k] = it.wg;
        S.ob[k][0] = S.ob[k][1] = 0x7fffffff;
        S.ob[k][2] = S.ob[k][3] = -1;
    }
    if (tid < kMaxTileItems / 32) S.set[tid] = 0u;
    __syncthreads();  // the set and boxes are cleared before any thread adds to them
    if (T.bands == 1)
    {
        // one band: the output is the owner's pixel (SeamBlend.cpp:527-545)
#pragma unroll
        for (int j = 0; j < kPx; ++j)
        {
            if (own[j] == -2) continue;
            const size_t q = (size_t)(oy0 + 4 * j) * W + ox;
            unsigned short* o = T.out + q * 3;
            if (own[j] < 0)
            {
                o[0] = o[1] = o[2] = 0;
                continue;
            }
            const unsigned short* p = S.img[own[j]] + q * 3;
            const float r[3] = {u2f(__ldg(p)), u2f(__ldg(p + 1)), u2f(__ldg(p + 2))};
            final_store(o, r);
        }
        return;
    }
    const int lw1 = T.lw[1], lh1 = T.lh[1];
    const bool top1 = T.bands == 2;
    // level-1 window: the Up taps of the block's first and last pixels
    // (monotonic in x and y)
    const UpCoef ca = up_coef_s(T.usx[0], T.usy[0], lw1, lh1, X0, Y0);
    const UpCoef cb = up_coef_s(T.usx[0], T.usy[0], lw1, lh1, xe, ye);
    const int A0 = ca.x0, A1 = cb.x1, B0 = ca.y0, B1 = cb.y1;
    const int nA = A1 - A0 + 1, nB = B1 - B0 + 1;
    const int cx0 = max(0, 2 * A0 - 2), cx1 = min(W - 1, 2 * A1 + 2);
    const int ry0 = max(0, 2 * B0 - 2), ry1 = min(H - 1, 2 * B1 + 2);
    const int cxa = cx0 & ~3;
    // level-2 window: the Up taps (level 2 -> 1) of the level-1 window's corners
    int P0 = 0, P1 = -1, Q0 = 0, Q1 = -1;
    const int lw2 = top1 ? 1 : T.lw[2], lh2 = top1 ? 1 : T.lh[2];
    if (!top1)
    {
        const UpCoef pa = up_coef_s(T.usx[1], T.usy[1], lw2, lh2, A0, B0);
        const UpCoef pb = up_coef_s(T.usx[1], T.usy[1], lw2, lh2, A1, B1);
        P0 = pa.x0;
        P1 = pb.x1;
        Q0 = pa.y0;
        Q1 = pb.y1;
    }
    const int nP = P1 - P0 + 1, nQ = Q1 - Q0 + 1;
    if (nA > kF1W || nB > kF1H || ry1 - ry0 + 1 > kF0H || ((cx1 - cxa + 4) & ~3) > kF0S || nP > kF2W || nQ > kF2H)
    {
        // outside the proven window bounds: report instead of overrunning
        if (tid == 0)
        {
            atomicExch(a.error, 1);
            atomicExch(a.error + 1, 1);
        }
        return;
    }
    // Up tap tables (see FineSmem); indices relative to the windows
    for (int i = tid; i < kFW + kFH + kF1W + kF1H; i += blockDim.x)
    {
        if (i < kFW)
        {
            const UpCoef q = up_coef_s(T.usx[0], T.usy[0], lw1, lh1, min(X0 + i, xe), Y0);
            S.tx0[i] = make_short2((short)(q.x0 - A0), (short)(q.x1 - A0));
            S.fx0[i] = q.wx;
        }
        else if (i < kFW + kFH)
        {
            const int j = i - kFW;
            const UpCoef q = up_coef_s(T.usx[0], T.usy[0], lw1, lh1, X0, min(Y0 + j, ye));
            S.ty0[j] = make_short2((short)(q.y0 - B0), (short)(q.y1 - B0));
            S.fy0[j] = q.wy;
        }
        else if (!top1 && i < kFW + kFH + kF1W)
        {
            const int c = i - kFW - kFH;
            const UpCoef q = up_coef_s(T.usx[1], T.usy[1], lw2, lh2, min(A0 + c, A1), B0);
            S.tx1[c] = make_short2((short)(q.x0 - P0), (short)(q.x1 - P0));
            S.fx1[c] = q.wx;
        }
        else if (!top1)
        {
            const int r = i - kFW - kFH - kF1W;
            const UpCoef q = up_coef_s(T.usx[1], T.usy[1], lw2, lh2, A0, min(B0 + r, B1));
            S.ty1[r] = make_short2((short)(q.y0 - Q0), (short)(q.y1 - Q0));
            S.fy1[r] = q.wy;
        }
    }
    // owner map over the footprint (a warp per row): the contributors it
    // names and, for the recomputing form, the box of the pixels each owns
    // (lanes grouped by owner, one atomic update per group)
    const int nr = ry1 - ry0 + 1, ncol = cx1 - cxa + 1;
    for (int r = warp; r < nr; r += 8)
    {
        for (int c0 = 0; c0 < ncol; c0 += 32)
        {
            const int c = c0 + lane;
            const int x = cxa + c;
            int o = -1;
            if (c < ncol && x < W) o = (int)__ldg(T.owner + (size_t)(ry0 + r) * W + x);
            if (!L1MEM && c < ncol) S.own[r * kF0S + c] = (signed char)o;
            const bool named = x >= cx0 && o >= 0 && o < K;
            if (named) atomicOr(&S.set[o >> 5], 1u << (o & 31));
            if (!L1MEM)
            {
                const int key = (o >= 0 && o < K && c < ncol) ? o : -1;
                const unsigned grp = __match_any_sync(kFull, key);
                const int cmin = __reduce_min_sync(grp, c), cmax = __reduce_max_sync(grp, c);
                if (key >= 0 && lane == __ffs(grp) - 1)
                {
                    atomicMin(&S.ob[key][0], cmin);
                    atomicMax(&S.ob[key][2], cmax);
                    atomicMin(&S.ob[key][1], r);
                    atomicMax(&S.ob[key][3], r);
                }
            }
        }
    }
    // recon2 on the level-2 window
    if (!top1)
    {
        const float* rc2 = T.blend + T.loff[2] * 3;
        for (int idx = tid; idx < nP * nQ; idx += blockDim.x)
        {
            const int r = idx / nP, c = idx - r * nP;
            const float* src = rc2 + ((size_t)(Q0 + r) * lw2 + P0 + c) * 3;
            S.r2[0][r][c] = __ldg(src);
            S.r2[1][r][c] = __ldg(src + 1);
            S.r2[2][r][c] = __ldg(src + 2);
        }
    }
    __syncthreads();
    // this thread's level-1 window pixels: tid, tid + 256, tid + 512
    float acc[3][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) acc[j][0] = acc[j][1] = acc[j][2] = 0.0f;
    float lap[kPx][3];
#pragma unroll
    for (int j = 0; j < kPx; ++j) lap[j][0] = lap[j][1] = lap[j][2] = 0.0f;
    const int nWin = nA * nB;
    const int nPairs = (nA + 1) >> 1;
    const int nRuns = (nB + kFRun - 1) / kFRun;
    const short2 xt0 = S.tx0[tid & (kFW - 1)];
    const float wx0 = S.fx0[tid & (kFW - 1)];
    for (int w = 0; w < kMaxTileItems / 32; ++w)
    {
        uint32_t m = S.set[w];
        while (m)
        {
            const int k = 32 * w + __ffs(m) - 1;
            m &= m - 1;
            if (!top1)
            {
                const size_t g2 = T.loff[2];
                for (int idx = tid; idx < nP * nQ; idx += blockDim.x)
                {
                    const int r = idx / nP, c = idx - r * nP;
                    const float3 g = g_at(S.nd[k], g2 + (size_t)(Q0 + r) * lw2 + P0 + c, 2, a.gmin, a.half);
                    S.g2[0][r][c] = g.x;
                    S.g2[1][r][c] = g.y;
                    S.g2[2][r][c] = g.z;
                }
            }
            if (L1MEM)
            {
                // level 1 from memory: the weight everywhere on the window,
                // G1 where the weight is non-zero (where it is used)
                const size_t l1 = T.loff[1];
#pragma unroll
                for (int j = 0; j < 3; ++j)
                {
                    const int p = tid + 256 * j;
                    if (p >= nWin) continue;
                    const int r = p / nA, c = p - r * nA;
                    const size_t q = l1 + (size_t)(B0 + r) * lw1 + A0 + c;
                    const float wv = wg_at(S.wg[k], q, a.half);
                    S.w1[r][c] = wv;
                    if (wv != 0.0f)
                    {
                        const float3 g = gauss_of(nd_at(S.nd[k], q, a.half));
                        S.g1[0][r][c] = g.x;
                        S.g1[1][r][c] = g.y;
                        S.g1[2][r][c] = g.z;
                    }
                }
                __syncthreads();
            }
            else
            {
                const int ob0 = S.ob[k][0], ob1 = S.ob[k][1], ob2 = S.ob[k][2], ob3 = S.ob[k][3];
                // stage the footprint within 6 of the owned box
                const int sy0 = max(ry0, ry0 + ob1 - 6), sy1 = min(ry1, ry0 + ob3 + 6);
                const int sx0 = max(cx0, cxa + ob0 - 6), sx1 = min(cx1, cxa + ob2 + 6);
                stage_level0(S.img[k], S.own, kF0S, true, (signed char)k, W, sy0, sy1, sx0, sx1, S.px, kF0S, ry0,
                             cxa);
                __syncthreads();
                // level-1 values of contributor k on the window: the tasks whose
                // level-0 footprint meets the owned box; zero weight elsewhere
                for (int task = tid; task < nPairs * nRuns; task += blockDim.x)
                {
                    const int run = task / nPairs, c = 2 * (task - run * nPairs);
                    const int Y1s = B0 + run * kFRun;
                    const int R = min(kFRun, B1 - Y1s + 1);
                    const bool two = c + 1 < nA;
                    const int X1 = A0 + c;
                    const int fr0 = max(2 * Y1s - 2, 0) - ry0, fr1 = min(2 * (Y1s + R - 1) + 2, H - 1) - ry0;
                    const int fc0 = max(2 * X1 - 2, 0) - cxa, fc1 = min(2 * (X1 + (two ? 1 : 0)) + 2, W - 1) - cxa;
                    if (fr1 < ob1 || fr0 > ob3 || fc1 < ob0 || fc0 > ob2)
                    {
                        for (int rr = 0; rr < R; ++rr)
                        {
                            S.w1[Y1s + rr - B0][c] = 0.0f;
                            if (two) S.w1[Y1s + rr - B0][c + 1] = 0.0f;
                        }
                        continue;
                    }
                    level1_pair(S.px, kF0S, ry0, cxa, cx1, W, H, X1, two, Y1s, R,
                                [&](int cc, int mm, float n0, float n1, float n2, float den, float wg) {
                                    const int r = Y1s + mm - B0;
                                    const float3 g = gauss_of(make_float4(n0, n1, n2, den));
                                    S.g1[0][r][c + cc] = g.x;
                                    S.g1[1][r][c + cc] = g.y;
                                    S.g1[2][r][c + cc] = g.z;
                                    S.w1[r][c + cc] = wg;
                                });
                }
                __syncthreads();
            }
            // blended level-1 band: weight x Laplacian, in contributor order
#pragma unroll
            for (int j = 0; j < 3; ++j)
            {
                const int p = tid + 256 * j;
                if (p >= nWin) continue;
                const int r = p / nA, c = p - r * nA;
                const float wv = S.w1[r][c];
                if (wv == 0.0f) continue;  // the term is +-0
                float g[3] = {S.g1[0][r][c], S.g1[1][r][c], S.g1[2][r][c]};
                if (!top1)
                {
                    const short2 xt = S.tx1[c], yt = S.ty1[r];
                    const float wx = S.fx1[c], wy = S.fy1[r];
#pragma unroll
                    for (int ch = 0; ch < 3; ++ch)
                        g[ch] = fsub(g[ch], up_mix(S.g2[ch][yt.x][xt.x], S.g2[ch][yt.x][xt.y], S.g2[ch][yt.y][xt.x],
                                                   S.g2[ch][yt.y][xt.y], wx, wy));
                }
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) acc[j][ch] = fadd(acc[j][ch], fmul(wv, g[ch]));
            }
            // level-0 Laplacian of the pixels k owns: img - Up(G1)
#pragma unroll
            for (int j = 0; j < kPx; ++j)
            {
                if (own[j] != k) continue;
                const int y = oy0 + 4 * j;
                const short2 yt = S.ty0[y - Y0];
                const float wy = S.fy0[y - Y0];
                float v[3];
                if (L1MEM)
                {
                    const unsigned short* q = S.img[k] + ((size_t)y * W + ox) * 3;
                    v[0] = u2f(__ldg(q));
                    v[1] = u2f(__ldg(q + 1));
                    v[2] = u2f(__ldg(q + 2));
                }
                else
                {
                    int cv[4];
                    px_channels(S.px[(y - ry0) * kF0S + (ox - cxa)], cv);
                    v[0] = u2f((uint32_t)cv[0]);
                    v[1] = u2f((uint32_t)cv[1]);
                    v[2] = u2f((uint32_t)cv[2]);
                }
#pragma unroll
                for (int ch = 0; ch < 3; ++ch)
                    lap[j][ch] = fsub(v[ch], up_mix(S.g1[ch][yt.x][xt0.x], S.g1[ch][yt.x][xt0.y], S.g1[ch][yt.y][xt0.x],
                                                    S.g1[ch][yt.y][xt0.y], wx0, wy));
            }
            __syncthreads();
        }
    }
    // recon1 = blended1 + Up(recon2) on the window (in g1's place)
#pragma unroll
    for (int j = 0; j < 3; ++j)
    {
        const int p = tid + 256 * j;
        if (p >= nWin) continue;
        const int r = p / nA, c = p - r * nA;
        float v[3] = {acc[j][0], acc[j][1], acc[j][2]};
        if (!top1)
        {
            const short2 xt = S.tx1[c], yt = S.ty1[r];
            const float wx = S.fx1[c], wy = S.fy1[r];
#pragma unroll
            for (int ch = 0; ch < 3; ++ch)
                v[ch] = fadd(v[ch], up_mix(S.r2[ch][yt.x][xt.x], S.r2[ch][yt.x][xt.y], S.r2[ch][yt.y][xt.x],
                                           S.r2[ch][yt.y][xt.y], wx, wy));
        }
        S.g1[0][r][c] = v[0];
        S.g1[1][r][c] = v[1];
        S.g1[2][r][c] = v[2];
    }
    __syncthreads();
    // output: clamp(lap0 + Up(recon1)) + 0.5, zero where nobody owns
#pragma unroll
    for (int j = 0; j < kPx; ++j)
    {
        if (own[j] == -2) continue;
        const int y = oy0 + 4 * j;
        unsigned short res[3] = {0, 0, 0};
        if (own[j] >= 0)
        {
            const short2 yt = S.ty0[y - Y0];
            const float wy = S.fy0[y - Y0];
            float r[3];
#pragma unroll
            for (int ch = 0; ch < 3; ++ch)
                r[ch] = fadd(lap[j][ch], up_mix(S.g1[ch][yt.x][xt0.x], S.g1[ch][yt.x][xt0.y], S.g1[ch][yt.y][xt0.x],
                                                S.g1[ch][yt.y][xt0.y], wx0, wy));
            final_store(res, r);
        }
        unsigned short* o = T.out + ((size_t)y * W + ox) * 3;
        o[0] = res[0];
        o[1] = res[1];
        o[2] = res[2];
    }
}
}  // namespace

// Shared-memory bytes of the per-row-group progress counters.
size_t dt_prog_bytes(int maxH) { return (size_t)(((maxH + 31) >> 5) + 1) * sizeof(int); }

int dt_rows_in_flight(int maxW, int maxH)
{
    const size_t row = (size_t)dt_ring_stride(maxW) * sizeof(float);
    const size_t fixed = dt_prog_bytes(maxH) + kDtStageBytes;
    auto fit = [&](size_t budget) { return budget > fixed ? (int)((budget - fixed) / row) : 0; };
    int n = fit(110 * 1024);  // two CTAs per SM
    if (n < 2) n = fit(220 * 1024);
    return n > kDtRing ? kDtRing : n;
}

int launch_coverage(const BlendArgs& a, const Unit* units, int n, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    k_coverage<<<n, 256, 0, s>>>(a, units);
    return check_launch("coverage kernel");
}

int launch_warp_tiles(const BlendArgs& a, const Unit* units, int n, int shape, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    if (shape == 1)
    {
        const int smem = (int)sizeof(WarpSmem);
        cudaFuncSetAttribute(k_warp_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        k_warp_tiles<<<n, 256, smem, s>>>(a, units);
    }
    else k_warp_rows<<<n, 256, 0, s>>>(a, units);
    return check_launch("tile warp kernel");
}

int launch_dt(const BlendArgs& a, const int* itemList, int n, bool backward, int maxW, int maxH, int slotsWanted,
              cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    int slots = dt_rows_in_flight(maxW, maxH);
    if (slotsWanted >= 2 && slotsWanted < slots) slots = slotsWanted;
    if (slots < 2)
        return fail(I360B_NOT_SUPPORTED, "Chunk %dx%d exceeds the distance-transform row ring.", maxW, maxH);
    size_t smem = kDtStageBytes + (size_t)slots * dt_ring_stride(maxW) * sizeof(float) + dt_prog_bytes(maxH);
    if (backward)
    {
        cudaFuncSetAttribute(k_dt<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_dt<true><<<n, 32 * kDtWarps, smem, s>>>(a, itemList, slots);
    }
    else
    {
        cudaFuncSetAttribute(k_dt<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_dt<false><<<n, 32 * kDtWarps, smem, s>>>(a, itemList, slots);
    }
    return check_launch("distance transform kernel");
}

int launch_owner(const BlendArgs& a, const Unit* units, int n, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    k_owner<<<n, 256, 0, s>>>(a, units);
    return check_launch("ownership kernel");
}

int launch_seam(const BlendArgs& a, const int* tileList, int n, int maxLines, cudaStream_t s);

int launch_seam(const BlendArgs& a, const int* tileList, int n, cudaStream_t s)
{
    // Per-line state (lo, hi, prev: 3 ints; back pointers: kSeamBand bytes)
    // is kept in shared memory for lines up to this count.
    const int smemLines = 3072;
    size_t smem = (size_t)smemLines * (4 * sizeof(int) + kSeamBand);
    if (n <= 0) return I360B_SUCCESS;
    cudaFuncSetAttribute(k_seam, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_seam<<<n, kSeamThreads, smem, s>>>(a, tileList, smemLines);
    return check_launch("seam kernel");
}

int launch_down(const BlendArgs& a, const Unit* units, int n, int level, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    const int smem = (10 * kDnSH * (kDnSW / 2) + 5 * kDnSH * kDnTW) * (int)sizeof(float);
    if (level == 0)
    {
        k_down0s<<<(n + kDnWarps - 1) / kDnWarps, 32 * kDnWarps, 0, s>>>(a, units, n);
    }
    else
    {
        cudaFuncSetAttribute(k_down, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        k_down<<<n, 256, smem, s>>>(a, units, level);
    }
    return check_launch("pyramid down kernel");
}

int launch_blend_level(const BlendArgs& a, const Unit* units, int n, int level, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    k_blend_level<<<n, 256, 0, s>>>(a, units, level);
    return check_launch("blend level kernel");
}

int launch_collapse(const BlendArgs& a, const Unit* units, int n, int level, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    k_collapse<<<n, 256, 0, s>>>(a, units, level);
    return check_launch("collapse kernel");
}

int launch_final0(const BlendArgs& a, const Unit* units, int n, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    k_final0<<<n, 256, 0, s>>>(a, units);
    return check_launch("final level kernel");
}

int launch_base2(const BlendArgs& a, const Unit* units, int n, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    const int smem = (int)sizeof(Base2Smem);
    cudaFuncSetAttribute(k_base2, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_base2<<<n, 256, smem, s>>>(a, units);
    return check_launch("pyramid base kernel");
}

int launch_fine(const BlendArgs& a, const Unit* units, int n, bool level1InMemory, cudaStream_t s)
{
    if (n <= 0) return I360B_SUCCESS;
    if (level1InMemory)
    {
        // the level-0 staging arrays (the struct's tail) are not used
        const int smem = (int)offsetof(FineSmem, px);
        cudaFuncSetAttribute(k_fine<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        k_fine<true><<<n, 256, smem, s>>>(a, units);
    }
    else
    {
        const int smem = (int)sizeof(FineSmem);
        cudaFuncSetAttribute(k_fine<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        k_fine<false><<<n, 256, smem, s>>>(a, units);
    }
    return check_launch("fine levels kernel");
}
}  // namespace i360b
