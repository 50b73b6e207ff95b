// Per-pixel render-path kernels: fused Bayer demosaic, backward homography
// warp (+ gain), sigma-clipped median stack and gain.  Each reproduces the
// reference CPU backend's arithmetic bit for bit (FP32, no FMA contraction,
// truncation at the same points) so outputs match Kernels::Scalar::* exactly.
#include "common.cuh"

namespace i360b
{
// ---------------------------------------------------------------------------
// Demosaic: BlackLevelSubtract -> WhiteBalance -> bilinear 3x3 -> 3x4 matrix,
// one pass (BayerDemosaic_Scalar.cpp:9-50, BayerDemosaicKernels.h:10-75).
// A CTA stages its (TH+2) x (TW+2) CFA footprint in shared memory with the
// black level and white balance already applied, then each thread demosaics
// and colour-corrects 2x2 output pixels.
// ---------------------------------------------------------------------------
namespace
{
constexpr int kDmTW = 64, kDmTH = 16;

struct DemosaicParams
{
    float camMul[4];
    float rgbCam[12];
    uint32_t filters;
    unsigned short black;
    // Standard Bayer layout (2x2-periodic, one R, one B, G on a diagonal):
    // colour of site (y & 1, x & 1), else std2x2 = 0 and only the generic
    // path runs.
    int std2x2;
    int color2x2[4];
};

__device__ __forceinline__ int bayer_color(int row, int col, uint32_t filters)
{
    // BayerDemosaicKernels.h:10-13.
    return (int)((filters >> ((((row << 1) & 14) | (col & 1)) << 1)) & 3u);
}

// 3x3 same-colour average of DemosaicPixel (BayerDemosaicKernels.h:25-60) for
// any filter word and any position (borders average fewer neighbours).
__device__ __forceinline__ void demosaic_generic(const float (*s)[kDmTW + 2], int lx, int ly, int x, int y,
                                                 int w, int h, uint32_t filters, float rgb[3])
{
    float acc[3] = {0.0f, 0.0f, 0.0f};
    int cnt[3] = {0, 0, 0};
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx)
        {
            int nx = x + dx, ny = y + dy;
            if (nx < 0 || ny < 0 || nx >= w || ny >= h) continue;
            int ch = bayer_color(ny, nx, filters);
            int slot = ch == 3 ? 1 : ch;
            float v = s[ly + 1 + dy][lx + 1 + dx];
            // Integer-valued sums below 2^24: exact in any order.
            if (slot == 0) { acc[0] += v; cnt[0]++; }
            else if (slot == 1) { acc[1] += v; cnt[1]++; }
            else { acc[2] += v; cnt[2]++; }
        }
    int mine = bayer_color(y, x, filters);
    int my = mine == 3 ? 1 : mine;
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        float v = acc[c];
        if (c == my) v = s[ly + 1][lx + 1];
        else if (cnt[c] != 0) v = fdiv(v, u2f((uint32_t)cnt[c]));
        rgb[c] = v;
    }
}

__global__ void __launch_bounds__(256) k_demosaic(const unsigned short* __restrict__ cfa, int w, int h,
                                                  DemosaicParams P, unsigned short* __restrict__ out)
{
    __shared__ float s[kDmTH + 2][kDmTW + 2];
    const int tx0 = blockIdx.x * kDmTW, ty0 = blockIdx.y * kDmTH;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    // Black level and white balance of one CFA value (BayerDemosaicKernels.h
    // BLS/WB steps), as the float the interpolation reads.
    // The uint16 truncation and the float the interpolation reads in one step
    // (clamp_floor_u16f); `mul` is the multiplier of the value's colour.
    auto level_m = [&](unsigned raw, float mul) {
        raw = raw > P.black ? raw - P.black : 0u;
        return clamp_floor_u16f(fmul(u2f(raw), mul));
    };
    auto level = [&](unsigned short raw, int gy, int gx) {
        return level_m(raw, P.camMul[bayer_color(gy, gx, P.filters)]);
    };
    if ((w & 3) == 0 && (reinterpret_cast<uintptr_t>(cfa) & 7) == 0 && tx0 >= 4 && tx0 + kDmTW + 4 <= w)
    {
        // Interior column of tiles on 8-byte aligned rows: the footprint
        // (columns tx0-1 .. tx0+64) read as 8-byte words of four values,
        // columns tx0-4 .. tx0+67.
        constexpr int kWords = kDmTW / 4 + 2;
        for (int i = tid; i < (kDmTH + 2) * kWords; i += 256)
        {
            const int r = i / kWords, wi = i - r * kWords;
            const int gy = ty0 - 1 + r, gx0 = tx0 - 4 + 4 * wi;
            float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (gy >= 0 && gy < h)
            {
                // gx0 is even: the four values alternate between two colours
                // (a site's colour depends on its column only through x & 1)
                const float me = P.camMul[bayer_color(gy, gx0, P.filters)];
                const float mo = P.camMul[bayer_color(gy, gx0 + 1, P.filters)];
                const uint2 q = __ldg(reinterpret_cast<const uint2*>(cfa + (size_t)gy * w + gx0));
                v[0] = level_m(q.x & 0xffffu, me);
                v[1] = level_m(q.x >> 16, mo);
                v[2] = level_m(q.y & 0xffffu, me);
                v[3] = level_m(q.y >> 16, mo);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                const int c = gx0 + k - (tx0 - 1);
                if (c >= 0 && c < kDmTW + 2) s[r][c] = v[k];
            }
        }
    }
    else
    {
        for (int i = tid; i < (kDmTH + 2) * (kDmTW + 2); i += 256)
        {
            int r = i / (kDmTW + 2), c = i % (kDmTW + 2);
            int gx = tx0 - 1 + c, gy = ty0 - 1 + r;
            float v = 0.0f;
            if (gx >= 0 && gy >= 0 && gx < w && gy < h) v = level(__ldg(cfa + (size_t)gy * w + gx), gy, gx);
            s[r][c] = v;
        }
    }
    __syncthreads();
    const bool evenW = (w & 1) == 0;
    // Every pixel of the block is an interior pixel (1 <= x <= w-2, 1 <= y <= h-2).
    const bool blockInterior = tx0 >= 1 && ty0 >= 1 && tx0 + kDmTW <= w - 1 && ty0 + kDmTH <= h - 1;
    // The quad's 4x4 neighbourhood, read once.
    float nb[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) nb[r][c] = s[threadIdx.y * 2 + r][threadIdx.x * 2 + c];
#pragma unroll
    for (int oy = 0; oy < 2; ++oy)
    {
        unsigned short px[2][3];
        const int ly = threadIdx.y * 2 + oy, y = ty0 + ly;
#pragma unroll
        for (int ox = 0; ox < 2; ++ox)
        {
            const int lx = threadIdx.x * 2 + ox, x = tx0 + lx;
            float R = 0.0f, G = 0.0f, B = 0.0f;
            if (P.std2x2 && (blockInterior || (x >= 1 && y >= 1 && x < w - 1 && y < h - 1)))
            {
                // Interior of a standard Bayer layout: the same-colour
                // neighbours are the cross (4), the diagonals (4), or a
                // horizontal / vertical pair (2 each); dividing by 4 or 2 is
                // exact, so these are the reference's averages bit for bit.
                // quad-local neighbourhood: centre at nb[oy + 1][ox + 1]
                const float c = nb[oy + 1][ox + 1];
                const float n = nb[oy][ox + 1], so = nb[oy + 2][ox + 1];
                const float we = nb[oy + 1][ox], ea = nb[oy + 1][ox + 2];
                // tx0, ty0 and the quad's corner are even: y & 1 = oy, x & 1 = ox
                const int cls = P.color2x2[(oy << 1) | ox];
                if (cls != 1)
                {
                    const float cross = ((n + we) + ea) + so;
                    const float diag = ((nb[oy][ox] + nb[oy][ox + 2]) + nb[oy + 2][ox]) + nb[oy + 2][ox + 2];
                    G = fmul(cross, 0.25f);
                    const float other = fmul(diag, 0.25f);
                    R = cls == 0 ? c : other;
                    B = cls == 0 ? other : c;
                }
                else
                {
                    const int hc = P.color2x2[(oy << 1) | (ox ^ 1)];  // colour of the left/right pair
                    const float hp = fmul(we + ea, 0.5f), vp = fmul(n + so, 0.5f);
                    G = c;
                    R = hc == 0 ? hp : vp;
                    B = hc == 0 ? vp : hp;
                }
            }
            else if (x < w && y < h)
            {
                float rgb[3];
                demosaic_generic(s, lx, ly, x, y, w, h, P.filters, rgb);
                R = rgb[0];
                G = rgb[1];
                B = rgb[2];
            }
            // Truncate to uint16 (DemosaicPixel), then the 3x4 colour matrix
            // (ApplyColorMatrixPixel, BayerDemosaicKernels.h:64-75).
            const float r = clamp_floor_u16f(R), g = clamp_floor_u16f(G), b = clamp_floor_u16f(B);
#pragma unroll
            for (int row = 0; row < 3; ++row)
            {
                float val = fadd(fadd(fadd(fmul(P.rgbCam[row * 4 + 0], r), fmul(P.rgbCam[row * 4 + 1], g)),
                                      fmul(P.rgbCam[row * 4 + 2], b)),
                                 P.rgbCam[row * 4 + 3]);
                px[ox][row] = clamp_trunc_u16(val);
            }
        }
        const int x0 = tx0 + threadIdx.x * 2;
        if (y >= h || x0 >= w) continue;
        unsigned short* o = out + ((size_t)y * w + x0) * 3;
        if (evenW && x0 + 1 < w)
        {
            // x0 even and w even: 12 bytes at a 4-byte-aligned address.
            uint32_t* o32 = reinterpret_cast<uint32_t*>(o);
            o32[0] = (uint32_t)px[0][0] | ((uint32_t)px[0][1] << 16);
            o32[1] = (uint32_t)px[0][2] | ((uint32_t)px[1][0] << 16);
            o32[2] = (uint32_t)px[1][1] | ((uint32_t)px[1][2] << 16);
        }
        else
        {
            o[0] = px[0][0];
            o[1] = px[0][1];
            o[2] = px[0][2];
            if (x0 + 1 < w)
            {
                o[3] = px[1][0];
                o[4] = px[1][1];
                o[5] = px[1][2];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Warp: backward bilinear homography warp (WarpPerspective_Scalar.cpp:8-45,
// WarpPerspectiveKernels.h:16-43), with RenderExecutor's ApplyGain fused.
// ---------------------------------------------------------------------------
struct WarpParams
{
    float H[9];
    float gain;
    int applyGain;
};

__device__ __forceinline__ void warp_pixel(const unsigned short* __restrict__ src, int sw, int sh, const WarpParams& P,
                                           float dX, float dY, unsigned short o[3])
{
    float sx = fadd(fadd(fmul(P.H[0], dX), fmul(P.H[1], dY)), P.H[2]);
    float sy = fadd(fadd(fmul(P.H[3], dX), fmul(P.H[4], dY)), P.H[5]);
    float sw1 = fadd(fadd(fmul(P.H[6], dX), fmul(P.H[7], dY)), P.H[8]);
    o[0] = o[1] = o[2] = 0;
    if (fabsf(sw1) < 1e-10f) return;
    sx = fdiv(sx, sw1);
    sy = fdiv(sy, sw1);
    // floor(s) >= 0 && floor(s) + 1 < size, stated on the float: NaN and
    // out-of-int-range positions are invalid, as the reference's int
    // conversion makes them.
    if (!(sx >= 0.0f && sx < (float)(sw - 1) && sy >= 0.0f && sy < (float)(sh - 1))) return;
    int x0 = (int)f2u_floor(sx), y0 = (int)f2u_floor(sy);  // 0 <= sx, sy < 2^23 here
    float fx = fsub(sx, u2f((uint32_t)x0)), fy = fsub(sy, u2f((uint32_t)y0));
    float gx = fsub(1.0f, fx), gy = fsub(1.0f, fy);
    float w00 = fmul(gx, gy), w10 = fmul(fx, gy), w01 = fmul(gx, fy), w11 = fmul(fx, fy);
    const unsigned short* r0 = src + ((size_t)y0 * sw + x0) * 3;
    const unsigned short* r1 = r0 + (size_t)sw * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        float v = fadd(fadd(fadd(fmul(w00, u2f(__ldg(r0 + c))), fmul(w10, u2f(__ldg(r0 + 3 + c)))),
                            fmul(w01, u2f(__ldg(r1 + c)))),
                       fmul(w11, u2f(__ldg(r1 + 3 + c))));
        o[c] = P.applyGain ? clamp_trunc_u16(fmul(clamp_floor_u16f(v), P.gain)) : clamp_trunc_u16(v);
    }
}

__global__ void __launch_bounds__(256) k_warp(const unsigned short* __restrict__ src, int sw, int sh,
                                              unsigned short* __restrict__ dst, int dw, int dh, int offX, int offY,
                                              WarpParams P)
{
    int x = blockIdx.x * 32 + threadIdx.x;
    int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= dw || y >= dh) return;
    unsigned short o[3];
    warp_pixel(src, sw, sh, P, (float)(x + offX), (float)(y + offY), o);
    unsigned short* d = dst + ((size_t)y * dw + x) * 3;
    d[0] = o[0];
    d[1] = o[1];
    d[2] = o[2];
}

// ---------------------------------------------------------------------------
// Median stack (MedianStackKernels.h:19-55, MedianStack_Scalar.cpp:8-24).
//
// Two output scalars per thread, packed as the low and high halves of one
// 32-bit word per input (one 4-byte load per input: a warp reads 128
// contiguous bytes of each input).  Per scalar the statistics are
// accumulated sequentially in input order in FP32 (sumSq exceeds 2^24, so
// the order is part of the result), exactly as the reference.  The sort is a
// bitonic network on the packed words with __vminu2/__vmaxu2, so one
// compare-exchange instruction pair sorts both scalars' stacks.  A clipped
// value, and every slot past the input count, becomes 0xFFFF: the maximum of
// the type, so the first keptCount sorted positions hold exactly the sorted
// kept values (ties with a kept 65535 do not change any value there), and
// the median is element keptCount/2 - the reference's values[count / 2].
// ---------------------------------------------------------------------------
struct MedianInputs
{
    const unsigned short* p[kMaxContributors];
};

template <int P>
__device__ __forceinline__ void bitonic_sort_u16x2(uint32_t (&v)[P])
{
#pragma unroll
    for (int k = 2; k <= P; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < P; ++i)
            {
                const int l = i ^ j;
                if (l > i)
                {
                    const uint32_t lo = __vminu2(v[i], v[l]), hi = __vmaxu2(v[i], v[l]);
                    const bool up = (i & k) == 0;
                    v[i] = up ? lo : hi;
                    v[l] = up ? hi : lo;
                }
            }
}

// Sigma bounds of one scalar's stack (MedianStackKernels.h:22-27).
__device__ __forceinline__ void clip_bounds(float sum, float sumSq, int n, float sigma, float& lo, float& hi)
{
    const float fn = (float)n;
    const float mean = fdiv(sum, fn);
    const float var = fsub(fdiv(sumSq, fn), fmul(mean, mean));
    const float sd = __fsqrt_rn(var < 0.0f ? 0.0f : var);
    lo = fsub(mean, fmul(sigma, sd));
    hi = fadd(mean, fmul(sigma, sd));
}

// The sigma-clipped median of both halves of v[0..n) (v[i] for i >= n must
// be 0xFFFFFFFF), packed the same way.  v is sorted in place.
template <int P>
__device__ __forceinline__ uint32_t median_pair(uint32_t (&v)[P], int n, float sigma)
{
    int cntL = n, cntH = n;
    if (n > 3)
    {
        float sL = 0.0f, qL = 0.0f, sH = 0.0f, qH = 0.0f;
#pragma unroll
        for (int i = 0; i < P; ++i)
            if (i < n)
            {
                const float a = u2f(v[i] & 0xffffu), b = u2f(v[i] >> 16);
                sL = fadd(sL, a);
                qL = fadd(qL, fmul(a, a));
                sH = fadd(sH, b);
                qH = fadd(qH, fmul(b, b));
            }
        float loL, hiL, loH, hiH;
        clip_bounds(sL, qL, n, sigma, loL, hiL);
        clip_bounds(sH, qH, n, sigma, loH, hiH);
        uint32_t outL = 0, outH = 0;  // bit i: value i is clipped
        int kL = 0, kH = 0;
#pragma unroll
        for (int i = 0; i < P; ++i)
            if (i < n)
            {
                const float a = u2f(v[i] & 0xffffu), b = u2f(v[i] >> 16);
                const bool keepA = a >= loL && a <= hiL, keepB = b >= loH && b <= hiH;
                kL += keepA ? 1 : 0;
                kH += keepB ? 1 : 0;
                outL |= keepA ? 0u : (1u << i);
                outH |= keepB ? 0u : (1u << i);
            }
        // if nothing is kept the reference keeps every value
        if (kL == 0) outL = 0;
        else cntL = kL;
        if (kH == 0) outH = 0;
        else cntH = kH;
#pragma unroll
        for (int i = 0; i < P; ++i)
        {
            if ((outL >> i) & 1u) v[i] |= 0x0000ffffu;
            if ((outH >> i) & 1u) v[i] |= 0xffff0000u;
        }
    }
    bitonic_sort_u16x2<P>(v);
    const int mL = cntL >> 1, mH = cntH >> 1;
    uint32_t rL = v[0], rH = v[0];
#pragma unroll
    for (int i = 1; i < P; ++i)
    {
        rL = (i == mL) ? v[i] : rL;
        rH = (i == mH) ? v[i] : rH;
    }
    return (rL & 0x0000ffffu) | (rH & 0xffff0000u);
}

// Packed path: scalars 2t and 2t+1 of every input (4-byte aligned inputs
// and output, even scalar count).
template <int P>
__global__ void __launch_bounds__(256) k_median2(MedianInputs in, int n, long long pairs, float sigma,
                                                 uint32_t* __restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= pairs) return;
    uint32_t v[P];
#pragma unroll
    for (int i = 0; i < P; ++i)
        v[i] = i < n ? __ldg(reinterpret_cast<const uint32_t*>(in.p[i]) + t) : 0xffffffffu;
    out[t] = median_pair<P>(v, n, sigma);
}

// General path (any alignment or odd count): one scalar per thread, in the
// low half of the packed words.
template <int P>
__global__ void __launch_bounds__(256) k_median1(MedianInputs in, int n, long long total, float sigma,
                                                 unsigned short* __restrict__ out)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    uint32_t v[P];
#pragma unroll
    for (int i = 0; i < P; ++i) v[i] = i < n ? ((uint32_t)__ldg(in.p[i] + idx) | 0xffff0000u) : 0xffffffffu;
    out[idx] = (unsigned short)(median_pair<P>(v, n, sigma) & 0xffffu);
}

// ---------------------------------------------------------------------------
// Warp + median stack fused: the median of n frames each warped onto the
// same destination grid (IComputeBackend::WarpPerspective of every frame,
// then MedianStack over the warped buffers: CpuComputeBackend.cpp:112-159).
// Each destination pixel's n samples are computed with the warp's exact FP32
// arithmetic and stacked in registers, so the warped frames are never
// written; a thread makes two horizontally adjacent pixels and stacks their
// channels as three packed pairs (r, g, b of pixel x in the low halves, of
// pixel x+1 in the high halves).
// ---------------------------------------------------------------------------
struct StackParams
{
    const unsigned short* src[kMaxContributors];
    float H[kMaxContributors][9];
};

template <int P>
__global__ void __launch_bounds__(256) k_warp_median(StackParams S, int n, int sw, int sh,
                                                     unsigned short* __restrict__ dst, int dw, int dh, int offX,
                                                     int offY, float sigma)
{
    const int x = (blockIdx.x * 32 + threadIdx.x) * 2;
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= dw || y >= dh) return;
    const bool two = x + 1 < dw;
    const float dX = (float)(x + offX), dY = (float)(y + offY);
    uint32_t r[P], g[P], b[P];
#pragma unroll
    for (int i = 0; i < P; ++i)
    {
        r[i] = g[i] = b[i] = 0xffffffffu;
        if (i < n)
        {
            WarpParams W;
#pragma unroll
            for (int q = 0; q < 9; ++q) W.H[q] = S.H[i][q];
            W.gain = 1.0f;
            W.applyGain = 0;
            unsigned short a[3], c[3] = {0, 0, 0};
            warp_pixel(S.src[i], sw, sh, W, dX, dY, a);
            if (two) warp_pixel(S.src[i], sw, sh, W, (float)(x + 1 + offX), dY, c);
            r[i] = (uint32_t)a[0] | ((uint32_t)c[0] << 16);
            g[i] = (uint32_t)a[1] | ((uint32_t)c[1] << 16);
            b[i] = (uint32_t)a[2] | ((uint32_t)c[2] << 16);
        }
    }
    const uint32_t mr = median_pair<P>(r, n, sigma);
    const uint32_t mg = median_pair<P>(g, n, sigma);
    const uint32_t mb = median_pair<P>(b, n, sigma);
    unsigned short* o = dst + ((size_t)y * dw + x) * 3;
    if (two && ((reinterpret_cast<uintptr_t>(o) & 3) == 0))
    {
        uint32_t* o32 = reinterpret_cast<uint32_t*>(o);
        o32[0] = (mr & 0xffffu) | (mg << 16);
        o32[1] = (mb & 0xffffu) | (mr & 0xffff0000u);
        o32[2] = (mg >> 16) | (mb & 0xffff0000u);
    }
    else
    {
        o[0] = (unsigned short)(mr & 0xffffu);
        o[1] = (unsigned short)(mg & 0xffffu);
        o[2] = (unsigned short)(mb & 0xffffu);
        if (two)
        {
            o[3] = (unsigned short)(mr >> 16);
            o[4] = (unsigned short)(mg >> 16);
            o[5] = (unsigned short)(mb >> 16);
        }
    }
}

// ---------------------------------------------------------------------------
// Gain (GainColorOps.cpp:16-26), 8 values per thread with 16-byte accesses.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_gain(unsigned short* __restrict__ d, long long n, float gain)
{
    long long i8 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 8;
    if (i8 >= n) return;
    if (i8 + 8 <= n && ((reinterpret_cast<uintptr_t>(d + i8) & 15) == 0))
    {
        uint4 q = *reinterpret_cast<uint4*>(d + i8);
        unsigned short* s = reinterpret_cast<unsigned short*>(&q);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] = clamp_trunc_u16(fmul(u2f(s[k]), gain));
        *reinterpret_cast<uint4*>(d + i8) = q;
    }
    else
    {
        for (long long i = i8; i < n && i < i8 + 8; ++i) d[i] = clamp_trunc_u16(fmul(u2f(d[i]), gain));
    }
}
}  // namespace

int launch_demosaic(const unsigned short* cfa, int w, int h, unsigned short black, const float* camMul,
                    const float* rgbCam, uint32_t filters, unsigned short* out, cudaStream_t s)
{
    DemosaicParams P;
    for (int i = 0; i < 4; ++i) P.camMul[i] = camMul[i];
    for (int i = 0; i < 12; ++i) P.rgbCam[i] = rgbCam[i];
    P.filters = filters;
    P.black = black;
    // Standard Bayer layout test on the filter word (rows repeat with period
    // 2; one R, one B, G/G2 on a diagonal).
    {
        auto col = [&](int r, int c) { return (int)((filters >> ((((r << 1) & 14) | (c & 1)) << 1)) & 3u); };
        bool periodic = true;
        for (int r = 2; r < 8; ++r)
            for (int c = 0; c < 2; ++c) periodic = periodic && col(r, c) == col(r & 1, c);
        int c00 = col(0, 0), c01 = col(0, 1), c10 = col(1, 0), c11 = col(1, 1);
        auto isG = [](int v) { return v == 1 || v == 3; };
        bool diagG = (isG(c00) && isG(c11) && ((c01 == 0 && c10 == 2) || (c01 == 2 && c10 == 0))) ||
                     (isG(c01) && isG(c10) && ((c00 == 0 && c11 == 2) || (c00 == 2 && c11 == 0)));
        P.std2x2 = (periodic && diagG) ? 1 : 0;
        P.color2x2[0] = isG(c00) ? 1 : c00;
        P.color2x2[1] = isG(c01) ? 1 : c01;
        P.color2x2[2] = isG(c10) ? 1 : c10;
        P.color2x2[3] = isG(c11) ? 1 : c11;
    }
    dim3 grid((w + kDmTW - 1) / kDmTW, (h + kDmTH - 1) / kDmTH);
    k_demosaic<<<grid, dim3(32, 8), 0, s>>>(cfa, w, h, P, out);
    return check_launch("demosaic kernel");
}

int launch_warp(const unsigned short* src, int sw, int sh, unsigned short* dst, int dw, int dh, const float* H,
                int offX, int offY, float gain, cudaStream_t s)
{
    WarpParams P;
    for (int i = 0; i < 9; ++i) P.H[i] = H[i];
    P.gain = gain;
    P.applyGain = gain_is_identity(gain) ? 0 : 1;
    dim3 grid((dw + 31) / 32, (dh + 7) / 8);
    k_warp<<<grid, dim3(32, 8), 0, s>>>(src, sw, sh, dst, dw, dh, offX, offY, P);
    return check_launch("warp kernel");
}

int launch_median(const unsigned short* const* inputs, int n, unsigned short* out, int w, int h, float sigma,
                  cudaStream_t s)
{
    MedianInputs in;
    const int cnt = n < kMaxContributors ? n : kMaxContributors;
    uintptr_t align = reinterpret_cast<uintptr_t>(out);
    for (int i = 0; i < kMaxContributors; ++i)
    {
        in.p[i] = i < cnt ? inputs[i] : nullptr;
        if (i < cnt) align |= reinterpret_cast<uintptr_t>(inputs[i]);
    }
    const long long total = (long long)w * h * 3;
    if ((total & 1) == 0 && (align & 3) == 0)
    {
        const long long pairs = total >> 1;
        const unsigned blocks = (unsigned)((pairs + 255) / 256);
        uint32_t* o = reinterpret_cast<uint32_t*>(out);
        if (cnt <= 4) k_median2<4><<<blocks, 256, 0, s>>>(in, cnt, pairs, sigma, o);
        else if (cnt <= 8) k_median2<8><<<blocks, 256, 0, s>>>(in, cnt, pairs, sigma, o);
        else if (cnt <= 16) k_median2<16><<<blocks, 256, 0, s>>>(in, cnt, pairs, sigma, o);
        else k_median2<32><<<blocks, 256, 0, s>>>(in, cnt, pairs, sigma, o);
    }
    else
    {
        const unsigned blocks = (unsigned)((total + 255) / 256);
        if (cnt <= 4) k_median1<4><<<blocks, 256, 0, s>>>(in, cnt, total, sigma, out);
        else if (cnt <= 8) k_median1<8><<<blocks, 256, 0, s>>>(in, cnt, total, sigma, out);
        else if (cnt <= 16) k_median1<16><<<blocks, 256, 0, s>>>(in, cnt, total, sigma, out);
        else k_median1<32><<<blocks, 256, 0, s>>>(in, cnt, total, sigma, out);
    }
    return check_launch("median kernel");
}

int launch_warp_median(const unsigned short* const* frames, int n, int sw, int sh, const float* H, unsigned short* out,
                       int dw, int dh, int offX, int offY, float sigma, cudaStream_t s)
{
    StackParams S;
    const int cnt = n < kMaxContributors ? n : kMaxContributors;
    for (int i = 0; i < kMaxContributors; ++i)
    {
        S.src[i] = i < cnt ? frames[i] : nullptr;
        for (int q = 0; q < 9; ++q) S.H[i][q] = i < cnt ? H[(size_t)i * 9 + q] : 0.0f;
    }
    dim3 grid((unsigned)((dw + 63) / 64), (unsigned)((dh + 7) / 8));
    dim3 block(32, 8);
    if (cnt <= 4) k_warp_median<4><<<grid, block, 0, s>>>(S, cnt, sw, sh, out, dw, dh, offX, offY, sigma);
    else if (cnt <= 8) k_warp_median<8><<<grid, block, 0, s>>>(S, cnt, sw, sh, out, dw, dh, offX, offY, sigma);
    else if (cnt <= 16) k_warp_median<16><<<grid, block, 0, s>>>(S, cnt, sw, sh, out, dw, dh, offX, offY, sigma);
    else k_warp_median<32><<<grid, block, 0, s>>>(S, cnt, sw, sh, out, dw, dh, offX, offY, sigma);
    return check_launch("warp + median kernel");
}

int launch_gain(unsigned short* data, long long n, float gain, cudaStream_t s)
{
    if (gain_is_identity(gain) || n <= 0) return I360B_SUCCESS;
    long long threads = (n + 7) / 8;
    k_gain<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(data, n, gain);
    return check_launch("gain kernel");
}
}  // namespace i360b
