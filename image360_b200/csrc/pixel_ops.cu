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
};

__device__ __forceinline__ int bayer_color(int row, int col, uint32_t filters)
{
    // BayerDemosaicKernels.h:10-13.
    return (int)((filters >> ((((row << 1) & 14) | (col & 1)) << 1)) & 3u);
}

__global__ void __launch_bounds__(256) k_demosaic(const unsigned short* __restrict__ cfa, int w, int h,
                                                  DemosaicParams P, unsigned short* __restrict__ out)
{
    __shared__ unsigned short s[kDmTH + 2][kDmTW + 2];
    const int tx0 = blockIdx.x * kDmTW, ty0 = blockIdx.y * kDmTH;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int i = tid; i < (kDmTH + 2) * (kDmTW + 2); i += 256)
    {
        int r = i / (kDmTW + 2), c = i % (kDmTW + 2);
        int gx = tx0 - 1 + c, gy = ty0 - 1 + r;
        unsigned short v = 0;
        if (gx >= 0 && gy >= 0 && gx < w && gy < h)
        {
            unsigned short raw = __ldg(cfa + (size_t)gy * w + gx);
            raw = raw > P.black ? (unsigned short)(raw - P.black) : (unsigned short)0;
            v = clamp_trunc_u16(fmul((float)raw, P.camMul[bayer_color(gy, gx, P.filters)]));
        }
        s[r][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int oy = 0; oy < 2; ++oy)
#pragma unroll
        for (int ox = 0; ox < 2; ++ox)
        {
            int lx = threadIdx.x * 2 + ox, ly = threadIdx.y * 2 + oy;
            int x = tx0 + lx, y = ty0 + ly;
            if (x >= w || y >= h) continue;
            float rgb[3] = {0.0f, 0.0f, 0.0f};
            int cnt[3] = {0, 0, 0};
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx)
                {
                    int nx = x + dx, ny = y + dy;
                    if (nx < 0 || ny < 0 || nx >= w || ny >= h) continue;
                    int ch = bayer_color(ny, nx, P.filters);
                    int slot = ch == 3 ? 1 : ch;
                    float v = (float)s[ly + 1 + dy][lx + 1 + dx];
                    // Integer-valued sums below 2^24: exact in any order.
                    if (slot == 0) { rgb[0] += v; cnt[0]++; }
                    else if (slot == 1) { rgb[1] += v; cnt[1]++; }
                    else { rgb[2] += v; cnt[2]++; }
                }
            int mine = bayer_color(y, x, P.filters);
            int my = mine == 3 ? 1 : mine;
            float own = (float)s[ly + 1][lx + 1];
            unsigned short px[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
                float v = rgb[c];
                if (c == my) v = own;
                else if (cnt[c] != 0) v = fdiv(v, (float)cnt[c]);
                px[c] = clamp_trunc_u16(v);
            }
            float r = (float)px[0], g = (float)px[1], b = (float)px[2];
            unsigned short* o = out + ((size_t)y * w + x) * 3;
#pragma unroll
            for (int row = 0; row < 3; ++row)
            {
                float val = fadd(fadd(fadd(fmul(P.rgbCam[row * 4 + 0], r), fmul(P.rgbCam[row * 4 + 1], g)),
                                      fmul(P.rgbCam[row * 4 + 2], b)),
                                 P.rgbCam[row * 4 + 3]);
                o[row] = clamp_trunc_u16(val);
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
    int x0 = (int)floorf(sx), y0 = (int)floorf(sy);
    float fx = fsub(sx, (float)x0), fy = fsub(sy, (float)y0);
    float gx = fsub(1.0f, fx), gy = fsub(1.0f, fy);
    float w00 = fmul(gx, gy), w10 = fmul(fx, gy), w01 = fmul(gx, fy), w11 = fmul(fx, fy);
    const unsigned short* r0 = src + ((size_t)y0 * sw + x0) * 3;
    const unsigned short* r1 = r0 + (size_t)sw * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        float v = fadd(fadd(fadd(fmul(w00, (float)__ldg(r0 + c)), fmul(w10, (float)__ldg(r0 + 3 + c))),
                            fmul(w01, (float)__ldg(r1 + c))),
                       fmul(w11, (float)__ldg(r1 + 3 + c)));
        unsigned short q = clamp_trunc_u16(v);
        if (P.applyGain) q = clamp_trunc_u16(fmul((float)q, P.gain));
        o[c] = q;
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
// One output scalar per thread.  Statistics are accumulated sequentially in
// input order in FP32 (sumSq exceeds 2^24, so the order is part of the
// result).  Clipped-out values become INT_MAX and a register bitonic network
// of the padded width sorts; the median is element keptCount/2.
// ---------------------------------------------------------------------------
struct MedianInputs
{
    const unsigned short* p[kMaxContributors];
};

template <int P>
__device__ __forceinline__ void bitonic_sort(int (&v)[P])
{
#pragma unroll
    for (int k = 2; k <= P; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < P; ++i)
            {
                int l = i ^ j;
                if (l > i)
                {
                    int a = v[i], b = v[l];
                    int lo = min(a, b), hi = max(a, b);
                    bool up = (i & k) == 0;
                    v[i] = up ? lo : hi;
                    v[l] = up ? hi : lo;
                }
            }
}

template <int P>
__global__ void __launch_bounds__(256) k_median(MedianInputs in, int n, long long total, float sigma,
                                                unsigned short* __restrict__ out)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int v[P];
#pragma unroll
    for (int i = 0; i < P; ++i) v[i] = i < n ? (int)__ldg(in.p[i] + idx) : 0x7fffffff;
    int count = n;
    if (n > 3)
    {
        float sum = 0.0f, sumSq = 0.0f;
#pragma unroll
        for (int i = 0; i < P; ++i)
            if (i < n)
            {
                float f = (float)v[i];
                sum = fadd(sum, f);
                sumSq = fadd(sumSq, fmul(f, f));
            }
        float fn = (float)n;
        float mean = fdiv(sum, fn);
        float var = fsub(fdiv(sumSq, fn), fmul(mean, mean));
        float sd = __fsqrt_rn(var < 0.0f ? 0.0f : var);
        float lo = fsub(mean, fmul(sigma, sd));
        float hi = fadd(mean, fmul(sigma, sd));
        int kept = 0;
#pragma unroll
        for (int i = 0; i < P; ++i)
            if (i < n)
            {
                float f = (float)v[i];
                kept += (f >= lo && f <= hi) ? 1 : 0;
            }
        if (kept > 0)
        {
#pragma unroll
            for (int i = 0; i < P; ++i)
                if (i < n)
                {
                    float f = (float)v[i];
                    if (!(f >= lo && f <= hi)) v[i] = 0x7fffffff;
                }
            count = kept;
        }
    }
    bitonic_sort<P>(v);
    int m = count >> 1;
    int r = v[0];
#pragma unroll
    for (int i = 1; i < P; ++i)
        if (i == m) r = v[i];
    out[idx] = (unsigned short)r;
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
        for (int k = 0; k < 8; ++k) s[k] = clamp_trunc_u16(fmul((float)s[k], gain));
        *reinterpret_cast<uint4*>(d + i8) = q;
    }
    else
    {
        for (long long i = i8; i < n && i < i8 + 8; ++i) d[i] = clamp_trunc_u16(fmul((float)d[i], gain));
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
    int cnt = n < kMaxContributors ? n : kMaxContributors;
    for (int i = 0; i < kMaxContributors; ++i) in.p[i] = i < cnt ? inputs[i] : nullptr;
    long long total = (long long)w * h * 3;
    unsigned blocks = (unsigned)((total + 255) / 256);
    if (cnt <= 4) k_median<4><<<blocks, 256, 0, s>>>(in, cnt, total, sigma, out);
    else if (cnt <= 8) k_median<8><<<blocks, 256, 0, s>>>(in, cnt, total, sigma, out);
    else if (cnt <= 16) k_median<16><<<blocks, 256, 0, s>>>(in, cnt, total, sigma, out);
    else k_median<32><<<blocks, 256, 0, s>>>(in, cnt, total, sigma, out);
    return check_launch("median kernel");
}

int launch_gain(unsigned short* data, long long n, float gain, cudaStream_t s)
{
    if (gain_is_identity(gain) || n <= 0) return I360B_SUCCESS;
    long long threads = (n + 7) / 8;
    k_gain<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(data, n, gain);
    return check_launch("gain kernel");
}
}  // namespace i360b
