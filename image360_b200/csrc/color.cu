// CIE Lab colour statistics and Reinhard colour transfer of RGB48 images: the
// Optimize-stage colour correction that feeds the render path
// (OptimizeExecutor.cpp:308-330 calls ComputeLabStats on the reference and the
// target image, then ApplyReinhardColorTransfer on the target).
//
// Arithmetic follows the reference's CPU implementation (GainColorOps.cpp:28-156)
// step by step in FP32 with every product and sum rounded separately (this file
// is built without FMA contraction) and the statistics in FP64.  The
// reference's FP64 transfer (lab - mean) * scale + refMean is carried in
// float-float arithmetic (hi + lo pairs, ~48 bits) and rounded once to FP32,
// which gives the FP64 result's FP32 rounding except when that lies within
// ~2^-48 of a rounding boundary (about 1 value in 10^7, mostly where the sum
// cancels toward 0).  The transcendental steps are evaluated to the correctly
// rounded FP32 result:
//   * sRGB decode of a 16-bit code, ((c + 0.055f) / 1.055f)^2.4f
//     (GainColorOps.cpp:30-33): a 65536-entry table, each entry the FP64 power
//     rounded to FP32, built on the device once per process;
//   * the cube root of LabF (GainColorOps.cpp:40-44): a 2^(log2(t)/3) seed
//     refined by one Newton step y -= (y^3 - t) / (3 y^2) whose residual
//     y^3 - t is formed exactly from FMA product error terms, in FP32;
//   * the sRGB encode power c^(1/2.4f) (GainColorOps.cpp:35-38): a
//     2^(e log2 c) seed refined by one Newton step on z^12 = c^5 whose
//     residual is formed from FMA error terms in FP32, together with the
//     first-order factor 1 + (e - 5/12) ln c for the FP32 exponent e = 1/2.4f
//     (|e - 5/12| ~ 1e-8), rounded once.
// Divisions by the conversion's constants use the reciprocal and one FMA
// residual correction, which equals IEEE division for 2^-99 <= |x| < 2^100
// (checked for every float in that range and each divisor by
// tests/color_arith_check.c); outside it they divide.
// The reference's libm powf/cbrtf are within about one ulp of those values, so
// outputs agree within 1 LSB at 16 bits, and the statistics to FP64 summation
// order.
//
// Layout: RGB48 interleaved, row-major, 6 bytes per pixel.  When the image base
// is 16-byte aligned a block moves chunks of 2048 pixels through shared memory
// with 16-byte loads and stores; the remainder (and unaligned images) go one
// pixel per thread.  The statistics are reduced per block in
// FP64 into a partials array and summed by one block in a fixed order, so they
// are deterministic from run to run.
#include "common.cuh"

#include <mutex>

using namespace i360b;

namespace
{
// ---------------------------------------------------------------------------
// Constants (GainColorOps.cpp:40-54), folded in FP32 exactly as the reference's
// compiler folds them.
// ---------------------------------------------------------------------------
constexpr float kDelta = 6.0f / 29.0f;
constexpr float kDelta3 = kDelta * kDelta * kDelta;
constexpr float kThreeDelta2 = 3.0f * kDelta * kDelta;
constexpr float kFourOver29 = 4.0f / 29.0f;
constexpr float kXn = 0.95047f;
constexpr float kYn = 1.0f;
constexpr float kZn = 1.08883f;
constexpr float kInvGamma = 1.0f / 2.4f;
// (FP32 exponent - 5/12) ln 2: the correction of the encode power per unit of log2 c.
constexpr float kInvGammaDeltaLn2 = (float)(((double)kInvGamma - 5.0 / 12.0) * 0.69314718055994530942);

constexpr int kMaxImages = 64;   // images per batched launch
constexpr int kThreads = 256;
constexpr int kPixPerThread = 8;

__device__ float g_srgbDecode[65536];

__global__ void k_build_decode_table()
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 65536) return;
    const float c = fdiv((float)i, 65535.0f);
    float v;
    if (c <= 0.04045f)
        v = fdiv(c, 12.92f);
    else
        v = __double2float_rn(pow((double)fdiv(fadd(c, 0.055f), 1.055f), (double)2.4f));
    g_srgbDecode[i] = v;
}

// x / d for the constant divisor d with r = 1.0f / d (see the header comment).
__device__ __forceinline__ float div_const(float x, float d, float r)
{
    const float ax = fabsf(x);
    if (ax >= 0x1p-99f && ax < 0x1p100f)
    {
        const float q = fmul(x, r);
        return __fmaf_rn(__fmaf_rn(-q, d, x), r, q);
    }
    return fdiv(x, d);
}

// x / d without the range guard, for x = 0 or x >= 2^-99 (the reciprocal
// step gives +0 for x = 0, like the division).
__device__ __forceinline__ float div_const_nonneg(float x, float d, float r)
{
    const float q = fmul(x, r);
    return __fmaf_rn(__fmaf_rn(-q, d, x), r, q);
}

constexpr float kRcpXn = 1.0f / kXn;
constexpr float kRcpZn = 1.0f / kZn;
constexpr float kRcpThreeDelta2 = 1.0f / kThreeDelta2;

// Correctly rounded cube root for t in (kDelta3, 2]: p + pl = y^2 and
// c + cl = p y exactly (FMA error terms), c - t is exact (Sterbenz), so the
// residual y^3 - t carries only the rounding of the tiny pl y term.
__device__ __forceinline__ float cbrt_rn(float t)
{
    const float y = exp2f(fmul(__log2f(t), 0.333333343f));
    const float p = fmul(y, y), pl = __fmaf_rn(y, y, -p);
    const float c = fmul(p, y), cl = __fmaf_rn(p, y, -c);
    const float e = fadd(fsub(c, t), __fmaf_rn(pl, y, cl));
    return fsub(y, __fdividef(e, fmul(3.0f, p)));
}

// c^(1/2.4f) correctly rounded for c in [0.0031308, 2]; above 2 the encoded
// value exceeds 1 and clamps to 65535 whatever its last bits.  z^12 and c^5
// are carried as hi + lo pairs from FMA error terms; their hi parts agree to a
// few ulp, so hi - hi is exact (Sterbenz) and the residual keeps ~2^-46.
__device__ __forceinline__ float encode_pow_rn(float c)
{
    const float l2 = __log2f(c);
    const float z = exp2f(fmul(l2, kInvGamma));
    if (!(c <= 2.0f)) return z;
    const float z2 = fmul(z, z), z2l = __fmaf_rn(z, z, -z2);
    const float z4 = fmul(z2, z2), z4l = fadd(__fmaf_rn(z2, z2, -z4), fmul(fmul(2.0f, z2), z2l));
    const float z8 = fmul(z4, z4), z8l = fadd(__fmaf_rn(z4, z4, -z8), fmul(fmul(2.0f, z4), z4l));
    const float z12 = fmul(z8, z4), z12l = fadd(__fmaf_rn(z8, z4, -z12), fadd(fmul(z8, z4l), fmul(z4, z8l)));
    const float c2 = fmul(c, c), c2l = __fmaf_rn(c, c, -c2);
    const float c4 = fmul(c2, c2), c4l = fadd(__fmaf_rn(c2, c2, -c4), fmul(fmul(2.0f, c2), c2l));
    const float c5 = fmul(c4, c), c5l = fadd(__fmaf_rn(c4, c, -c5), fmul(c4l, c));
    const float q = __fdividef(fadd(fsub(z12, c5), fsub(z12l, c5l)), z12);
    const float corr = fsub(fmul(kInvGammaDeltaLn2, l2), fmul(q, 1.0f / 12.0f));
    return __fmaf_rn(z, corr, z);
}

// (unsigned short) of v clamped to [0, 65535], truncated (NaN -> 0): v + 2^23
// rounded toward zero holds trunc(v) in its low mantissa bits (no conversion
// instruction).
__device__ __forceinline__ unsigned short trunc_u16(float v)
{
    v = v > 0.0f ? v : 0.0f;
    v = v < 65535.0f ? v : 65535.0f;
    return (unsigned short)(__float_as_uint(__fadd_rz(v, 8388608.0f)) & 0xffffu);
}

__device__ __forceinline__ float lab_f(float t)  // GainColorOps.cpp:40-44
{
    return t > kDelta3 ? cbrt_rn(t) : fadd(div_const_nonneg(t, kThreeDelta2, kRcpThreeDelta2), kFourOver29);
}

__device__ __forceinline__ float lab_f_inv(float t)  // GainColorOps.cpp:46-50
{
    return t > kDelta ? fmul(fmul(t, t), t) : fmul(kThreeDelta2, fsub(t, kFourOver29));
}

__device__ __forceinline__ float srgb_encode(float c)  // GainColorOps.cpp:35-38
{
    return c <= 0.0031308f ? fmul(c, 12.92f) : fsub(fmul(1.055f, encode_pow_rn(c)), 0.055f);
}

struct Lab
{
    float v[3];
};

// GainColorOps.cpp:56-73.
__device__ __forceinline__ Lab rgb_to_lab(unsigned r16, unsigned g16, unsigned b16)
{
    const float r = __ldg(&g_srgbDecode[r16]);
    const float g = __ldg(&g_srgbDecode[g16]);
    const float b = __ldg(&g_srgbDecode[b16]);
    const float X = fadd(fadd(fmul(0.4124564f, r), fmul(0.3575761f, g)), fmul(0.1804375f, b));
    const float Y = fadd(fadd(fmul(0.2126729f, r), fmul(0.7151522f, g)), fmul(0.0721750f, b));
    const float Z = fadd(fadd(fmul(0.0193339f, r), fmul(0.1191920f, g)), fmul(0.9503041f, b));
    // X, Y, Z are 0 or at least ~2e-8 (the smallest non-zero table entry,
    // (1 / 65535) / 12.92, times the smallest coefficient of a row), inside
    // the unguarded division's exact range.
    const float fx = lab_f(div_const_nonneg(X, kXn, kRcpXn));
    const float fy = lab_f(Y);  // Y / kYn with kYn = 1 is Y exactly
    const float fz = lab_f(div_const_nonneg(Z, kZn, kRcpZn));
    Lab o;
    o.v[0] = fsub(fmul(116.0f, fy), 16.0f);
    o.v[1] = fmul(500.0f, fsub(fx, fy));
    o.v[2] = fmul(200.0f, fsub(fy, fz));
    return o;
}

// GainColorOps.cpp:75-100.
__device__ __forceinline__ void lab_to_rgb(const Lab& lab, unsigned short* out)
{
    const float fy = div_const(fadd(lab.v[0], 16.0f), 116.0f, 1.0f / 116.0f);
    const float fx = fadd(fy, div_const(lab.v[1], 500.0f, 1.0f / 500.0f));
    const float fz = fsub(fy, div_const(lab.v[2], 200.0f, 1.0f / 200.0f));
    const float X = fmul(kXn, lab_f_inv(fx));
    const float Y = lab_f_inv(fy);  // kYn * v with kYn = 1 is v exactly
    const float Z = fmul(kZn, lab_f_inv(fz));
    const float rl = fsub(fsub(fmul(3.2404542f, X), fmul(1.5371385f, Y)), fmul(0.4985314f, Z));
    const float gl = fadd(fadd(fmul(-0.9692660f, X), fmul(1.8760108f, Y)), fmul(0.0415560f, Z));
    const float bl = fadd(fsub(fmul(0.0556434f, X), fmul(0.2040259f, Y)), fmul(1.0572252f, Z));
    // (std::max)(x, 0.0f) keeps a NaN x, as the reference does.
    const float r = srgb_encode(rl < 0.0f ? 0.0f : rl);
    const float g = srgb_encode(gl < 0.0f ? 0.0f : gl);
    const float b = srgb_encode(bl < 0.0f ? 0.0f : bl);
    out[0] = trunc_u16(fmul(r, 65535.0f));
    out[1] = trunc_u16(fmul(g, 65535.0f));
    out[2] = trunc_u16(fmul(b, 65535.0f));
}

// A batch of images, each covered by a run of blocks.
struct ImageSet
{
    unsigned short* img[kMaxImages];
    long long pixels[kMaxImages];
    int blockStart[kMaxImages + 1];  // prefix of blocks per image
    int statIndex[kMaxImages];       // transfer: row of dStats holding the image's own statistics
    int n;
};

__device__ __forceinline__ int image_of_block(const ImageSet& s, int b)
{
    int lo = 0, hi = s.n - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (s.blockStart[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// A block's chunk of kChunkPx consecutive pixels (kChunkPx * 6 bytes) staged in
// shared memory: loaded and stored as 16-byte words by consecutive threads,
// processed with thread t on pixels t, t + kThreads, ... so that a warp reads 32
// consecutive pixels.  The per-pixel code is a rolled loop, small enough for
// the instruction cache.
constexpr int kChunkPx = kThreads * kPixPerThread;
constexpr int kChunkWords = kChunkPx * 6 / 16;

__device__ __forceinline__ void stage_load(uint4* stage, const unsigned short* src)
{
    const uint4* q = reinterpret_cast<const uint4*>(src);
    for (int i = threadIdx.x; i < kChunkWords; i += kThreads) stage[i] = __ldcs(q + i);
}

__device__ __forceinline__ void stage_store(const uint4* stage, unsigned short* dst)
{
    uint4* q = reinterpret_cast<uint4*>(dst);
    for (int i = threadIdx.x; i < kChunkWords; i += kThreads) __stcs(q + i, stage[i]);
}

__device__ __forceinline__ void accumulate(const Lab& lab, double* acc)
{
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        const double v = lab.v[c];
        acc[c] += v;
        acc[3 + c] += v * v;
    }
}

// Per-block FP64 sums (sum L, a, b, sum of squares L, a, b) of each image's
// pixels, written to partials[block][6].
__global__ void __launch_bounds__(kThreads) k_lab_partials(const __grid_constant__ ImageSet set, double* partials)
{
    const int im = image_of_block(set, blockIdx.x);
    const int nb = set.blockStart[im + 1] - set.blockStart[im];
    const int bi = blockIdx.x - set.blockStart[im];
    const unsigned short* img = set.img[im];
    const long long npx = set.pixels[im];
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    __shared__ uint4 stage[kChunkWords];
    const bool vec = (reinterpret_cast<uintptr_t>(img) & 15) == 0;
    const long long chunks = vec ? npx / kChunkPx : 0;
    for (long long ch = bi; ch < chunks; ch += nb)
    {
        stage_load(stage, img + ch * kChunkPx * 3);
        __syncthreads();
        const unsigned short* sp = reinterpret_cast<const unsigned short*>(stage);
#pragma unroll 1
        for (int p = 0; p < kPixPerThread; ++p)
        {
            const unsigned short* q = sp + (threadIdx.x + p * kThreads) * 3;
            accumulate(rgb_to_lab(q[0], q[1], q[2]), acc);
        }
        __syncthreads();
    }
    const long long stride = (long long)nb * kThreads;
    for (long long px = chunks * kChunkPx + (long long)bi * kThreads + threadIdx.x; px < npx; px += stride)
    {
        const unsigned short* q = img + px * 3;
        accumulate(rgb_to_lab(q[0], q[1], q[2]), acc);
    }
    __shared__ double red[kThreads / 32][6];
#pragma unroll
    for (int c = 0; c < 6; ++c)
    {
        double x = acc[c];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        acc[c] = x;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int c = 0; c < 6; ++c) red[warp][c] = acc[c];
    __syncthreads();
    if (threadIdx.x < 6)
    {
        double x = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) x += red[w][threadIdx.x];
        partials[(size_t)blockIdx.x * 6 + threadIdx.x] = x;
    }
}

// One block per image: sums the image's partials in block order and writes
// stats[image] = {mean L, a, b, std L, a, b} (GainColorOps.cpp:123-129).
__global__ void k_lab_finish(const __grid_constant__ ImageSet set, const double* partials, double* stats)
{
    const int im = blockIdx.x;
    const int b0 = set.blockStart[im], b1 = set.blockStart[im + 1];
    __shared__ double red[32][6];
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x)
        for (int c = 0; c < 6; ++c) acc[c] += partials[(size_t)b * 6 + c];
#pragma unroll
    for (int c = 0; c < 6; ++c)
    {
        double x = acc[c];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        acc[c] = x;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int c = 0; c < 6; ++c) red[warp][c] = acc[c];
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double sum[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            for (int c = 0; c < 6; ++c) sum[c] += red[w][c];
        const double n = (double)set.pixels[im];
        for (int c = 0; c < 3; ++c)
        {
            const double mean = sum[c] / n;
            const double var = sum[3 + c] / n - mean * mean;
            stats[(size_t)im * 6 + c] = mean;
            stats[(size_t)im * 6 + 3 + c] = sqrt(var > 0.0 ? var : 0.0);
        }
    }
}

// Per-channel transfer coefficients (GainColorOps.cpp:146-151): lab' =
// (lab - srcMean) * (refStd / stdSrc) + refMean, stdSrc = srcStd or 1 when
// srcStd <= 1e-6, the FP64 coefficients held as float pairs hi + lo.
struct FloatPair
{
    float h, l;
};

__device__ __forceinline__ FloatPair split(double x)
{
    FloatPair p;
    p.h = __double2float_rn(x);
    p.l = __double2float_rn(x - (double)p.h);
    return p;
}

struct Transfer
{
    FloatPair srcMean[3], scale[3], refMean[3];
};

__device__ __forceinline__ Transfer make_transfer(const double* src, const double* ref)
{
    Transfer t;
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        const double s = src[3 + c] > 1e-6 ? src[3 + c] : 1.0;
        t.srcMean[c] = split(src[c]);
        t.scale[c] = split(ref[3 + c] / s);
        t.refMean[c] = split(ref[c]);
    }
    return t;
}

// (v - m) * k + r in float-float, rounded once: two-sum for the differences
// and sums, an FMA error term for the product.
__device__ __forceinline__ float transfer_value(float v, const FloatPair& m, const FloatPair& k, const FloatPair& r)
{
    const float s = fsub(v, m.h);
    const float sb = fsub(s, v);
    const float se = fsub(fadd(fsub(v, fsub(s, sb)), fsub(-m.h, sb)), m.l);
    const float dh = fadd(s, se);
    const float dl = fsub(se, fsub(dh, s));
    const float ph = fmul(dh, k.h);
    const float pl = fadd(__fmaf_rn(dh, k.h, -ph), fadd(fmul(dh, k.l), fmul(dl, k.h)));
    const float th = fadd(ph, r.h);
    const float tb = fsub(th, ph);
    const float te = fadd(fadd(fsub(ph, fsub(th, tb)), fsub(r.h, tb)), fadd(pl, r.l));
    return fadd(th, te);
}

__device__ __forceinline__ void transfer_pixel(const Transfer& t, const unsigned short* in, unsigned short* out)
{
    Lab lab = rgb_to_lab(in[0], in[1], in[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) lab.v[c] = transfer_value(lab.v[c], t.srcMean[c], t.scale[c], t.refMean[c]);
    lab_to_rgb(lab, out);
}

// In-place transfer of each image of the set from its own statistics
// (stats[set.statIndex[image]]) to refStats.
__global__ void __launch_bounds__(kThreads) k_reinhard(const __grid_constant__ ImageSet set, const double* stats,
                                                       const double* refStats)
{
    const int im = image_of_block(set, blockIdx.x);
    const int nb = set.blockStart[im + 1] - set.blockStart[im];
    const int bi = blockIdx.x - set.blockStart[im];
    unsigned short* img = set.img[im];
    const long long npx = set.pixels[im];
    const Transfer t = make_transfer(stats + (size_t)set.statIndex[im] * 6, refStats);
    __shared__ uint4 stage[kChunkWords];
    const bool vec = (reinterpret_cast<uintptr_t>(img) & 15) == 0;
    const long long chunks = vec ? npx / kChunkPx : 0;
    for (long long ch = bi; ch < chunks; ch += nb)
    {
        // each thread stores back exactly the words it loaded, so no barrier
        // is needed between one chunk's store and the next chunk's load
        stage_load(stage, img + ch * kChunkPx * 3);
        __syncthreads();
        unsigned short* sp = reinterpret_cast<unsigned short*>(stage);
#pragma unroll 1
        for (int p = 0; p < kPixPerThread; ++p)
        {
            unsigned short* q = sp + (threadIdx.x + p * kThreads) * 3;
            unsigned short o[3];
            transfer_pixel(t, q, o);
            q[0] = o[0];
            q[1] = o[1];
            q[2] = o[2];
        }
        __syncthreads();
        stage_store(stage, img + ch * kChunkPx * 3);
    }
    const long long stride = (long long)nb * kThreads;
    for (long long px = chunks * kChunkPx + (long long)bi * kThreads + threadIdx.x; px < npx; px += stride)
    {
        unsigned short o[3];
        transfer_pixel(t, img + px * 3, o);
        img[px * 3] = o[0];
        img[px * 3 + 1] = o[1];
        img[px * 3 + 2] = o[2];
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

int ensure_decode_table(cudaStream_t s)
{
    static std::mutex mu;
    static bool built[64] = {};
    const int dev = device();
    if (dev < 0 || dev >= 64) return fail(I360B_CUDA_ERROR, "Colour transfer: unsupported device index %d.", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (built[dev]) return I360B_SUCCESS;
    k_build_decode_table<<<256, 256, 0, s>>>();
    I360B_TRY(check_launch("sRGB decode table kernel"));
    I360B_CUDA(cudaStreamSynchronize(s), "sRGB decode table");
    built[dev] = true;
    return I360B_SUCCESS;
}

// Blocks per image: one wave of resident blocks (`perSm` per SM) over the
// whole batch, shared in proportion to pixel count, at least one per image and
// no more than the image has chunks.
int plan_blocks(ImageSet& set, int perSm)
{
    long long total = 0;
    for (int i = 0; i < set.n; ++i) total += set.pixels[i];
    const long long target = (long long)sm_count() * (perSm > 0 ? perSm : 1);
    set.blockStart[0] = 0;
    for (int i = 0; i < set.n; ++i)
    {
        const long long groups = (set.pixels[i] + kPixPerThread - 1) / kPixPerThread;
        long long b = total > 0 ? (target * set.pixels[i] + total - 1) / total : 1;
        const long long cap = (groups + kThreads - 1) / kThreads;  // no block without work
        b = b < 1 ? 1 : (b > cap ? cap : b);
        set.blockStart[i + 1] = set.blockStart[i] + (int)b;
    }
    return set.blockStart[set.n];
}

int check_images(unsigned short* const* imgs, const int* w, const int* h, int n)
{
    if (!imgs || !w || !h) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (n <= 0 || n > kMaxImages) return fail(I360B_INVALID_PARAM, "Image count must be 1-%d.", kMaxImages);
    for (int i = 0; i < n; ++i)
    {
        if (!imgs[i]) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
        if (w[i] <= 0 || h[i] <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    }
    return I360B_SUCCESS;
}

// Resident blocks per SM of a colour kernel (occupancy query, once per process).
template <typename K>
int resident_blocks(K kernel)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreads, 0) != cudaSuccess) n = 4;
    return n > 0 ? n : 1;
}

int stats_blocks_per_sm()
{
    static const int n = resident_blocks(k_lab_partials);
    return n;
}

int transfer_blocks_per_sm()
{
    static const int n = resident_blocks(k_reinhard);
    return n;
}

ImageSet make_set(unsigned short* const* imgs, const int* w, const int* h, int n)
{
    ImageSet set{};
    set.n = n;
    for (int i = 0; i < n; ++i)
    {
        set.img[i] = imgs[i];
        set.pixels[i] = (long long)w[i] * h[i];
        set.statIndex[i] = i;
    }
    return set;
}

struct Scratch
{
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() { dev_free(p, s); }
};

// Statistics of every image of the set into dStats[i * 6 .. i * 6 + 5].
int run_stats(const ImageSet& set, int blocks, double* dStats, cudaStream_t s)
{
    Scratch part;
    part.s = s;
    I360B_TRY(dev_alloc(&part.p, (size_t)blocks * 6 * sizeof(double), s, "Lab statistics"));
    k_lab_partials<<<blocks, kThreads, 0, s>>>(set, static_cast<double*>(part.p));
    I360B_TRY(check_launch("Lab statistics kernel"));
    k_lab_finish<<<set.n, 256, 0, s>>>(set, static_cast<const double*>(part.p), dStats);
    return check_launch("Lab statistics reduction kernel");
}
}  // namespace

namespace i360b
{
int launch_lab_stats(const unsigned short* const* dImgs, const int* w, const int* h, int n, double* dStats,
                     cudaStream_t s)
{
    I360B_TRY(check_images(const_cast<unsigned short* const*>(dImgs), w, h, n));
    if (!dStats) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    I360B_TRY(ensure_decode_table(s));
    ImageSet set = make_set(const_cast<unsigned short* const*>(dImgs), w, h, n);
    const int blocks = plan_blocks(set, stats_blocks_per_sm());
    return run_stats(set, blocks, dStats, s);
}

int launch_reinhard(unsigned short* const* dImgs, const int* w, const int* h, int n, const double* dSrcStats,
                    const double* dRefStats, cudaStream_t s)
{
    I360B_TRY(check_images(dImgs, w, h, n));
    if (!dSrcStats || !dRefStats) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    I360B_TRY(ensure_decode_table(s));
    ImageSet set = make_set(dImgs, w, h, n);
    const int blocks = plan_blocks(set, transfer_blocks_per_sm());
    k_reinhard<<<blocks, kThreads, 0, s>>>(set, dSrcStats, dRefStats);
    return check_launch("Reinhard transfer kernel");
}

int launch_color_correct(unsigned short* const* dImgs, const int* w, const int* h, int n, int refIndex,
                         double* dStats, cudaStream_t s)
{
    I360B_TRY(check_images(dImgs, w, h, n));
    if (refIndex < 0 || refIndex >= n) return fail(I360B_INVALID_PARAM, "Reference index out of range.");
    I360B_TRY(ensure_decode_table(s));
    Scratch own;
    own.s = s;
    if (!dStats)
    {
        I360B_TRY(dev_alloc(&own.p, (size_t)n * 6 * sizeof(double), s, "colour correction"));
        dStats = static_cast<double*>(own.p);
    }
    ImageSet all = make_set(dImgs, w, h, n);
    const int blocks = plan_blocks(all, stats_blocks_per_sm());
    I360B_TRY(run_stats(all, blocks, dStats, s));
    if (n == 1) return I360B_SUCCESS;
    // The reference image passes through unchanged (OptimizeExecutor.cpp:290-296).
    ImageSet targets{};
    for (int i = 0; i < n; ++i)
    {
        if (i == refIndex) continue;
        targets.img[targets.n] = all.img[i];
        targets.pixels[targets.n] = all.pixels[i];
        targets.statIndex[targets.n] = i;
        ++targets.n;
    }
    const int tblocks = plan_blocks(targets, transfer_blocks_per_sm());
    k_reinhard<<<tblocks, kThreads, 0, s>>>(targets, dStats, dStats + (size_t)refIndex * 6);
    return check_launch("Reinhard transfer kernel");
}
}  // namespace i360b
