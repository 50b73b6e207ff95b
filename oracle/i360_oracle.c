/*
 * Test infrastructure only (the oracle): a plain-C restatement of the
 * reference's CPU render path (thnak/Image360, WindowsApp.Core).  Used by the
 * tests and bench.py's CPU-baseline leg as the checker; never by the product.
 *
 * Pinned against the reference itself: tests/test_oracle_ref.py compares every
 * function here with the reference's own code (oracle/_ref, compiled from the
 * reference sources) and tests/test_oracle_golden.py with the committed golden
 * vectors that the reference produced (tests/golden/make_golden.py).
 *
 * Built with -ffp-contract=off and no FMA so each FP32 expression is evaluated
 * exactly as written, in the reference's order.
 */
#define _POSIX_C_SOURCE 200809L
#include "i360_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static inline uint16_t clamp_trunc_u16(float v)
{
    /* (unsigned short)min(max(v, 0), 65535): truncation toward zero. */
    if (!(v > 0.0f)) v = 0.0f;
    if (v > 65535.0f) v = 65535.0f;
    return (uint16_t)v;
}

static inline uint16_t clamp_trunc_u16_d(double v)
{
    if (!(v > 0.0)) v = 0.0;
    if (v > 65535.0) v = 65535.0;
    return (uint16_t)v;
}

/* ------------------------------------------------------------------------ */
/* Demosaic: BayerDemosaic_Scalar.cpp:9-50, BayerDemosaicKernels.h:10-75.     */
/* ------------------------------------------------------------------------ */

static inline int bayer_color(int row, int col, uint32_t filters)
{
    /* BayerDemosaicKernels.h:10-13 (LibRaw's 2-bit-per-site filter word). */
    return (int)((filters >> ((((row << 1) & 14) | (col & 1)) << 1)) & 3u);
}

void or_demosaic(const uint16_t* cfaIn, int w, int h, uint16_t black, const float* camMul,
                 const float* rgbCam, uint32_t filters, uint16_t* out)
{
    size_t n = (size_t)w * h;
    uint16_t* cfa = (uint16_t*)malloc(n * sizeof(uint16_t));
    /* Black level subtract, saturating (BayerDemosaic_Scalar.cpp:18-22). */
    for (size_t i = 0; i < n; ++i) cfa[i] = cfaIn[i] > black ? (uint16_t)(cfaIn[i] - black) : 0;
    /* White balance, truncating (BayerDemosaic_Scalar.cpp:24-35). */
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
        {
            size_t i = (size_t)y * w + x;
            float val = (float)cfa[i] * camMul[bayer_color(y, x, filters)];
            cfa[i] = clamp_trunc_u16(val);
        }
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
        {
            /* DemosaicPixel (BayerDemosaicKernels.h:25-60). */
            float rgb[3] = {0.0f, 0.0f, 0.0f};
            int counts[3] = {0, 0, 0};
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    int nx = x + dx, ny = y + dy;
                    if (nx < 0 || ny < 0 || nx >= w || ny >= h) continue;
                    int ch = bayer_color(ny, nx, filters);
                    int slot = ch == 3 ? 1 : ch;
                    rgb[slot] += (float)cfa[(size_t)ny * w + nx];
                    counts[slot]++;
                }
            int mine = bayer_color(y, x, filters);
            int mySlot = mine == 3 ? 1 : mine;
            for (int c = 0; c < 3; ++c)
            {
                if (c == mySlot || counts[c] == 0) continue;
                rgb[c] /= (float)counts[c];
            }
            rgb[mySlot] = (float)cfa[(size_t)y * w + x];
            uint16_t px[3];
            for (int c = 0; c < 3; ++c) px[c] = clamp_trunc_u16(rgb[c]);
            /* ApplyColorMatrixPixel (BayerDemosaicKernels.h:64-75). */
            float r = (float)px[0], g = (float)px[1], b = (float)px[2];
            uint16_t* o = out + ((size_t)y * w + x) * 3;
            for (int row = 0; row < 3; ++row)
            {
                const float* m = rgbCam + row * 4;
                float val = m[0] * r + m[1] * g + m[2] * b + m[3];
                o[row] = clamp_trunc_u16(val);
            }
        }
    free(cfa);
}

void or_demosaic_f64(const uint16_t* cfaIn, int w, int h, uint16_t black, const float* camMul,
                     const float* rgbCam, uint32_t filters, uint16_t* out)
{
    size_t n = (size_t)w * h;
    uint16_t* cfa = (uint16_t*)malloc(n * sizeof(uint16_t));
    for (size_t i = 0; i < n; ++i) cfa[i] = cfaIn[i] > black ? (uint16_t)(cfaIn[i] - black) : 0;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
        {
            size_t i = (size_t)y * w + x;
            cfa[i] = clamp_trunc_u16_d((double)cfa[i] * (double)camMul[bayer_color(y, x, filters)]);
        }
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
        {
            double rgb[3] = {0, 0, 0};
            int counts[3] = {0, 0, 0};
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    int nx = x + dx, ny = y + dy;
                    if (nx < 0 || ny < 0 || nx >= w || ny >= h) continue;
                    int ch = bayer_color(ny, nx, filters);
                    int slot = ch == 3 ? 1 : ch;
                    rgb[slot] += (double)cfa[(size_t)ny * w + nx];
                    counts[slot]++;
                }
            int mine = bayer_color(y, x, filters);
            int mySlot = mine == 3 ? 1 : mine;
            for (int c = 0; c < 3; ++c)
                if (c != mySlot && counts[c] != 0) rgb[c] /= (double)counts[c];
            rgb[mySlot] = (double)cfa[(size_t)y * w + x];
            uint16_t px[3];
            for (int c = 0; c < 3; ++c) px[c] = clamp_trunc_u16_d(rgb[c]);
            uint16_t* o = out + ((size_t)y * w + x) * 3;
            for (int row = 0; row < 3; ++row)
            {
                const float* m = rgbCam + row * 4;
                o[row] = clamp_trunc_u16_d((double)m[0] * px[0] + (double)m[1] * px[1] + (double)m[2] * px[2] + (double)m[3]);
            }
        }
    free(cfa);
}

/* ------------------------------------------------------------------------ */
/* Warp: WarpPerspective_Scalar.cpp:8-45, WarpPerspectiveKernels.h:16-43.     */
/* ------------------------------------------------------------------------ */

void or_warp(const uint16_t* src, int sw, int sh, uint16_t* dst, int dw, int dh, const float* H,
             int offX, int offY)
{
    for (int y = 0; y < dh; ++y)
    {
        float dstY = (float)(y + offY);
        for (int x = 0; x < dw; ++x)
        {
            float dstX = (float)(x + offX);
            float srcX = H[0] * dstX + H[1] * dstY + H[2];
            float srcY = H[3] * dstX + H[4] * dstY + H[5];
            float srcW1 = H[6] * dstX + H[7] * dstY + H[8];
            uint16_t* o = dst + ((size_t)y * dw + x) * 3;
            if (fabsf(srcW1) < 1e-10f) { o[0] = o[1] = o[2] = 0; continue; }
            srcX /= srcW1;
            srcY /= srcW1;
            /* valid iff floor(sx) >= 0 && floor(sx)+1 < sw (and the same in y);
             * stated on the float so NaN and out-of-int-range coordinates are
             * invalid, as the reference's int conversion makes them. */
            if (!(srcX >= 0.0f && srcX < (float)(sw - 1) && srcY >= 0.0f && srcY < (float)(sh - 1)))
            {
                o[0] = o[1] = o[2] = 0;
                continue;
            }
            int sx0 = (int)floorf(srcX), sy0 = (int)floorf(srcY);
            float fx = srcX - (float)sx0, fy = srcY - (float)sy0;
            float w00 = (1.0f - fx) * (1.0f - fy);
            float w10 = fx * (1.0f - fy);
            float w01 = (1.0f - fx) * fy;
            float w11 = fx * fy;
            const uint16_t* r0 = src + ((size_t)sy0 * sw + sx0) * 3;
            const uint16_t* r1 = r0 + (size_t)sw * 3;
            for (int c = 0; c < 3; ++c)
            {
                float val = w00 * (float)r0[c] + w10 * (float)r0[3 + c] + w01 * (float)r1[c] + w11 * (float)r1[3 + c];
                o[c] = clamp_trunc_u16(val);
            }
        }
    }
}

void or_warp_f64(const uint16_t* src, int sw, int sh, uint16_t* dst, int dw, int dh, const double* H,
                 int offX, int offY)
{
    for (int y = 0; y < dh; ++y)
        for (int x = 0; x < dw; ++x)
        {
            double dX = (double)x + offX, dY = (double)y + offY;
            double sx = H[0] * dX + H[1] * dY + H[2];
            double sy = H[3] * dX + H[4] * dY + H[5];
            double sw1 = H[6] * dX + H[7] * dY + H[8];
            uint16_t* o = dst + ((size_t)y * dw + x) * 3;
            if (fabs(sw1) < 1e-10) { o[0] = o[1] = o[2] = 0; continue; }
            sx /= sw1;
            sy /= sw1;
            if (!(sx >= 0.0 && sx < (double)(sw - 1) && sy >= 0.0 && sy < (double)(sh - 1)))
            {
                o[0] = o[1] = o[2] = 0;
                continue;
            }
            int sx0 = (int)floor(sx), sy0 = (int)floor(sy);
            double fx = sx - sx0, fy = sy - sy0;
            const uint16_t* r0 = src + ((size_t)sy0 * sw + sx0) * 3;
            const uint16_t* r1 = r0 + (size_t)sw * 3;
            for (int c = 0; c < 3; ++c)
            {
                double val = (1 - fx) * (1 - fy) * r0[c] + fx * (1 - fy) * r0[3 + c] + (1 - fx) * fy * r1[c] + fx * fy * r1[3 + c];
                o[c] = clamp_trunc_u16_d(val);
            }
        }
}

/* ------------------------------------------------------------------------ */
/* Median stack: MedianStack_Scalar.cpp:8-24, MedianStackKernels.h:19-55.    */
/* ------------------------------------------------------------------------ */

static int cmp_u16(const void* a, const void* b)
{
    return (int)*(const uint16_t*)a - (int)*(const uint16_t*)b;
}

void or_median(const uint16_t* const* inputs, int n, uint16_t* out, int w, int h, float sigma)
{
    int count0 = n < 32 ? n : 32;
    long long total = (long long)w * h * 3;
    uint16_t values[32];
    for (long long idx = 0; idx < total; ++idx)
    {
        int count = count0;
        for (int i = 0; i < count; ++i) values[i] = inputs[i][idx];
        if (count > 3)
        {
            float sum = 0.0f, sumSq = 0.0f;
            for (int i = 0; i < count; ++i)
            {
                float v = (float)values[i];
                sum += v;
                sumSq += v * v;
            }
            float mean = sum / (float)count;
            float variance = sumSq / (float)count - mean * mean;
            float sd = sqrtf(variance > 0.0f ? variance : 0.0f);
            float lower = mean - sigma * sd;
            float upper = mean + sigma * sd;
            int valid = 0;
            for (int i = 0; i < count; ++i)
            {
                float v = (float)values[i];
                if (v >= lower && v <= upper) values[valid++] = values[i];
            }
            if (valid > 0) count = valid;
        }
        qsort(values, (size_t)count, sizeof(uint16_t), cmp_u16);
        out[idx] = values[count / 2];
    }
}

/* ------------------------------------------------------------------------ */
/* Gain (GainColorOps.cpp:16-26) and homography inverse (HomographyMath.cpp). */
/* ------------------------------------------------------------------------ */

void or_gain(uint16_t* data, int n, float gain)
{
    if (!data || n <= 0) return;
    if (fabsf(gain - 1.0f) < 1e-6f) return;
    for (int i = 0; i < n; ++i) data[i] = clamp_trunc_u16((float)data[i] * gain);
}

/* ------------------------------------------------------------------------ */
/* Lab statistics and Reinhard colour transfer: GainColorOps.cpp:28-156.      */
/* FP32 per pixel, FP64 sums and transfer; libm powf/cbrtf as the reference.  */
/* ------------------------------------------------------------------------ */
#define LAB_DELTA (6.0f / 29.0f)

static float lab_decode(float c) /* GainColorOps.cpp:30-33 */
{
    if (c <= 0.04045f) return c / 12.92f;
    return powf((c + 0.055f) / 1.055f, 2.4f);
}

static float lab_encode(float c) /* GainColorOps.cpp:35-38 */
{
    if (c <= 0.0031308f) return c * 12.92f;
    return 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
}

static float lab_fwd(float t) /* GainColorOps.cpp:40-44 */
{
    const float d = LAB_DELTA;
    if (t > d * d * d) return cbrtf(t);
    return t / (3.0f * d * d) + 4.0f / 29.0f;
}

static float lab_inv(float t) /* GainColorOps.cpp:46-50 */
{
    const float d = LAB_DELTA;
    if (t > d) return t * t * t;
    return 3.0f * d * d * (t - 4.0f / 29.0f);
}

static void lab_of_pixel(const uint16_t* px, float* lab) /* GainColorOps.cpp:56-73 */
{
    float r = lab_decode(px[0] / 65535.0f);
    float g = lab_decode(px[1] / 65535.0f);
    float b = lab_decode(px[2] / 65535.0f);
    float X = 0.4124564f * r + 0.3575761f * g + 0.1804375f * b;
    float Y = 0.2126729f * r + 0.7151522f * g + 0.0721750f * b;
    float Z = 0.0193339f * r + 0.1191920f * g + 0.9503041f * b;
    float fx = lab_fwd(X / 0.95047f);
    float fy = lab_fwd(Y / 1.0f);
    float fz = lab_fwd(Z / 1.08883f);
    lab[0] = 116.0f * fy - 16.0f;
    lab[1] = 500.0f * (fx - fy);
    lab[2] = 200.0f * (fy - fz);
}

static void pixel_of_lab(const float* lab, uint16_t* px) /* GainColorOps.cpp:75-100 */
{
    float fy = (lab[0] + 16.0f) / 116.0f;
    float fx = fy + lab[1] / 500.0f;
    float fz = fy - lab[2] / 200.0f;
    float X = 0.95047f * lab_inv(fx);
    float Y = 1.0f * lab_inv(fy);
    float Z = 1.08883f * lab_inv(fz);
    float lin[3];
    lin[0] = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
    lin[1] = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
    lin[2] = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
    for (int c = 0; c < 3; ++c)
    {
        float v = lin[c] < 0.0f ? 0.0f : lin[c]; /* a NaN stays NaN, as (std::max)(v, 0.0f) */
        px[c] = clamp_trunc_u16(lab_encode(v) * 65535.0f);
    }
}

void or_lab_stats(const uint16_t* rgb, int w, int h, double* mean3, double* std3)
{
    if (!rgb || !mean3 || !std3 || w <= 0 || h <= 0) return;
    const long long n = (long long)w * h;
    double sum[3] = {0.0, 0.0, 0.0}, sq[3] = {0.0, 0.0, 0.0};
    for (long long i = 0; i < n; ++i)
    {
        float lab[3];
        lab_of_pixel(rgb + i * 3, lab);
        for (int c = 0; c < 3; ++c)
        {
            double v = (double)lab[c];
            sum[c] += v;
            sq[c] += v * v;
        }
    }
    for (int c = 0; c < 3; ++c)
    {
        double m = sum[c] / (double)n;
        double var = sq[c] / (double)n - m * m;
        mean3[c] = m;
        std3[c] = sqrt(var > 0.0 ? var : 0.0);
    }
}

void or_reinhard(uint16_t* rgb, int w, int h, const double* srcMean, const double* srcStd,
                 const double* refMean, const double* refStd)
{
    if (!rgb || !srcMean || !srcStd || !refMean || !refStd || w <= 0 || h <= 0) return;
    const long long n = (long long)w * h;
    for (long long i = 0; i < n; ++i)
    {
        uint16_t* px = rgb + i * 3;
        float lab[3];
        lab_of_pixel(px, lab);
        for (int c = 0; c < 3; ++c)
        {
            double s = srcStd[c] > 1e-6 ? srcStd[c] : 1.0;
            lab[c] = (float)(((double)lab[c] - srcMean[c]) * (refStd[c] / s) + refMean[c]);
        }
        pixel_of_lab(lab, px);
    }
}

/* FP64 restatement of the same conversions (exact powers and cube roots in
 * double), quantised only at the RGB48 output, for error reporting. */
static double lab_fwd_d(double t)
{
    const double d = 6.0 / 29.0;
    return t > d * d * d ? cbrt(t) : t / (3.0 * d * d) + 4.0 / 29.0;
}

static double lab_inv_d(double t)
{
    const double d = 6.0 / 29.0;
    return t > d ? t * t * t : 3.0 * d * d * (t - 4.0 / 29.0);
}

static void lab_of_pixel_d(const uint16_t* px, double* lab)
{
    double lin[3];
    for (int c = 0; c < 3; ++c)
    {
        double v = px[c] / 65535.0;
        lin[c] = v <= 0.04045 ? v / 12.92 : pow((v + 0.055) / 1.055, 2.4);
    }
    double X = 0.4124564 * lin[0] + 0.3575761 * lin[1] + 0.1804375 * lin[2];
    double Y = 0.2126729 * lin[0] + 0.7151522 * lin[1] + 0.0721750 * lin[2];
    double Z = 0.0193339 * lin[0] + 0.1191920 * lin[1] + 0.9503041 * lin[2];
    double fx = lab_fwd_d(X / 0.95047), fy = lab_fwd_d(Y), fz = lab_fwd_d(Z / 1.08883);
    lab[0] = 116.0 * fy - 16.0;
    lab[1] = 500.0 * (fx - fy);
    lab[2] = 200.0 * (fy - fz);
}

void or_lab_stats_f64(const uint16_t* rgb, int w, int h, double* mean3, double* std3)
{
    if (!rgb || !mean3 || !std3 || w <= 0 || h <= 0) return;
    const long long n = (long long)w * h;
    double sum[3] = {0.0, 0.0, 0.0}, sq[3] = {0.0, 0.0, 0.0};
    for (long long i = 0; i < n; ++i)
    {
        double lab[3];
        lab_of_pixel_d(rgb + i * 3, lab);
        for (int c = 0; c < 3; ++c)
        {
            sum[c] += lab[c];
            sq[c] += lab[c] * lab[c];
        }
    }
    for (int c = 0; c < 3; ++c)
    {
        double m = sum[c] / (double)n;
        double var = sq[c] / (double)n - m * m;
        mean3[c] = m;
        std3[c] = sqrt(var > 0.0 ? var : 0.0);
    }
}

void or_reinhard_f64(uint16_t* rgb, int w, int h, const double* srcMean, const double* srcStd,
                     const double* refMean, const double* refStd)
{
    if (!rgb || !srcMean || !srcStd || !refMean || !refStd || w <= 0 || h <= 0) return;
    const long long n = (long long)w * h;
    for (long long i = 0; i < n; ++i)
    {
        uint16_t* px = rgb + i * 3;
        double lab[3];
        lab_of_pixel_d(px, lab);
        for (int c = 0; c < 3; ++c)
        {
            double s = srcStd[c] > 1e-6 ? srcStd[c] : 1.0;
            lab[c] = (lab[c] - srcMean[c]) * (refStd[c] / s) + refMean[c];
        }
        double fy = (lab[0] + 16.0) / 116.0, fx = fy + lab[1] / 500.0, fz = fy - lab[2] / 200.0;
        double X = 0.95047 * lab_inv_d(fx), Y = lab_inv_d(fy), Z = 1.08883 * lab_inv_d(fz);
        double lin[3] = {3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z,
                         -0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z,
                         0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z};
        for (int c = 0; c < 3; ++c)
        {
            double v = lin[c] < 0.0 ? 0.0 : lin[c];
            double e = v <= 0.0031308 ? v * 12.92 : 1.055 * pow(v, 1.0 / 2.4) - 0.055;
            px[c] = clamp_trunc_u16_d(e * 65535.0);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Overlap culling: OverlapCulling.cpp:36-71.                                 */
/* ------------------------------------------------------------------------ */
int or_image_overlaps_chunk(const float* m, int imageW, int imageH, int chunkX, int chunkY, int chunkW, int chunkH)
{
    const float cx[4] = {0.0f, (float)imageW, 0.0f, (float)imageW};
    const float cy[4] = {0.0f, 0.0f, (float)imageH, (float)imageH};
    float minX = FLT_MAX, minY = FLT_MAX, maxX = -FLT_MAX, maxY = -FLT_MAX;
    for (int k = 0; k < 4; ++k)
    {
        float den = m[6] * cx[k] + m[7] * cy[k] + m[8];
        if (fabsf(den) < 1e-10f) den = den >= 0.0f ? 1e-10f : -1e-10f;
        float px = (m[0] * cx[k] + m[1] * cy[k] + m[2]) / den;
        float py = (m[3] * cx[k] + m[4] * cy[k] + m[5]) / den;
        if (px < minX) minX = px;
        if (py < minY) minY = py;
        if (maxX < px) maxX = px;
        if (maxY < py) maxY = py;
    }
    float x0 = (float)chunkX, y0 = (float)chunkY;
    float x1 = x0 + (float)chunkW, y1 = y0 + (float)chunkH;
    return minX < x1 && maxX > x0 && minY < y1 && maxY > y0;
}

int or_image_overlaps_chunk_f64(const float* m, int imageW, int imageH, int chunkX, int chunkY, int chunkW,
                                int chunkH)
{
    const double cx[4] = {0.0, (double)imageW, 0.0, (double)imageW};
    const double cy[4] = {0.0, 0.0, (double)imageH, (double)imageH};
    double minX = DBL_MAX, minY = DBL_MAX, maxX = -DBL_MAX, maxY = -DBL_MAX;
    for (int k = 0; k < 4; ++k)
    {
        double den = (double)m[6] * cx[k] + (double)m[7] * cy[k] + (double)m[8];
        if (fabs(den) < 1e-10) den = den >= 0.0 ? 1e-10 : -1e-10;
        double px = ((double)m[0] * cx[k] + (double)m[1] * cy[k] + (double)m[2]) / den;
        double py = ((double)m[3] * cx[k] + (double)m[4] * cy[k] + (double)m[5]) / den;
        if (px < minX) minX = px;
        if (py < minY) minY = py;
        if (maxX < px) maxX = px;
        if (maxY < py) maxY = py;
    }
    double x1 = (double)chunkX + (double)chunkW, y1 = (double)chunkY + (double)chunkH;
    return minX < x1 && maxX > (double)chunkX && minY < y1 && maxY > (double)chunkY;
}

/* ------------------------------------------------------------------------ */
/* Export: PanoramaExporter.cpp:9-102, StorageEngine.cpp:130-144,             */
/* Tiff16Writer.cpp:40-97.                                                    */
/* ------------------------------------------------------------------------ */
float or_export_scale(int totalW, int totalH, int maxDimension)
{
    int longest = totalW > totalH ? totalW : totalH;
    if (longest <= 0) return 1.0f;
    return (float)maxDimension / (float)longest;
}

void or_chunk_placement(int x, int y, int w, int h, float scale, int* out4)
{
    int dw = (int)((float)w * scale), dh = (int)((float)h * scale);
    out4[0] = (int)((float)x * scale);
    out4[1] = (int)((float)y * scale);
    out4[2] = dw > 1 ? dw : 1;
    out4[3] = dh > 1 ? dh : 1;
}

int or_export_preview(const uint16_t* const* tiles, const int32_t* rects, int numTiles, int totalW, int totalH,
                      int maxDimension, uint8_t* out, long long capacity, int* outW, int* outH)
{
    if (maxDimension <= 0 || totalW <= 0 || totalH <= 0) return 0;
    float scale = or_export_scale(totalW, totalH, maxDimension);
    int ow = (int)((float)totalW * scale), oh = (int)((float)totalH * scale);
    ow = ow > 1 ? ow : 1;
    oh = oh > 1 ? oh : 1;
    if ((long long)ow * oh * 3 > capacity) return 0;
    memset(out, 0, (size_t)ow * oh * 3);
    for (int c = 0; c < numTiles; ++c)
    {
        const uint16_t* src = tiles[c];
        if (!src) continue;
        const int32_t* r = rects + 4 * c;
        int p[4];
        or_chunk_placement(r[0], r[1], r[2], r[3], scale, p);
        for (int dy = 0; dy < p[3]; ++dy)
        {
            int oy = p[1] + dy;
            if (oy < 0 || oy >= oh) continue;
            for (int dx = 0; dx < p[2]; ++dx)
            {
                int ox = p[0] + dx;
                if (ox < 0 || ox >= ow) continue;
                int sx = (int)((float)dx / scale), sy = (int)((float)dy / scale);
                if (sx < 0 || sx >= r[2] || sy < 0 || sy >= r[3]) continue;
                const uint16_t* s = src + ((size_t)sy * r[2] + sx) * 3;
                uint8_t* d = out + ((size_t)oy * ow + ox) * 3;
                d[0] = (uint8_t)(s[0] >> 8);
                d[1] = (uint8_t)(s[1] >> 8);
                d[2] = (uint8_t)(s[2] >> 8);
            }
        }
    }
    *outW = ow;
    *outH = oh;
    return 1;
}

static void put_u16(uint8_t* p, uint16_t v)
{
    p[0] = (uint8_t)(v & 0xff);
    p[1] = (uint8_t)(v >> 8);
}

static void put_u32(uint8_t* p, uint32_t v)
{
    for (int i = 0; i < 4; ++i) p[i] = (uint8_t)(v >> (8 * i));
}

void or_frame_pixel_buffer(const uint16_t* data, int w, int h, uint8_t* out)
{
    put_u32(out, (uint32_t)w);
    put_u32(out + 4, (uint32_t)h);
    memcpy(out + 8, data, (size_t)w * h * 6);
}

long long or_tiff16_size(int w, int h)
{
    return 8 + (long long)w * h * 6 + 6 + 8 + 8 + 2 + 12 * 12 + 4;
}

void or_tiff16_bytes(const uint16_t* data, int w, int h, uint8_t* out)
{
    const uint32_t pix = (uint32_t)((size_t)w * h * 6);
    const uint32_t bps = 8 + pix, xres = bps + 6, yres = xres + 8, ifd = yres + 8;
    out[0] = 'I';
    out[1] = 'I';
    put_u16(out + 2, 42);
    put_u32(out + 4, ifd);
    memcpy(out + 8, data, pix);
    uint8_t* p = out + bps;
    put_u16(p, 16), put_u16(p + 2, 16), put_u16(p + 4, 16);
    put_u32(p + 6, 72), put_u32(p + 10, 1), put_u32(p + 14, 72), put_u32(p + 18, 1);
    p = out + ifd;
    put_u16(p, 12);
    const uint32_t e[12][4] = {{256, 4, 1, (uint32_t)w}, {257, 4, 1, (uint32_t)h}, {258, 3, 3, bps},
                               {259, 3, 1, 1},          {262, 3, 1, 2},          {273, 4, 1, 8},
                               {277, 3, 1, 3},          {278, 4, 1, (uint32_t)h}, {279, 4, 1, pix},
                               {282, 5, 1, xres},       {283, 5, 1, yres},       {296, 3, 1, 2}};
    for (int i = 0; i < 12; ++i)
    {
        uint8_t* q = p + 2 + 12 * i;
        put_u16(q, (uint16_t)e[i][0]);
        put_u16(q + 2, (uint16_t)e[i][1]);
        put_u32(q + 4, e[i][2]);
        put_u32(q + 8, e[i][3]);
    }
    put_u32(p + 2 + 12 * 12, 0);
}

int or_invert_h(const float* m, float* out)
{
    if (!m || !out) return 0;
    float a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], i2 = m[7], j = m[8];
    float det = a * (e * j - f * i2) - b * (d * j - f * g) + c * (d * i2 - e * g);
    if (fabsf(det) < 1e-12f) return 0;
    float inv = 1.0f / det;
    out[0] = (e * j - f * i2) * inv;
    out[1] = (c * i2 - b * j) * inv;
    out[2] = (b * f - c * e) * inv;
    out[3] = (f * g - d * j) * inv;
    out[4] = (a * j - c * g) * inv;
    out[5] = (c * d - a * f) * inv;
    out[6] = (d * i2 - e * g) * inv;
    out[7] = (b * g - a * i2) * inv;
    out[8] = (a * e - b * d) * inv;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Seam blend: SeamBlend.cpp.                                                */
/* ------------------------------------------------------------------------ */

void or_coverage(const uint16_t* img, int w, int h, uint8_t* cov)
{
    size_t n = (size_t)w * h;
    for (size_t p = 0; p < n; ++p) cov[p] = (img[p * 3] | img[p * 3 + 1] | img[p * 3 + 2]) != 0;
}

static inline float fminf_keep(float a, float b) { return b < a ? b : a; }

void or_coverage_distance(const uint8_t* cov, int w, int h, float* d)
{
    /* SeamBlend.cpp:206-242: two-pass 3x3 chamfer, kInf = w + h. */
    const float kDiag = 1.41421356f;
    const float kInf = (float)(w + h);
    size_t n = (size_t)w * h;
    for (size_t p = 0; p < n; ++p) d[p] = cov[p] ? kInf : 0.0f;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
        {
            size_t p = (size_t)y * w + x;
            float best = d[p];
            if (x > 0) best = fminf_keep(best, d[p - 1] + 1.0f);
            if (y > 0) best = fminf_keep(best, d[p - w] + 1.0f);
            if (x > 0 && y > 0) best = fminf_keep(best, d[p - w - 1] + kDiag);
            if (x < w - 1 && y > 0) best = fminf_keep(best, d[p - w + 1] + kDiag);
            d[p] = best;
        }
    for (int y = h - 1; y >= 0; --y)
        for (int x = w - 1; x >= 0; --x)
        {
            size_t p = (size_t)y * w + x;
            float best = d[p];
            if (x < w - 1) best = fminf_keep(best, d[p + 1] + 1.0f);
            if (y < h - 1) best = fminf_keep(best, d[p + w] + 1.0f);
            if (x < w - 1 && y < h - 1) best = fminf_keep(best, d[p + w + 1] + kDiag);
            if (x > 0 && y < h - 1) best = fminf_keep(best, d[p + w - 1] + kDiag);
            d[p] = best;
        }
}

void or_ownership(const float* const* dists, int k, int w, int h, int32_t* owner)
{
    /* SeamBlend.cpp:244-261: strict '>' so ties keep the lowest index. */
    size_t n = (size_t)w * h;
    for (size_t p = 0; p < n; ++p)
    {
        int best = -1;
        float bestD = 0.0f;
        for (int i = 0; i < k; ++i)
        {
            float v = dists[i][p];
            if (v > bestD) { bestD = v; best = i; }
        }
        owner[p] = best;
    }
}

int or_bbox(const uint8_t* cov, int w, int h, int32_t* box)
{
    /* SeamBlend.cpp:263-280. */
    int valid = 0;
    box[0] = 0; box[1] = 0; box[2] = -1; box[3] = -1;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
        {
            if (!cov[(size_t)y * w + x]) continue;
            if (!valid) { box[0] = box[2] = x; box[1] = box[3] = y; valid = 1; }
            else
            {
                if (x < box[0]) box[0] = x;
                if (x > box[2]) box[2] = x;
                if (y < box[1]) box[1] = y;
                if (y > box[3]) box[3] = y;
            }
        }
    return valid;
}

static int intersect_bbox(const int32_t* a, int va, const int32_t* b, int vb, int32_t* o)
{
    /* SeamBlend.cpp:282-291. */
    if (!va || !vb) { o[0] = 0; o[1] = 0; o[2] = -1; o[3] = -1; return 0; }
    o[0] = a[0] > b[0] ? a[0] : b[0];
    o[1] = a[1] > b[1] ? a[1] : b[1];
    o[2] = a[2] < b[2] ? a[2] : b[2];
    o[3] = a[3] < b[3] ? a[3] : b[3];
    return o[0] <= o[2] && o[1] <= o[3];
}

void or_refine_seam(const uint16_t* imgI, const uint16_t* imgJ, const float* distI, const float* distJ,
                    int width, int height, int ci, int cj, const int32_t* boxI, const int32_t* boxJ,
                    const int32_t* ov, int32_t* owner)
{
    /* SeamBlend.cpp:293-445. */
    (void)height;
    int bw = ov[2] - ov[0] + 1, bh = ov[3] - ov[1] + 1;
    int rowScan = bw >= bh;
    float centerI = rowScan ? (float)(boxI[0] + boxI[2]) * 0.5f : (float)(boxI[1] + boxI[3]) * 0.5f;
    float centerJ = rowScan ? (float)(boxJ[0] + boxJ[2]) * 0.5f : (float)(boxJ[1] + boxJ[3]) * 0.5f;
    int iLow = centerI <= centerJ;
    const float kSmooth = 2.0f;
    const int kRadius = 24;
    int numLines = rowScan ? bh : bw;
    int lineLen = rowScan ? bw : bh;
    int* lo = (int*)malloc(sizeof(int) * (size_t)numLines);
    int* hi = (int*)malloc(sizeof(int) * (size_t)numLines);
    for (int l = 0; l < numLines; ++l) { lo[l] = 1; hi[l] = 0; }
#define PIX(line, t) (rowScan ? ((size_t)(ov[1] + (line)) * width + (size_t)(ov[0] + (t))) \
                              : ((size_t)(ov[1] + (t)) * width + (size_t)(ov[0] + (line))))
    for (int line = 0; line < numLines; ++line)
    {
        int cross = -1, first = -1;
        for (int t = 0; t < lineLen; ++t)
        {
            int o = owner[PIX(line, t)];
            if (o != ci && o != cj) continue;
            if (first < 0) { first = o; continue; }
            if (o != first) { cross = t; break; }
        }
        if (cross < 0) continue;
        int bLo = cross - kRadius < 0 ? 0 : cross - kRadius;
        int bHi = cross + kRadius > lineLen - 1 ? lineLen - 1 : cross + kRadius;
        for (int t = bLo; t <= bHi; ++t)
        {
            size_t p = PIX(line, t);
            if (distI[p] > 0.0f && distJ[p] > 0.0f)
            {
                if (hi[line] < lo[line]) { lo[line] = t; hi[line] = t; }
                else
                {
                    if (t < lo[line]) lo[line] = t;
                    if (t > hi[line]) hi[line] = t;
                }
            }
        }
    }
    /* dp / back stored per line with a fixed stride (lineWidth <= 49). */
    const int S = 2 * kRadius + 1;
    float* dp = (float*)malloc(sizeof(float) * (size_t)numLines * S);
    int* back = (int*)malloc(sizeof(int) * (size_t)numLines * S);
    int* prevLine = (int*)malloc(sizeof(int) * (size_t)numLines);
    int last = -1;
    for (int line = 0; line < numLines; ++line)
    {
        prevLine[line] = -1;
        if (hi[line] < lo[line]) continue;
        int lw = hi[line] - lo[line] + 1;
        for (int k = 0; k < lw; ++k)
        {
            int t = lo[line] + k;
            size_t p = PIX(line, t);
            float cost = 0.0f;
            for (int c = 0; c < 3; ++c) cost += fabsf((float)imgI[p * 3 + c] - (float)imgJ[p * 3 + c]);
            if (last < 0)
            {
                dp[(size_t)line * S + k] = cost;
                back[(size_t)line * S + k] = -1;
            }
            else
            {
                float best = 3.402823466e+38f;
                int bestPrev = -1;
                int pLo = lo[last], pW = hi[last] - lo[last] + 1;
                for (int pk = 0; pk < pW; ++pk)
                {
                    int pt = pLo + pk;
                    float c2 = dp[(size_t)last * S + pk] + kSmooth * fabsf((float)(t - pt));
                    if (c2 < best) { best = c2; bestPrev = pk; }
                }
                dp[(size_t)line * S + k] = cost + best;
                back[(size_t)line * S + k] = bestPrev;
            }
        }
        prevLine[line] = last;
        last = line;
    }
    if (last >= 0)
    {
        int* chosen = (int*)malloc(sizeof(int) * (size_t)numLines);
        for (int l = 0; l < numLines; ++l) chosen[l] = -1;
        int line = last, bestK = 0;
        {
            float best = 3.402823466e+38f;
            int lw = hi[line] - lo[line] + 1;
            for (int k = 0; k < lw; ++k)
                if (dp[(size_t)line * S + k] < best) { best = dp[(size_t)line * S + k]; bestK = k; }
        }
        while (line >= 0)
        {
            chosen[line] = lo[line] + bestK;
            int pl = prevLine[line];
            int pk = back[(size_t)line * S + bestK];
            line = pl;
            bestK = pk;
        }
        for (int l = 0; l < numLines; ++l)
        {
            if (chosen[l] < 0) continue;
            for (int t = lo[l]; t <= hi[l]; ++t)
            {
                size_t p = PIX(l, t);
                if (owner[p] != ci && owner[p] != cj) continue;
                int onLow = t < chosen[l];
                owner[p] = (onLow == iLow) ? ci : cj;
            }
        }
        free(chosen);
    }
#undef PIX
    free(lo); free(hi); free(dp); free(back); free(prevLine);
}

/* --- pyramid helpers (SeamBlend.cpp:15-201), generic over float/double --- */

#define DEFINE_PYR(T, SUF)                                                                           \
static void blur5_##SUF(const T* src, int w, int h, int ch, T* dst, T* tmp)                          \
{                                                                                                    \
    const T k0 = (T)1 / (T)16, k1 = (T)4 / (T)16, k2 = (T)6 / (T)16;                                 \
    for (int y = 0; y < h; ++y)                                                                      \
        for (int x = 0; x < w; ++x)                                                                  \
        {                                                                                            \
            int xm2 = x - 2 < 0 ? 0 : x - 2, xm1 = x - 1 < 0 ? 0 : x - 1;                            \
            int xp1 = x + 1 > w - 1 ? w - 1 : x + 1, xp2 = x + 2 > w - 1 ? w - 1 : x + 2;            \
            const T* r = src + (size_t)y * w * ch;                                                   \
            for (int c = 0; c < ch; ++c)                                                             \
                tmp[((size_t)y * w + x) * ch + c] = k0 * r[xm2 * ch + c] + k1 * r[xm1 * ch + c] +    \
                    k2 * r[x * ch + c] + k1 * r[xp1 * ch + c] + k0 * r[xp2 * ch + c];                \
        }                                                                                            \
    for (int y = 0; y < h; ++y)                                                                      \
    {                                                                                                \
        int ym2 = y - 2 < 0 ? 0 : y - 2, ym1 = y - 1 < 0 ? 0 : y - 1;                                \
        int yp1 = y + 1 > h - 1 ? h - 1 : y + 1, yp2 = y + 2 > h - 1 ? h - 1 : y + 2;                \
        for (int x = 0; x < w; ++x)                                                                  \
            for (int c = 0; c < ch; ++c)                                                             \
            {                                                                                        \
                size_t o = (size_t)x * ch + c;                                                       \
                size_t rs = (size_t)w * ch;                                                          \
                dst[(size_t)y * rs + o] = k0 * tmp[(size_t)ym2 * rs + o] + k1 * tmp[(size_t)ym1 * rs + o] + \
                    k2 * tmp[(size_t)y * rs + o] + k1 * tmp[(size_t)yp1 * rs + o] + k0 * tmp[(size_t)yp2 * rs + o]; \
            }                                                                                        \
    }                                                                                                \
}                                                                                                    \
/* Blur then pick (min(2x,w-1), min(2y,h-1)) (SeamBlend.cpp:60-79). */                               \
static T* down2_##SUF(const T* src, int w, int h, int ch, int* ow, int* oh)                          \
{                                                                                                    \
    size_t n = (size_t)w * h * ch;                                                                   \
    T* bl = (T*)malloc(n * sizeof(T));                                                               \
    T* tmp = (T*)malloc(n * sizeof(T));                                                              \
    blur5_##SUF(src, w, h, ch, bl, tmp);                                                             \
    free(tmp);                                                                                       \
    *ow = (w + 1) / 2;                                                                               \
    *oh = (h + 1) / 2;                                                                               \
    T* dst = (T*)malloc((size_t)(*ow) * (*oh) * ch * sizeof(T));                                     \
    for (int y = 0; y < *oh; ++y)                                                                    \
    {                                                                                                \
        int sy = 2 * y < h - 1 ? 2 * y : h - 1;                                                      \
        for (int x = 0; x < *ow; ++x)                                                                \
        {                                                                                            \
            int sx = 2 * x < w - 1 ? 2 * x : w - 1;                                                  \
            for (int c = 0; c < ch; ++c)                                                             \
                dst[((size_t)y * (*ow) + x) * ch + c] = bl[((size_t)sy * w + sx) * ch + c];          \
        }                                                                                            \
    }                                                                                                \
    free(bl);                                                                                        \
    return dst;                                                                                      \
}                                                                                                    \
/* Align-corners bilinear resize (SeamBlend.cpp:85-115). */                                          \
static void up_##SUF(const T* src, int w, int h, int ch, int ow, int oh, T* dst)                     \
{                                                                                                    \
    T sx = (w > 1) ? (T)(w - 1) / (T)(ow - 1 > 1 ? ow - 1 : 1) : (T)0;                               \
    T sy = (h > 1) ? (T)(h - 1) / (T)(oh - 1 > 1 ? oh - 1 : 1) : (T)0;                               \
    for (int y = 0; y < oh; ++y)                                                                     \
    {                                                                                                \
        T fy = sy * (T)y;                                                                            \
        int y0 = (int)fy < h - 1 ? (int)fy : h - 1;                                                  \
        int y1 = y0 + 1 < h - 1 ? y0 + 1 : h - 1;                                                    \
        T wy = fy - (T)y0;                                                                           \
        for (int x = 0; x < ow; ++x)                                                                 \
        {                                                                                            \
            T fx = sx * (T)x;                                                                        \
            int x0 = (int)fx < w - 1 ? (int)fx : w - 1;                                              \
            int x1 = x0 + 1 < w - 1 ? x0 + 1 : w - 1;                                                \
            T wx = fx - (T)x0;                                                                       \
            for (int c = 0; c < ch; ++c)                                                             \
            {                                                                                        \
                T v00 = src[((size_t)y0 * w + x0) * ch + c];                                         \
                T v10 = src[((size_t)y0 * w + x1) * ch + c];                                         \
                T v01 = src[((size_t)y1 * w + x0) * ch + c];                                         \
                T v11 = src[((size_t)y1 * w + x1) * ch + c];                                         \
                dst[((size_t)y * ow + x) * ch + c] = ((T)1 - wy) * (((T)1 - wx) * v00 + wx * v10) +  \
                                                     wy * (((T)1 - wx) * v01 + wx * v11);            \
            }                                                                                        \
        }                                                                                            \
    }                                                                                                \
}                                                                                                    \
typedef struct { T* d; int w, h; } lvl_##SUF;                                                        \
/* BuildGaussianPyramid (SeamBlend.cpp:125-140); level 0 takes ownership of base. */                 \
static void gauss_##SUF(T* base, int w, int h, int ch, int bands, lvl_##SUF* out)                    \
{                                                                                                    \
    out[0].d = base; out[0].w = w; out[0].h = h;                                                     \
    for (int l = 1; l < bands; ++l)                                                                  \
        out[l].d = down2_##SUF(out[l - 1].d, out[l - 1].w, out[l - 1].h, ch, &out[l].w, &out[l].h);  \
}                                                                                                    \
/* Compose given owner and coverage (SeamBlend.cpp:447-546). */                                      \
static void compose_##SUF(const uint16_t* const* bufs, const uint8_t* const* cover, const int32_t* owner, \
                          int k, int width, int height, int bands, uint16_t* out)                   \
{                                                                                                    \
    size_t count = (size_t)width * height;                                                           \
    memset(out, 0, count * 3 * sizeof(uint16_t));                                                    \
    bands = or_clamp_bands(width, height, bands);                                                    \
    lvl_##SUF blended[16];                                                                           \
    int init = 0;                                                                                    \
    for (int i = 0; i < k; ++i)                                                                      \
    {                                                                                                \
        int any = 0;                                                                                 \
        for (size_t p = 0; p < count && !any; ++p) any = owner[p] == i;                              \
        if (!any) continue;                                                                          \
        T* wm = (T*)malloc(count * sizeof(T));                                                       \
        for (size_t p = 0; p < count; ++p) wm[p] = owner[p] == i ? (T)1 : (T)0;                      \
        lvl_##SUF wp[16];                                                                            \
        gauss_##SUF(wm, width, height, 1, bands, wp);                                                \
        T* num = (T*)malloc(count * 3 * sizeof(T));                                                  \
        T* den = (T*)malloc(count * sizeof(T));                                                      \
        for (size_t p = 0; p < count; ++p)                                                           \
        {                                                                                            \
            T m = cover[i][p] ? (T)1 : (T)0;                                                         \
            den[p] = m;                                                                              \
            for (int c = 0; c < 3; ++c) num[p * 3 + c] = (T)bufs[i][p * 3 + c] * m;                  \
        }                                                                                            \
        lvl_##SUF np[16], dpyr[16], g[16];                                                           \
        gauss_##SUF(num, width, height, 3, bands, np);                                               \
        gauss_##SUF(den, width, height, 1, bands, dpyr);                                             \
        for (int l = 0; l < bands; ++l)                                                              \
        {                                                                                            \
            size_t lc = (size_t)np[l].w * np[l].h;                                                   \
            g[l].w = np[l].w; g[l].h = np[l].h;                                                      \
            g[l].d = (T*)malloc(lc * 3 * sizeof(T));                                                 \
            for (size_t p = 0; p < lc; ++p)                                                          \
            {                                                                                        \
                T dv = dpyr[l].d[p];                                                                 \
                T inv = (dv > (T)1e-6f) ? (T)1 / dv : (T)0;                                          \
                for (int c = 0; c < 3; ++c) g[l].d[p * 3 + c] = np[l].d[p * 3 + c] * inv;            \
            }                                                                                        \
        }                                                                                            \
        if (!init)                                                                                   \
        {                                                                                            \
            for (int l = 0; l < bands; ++l)                                                          \
            {                                                                                        \
                blended[l].w = g[l].w; blended[l].h = g[l].h;                                        \
                blended[l].d = (T*)calloc((size_t)g[l].w * g[l].h * 3, sizeof(T));                   \
            }                                                                                        \
            init = 1;                                                                                \
        }                                                                                            \
        for (int l = 0; l < bands; ++l)                                                              \
        {                                                                                            \
            size_t lc = (size_t)g[l].w * g[l].h;                                                     \
            T* up = NULL;                                                                            \
            if (l < bands - 1)                                                                       \
            {                                                                                        \
                up = (T*)malloc(lc * 3 * sizeof(T));                                                 \
                up_##SUF(g[l + 1].d, g[l + 1].w, g[l + 1].h, 3, g[l].w, g[l].h, up);                 \
            }                                                                                        \
            for (size_t p = 0; p < lc; ++p)                                                          \
            {                                                                                        \
                T wv = wp[l].d[p];                                                                   \
                for (int c = 0; c < 3; ++c)                                                          \
                {                                                                                    \
                    T lap = up ? g[l].d[p * 3 + c] - up[p * 3 + c] : g[l].d[p * 3 + c];              \
                    blended[l].d[p * 3 + c] += wv * lap;                                             \
                }                                                                                    \
            }                                                                                        \
            free(up);                                                                                \
        }                                                                                            \
        for (int l = 0; l < bands; ++l) { free(wp[l].d); free(np[l].d); free(dpyr[l].d); free(g[l].d); } \
    }                                                                                                \
    if (!init) return;                                                                               \
    T* recon = blended[bands - 1].d;                                                                 \
    int rw = blended[bands - 1].w, rh = blended[bands - 1].h;                                        \
    for (int l = bands - 2; l >= 0; --l)                                                             \
    {                                                                                                \
        size_t n3 = (size_t)blended[l].w * blended[l].h * 3;                                         \
        T* up = (T*)malloc(n3 * sizeof(T));                                                          \
        up_##SUF(recon, rw, rh, 3, blended[l].w, blended[l].h, up);                                  \
        for (size_t p = 0; p < n3; ++p) up[p] = blended[l].d[p] + up[p];                             \
        free(recon);                                                                                 \
        recon = up;                                                                                  \
        rw = blended[l].w; rh = blended[l].h;                                                        \
    }                                                                                                \
    for (int l = 0; l < bands - 1; ++l) free(blended[l].d);                                          \
    for (size_t p = 0; p < count; ++p)                                                               \
        for (int c = 0; c < 3; ++c)                                                                  \
        {                                                                                            \
            T v = recon[p * 3 + c];                                                                  \
            v = (T)0 > ((T)65535 < v ? (T)65535 : v) ? (T)0 : ((T)65535 < v ? (T)65535 : v);         \
            out[p * 3 + c] = (uint16_t)(v + (T)0.5f);                                                \
        }                                                                                            \
    free(recon);                                                                                     \
    for (size_t p = 0; p < count; ++p)                                                               \
        if (owner[p] < 0) out[p * 3] = out[p * 3 + 1] = out[p * 3 + 2] = 0;                          \
}

DEFINE_PYR(float, f32)
DEFINE_PYR(double, f64)

int or_clamp_bands(int w, int h, int bands)
{
    /* SeamBlend.cpp:457-459. */
    int maxBands = 1;
    while (w > 1 && h > 1 && maxBands < bands) { w = (w + 1) / 2; h = (h + 1) / 2; ++maxBands; }
    int lim = maxBands > 1 ? maxBands : 1;
    return bands < lim ? bands : lim;
}

void or_compose(const uint16_t* const* bufs, const float* const* dists, const int32_t* owner, int k,
                int w, int h, int bands, uint16_t* out)
{
    size_t count = (size_t)w * h;
    uint8_t** cov = (uint8_t**)malloc(sizeof(uint8_t*) * (size_t)(k > 0 ? k : 1));
    for (int i = 0; i < k; ++i)
    {
        cov[i] = (uint8_t*)malloc(count);
        for (size_t p = 0; p < count; ++p) cov[i][p] = dists[i][p] > 0.0f;
    }
    compose_f32(bufs, (const uint8_t* const*)cov, owner, k, w, h, bands, out);
    for (int i = 0; i < k; ++i) free(cov[i]);
    free(cov);
}

void or_compose_f64(const uint16_t* const* bufs, const int32_t* owner, int k, int w, int h, int bands,
                    uint16_t* out)
{
    size_t count = (size_t)w * h;
    uint8_t** cov = (uint8_t**)malloc(sizeof(uint8_t*) * (size_t)(k > 0 ? k : 1));
    for (int i = 0; i < k; ++i)
    {
        cov[i] = (uint8_t*)malloc(count);
        or_coverage(bufs[i], w, h, cov[i]);
    }
    compose_f64(bufs, (const uint8_t* const*)cov, owner, k, w, h, bands, out);
    for (int i = 0; i < k; ++i) free(cov[i]);
    free(cov);
}

void or_blend_chunk_ex(const uint16_t* const* bufs, int k, int w, int h, int bands, uint16_t* out,
                       int32_t* ownerOut)
{
    /* SeamBlend.cpp:549-587. */
    size_t count = (size_t)w * h;
    memset(out, 0, count * 3 * sizeof(uint16_t));
    if (k <= 0) { if (ownerOut) for (size_t p = 0; p < count; ++p) ownerOut[p] = -1; return; }
    uint8_t** cov = (uint8_t**)malloc(sizeof(uint8_t*) * (size_t)k);
    float** dist = (float**)malloc(sizeof(float*) * (size_t)k);
    int32_t* boxes = (int32_t*)malloc(sizeof(int32_t) * 4 * (size_t)k);
    int* valid = (int*)malloc(sizeof(int) * (size_t)k);
    for (int i = 0; i < k; ++i)
    {
        cov[i] = (uint8_t*)malloc(count);
        dist[i] = (float*)malloc(count * sizeof(float));
        or_coverage(bufs[i], w, h, cov[i]);
        or_coverage_distance(cov[i], w, h, dist[i]);
        valid[i] = or_bbox(cov[i], w, h, boxes + 4 * i);
    }
    int32_t* owner = ownerOut ? ownerOut : (int32_t*)malloc(count * sizeof(int32_t));
    or_ownership((const float* const*)dist, k, w, h, owner);
    for (int i = 0; i < k; ++i)
    {
        if (!valid[i]) continue;
        for (int j = i + 1; j < k; ++j)
        {
            if (!valid[j]) continue;
            int32_t ov[4];
            if (!intersect_bbox(boxes + 4 * i, 1, boxes + 4 * j, 1, ov)) continue;
            or_refine_seam(bufs[i], bufs[j], dist[i], dist[j], w, h, i, j, boxes + 4 * i, boxes + 4 * j, ov, owner);
        }
    }
    compose_f32(bufs, (const uint8_t* const*)cov, owner, k, w, h, bands, out);
    for (int i = 0; i < k; ++i) { free(cov[i]); free(dist[i]); }
    free(cov); free(dist); free(boxes); free(valid);
    if (!ownerOut) free(owner);
}

void or_blend_chunk(const uint16_t* const* bufs, int k, int w, int h, int bands, uint16_t* out)
{
    or_blend_chunk_ex(bufs, k, w, h, bands, out, NULL);
}

/* ------------------------------------------------------------------------ */
/* Multi-threaded tile render (RenderExecutor.cpp:70-140 per chunk).          */
/* ------------------------------------------------------------------------ */

typedef struct
{
    const uint16_t* const* frames;
    const int32_t *frameW, *frameH;
    const float *invH, *gains;
    int nTiles;
    const int32_t *rect, *off, *contrib;
    int bands;
    uint16_t** out;
    int next;
    pthread_mutex_t mu;
} render_job;

static void* render_worker(void* arg)
{
    render_job* j = (render_job*)arg;
    for (;;)
    {
        pthread_mutex_lock(&j->mu);
        int t = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (t >= j->nTiles) break;
        int tx = j->rect[4 * t], ty = j->rect[4 * t + 1], tw = j->rect[4 * t + 2], th = j->rect[4 * t + 3];
        size_t n3 = (size_t)tw * th * 3;
        int kb = j->off[t], ke = j->off[t + 1];
        int k = ke - kb;
        uint16_t** warped = (uint16_t**)malloc(sizeof(uint16_t*) * (size_t)(k > 0 ? k : 1));
        for (int q = 0; q < k; ++q)
        {
            int f = j->contrib[kb + q];
            warped[q] = (uint16_t*)calloc(n3, sizeof(uint16_t));
            or_warp(j->frames[f], j->frameW[f], j->frameH[f], warped[q], tw, th, j->invH + 9 * f, tx, ty);
            if (fabsf(j->gains[f] - 1.0f) > 1e-6f) or_gain(warped[q], (int)n3, j->gains[f]);
        }
        uint16_t* res = (j->out && j->out[t]) ? j->out[t] : (uint16_t*)malloc(n3 * sizeof(uint16_t));
        or_blend_chunk((const uint16_t* const*)warped, k, tw, th, j->bands, res);
        if (!(j->out && j->out[t])) free(res);
        for (int q = 0; q < k; ++q) free(warped[q]);
        free(warped);
    }
    return NULL;
}

double or_render_tiles(int threads, const uint16_t* const* frames, const int32_t* frameW,
                       const int32_t* frameH, const float* invH, const float* gains, int nTiles,
                       const int32_t* tileRect, const int32_t* contribOffset, const int32_t* contrib,
                       int bands, uint16_t** out)
{
    render_job j = {frames, frameW, frameH, invH, gains, nTiles, tileRect, contribOffset, contrib,
                    bands, out, 0, PTHREAD_MUTEX_INITIALIZER};
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    int nt = threads < 1 ? 1 : threads;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nt);
    for (int i = 0; i < nt; ++i) pthread_create(&th[i], NULL, render_worker, &j);
    for (int i = 0; i < nt; ++i) pthread_join(th[i], NULL);
    free(th);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}
