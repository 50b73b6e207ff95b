/*
 * Checks two FP32 identities the GPU colour conversion (image360_b200/csrc/color.cu)
 * relies on, with the host's IEEE arithmetic (the GPU's fmul/fma/fsub round the
 * same way):
 *
 *  1. Division by each conversion constant d as q = x * r, r = 1.0f / d,
 *     corrected by one FMA residual step, equals the IEEE quotient x / d for
 *     every float x with 2^-99 <= |x| < 2^100.
 *  2. One Newton step y - (y^3 - t) / (3 y^2) whose residual is formed from
 *     FMA product error terms turns a cube-root seed within 4 ulp into the
 *     correctly rounded cube root for almost every t in (delta^3, 2] (the
 *     count of exceptions is printed; the bound is 1 in 10^5).
 *  3. One Newton step on z^12 = c^5 (residual from FMA error terms) with the
 *     first-order exponent correction turns a seed of c^(1/2.4f) within 4 ulp
 *     into the correctly rounded power for almost every c in
 *     (0.0031308, 2] (bound: 1 in 10^5).
 *
 * Usage: color_arith_check [--all]   (default: every 251st float; --all:
 * every float, several minutes).  Exit status 0 when both hold.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static float from_bits(uint32_t u)
{
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static uint32_t to_bits(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

static float div_const(float x, float d, float r)
{
    float q = x * r;
    return fmaf(fmaf(-q, d, x), r, q);
}

static float cbrt_step(float y, float t)
{
    float p = y * y, pl = fmaf(y, y, -p);
    float c = p * y, cl = fmaf(p, y, -c);
    float e = (c - t) + fmaf(pl, y, cl);
    return y - e / (3.0f * p);
}

static const float kInvGamma = 1.0f / 2.4f;

static float encode_step(float c, float z, float l2)
{
    const float dl = (float)(((double)kInvGamma - 5.0 / 12.0) * 0.69314718055994530942);
    float z2 = z * z, z2l = fmaf(z, z, -z2);
    float z4 = z2 * z2, z4l = fmaf(z2, z2, -z4) + 2.0f * z2 * z2l;
    float z8 = z4 * z4, z8l = fmaf(z4, z4, -z8) + 2.0f * z4 * z4l;
    float z12 = z8 * z4, z12l = fmaf(z8, z4, -z12) + (z8 * z4l + z4 * z8l);
    float c2 = c * c, c2l = fmaf(c, c, -c2);
    float c4 = c2 * c2, c4l = fmaf(c2, c2, -c4) + 2.0f * c2 * c2l;
    float c5 = c4 * c, c5l = fmaf(c4, c, -c5) + c4l * c;
    float q = ((z12 - c5) + (z12l - c5l)) / z12;
    return fmaf(z, dl * l2 - q * (1.0f / 12.0f), z);
}

int main(int argc, char** argv)
{
    const uint32_t stride = (argc > 1 && strcmp(argv[1], "--all") == 0) ? 1u : 251u;
    const float delta = 6.0f / 29.0f;
    const float divisors[] = {0.95047f, 1.08883f, 116.0f, 500.0f, 200.0f, 3.0f * delta * delta};
    int ok = 1;
    const uint32_t lo = to_bits(0x1p-99f), hi = to_bits(0x1p100f);
    for (int k = 0; k < 6; ++k)
    {
        const float d = divisors[k], r = 1.0f / d;
        long long n = 0, bad = 0;
        for (uint32_t u = lo; u < hi; u += stride)
            for (int s = 0; s < 2; ++s)
            {
                float x = s ? -from_bits(u) : from_bits(u);
                ++n;
                if (to_bits(div_const(x, d, r)) != to_bits(x / d)) ++bad;
            }
        printf("divide by %.9g: %lld values, %lld differ from IEEE division\n", d, n, bad);
        if (bad) ok = 0;
    }
    const uint32_t c0 = to_bits(delta * delta * delta) + 1, c1 = to_bits(2.0f);
    for (int pert = -4; pert <= 4; pert += 4)
    {
        long long n = 0, bad = 0;
        for (uint32_t u = c0; u <= c1; u += stride)
        {
            float t = from_bits(u);
            float exact = (float)cbrt((double)t);
            float seed = from_bits(to_bits(exact) + (uint32_t)pert);
            ++n;
            if (to_bits(cbrt_step(seed, t)) != to_bits(exact)) ++bad;
        }
        printf("cube root, seed %+d ulp: %lld values, %lld not correctly rounded\n", pert, n, bad);
        if (bad * 100000LL > n) ok = 0;
    }
    const uint32_t e0 = to_bits(0.0031308f) + 1, e1 = to_bits(2.0f);
    for (int pert = -4; pert <= 4; pert += 4)
    {
        long long n = 0, bad = 0;
        for (uint32_t u = e0; u <= e1; u += stride)
        {
            float c = from_bits(u);
            float exact = (float)pow((double)c, (double)kInvGamma);
            float seed = from_bits(to_bits(exact) + (uint32_t)pert);
            ++n;
            if (to_bits(encode_step(c, seed, log2f(c))) != to_bits(exact)) ++bad;
        }
        printf("encode power, seed %+d ulp: %lld values, %lld not correctly rounded\n", pert, n, bad);
        if (bad * 100000LL > n) ok = 0;
    }
    return ok ? 0 : 1;
}
