// Tile -> contributor lists of a panorama on the device: the overlap test of
// OverlapCulling.cpp:10-45 (ImageOverlapsChunk) for every (tile, frame) pair,
// each tile's list in frame order as FindOverlappingImages builds it
// (OverlapCulling.cpp:47-89), including its conservative rule that a frame of
// unknown size (width or height <= 0) overlaps every tile.
//
// The test projects the frame's four corners (0,0), (W,0), (0,H), (W,H)
// through its frame -> canvas homography, takes the axis-aligned box of the
// projected points and compares it with the tile rectangle with strict
// inequalities.  The box depends on the frame only, so it is computed once
// per frame (k_frame_boxes), then one warp per tile tests the frames 32 at a
// time and ballots the hits (k_cull_count / k_cull_write), writing the
// tile's contributors in frame order at an offset from an exclusive scan of
// the counts (k_cull_scan).  Modes:
//   I360B_CULL_REFERENCE  FP32 as the reference: products and sums rounded
//                         separately (this file is built without FMA
//                         contraction), the tile bounds as float(x) +
//                         float(w) - decisions identical to the CPU's;
//   I360B_CULL_FP64       the corners and the tile bounds in FP64, for
//                         canvases beyond 2^24 pixels where FP32 tile bounds
//                         round.
#include "common.cuh"

using namespace i360b;

namespace
{
struct Box
{
    double x0, y0, x1, y1;
    int known;  // 0: size unknown, the frame overlaps every tile
};

constexpr int kWarpsPerBlock = 8;

// OverlapCulling.cpp:36-63 in FP32.
__device__ Box frame_box_f32(const float* m, int w, int h)
{
    const float cx[4] = {0.0f, (float)w, 0.0f, (float)w};
    const float cy[4] = {0.0f, 0.0f, (float)h, (float)h};
    const float big = 3.402823466e38f;
    float minX = big, minY = big, maxX = -big, maxY = -big;
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        float den = fadd(fadd(fmul(m[6], cx[k]), fmul(m[7], cy[k])), m[8]);
        if (fabsf(den) < 1e-10f) den = den >= 0.0f ? 1e-10f : -1e-10f;
        const float px = fdiv(fadd(fadd(fmul(m[0], cx[k]), fmul(m[1], cy[k])), m[2]), den);
        const float py = fdiv(fadd(fadd(fmul(m[3], cx[k]), fmul(m[4], cy[k])), m[5]), den);
        // (std::min)(a, b) is (b < a) ? b : a: a NaN corner leaves the box as is
        minX = px < minX ? px : minX;
        minY = py < minY ? py : minY;
        maxX = maxX < px ? px : maxX;
        maxY = maxY < py ? py : maxY;
    }
    return Box{minX, minY, maxX, maxY, 1};
}

__device__ Box frame_box_f64(const float* m, int w, int h)
{
    const double cx[4] = {0.0, (double)w, 0.0, (double)w};
    const double cy[4] = {0.0, 0.0, (double)h, (double)h};
    double minX = 1.7976931348623157e308, minY = minX, maxX = -minX, maxY = -minX;
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        double den = __dadd_rn(__dadd_rn(__dmul_rn(m[6], cx[k]), __dmul_rn(m[7], cy[k])), (double)m[8]);
        if (fabs(den) < 1e-10) den = den >= 0.0 ? 1e-10 : -1e-10;
        const double px =
            __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], cx[k]), __dmul_rn(m[1], cy[k])), (double)m[2]), den);
        const double py =
            __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[3], cx[k]), __dmul_rn(m[4], cy[k])), (double)m[5]), den);
        minX = px < minX ? px : minX;
        minY = py < minY ? py : minY;
        maxX = maxX < px ? px : maxX;
        maxY = maxY < py ? py : maxY;
    }
    return Box{minX, minY, maxX, maxY, 1};
}

struct CullArgs
{
    const float* H;  // numFrames x 9, row-major, frame -> canvas
    const int* frameW;
    const int* frameH;
    int numFrames;
    const int* tiles;  // numTiles x 4: x, y, w, h
    int numTiles;
    int mode;
    Box* boxes;  // numFrames
    int* first;
    int* count;
    int* contrib;
    int capacity;
    int* total;
};

__global__ void k_frame_boxes(CullArgs a)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.numFrames) return;
    const int w = a.frameW[f], h = a.frameH[f];
    Box b{0.0, 0.0, 0.0, 0.0, 0};
    if (w > 0 && h > 0)
        b = a.mode == I360B_CULL_FP64 ? frame_box_f64(a.H + (size_t)f * 9, w, h)
                                      : frame_box_f32(a.H + (size_t)f * 9, w, h);
    a.boxes[f] = b;
}

// OverlapCulling.cpp:65-70.
__device__ __forceinline__ bool hits(const CullArgs& a, const Box& b, int x, int y, int w, int h)
{
    if (!b.known) return true;  // OverlapCulling.cpp:100-106
    if (a.mode == I360B_CULL_FP64)
    {
        const double cx0 = x, cy0 = y, cx1 = (double)x + (double)w, cy1 = (double)y + (double)h;
        return b.x0 < cx1 && b.x1 > cx0 && b.y0 < cy1 && b.y1 > cy0;
    }
    const float cx0 = (float)x, cy0 = (float)y;
    const float cx1 = fadd(cx0, (float)w), cy1 = fadd(cy0, (float)h);
    return (float)b.x0 < cx1 && (float)b.x1 > cx0 && (float)b.y0 < cy1 && (float)b.y1 > cy0;
}

template <bool WRITE>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_cull(CullArgs a)
{
    const int t = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= a.numTiles) return;
    const int x = a.tiles[t * 4], y = a.tiles[t * 4 + 1], w = a.tiles[t * 4 + 2], h = a.tiles[t * 4 + 3];
    int n = 0;
    const int base = WRITE ? a.first[t] : 0;
    for (int f0 = 0; f0 < a.numFrames; f0 += 32)
    {
        const int f = f0 + lane;
        const bool hit = f < a.numFrames && hits(a, a.boxes[f], x, y, w, h);
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        if (WRITE && hit)
        {
            const int pos = base + n + __popc(mask & ((1u << lane) - 1u));
            if (pos < a.capacity) a.contrib[pos] = f;
        }
        n += __popc(mask);
    }
    if (!WRITE && lane == 0) a.count[t] = n;
}

// Exclusive scan of the counts into first[], total into *total (one block).
__global__ void k_cull_scan(CullArgs a)
{
    __shared__ int carry;
    __shared__ int warpSums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < a.numTiles; base += blockDim.x)
    {
        const int i = base + threadIdx.x;
        const int v = i < a.numTiles ? a.count[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1)
        {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) warpSums[warp] = incl;
        __syncthreads();
        int before = carry;
        for (int k = 0; k < warp; ++k) before += warpSums[k];
        if (i < a.numTiles) a.first[i] = before + incl - v;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            int s = 0;
            for (int k = 0; k < nw; ++k) s += warpSums[k];
            carry += s;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *a.total = carry;
}

int check_cull(int numFrames, int numTiles, int mode, int capacity)
{
    if (numFrames < 0 || numTiles < 0) return fail(I360B_INVALID_PARAM, "Invalid frame or tile count.");
    if (mode != I360B_CULL_REFERENCE && mode != I360B_CULL_FP64)
        return fail(I360B_INVALID_PARAM, "Unknown culling mode %d.", mode);
    if (capacity < 0) return fail(I360B_INVALID_PARAM, "Invalid contributor capacity.");
    return I360B_SUCCESS;
}

int run_cull(CullArgs a, cudaStream_t s)
{
    if (a.numTiles == 0)
    {
        I360B_CUDA(cudaMemsetAsync(a.total, 0, sizeof(int), s), "tile culling");
        return I360B_SUCCESS;
    }
    if (a.numFrames > 0)
    {
        k_frame_boxes<<<(a.numFrames + 127) / 128, 128, 0, s>>>(a);
        I360B_TRY(check_launch("frame box kernel"));
    }
    const int blocks = (a.numTiles + kWarpsPerBlock - 1) / kWarpsPerBlock;
    k_cull<false><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a);
    I360B_TRY(check_launch("tile culling kernel"));
    k_cull_scan<<<1, 1024, 0, s>>>(a);
    I360B_TRY(check_launch("tile culling scan kernel"));
    k_cull<true><<<blocks, kWarpsPerBlock * 32, 0, s>>>(a);
    return check_launch("tile culling kernel");
}

struct Scratch
{
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() { dev_free(p, s); }
};
}  // namespace

extern "C" int i360b_launch_cull_tiles(const float* dHomographies, const int* dFrameWidths, const int* dFrameHeights,
                                       int numFrames, const int* dTiles, int numTiles, int mode, int* dFirst,
                                       int* dCount, int* dContrib, int contribCapacity, int* dTotal, void* stream)
{
    clear_error();
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    I360B_TRY(check_cull(numFrames, numTiles, mode, contribCapacity));
    if (!dTotal || (numFrames > 0 && (!dHomographies || !dFrameWidths || !dFrameHeights)) ||
        (numTiles > 0 && (!dTiles || !dFirst || !dCount)) || (contribCapacity > 0 && !dContrib))
        return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch boxes;
    boxes.s = s;
    if (numFrames > 0) I360B_TRY(dev_alloc(&boxes.p, (size_t)numFrames * sizeof(Box), s, "tile culling"));
    CullArgs a{dHomographies, dFrameWidths, dFrameHeights, numFrames, dTiles, numTiles, mode,
               static_cast<Box*>(boxes.p), dFirst, dCount, dContrib, contribCapacity, dTotal};
    return run_cull(a, s);
}

extern "C" int i360b_cull_tiles(const float* homographies, const int* frameWidths, const int* frameHeights,
                                int numFrames, const int* tiles, int numTiles, int mode, int* first, int* count,
                                int* contrib, int contribCapacity, int* total)
{
    clear_error();
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    I360B_TRY(check_cull(numFrames, numTiles, mode, contribCapacity));
    if (!total || (numFrames > 0 && (!homographies || !frameWidths || !frameHeights)) ||
        (numTiles > 0 && (!tiles || !first || !count)) || (contribCapacity > 0 && !contrib))
        return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    cudaStream_t s = thread_stream();
    if (!s) return fail(I360B_CUDA_ERROR, "Could not create a CUDA stream for this thread.");
    const size_t fb = (size_t)numFrames, tb = (size_t)numTiles;
    const size_t bytes = fb * 9 * sizeof(float) + fb * 2 * sizeof(int) + tb * 4 * sizeof(int) + tb * 2 * sizeof(int) +
                         (size_t)contribCapacity * sizeof(int) + sizeof(int) + fb * sizeof(Box) + 64;
    Scratch buf;
    buf.s = s;
    I360B_TRY(dev_alloc(&buf.p, bytes, s, "tile culling"));
    char* p = static_cast<char*>(buf.p);
    auto take = [&p](size_t n) {
        char* q = p;
        p += (n + 7) & ~size_t(7);
        return q;
    };
    Box* dBoxes = reinterpret_cast<Box*>(take(fb * sizeof(Box)));
    float* dH = reinterpret_cast<float*>(take(fb * 9 * sizeof(float)));
    int* dW = reinterpret_cast<int*>(take(fb * sizeof(int)));
    int* dHt = reinterpret_cast<int*>(take(fb * sizeof(int)));
    int* dT = reinterpret_cast<int*>(take(tb * 4 * sizeof(int)));
    int* dFirst = reinterpret_cast<int*>(take(tb * sizeof(int)));
    int* dCount = reinterpret_cast<int*>(take(tb * sizeof(int)));
    int* dContrib = reinterpret_cast<int*>(take((size_t)contribCapacity * sizeof(int)));
    int* dTotal = reinterpret_cast<int*>(take(sizeof(int)));
    if (numFrames > 0)
    {
        I360B_CUDA(cudaMemcpyAsync(dH, homographies, fb * 9 * sizeof(float), cudaMemcpyHostToDevice, s), "culling upload");
        I360B_CUDA(cudaMemcpyAsync(dW, frameWidths, fb * sizeof(int), cudaMemcpyHostToDevice, s), "culling upload");
        I360B_CUDA(cudaMemcpyAsync(dHt, frameHeights, fb * sizeof(int), cudaMemcpyHostToDevice, s), "culling upload");
    }
    if (numTiles > 0)
        I360B_CUDA(cudaMemcpyAsync(dT, tiles, tb * 4 * sizeof(int), cudaMemcpyHostToDevice, s), "culling upload");
    CullArgs a{dH, dW, dHt, numFrames, dT, numTiles, mode, dBoxes, dFirst, dCount, dContrib, contribCapacity, dTotal};
    I360B_TRY(run_cull(a, s));
    if (numTiles > 0)
    {
        I360B_CUDA(cudaMemcpyAsync(first, dFirst, tb * sizeof(int), cudaMemcpyDeviceToHost, s), "culling download");
        I360B_CUDA(cudaMemcpyAsync(count, dCount, tb * sizeof(int), cudaMemcpyDeviceToHost, s), "culling download");
    }
    I360B_CUDA(cudaMemcpyAsync(total, dTotal, sizeof(int), cudaMemcpyDeviceToHost, s), "culling download");
    I360B_CUDA(cudaStreamSynchronize(s), "tile culling");
    if (*total > contribCapacity)
        return fail(I360B_INVALID_PARAM, "Contributor capacity %d is below the %d contributors found.", contribCapacity,
                    *total);
    if (*total > 0)
    {
        I360B_CUDA(cudaMemcpyAsync(contrib, dContrib, (size_t)*total * sizeof(int), cudaMemcpyDeviceToHost, s),
                   "culling download");
        I360B_CUDA(cudaStreamSynchronize(s), "tile culling");
    }
    return I360B_SUCCESS;
}
