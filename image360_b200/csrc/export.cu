// Export of a panorama's rendered chunk outputs, device-resident:
//   * the preview composite of PanoramaExporter::ExportPreviewJpeg
//     (PanoramaExporter.cpp:46-102): every chunk's RGB48 output placed, in
//     chunk order, into an RGB8 canvas scaled so its longest edge is
//     maxDimension - placement and source pixel by the FP32 steps of
//     ComputeExportScale / ComputeChunkPlacement (PanoramaExporter.cpp:9-24)
//     and int(d / scale) (a table over d, shared by all chunks), samples >> 8,
//     pixels without a source left at 0.  When no two placements overlap (a
//     chunk grid) one launch covers every chunk; otherwise one launch per
//     chunk in chunk order reproduces the reference loop's last-writer-wins;
//   * the framed chunk blob of StorageEngine::WritePixelBuffer
//     (StorageEngine.cpp:130-144): int32 width, int32 height, the samples;
//   * the 16-bit RGB TIFF of WriteTiff16RGB (Tiff16Writer.cpp:40-97) of a
//     whole canvas of chunk outputs, assembled band by band on the device
//     (2-D copies of every chunk row range into a zeroed band) and streamed
//     to the file through two pinned buffers, so the host writes one band
//     while the next is copied.
// The JPEG encode of the preview is left to the caller's codec (nvJPEG in the
// reference, IImageCodec::Encode).
#include "render_plan.hpp"

#include <algorithm>
#include <cstdio>
#include <vector>

using namespace i360b;

namespace
{
struct ExportTile
{
    const unsigned short* src;
    int x, y, w, h;
};

// ComputeChunkPlacement (PanoramaExporter.cpp:16-24).
__host__ __device__ __forceinline__ void placement(const ExportTile& t, float scale, int* p)
{
#ifdef __CUDA_ARCH__
    p[0] = __float2int_rz(__fmul_rn((float)t.x, scale));
    p[1] = __float2int_rz(__fmul_rn((float)t.y, scale));
    const int w = __float2int_rz(__fmul_rn((float)t.w, scale)), h = __float2int_rz(__fmul_rn((float)t.h, scale));
#else
    p[0] = (int)((float)t.x * scale);
    p[1] = (int)((float)t.y * scale);
    const int w = (int)((float)t.w * scale), h = (int)((float)t.h * scale);
#endif
    p[2] = w > 1 ? w : 1;
    p[3] = h > 1 ? h : 1;
}

// int(d / scale) for every placement offset d (PanoramaExporter.cpp:86-87).
__global__ void k_export_source_table(float scale, int n, int* tab)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < n) tab[d] = __float2int_rz(__fdiv_rn((float)d, scale));
}

// Chunks [t0, t0 + gridDim.z) write their placements (PanoramaExporter.cpp:74-101).
__global__ void k_export_place(const ExportTile* __restrict__ tiles, int t0, float scale, int ow, int oh,
                               const int* __restrict__ srcOf, unsigned char* __restrict__ out)
{
    const ExportTile T = tiles[t0 + blockIdx.z];
    int p[4];
    placement(T, scale, p);
    const int dx = blockIdx.x * blockDim.x + threadIdx.x, dy = blockIdx.y * blockDim.y + threadIdx.y;
    if (dx >= p[2] || dy >= p[3]) return;
    const int ox = p[0] + dx, oy = p[1] + dy;
    if (ox < 0 || ox >= ow || oy < 0 || oy >= oh) return;
    const int sx = srcOf[dx], sy = srcOf[dy];
    if (sx < 0 || sx >= T.w || sy < 0 || sy >= T.h) return;
    const unsigned short* s = T.src + ((size_t)sy * T.w + sx) * 3;
    unsigned char* o = out + ((size_t)oy * ow + ox) * 3;
    o[0] = (unsigned char)(s[0] >> 8);
    o[1] = (unsigned char)(s[1] >> 8);
    o[2] = (unsigned char)(s[2] >> 8);
}

struct Scratch
{
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~Scratch() { dev_free(p, s); }
};

// ComputeExportScale (PanoramaExporter.cpp:9-14) and the composite size
// (PanoramaExporter.cpp:50-52).
void export_size(int totalW, int totalH, int maxDimension, float* scale, int* ow, int* oh)
{
    const int longest = totalW > totalH ? totalW : totalH;
    *scale = longest <= 0 ? 1.0f : (float)maxDimension / (float)longest;
    const int w = (int)((float)totalW * *scale), h = (int)((float)totalH * *scale);
    *ow = w > 1 ? w : 1;
    *oh = h > 1 ? h : 1;
}

int export_preview(const std::vector<ExportTile>& tiles, int totalW, int totalH, int maxDimension, unsigned char* dOut,
                   long long capacity, int* outW, int* outH, cudaStream_t s)
{
    if (!outW || !outH) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (maxDimension <= 0 || totalW <= 0 || totalH <= 0)
        return fail(I360B_INVALID_PARAM, "Invalid canvas size or maximum dimension.");
    if (tiles.size() > 65535) return fail(I360B_INVALID_PARAM, "More than 65535 chunks.");
    float scale;
    int ow, oh;
    export_size(totalW, totalH, maxDimension, &scale, &ow, &oh);
    *outW = ow;
    *outH = oh;
    if ((long long)ow * oh * 3 > capacity)
        return fail(I360B_INVALID_PARAM, "The %dx%d preview needs %lld bytes (capacity %lld).", ow, oh,
                    (long long)ow * oh * 3, capacity);
    if (!dOut) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    I360B_CUDA(cudaMemsetAsync(dOut, 0, (size_t)ow * oh * 3, s), "preview export");
    if (tiles.empty()) return I360B_SUCCESS;
    // placements clipped to the canvas; overlap decides between one launch
    // and one launch per chunk
    std::vector<int> pl(tiles.size() * 4);
    int maxW = 1, maxH = 1;
    for (size_t t = 0; t < tiles.size(); ++t)
    {
        placement(tiles[t], scale, &pl[t * 4]);
        maxW = pl[t * 4 + 2] > maxW ? pl[t * 4 + 2] : maxW;
        maxH = pl[t * 4 + 3] > maxH ? pl[t * 4 + 3] : maxH;
    }
    bool overlap = false;
    for (size_t a = 0; a < tiles.size() && !overlap; ++a)
        for (size_t b = a + 1; b < tiles.size() && !overlap; ++b)
        {
            const int* A = &pl[a * 4];
            const int* B = &pl[b * 4];
            const int x0 = std::max(std::max(A[0], B[0]), 0), x1 = std::min(std::min(A[0] + A[2], B[0] + B[2]), ow);
            const int y0 = std::max(std::max(A[1], B[1]), 0), y1 = std::min(std::min(A[1] + A[3], B[1] + B[3]), oh);
            overlap = x0 < x1 && y0 < y1;
        }
    Scratch desc, tab;
    desc.s = tab.s = s;
    const int tabN = std::max(maxW, maxH);
    I360B_TRY(dev_alloc(&desc.p, tiles.size() * sizeof(ExportTile), s, "preview export"));
    I360B_TRY(dev_alloc(&tab.p, (size_t)tabN * sizeof(int), s, "preview export"));
    I360B_CUDA(cudaMemcpyAsync(desc.p, tiles.data(), tiles.size() * sizeof(ExportTile), cudaMemcpyHostToDevice, s),
               "preview export");
    k_export_source_table<<<(tabN + 255) / 256, 256, 0, s>>>(scale, tabN, static_cast<int*>(tab.p));
    I360B_TRY(check_launch("preview source table kernel"));
    const dim3 block(32, 8);
    const ExportTile* dT = static_cast<const ExportTile*>(desc.p);
    const int* dTab = static_cast<const int*>(tab.p);
    if (!overlap)
    {
        const dim3 grid((maxW + 31) / 32, (maxH + 7) / 8, (unsigned)tiles.size());
        k_export_place<<<grid, block, 0, s>>>(dT, 0, scale, ow, oh, dTab, dOut);
        return check_launch("preview placement kernel");
    }
    for (size_t t = 0; t < tiles.size(); ++t)
    {
        const dim3 grid((pl[t * 4 + 2] + 31) / 32, (pl[t * 4 + 3] + 7) / 8, 1);
        k_export_place<<<grid, block, 0, s>>>(dT, (int)t, scale, ow, oh, dTab, dOut);
        I360B_TRY(check_launch("preview placement kernel"));
    }
    return I360B_SUCCESS;
}

void put_u16(unsigned char* p, uint16_t v)
{
    p[0] = (unsigned char)(v & 0xff);
    p[1] = (unsigned char)(v >> 8);
}

void put_u32(unsigned char* p, uint32_t v)
{
    for (int i = 0; i < 4; ++i) p[i] = (unsigned char)(v >> (8 * i));
}

// The bytes of Tiff16Writer.cpp:58-61 (header) and :69-90 (blocks after the
// pixel data, then the IFD) for a w x h image.
void tiff_header(int w, int h, unsigned char* hdr8, std::vector<unsigned char>& trailer)
{
    const uint32_t pix = (uint32_t)((size_t)w * h * 6);
    const uint32_t bps = 8 + pix, xres = bps + 6, yres = xres + 8, ifd = yres + 8;
    hdr8[0] = 'I';
    hdr8[1] = 'I';
    put_u16(hdr8 + 2, 42);
    put_u32(hdr8 + 4, ifd);
    trailer.assign(6 + 16 + 2 + 12 * 12 + 4, 0);
    unsigned char* p = trailer.data();
    put_u16(p, 16);
    put_u16(p + 2, 16);
    put_u16(p + 4, 16);
    put_u32(p + 6, 72);
    put_u32(p + 10, 1);
    put_u32(p + 14, 72);
    put_u32(p + 18, 1);
    p += 22;
    put_u16(p, 12);
    const uint32_t e[12][4] = {{256, 4, 1, (uint32_t)w}, {257, 4, 1, (uint32_t)h}, {258, 3, 3, bps},
                               {259, 3, 1, 1},          {262, 3, 1, 2},          {273, 4, 1, 8},
                               {277, 3, 1, 3},          {278, 4, 1, (uint32_t)h}, {279, 4, 1, pix},
                               {282, 5, 1, xres},       {283, 5, 1, yres},       {296, 3, 1, 2}};
    for (int i = 0; i < 12; ++i)
    {
        unsigned char* q = p + 2 + 12 * i;
        put_u16(q, (uint16_t)e[i][0]);
        put_u16(q + 2, (uint16_t)e[i][1]);
        put_u32(q + 4, e[i][2]);
        put_u32(q + 8, e[i][3]);
    }
}

struct HostBuf
{
    void* p = nullptr;
    ~HostBuf()
    {
        if (p) cudaFreeHost(p);
    }
};

struct File
{
    FILE* f = nullptr;
    ~File()
    {
        if (f) fclose(f);
    }
};

int write_tiff(const char* path, const std::vector<ExportTile>& tiles, int W, int H, cudaStream_t s)
{
    if (!path) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (W <= 0 || H <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    const unsigned long long pix = (unsigned long long)W * H * 6;
    if (pix + 8 + 64 > 0xffffffffull)
        return fail(I360B_INVALID_PARAM, "A %dx%d RGB48 image does not fit the 32-bit offsets of a baseline TIFF.", W, H);
    const size_t rowBytes = (size_t)W * 6;
    int band = (int)((size_t)(256u << 20) / rowBytes);
    band = band < 1 ? 1 : (band > H ? H : band);
    const size_t bandBytes = rowBytes * band;
    Scratch dBand;
    dBand.s = s;
    I360B_TRY(dev_alloc(&dBand.p, bandBytes, s, "TIFF export"));
    HostBuf hb[2];
    for (auto& b : hb) I360B_CUDA(cudaHostAlloc(&b.p, bandBytes, cudaHostAllocDefault), "TIFF export staging");
    cudaEvent_t ev[2] = {nullptr, nullptr};
    for (auto& e : ev) I360B_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "TIFF export");
    struct Events
    {
        cudaEvent_t* e;
        ~Events()
        {
            cudaEventDestroy(e[0]);
            cudaEventDestroy(e[1]);
        }
    } evGuard{ev};
    File file;
    file.f = fopen(path, "wb");
    if (!file.f) return fail(I360B_INVALID_PARAM, "Cannot open %s for writing.", path);
    unsigned char hdr[8];
    std::vector<unsigned char> trailer;
    tiff_header(W, H, hdr, trailer);
    if (fwrite(hdr, 1, 8, file.f) != 8) return fail(I360B_INVALID_PARAM, "Cannot write %s.", path);
    const int nb = (H + band - 1) / band;
    size_t pending = 0;
    for (int b = 0; b <= nb; ++b)
    {
        if (b < nb)
        {
            const int y0 = b * band, y1 = y0 + band < H ? y0 + band : H;
            I360B_CUDA(cudaMemsetAsync(dBand.p, 0, rowBytes * (y1 - y0), s), "TIFF export");
            for (const ExportTile& t : tiles)
            {
                const int r0 = t.y > y0 ? t.y : y0, r1 = t.y + t.h < y1 ? t.y + t.h : y1;
                const int c0 = t.x > 0 ? t.x : 0, c1 = t.x + t.w < W ? t.x + t.w : W;
                if (r0 >= r1 || c0 >= c1) continue;
                const unsigned short* src = t.src + ((size_t)(r0 - t.y) * t.w + (c0 - t.x)) * 3;
                unsigned char* dst = static_cast<unsigned char*>(dBand.p) + (size_t)(r0 - y0) * rowBytes + (size_t)c0 * 6;
                I360B_CUDA(cudaMemcpy2DAsync(dst, rowBytes, src, (size_t)t.w * 6, (size_t)(c1 - c0) * 6, r1 - r0,
                                             cudaMemcpyDeviceToDevice, s),
                           "TIFF export band copy");
            }
            I360B_CUDA(cudaMemcpyAsync(hb[b & 1].p, dBand.p, rowBytes * (y1 - y0), cudaMemcpyDeviceToHost, s),
                       "TIFF export download");
            I360B_CUDA(cudaEventRecord(ev[b & 1], s), "TIFF export");
        }
        if (b > 0)
        {
            const int p = (b - 1) & 1;
            I360B_CUDA(cudaEventSynchronize(ev[p]), "TIFF export");
            if (fwrite(hb[p].p, 1, pending, file.f) != pending) return fail(I360B_INVALID_PARAM, "Cannot write %s.", path);
        }
        if (b < nb)
        {
            const int y0 = b * band, y1 = y0 + band < H ? y0 + band : H;
            pending = rowBytes * (y1 - y0);
        }
    }
    if (fwrite(trailer.data(), 1, trailer.size(), file.f) != trailer.size())
        return fail(I360B_INVALID_PARAM, "Cannot write %s.", path);
    if (fclose(file.f) != 0)
    {
        file.f = nullptr;
        return fail(I360B_INVALID_PARAM, "Cannot write %s.", path);
    }
    file.f = nullptr;
    return I360B_SUCCESS;
}

int require_ready()
{
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    return ensure_ready();
}

int gather_tiles(const unsigned short* const* dTiles, const int* rects, int numTiles, bool skipNull,
                 std::vector<ExportTile>& out)
{
    if (numTiles < 0) return fail(I360B_INVALID_PARAM, "Invalid chunk count.");
    if (numTiles > 0 && (!dTiles || !rects)) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    for (int t = 0; t < numTiles; ++t)
    {
        const int* r = rects + 4 * t;
        if (r[2] <= 0 || r[3] <= 0) return fail(I360B_INVALID_PARAM, "Chunk %d has invalid dimensions.", t);
        if (!dTiles[t])
        {
            if (skipNull) continue;
            return fail(I360B_INVALID_PARAM, "Chunk %d has no output buffer.", t);
        }
        out.push_back(ExportTile{dTiles[t], r[0], r[1], r[2], r[3]});
    }
    return I360B_SUCCESS;
}

void plan_tiles(const i360b_render_plan* plan, bool renderedOnly, std::vector<ExportTile>& out)
{
    const Plan& P = plan->plan;
    for (int t = 0; t < P.nTiles; ++t)
    {
        if (renderedOnly && P.tileListed[t] == 0) continue;  // no render task (PanoramaExporter.cpp:69)
        const int* r = &P.tileRects[(size_t)t * 4];
        out.push_back(ExportTile{P.tiles[t].out, r[0], r[1], r[2], r[3]});
    }
}
}  // namespace

extern "C" int i360b_launch_export_preview(const unsigned short* const* dChunks, const int* rects, int numChunks,
                                           int totalW, int totalH, int maxDimension, unsigned char* dOut,
                                           long long capacity, int* outW, int* outH, void* stream)
{
    clear_error();
    I360B_TRY(require_ready());
    std::vector<ExportTile> tiles;
    I360B_TRY(gather_tiles(dChunks, rects, numChunks, true, tiles));
    return export_preview(tiles, totalW, totalH, maxDimension, dOut, capacity, outW, outH,
                          static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_render_plan_export_preview(i360b_render_plan* plan, int totalW, int totalH, int maxDimension,
                                                unsigned char* dOut, long long capacity, int* outW, int* outH,
                                                void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(require_ready());
    std::vector<ExportTile> tiles;
    plan_tiles(plan, true, tiles);
    return export_preview(tiles, totalW, totalH, maxDimension, dOut, capacity, outW, outH,
                          static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_write_tiff16_chunks(const char* path, const unsigned short* const* dChunks, const int* rects,
                                         int numChunks, int canvasW, int canvasH, void* stream)
{
    clear_error();
    I360B_TRY(require_ready());
    std::vector<ExportTile> tiles;
    I360B_TRY(gather_tiles(dChunks, rects, numChunks, true, tiles));
    return write_tiff(path, tiles, canvasW, canvasH, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_render_plan_write_tiff16(i360b_render_plan* plan, const char* path, int canvasW, int canvasH,
                                              void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(require_ready());
    std::vector<ExportTile> tiles;
    plan_tiles(plan, false, tiles);
    return write_tiff(path, tiles, canvasW, canvasH, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_download_framed(const unsigned short* dData, int width, int height, void* hostOut, void* stream)
{
    clear_error();
    I360B_TRY(require_ready());
    if (!dData || !hostOut) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (width <= 0 || height <= 0) return fail(I360B_INVALID_PARAM, "Invalid dimensions.");
    unsigned char* o = static_cast<unsigned char*>(hostOut);
    put_u32(o, (uint32_t)width);
    put_u32(o + 4, (uint32_t)height);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    I360B_CUDA(cudaMemcpyAsync(o + 8, dData, (size_t)width * height * 6, cudaMemcpyDeviceToHost, s),
               "framed download");
    I360B_CUDA(cudaStreamSynchronize(s), "framed download");
    return I360B_SUCCESS;
}
