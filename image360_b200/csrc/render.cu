// Batched seam-blend render of many uneven output tiles.
//
// A plan turns a tile list into flat per-kernel work lists ("units": one CTA
// each) over all tiles at once, carves every intermediate out of one device
// arena, and enqueues the fixed kernel sequence
//     warp(+gain, coverage) -> chamfer fwd -> chamfer bwd -> ownership ->
//     seam DP -> pyramid down x(L-1) -> blended bands -> collapse -> level 0
// which is captured once into a CUDA graph and replayed.  The same machinery
// serves the single-chunk blend API (one tile, pre-warped contributors).
#include "blend_kernels.cuh"
#include "render_plan.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace i360b
{
namespace
{
__global__ void k_init_bbox(ItemDev* items, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int* b = items[i].bbox;
    b[0] = 0x7fffffff;
    b[1] = 0x7fffffff;
    b[2] = -1;
    b[3] = -1;
    b[4] = 0;
    b[kOwnedBox] = 0x7fffffff;
    b[kOwnedBox + 1] = 0x7fffffff;
    b[kOwnedBox + 2] = -1;
    b[kOwnedBox + 3] = -1;
}

// Frame homography -> per-item destination->source matrix.
//  REFERENCE: round the frame->canvas matrix to float, invert it with the FP32
//  adjugate of HomographyMath.cpp:94-116, keep the tile origin as the integer
//  offset RenderExecutor passes (RenderExecutor.cpp:101-108).
//  FP64_ORIGIN: invert in FP64 and fold the tile origin into the matrix in
//  FP64 (H * T(x0, y0)), rounding to float once; offsets become 0.
__global__ void k_setup_items(ItemDev* items, const double* toCanvas, const int* itemFrame, const int* tileXY,
                              int n, int mode, int* singular)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* m = toCanvas + 9 * itemFrame[i];
    ItemDev& it = items[i];
    int tx = tileXY[2 * i], ty = tileXY[2 * i + 1];
    if (mode == I360B_COORDS_REFERENCE)
    {
        float a = (float)m[0], b = (float)m[1], c = (float)m[2], d = (float)m[3], e = (float)m[4], f = (float)m[5],
              g = (float)m[6], i2 = (float)m[7], j = (float)m[8];
        float det = fadd(fsub(fmul(a, fsub(fmul(e, j), fmul(f, i2))), fmul(b, fsub(fmul(d, j), fmul(f, g)))),
                         fmul(c, fsub(fmul(d, i2), fmul(e, g))));
        if (fabsf(det) < 1e-12f)
        {
            singular[i] = 1;
            return;
        }
        float inv = fdiv(1.0f, det);
        it.H[0] = fmul(fsub(fmul(e, j), fmul(f, i2)), inv);
        it.H[1] = fmul(fsub(fmul(c, i2), fmul(b, j)), inv);
        it.H[2] = fmul(fsub(fmul(b, f), fmul(c, e)), inv);
        it.H[3] = fmul(fsub(fmul(f, g), fmul(d, j)), inv);
        it.H[4] = fmul(fsub(fmul(a, j), fmul(c, g)), inv);
        it.H[5] = fmul(fsub(fmul(c, d), fmul(a, f)), inv);
        it.H[6] = fmul(fsub(fmul(d, i2), fmul(e, g)), inv);
        it.H[7] = fmul(fsub(fmul(b, g), fmul(a, i2)), inv);
        it.H[8] = fmul(fsub(fmul(a, e), fmul(b, d)), inv);
        it.offX = tx;
        it.offY = ty;
        singular[i] = 0;
    }
    else
    {
        double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], i2 = m[7], j = m[8];
        double det = a * (e * j - f * i2) - b * (d * j - f * g) + c * (d * i2 - e * g);
        if (fabs(det) < 1e-12)
        {
            singular[i] = 1;
            return;
        }
        double inv = 1.0 / det;
        double Hi[9] = {(e * j - f * i2) * inv, (c * i2 - b * j) * inv, (b * f - c * e) * inv,
                        (f * g - d * j) * inv,  (a * j - c * g) * inv,  (c * d - a * f) * inv,
                        (d * i2 - e * g) * inv, (b * g - a * i2) * inv, (a * e - b * d) * inv};
        for (int r = 0; r < 3; ++r)
        {
            it.H[r * 3 + 0] = (float)Hi[r * 3 + 0];
            it.H[r * 3 + 1] = (float)Hi[r * 3 + 1];
            it.H[r * 3 + 2] = (float)(Hi[r * 3 + 0] * tx + Hi[r * 3 + 1] * ty + Hi[r * 3 + 2]);
        }
        it.offX = 0;
        it.offY = 0;
        singular[i] = 0;
    }
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

__global__ void k_count_cov(const ItemDev* items, const TileDev* tiles, int n, unsigned long long* out)
{
    int i = blockIdx.x;
    if (i >= n) return;
    const ItemDev& it = items[i];
    const TileDev& T = tiles[it.tile];
    long long words = (long long)T.h * T.covWords;
    unsigned long long c = 0;
    for (long long q = threadIdx.x; q < words; q += blockDim.x) c += __popc(it.cov[q]);
    atomicAdd(out, c);
}
}  // namespace

int Plan::build(const std::vector<TileSpec>& specs, int numBands, bool renderPath, void* extArena, size_t extBytes,
                cudaStream_t stream)
{
    render = renderPath;
    nTiles = (int)specs.size();
    if (numBands < 1) return fail(I360B_INVALID_PARAM, "numBands must be >= 1.");
    bandsReq = std::min(numBands, kMaxBands);
    if (numBands > kMaxBands)
        bandsReq = kMaxBands;  // a band count above what any tile can hold is clamped per tile anyway
    // ---- host layout ------------------------------------------------------
    tiles.assign(nTiles, TileDev{});
    items.clear();
    itemEdges.clear();
    size_t bytes = 0;
    struct Off
    {
        size_t warped, cov, d1, d, bbox, nd, wg;
    };
    std::vector<Off> itemOff;
    struct TOff
    {
        size_t owner, blend, lo, hi, prev, chosen, list, cost, back;
    };
    std::vector<TOff> tileOff(nTiles);
    maxW = 1;
    maxH = 1;
    for (int t = 0; t < nTiles; ++t)
    {
        const TileSpec& S = specs[t];
        TileDev& T = tiles[t];
        T.w = S.w;
        T.h = S.h;
        // SeamBlend.cpp:457-459.
        int maxBands = 1;
        {
            int w = S.w, h = S.h;
            while (w > 1 && h > 1 && maxBands < numBands)
            {
                w = (w + 1) / 2;
                h = (h + 1) / 2;
                ++maxBands;
            }
        }
        T.bands = std::min(numBands, std::max(1, maxBands));
        if (T.bands > kMaxBands) return fail(I360B_INVALID_PARAM, "numBands above %d is not supported.", kMaxBands);
        T.firstItem = (int)items.size();
        T.numItems = (int)S.items.size();
        T.covWords = (S.w + 31) / 32;
        T.out = S.out;
        T.maxLines = std::max(S.w, S.h);
        T.lw[0] = S.w;
        T.lh[0] = S.h;
        long long acc = 0;
        T.loff[0] = 0;
        for (int l = 1; l < kMaxBands; ++l)
        {
            T.lw[l] = (T.lw[l - 1] + 1) / 2;
            T.lh[l] = (T.lh[l - 1] + 1) / 2;
            T.loff[l] = acc;
            if (l < T.bands) acc += (long long)T.lw[l] * T.lh[l];
        }
        for (int l = 0; l + 1 < kMaxBands; ++l)
        {
            // SeamBlend.cpp:89-90: (w-1)/max(1, outW-1), 0 when w <= 1 (host
            // float division is IEEE round-to-nearest, as on the device).
            const int sw = T.lw[l + 1], sh = T.lh[l + 1], dw = T.lw[l], dh = T.lh[l];
            T.usx[l] = (sw > 1) ? (float)(sw - 1) / (float)std::max(1, dw - 1) : 0.0f;
            T.usy[l] = (sh > 1) ? (float)(sh - 1) / (float)std::max(1, dh - 1) : 0.0f;
        }
        T.usx[kMaxBands - 1] = T.usy[kMaxBands - 1] = 0.0f;
        size_t pyrPx = (size_t)acc;
        maxW = std::max(maxW, S.w);
        maxH = std::max(maxH, S.h);
        size_t px = (size_t)S.w * S.h;
        TOff& to = tileOff[t];
        to.owner = bytes; bytes += align256(px + 16);  // + 16: the seam scan's 16-byte chunk reads past a row end stay inside
        to.blend = bytes; bytes += align256(std::max<size_t>(pyrPx, 1) * 12);
        size_t ml = (size_t)T.maxLines;
        to.lo = bytes; bytes += align256(ml * 4);
        to.hi = bytes; bytes += align256(ml * 4);
        to.prev = bytes; bytes += align256(ml * 4);
        to.chosen = bytes; bytes += align256(ml * 4);
        to.list = bytes; bytes += align256(ml * 4);
        to.cost = bytes; bytes += align256(ml * kSeamBand * 4);
        to.back = bytes; bytes += align256(ml * kSeamBand);
        for (int k = 0; k < T.numItems; ++k)
        {
            const ItemSpec& I = S.items[k];
            ItemDev it{};
            it.tile = t;
            it.k = k;
            it.img = I.img;
            it.src = I.src;
            it.srcW = I.srcW;
            it.srcH = I.srcH;
            it.gain = I.gain;
            for (int q = 0; q < 9; ++q) it.H[q] = I.H[q];
            it.offX = I.offX;
            it.offY = I.offY;
            it.vx0 = I.vx0;
            it.vy0 = I.vy0;
            it.vx1 = I.vx1;
            it.vy1 = I.vy1;
            Off o{};
            if (renderPath) { o.warped = bytes; bytes += align256(px * 6); }
            o.cov = bytes; bytes += align256((size_t)S.h * T.covWords * 4);
            o.d1 = bytes; bytes += align256(px * 4);
            o.d = bytes; bytes += align256(px * 4);
            o.bbox = bytes; bytes += 256;
            o.nd = bytes; bytes += align256(std::max<size_t>(pyrPx, 1) * 16);
            o.wg = bytes; bytes += align256(std::max<size_t>(pyrPx, 1) * 4);
            items.push_back(it);
            itemOff.push_back(o);
            itemEdges.insert(itemEdges.end(), I.edges, I.edges + 16);
        }
    }
    nItems = (int)items.size();
    // ---- chains: tiles split into groups of about equal work -------------
    nChains = std::min(nTiles, (int)kMaxChains);
    if (nChains < 1) nChains = 1;
    balanced_chains();
    // ---- work lists -------------------------------------------------------
    std::vector<Unit> units;
    {
        // the largest list any band height and warp form needs
        const int shape = warpShape;
        size_t cap = 0;
        for (int ws : {0, 1})
        {
            warpShape = ws;
            make_units(8, units);
            cap = std::max(cap, units.size());
        }
        warpShape = shape;
        unitCap = (int)cap;
    }
    make_units(bandRows, units);
    std::vector<int> ints;
    const int seamStart = chain_lists(ints);
    if (nChains > 1)
    {
        I360B_CUDA(cudaEventCreateWithFlags(&evFork, cudaEventDisableTiming), "chain event");
        I360B_CUDA(cudaEventCreateWithFlags(&evLag, cudaEventDisableTiming), "chain event");
        for (int c = 1; c < nChains; ++c)
        {
            I360B_CUDA(cudaStreamCreateWithFlags(&side[c - 1], cudaStreamNonBlocking), "chain stream");
            I360B_CUDA(cudaEventCreateWithFlags(&evJoin[c - 1], cudaEventDisableTiming), "chain event");
        }
    }
    // ---- device allocation -----------------------------------------------
    size_t unitBytes = align256(std::max<size_t>(unitCap, 1) * sizeof(Unit));
    size_t intBytes = align256(std::max<size_t>(ints.size(), 1) * sizeof(int));
    size_t itemBytes = align256(std::max(nItems, 1) * sizeof(ItemDev));
    size_t tileBytes = align256(std::max(nTiles, 1) * sizeof(TileDev));
    size_t metaOff = bytes;
    bytes += unitBytes + intBytes + itemBytes + tileBytes + 256 + 256 + align256(std::max(nTiles, 1) * 8);
    arenaBytes = bytes;
    if (extArena)
    {
        if (bytes > extBytes)
            return fail(I360B_INVALID_PARAM,
                        "chunk needs %zu bytes of device scratch; the allocation-free entry point holds %zu", bytes,
                        extBytes);
        arena = extArena;
        ownsArena = false;
    }
    else
    {
        if (inject_alloc_failure())
            return fail(I360B_OUT_OF_MEMORY, "render plan: device allocation of %zu bytes failed (injected)", bytes);
        cudaError_t e = cudaMalloc(&arena, bytes);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            arena = nullptr;
            return fail(e == cudaErrorMemoryAllocation ? I360B_OUT_OF_MEMORY : I360B_CUDA_ERROR,
                        "render plan: device allocation of %zu bytes failed (%s)", bytes, cudaGetErrorString(e));
        }
    }
    char* base = static_cast<char*>(arena);
    for (int t = 0; t < nTiles; ++t)
    {
        TileDev& T = tiles[t];
        const TOff& to = tileOff[t];
        T.owner = reinterpret_cast<signed char*>(base + to.owner);
        T.blend = reinterpret_cast<float*>(base + to.blend);
        T.lo = reinterpret_cast<int*>(base + to.lo);
        T.hi = reinterpret_cast<int*>(base + to.hi);
        T.prevLine = reinterpret_cast<int*>(base + to.prev);
        T.chosen = reinterpret_cast<int*>(base + to.chosen);
        T.list = reinterpret_cast<int*>(base + to.list);
        T.cost = reinterpret_cast<float*>(base + to.cost);
        T.back = reinterpret_cast<unsigned char*>(base + to.back);
    }
    for (int i = 0; i < nItems; ++i)
    {
        ItemDev& it = items[i];
        const Off& o = itemOff[i];
        if (renderPath) it.img = reinterpret_cast<unsigned short*>(base + o.warped);
        it.cov = reinterpret_cast<uint32_t*>(base + o.cov);
        it.d1 = reinterpret_cast<float*>(base + o.d1);
        it.d = reinterpret_cast<float*>(base + o.d);
        it.bbox = reinterpret_cast<int*>(base + o.bbox);
        it.nd = reinterpret_cast<float4*>(base + o.nd);
        it.wg = reinterpret_cast<float*>(base + o.wg);
    }
    dUnits = reinterpret_cast<Unit*>(base + metaOff);
    dInts = reinterpret_cast<int*>(base + metaOff + unitBytes);
    dItems = reinterpret_cast<ItemDev*>(base + metaOff + unitBytes + intBytes);
    dTiles = reinterpret_cast<TileDev*>(base + metaOff + unitBytes + intBytes + itemBytes);
    dError = reinterpret_cast<int*>(base + metaOff + unitBytes + intBytes + itemBytes + tileBytes);
    dSeamCycles = reinterpret_cast<unsigned long long*>(base + metaOff + unitBytes + intBytes + itemBytes + tileBytes + 256);
    dSeamTile = reinterpret_cast<unsigned long long*>(base + metaOff + unitBytes + intBytes + itemBytes + tileBytes + 512);
    if (extArena)
    {
        // Caller-provided scratch: upload the tables on the caller's stream
        // (the scratch may still be in use by earlier work on that stream).
        I360B_CUDA(cudaMemcpyAsync(dUnits, units.data(), units.size() * sizeof(Unit), cudaMemcpyHostToDevice, stream),
                   "plan upload");
        I360B_CUDA(cudaMemcpyAsync(dInts, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice, stream),
                   "plan upload");
        if (nItems)
            I360B_CUDA(cudaMemcpyAsync(dItems, items.data(), nItems * sizeof(ItemDev), cudaMemcpyHostToDevice, stream),
                       "plan upload");
        if (nTiles)
            I360B_CUDA(cudaMemcpyAsync(dTiles, tiles.data(), nTiles * sizeof(TileDev), cudaMemcpyHostToDevice, stream),
                       "plan upload");
        I360B_CUDA(cudaMemsetAsync(dError, 0, 2 * sizeof(int), stream), "plan upload");
        I360B_CUDA(cudaMemsetAsync(dSeamCycles, 0, 5 * sizeof(unsigned long long), stream), "plan upload");
        I360B_CUDA(cudaMemsetAsync(dSeamTile, 0, std::max(nTiles, 1) * sizeof(unsigned long long), stream),
                   "plan upload");
        I360B_CUDA(cudaStreamSynchronize(stream), "plan upload");
    }
    else
    {
        I360B_CUDA(cudaMemcpy(dUnits, units.data(), units.size() * sizeof(Unit), cudaMemcpyHostToDevice), "plan upload");
        I360B_CUDA(cudaMemcpy(dInts, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice), "plan upload");
        if (nItems) I360B_CUDA(cudaMemcpy(dItems, items.data(), nItems * sizeof(ItemDev), cudaMemcpyHostToDevice), "plan upload");
        if (nTiles) I360B_CUDA(cudaMemcpy(dTiles, tiles.data(), nTiles * sizeof(TileDev), cudaMemcpyHostToDevice), "plan upload");
        I360B_CUDA(cudaMemset(dError, 0, 2 * sizeof(int)), "plan upload");
        I360B_CUDA(cudaMemset(dSeamCycles, 0, 5 * sizeof(unsigned long long)), "plan upload");
        I360B_CUDA(cudaMemset(dSeamTile, 0, std::max(nTiles, 1) * sizeof(unsigned long long)), "plan upload");
    }
    seamList = dInts + seamStart;
    return I360B_SUCCESS;
}

// Lists per chain, kListsPerChain each (index chain * kListsPerChain + list):
// warp, ownership, level-0 output, down from each level, blend and collapse
// at each level, then the fused pyramid's level-2 base and fine blocks.
constexpr int kListBase2 = 3 + (kMaxBands - 1) + kMaxBands + kMaxBands;
constexpr int kListFine = kListBase2 + 1;
constexpr int kListsPerChain = kListFine + 1;

void Plan::make_units(int rows, std::vector<Unit>& units)
{
    units.clear();
    // Band units: `rows` full-width rows each (per-pixel kernels).
    auto addBands = [&](int id, int h) {
        for (int by = 0; by < (h + rows - 1) / rows; ++by) units.push_back(Unit{id, 0, by, 0});
    };
    // Block units of the pyramid down kernels: bw x 16 outputs each (64 wide
    // for the level-0 step, whose lanes make two columns each; 32 above).
    auto addBlocks = [&](int id, int w, int h, int bw) {
        for (int by = 0; by < (h + 15) / 16; ++by)
            for (int bx = 0; bx < (w + bw - 1) / bw; ++bx) units.push_back(Unit{id, bx, by, 0});
    };
    lists.clear();
    auto beginList = [&]() { return (int)units.size(); };
    auto endList = [&](int start) { lists.push_back(Range{start, (int)units.size() - start}); };
    for (int c = 0; c < nChains; ++c)
    {
        auto inT = [&](int t) { return tileChain.empty() || tileChain[t] == c; };
        auto inI = [&](int i) { return inT(items[i].tile); };
        int s;
        s = beginList();  // 0: warp (render path: 128x16 blocks) / coverage (bands)
        for (int i = 0; i < nItems; ++i)
        {
            if (!inI(i)) continue;
            const TileDev& T = tiles[items[i].tile];
            if (render && warpShape == 1)
            {
                for (int by = 0; by < (T.h + kWarpBlockH - 1) / kWarpBlockH; ++by)
                    for (int bx = 0; bx < (T.w + kWarpBlockW - 1) / kWarpBlockW; ++bx) units.push_back(Unit{i, bx, by, 0});
            }
            else
                addBands(i, T.h);
        }
        endList(s);
        s = beginList();  // 1: ownership
        for (int t = 0; t < nTiles; ++t)
            if (inT(t)) addBands(t, tiles[t].h);
        endList(s);
        s = beginList();  // 2: level 0 output
        for (int t = 0; t < nTiles; ++t)
            if (inT(t)) addBands(t, tiles[t].h);
        endList(s);
        for (int l = 0; l < kMaxBands - 1; ++l)  // 3 + l: down from level l
        {
            s = beginList();
            for (int i = 0; i < nItems; ++i)
            {
                const TileDev& T = tiles[items[i].tile];
                if (inI(i) && T.bands > l + 1) addBlocks(i, T.lw[l + 1], T.lh[l + 1], l == 0 ? 64 : 32);
            }
            endList(s);
        }
        for (int l = 0; l < kMaxBands; ++l)  // 3 + (kMaxBands-1) + l: blend band at level l (l >= 1)
        {
            s = beginList();
            if (l >= 1)
                for (int t = 0; t < nTiles; ++t)
                    if (inT(t) && tiles[t].bands > l) addBands(t, tiles[t].lh[l]);
            endList(s);
        }
        for (int l = 0; l < kMaxBands; ++l)  // 3 + 2*kMaxBands - 1 + l: collapse at level l (1 <= l <= bands-2)
        {
            s = beginList();
            if (l >= 1)
                for (int t = 0; t < nTiles; ++t)
                    if (inT(t) && tiles[t].bands > l + 1) addBands(t, tiles[t].lh[l]);
            endList(s);
        }
        s = beginList();  // kListBase2: level-2 blocks of every contributor of a tile with >= 3 bands
        for (int i = 0; i < nItems; ++i)
        {
            const TileDev& T = tiles[items[i].tile];
            if (!inI(i) || T.bands < 3) continue;
            for (int by = 0; by < (T.lh[2] + kBase2H - 1) / kBase2H; ++by)
                for (int bx = 0; bx < (T.lw[2] + kBase2W - 1) / kBase2W; ++bx) units.push_back(Unit{i, bx, by, 0});
        }
        endList(s);
        s = beginList();  // kListFine: output blocks of every tile
        for (int t = 0; t < nTiles; ++t)
        {
            if (!inT(t)) continue;
            for (int by = 0; by < (tiles[t].h + kFineH - 1) / kFineH; ++by)
                for (int bx = 0; bx < (tiles[t].w + kFineW - 1) / kFineW; ++bx) units.push_back(Unit{t, bx, by, 0});
        }
        endList(s);
    }
}

int Plan::set_tuning(int rows, int slots, cudaStream_t s)
{
    if (rows < 8 || rows > 64 || (rows & 7)) return fail(I360B_INVALID_PARAM, "band rows must be 8..64, a multiple of 8");
    std::vector<Unit> units;
    make_units(rows, units);
    if ((int)units.size() > unitCap) return fail(I360B_INVALID_PARAM, "work list exceeds its capacity");
    I360B_CUDA(cudaStreamSynchronize(s), "plan tuning");
    I360B_CUDA(cudaMemcpyAsync(dUnits, units.data(), units.size() * sizeof(Unit), cudaMemcpyHostToDevice, s),
               "plan tuning");
    I360B_CUDA(cudaStreamSynchronize(s), "plan tuning");
    bandRows = rows;
    dtSlots = slots;
    drop_graphs();
    return I360B_SUCCESS;
}

int Plan::set_warp_shape(int shape, cudaStream_t s)
{
    if (shape != 0 && shape != 1) return fail(I360B_INVALID_PARAM, "warp shape must be 0 or 1");
    const int old = warpShape;
    warpShape = shape;
    const int rc = set_tuning(bandRows, dtSlots, s);  // remakes and uploads the work lists
    if (rc != I360B_SUCCESS) warpShape = old;
    return rc;
}

int Plan::set_precision(int mode, cudaStream_t s)
{
    if (mode != I360B_PRECISION_EXACT && mode != I360B_PRECISION_FP16)
        return fail(I360B_INVALID_PARAM, "Unknown precision mode %d.", mode);
    I360B_CUDA(cudaStreamSynchronize(s), "plan precision");
    storage16 = mode == I360B_PRECISION_FP16 ? 1 : 0;
    drop_graphs();
    return I360B_SUCCESS;
}

void Plan::balanced_chains()
{
    tileChain.assign(nTiles, 0);
    if (nChains < 2) return;
    std::vector<int> order(nTiles);
    for (int t = 0; t < nTiles; ++t) order[t] = t;
    auto load = [&](int t) { return (double)tiles[t].w * tiles[t].h * (1 + tiles[t].numItems); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return load(a) > load(b); });
    double sum[kMaxChains] = {};
    for (int t : order)
    {
        int c = 0;
        for (int q = 1; q < nChains; ++q)
            if (sum[q] < sum[c]) c = q;
        tileChain[t] = c;
        sum[c] += load(t);
    }
}

int Plan::chain_lists(std::vector<int>& ints)
{
    ints.clear();
    for (int c = 0; c < nChains; ++c)
    {
        dtRange[c].start = (int)ints.size();
        for (int i = 0; i < nItems; ++i)
            if (tileChain[items[i].tile] == c) ints.push_back(i);
        dtRange[c].count = (int)ints.size() - dtRange[c].start;
    }
    const int seamStart = (int)ints.size();
    for (int c = 0; c < nChains; ++c)
    {
        seamRange[c].start = (int)ints.size() - seamStart;
        for (int t = 0; t < nTiles; ++t)
            if (tileChain[t] == c && tiles[t].numItems >= 2) ints.push_back(t);
        seamRange[c].count = (int)ints.size() - seamStart - seamRange[c].start;
    }
    nSeam = (int)ints.size() - seamStart;
    return seamStart;
}

int Plan::set_chain_split(int percent, cudaStream_t s)
{
    if (percent < 0 || percent > 50) return fail(I360B_INVALID_PARAM, "chain split must be 0 (balanced) to 50 percent");
    I360B_CUDA(cudaStreamSynchronize(s), "plan chain split");
    if (nChains < 2)
    {
        chainSplit = 0;
        return I360B_SUCCESS;
    }
    if (percent == 0)
        balanced_chains();
    else
    {
        // the seam step's cycles per tile from the last execution: the
        // slowest seams first, in the first chain
        std::vector<unsigned long long> cyc(nTiles);
        I360B_CUDA(cudaMemcpy(cyc.data(), dSeamTile, nTiles * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
                   "plan chain split");
        bool any = false;
        for (unsigned long long v : cyc) any = any || v != 0;
        if (!any) return fail(I360B_INVALID_PARAM, "chain split by seam time needs an execution of the plan first");
        std::vector<int> order(nTiles);
        for (int t = 0; t < nTiles; ++t) order[t] = t;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cyc[a] > cyc[b]; });
        // chain c < nChains - 1 takes the next `percent` of the tiles in that
        // order (at least one), the last chain the rest
        const int per = std::max(1, (nTiles * percent + 50) / 100);
        tileChain.assign(nTiles, nChains - 1);
        for (int k = 0; k < nTiles; ++k)
        {
            const int c = k / per;
            if (c >= nChains - 1 || nTiles - k <= 1) break;  // the last chain keeps at least one tile
            tileChain[order[k]] = c;
        }
    }
    std::vector<int> ints;
    const int seamStart = chain_lists(ints);
    std::vector<Unit> units;
    make_units(bandRows, units);
    if ((int)units.size() > unitCap) return fail(I360B_INVALID_PARAM, "work list exceeds its capacity");
    I360B_CUDA(cudaMemcpy(dInts, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice), "plan chain split");
    I360B_CUDA(cudaMemcpy(dUnits, units.data(), units.size() * sizeof(Unit), cudaMemcpyHostToDevice),
               "plan chain split");
    seamList = dInts + seamStart;
    chainSplit = percent;
    drop_graphs();
    return I360B_SUCCESS;
}

int Plan::set_chain_lag(int stage, cudaStream_t s)
{
    if (stage < -1 || stage >= kStages - 1) return fail(I360B_INVALID_PARAM, "chain stagger must be -1 or a stage 0-8");
    I360B_CUDA(cudaStreamSynchronize(s), "plan stagger");
    chainLag = stage;
    drop_graphs();
    return I360B_SUCCESS;
}

int Plan::set_fusion(int levels, cudaStream_t s)
{
    if (levels < 0 || levels > 2) return fail(I360B_INVALID_PARAM, "fused pyramid levels must be 0, 1 or 2");
    I360B_CUDA(cudaStreamSynchronize(s), "plan fusion");
    fusedLevels = levels;
    drop_graphs();
    return I360B_SUCCESS;
}

void Plan::drop_graphs()
{
    for (auto& g : rangeGraphs) cudaGraphExecDestroy(g.second);
    rangeGraphs.clear();
    if (graphExec) cudaGraphExecDestroy(graphExec);
    if (graph) cudaGraphDestroy(graph);
    graphExec = nullptr;
    graph = nullptr;
}

int Plan::set_wait_limit(long long cycles, cudaStream_t s)
{
    I360B_CUDA(cudaStreamSynchronize(s), "plan wait limit");
    spinLimit = cycles < 0 ? kSpinCyclesDefault : cycles;
    drop_graphs();
    return I360B_SUCCESS;
}

Plan::~Plan()
{
    for (auto& g : rangeGraphs) cudaGraphExecDestroy(g.second);
    for (int c = 0; c + 1 < kMaxChains; ++c)
    {
        if (side[c]) cudaStreamSynchronize(side[c]);
        if (evJoin[c]) cudaEventDestroy(evJoin[c]);
        if (side[c]) cudaStreamDestroy(side[c]);
    }
    if (evFork) cudaEventDestroy(evFork);
    if (evLag) cudaEventDestroy(evLag);
    if (graphExec) cudaGraphExecDestroy(graphExec);
    if (graph) cudaGraphDestroy(graph);
    if (hostErr) cudaFreeHost(hostErr);
    if (arena && ownsArena) cudaFree(arena);
}

// Stages 5-9 with the fused pyramid (depth 2): level 0 -> 2 of every
// contributor; down from level 2; blended bands >= 2; collapse to level 2;
// level-1 blend, collapse and output from level 0.  Depth 1: level 0 -> 1;
// down from level 1; bands >= 2; collapse to level 2; level-1 blend, collapse
// and output reading level 1.  Materialised (depth 0): level 0 -> 1; down
// from level 1; bands >= 1; collapse to level 1; level-0 output.
const char* const kStageNames[kStages] = {"warp_gain_coverage", "chamfer_forward", "chamfer_backward",
                                          "ownership",          "seam_dp",         "pyramid_base",
                                          "pyramid_down",       "blend_bands",     "collapse",
                                          "fine_output"};

int Plan::kernels_per_execute() const
{
    int n = (nItems > 0 ? 1 : 0);  // bbox reset
    const int lo = fusedLevels > 0 ? 2 : 1, downLo = fusedLevels == 2 ? 2 : 1;
    for (int c = 0; c < nChains; ++c)
    {
        const Range* L = &lists[(size_t)c * kListsPerChain];
        n += (L[0].count > 0 ? 1 : 0) + (dtRange[c].count > 0 ? 2 : 0) + (L[1].count > 0 ? 1 : 0) +
             (seamRange[c].count > 0 ? 1 : 0);
        n += fusedLevels == 2 ? (L[kListBase2].count > 0 ? 1 : 0) : (L[3].count > 0 ? 1 : 0);
        n += fusedLevels > 0 ? (L[kListFine].count > 0 ? 1 : 0) : (L[2].count > 0 ? 1 : 0);
        for (int l = downLo; l < kMaxBands - 1; ++l) n += L[3 + l].count > 0 ? 1 : 0;           // down
        for (int l = lo; l < kMaxBands; ++l) n += L[3 + (kMaxBands - 1) + l].count > 0 ? 1 : 0;  // blend
        for (int l = lo; l < kMaxBands; ++l) n += L[3 + 2 * kMaxBands - 1 + l].count > 0 ? 1 : 0;  // collapse
    }
    return n;
}

int Plan::enqueue_warp(cudaStream_t s)
{
    if (nItems > 0) k_init_bbox<<<(nItems + 127) / 128, 128, 0, s>>>(dItems, nItems);
    I360B_TRY(check_launch("bbox init kernel"));
    I360B_CUDA(cudaMemsetAsync(dError, 0, sizeof(int), s), "error flag reset");
    for (int c = 0; c < nChains; ++c) I360B_TRY(enqueue_chain(c, 0, 0, s));
    return I360B_SUCCESS;
}

int Plan::enqueue_chain(int c, int first, int last, cudaStream_t s)
{
    // levels whose band blend stores G in place (see g_at in blend_kernels.cu)
    const int gmin = fusedLevels == 0 ? 1 : 2;
    BlendArgs a{dItems, dTiles, dError, dSeamCycles, dSeamTile, bandRows, spinLimit, storage16, gmin};
    const Range* L = &lists[(size_t)c * kListsPerChain];
    const bool base2 = fusedLevels == 2, fine = fusedLevels > 0;
    const int lo = fine ? 2 : 1;        // lowest level of the materialised blend and collapse
    const int downLo = base2 ? 2 : 1;   // lowest level the down steps start from
    for (int stage = first; stage <= last; ++stage)
    {
        Range r;
        switch (stage)
        {
        case 0:
            r = L[0];
            I360B_TRY(render ? launch_warp_tiles(a, dUnits + r.start, r.count, warpShape, s)
                             : launch_coverage(a, dUnits + r.start, r.count, s));
            break;
        case 1:
        case 2:
            I360B_TRY(launch_dt(a, dInts + dtRange[c].start, dtRange[c].count, stage == 2, maxW, maxH, dtSlots, s));
            break;
        case 3:
            r = L[1];
            I360B_TRY(launch_owner(a, dUnits + r.start, r.count, s));
            break;
        case 4:
            I360B_TRY(launch_seam(a, seamList + seamRange[c].start, seamRange[c].count, s));
            break;
        case 5:  // pyramid base: level 0 -> 2 (depth 2) or level 0 -> 1
            if (base2)
            {
                r = L[kListBase2];
                I360B_TRY(launch_base2(a, dUnits + r.start, r.count, s));
            }
            else
            {
                r = L[3];
                I360B_TRY(launch_down(a, dUnits + r.start, r.count, 0, s));
            }
            break;
        case 6:  // the levels above the base
            for (int l = downLo; l < kMaxBands - 1; ++l)
            {
                r = L[3 + l];
                I360B_TRY(launch_down(a, dUnits + r.start, r.count, l, s));
            }
            break;
        case 7:
            for (int l = kMaxBands - 1; l >= lo; --l)
            {
                r = L[3 + (kMaxBands - 1) + l];
                I360B_TRY(launch_blend_level(a, dUnits + r.start, r.count, l, s));
            }
            break;
        case 8:
            for (int l = kMaxBands - 1; l >= lo; --l)
            {
                r = L[3 + 2 * kMaxBands - 1 + l];
                I360B_TRY(launch_collapse(a, dUnits + r.start, r.count, l, s));
            }
            break;
        case 9:  // depths 1, 2: level-1 blend + collapse + output; else the level-0 output
            r = fine ? L[kListFine] : L[2];
            I360B_TRY(fine ? launch_fine(a, dUnits + r.start, r.count, !base2, s)
                           : launch_final0(a, dUnits + r.start, r.count, s));
            break;
        }
    }
    return I360B_SUCCESS;
}

int Plan::enqueue(cudaStream_t s, cudaEvent_t* ev) { return enqueue_range(s, 0, kStages - 1, ev); }

int Plan::enqueue_range(cudaStream_t s, int first, int last, cudaEvent_t* ev)
{
    if (!ev && nChains > 1)
    {
        // Stage 0's bbox reset and error flag for all items, then each chain's
        // stages on its own stream (chains 1.. forked onto `side`), joined.
        if (first == 0)
        {
            if (nItems > 0) k_init_bbox<<<(nItems + 127) / 128, 128, 0, s>>>(dItems, nItems);
            I360B_TRY(check_launch("bbox init kernel"));
            I360B_CUDA(cudaMemsetAsync(dError, 0, sizeof(int), s), "error flag reset");
        }
        if (chainLag >= first && chainLag < last)
        {
            // staggered: the other chains start once chain 0 has finished stage chainLag
            I360B_TRY(enqueue_chain(0, first, chainLag, s));
            I360B_CUDA(cudaEventRecord(evLag, s), "chain stagger");
            for (int c = 1; c < nChains; ++c) I360B_CUDA(cudaStreamWaitEvent(side[c - 1], evLag, 0), "chain stagger");
            I360B_TRY(enqueue_chain(0, chainLag + 1, last, s));
        }
        else
        {
            I360B_CUDA(cudaEventRecord(evFork, s), "chain fork");
            for (int c = 1; c < nChains; ++c) I360B_CUDA(cudaStreamWaitEvent(side[c - 1], evFork, 0), "chain fork");
            I360B_TRY(enqueue_chain(0, first, last, s));
        }
        for (int c = 1; c < nChains; ++c)
        {
            I360B_TRY(enqueue_chain(c, first, last, side[c - 1]));
            I360B_CUDA(cudaEventRecord(evJoin[c - 1], side[c - 1]), "chain join");
            I360B_CUDA(cudaStreamWaitEvent(s, evJoin[c - 1], 0), "chain join");
        }
        return I360B_SUCCESS;
    }
    // Stage by stage (every chain's part of a stage, forked and joined,
    // before the next stage), so `ev[i]` brackets stage i (kStageNames order)
    // as it runs when the chains overlap.
    auto mark = [&](int i) {
        if (ev) cudaEventRecord(ev[i], s);
    };
    mark(first);
    if (first == 0)
    {
        if (nItems > 0) k_init_bbox<<<(nItems + 127) / 128, 128, 0, s>>>(dItems, nItems);
        I360B_TRY(check_launch("bbox init kernel"));
        I360B_CUDA(cudaMemsetAsync(dError, 0, sizeof(int), s), "error flag reset");
    }
    for (int stage = first; stage <= last; ++stage)
    {
        if (stage > first) mark(stage);
        if (nChains > 1)
        {
            I360B_CUDA(cudaEventRecord(evFork, s), "chain fork");
            for (int c = 1; c < nChains; ++c) I360B_CUDA(cudaStreamWaitEvent(side[c - 1], evFork, 0), "chain fork");
            I360B_TRY(enqueue_chain(0, stage, stage, s));
            for (int c = 1; c < nChains; ++c)
            {
                I360B_TRY(enqueue_chain(c, stage, stage, side[c - 1]));
                I360B_CUDA(cudaEventRecord(evJoin[c - 1], side[c - 1]), "chain join");
                I360B_CUDA(cudaStreamWaitEvent(s, evJoin[c - 1], 0), "chain join");
            }
        }
        else
            I360B_TRY(enqueue_chain(0, stage, stage, s));
    }
    mark(last + 1);
    return I360B_SUCCESS;
}

int Plan::execute(cudaStream_t s, bool useGraph)
{
    if (!useGraph) return enqueue(s);
    if (!graphExec)
    {
        cudaStream_t cap = nullptr;
        I360B_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "graph capture stream");
        I360B_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "graph capture");
        int rc = enqueue(cap);
        cudaError_t e = cudaStreamEndCapture(cap, &graph);
        cudaStreamDestroy(cap);
        if (rc != I360B_SUCCESS) return rc;
        if (e != cudaSuccess) return cuda_fail(e, "graph capture");
        I360B_CUDA(cudaGraphInstantiate(&graphExec, graph, 0), "graph instantiate");
    }
    I360B_CUDA(cudaGraphLaunch(graphExec, s), "graph launch");
    return I360B_SUCCESS;
}

int Plan::execute_range(cudaStream_t s, int first, int last)
{
    if (first == 0 && last == kStages - 1) return execute(s, true);
    if (first < 0 || last >= kStages || first > last) return fail(I360B_INVALID_PARAM, "Invalid stage range.");
    const int key = first * kStages + last;
    for (auto& g : rangeGraphs)
        if (g.first == key)
        {
            I360B_CUDA(cudaGraphLaunch(g.second, s), "graph launch");
            return I360B_SUCCESS;
        }
    cudaStream_t cap = nullptr;
    I360B_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "graph capture stream");
    I360B_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "graph capture");
    int rc = enqueue_range(cap, first, last, nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (rc != I360B_SUCCESS)
    {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "graph capture");
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
    rangeGraphs.push_back({key, x});
    I360B_CUDA(cudaGraphLaunch(x, s), "graph launch");
    return I360B_SUCCESS;
}

int Plan::check(cudaStream_t s)
{
    if (!hostErr) I360B_CUDA(cudaMallocHost(&hostErr, 2 * sizeof(int)), "pinned flag");
    I360B_CUDA(cudaMemcpyAsync(hostErr, dError, 2 * sizeof(int), cudaMemcpyDeviceToHost, s), "error flag readback");
    I360B_CUDA(cudaStreamSynchronize(s), "render synchronize");
    // error[1] holds a give-up of any execution since the last check (each
    // execution clears error[0] when it starts), so a failed run is reported
    // even when later runs of the same plan succeeded.
    if (hostErr[0] || hostErr[1])
    {
        I360B_CUDA(cudaMemsetAsync(dError + 1, 0, sizeof(int), s), "error flag reset");
        I360B_CUDA(cudaStreamSynchronize(s), "error flag reset");
        return fail(I360B_KERNEL_LAUNCH_FAILED, "A render kernel gave up waiting (bounded spin); output invalid.");
    }
    return I360B_SUCCESS;
}

// Device-side setup of render-path items: matrices, singular contributors.
int setup_render_items(const std::vector<double>& toCanvas, const std::vector<int>& itemFrame,
                       const std::vector<int>& tileXY, int mode, std::vector<float>& Hout, std::vector<int>& offOut,
                       std::vector<int>& singular)
{
    int n = (int)itemFrame.size();
    Hout.assign((size_t)n * 9, 0.0f);
    offOut.assign((size_t)n * 2, 0);
    singular.assign(n, 0);
    if (n == 0) return I360B_SUCCESS;
    cudaStream_t s = thread_stream();
    void *dM = nullptr, *dF = nullptr, *dXY = nullptr, *dS = nullptr, *dIt = nullptr;
    int rc = I360B_SUCCESS;
    std::vector<ItemDev> tmp(n);
    if ((rc = dev_alloc(&dM, toCanvas.size() * 8, s, "setup")) || (rc = dev_alloc(&dF, n * 4, s, "setup")) ||
        (rc = dev_alloc(&dXY, n * 8, s, "setup")) || (rc = dev_alloc(&dS, n * 4, s, "setup")) ||
        (rc = dev_alloc(&dIt, n * sizeof(ItemDev), s, "setup")))
        goto done;
    cudaMemcpyAsync(dM, toCanvas.data(), toCanvas.size() * 8, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dF, itemFrame.data(), n * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dXY, tileXY.data(), n * 8, cudaMemcpyHostToDevice, s);
    k_setup_items<<<(n + 127) / 128, 128, 0, s>>>(static_cast<ItemDev*>(dIt), static_cast<double*>(dM),
                                                 static_cast<int*>(dF), static_cast<int*>(dXY), n, mode,
                                                 static_cast<int*>(dS));
    if ((rc = check_launch("homography setup kernel"))) goto done;
    cudaMemcpyAsync(tmp.data(), dIt, n * sizeof(ItemDev), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(singular.data(), dS, n * 4, cudaMemcpyDeviceToHost, s);
    {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { rc = cuda_fail(e, "homography setup"); goto done; }
    }
    for (int i = 0; i < n; ++i)
    {
        for (int q = 0; q < 9; ++q) Hout[(size_t)i * 9 + q] = tmp[i].H[q];
        offOut[2 * i] = tmp[i].offX;
        offOut[2 * i + 1] = tmp[i].offY;
    }
done:
    dev_free(dM, s);
    dev_free(dF, s);
    dev_free(dXY, s);
    dev_free(dS, s);
    dev_free(dIt, s);
    return rc;
}

int launch_blend_chunk(const unsigned short* const* warped, int k, int w, int h, int bands, unsigned short* out,
                       cudaStream_t s)
{
    std::vector<TileSpec> specs(1);
    specs[0].w = w;
    specs[0].h = h;
    specs[0].out = out;
    for (int i = 0; i < k; ++i)
    {
        ItemSpec it{};
        it.img = warped[i];
        specs[0].items.push_back(it);
    }
    Plan p;
    I360B_TRY(p.build(specs, bands, false));
    I360B_TRY(p.execute(s, false));
    return p.check(s);
}

int launch_blend_chunk_in(void* arena, size_t arenaBytes, const unsigned short* const* warped, int k, int w, int h,
                          int bands, unsigned short* out, cudaStream_t s)
{
    std::vector<TileSpec> specs(1);
    specs[0].w = w;
    specs[0].h = h;
    specs[0].out = out;
    for (int i = 0; i < k; ++i)
    {
        ItemSpec it{};
        it.img = warped[i];
        specs[0].items.push_back(it);
    }
    Plan p;
    I360B_TRY(p.build(specs, bands, false, arena, arenaBytes, s));
    I360B_TRY(p.enqueue(s));
    // Status of the bounded waits, read without a pinned staging buffer.
    int flag = 0;
    I360B_CUDA(cudaMemcpyAsync(&flag, p.dError + 1, sizeof(int), cudaMemcpyDeviceToHost, s), "error flag readback");
    I360B_CUDA(cudaStreamSynchronize(s), "blend synchronize");
    if (flag) return fail(I360B_KERNEL_LAUNCH_FAILED, "A blend kernel gave up waiting (bounded spin); output invalid.");
    return I360B_SUCCESS;
}
}  // namespace i360b

// ---------------------------------------------------------------------------
// C-ABI: render plans.
// ---------------------------------------------------------------------------
using namespace i360b;

namespace
{
// The coverage boundary of a frame in tile coordinates: the warp writes
// destination pixel (x, y) when its source position lies in [0, srcW-1) x
// [0, srcH-1), so the boundary is that source rectangle mapped by the
// frame->canvas homography (FP64) and shifted by the tile origin.  Each of
// its 4 edges is clipped to the tile's pixel centres [0, w-1] x [0, h-1]
// (Liang-Barsky); an edge outside the tile is absent (NaN x0).
void coverage_edges(const double* m, int srcW, int srcH, int tx, int ty, int w, int h, float* out)
{
    const double sx[4] = {0.0, (double)(srcW - 1), (double)(srcW - 1), 0.0};
    const double sy[4] = {0.0, 0.0, (double)(srcH - 1), (double)(srcH - 1)};
    double px[4], py[4];
    for (int q = 0; q < 4; ++q)
    {
        const double wq = m[6] * sx[q] + m[7] * sy[q] + m[8];
        px[q] = (m[0] * sx[q] + m[1] * sy[q] + m[2]) / wq - tx;
        py[q] = (m[3] * sx[q] + m[4] * sy[q] + m[5]) / wq - ty;
    }
    for (int e = 0; e < 4; ++e)
    {
        const double x0 = px[e], y0 = py[e], dx = px[(e + 1) & 3] - x0, dy = py[(e + 1) & 3] - y0;
        double t0 = 0.0, t1 = 1.0;
        const double pp[4] = {-dx, dx, -dy, dy};
        const double qq[4] = {x0 - 0.0, (w - 1) - x0, y0 - 0.0, (h - 1) - y0};
        bool in = true;
        for (int k = 0; k < 4 && in; ++k)
        {
            if (pp[k] == 0.0)
            {
                if (qq[k] < 0.0) in = false;
            }
            else
            {
                const double r = qq[k] / pp[k];
                if (pp[k] < 0.0) t0 = std::max(t0, r);
                else t1 = std::min(t1, r);
                if (t0 > t1) in = false;
            }
        }
        float* o = out + 4 * e;
        if (!in)
        {
            o[0] = __builtin_nanf("");
            o[1] = o[2] = o[3] = 0.0f;
            continue;
        }
        o[0] = (float)(x0 + t0 * dx);
        o[1] = (float)(y0 + t0 * dy);
        o[2] = (float)(x0 + t1 * dx);
        o[3] = (float)(y0 + t1 * dy);
    }
}
}  // namespace

extern "C" int i360b_render_plan_create(const i360b_frame* frames, int numFrames, const i360b_tile* tiles,
                                        int numTiles, const int* contributors, int numBands, int coordMode,
                                        i360b_render_plan** outPlan)
{
    clear_error();
    if (!outPlan) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    *outPlan = nullptr;
    if (!frames || !tiles || numFrames <= 0 || numTiles <= 0) return fail(I360B_INVALID_PARAM, "Null or empty frame/tile list.");
    if (numBands < 1) return fail(I360B_INVALID_PARAM, "numBands must be >= 1.");
    if (coordMode != I360B_COORDS_REFERENCE && coordMode != I360B_COORDS_FP64_ORIGIN)
        return fail(I360B_INVALID_PARAM, "Unknown coordinate mode %d.", coordMode);
    I360B_TRY(ensure_ready());
    for (int f = 0; f < numFrames; ++f)
        if (!frames[f].rgb || frames[f].width <= 0 || frames[f].height <= 0)
            return fail(I360B_INVALID_PARAM, "Frame %d has a null buffer or invalid dimensions.", f);
    std::vector<double> M((size_t)numFrames * 9);
    for (int f = 0; f < numFrames; ++f)
        for (int q = 0; q < 9; ++q) M[(size_t)f * 9 + q] = frames[f].toCanvas[q];
    std::vector<int> itemFrame, tileXY;
    for (int t = 0; t < numTiles; ++t)
    {
        const i360b_tile& T = tiles[t];
        if (T.width <= 0 || T.height <= 0 || !T.dOut || T.count < 0 || T.first < 0)
            return fail(I360B_INVALID_PARAM, "Tile %d has invalid geometry or a null output.", t);
        if (T.count > 0 && !contributors) return fail(I360B_INVALID_PARAM, "Null contributor list.");
        if (T.count > kMaxContributors) return fail(I360B_INVALID_PARAM, "Tile %d has %d contributors (max %d).", t, T.count, kMaxContributors);
        for (int k = 0; k < T.count; ++k)
        {
            int f = contributors[T.first + k];
            if (f < 0 || f >= numFrames) return fail(I360B_INVALID_PARAM, "Tile %d names frame %d.", t, f);
            itemFrame.push_back(f);
            tileXY.push_back(T.x);
            tileXY.push_back(T.y);
        }
    }
    std::vector<float> H;
    std::vector<int> off, singular;
    I360B_TRY(setup_render_items(M, itemFrame, tileXY, coordMode, H, off, singular));
    std::vector<TileSpec> specs(numTiles);
    int idx = 0;
    for (int t = 0; t < numTiles; ++t)
    {
        const i360b_tile& T = tiles[t];
        specs[t].w = T.width;
        specs[t].h = T.height;
        specs[t].out = T.dOut;
        for (int k = 0; k < T.count; ++k, ++idx)
        {
            // RenderExecutor.cpp:102 skips a contributor whose homography does
            // not invert; it then takes no part in the blend.
            if (singular[idx]) continue;
            const i360b_frame& F = frames[contributors[T.first + k]];
            ItemSpec it{};
            it.src = F.rgb;
            it.srcW = F.width;
            it.srcH = F.height;
            it.gain = F.gain;
            for (int q = 0; q < 9; ++q) it.H[q] = H[(size_t)idx * 9 + q];
            it.offX = off[2 * idx];
            it.offY = off[2 * idx + 1];
            // Canvas footprint of the frame (corners through the FP64
            // homography) in tile coordinates, widened by 2 px: outside it
            // every destination pixel maps outside the source, so the tile
            // warp writes (0,0,0) there without evaluating the mapping.  Only
            // used when the frame->canvas map keeps w > 0 at the corners.
            {
                const double* m = F.toCanvas;
                double mnx = 1e300, mny = 1e300, mxx = -1e300, mxy = -1e300;
                bool ok = true;
                const double cx[4] = {0.0, (double)F.width, 0.0, (double)F.width};
                const double cy[4] = {0.0, 0.0, (double)F.height, (double)F.height};
                for (int q = 0; q < 4; ++q)
                {
                    double wq = m[6] * cx[q] + m[7] * cy[q] + m[8];
                    if (!(wq > 1e-9)) { ok = false; break; }
                    double px = (m[0] * cx[q] + m[1] * cy[q] + m[2]) / wq;
                    double py = (m[3] * cx[q] + m[4] * cy[q] + m[5]) / wq;
                    mnx = std::min(mnx, px); mxx = std::max(mxx, px);
                    mny = std::min(mny, py); mxy = std::max(mxy, py);
                }
                if (ok)
                {
                    it.vx0 = (int)std::max(-1.0, std::floor(mnx - 2.0 - T.x));
                    it.vy0 = (int)std::max(-1.0, std::floor(mny - 2.0 - T.y));
                    it.vx1 = (int)std::min((double)T.width, std::ceil(mxx + 2.0 - T.x));
                    it.vy1 = (int)std::min((double)T.height, std::ceil(mxy + 2.0 - T.y));
                    coverage_edges(m, F.width, F.height, T.x, T.y, T.width, T.height, it.edges);
                }
            }
            specs[t].items.push_back(it);
        }
    }
    auto* p = new (std::nothrow) i360b_render_plan;
    if (!p) return fail(I360B_OUT_OF_MEMORY, "Host allocation failed.");
    int rc = p->plan.build(specs, numBands, true);
    if (rc != I360B_SUCCESS)
    {
        delete p;
        return rc;
    }
    p->plan.tileRects.resize((size_t)numTiles * 4);
    p->plan.tileListed.resize(numTiles);
    for (int t = 0; t < numTiles; ++t)
    {
        const int r[4] = {tiles[t].x, tiles[t].y, tiles[t].width, tiles[t].height};
        for (int q = 0; q < 4; ++q) p->plan.tileRects[(size_t)t * 4 + q] = r[q];
        p->plan.tileListed[t] = tiles[t].count;
    }
    *outPlan = p;
    return I360B_SUCCESS;
}

extern "C" int i360b_render_plan_execute(i360b_render_plan* plan, void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    return plan->plan.execute(static_cast<cudaStream_t>(stream), true);
}

extern "C" int i360b_render_plan_execute_stages(i360b_render_plan* plan, int firstStage, int lastStage,
                                                void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    return plan->plan.execute_range(static_cast<cudaStream_t>(stream), firstStage, lastStage);
}

extern "C" int i360b_render_plan_wait(i360b_render_plan* plan, void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    return plan->plan.check(static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_render_plan_autotune(i360b_render_plan* plan, void* stream, int* bandRows, int* dtSlots,
                                          float* bestMs)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    Plan& P = plan->plan;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int maxSlots = dt_rows_in_flight(P.maxW, P.maxH);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    I360B_CUDA(cudaEventCreate(&e0), "autotune events");
    I360B_CUDA(cudaEventCreate(&e1), "autotune events");
    int bestR = P.bandRows, bestS = P.dtSlots, bestF = P.fusedLevels, bestW = P.warpShape;
    float best = INFINITY;
    int rc = I360B_SUCCESS;
    // One trial: a warm-up run (which also captures the graphs), then two
    // timed runs, each in the form that lets a caller refill the frames early:
    // stage 0, then stages 1-9 (execute_stages).
    auto run = [&]() -> int {
        int r = P.execute_range(s, 0, 0);
        return r == I360B_SUCCESS ? P.execute_range(s, 1, kStages - 1) : r;
    };
    auto trial = [&](float& ms) -> int {
        int r = run();
        if (r != I360B_SUCCESS) return r;
        cudaEventRecord(e0, s);
        for (int k = 0; k < 2 && r == I360B_SUCCESS; ++k) r = run();
        cudaEventRecord(e1, s);
        if (r == I360B_SUCCESS) r = P.check(s);
        ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        return r;
    };
    // 1: warp form x fusion depth at the current band height and ring depth
    for (int shape : {1, 0})
    {
        for (int fused : {2, 1, 0})
        {
            if ((rc = P.set_warp_shape(shape, s)) != I360B_SUCCESS || (rc = P.set_fusion(fused, s)) != I360B_SUCCESS)
                break;
            float ms;
            if ((rc = trial(ms)) != I360B_SUCCESS) break;
            if (ms < best)
            {
                best = ms;
                bestW = shape;
                bestF = fused;
            }
        }
        if (rc != I360B_SUCCESS) break;
    }
    // 2: band height x ring depth with those
    if (rc == I360B_SUCCESS && (rc = P.set_warp_shape(bestW, s)) == I360B_SUCCESS &&
        (rc = P.set_fusion(bestF, s)) == I360B_SUCCESS)
    {
        for (int rows : {8, 16, 32, 64})
        {
            for (int slots = 2; slots <= maxSlots && rc == I360B_SUCCESS; ++slots)
            {
                if ((rc = P.set_tuning(rows, slots, s)) != I360B_SUCCESS) break;
                float ms;
                if ((rc = trial(ms)) != I360B_SUCCESS) break;
                if (ms < best)
                {
                    best = ms;
                    bestR = rows;
                    bestS = slots;
                }
            }
            if (rc != I360B_SUCCESS) break;
        }
    }
    // 3: chain split by seam time (several chains only), with the best of the above
    int bestP = P.chainSplit;
    if (rc == I360B_SUCCESS && P.nChains > 1 && (rc = P.set_tuning(bestR, bestS, s)) == I360B_SUCCESS)
    {
        for (int pct : {0, 5, 10, 15, 20, 30})
        {
            if ((rc = P.set_chain_split(pct, s)) != I360B_SUCCESS) break;
            float ms;
            if ((rc = trial(ms)) != I360B_SUCCESS) break;
            if (ms < best)
            {
                best = ms;
                bestP = pct;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != I360B_SUCCESS) return rc;
    I360B_TRY(P.set_warp_shape(bestW, s));
    I360B_TRY(P.set_fusion(bestF, s));
    I360B_TRY(P.set_chain_split(bestP, s));
    I360B_TRY(P.set_tuning(bestR, bestS, s));
    if (bandRows) *bandRows = bestR;
    if (dtSlots) *dtSlots = bestS;
    if (bestMs) *bestMs = best / 2.0f;
    return I360B_SUCCESS;
}

extern "C" int i360b_render_plan_set_chain_lag(i360b_render_plan* plan, int stage, void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    return plan->plan.set_chain_lag(stage, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_render_plan_set_chain_split(i360b_render_plan* plan, int percent, void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    return plan->plan.set_chain_split(percent, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_render_plan_seam_tile_cycles(i360b_render_plan* plan, unsigned long long* cycles, int maxTiles,
                                                  void* stream)
{
    clear_error();
    if (!plan || (!cycles && maxTiles > 0)) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    I360B_TRY(ensure_ready());
    Plan& P = plan->plan;
    const int n = std::min(maxTiles, P.nTiles);
    if (n <= 0) return I360B_SUCCESS;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    I360B_CUDA(cudaMemcpyAsync(cycles, P.dSeamTile, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
               "seam tile cycles");
    I360B_CUDA(cudaStreamSynchronize(s), "seam tile cycles");
    return I360B_SUCCESS;
}

extern "C" int i360b_render_plan_get_chain_split(i360b_render_plan* plan, int* percent)
{
    clear_error();
    if (!plan || !percent) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    *percent = plan->plan.chainSplit;
    return I360B_SUCCESS;
}

extern "C" int i360b_render_plan_get_chain_lag(i360b_render_plan* plan, int* stage)
{
    clear_error();
    if (!plan || !stage) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    *stage = plan->plan.nChains > 1 ? plan->plan.chainLag : -1;
    return I360B_SUCCESS;
}

extern "C" int i360b_render_plan_get_tuning(i360b_render_plan* plan, int* bandRows, int* dtSlots, int* fusedLevels,
                                            int* warpShape)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    if (bandRows) *bandRows = plan->plan.bandRows;
    if (dtSlots) *dtSlots = plan->plan.dtSlots;
    if (fusedLevels) *fusedLevels = plan->plan.fusedLevels;
    if (warpShape) *warpShape = plan->plan.warpShape;
    return I360B_SUCCESS;
}

extern "C" int i360b_render_plan_set_tuning(i360b_render_plan* plan, int bandRows, int dtSlots, int fusedLevels,
                                            int warpShape, void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int maxSlots = dt_rows_in_flight(plan->plan.maxW, plan->plan.maxH);
    if (dtSlots != 0 && (dtSlots < 2 || dtSlots > maxSlots))
        return fail(I360B_INVALID_PARAM, "dtSlots must be 0 or 2-%d for this plan.", maxSlots);
    if (warpShape != 0 && warpShape != 1) return fail(I360B_INVALID_PARAM, "warp shape must be 0 or 1");
    I360B_TRY(plan->plan.set_fusion(fusedLevels, s));
    plan->plan.warpShape = warpShape;
    return plan->plan.set_tuning(bandRows, dtSlots, s);
}

extern "C" int i360b_render_plan_set_precision(i360b_render_plan* plan, int mode, void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    return plan->plan.set_precision(mode, static_cast<cudaStream_t>(stream));
}

extern "C" int i360b_render_plan_set_wait_limit(i360b_render_plan* plan, long long cycles, void* stream)
{
    clear_error();
    if (!plan) return fail(I360B_INVALID_PARAM, "Null plan.");
    I360B_TRY(ensure_ready());
    return plan->plan.set_wait_limit(cycles, static_cast<cudaStream_t>(stream));
}

extern "C" size_t i360b_render_plan_scratch_bytes(const i360b_render_plan* plan)
{
    return plan ? plan->plan.arenaBytes : 0;
}

extern "C" void i360b_render_plan_destroy(i360b_render_plan* plan)
{
    if (!plan) return;
    cudaDeviceSynchronize();
    release_learned_scratch(&plan->plan);
    delete plan;
}


extern "C" int i360b_render_plan_stats(i360b_render_plan* plan, void* stream, i360b_render_stats* out)
{
    clear_error();
    if (!plan || !out) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    I360B_TRY(ensure_ready());
    Plan& P = plan->plan;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::memset(out, 0, sizeof(*out));
    out->numTiles = P.nTiles;
    out->numItems = P.nItems;
    out->kernelsPerExecute = P.kernels_per_execute();
    long long px = 0;
    for (const TileDev& T : P.tiles) px += (long long)T.w * T.h;
    out->outputPixels = px;
    out->scratchBytes = (long long)P.arenaBytes;
    void* d = nullptr;
    I360B_TRY(dev_alloc(&d, sizeof(unsigned long long), s, "stats"));
    cudaMemsetAsync(d, 0, sizeof(unsigned long long), s);
    if (P.nItems > 0)
        k_count_cov<<<P.nItems, 256, 0, s>>>(P.dItems, P.dTiles, P.nItems, static_cast<unsigned long long*>(d));
    unsigned long long c = 0;
    cudaMemcpyAsync(&c, d, sizeof(c), cudaMemcpyDeviceToHost, s);
    dev_free(d, s);
    I360B_CUDA(cudaStreamSynchronize(s), "stats");
    out->coveredItemPixels = (long long)c;
    unsigned long long cyc[5];
    I360B_CUDA(cudaMemcpy(cyc, P.dSeamCycles, sizeof(cyc), cudaMemcpyDeviceToHost), "stats");
    for (int i = 0; i < 5; ++i) out->seamPhaseCycles[i] = (long long)cyc[i];
    return I360B_SUCCESS;
}

extern "C" int i360b_render_plan_profile(i360b_render_plan* plan, void* stream, float* stageMs, int maxStages)
{
    clear_error();
    if (!plan || !stageMs) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    I360B_TRY(ensure_ready());
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t ev[kStages + 1];
    for (int i = 0; i <= kStages; ++i) I360B_CUDA(cudaEventCreate(&ev[i]), "profile events");
    int rc = plan->plan.enqueue(s, ev);
    if (rc == I360B_SUCCESS) rc = plan->plan.check(s);
    for (int i = 0; i < kStages && i < maxStages && rc == I360B_SUCCESS; ++i)
        cudaEventElapsedTime(&stageMs[i], ev[i], ev[i + 1]);
    for (int i = 0; i <= kStages; ++i) cudaEventDestroy(ev[i]);
    return rc;
}

extern "C" const char* i360b_render_stage_name(int stage)
{
    return (stage >= 0 && stage < kStages) ? kStageNames[stage] : "";
}
