// Device data layout and kernels of the seam blend
// (Kernels::SeamBlend::BlendChunkContributors, SeamBlend.cpp:549-587) for a
// batch of output tiles ("chunks"), each with its own contributors ("items").
#pragma once

#include "common.cuh"

namespace i360b
{
constexpr int kMaxBands = 8;
constexpr int kBandRows = 16;  // default rows per CTA of the per-pixel band kernels
constexpr int kSeamRadius = 24;                 // SeamBlend.cpp:319
constexpr int kSeamBand = 2 * kSeamRadius + 1;  // candidates per line
constexpr float kSeamSmooth = 2.0f;             // SeamBlend.cpp:309

// One (tile, contributor) pair.  All buffers live in the plan's arena.
struct ItemDev
{
    const unsigned short* img;  // warped RGB48, tile-sized, (0,0,0) = no data
    uint32_t* cov;              // coverage bits, covWords per row
    float* d1;                  // chamfer forward pass
    float* d;                   // chamfer distance (final)
    int* bbox;                  // x0, y0, x1, y1 of covered pixels (x0 > x1 = empty), then the covered count;
                                // at 8..11 the box of the pixels it owns after the seam step (see kOwnedBox)
    float4* nd;                 // pyramid levels 1.. : (num.rgb, den)
    float* wg;                  // pyramid levels 1.. : weight
    float H[9];                 // destination(tile) -> source(frame) matrix
    const unsigned short* src;  // source frame (render path)
    int srcW, srcH;
    int offX, offY;             // added to tile-local x, y before H
    float gain;
    int tile;
    int k;                      // contributor index inside its tile
    int vx0, vy0, vx1, vy1;     // tile-local box outside which the warp is surely (0,0,0)
};

struct TileDev
{
    int w, h;
    int bands;       // clamped band count (SeamBlend.cpp:457-459)
    int firstItem;   // items [firstItem, firstItem + numItems)
    int numItems;
    int covWords;    // 32-bit words per coverage row
    signed char* owner;
    float* blend;    // levels 1.. : 3 floats per pixel (blended band, then reconstruction)
    unsigned short* out;
    int lw[kMaxBands], lh[kMaxBands];
    long long loff[kMaxBands];  // pixel offset of level l (l >= 1) in the per-level arrays
    float usx[kMaxBands], usy[kMaxBands];  // align-corners scales of Up(level l+1 -> l), FP32 as SeamBlend.cpp:89-90
    // seam scratch
    int* lo;
    int* hi;
    int* prevLine;
    int* chosen;
    int* list;
    float* cost;
    unsigned char* back;
    int maxLines;
};

// A CTA's assignment inside a batched launch: object id and block coords.
struct Unit
{
    int id;
    int bx;
    int by;
    int level;
};

// Default limit of every bounded device wait, in SM cycles (~1 s at B200
// clocks).
constexpr long long kSpinCyclesDefault = 2000000000ll;

// Offset in an item's bbox record of its owned box: x0, y0, x1, y1 of the
// pixels it owns once the seam step has run (a superset: the argmax owner's
// box grown by the seam's contested bands), x0 > x1 when it owns none.
constexpr int kOwnedBox = 8;

struct BlendArgs
{
    ItemDev* items;
    TileDev* tiles;
    // error[0]: set by a kernel that gave up (bounded waits) in this execution;
    // error[1]: the same, kept across executions until the host reads it.
    int* error;
    unsigned long long* seamCycles;    // per-phase SM cycles of the seam kernel (5 counters)
    unsigned long long* seamTile;      // SM cycles of each tile's seam step in the last execution
    int bandRows;                      // rows per band unit (a multiple of 8; the plan's tuning)
    long long spinLimit;               // cycles a bounded wait may last (0: give up at the first miss)
    int half;                          // materialised pyramid levels stored as FP16 (the native mode)
    int gmin;                          // lowest level whose band blend stores G in place of num (see g_at)
};

// Kernel launchers (blend_kernels.cu).
int launch_coverage(const BlendArgs& a, const Unit* units, int n, cudaStream_t s);
// shape 1: staged 128x32 blocks (units: item, block); 0: row bands (units:
// item, band of BlendArgs::bandRows rows).
int launch_warp_tiles(const BlendArgs& a, const Unit* units, int n, int shape, cudaStream_t s);
int launch_dt(const BlendArgs& a, const int* itemList, int n, bool backward, int maxW, int maxH, int slots,
              cudaStream_t s);
int launch_owner(const BlendArgs& a, const Unit* units, int n, cudaStream_t s);
int launch_seam(const BlendArgs& a, const int* tileList, int n, cudaStream_t s);
int launch_down(const BlendArgs& a, const Unit* units, int n, int level, cudaStream_t s);
int launch_blend_level(const BlendArgs& a, const Unit* units, int n, int level, cudaStream_t s);
int launch_collapse(const BlendArgs& a, const Unit* units, int n, int level, cudaStream_t s);
int launch_final0(const BlendArgs& a, const Unit* units, int n, cudaStream_t s);
// Fused pyramid levels 0-1: level 2 of every contributor from level 0
// (units: item, 32x8 blocks of level 2), then per tile the level-1 blend,
// its collapse and the output (units: tile, 64x32 blocks of output pixels).
constexpr int kBase2W = 32, kBase2H = 8, kFineW = 64, kFineH = 32;
// Destination block of one tile-warp CTA (launch_warp_tiles units: item, block).
constexpr int kWarpBlockW = 128, kWarpBlockH = 32;
int launch_base2(const BlendArgs& a, const Unit* units, int n, cudaStream_t s);
int launch_fine(const BlendArgs& a, const Unit* units, int n, bool level1InMemory, cudaStream_t s);
int dt_rows_in_flight(int maxW, int maxH);
}  // namespace i360b
