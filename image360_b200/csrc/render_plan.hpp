// Host-side description of a batched seam-blend render (see render.cu).
#pragma once

#include "blend_kernels.cuh"

#include <utility>
#include <vector>

namespace i360b
{
// One contributor of one tile.  Either `img` (a pre-warped tile-sized RGB48
// device buffer) or the source frame + matrix for the fused warp.
struct ItemSpec
{
    const unsigned short* img = nullptr;
    const unsigned short* src = nullptr;
    int srcW = 0, srcH = 0;
    float H[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    int offX = 0, offY = 0;
    float gain = 1.0f;
    // Tile-local box outside which the warp is surely empty (default: all).
    int vx0 = 0, vy0 = 0, vx1 = 0x3fffffff, vy1 = 0x3fffffff;
    // The 4 edges of the coverage boundary clipped to the tile, {x0, y0, x1,
    // y1} each in tile pixels; NaN x0 = absent (the learned blend's feature).
    float edges[16] = {__builtin_nanf(""), 0, 0, 0, __builtin_nanf(""), 0, 0, 0,
                       __builtin_nanf(""), 0, 0, 0, __builtin_nanf(""), 0, 0, 0};
};

struct TileSpec
{
    int w = 0, h = 0;
    unsigned short* out = nullptr;
    std::vector<ItemSpec> items;
};

constexpr int kStages = 10;
extern const char* const kStageNames[kStages];

struct Range
{
    int start;
    int count;
};

// A 256x256 window of an output tile for the learned blend (partial at the
// tile's right and bottom edges): which contributors reach it.
struct SubTile
{
    int tile, ox, oy, w, h;
    int kind;     // 0 no contributor, 1 one (copied), 2 two to four (network)
    int overflow; // more than 4 reached it; the 4 with the largest overlap kept
    int item[4];  // global item indices, -1 unused
};

struct Plan
{
    bool render = false;
    int nTiles = 0, nItems = 0, nSeam = 0, bandsReq = 0, maxW = 1, maxH = 1;
    // Tuning: rows per band unit of the per-pixel kernels (8, 16, 32 or 64)
    // and ring slots of the chamfer transform (0 = as many as fit).
    int bandRows = kBandRows, dtSlots = 0;
    // Pyramid levels computed on chip (level-fusion depth): 2 = levels 0 and
    // 1 fused (k_base2 + k_fine, only levels >= 2 in memory), 1 = level 1
    // materialised by k_down0s and read by k_fine (the level-1 blend,
    // collapse and output fused), 0 = every level materialised (k_down0s,
    // k_blend_level / k_collapse at level 1, k_final0).
    int fusedLevels = 0;  // the fastest on the 90-tile panorama (the autotuner times all three)
    // Storage of the materialised pyramid levels (levels >= 1, or >= 2 at
    // fusion depth 2): 0 FP32 (exact, the reference's values bit for bit),
    // 1 FP16 with FP32 arithmetic (the native mode).
    int storage16 = 0;
    // Tile-warp form: 1 = staged 128x32 blocks (source footprint in shared
    // memory), 0 = row bands gathering through L1.
    int warpShape = 0;  // the faster form on the 90-tile panorama (the autotuner times both)
    // Limit of the bounded device waits (SM cycles; 0 = give up at the first
    // wait that is not satisfied at once, a test setting).
    long long spinLimit = kSpinCyclesDefault;
    int unitCap = 0;  // units the device list holds (sized for 8-row bands)
    std::vector<ItemDev> items;
    std::vector<TileDev> tiles;
    std::vector<Range> lists;
    void* arena = nullptr;
    size_t arenaBytes = 0;
    Unit* dUnits = nullptr;
    int* dInts = nullptr;
    int* seamList = nullptr;
    ItemDev* dItems = nullptr;
    TileDev* dTiles = nullptr;
    int* dError = nullptr;
    unsigned long long* dSeamCycles = nullptr;
    unsigned long long* dSeamTile = nullptr;  // seam cycles per tile, last execution
    int* hostErr = nullptr;
    std::vector<SubTile> subTiles;  // built on first learned render
    std::vector<float> itemEdges;   // 16 per item (ItemSpec::edges)
    std::vector<int> tileRects;     // x, y, width, height per tile (canvas)
    std::vector<int> tileListed;    // contributors listed per tile (0: no render output)
    // Tiles are independent, so they are split into up to three chains whose
    // stages are enqueued on their own streams inside the graph: the
    // latency-bound stages of one chain (chamfer wavefront, seam search) run
    // beside the full-GPU stages of the others.
    static constexpr int kMaxChains = 3;
    int nChains = 1;
    std::vector<int> tileChain;          // chain of each tile
    Range dtRange[kMaxChains] = {};      // chamfer item lists in dInts, per chain
    Range seamRange[kMaxChains] = {};    // seam tile lists in dInts, per chain
    cudaStream_t side[kMaxChains - 1] = {};     // the streams of chains 1..
    cudaEvent_t evFork = nullptr, evLag = nullptr, evJoin[kMaxChains - 1] = {};
    // Chain stagger: with chainLag = L >= 0, the other chains' first stage of
    // a run waits until chain 0 has finished stage L.  -1: all chains start
    // together.  Ordering only: the render is the same.
    int chainLag = -1;
    // Chain split: 0 = chains of about equal work (area x contributors);
    // p > 0 = tiles in order of their seam step's time in the last execution,
    // slowest first: the first p percent form chain 0, the next p percent
    // chain 1, the rest the last chain - so the slow seam searches (a CTA per
    // tile, sequential over lines) start early and run beside the full-GPU
    // stages of the chains behind them instead of deciding the end of a stage.
    int chainSplit = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;

    Plan() = default;
    Plan(const Plan&) = delete;
    Plan& operator=(const Plan&) = delete;
    ~Plan();

    // With extArena non-null the plan lives in that caller-provided device
    // buffer of extBytes bytes (no allocation; INVALID_PARAM if too small)
    // and its tables are uploaded on stream `s`.
    int build(const std::vector<TileSpec>& specs, int numBands, bool renderPath, void* extArena = nullptr,
              size_t extBytes = 0, cudaStream_t s = nullptr);
    bool ownsArena = true;
    // Enqueues the kernel sequence; with `ev` non-null records ev[i] before
    // stage i and ev[kStages] at the end (stage order of kStageNames).
    int enqueue(cudaStream_t s, cudaEvent_t* ev = nullptr);
    // Only the first stage: bounding-box reset and the warp (render path) or
    // coverage pass, leaving every contributor's tile-space image in the arena.
    int enqueue_warp(cudaStream_t s);
    // One chain's stages from `first` to `last` (kStageNames order, 0 = warp).
    int enqueue_chain(int chain, int first, int last, cudaStream_t s);
    // Stages `first` to `last` of every chain (with ev, one stage at a time).
    int enqueue_range(cudaStream_t s, int first, int last, cudaEvent_t* ev);
    // Stages `first` to `last` as a graph of their own (cached per range).
    int execute_range(cudaStream_t s, int first, int last);
    std::vector<std::pair<int, cudaGraphExec_t>> rangeGraphs;
    int kernels_per_execute() const;
    // Work lists for band height `rows` (fills `lists`).
    void make_units(int rows, std::vector<Unit>& units);
    // Switches the band height and chamfer ring depth; the next execute
    // recaptures the graph.  Synchronous on `s`.
    int set_tuning(int rows, int slots, cudaStream_t s);
    // Switches the level-fusion depth (0, 1 or 2); recaptures on next execute.
    int set_fusion(int levels, cudaStream_t s);
    // Switches the pyramid storage precision (0 exact, 1 FP16).
    int set_precision(int mode, cudaStream_t s);
    // Switches the tile-warp form (0 or 1); remakes the work lists.
    int set_warp_shape(int shape, cudaStream_t s);
    // Sets the chain stagger (-1 or a stage 0-8); recaptures on next execute.
    int set_chain_lag(int stage, cudaStream_t s);
    // Splits the tiles into the chains (see chainSplit); remakes the lists.
    int set_chain_split(int percent, cudaStream_t s);
    void balanced_chains();
    // The chamfer item and seam tile lists per chain into `ints`; returns
    // where the seam tiles start.
    int chain_lists(std::vector<int>& ints);
    // Changes the bounded-wait limit; the next execute recaptures the graph.
    int set_wait_limit(long long cycles, cudaStream_t s);
    void drop_graphs();
    int execute(cudaStream_t s, bool useGraph);
    // Waits for the stream and reports a kernel that gave up (bounded waits)
    // in any execution since the previous check.
    int check(cudaStream_t s);
};
}  // namespace i360b

namespace i360b
{
// Frees the learned-render scratch kept for a plan (learned.cu).
void release_learned_scratch(const Plan* p);
}  // namespace i360b

// The opaque handle of the C-ABI (include/image360_b200.h).
struct i360b_render_plan
{
    i360b::Plan plan;
};
