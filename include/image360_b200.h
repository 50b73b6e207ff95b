/*
 * image360_b200 - B200 (sm_100a) render backend for the Image360 stitching
 * engine: the C-ABI boundary.
 *
 * Every entry point takes plain pointers and sizes and returns an int that is
 * numerically identical to WindowsApp::Compute::ComputeResult
 * (WindowsApp.Compute/HeaderFiles/ComputeTypes.h:32-50).  No exception ever
 * crosses this boundary.  The last error message is kept per calling thread
 * (the reference keeps one char[512] per backend object,
 * WindowsApp.Core/HeaderFiles/CpuComputeBackend.h:88; calls arrive from several
 * TaskScheduler threads at once, TaskScheduler.cpp:67, so a per-thread message
 * is what makes GetLastError() meaningful here).
 *
 * Two kinds of entry point:
 *   - i360b_<op>: the IComputeBackend operations.  Host buffers in, host
 *     buffers out, synchronous: results are in host memory on return.  Each
 *     calling thread gets its own CUDA stream.  Device memory comes from a
 *     stream-ordered pool that is kept for the life of the process.
 *   - i360b_launch_<op> / i360b_render_*: device-resident, stream-ordered
 *     launchers for callers that keep frames in HBM.  `stream` is a
 *     cudaStream_t passed as void* (NULL = the legacy default stream).
 *
 * Pixel format: RGB48 = interleaved unsigned short x3, row-major; (0,0,0)
 * means "no data" (WindowsApp.Core/SourceFiles/SeamBlend.cpp:565).
 */
#ifndef IMAGE360_B200_H
#define IMAGE360_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define I360B_API __attribute__((visibility("default")))
#else
#define I360B_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ComputeResult values (ComputeTypes.h:32-50). */
enum
{
    I360B_SUCCESS = 0,
    I360B_NO_GPU = 1,
    I360B_INVALID_PARAM = 2,
    I360B_OUT_OF_MEMORY = 3,
    I360B_KERNEL_LAUNCH_FAILED = 4,
    I360B_CUDA_ERROR = 5,
    I360B_NOT_SUPPORTED = 6
};

/* Mirrors WindowsApp::Compute::GpuInfo (ComputeTypes.h:18-29), with the bool
 * stored as int for a stable C layout. */
typedef struct i360b_gpu_info
{
    int deviceId;
    char name[256];
    size_t totalMemory;
    size_t freeMemory;
    int computeMajor;
    int computeMinor;
    int maxThreadsPerBlock;
    int multiProcessorCount;
    int hasTensorCores;
} i360b_gpu_info;

/* ---- lifecycle: IComputeBackend::Initialize/Shutdown/IsInitialized/
 *      GetGpuInfo/GetLastError (IComputeBackend.h:21-25) ---------------- */

/* Picks the visible device with the most memory (as CudaPipeline::Initialize
 * does, CudaPipeline.cpp:137-152) and requires compute capability 10.x.
 * Returns I360B_NO_GPU when there is none. */
I360B_API int i360b_initialize(void);
I360B_API void i360b_shutdown(void);
I360B_API int i360b_is_initialized(void);
I360B_API int i360b_get_gpu_info(i360b_gpu_info* out);
/* Last error message of the calling thread ("" when none). */
I360B_API const char* i360b_get_last_error(void);
/* Records "<op> is not supported by the B200 backend" as the calling thread's
 * last error and returns I360B_NOT_SUPPORTED: the result of the eight
 * IComputeBackend operations outside the render path (IComputeBackend.h:53-168). */
I360B_API int i360b_not_supported(const char* op);

/* ---- IComputeBackend host-buffer operations ---------------------------- */

/* IComputeBackend::WarpPerspective (IComputeBackend.h:29-32).  Backward
 * bilinear warp; `homography` is 9 floats, row-major, mapping DESTINATION
 * pixel (x+offsetX, y+offsetY) to SOURCE (WarpPerspectiveKernels.h:46-53).
 * Out-of-bounds or singular pixels are written as (0,0,0). */
I360B_API int i360b_warp_perspective(const unsigned short* srcData, int srcW, int srcH, unsigned short* dstData,
                           int dstW, int dstH, const float* homography, int offsetX, int offsetY);

/* IComputeBackend::MedianStack (IComputeBackend.h:35-38).  numInputs must be
 * 1..32 (CpuComputeBackend.cpp:143).  Each input is width*height*3 values. */
I360B_API int i360b_median_stack(const unsigned short* const* inputs, int numInputs, unsigned short* output, int width,
                       int height, float sigmaThreshold);

/* IComputeBackend::ApplyGain (IComputeBackend.h:41-42).  numPixels counts
 * unsigned shorts (RenderExecutor passes width*height*3). */
I360B_API int i360b_apply_gain(unsigned short* data, int numPixels, float gain);

/* IComputeBackend::ComputeLabStats (IComputeBackend.h:65-67; CPU semantics
 * GainColorOps.cpp:103-130): mean and standard deviation of CIE L, a, b over
 * an RGB48 image (sRGB 16-bit -> linear -> XYZ -> Lab per pixel).  The
 * per-pixel conversion is the reference's FP32 arithmetic with correctly
 * rounded powers and cube roots, the sums are FP64 (reduction order differs
 * from the reference's sequential loop, so results agree to FP64 rounding). */
I360B_API int i360b_compute_lab_stats(const unsigned short* rgb, int width, int height, double outMean[3],
                                      double outStd[3]);

/* IComputeBackend::ApplyReinhardColorTransfer (IComputeBackend.h:69-73; CPU
 * semantics GainColorOps.cpp:132-156): in place, Lab of each pixel mapped to
 * (lab - srcMean) * (refStd / srcStd) + refMean (srcStd <= 1e-6 taken as 1)
 * and back to RGB48.  Outputs agree with the reference within 1 LSB (its libm
 * powf/cbrtf are not correctly rounded). */
I360B_API int i360b_apply_reinhard_color_transfer(unsigned short* rgbInOut, int width, int height,
                                                  const double srcMean[3], const double srcStd[3],
                                                  const double refMean[3], const double refStd[3]);

/* IComputeBackend::DemosaicBayer (IComputeBackend.h:46-49).  rgbCam is the
 * 3x4 matrix as 12 floats, row-major. */
I360B_API int i360b_demosaic_bayer(const unsigned short* cfaData, int width, int height, unsigned short blackLevel,
                         const float camMul[4], const float rgbCam[12], uint32_t filters, unsigned short* rgbOut);

/* ---- blend extension (no IComputeBackend counterpart) ------------------ */

/* Kernels::SeamBlend::BlendChunkContributors (SeamBlendKernels.h:91,
 * SeamBlend.cpp:549-587) with the band count exposed as
 * Detail::MultiBandCompose does (SeamBlendKernels.h:75-79); 5 reproduces the
 * reference's kDefaultNumBands.  numContributors may be 0 (all-zero output). */
I360B_API int i360b_blend_chunk_contributors(const unsigned short* const* warpedBuffers, int numContributors, int width,
                                   int height, int numBands, unsigned short* outResult);

/* ---- device-resident launchers ----------------------------------------- */

/* DemosaicBayer on device buffers. */
I360B_API int i360b_launch_demosaic(const unsigned short* dCfa, int width, int height, unsigned short blackLevel,
                          const float camMul[4], const float rgbCam[12], uint32_t filters, unsigned short* dRgbOut,
                          void* stream);

/* WarpPerspective on device buffers, followed by ApplyGain(gain) in the same
 * pass (RenderExecutor.cpp:105-114 does the two back to back; gain is skipped
 * when |gain-1| <= 1e-6 exactly as there). */
I360B_API int i360b_launch_warp(const unsigned short* dSrc, int srcW, int srcH, unsigned short* dDst, int dstW, int dstH,
                      const float* homography, int offsetX, int offsetY, float gain, void* stream);

/* MedianStack on device buffers; dInputs is a HOST array of numInputs device
 * pointers. */
I360B_API int i360b_launch_median(const unsigned short* const* dInputs, int numInputs, unsigned short* dOutput, int width,
                        int height, float sigmaThreshold, void* stream);

/* The median stack of a burst: WarpPerspective of every frame onto one
 * dstW x dstH grid (homographies: numFrames * 9 floats, each dst->src
 * row-major as WarpPerspective takes it; offsets added to every destination
 * coordinate), then MedianStack over the warped frames
 * (CpuComputeBackend.cpp:112-159, MedianStackKernels.h:19-55), in one pass
 * that never writes the warped frames: the result equals those two
 * operations bit for bit.  dFrames is a HOST array of numFrames (1-32)
 * device RGB48 frames of srcW x srcH. */
I360B_API int i360b_launch_warp_median(const unsigned short* const* dFrames, int numFrames, int srcW, int srcH,
                                       const float* homographies, unsigned short* dOutput, int dstW, int dstH,
                                       int offsetX, int offsetY, float sigmaThreshold, void* stream);

/* ApplyGain on a device buffer. */
I360B_API int i360b_launch_gain(unsigned short* dData, int numValues, float gain, void* stream);

/* ComputeLabStats of n device RGB48 images in one pass (dImages, widths and
 * heights are HOST arrays, n <= 64).  dStats: DEVICE array of n * 6 doubles,
 * per image {mean L, a, b, std L, a, b}. */
I360B_API int i360b_launch_lab_stats(const unsigned short* const* dImages, const int* widths, const int* heights,
                                     int n, double* dStats, void* stream);

/* ApplyReinhardColorTransfer of n device RGB48 images in place, image i from
 * its statistics dSrcStats[i * 6 ..] to dRefStats[0 .. 5] (DEVICE arrays in
 * the i360b_launch_lab_stats layout). */
I360B_API int i360b_launch_reinhard(unsigned short* const* dImages, const int* widths, const int* heights, int n,
                                    const double* dSrcStats, const double* dRefStats, void* stream);

/* The Optimize stage's colour correction of a frame set on the device
 * (OptimizeExecutor.cpp:283-330): the Lab statistics of all n frames in one
 * pass, then every frame except frames[refIndex] transferred in place to the
 * reference frame's statistics in a second pass, with no host round trip.
 * The reference frame passes through unchanged, as there.  dStats (optional,
 * DEVICE, n * 6 doubles) receives the statistics measured before the
 * transfer. */
I360B_API int i360b_launch_color_correct(unsigned short* const* dImages, const int* widths, const int* heights,
                                         int n, int refIndex, double* dStats, void* stream);

/* Seam blend of one chunk whose K warped buffers are already on the device
 * (dWarped is a HOST array of K device pointers). */
I360B_API int i360b_launch_blend(const unsigned short* const* dWarped, int numContributors, int width, int height,
                       int numBands, unsigned short* dOut, void* stream);

/* Allocation-free variant of i360b_launch_blend.  No counterpart in the
 * reference: it exists for callers that must not allocate device memory once
 * running - hosts that reserve the GPU's memory up front for their own pool
 * (where a cudaMalloc fails or breaks their budget) and latency-critical
 * render loops (where cudaMalloc/cudaFree would synchronise the device).  All
 * of the blend's scratch comes from one static 12 MiB device array compiled
 * into the library (held on every GPU that loads it until exit); a chunk
 * needing more - roughly width*height*(15*numContributors + 5) bytes, e.g.
 * 256x256 with 8 contributors fits - returns I360B_INVALID_PARAM.  The caller
 * passes device inputs and output as for i360b_launch_blend.  Synchronous: it
 * waits for `stream` before returning.  Every call reuses the same array, so
 * calls whose GPU work overlaps race; serialise them.  i360b_initialize
 * reserves the array on the device it selects and looks up its device
 * address, so the entry point itself never touches the allocator. */
I360B_API int i360b_launch_blend_noalloc(const unsigned short* const* dWarped, int numContributors, int width,
                                         int height, int numBands, unsigned short* dOut, void* stream);

/* ---- batched render of a panorama's output tiles ----------------------- */

/* One source frame: a demosaiced RGB48 image in device memory and its
 * homography from frame pixels to canvas pixels (Homography, Types.h:138-141,
 * in double).  gain is applied after the warp (RenderExecutor.cpp:111-114). */
/* ---- pipelined render executor ------------------------------------------ */

/* A device-resident RenderExecutor (RenderExecutor.cpp:40-147) for a sequence
 * of frame sets of one panorama geometry: each submission uploads its CFA
 * frames once, demosaics them (DemosaicBayer), renders every tile (the
 * render plan) and downloads every tile output once - no per-operation host
 * round trips (CudaPipeline.cpp:207-267 copies every operand on every call).
 * `depth` device slots (1-4), each with its own compute stream, let the
 * upload of one submission, the renders of the previous ones and the
 * download of an earlier one run at the same time (two renders overlap the
 * latency-bound stages of one with the bandwidth-bound stages of the other).  Host buffers must be pinned for the copies to overlap
 * and must stay valid until i360b_pipeline_wait returns. */
typedef struct i360b_pipeline_desc
{
    int numFrames, frameWidth, frameHeight;
    const double* toCanvas; /* numFrames x 9, frame -> canvas, row-major */
    const float* gains;     /* numFrames: ApplyGain after the warp (RenderExecutor.cpp:111) */
    unsigned short blackLevel;
    float camMul[4];
    float rgbCam[12]; /* 3x4, row-major */
    uint32_t filters;
    int numTiles;
    const int* tileRects;    /* numTiles x 4: x, y, width, height */
    const int* tileFirst;    /* numTiles: contributors[first .. first+count) */
    const int* tileCount;    /* numTiles */
    const int* contributors; /* frame indices */
    int numBands;
    int coordMode; /* I360B_COORDS_* */
    int depth;     /* device slots, 1-4 (2 overlaps all three stages) */
} i360b_pipeline_desc;

typedef struct i360b_pipeline i360b_pipeline;

I360B_API int i360b_pipeline_create(const i360b_pipeline_desc* desc, i360b_pipeline** out);
/* Enqueues one frame set: hostCfa[numFrames] (width x height samples each)
 * in, hostTiles[numTiles] (RGB48 tile outputs) out.  Returns at once. */
I360B_API int i360b_pipeline_submit(i360b_pipeline* pipeline, const unsigned short* const* hostCfa,
                                    unsigned short* const* hostTiles);
/* Waits for every submission; *elapsedMs (optional) receives the device
 * time from the first upload since the previous wait to the last download. */
I360B_API int i360b_pipeline_wait(i360b_pipeline* pipeline, float* elapsedMs);
/* i360b_render_plan_autotune on the first slot's plan (after a submission:
 * the plan needs real frames), applied to every slot. */
I360B_API int i360b_pipeline_autotune(i360b_pipeline* pipeline, int* bandRows, int* dtSlots, float* bestMs);
I360B_API void i360b_pipeline_destroy(i360b_pipeline* pipeline);

/* ---- export of rendered chunk outputs ----------------------------------- */

/* The preview composite of PanoramaExporter::ExportPreviewJpeg
 * (PanoramaExporter.cpp:46-102) on the device: chunk outputs (RGB48,
 * dChunks[c] with canvas rectangle rects[4c .. 4c+3] = x, y, width, height;
 * a null pointer = a chunk with no render output) placed in chunk order into
 * an RGB8 image whose longest edge is maxDimension (ComputeExportScale /
 * ComputeChunkPlacement, PanoramaExporter.cpp:9-24), nearest source pixel,
 * samples >> 8; the last chunk with a source pixel wins where placements
 * overlap, as in the reference's loop.  *outW / *outH receive the size;
 * returns INVALID_PARAM when capacity < outW * outH * 3 bytes.  The JPEG
 * encode is the caller's codec (IImageCodec::Encode).  dChunks and rects are
 * HOST arrays; dOut is device memory. */
I360B_API int i360b_launch_export_preview(const unsigned short* const* dChunks, const int* rects, int numChunks,
                                          int totalW, int totalH, int maxDimension, unsigned char* dOut,
                                          long long capacity, int* outW, int* outH, void* stream);

/* Writes the 16-bit RGB TIFF of WriteTiff16RGB (Tiff16Writer.cpp:40-97,
 * byte for byte) of a canvasW x canvasH canvas holding the chunk outputs at
 * their rectangles (zero elsewhere), assembled band by band on the device.
 * Canvases whose samples exceed the format's 32-bit offsets (4 GiB) are
 * rejected with INVALID_PARAM (the reference would write wrapped offsets).
 * Synchronous. */
I360B_API int i360b_write_tiff16_chunks(const char* path, const unsigned short* const* dChunks, const int* rects,
                                        int numChunks, int canvasW, int canvasH, void* stream);

/* StorageEngine::WritePixelBuffer's framing (StorageEngine.cpp:130-144) of a
 * device RGB48 image into hostOut: int32 width, int32 height (little
 * endian), then width * height * 3 samples - 8 + width * height * 6 bytes.
 * Synchronous. */
I360B_API int i360b_download_framed(const unsigned short* dData, int width, int height, void* hostOut, void* stream);

/* ---- tile -> contributor culling ---------------------------------------- */

/* Overlap test modes of i360b_cull_tiles / i360b_launch_cull_tiles. */
enum
{
    /* OverlapCulling.cpp:10-45 in FP32: decisions identical to the CPU's. */
    I360B_CULL_REFERENCE = 0,
    /* corners and tile bounds in FP64 (canvases beyond 2^24 pixels). */
    I360B_CULL_FP64 = 1
};

/* The contributor list of every output tile: ImageOverlapsChunk
 * (OverlapCulling.cpp:10-45) for every (tile, frame) pair - the box of the
 * frame's projected corners (0,0), (W,0), (0,H), (W,H) under its frame ->
 * canvas homography against the tile rectangle, strict inequalities - with
 * each tile's frames listed in frame order as FindOverlappingImages builds
 * them (OverlapCulling.cpp:47-89), and its rule that a frame of unknown size
 * (width or height <= 0) overlaps every tile.
 *   homographies  numFrames x 9 floats, row-major, frame -> canvas
 *   tiles         numTiles x 4 ints: x, y, width, height
 *   first, count  per tile: its contributors are contrib[first .. first+count)
 *   total         contributors over all tiles.
 * The output is the CSR form i360b_tile takes (first, count).  Host buffers;
 * returns INVALID_PARAM when contribCapacity < *total (first, count and
 * *total are still written, so the caller can size contrib and call again). */
I360B_API int i360b_cull_tiles(const float* homographies, const int* frameWidths, const int* frameHeights,
                               int numFrames, const int* tiles, int numTiles, int mode, int* first, int* count,
                               int* contrib, int contribCapacity, int* total);

/* The same on device buffers, stream-ordered (dTotal is a device int);
 * contributors beyond contribCapacity are not written - compare *dTotal with
 * the capacity. */
I360B_API int i360b_launch_cull_tiles(const float* dHomographies, const int* dFrameWidths, const int* dFrameHeights,
                                      int numFrames, const int* dTiles, int numTiles, int mode, int* dFirst,
                                      int* dCount, int* dContrib, int contribCapacity, int* dTotal, void* stream);

typedef struct i360b_frame
{
    const unsigned short* rgb;
    int width;
    int height;
    double toCanvas[9];
    float gain;
} i360b_frame;

/* One output tile (a RenderExecutor chunk, Types.h:143-152): canvas
 * rectangle, its contributors contributors[first .. first+count), and the
 * device RGB48 buffer (width*height*3) it is written to. */
typedef struct i360b_tile
{
    int x;
    int y;
    int width;
    int height;
    int first;
    int count;
    unsigned short* dOut;
} i360b_tile;

/* Coordinate modes of the tile warp. */
enum
{
    /* Inverse homography in FP32 by the adjugate (HomographyMath.cpp:94-116)
     * and destination coordinates (x + tile.x, y + tile.y) in FP32, exactly as
     * RenderExecutor feeds WarpPerspective: bit-identical to the CPU backend. */
    I360B_COORDS_REFERENCE = 0,
    /* Inverse homography in FP64 on the GPU and each tile's origin mapped in
     * FP64; FP32 only for offsets inside the tile. */
    I360B_COORDS_FP64_ORIGIN = 1
};

typedef struct i360b_render_plan i360b_render_plan;

/* Builds a reusable plan (work lists, device scratch) for rendering `numTiles`
 * uneven tiles from `numFrames` frames with `numBands` pyramid levels.  The
 * frame and tile arrays are copied; device pointers inside them must stay
 * valid while the plan is used. */
I360B_API int i360b_render_plan_create(const i360b_frame* frames, int numFrames, const i360b_tile* tiles, int numTiles,
                             const int* contributors, int numBands, int coordMode, i360b_render_plan** outPlan);
/* Enqueues the whole render on `stream` (captured once as a CUDA graph and
 * replayed on later calls).  Asynchronous: returns once enqueued. */
I360B_API int i360b_render_plan_execute(i360b_render_plan* plan, void* stream);
/* Waits for `stream` and reports a render kernel that gave up one of its
 * bounded waits (I360B_KERNEL_LAUNCH_FAILED; the output is then invalid). */
I360B_API int i360b_render_plan_wait(i360b_render_plan* plan, void* stream);
/* Plan statistics.  coveredItemPixels (sum over tile contributors of their
 * covered pixels after the last execute) needs a completed execute. */
typedef struct i360b_render_stats
{
    int numTiles;
    int numItems;          /* (tile, contributor) pairs */
    int kernelsPerExecute; /* kernel launches one execute enqueues */
    long long outputPixels;
    long long coveredItemPixels;
    long long scratchBytes;
    /* SM cycles spent in the seam kernel's five phases (crossover scan, colour
     * cost, dynamic program, backtrack, reassignment), summed over tiles and
     * executions since the plan was created. */
    long long seamPhaseCycles[5];
} i360b_render_stats;
I360B_API int i360b_render_plan_stats(i360b_render_plan* plan, void* stream, i360b_render_stats* out);
/* Runs the plan once without the graph, timing each stage with CUDA events on
 * `stream`; stageMs receives up to maxStages values (10 stages, names from
 * i360b_render_stage_name; stages 5-9 are the pyramid base, the levels above
 * it, the blended bands, the collapse and the fine levels with the output,
 * whose split depends on the level-fusion depth).  Synchronous. */
I360B_API int i360b_render_plan_profile(i360b_render_plan* plan, void* stream, float* stageMs, int maxStages);
I360B_API const char* i360b_render_stage_name(int stage);
/* Autotuner: times the plan's own render (two runs after a warm-up, CUDA
 * events on `stream`; each run as stage 0 then stages 1-9, the form
 * i360b_render_plan_execute_stages offers for early frame refills), first
 * for both tile-warp forms and level-fusion
 * depths, then with the faster pair for every band-unit height of the
 * per-pixel kernels (8, 16, 32, 64 rows) and every ring depth of the chamfer
 * transform that fits (2 to 4 row groups), then the chain split, and keeps
 * the fastest (read the fusion depth and warp form back with
 * i360b_render_plan_get_tuning, the split with
 * i360b_render_plan_get_chain_split).  The output of every
 * setting is identical (the settings only partition the same work), so
 * tuning never changes results.  The chosen values and the best time of one
 * execute are returned when the pointers are non-null.  Synchronous; the
 * plan's outputs are overwritten with its render. */
I360B_API int i360b_render_plan_autotune(i360b_render_plan* plan, void* stream, int* bandRows, int* dtSlots,
                                         float* bestMs);
/* The plan's tuning: rows per band unit of the per-pixel kernels (8, 16, 32
 * or 64), chamfer ring slots (0 = as many as fit, else 2 to the number that
 * fits), the level-fusion depth of the pyramid (2 computes levels 0 and 1 on
 * chip, so only levels >= 2 of the pyramids are written to memory; 1 writes
 * level 1 too and fuses the level-1 blend, the collapse and the output into
 * one kernel that reads it; 0 materialises every level) and the tile warp's form (1: 128x32 blocks whose
 * source footprint is staged in shared memory; 0: row bands gathering
 * through L1).  Every setting renders the same bits.  No reference
 * counterpart (the reference's blend is a fixed CPU loop).  set_tuning is
 * synchronous on `stream`; the next execute recaptures the plan's graph.
 * The autotuner searches all four. */
I360B_API int i360b_render_plan_get_tuning(i360b_render_plan* plan, int* bandRows, int* dtSlots, int* fusedLevels,
                                           int* warpShape);
I360B_API int i360b_render_plan_set_tuning(i360b_render_plan* plan, int bandRows, int dtSlots, int fusedLevels,
                                           int warpShape, void* stream);
/* Chain stagger.  A plan splits its tiles into up to three chains whose
 * stages run on their own streams inside its graph.  With stage L >= 0 the
 * other chains start only once the first has finished stage L (of the
 * stages a run covers); -1 starts them together (the default: on the
 * 90-tile panorama a stagger measured no faster for whole runs and slower
 * for runs split after stage 0, so the autotuner leaves it).  Ordering only:
 * every setting renders the same bits.  A plan with one chain reports -1.
 * Synchronous on `stream`; the next execute recaptures the plan's graph.
 * No reference counterpart. */
I360B_API int i360b_render_plan_set_chain_lag(i360b_render_plan* plan, int stage, void* stream);
/* Chain split.  0: the chains carry about equal work (area x contributors),
 * the default.  p in 1..50: the tiles ordered by the time their seam step
 * took in the plan's last execution, slowest first (the seam search runs one
 * CTA per tile, sequentially over contested lines, so its slowest tile sets
 * the stage's length while most SMs are free): the first p percent form the
 * first chain, the next p percent the second (with three chains), the rest
 * the last.  The slow seam searches start early and run beside the full-GPU
 * stages of the chains behind them.  INVALID_PARAM for p outside 0..50, or
 * for p > 0 before the plan has executed once.  Ordering only: every setting
 * renders the same bits.  The autotuner tries 0, 5, 10, 15, 20 and 30.  Synchronous on
 * `stream`; the next execute recaptures the plan's graph.  No reference
 * counterpart. */
I360B_API int i360b_render_plan_set_chain_split(i360b_render_plan* plan, int percent, void* stream);
I360B_API int i360b_render_plan_get_chain_split(i360b_render_plan* plan, int* percent);
/* SM cycles each tile's seam step took in the plan's last execution (0 for
 * tiles with fewer than two contributors or before a first execution), for
 * the first maxTiles tiles in plan order.  Synchronous on `stream`. */
I360B_API int i360b_render_plan_seam_tile_cycles(i360b_render_plan* plan, unsigned long long* cycles, int maxTiles,
                                                 void* stream);
I360B_API int i360b_render_plan_get_chain_lag(i360b_render_plan* plan, int* stage);
/* Precision of the render's stored pyramid levels.  EXACT keeps them in
 * FP32 and renders the CPU backend's output bit for bit.  FP16 is the native
 * mode: the levels a plan keeps in memory (levels >= 1, or >= 2 at
 * level-fusion depth 2; any depth may be combined with it) are stored as
 * FP16 (num / 256, den, weight) with every operation in FP32, halving their
 * traffic; its output is no longer bit-exact, and its
 * error against the FP64 restatement of the blend is what the tests and the
 * bench report.  Warped pixels stay 16-bit integers in both modes (the same
 * two bytes as FP16, without FP16's rounding of values above 2048).  No
 * reference counterpart.  Synchronous on `stream`; the next execute
 * recaptures the plan's graph. */
enum
{
    I360B_PRECISION_EXACT = 0,
    I360B_PRECISION_FP16 = 1
};
I360B_API int i360b_render_plan_set_precision(i360b_render_plan* plan, int mode, void* stream);
/* i360b_launch_export_preview over the plan's tiles in tile order (tiles that
 * list no contributor have no render output and are skipped). */
I360B_API int i360b_render_plan_export_preview(i360b_render_plan* plan, int totalW, int totalH, int maxDimension,
                                               unsigned char* dOut, long long capacity, int* outW, int* outH,
                                               void* stream);

/* i360b_write_tiff16_chunks over the plan's tile outputs. */
I360B_API int i360b_render_plan_write_tiff16(i360b_render_plan* plan, const char* path, int canvasW, int canvasH,
                                             void* stream);

/* Runs stages firstStage..lastStage of the plan (the order of
 * i360b_render_stage_name: 0 = warp, gain and coverage, which alone reads the
 * frames' RGB48 buffers; 1-9 the seam blend) as a CUDA graph of their own
 * (captured on first use).  Running stage 0, then 1-9, is the same render as
 * i360b_render_plan_execute; a caller that refills the frame buffers for the
 * next render may do so as soon as stage 0 has completed.  Stages run in
 * order and consume what the stages before them wrote: in particular the
 * band blend (stage 7) turns the stored coarse pyramid levels into their
 * Gaussian values in place, so a range starting after stage 5 must follow a
 * run of the stages before it. */
I360B_API int i360b_render_plan_execute_stages(i360b_render_plan* plan, int firstStage, int lastStage, void* stream);

/* Sets how long each bounded device wait of the plan's kernels may last, in
 * SM cycles (default about one second; a negative value restores it).  A
 * kernel whose wait runs out sets the plan's error flag and returns, and
 * i360b_render_plan_wait then reports I360B_KERNEL_LAUNCH_FAILED.  0 makes
 * every wait that is not satisfied at once give up, which tests use to
 * exercise that path without faulting the GPU.  No reference counterpart:
 * the reference's kernels have no inter-block waits.  Synchronous on
 * `stream`; the next execute recaptures the plan's graph. */
I360B_API int i360b_render_plan_set_wait_limit(i360b_render_plan* plan, long long cycles, void* stream);

/* Host-side failure injection for tests (StubTaskExecutor.h:27-56 injects at
 * task level; this injects at the device-call level).  kind
 * I360B_INJECT_ALLOC makes the next `count` device allocations of the library
 * fail as out of memory (I360B_OUT_OF_MEMORY); I360B_INJECT_LAUNCH makes the
 * next `count` launch checks report a failed launch
 * (I360B_KERNEL_LAUNCH_FAILED).  Nothing reaches the GPU: the failure is
 * decided on the host before the call.  count 0 disarms. */
enum
{
    I360B_INJECT_ALLOC = 1,
    I360B_INJECT_LAUNCH = 2
};
I360B_API int i360b_debug_inject_failure(int kind, int count);

/* Device bytes of scratch the plan holds. */
I360B_API size_t i360b_render_plan_scratch_bytes(const i360b_render_plan* plan);
I360B_API void i360b_render_plan_destroy(i360b_render_plan* plan);

#ifdef __cplusplus
}
#endif

#endif
