/*
 * image360_b200 - learned seam blend: the C-ABI of the blend network and its
 * tensor-core convolution primitives.
 *
 * No counterpart in the reference, which blends overlaps only with the
 * multi-band Laplacian seam blend (WindowsApp.Core/SourceFiles/SeamBlend.cpp:549-587).
 * The network stands in for that blend on overlap windows:
 *
 *   input   16 channels per pixel: up to 4 warped RGB48 layers, each as R, G, B
 *           (value / 32768) and a feathered coverage mask: 0 where the layer
 *           is (0,0,0) (uncovered, SeamBlend.cpp:565), else
 *           0.25 + 0.75 min(1, d / 2048) with d the distance from the pixel
 *           to the nearest of the layer's boundary edges given in the job
 *           (1 where none is given), in bf16;
 *   net     a 2-scale U-Net-lite of eight 3x3 convolutions with zero padding:
 *           16->32, 32->32 (full resolution, kept as the skip), 2x2 average
 *           pool, 32->64, 64->64, 64->64 (half resolution), nearest 2x
 *           upsample concatenated after the skip (96 channels), 96->32, 32->32,
 *           32->4; ReLU after all but the last; bf16 weights and activations,
 *           fp32 accumulation (tcgen05 tensor cores) and fp32 bias;
 *   head    the 4 outputs are per-layer blend logits; a softmax over the
 *           layers that cover the pixel weights the layers' original 16-bit
 *           values into the RGB48 output (no layer covers -> 0).
 *
 * With all logits equal (the untrained network: the last layer starts at
 * zero) the head is the coverage-weighted mean of the layers.  Training
 * minimises the mean squared error against the plain seam blend of the same
 * window (Adam).  Window width must be a multiple of 256, height even.
 *
 * All pointers named d* are device pointers; `stream` is a cudaStream_t.
 */
#ifndef IMAGE360_B200_BLENDNET_H
#define IMAGE360_B200_BLENDNET_H

#include "image360_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One window of a batch.  Slot i of pixel (x, y) of the window is
 * slot[i][y * rowStride + x * pixStride + c] for c = R, G, B (element
 * offsets); a null slot is an absent layer.  Pixels with x >= width or
 * y >= height lie outside the image (input zero, nothing written). */
typedef struct i360b_blend_job
{
    const unsigned short* slot[4];
    long long pixStride;
    long long rowStride;
    int width;
    int height;
    /* Training: target RGB48 of the window (same stride convention). */
    const unsigned short* target;
    long long targetRowStride;
    /* Inference: RGB48 output (3 elements per pixel). */
    unsigned short* out;
    long long outRowStride;
    /* Per slot, up to 4 line segments {x0, y0, x1, y1} in window pixel
     * coordinates: the parts of the layer's coverage boundary inside the
     * output tile (the distance of the feathered mask).  A segment whose x0
     * is NaN is absent. */
    float edges[4][16];
} i360b_blend_job;

typedef struct i360b_blendnet i360b_blendnet;

/* Number of fp32 parameters (weights [cout][ky][kx][cin] then bias, layer by
 * layer). */
I360B_API int i360b_blendnet_param_count(void);
/* A network with He-normal weights from `seed`, zero biases and a zero last
 * layer, on the current device. */
I360B_API int i360b_blendnet_create(unsigned long long seed, i360b_blendnet** outNet);
I360B_API void i360b_blendnet_destroy(i360b_blendnet* net);
I360B_API int i360b_blendnet_get_params(i360b_blendnet* net, float* hostParams, int count);
I360B_API int i360b_blendnet_set_params(i360b_blendnet* net, const float* hostParams, int count);
/* The optimiser state for checkpoints: Adam's first and second moments
 * (param_count floats each) and the step count its bias correction uses.
 * Saving it with the weights lets a resumed training continue exactly where
 * it stopped.  Synchronous. */
I360B_API int i360b_blendnet_get_adam(i360b_blendnet* net, float* hostM, float* hostV, int count, int* step);
I360B_API int i360b_blendnet_set_adam(i360b_blendnet* net, const float* hostM, const float* hostV, int count,
                                      int step);
/* Forward pass of `n` windows of w x h; writes the 4 logits per pixel as fp32
 * [n][h][w][4] to dLogits.  Synchronous. */
I360B_API int i360b_blendnet_logits(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                    float* dLogits);
/* Loss (mean squared error over n*h*w*3 values, in units of 1/32768) and its
 * gradient with respect to every parameter (hostGrad: param_count floats).
 * Synchronous. */
I360B_API int i360b_blendnet_gradients(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                       float* hostGrad, double* hostLoss);
/* One Adam step (beta 0.9/0.999, eps 1e-8) at learning rate lr on the batch.
 * hostLoss, when non-null, receives the batch loss before the step (the call
 * then waits for the stream). */
I360B_API int i360b_blendnet_train_step(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                        float lr, double* hostLoss, void* stream);
/* Inference: blends each window into its job's output.  Asynchronous. */
I360B_API int i360b_blendnet_infer(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                   void* stream);

/* One inference pass timed kernel by kernel with CUDA events: kernelMs
 * receives up to maxKernels times (10 kernels, names from
 * i360b_blendnet_kernel_name).  Synchronous. */
I360B_API int i360b_blendnet_profile(i360b_blendnet* net, const i360b_blend_job* jobs, int n, int w, int h,
                                     float* kernelMs, int maxKernels);
I360B_API const char* i360b_blendnet_kernel_name(int kernel);

/* ---- learned render of a panorama --------------------------------------- */

/* Every output tile of a render plan is cut into 256x256 windows (partial at
 * the tile's right and bottom edges).  A window that no contributor's
 * footprint reaches is cleared, one that a single contributor reaches gets
 * that contributor's warped pixels, and one that 2 to 4 reach is blended by
 * the network (with more than 4, the 4 with the largest footprint overlap). */
typedef struct i360b_learned_stats
{
    int subTiles;         /* windows of all output tiles */
    int netSubTiles;      /* blended by the network */
    int copySubTiles;     /* one contributor: copied */
    int emptySubTiles;    /* no contributor: zero */
    int overflowSubTiles; /* more than 4 contributors reached the window */
    int judgedSubTiles;   /* compared with the plain seam blend */
    int fallbackSubTiles; /* below the PSNR threshold: replaced by the plain blend */
    int maxAbsError;      /* largest |learned - plain| before fallback */
    double minPsnr;       /* lowest window PSNR before fallback (inf: identical) */
    double meanPsnr;      /* mean over windows with a finite PSNR */
} i360b_learned_stats;

/* Warps every contributor (the plan's first stage) and renders each tile with
 * the learned blend into dTileOut[t] (width*height*3 RGB48 per tile; NULL =
 * the plan's own outputs), at most maxBatch network windows per pass.
 * stageMs, when non-null, receives 3 times in ms (warp, copies, network).
 * Returns once the render has completed on `stream`. */
I360B_API int i360b_render_plan_learned(i360b_render_plan* plan, i360b_blendnet* net,
                                        unsigned short* const* dTileOut, int maxBatch, void* stream, float* stageMs);
/* The per-window judge and fallback: compares every window of dTileOut with
 * the plan's own outputs, which must hold the plain seam blend of a completed
 * i360b_render_plan_execute; PSNR = 10 log10(peak^2 / MSE) over the window's
 * RGB values.  Windows below minPsnrDb are overwritten with the plain blend.
 * hostSubTilePsnr (optional) receives up to maxSubTiles PSNRs in window order
 * (tile by tile, rows of windows).  Synchronous. */
I360B_API int i360b_render_plan_judge(i360b_render_plan* plan, unsigned short* const* dTileOut, double minPsnrDb,
                                      double peak, i360b_learned_stats* stats, float* hostSubTilePsnr,
                                      int maxSubTiles, void* stream);
/* The plan's windows in judge order: 6 ints per window {tile, x, y, kind
 * (0 clear, 1 copy, 2 network), overflow (more than 4 contributors reached
 * it), contributors kept}; numWindows receives the count, up to maxWindows
 * entries are written. */
I360B_API int i360b_render_plan_windows(i360b_render_plan* plan, int maxWindows, int* info, int* numWindows);
/* The warped contributor images of tile `tile` after an execute (device RGB48,
 * tile-sized), their footprint boxes {x0, y0, x1, y1} in tile pixels
 * (outside the box the image is zero) and, when `edges` is non-null, 16
 * floats per contributor: the 4 edges of its coverage boundary clipped to the
 * tile, as in i360b_blend_job (tile coordinates; NaN x0 = absent).
 * numItems receives the count; up to maxItems entries are written. */
I360B_API int i360b_render_plan_tile_items(i360b_render_plan* plan, int tile, int maxItems,
                                           const unsigned short** dImages, int* boxes, float* edges,
                                           int* numItems);

/* ---- convolution primitives (NHWC bf16) --------------------------------- */

/* Epilogues of i360b_conv3x3_forward. */
enum
{
    I360B_CONV_BIAS_RELU = 0, /* out = bf16(max(acc + bias, 0)) */
    I360B_CONV_LOGITS = 1,    /* out = fp32 (acc + bias) for channels 0..3 */
    I360B_CONV_MASK = 2,      /* out = bf16(dAct > 0 ? acc : 0) (ReLU backward) */
    I360B_CONV_RAW = 3        /* out = bf16(acc) */
};

/* 3x3 convolution, stride 1, zero padding 1.  dX is [n][h][w][cin]; with
 * skipChannels > 0 the input is instead the concatenation of dX
 * ([n][h][w][skipChannels]) and the nearest 2x upsample of dU
 * ([n][h/2][w/2][cin - skipChannels]).  dWeights is bf16 [cout][3][3][cin],
 * dBias fp32 [cout].  Supported (cin, cout): the layer shapes of the blend
 * network and of its backward pass.  Tensors 16-byte aligned. */
I360B_API int i360b_conv3x3_forward(const void* dX, const void* dU, int skipChannels, int n, int h, int w, int cin,
                                    int cout, const void* dWeights, const float* dBias, int epilogue,
                                    const void* dAct, void* dOut, void* stream);
/* Weight gradient of that convolution: dGradW[cout][3][3][cin] (fp32,
 * overwritten) = sum over pixels of dGrad[p][co] * input[p + tap][ci];
 * width a multiple of 128. */
I360B_API int i360b_conv3x3_wgrad(const void* dX, const void* dU, int skipChannels, const void* dGrad, int n, int h,
                                  int w, int cin, int cout, float* dGradW, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IMAGE360_B200_BLENDNET_H */
