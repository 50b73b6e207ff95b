// A pipelined, device-resident render executor: RenderExecutor::Execute
// (RenderExecutor.cpp:40-147) for every chunk of a panorama, fed with raw CFA
// frames and returning the chunk outputs to host memory, for a sequence of
// frame sets of one geometry (the same rig and homographies).
//
// The reference's compute backend copies every operand between host and
// device on every call (CudaPipeline.cpp:207-267); here each submission makes
// exactly one upload of its CFA frames and one download of its chunk outputs,
// and `depth` device slots (CFA frames, demosaiced frames, a render plan and
// its chunk outputs, and a compute stream of its own) let different
// submissions run at once: the upload of set k+1, the demosaic and render of
// sets k and k-1 (the latency-bound stages of one render - the chamfer
// wavefront, the seam search - overlap the bandwidth-bound stages of the
// other), the download of set k-2.  Per slot, events order the three stages
// against the slot's previous use: its upload waits until the previous render of the slot has
// read the CFA, its render waits for its upload and for the previous download
// of the slot's outputs, its download waits for its render.  Host buffers must
// be pinned for the copies to overlap, and must stay valid until the
// submission has been waited for.
#include "render_plan.hpp"

#include <new>
#include <vector>

using namespace i360b;

struct i360b_pipeline
{
    struct Slot
    {
        unsigned short* cfa = nullptr;   // numFrames x w x h
        unsigned short* rgb = nullptr;   // numFrames x w x h x 3
        unsigned short* outs = nullptr;  // every tile's output, back to back
        i360b_render_plan* plan = nullptr;
        cudaStream_t comp = nullptr;     // demosaic and render of this slot
        cudaEvent_t uploaded = nullptr, rendered = nullptr, downloaded = nullptr;
        bool used = false;
    };
    int nFrames = 0, w = 0, h = 0;
    unsigned short black = 0;
    float camMul[4] = {}, rgbCam[12] = {};
    uint32_t filters = 0;
    std::vector<size_t> tileOff;    // element offset of each tile output in a slot's `outs`
    std::vector<size_t> tileBytes;  // bytes of each tile output
    std::vector<Slot> slots;
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t start = nullptr, end = nullptr;
    long long submitted = 0;
    bool timing = false;

    ~i360b_pipeline()
    {
        for (cudaStream_t s : {up, down})
            if (s) cudaStreamSynchronize(s);
        for (Slot& S : slots)
        {
            if (S.comp) cudaStreamSynchronize(S.comp);
            if (S.plan) i360b_render_plan_destroy(S.plan);
            if (S.comp) cudaStreamDestroy(S.comp);
            cudaFree(S.cfa);
            cudaFree(S.rgb);
            cudaFree(S.outs);
            for (cudaEvent_t e : {S.uploaded, S.rendered, S.downloaded})
                if (e) cudaEventDestroy(e);
        }
        for (cudaEvent_t e : {start, end})
            if (e) cudaEventDestroy(e);
        for (cudaStream_t s : {up, down})
            if (s) cudaStreamDestroy(s);
    }
};

namespace
{
int make_slot(i360b_pipeline& P, const i360b_pipeline_desc& d, i360b_pipeline::Slot& S)
{
    const size_t px = (size_t)P.w * P.h;
    I360B_CUDA(cudaMalloc(&S.cfa, px * P.nFrames * sizeof(unsigned short)), "pipeline CFA frames");
    I360B_CUDA(cudaMalloc(&S.rgb, px * 3 * P.nFrames * sizeof(unsigned short)), "pipeline demosaiced frames");
    const size_t outElems = P.tileOff.back();
    I360B_CUDA(cudaMalloc(&S.outs, outElems * sizeof(unsigned short)), "pipeline chunk outputs");
    for (cudaEvent_t* e : {&S.uploaded, &S.rendered, &S.downloaded})
        I360B_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "pipeline event");
    I360B_CUDA(cudaStreamCreateWithFlags(&S.comp, cudaStreamNonBlocking), "pipeline stream");
    std::vector<i360b_frame> frames(P.nFrames);
    for (int f = 0; f < P.nFrames; ++f)
    {
        frames[f].rgb = S.rgb + px * 3 * f;
        frames[f].width = P.w;
        frames[f].height = P.h;
        for (int q = 0; q < 9; ++q) frames[f].toCanvas[q] = d.toCanvas[(size_t)f * 9 + q];
        frames[f].gain = d.gains[f];
    }
    std::vector<i360b_tile> tiles(d.numTiles);
    for (int t = 0; t < d.numTiles; ++t)
    {
        tiles[t].x = d.tileRects[4 * t];
        tiles[t].y = d.tileRects[4 * t + 1];
        tiles[t].width = d.tileRects[4 * t + 2];
        tiles[t].height = d.tileRects[4 * t + 3];
        tiles[t].first = d.tileFirst[t];
        tiles[t].count = d.tileCount[t];
        tiles[t].dOut = S.outs + P.tileOff[t];
    }
    return i360b_render_plan_create(frames.data(), P.nFrames, tiles.data(), d.numTiles, d.contributors, d.numBands,
                                    d.coordMode, &S.plan);
}
}  // namespace

extern "C" int i360b_pipeline_create(const i360b_pipeline_desc* d, i360b_pipeline** out)
{
    clear_error();
    if (!out) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    *out = nullptr;
    if (!d || !d->toCanvas || !d->gains || !d->tileRects || !d->tileFirst || !d->tileCount)
        return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (d->numFrames <= 0 || d->frameWidth <= 0 || d->frameHeight <= 0 || d->numTiles <= 0)
        return fail(I360B_INVALID_PARAM, "Invalid frame or tile counts or dimensions.");
    if (d->depth < 1 || d->depth > 4) return fail(I360B_INVALID_PARAM, "Pipeline depth must be 1-4.");
    if (!initialized()) return fail(I360B_CUDA_ERROR, "Not initialized.");
    I360B_TRY(ensure_ready());
    auto* P = new (std::nothrow) i360b_pipeline;
    if (!P) return fail(I360B_OUT_OF_MEMORY, "Host allocation failed.");
    struct Guard
    {
        i360b_pipeline* p;
        ~Guard() { delete p; }
    } guard{P};
    P->nFrames = d->numFrames;
    P->w = d->frameWidth;
    P->h = d->frameHeight;
    P->black = d->blackLevel;
    for (int i = 0; i < 4; ++i) P->camMul[i] = d->camMul[i];
    for (int i = 0; i < 12; ++i) P->rgbCam[i] = d->rgbCam[i];
    P->filters = d->filters;
    P->tileOff.assign(1, 0);
    for (int t = 0; t < d->numTiles; ++t)
    {
        const int tw = d->tileRects[4 * t + 2], th = d->tileRects[4 * t + 3];
        if (tw <= 0 || th <= 0) return fail(I360B_INVALID_PARAM, "Tile %d has invalid dimensions.", t);
        const size_t elems = (size_t)tw * th * 3;
        P->tileBytes.push_back(elems * sizeof(unsigned short));
        P->tileOff.push_back(P->tileOff.back() + ((elems + 127) & ~size_t(127)));  // 256-byte aligned outputs
    }
    for (cudaStream_t* s : {&P->up, &P->down})
        I360B_CUDA(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking), "pipeline stream");
    for (cudaEvent_t* e : {&P->start, &P->end}) I360B_CUDA(cudaEventCreate(e), "pipeline event");
    P->slots.resize(d->depth);
    for (auto& S : P->slots) I360B_TRY(make_slot(*P, *d, S));
    P->tileOff.pop_back();
    guard.p = nullptr;
    *out = P;
    return I360B_SUCCESS;
}

extern "C" int i360b_pipeline_submit(i360b_pipeline* P, const unsigned short* const* hostCfa,
                                     unsigned short* const* hostTiles)
{
    clear_error();
    if (!P || !hostCfa || !hostTiles) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    for (int f = 0; f < P->nFrames; ++f)
        if (!hostCfa[f]) return fail(I360B_INVALID_PARAM, "Null CFA frame %d.", f);
    for (size_t t = 0; t < P->tileOff.size(); ++t)
        if (!hostTiles[t]) return fail(I360B_INVALID_PARAM, "Null tile output %d.", (int)t);
    i360b_pipeline::Slot& S = P->slots[P->submitted % (long long)P->slots.size()];
    const size_t px = (size_t)P->w * P->h;
    if (!P->timing)
    {
        I360B_CUDA(cudaEventRecord(P->start, P->up), "pipeline timing");
        P->timing = true;
    }
    // upload: after the slot's previous render has read its CFA
    if (S.used) I360B_CUDA(cudaStreamWaitEvent(P->up, S.rendered, 0), "pipeline order");
    for (int f = 0; f < P->nFrames; ++f)
        I360B_CUDA(cudaMemcpyAsync(S.cfa + px * f, hostCfa[f], px * sizeof(unsigned short), cudaMemcpyHostToDevice,
                                   P->up),
                   "pipeline upload");
    I360B_CUDA(cudaEventRecord(S.uploaded, P->up), "pipeline order");
    // demosaic and render: after the upload and the slot's previous download
    I360B_CUDA(cudaStreamWaitEvent(S.comp, S.uploaded, 0), "pipeline order");
    if (S.used) I360B_CUDA(cudaStreamWaitEvent(S.comp, S.downloaded, 0), "pipeline order");
    for (int f = 0; f < P->nFrames; ++f)
        I360B_TRY(launch_demosaic(S.cfa + px * f, P->w, P->h, P->black, P->camMul, P->rgbCam, P->filters,
                                  S.rgb + px * 3 * f, S.comp));
    I360B_TRY(S.plan->plan.execute(S.comp, true));
    I360B_CUDA(cudaEventRecord(S.rendered, S.comp), "pipeline order");
    // download: after the render
    I360B_CUDA(cudaStreamWaitEvent(P->down, S.rendered, 0), "pipeline order");
    for (size_t t = 0; t < P->tileOff.size(); ++t)
        I360B_CUDA(cudaMemcpyAsync(hostTiles[t], S.outs + P->tileOff[t], P->tileBytes[t], cudaMemcpyDeviceToHost,
                                   P->down),
                   "pipeline download");
    I360B_CUDA(cudaEventRecord(S.downloaded, P->down), "pipeline order");
    S.used = true;
    ++P->submitted;
    return I360B_SUCCESS;
}

extern "C" int i360b_pipeline_wait(i360b_pipeline* P, float* elapsedMs)
{
    clear_error();
    if (!P) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (elapsedMs) *elapsedMs = 0.0f;
    I360B_CUDA(cudaEventRecord(P->end, P->down), "pipeline timing");
    I360B_CUDA(cudaEventSynchronize(P->end), "pipeline wait");
    if (P->timing && elapsedMs) I360B_CUDA(cudaEventElapsedTime(elapsedMs, P->start, P->end), "pipeline timing");
    P->timing = false;
    for (auto& S : P->slots)
        if (S.used) I360B_TRY(S.plan->plan.check(S.comp));
    return I360B_SUCCESS;
}

extern "C" int i360b_pipeline_autotune(i360b_pipeline* P, int* bandRows, int* dtSlots, float* bestMs)
{
    clear_error();
    if (!P) return fail(I360B_INVALID_PARAM, "Null pointer argument.");
    if (!P->slots[0].used) return fail(I360B_INVALID_PARAM, "Tune after a first submission (the plan needs frames).");
    I360B_TRY(i360b_pipeline_wait(P, nullptr));
    int rows = 0, ring = 0;
    float ms = 0.0f;
    I360B_TRY(i360b_render_plan_autotune(P->slots[0].plan, P->slots[0].comp, &rows, &ring, &ms));
    const int fused = P->slots[0].plan->plan.fusedLevels, shape = P->slots[0].plan->plan.warpShape;
    for (size_t k = 1; k < P->slots.size(); ++k)
    {
        I360B_TRY(P->slots[k].plan->plan.set_fusion(fused, P->slots[k].comp));
        I360B_TRY(P->slots[k].plan->plan.set_warp_shape(shape, P->slots[k].comp));
        I360B_TRY(P->slots[k].plan->plan.set_tuning(rows, ring, P->slots[k].comp));
    }
    if (bandRows) *bandRows = rows;
    if (dtSlots) *dtSlots = ring;
    if (bestMs) *bestMs = ms;
    return I360B_SUCCESS;
}

extern "C" void i360b_pipeline_destroy(i360b_pipeline* P) { delete P; }
