// C ABI of the engine (include/hbp_b200.h): context, device arena, the
// single-pair pipeline and the stage entry points.
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <cstdlib>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "engine.h"

namespace hbp
{
std::atomic<long> g_launches{0};

void Arena::init(size_t bytes)
{
    release();
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        throw StatusError{HBP_ERR_OUT_OF_MEMORY, "device slab allocation failed"};
    }
    base = static_cast<char *>(p);
    cap = bytes;
    off = 0;
    owned = true;
}

void Arena::attach(void *p, size_t bytes)
{
    release();
    base = static_cast<char *>(p);
    cap = bytes;
    off = 0;
    owned = false;
}

void Arena::release()
{
    if (owned && base)
        cudaFree(base);
    base = nullptr;
    cap = off = 0;
    owned = false;
}

void *Arena::raw(size_t bytes, size_t align)
{
    size_t o = (off + align - 1) / align * align;
    if (o + bytes > cap)
        throw StatusError{HBP_ERR_OUT_OF_MEMORY, "device slab exhausted"};
    off = o + bytes;
    return base + o;
}
} // namespace hbp

using namespace hbp;

// Per-stream state: one lane runs one pair at a time. The context itself is
// lane 0 (used by the stage entry points); batches add lanes so that pairs
// run concurrently, each lane driven by its own host thread.
struct Lane
{
    int device = 0;
    cudaStream_t st = nullptr;
    Arena arena; // pipeline buffers and pyramid
    Arena tmp;   // scratch of sorts / scans / segmentation / BP levels
    Pyramid pyr;
    bool have_pyr = false;
    int *err_dev = nullptr;
    long cap_pixels = 0;
    int cap_disp = 0;
    int bp_blocks = 0; // grid of the persistent BP kernel (0 = whole device)
    KernelProf prof;
};

// Device memory of one pair while its batch is in flight: cost volume(s),
// pyramid(s), per-level BP data and outputs of the right view.
struct Slot
{
    Arena mem;
    long cap_pixels = 0;
    int cap_disp = 0;
    Pyramid pyr, pyrR;
    ViewPlan plan, planR;
    float *dispR = nullptr, *planeR = nullptr, *plane = nullptr;
};

// Online choice of the number of BP streams of a batch, per workload class
// (image size, disparity range, message storage, post mode, views per batch):
// the first batches of a class try each candidate twice (two rounds), timing
// the BP phase on the host clock and keeping each candidate's faster trial (a
// single trial can catch a one-off stall), and later batches use the fastest.
// Views never read one another's data, so the streams change no result, only
// the speed.
struct AutoTune
{
    static constexpr int ROUNDS = 2;
    struct Entry
    {
        std::vector<int> cand;   // stream counts to try
        std::vector<double> ms;  // BP ms per view of each candidate (the faster trial)
        int trials = 0;          // batches measured
        int best = -1;           // index into cand once every candidate ran ROUNDS times
    };
    bool on = true;
    std::map<std::array<int, 6>, Entry> table;
};

struct hbp_ctx : Lane
{
    float *wtab = nullptr; // weighted-median weight table (766 floats)
    int prof_mode = 0;     // 0 off, 1 every pair, 2 first pair of each batch call
    int bp_streams = 0;    // hbp_set_bp_streams
    AutoTune tune;         // used while bp_streams == 0
    int max_lanes = 8;
    std::vector<std::unique_ptr<Lane>> lanes; // extra lanes (1..)
    std::vector<std::unique_ptr<Slot>> slots;
    double phase_ms[4] = {0, 0, 0, 0}; // last batch: prepare, bp, post, total
};

namespace
{
thread_local std::string g_err;
thread_local std::string g_lane_err; // message of a failed batch lane

hbp_status fail(hbp_status s, const std::string &msg)
{
    g_err = msg;
    return s;
}

template <typename F>
hbp_status guarded(F &&f)
{
    try
    {
        f();
        return HBP_OK;
    }
    catch (const CudaFailure &e)
    {
        return fail(HBP_ERR_CUDA, std::string("CUDA error ") + cudaGetErrorString(e.err) + " at " +
                                      e.file + ":" + std::to_string(e.line));
    }
    catch (const StatusError &e)
    {
        return fail(e.st, e.what);
    }
    catch (const std::bad_alloc &)
    {
        return fail(HBP_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    catch (const std::exception &e)
    {
        return fail(HBP_ERR_INTERNAL, e.what());
    }
}

// per pixel: the volume(s), the pyramid (room for the 8-neighbour grid's
// edges) and the BP data; temporaries of the segmentation and the BP setup
size_t slab_bytes(long pixels, int D)
{
    return (size_t)pixels * (size_t)(2 * (D + 16) + 1296) + ((size_t)96 << 20);
}
size_t tmp_bytes(long pixels) { return (size_t)pixels * 560 + ((size_t)64 << 20); }

SegConfig seg_config(const hbp_params &p)
{
    SegConfig s;
    s.link = p.linkage;
    s.num_nb = p.num_nb;
    s.sigma = p.sigma;
    return s;
}

void ensure_capacity(Lane *c, long pixels, int D)
{
    if (pixels <= c->cap_pixels && D <= c->cap_disp)
        return;
    long np = std::max(pixels, c->cap_pixels);
    int nd = std::max(D, c->cap_disp);
    HBP_CUDA(cudaSetDevice(c->device));
    HBP_CUDA(cudaStreamSynchronize(c->st));
    c->have_pyr = false;
    c->arena.init(slab_bytes(np, nd));
    c->tmp.init(tmp_bytes(np));
    c->cap_pixels = np;
    c->cap_disp = nd;
}

void check_device_error(Lane *c)
{
    int h = 0;
    HBP_CUDA(cudaMemcpyAsync(&h, c->err_dev, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    HBP_CUDA(cudaStreamSynchronize(c->st));
    if (h == DERR_BARRIER_TIMEOUT)
        throw StatusError{HBP_ERR_TIMEOUT, "a grid barrier timed out"};
    if (h == DERR_NO_CONVERGENCE)
        throw StatusError{HBP_ERR_NO_CONVERGENCE, "CRTrees did not converge within its bound"};
    if (h != 0)
        throw StatusError{HBP_ERR_INTERNAL, "device error word set"};
}

cudaStream_t pick(hbp_ctx *c, void *s) { return s ? (cudaStream_t)s : c->st; }

void check_dims(int W, int H, int D)
{
    if (W < 16 || H < 16 || W > 65535 || H > 65535 || D < 2 || D > 1024 || D >= W)
        throw StatusError{HBP_ERR_INVALID_ARG, "need 16 <= W,H <= 65535 and 2 <= D <= min(1024, W-1)"};
}

HbpParams to_params(const hbp_params *p, KernelProf *prof = nullptr)
{
    HbpParams q;
    q.prof = prof;
    if (p)
    {
        q.alpha = p->alpha;
        q.tau_smooth = p->tau_smooth;
        q.min_level = p->min_level;
        q.msg_fp16 = p->msg_fp16;
    }
    return q;
}

void ensure_slot(Slot *sl, long pixels, int D)
{
    if (pixels <= sl->cap_pixels && D <= sl->cap_disp)
        return;
    long np = std::max(pixels, sl->cap_pixels);
    int nd = std::max(D, sl->cap_disp);
    sl->mem.init(slab_bytes(np, nd));
    sl->cap_pixels = np;
    sl->cap_disp = nd;
}

// Stages of one pair before BP (main_stereo_hbp_isp.cu:33-64; right view of
// main_bench_middv3.cu:189-202 when post == 2): cost volume(s), segmentation
// pyramid(s) and BP level setup, all on the lane's stream; persistent data in
// the pair's slot.
void prepare_pair(hbp_ctx *ctx, Lane *L, Slot *sl, const uint8_t *dL, const uint8_t *dR, int W, int H,
                  int D, const hbp_params &p, float *disp, float *plane, bool reset_slot = true)
{
    const long n = (long)W * H;
    cudaStream_t st = L->st;
    Arena &a = sl->mem;
    if (reset_slot)
        a.reset();
    L->tmp.reset();
    HBP_CUDA(cudaMemsetAsync(L->err_dev, 0, sizeof(int), st));
    const bool lr = p.post == 2;
    uint32_t *cL = a.alloc<uint32_t>(n), *cR = a.alloc<uint32_t>(n);
    uint8_t *vol = a.alloc<uint8_t>(volume_bytes(W, H, D));
    uint8_t *volR = lr ? a.alloc<uint8_t>(volume_bytes(W, H, D)) : nullptr;
    float *wta = a.alloc<float>(n), *wtaR = lr ? a.alloc<float>(n) : nullptr;
    sl->plane = plane ? plane : a.alloc<float>(3 * n);
    {
        NvtxRange r("cost_volume");
        launch_cost(dL, dR, W, H, D, cL, cR, vol, wta, volR, wtaR, st);
    }
    HbpParams q = to_params(&p);
    const SegConfig seg = seg_config(p);
    {
        NvtxRange r("segmentation");
        segment_image(dL, W, H, sl->pyr, a, L->tmp, L->err_dev, st, seg);
        check_device_error(L);
    }
    L->tmp.reset();
    {
        NvtxRange r("bp_setup");
        hbp_prepare(sl->pyr, vol, wta, D, q, disp, sl->plane, a, L->tmp, st, sl->plan);
    }
    if (lr)
    {
        sl->dispR = a.alloc<float>(n);
        sl->planeR = a.alloc<float>(3 * n);
        L->tmp.reset();
        segment_image(dR, W, H, sl->pyrR, a, L->tmp, L->err_dev, st, seg);
        check_device_error(L);
        L->tmp.reset();
        hbp_prepare(sl->pyrR, volR, wtaR, D, q, sl->dispR, sl->planeR, a, L->tmp, st, sl->planR);
    }
    HBP_CUDA(cudaStreamSynchronize(st));
}

// Stages after BP: the driver's median (post 1) or LR check + fill, weighted
// median and plane -> disparity (post 2). Returns the final plane buffer.
const float *finish_pair(hbp_ctx *ctx, Lane *L, Slot *sl, const uint8_t *dL, int W, int H,
                         const hbp_params &p, float *disp)
{
    const long n = (long)W * H;
    cudaStream_t st = L->st;
    if (p.post == 2)
    {
        size_t m = sl->mem.mark();
        uint8_t *fail1 = sl->mem.alloc<uint8_t>(n), *fail2 = sl->mem.alloc<uint8_t>(n);
        float *plane2 = sl->mem.alloc<float>(3 * n);
        launch_lr_check(disp, sl->dispR, sl->plane, fail1, fail2, W, H, st);
        L->tmp.reset();
        launch_weighted_median(dL, fail1, sl->plane, plane2, W, H, ctx->wtab, L->tmp, st);
        launch_plane_to_disp(plane2, disp, W, H, st);
        HBP_CUDA(cudaMemcpyAsync(sl->plane, plane2, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, st));
        sl->mem.rewind(m);
    }
    else if (p.post == 1)
    {
        L->tmp.reset();
        float *t = L->tmp.alloc<float>(n);
        launch_driver_median(disp, t, W, H, st);
    }
    return sl->plane;
}

void lane_init(Lane *l, int device)
{
    l->device = device;
    HBP_CUDA(cudaSetDevice(device));
    HBP_CUDA(cudaStreamCreateWithFlags(&l->st, cudaStreamNonBlocking));
    HBP_CUDA(cudaMalloc(&l->err_dev, sizeof(int) * 4));
    HBP_CUDA(cudaMemset(l->err_dev, 0, sizeof(int) * 4));
}

void lane_release(Lane *l)
{
    if (l->st)
        cudaStreamSynchronize(l->st);
    l->arena.release();
    l->tmp.release();
    if (l->err_dev)
        cudaFree(l->err_dev);
    if (l->st)
        cudaStreamDestroy(l->st);
    l->st = nullptr;
    l->err_dev = nullptr;
}

Slot *slot_at(hbp_ctx *c, int i)
{
    while ((int)c->slots.size() <= i)
        c->slots.push_back(std::make_unique<Slot>());
    return c->slots[i].get();
}

Lane *lane_at(hbp_ctx *c, int i)
{
    if (i == 0)
        return c;
    while ((int)c->lanes.size() < i)
    {
        auto l = std::make_unique<Lane>();
        lane_init(l.get(), c->device);
        c->lanes.push_back(std::move(l));
    }
    return c->lanes[i - 1].get();
}
} // namespace

extern "C" {

size_t hbp_params_size(void) { return sizeof(hbp_params); }

void hbp_default_params(hbp_params *p)
{
    if (!p)
        return;
    p->alpha = 1000.1f;
    p->tau_smooth = 0.6f;
    p->min_level = 2;
    p->msg_fp16 = 0;
    p->post = 1;
    p->linkage = 2; // CentoridLink, 4-neighbour grid, no blur (test_stereo_hbp_isp.sh:4)
    p->num_nb = 4;
    p->sigma = 0.0;
}

const char *hbp_status_string(hbp_status s)
{
    switch (s)
    {
    case HBP_OK: return "ok";
    case HBP_ERR_INVALID_ARG: return "invalid argument";
    case HBP_ERR_OUT_OF_MEMORY: return "out of memory";
    case HBP_ERR_ADMISSION_REJECTED: return "admission rejected";
    case HBP_ERR_NO_CONVERGENCE: return "no convergence";
    case HBP_ERR_CUDA: return "CUDA error";
    case HBP_ERR_TIMEOUT: return "timeout";
    case HBP_ERR_NOT_READY: return "not ready";
    case HBP_ERR_INTERNAL: return "internal error";
    case HBP_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

const char *hbp_last_error(void) { return g_err.c_str(); }

hbp_status hbp_ctx_create(int device, long max_pixels, int max_disp, hbp_ctx **out)
{
    if (!out || max_pixels < 0 || max_disp < 0)
        return fail(HBP_ERR_INVALID_ARG, "bad context arguments");
    *out = nullptr;
    hbp_ctx *c = new (std::nothrow) hbp_ctx;
    if (!c)
        return fail(HBP_ERR_OUT_OF_MEMORY, "host allocation failed");
    hbp_status s = guarded([&] {
        lane_init(c, device);
        if (const char *e = std::getenv("HBP_LANES"))
            c->max_lanes = std::max(1, std::min(64, std::atoi(e)));
        float tab[766];
        median_weight_table(tab);
        HBP_CUDA(cudaMalloc(&c->wtab, sizeof(tab)));
        HBP_CUDA(cudaMemcpy(c->wtab, tab, sizeof(tab), cudaMemcpyHostToDevice));
        if (max_pixels > 0)
            ensure_capacity(c, max_pixels, max_disp > 0 ? max_disp : 256);
    });
    if (s != HBP_OK)
    {
        hbp_ctx_destroy(c);
        return s;
    }
    *out = c;
    return HBP_OK;
}

void hbp_ctx_destroy(hbp_ctx *c)
{
    if (!c)
        return;
    cudaSetDevice(c->device);
    for (auto &l : c->lanes)
        lane_release(l.get());
    c->lanes.clear();
    for (auto &sl : c->slots)
        sl->mem.release();
    c->slots.clear();
    if (c->wtab)
        cudaFree(c->wtab);
    lane_release(c);
    delete c;
}

void *hbp_ctx_stream(hbp_ctx *c) { return c ? (void *)c->st : nullptr; }

size_t hbp_volume_bytes(int W, int H, int D)
{
    return W > 0 && H > 0 && D > 0 ? volume_bytes(W, H, D) : 0;
}

hbp_status hbp_cost_census_d(hbp_ctx *c, const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D,
                             uint32_t *censusL, uint32_t *censusR, uint8_t *vol, float *wta,
                             uint8_t *volR, float *wtaR, void *stream)
{
    if (!c || !bgrL || !bgrR || !censusL || !censusR || !vol || !wta || (!volR) != (!wtaR))
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        check_dims(W, H, D);
        HBP_CUDA(cudaSetDevice(c->device));
        launch_cost(bgrL, bgrR, W, H, D, censusL, censusR, vol, wta, volR, wtaR, pick(c, stream));
    });
}

hbp_status hbp_lab_d(hbp_ctx *c, const uint8_t *bgr, long n, float *lab4, void *stream)
{
    if (!c || !bgr || !lab4 || n <= 0 || n > (1l << 31) - 1)
        return fail(HBP_ERR_INVALID_ARG, "bad arguments");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        launch_lab(bgr, (int)n, (float4 *)lab4, pick(c, stream));
    });
}

hbp_status hbp_crtrees_d(hbp_ctx *c, const int *nn, int N, int *clus, int *num_clusters, void *stream)
{
    if (!c || !nn || !clus || !num_clusters || N <= 0)
        return fail(HBP_ERR_INVALID_ARG, "bad arguments");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        ensure_capacity(c, std::max<long>(N, c->cap_pixels), std::max(c->cap_disp, 16));
        cudaStream_t st = pick(c, stream);
        // every successor must name a node: check on the host before launching
        std::vector<int> h(N);
        HBP_CUDA(cudaMemcpyAsync(h.data(), nn, sizeof(int) * N, cudaMemcpyDeviceToHost, st));
        HBP_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < N; ++i)
            if (h[i] < 0 || h[i] >= N)
                throw StatusError{HBP_ERR_INVALID_ARG, "successor out of range"};
        c->tmp.reset();
        HBP_CUDA(cudaMemsetAsync(c->err_dev, 0, sizeof(int), st));
        int *num_dev = c->tmp.alloc<int>(1);
        crtrees_labels(nn, N, clus, num_dev, c->err_dev, c->tmp, st);
        HBP_CUDA(cudaMemcpyAsync(num_clusters, num_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
        HBP_CUDA(cudaStreamSynchronize(st));
        int herr = 0;
        HBP_CUDA(cudaMemcpy(&herr, c->err_dev, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr)
            throw StatusError{HBP_ERR_NO_CONVERGENCE, "CRTrees gave up"};
    });
}

hbp_status hbp_segment_d(hbp_ctx *c, const uint8_t *bgr, int W, int H, int *levels, void *stream)
{
    return hbp_segment_cfg_d(c, bgr, W, H, 2, 4, 0.0, levels, stream);
}

hbp_status hbp_lab_sigma_d(hbp_ctx *c, const uint8_t *bgr, int W, int H, double sigma, float *lab4, void *stream)
{
    if (!c || !bgr || !lab4)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        check_dims(W, H, 16);
        SegConfig cfg;
        cfg.sigma = sigma;
        check_seg_config(cfg);
        HBP_CUDA(cudaSetDevice(c->device));
        ensure_capacity(c, (long)W * H, std::max(c->cap_disp, 16));
        cudaStream_t st = pick(c, stream);
        if (sigma > 1.1754943508222875e-38) // FLT_MIN, as segment.cu:805
        {
            c->tmp.reset();
            float4 *blur = c->tmp.alloc<float4>((size_t)W * H);
            launch_lab_blur(bgr, W, H, sigma, blur, (float4 *)lab4, st);
        }
        else
            launch_lab(bgr, W * H, (float4 *)lab4, st);
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_segment_cfg_d(hbp_ctx *c, const uint8_t *bgr, int W, int H, int linkage, int num_nb, double sigma,
                             int *levels, void *stream)
{
    return hbp_segment_target_d(c, bgr, W, H, linkage, num_nb, sigma, 1, levels, stream);
}

hbp_status hbp_segment_target_d(hbp_ctx *c, const uint8_t *bgr, int W, int H, int linkage, int num_nb,
                                double sigma, int target_clus, int *levels, void *stream)
{
    if (!c || !bgr || !levels)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        SegConfig cfg;
        cfg.link = linkage;
        cfg.num_nb = num_nb;
        cfg.sigma = sigma;
        cfg.target = target_clus;
        check_seg_config(cfg);
        if ((long)target_clus >= (long)W * H)
            throw StatusError{HBP_ERR_INVALID_ARG, "target_clus must be below W * H"};
        check_dims(W, H, 16);
        HBP_CUDA(cudaSetDevice(c->device));
        ensure_capacity(c, (long)W * H, std::max(c->cap_disp, 16));
        cudaStream_t st = pick(c, stream);
        c->arena.reset();
        c->tmp.reset();
        HBP_CUDA(cudaMemsetAsync(c->err_dev, 0, sizeof(int), st));
        c->have_pyr = false;
        segment_image(bgr, W, H, c->pyr, c->arena, c->tmp, c->err_dev, st, cfg);
        check_device_error(c);
        c->have_pyr = true;
        *levels = c->pyr.L;
    });
}

hbp_status hbp_segment_draw_d(hbp_ctx *c, int level, int format, const uint8_t *bgr, void *out, void *stream)
{
    if (!c || !out || !c->have_pyr)
        return fail(HBP_ERR_INVALID_ARG, "null pointer or no pyramid");
    if (level < -1 || level >= c->pyr.L)
        return fail(HBP_ERR_INVALID_ARG, "level must be -1 (the last) or 0 .. levels-1");
    if (format < SEG_DRAW_UCHAR3 || format > SEG_DRAW_BOUNDARY)
        return fail(HBP_ERR_INVALID_ARG, "format must be 0 (label BGR bytes), 1 (label ints) or 2 (boundaries)");
    if (format == SEG_DRAW_BOUNDARY && !bgr)
        return fail(HBP_ERR_INVALID_ARG, "the boundary picture needs the BGR image");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = pick(c, stream);
        c->tmp.reset();
        launch_draw_segmentation(c->pyr, level < 0 ? c->pyr.L - 1 : level, format, bgr, out, c->tmp, st);
    });
}

hbp_status hbp_segment_labels_d(hbp_ctx *c, int level, int *labels, int *num_clusters, void *stream)
{
    if (!c || !labels || !c->have_pyr)
        return fail(HBP_ERR_INVALID_ARG, "null pointer or no pyramid");
    if (level < -1 || level >= c->pyr.L)
        return fail(HBP_ERR_INVALID_ARG, "level must be -1 (the last) or 0 .. levels-1");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = pick(c, stream);
        const int lv = level < 0 ? c->pyr.L - 1 : level;
        c->tmp.reset();
        launch_level_labels(c->pyr, lv, labels, c->tmp, st);
        if (num_clusters)
            *num_clusters = level_cluster_count(c->pyr, lv, c->tmp, st);
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_pyramid_levels(hbp_ctx *c, int *sizes, int max_levels)
{
    if (!c || !sizes || !c->have_pyr)
        return fail(HBP_ERR_INVALID_ARG, "no pyramid");
    for (int l = 0; l < c->pyr.L && l < max_levels; ++l)
    {
        sizes[2 * l] = c->pyr.N[l];
        sizes[2 * l + 1] = c->pyr.E[l];
    }
    return HBP_OK;
}

hbp_status hbp_pyramid_device(hbp_ctx *c, const int **clus, const float **mean, const int **bd, const int **bdl)
{
    if (!c || !c->have_pyr)
        return fail(HBP_ERR_INVALID_ARG, "no pyramid");
    if (clus)
        *clus = c->pyr.clus;
    if (mean)
        *mean = c->pyr.sums;
    if (bd)
        *bd = reinterpret_cast<const int *>(c->pyr.bd);
    if (bdl)
        *bdl = c->pyr.bdl;
    return HBP_OK;
}

hbp_status hbp_pyramid_copy(hbp_ctx *c, int *clus, float *mean, int *bd, int *bdl)
{
    if (!c || !c->have_pyr)
        return fail(HBP_ERR_INVALID_ARG, "no pyramid");
    return guarded([&] {
        size_t tn = 0, te = 0;
        for (int l = 0; l < c->pyr.L; ++l)
        {
            tn += c->pyr.N[l];
            te += c->pyr.E[l];
        }
        HBP_CUDA(cudaStreamSynchronize(c->st));
        if (clus)
            HBP_CUDA(cudaMemcpy(clus, c->pyr.clus, sizeof(int) * tn, cudaMemcpyDeviceToHost));
        if (mean)
            HBP_CUDA(cudaMemcpy(mean, c->pyr.sums, sizeof(float) * 6 * tn, cudaMemcpyDeviceToHost));
        if (bd)
            HBP_CUDA(cudaMemcpy(bd, c->pyr.bd, sizeof(int2) * te, cudaMemcpyDeviceToHost));
        if (bdl)
            HBP_CUDA(cudaMemcpy(bdl, c->pyr.bdl, sizeof(int) * te, cudaMemcpyDeviceToHost));
    });
}

hbp_status hbp_infer_d(hbp_ctx *c, const uint8_t *vol, const float *wta, int D, const hbp_params *prm,
                       float *disp, float *plane, void *stream)
{
    if (!c || !vol || !wta || !disp || !c->have_pyr)
        return fail(HBP_ERR_INVALID_ARG, "bad arguments or no pyramid");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        check_dims(c->pyr.W, c->pyr.H, D);
        cudaStream_t st = pick(c, stream);
        HbpParams q = to_params(prm, c->prof.on ? &c->prof : nullptr);
        Slot *sl = slot_at(c, 0);
        ensure_slot(sl, (long)c->pyr.W * c->pyr.H, D);
        sl->mem.reset();
        c->tmp.reset();
        hbp_prepare(c->pyr, vol, wta, D, q, disp, plane, sl->mem, c->tmp, st, sl->plan);
        c->tmp.reset();
        std::vector<ViewPlan *> views{&sl->plan};
        hbp_run_views(views, q, c->tmp, st);
    });
}

size_t hbp_volume_f32_bytes(int W, int H, int D)
{
    return W > 0 && H > 0 && D > 0 ? volume_f32_bytes(W, H, D) : 0;
}

hbp_status hbp_cost_f32_d(hbp_ctx *c, const float *src, int W, int H, int D, float tau, float *vol, float *wta,
                          float *volR, float *wtaR, void *stream)
{
    if (!c || !src || !(tau > 0.0f))
        return fail(HBP_ERR_INVALID_ARG, "null pointer or tau <= 0");
    if (!vol != !wta || !volR != !wtaR || (!vol && !volR))
        return fail(HBP_ERR_INVALID_ARG, "give vol and wta, volR and wtaR, or both pairs");
    return guarded([&] {
        check_dims(W, H, D);
        HBP_CUDA(cudaSetDevice(c->device));
        launch_ingest_f32(src, W, H, D, tau, vol, wta, volR, wtaR, pick(c, stream));
    });
}

hbp_status hbp_cost_ad_d(hbp_ctx *c, const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, float *greyL,
                         float *greyR, float *vol, float *wta, float *volR, float *wtaR, void *stream)
{
    if (!c || !bgrL || !bgrR || !greyL || !greyR)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    if (!vol != !wta || !volR != !wtaR || (!vol && !volR))
        return fail(HBP_ERR_INVALID_ARG, "give vol and wta, volR and wtaR, or both pairs");
    return guarded([&] {
        check_dims(W, H, D);
        HBP_CUDA(cudaSetDevice(c->device));
        launch_cost_ad(bgrL, bgrR, W, H, D, AD_TAU, greyL, greyR, vol, wta, volR, wtaR, pick(c, stream));
    });
}

hbp_status hbp_infer_f32_d(hbp_ctx *c, const float *vol, const float *wta, int D, float tau, const hbp_params *prm,
                           float *disp, float *plane, void *stream)
{
    if (!c || !vol || !wta || !disp || !c->have_pyr || !(tau > 0.0f))
        return fail(HBP_ERR_INVALID_ARG, "bad arguments, tau <= 0 or no pyramid");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        check_dims(c->pyr.W, c->pyr.H, D);
        cudaStream_t st = pick(c, stream);
        HbpParams q = to_params(prm, c->prof.on ? &c->prof : nullptr);
        Slot *sl = slot_at(c, 0);
        ensure_slot(sl, (long)c->pyr.W * c->pyr.H, D);
        sl->mem.reset();
        c->tmp.reset();
        CostVolume cv;
        cv.f32 = vol;
        cv.tau = tau;
        hbp_prepare(c->pyr, cv, wta, D, q, disp, plane, sl->mem, c->tmp, st, sl->plan);
        c->tmp.reset();
        std::vector<ViewPlan *> views{&sl->plan};
        hbp_run_views(views, q, c->tmp, st);
    });
}

hbp_status hbp_infer_levels_d(hbp_ctx *c, const uint8_t *vol, const float *volf, const float *wta, int D, float tau,
                              const hbp_params *prm, int max_levels, float *disp_levels, float *plane_levels,
                              int *num_levels, void *stream)
{
    if (!c || !wta || !disp_levels || !c->have_pyr || (vol == nullptr) == (volf == nullptr))
        return fail(HBP_ERR_INVALID_ARG, "bad arguments (one of vol, volf), or no pyramid");
    if (volf && !(tau > 0.0f))
        return fail(HBP_ERR_INVALID_ARG, "tau <= 0");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        check_dims(c->pyr.W, c->pyr.H, D);
        cudaStream_t st = pick(c, stream);
        HbpParams q = to_params(prm, c->prof.on ? &c->prof : nullptr);
        const int n = c->pyr.L - q.min_level;
        if (q.min_level < 0 || n < 1)
            throw StatusError{HBP_ERR_INVALID_ARG, "min_level must lie in [0, levels-1]"};
        if (n > max_levels)
            throw StatusError{HBP_ERR_INVALID_ARG, "the output holds fewer levels than levels - min_level"};
        q.level_disp = disp_levels;
        q.level_plane = plane_levels;
        Slot *sl = slot_at(c, 0);
        const long HW = (long)c->pyr.W * c->pyr.H;
        ensure_slot(sl, HW, D);
        sl->mem.reset();
        c->tmp.reset();
        CostVolume cv;
        cv.u8 = vol;
        cv.f32 = volf;
        cv.tau = volf ? tau : CENSUS_TAU;
        float *disp = sl->mem.alloc<float>((size_t)HW);
        hbp_prepare(c->pyr, cv, wta, D, q, disp, nullptr, sl->mem, c->tmp, st, sl->plan);
        c->tmp.reset();
        std::vector<ViewPlan *> views{&sl->plan};
        hbp_run_views(views, q, c->tmp, st);
        if (num_levels)
            *num_levels = n;
    });
}

hbp_status hbp_lr_check_d(hbp_ctx *c, const float *dispL, const float *dispR, float *planeL,
                          uint8_t *fail_mask, float *disp_out, int W, int H, void *stream)
{
    if (!c || !dispL || !dispR || !planeL || !fail_mask)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        check_dims(W, H, 2);
        HBP_CUDA(cudaSetDevice(c->device));
        ensure_capacity(c, (long)W * H, std::max(c->cap_disp, 16));
        cudaStream_t st = pick(c, stream);
        c->tmp.reset();
        uint8_t *fail2 = c->tmp.alloc<uint8_t>((size_t)W * H);
        launch_lr_check(dispL, dispR, planeL, fail_mask, fail2, W, H, st);
        if (disp_out)
            launch_plane_to_disp(planeL, disp_out, W, H, st);
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_weighted_median_d(hbp_ctx *c, const uint8_t *bgrL, const uint8_t *fail_mask,
                                 float *plane, float *disp_out, int W, int H, void *stream)
{
    if (!c || !bgrL || !fail_mask || !plane)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        check_dims(W, H, 2);
        HBP_CUDA(cudaSetDevice(c->device));
        ensure_capacity(c, (long)W * H, std::max(c->cap_disp, 16));
        cudaStream_t st = pick(c, stream);
        c->tmp.reset();
        float *copy = c->tmp.alloc<float>(3 * (size_t)W * H);
        HBP_CUDA(cudaMemcpyAsync(copy, plane, sizeof(float) * 3 * W * H, cudaMemcpyDeviceToDevice, st));
        launch_weighted_median(bgrL, fail_mask, copy, plane, W, H, c->wtab, c->tmp, st);
        if (disp_out)
            launch_plane_to_disp(plane, disp_out, W, H, st);
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_weighted_median_gpu_d(hbp_ctx *c, const uint8_t *bgrL, const uint8_t *fail_mask, float *plane,
                                     float *disp_out, int W, int H, void *stream)
{
    if (!c || !bgrL || !fail_mask || !plane)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        check_dims(W, H, 2);
        HBP_CUDA(cudaSetDevice(c->device));
        ensure_capacity(c, (long)W * H, std::max(c->cap_disp, 16));
        cudaStream_t st = pick(c, stream);
        c->tmp.reset();
        float *copy = c->tmp.alloc<float>(3 * (size_t)W * H);
        float *wtab = c->tmp.alloc<float>(766);
        HBP_CUDA(cudaMemcpyAsync(copy, plane, sizeof(float) * 3 * W * H, cudaMemcpyDeviceToDevice, st));
        launch_patch_weights(wtab, st);
        launch_weighted_median_gpu(bgrL, fail_mask, copy, plane, W, H, wtab, c->tmp, st);
        if (disp_out)
            launch_plane_to_disp(plane, disp_out, W, H, st);
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_check_bounded_wait(hbp_ctx *c, int *timed_out)
{
    if (!c || !timed_out)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        ensure_capacity(c, std::max<long>(c->cap_pixels, 1), std::max(c->cap_disp, 16)); // keeps a pyramid
        cudaStream_t st = c->st;
        c->tmp.reset();
        unsigned int *count2 = c->tmp.alloc<unsigned int>(2);
        int *err = c->tmp.alloc<int>(1);
        HBP_CUDA(cudaMemsetAsync(count2, 0, 2 * sizeof(unsigned int), st));
        HBP_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
        launch_barrier_probe(count2, err, 200000, st); // ~50 ms of polls
        int h = 0;
        HBP_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        HBP_CUDA(cudaStreamSynchronize(st));
        *timed_out = h == DERR_BARRIER_TIMEOUT ? 1 : 0;
    });
}

hbp_status hbp_patch_weights_d(hbp_ctx *c, float *wtab766, void *stream)
{
    if (!c || !wtab766)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = pick(c, stream);
        launch_patch_weights(wtab766, st);
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_plane_to_disp_d(hbp_ctx *c, const float *plane, float *disp, int W, int H, void *stream)
{
    if (!c || !plane || !disp)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        check_dims(W, H, 2);
        HBP_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = pick(c, stream);
        launch_plane_to_disp(plane, disp, W, H, st);
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_dev_alloc(int device, size_t bytes, void **ptr)
{
    if (!ptr || bytes == 0)
        return fail(HBP_ERR_INVALID_ARG, "bad arguments");
    *ptr = nullptr;
    return guarded([&] {
        HBP_CUDA(cudaSetDevice(device));
        if (cudaMalloc(ptr, bytes) != cudaSuccess)
        {
            cudaGetLastError();
            *ptr = nullptr;
            throw StatusError{HBP_ERR_OUT_OF_MEMORY, "device allocation failed"};
        }
    });
}

hbp_status hbp_dev_free(void *ptr)
{
    return guarded([&] {
        if (ptr)
            HBP_CUDA(cudaFree(ptr));
    });
}

hbp_status hbp_copy(void *dst, const void *src, size_t bytes)
{
    if ((!dst || !src) && bytes)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        if (bytes)
            HBP_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
    });
}

hbp_status hbp_driver_median_d(hbp_ctx *c, float *disp, int W, int H, void *stream)
{
    if (!c || !disp)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        check_dims(W, H, 2);
        HBP_CUDA(cudaSetDevice(c->device));
        ensure_capacity(c, (long)W * H, std::max(c->cap_disp, 16));
        cudaStream_t st = pick(c, stream);
        c->tmp.reset();
        float *t = c->tmp.alloc<float>((size_t)W * H);
        launch_driver_median(disp, t, W, H, st);
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_driver_median_noalloc_d(float *disp, int W, int H, void *stream)
{
    if (!disp)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    if (W <= 0 || H <= 0)
        return fail(HBP_ERR_INVALID_ARG, "W and H must be positive");
    if ((long)W * H > HBP_NOALLOC_MAX_PIXELS)
        return fail(HBP_ERR_INVALID_ARG, "W*H exceeds HBP_NOALLOC_MAX_PIXELS (2097152), the size of the static scratch");
    return guarded([&] { launch_driver_median_noalloc(disp, W, H, static_cast<cudaStream_t>(stream)); });
}

namespace
{
// Every pair of a batch: preparation on the lanes (one host thread each),
// batched BP of all views on lane 0, then the post stages per pair.
void run_pairs(hbp_ctx *c, int npairs, const uint8_t *const *bgrL, const uint8_t *const *bgrR, int W,
               int H, int D, const hbp_params &p, float *const *disp, float *const *plane)
{
    const long n = (long)W * H;
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point t0) {
        return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    };
    for (double &x : c->phase_ms)
        x = 0;
    const auto t_all = clk::now();
    const int views_per_pair = p.post == 2 ? 2 : 1;
    const int group = 32 / views_per_pair; // pairs per BP batch
    for (int g0 = 0; g0 < npairs; g0 += group)
    {
        const int ng = std::min(group, npairs - g0);
        const int nl = std::max(1, std::min(c->max_lanes, ng));
        std::vector<Lane *> lanes(nl);
        for (int k = 0; k < nl; ++k)
        {
            lanes[k] = lane_at(c, k);
            ensure_capacity(lanes[k], n, D);
        }
        for (int i = 0; i < ng; ++i)
            ensure_slot(slot_at(c, i), n, D);
        std::vector<hbp_status> st(nl, HBP_OK);
        std::vector<std::string> msg(nl);
        const auto t_prep = clk::now();
        auto work = [&](int k) {
            st[k] = guarded([&] {
                HBP_CUDA(cudaSetDevice(c->device));
                for (int i = k; i < ng; i += nl)
                    prepare_pair(c, lanes[k], c->slots[i].get(), bgrL[g0 + i], bgrR[g0 + i], W, H, D, p,
                                 disp[g0 + i], plane ? plane[g0 + i] : nullptr);
            });
            if (st[k] != HBP_OK)
                msg[k] = g_err;
        };
        std::vector<std::thread> th;
        for (int k = 1; k < nl; ++k)
            th.emplace_back(work, k);
        work(0);
        for (auto &t : th)
            t.join();
        for (int k = 0; k < nl; ++k)
            if (st[k] != HBP_OK)
            {
                g_lane_err = "lane " + std::to_string(k) + ": " + msg[k];
                throw StatusError{st[k], g_lane_err.c_str()};
            }
        c->phase_ms[0] += ms_since(t_prep);
        const auto t_bp = clk::now();
        std::vector<ViewPlan *> views;
        for (int i = 0; i < ng; ++i)
        {
            views.push_back(&c->slots[i]->plan);
            if (p.post == 2)
                views.push_back(&c->slots[i]->planR);
        }
        HbpParams q = to_params(&p, c->prof_mode ? &c->prof : nullptr);
        q.bp_streams = c->bp_streams;
        AutoTune::Entry *tune = nullptr;
        if (q.bp_streams == 0 && c->tune.on)
        {
            const std::array<int, 6> key{W, H, D, p.msg_fp16, p.post, (int)views.size()};
            tune = &c->tune.table[key];
            if (tune->cand.empty())
                for (int s : {2, 4, 8, 12, 16})
                    if (s <= (int)views.size())
                        tune->cand.push_back(s);
            if (tune->cand.empty())
                tune->cand.push_back(1);
            q.bp_streams = tune->best >= 0 ? tune->cand[(size_t)tune->best]
                                           : tune->cand[(size_t)tune->trials % tune->cand.size()];
        }
        c->prof.on = c->prof_mode != 0;
        c->tmp.reset();
        const auto t_views = clk::now();
        {
            NvtxRange r("bp");
            hbp_run_views(views, q, c->tmp, c->st);
        }
        if (tune && tune->best < 0)
        {
            const double ms = ms_since(t_views) / (double)views.size();
            const size_t i = (size_t)tune->trials % tune->cand.size();
            if (i >= tune->ms.size())
                tune->ms.push_back(ms);
            else
                tune->ms[i] = std::min(tune->ms[i], ms);
            if (++tune->trials == AutoTune::ROUNDS * (int)tune->cand.size())
                tune->best = (int)(std::min_element(tune->ms.begin(), tune->ms.end()) - tune->ms.begin());
        }
        c->phase_ms[1] += ms_since(t_bp);
        const auto t_post = clk::now();
        NvtxRange rp("post");
        for (int i = 0; i < ng; ++i)
        {
            const float *po = finish_pair(c, c, c->slots[i].get(), bgrL[g0 + i], W, H, p, disp[g0 + i]);
            if (plane && plane[g0 + i] && po != plane[g0 + i])
                HBP_CUDA(cudaMemcpyAsync(plane[g0 + i], po, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, c->st));
        }
        HBP_CUDA(cudaStreamSynchronize(c->st));
        c->phase_ms[2] += ms_since(t_post);
    }
    c->phase_ms[3] = ms_since(t_all);
}
} // namespace

hbp_status hbp_run_pair(hbp_ctx *c, const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D,
                        const hbp_params *prm, float *disp_h, float *plane_h)
{
    if (!c || !bgrL || !bgrR || !disp_h)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    hbp_params def;
    hbp_default_params(&def);
    const hbp_params &p = prm ? *prm : def;
    if (p.post < 0 || p.post > 2)
        return fail(HBP_ERR_INVALID_ARG, "post must be 0, 1 or 2");
    return guarded([&] {
        check_seg_config(seg_config(p));
        check_dims(W, H, D);
        HBP_CUDA(cudaSetDevice(c->device));
        const long n = (long)W * H;
        ensure_capacity(c, n, D);
        cudaStream_t st = c->st;
        c->arena.reset();
        uint8_t *dL = c->arena.alloc<uint8_t>(3 * n), *dR = c->arena.alloc<uint8_t>(3 * n);
        float *disp = c->arena.alloc<float>(n), *plane = c->arena.alloc<float>(3 * n);
        HBP_CUDA(cudaMemcpyAsync(dL, bgrL, 3 * n, cudaMemcpyHostToDevice, st));
        HBP_CUDA(cudaMemcpyAsync(dR, bgrR, 3 * n, cudaMemcpyHostToDevice, st));
        HBP_CUDA(cudaStreamSynchronize(st));
        const uint8_t *pl[1] = {dL}, *pr[1] = {dR};
        float *pd[1] = {disp}, *pp[1] = {plane};
        int keep = c->max_lanes;
        c->max_lanes = 1;
        try
        {
            run_pairs(c, 1, pl, pr, W, H, D, p, pd, pp);
        }
        catch (...)
        {
            c->max_lanes = keep;
            throw;
        }
        c->max_lanes = keep;
        HBP_CUDA(cudaMemcpyAsync(disp_h, disp, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        if (plane_h)
            HBP_CUDA(cudaMemcpyAsync(plane_h, plane, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st));
        HBP_CUDA(cudaStreamSynchronize(st));
    });
}

hbp_status hbp_run_batch_d(hbp_ctx *c, int npairs, const uint8_t *const *bgrL, const uint8_t *const *bgrR,
                           int W, int H, int D, const hbp_params *prm, float *const *disp,
                           float *const *plane)
{
    if (!c || npairs < 0 || (npairs && (!bgrL || !bgrR || !disp)))
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    hbp_params def;
    hbp_default_params(&def);
    const hbp_params &p = prm ? *prm : def;
    if (p.post < 0 || p.post > 2)
        return fail(HBP_ERR_INVALID_ARG, "post must be 0, 1 or 2");
    {
        hbp_status st = guarded([&] { check_seg_config(seg_config(p)); });
        if (st != HBP_OK)
            return st;
    }
    for (int i = 0; i < npairs; ++i)
        if (!bgrL[i] || !bgrR[i] || !disp[i])
            return fail(HBP_ERR_INVALID_ARG, "null pair pointer");
    return guarded([&] {
        check_dims(W, H, D);
        HBP_CUDA(cudaSetDevice(c->device));
        run_pairs(c, npairs, bgrL, bgrR, W, H, D, p, disp, plane);
    });
}

hbp_status hbp_set_lanes(hbp_ctx *c, int lanes)
{
    if (!c || lanes < 1 || lanes > 64)
        return fail(HBP_ERR_INVALID_ARG, "lanes must be in [1, 64]");
    c->max_lanes = lanes;
    return HBP_OK;
}

long hbp_launch_count(void) { return g_launches.load(); }

hbp_status hbp_last_phase_ms(hbp_ctx *c, double *out4)
{
    if (!c || !out4)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    for (int i = 0; i < 4; ++i)
        out4[i] = c->phase_ms[i];
    return HBP_OK;
}

hbp_status hbp_profile_enable(hbp_ctx *c, int on)
{
    if (!c)
        return fail(HBP_ERR_INVALID_ARG, "null context");
    if (on < 0 || on > 3)
        return fail(HBP_ERR_INVALID_ARG, "profile mode must be 0, 1, 2 or 3");
    c->prof_mode = on;
    c->prof.on = on != 0;
    c->prof.breakdown = on == 3;
    c->prof.reset();
    for (auto &l : c->lanes)
        l->prof.reset();
    return HBP_OK;
}

hbp_status hbp_profile_read(hbp_ctx *c, double *ms, long *launches, double *bytes, double *pixels)
{
    if (!c || !ms || !launches || !bytes)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        *ms = c->prof.total_ms();
        *launches = c->prof.launches;
        *bytes = c->prof.bytes;
        if (pixels)
            *pixels = c->prof.pixels;
    });
}

hbp_status hbp_profile_read_kernel(hbp_ctx *c, int kernel, double *ms, long *launches, double *bytes,
                                   double *units)
{
    if (!c || !ms || !launches || !bytes || !units || kernel < 0 || kernel > 1)
        return fail(HBP_ERR_INVALID_ARG, "kernel 0 (data cost) or 1 (edge messages) and four outputs");
    return guarded([&] {
        if (kernel == 0)
        {
            *ms = c->prof.total_ms();
            *launches = c->prof.launches;
            *bytes = c->prof.bytes;
            *units = c->prof.pixels;
        }
        else
        {
            *ms = c->prof.edges.total_ms();
            *launches = c->prof.edges.launches;
            *bytes = c->prof.edges.bytes;
            *units = c->prof.edges.units;
        }
    });
}

hbp_status hbp_set_autotune(hbp_ctx *c, int on)
{
    if (!c)
        return fail(HBP_ERR_INVALID_ARG, "null context");
    c->tune.on = on != 0;
    return HBP_OK;
}

int hbp_autotune_table(hbp_ctx *c, double *rows, int max_rows)
{
    if (!c)
        return -1;
    int n = 0;
    for (const auto &kv : c->tune.table)
        for (size_t i = 0; i < kv.second.ms.size(); ++i, ++n)
            if (rows && n < max_rows)
            {
                double *r = rows + 9 * (size_t)n;
                for (int k = 0; k < 6; ++k)
                    r[k] = kv.first[(size_t)k];
                r[6] = kv.second.cand[i];
                r[7] = kv.second.ms[i];
                r[8] = kv.second.best == (int)i ? 1.0 : 0.0;
            }
    return n;
}

hbp_status hbp_set_bp_streams(hbp_ctx *c, int streams)
{
    if (!c || streams < 0 || streams > 64)
        return fail(HBP_ERR_INVALID_ARG, "streams must be 0 (automatic) .. 64");
    c->bp_streams = streams;
    return HBP_OK;
}

hbp_status hbp_profile_breakdown(hbp_ctx *c, double *ms, long *timed, long *all)
{
    if (!c || !ms || !timed || !all)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] { c->prof.read_breakdown(ms, timed, all); });
}

} // extern "C"

// ---------------------------------------------------------------------------
// Request server: continuous batching of pairs of any size.
//
// Requests are admitted by their device footprint against the server's
// budget, prepared (upload, cost volume, pyramid, BP setup) by preparation
// lanes on their own streams, then join the BP scheduler at its next tick;
// each tick advances every pair in flight by one BP action with one launch per
// kernel kind. A pair leaves after its MAP, runs the driver's median and is
// copied to pinned staging on the scheduler stream; its result reaches the
// caller's buffer when that copy has completed.
namespace
{
double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct ServerSlot
{
    Slot slot;
    size_t bytes = 0;       // device bytes of slot.mem
    float *pinned = nullptr; // disparity staging (cap_pixels floats)
    ~ServerSlot()
    {
        if (pinned)
            cudaFreeHost(pinned);
    }
};

enum ReqState
{
    RQ_QUEUED,
    RQ_PREPARING,
    RQ_BP,
    RQ_FINISHING,
    RQ_DONE
};

struct ServerReq
{
    long long id = 0;
    const uint8_t *L = nullptr, *R = nullptr;
    float *out = nullptr;
    int W = 0, H = 0, D = 0;
    size_t need = 0;
    int state = RQ_QUEUED;
    hbp_status st = HBP_OK;
    std::string err;
    double t_submit = 0, t_done = 0;
    ServerSlot *ss = nullptr;
    bool new_slot = false;
    float *ddisp = nullptr, *dtmp = nullptr;
    cudaEvent_t ev_ready = nullptr, ev_done = nullptr;
};

size_t request_bytes(int W, int H, int D) { return slab_bytes((long)W * H, D); }

// BP streams of the server's scheduler (pairs join the least-loaded one)
#ifndef SERVER_BP_STREAMS
#define SERVER_BP_STREAMS 8
#endif
} // namespace

struct hbp_server
{
    int device = 0;
    hbp_params prm{};
    size_t budget = 0, allocated = 0;
    std::mutex mu;
    std::condition_variable cv_prep, cv_sched, cv_done;
    std::deque<ServerReq *> queued, to_prep, ready;
    std::unordered_map<long long, std::unique_ptr<ServerReq>> reqs;
    std::vector<std::unique_ptr<ServerSlot>> pool; // free slots
    std::vector<std::unique_ptr<ServerSlot>> busy;  // slots of admitted requests
    std::vector<std::unique_ptr<Lane>> lanes;
    std::vector<std::thread> threads;
    long long next_id = 1;
    double bypass_ms = 2000.0; // how long a request that does not fit may be passed
    int preparing = 0; // requests a preparation lane has taken from to_prep
    bool stop = false;
    hbp_status fatal = HBP_OK;
    std::string fatal_msg;
    Lane sched; // error word and stream of the scheduler thread's own work

    // A slot for r: a pooled slot large enough (the smallest), else a new
    // one within the budget, freeing pooled slots (the most recently pooled
    // first) only when that makes room. False when r must wait for requests
    // in flight to finish. Caller holds mu.
    bool take_slot_locked(ServerReq *r)
    {
        const long px = (long)r->W * r->H;
        int pick = -1;
        for (size_t i = 0; i < pool.size(); ++i)
            if (pool[i]->slot.cap_pixels >= px && pool[i]->slot.cap_disp >= r->D &&
                (pick < 0 || pool[i]->bytes < pool[(size_t)pick]->bytes))
                pick = (int)i;
        if (pick >= 0)
        {
            r->ss = pool[(size_t)pick].get();
            busy.push_back(std::move(pool[(size_t)pick]));
            pool.erase(pool.begin() + pick);
            return true;
        }
        size_t pooled = 0;
        for (auto &p : pool)
            pooled += p->bytes;
        if (allocated - pooled + r->need > budget)
            return false; // even an empty pool leaves no room
        while (allocated + r->need > budget && !pool.empty())
        {
            allocated -= pool.back()->bytes;
            pool.pop_back(); // frees its device and pinned memory
        }
        auto ns = std::make_unique<ServerSlot>();
        ns->bytes = r->need;
        allocated += r->need;
        r->ss = ns.get();
        r->new_slot = true;
        busy.push_back(std::move(ns));
        return true;
    }

    // Admit queued requests while memory allows, in arrival order, letting a
    // request that fits pass one that does not (a large pair at the head does
    // not block the small ones behind it) until the oldest waiting request
    // has waited bypass_ms: from then on nothing passes it, so the pairs in
    // flight drain and it is admitted next. Caller holds mu.
    void admit_locked()
    {
        const double now = now_ms();
        for (auto it = queued.begin(); it != queued.end();)
        {
            ServerReq *r = *it;
            if (!take_slot_locked(r))
            {
                if (now - r->t_submit >= bypass_ms)
                    break; // r has waited long enough: hold the rest back
                ++it;
                continue;
            }
            it = queued.erase(it);
            r->state = RQ_PREPARING;
            to_prep.push_back(r);
            cv_prep.notify_one();
        }
    }

    void release_slot_locked(ServerSlot *ss)
    {
        for (size_t i = 0; i < busy.size(); ++i)
            if (busy[i].get() == ss)
            {
                pool.push_back(std::move(busy[i]));
                busy.erase(busy.begin() + (long)i);
                return;
            }
    }

    void finish_locked(ServerReq *r, hbp_status st, const std::string &msg)
    {
        r->st = st;
        r->err = msg;
        r->t_done = now_ms();
        r->state = RQ_DONE;
        if (r->ss)
            release_slot_locked(r->ss);
        r->ss = nullptr;
        admit_locked();
        cv_done.notify_all();
    }

    void prep_loop(Lane *L)
    {
        cudaSetDevice(device);
        for (;;)
        {
            ServerReq *r;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_prep.wait(lk, [&] { return stop || !to_prep.empty(); });
                if (stop && to_prep.empty())
                    return;
                r = to_prep.front();
                to_prep.pop_front();
                ++preparing;
            }
            std::string msg;
            hbp_status st = guarded([&] {
                ServerSlot *ss = r->ss;
                const long n = (long)r->W * r->H;
                if (!ss->pinned || ss->slot.cap_pixels < n)
                {
                    ensure_slot(&ss->slot, n, r->D);
                    if (ss->pinned)
                        cudaFreeHost(ss->pinned);
                    ss->pinned = nullptr;
                    HBP_CUDA(cudaMallocHost(&ss->pinned, sizeof(float) * (size_t)ss->slot.cap_pixels));
                }
                ensure_slot(&ss->slot, n, r->D);
                if (L->cap_pixels < n)
                {
                    L->tmp.init(tmp_bytes(std::max<long>(n, L->cap_pixels)));
                    L->cap_pixels = std::max<long>(n, L->cap_pixels);
                }
                Arena &a = ss->slot.mem;
                a.reset();
                uint8_t *dL = a.alloc<uint8_t>(3 * (size_t)n), *dR = a.alloc<uint8_t>(3 * (size_t)n);
                r->ddisp = a.alloc<float>(n);
                r->dtmp = a.alloc<float>(n);
                HBP_CUDA(cudaMemcpyAsync(dL, r->L, 3 * (size_t)n, cudaMemcpyHostToDevice, L->st));
                HBP_CUDA(cudaMemcpyAsync(dR, r->R, 3 * (size_t)n, cudaMemcpyHostToDevice, L->st));
                hbp_params p = prm;
                p.post = 1;
                prepare_pair(nullptr, L, &ss->slot, dL, dR, r->W, r->H, r->D, p, r->ddisp, nullptr, false);
                if (!r->ev_ready)
                    HBP_CUDA(cudaEventCreateWithFlags(&r->ev_ready, cudaEventDisableTiming));
                HBP_CUDA(cudaEventRecord(r->ev_ready, L->st));
            });
            if (st != HBP_OK)
                msg = g_err;
            std::lock_guard<std::mutex> lk(mu);
            if (st == HBP_OK && fatal != HBP_OK)
            {
                st = fatal;
                msg = fatal_msg;
            }
            if (st != HBP_OK)
                finish_locked(r, st, msg);
            else
            {
                r->state = RQ_BP;
                ready.push_back(r);
            }
            --preparing;
            // the scheduler waits for prepared requests, and at shutdown for
            // the last preparation to end
            cv_sched.notify_one();
        }
    }

    // Fails every request that reached the scheduler (prepared, in BP or
    // finishing) after a fatal error; requests still being prepared fail
    // when their lane sees `fatal`. Caller holds mu.
    void fail_scheduled_locked(hbp_status st, const std::string &msg)
    {
        ready.clear();
        for (auto &kv : reqs)
        {
            const int q = kv.second->state;
            if (q == RQ_BP || q == RQ_FINISHING)
                finish_locked(kv.second.get(), st, msg);
        }
    }

    // Nothing left for the scheduler: no prepared request waiting and none
    // queued for or inside a preparation lane. Caller holds mu.
    bool drained_locked() const { return ready.empty() && to_prep.empty() && preparing == 0; }

    void sched_loop()
    {
        cudaSetDevice(device);
        HbpParams q = to_params(&prm);
        // 8 schedulers on their own streams, ticked in turn; a joining pair
        // goes to the one with the fewest pairs in flight
        std::unique_ptr<BpPool> pool;
        hbp_status pst = guarded([&] { pool = std::make_unique<BpPool>(q, SERVER_BP_STREAMS); });
        if (pst != HBP_OK)
        {
            std::lock_guard<std::mutex> lk(mu);
            fatal = pst;
            fatal_msg = g_err;
            fail_scheduled_locked(fatal, fatal_msg);
            return;
        }
        auto active = [&] { return pool->active(); };
        std::deque<ServerReq *> finishing;
        std::vector<std::pair<void *, int>> fin;
        for (;;)
        {
            std::vector<ServerReq *> join;
            {
                std::unique_lock<std::mutex> lk(mu);
                // at shutdown the scheduler stays until every admitted request
                // has been prepared and run
                if (!active() && finishing.empty())
                    cv_sched.wait(lk, [&] { return !ready.empty() || (stop && drained_locked()); });
                if (stop && !active() && finishing.empty() && drained_locked())
                    return;
                join.assign(ready.begin(), ready.end());
                ready.clear();
            }
            hbp_status st = guarded([&] {
                for (ServerReq *r : join)
                {
                    const int bi = pool->least_loaded();
                    HBP_CUDA(cudaStreamWaitEvent(pool->stream(bi), r->ev_ready, 0));
                    pool->add(bi, &r->ss->slot.plan, r);
                }
                if (pool->active())
                {
                    fin.clear();
                    pool->tick(fin);
                    for (auto &f : fin)
                    {
                        ServerReq *r = static_cast<ServerReq *>(f.first);
                        const cudaStream_t bs = pool->stream(f.second);
                        const long n = (long)r->W * r->H;
                        launch_driver_median(r->ddisp, r->dtmp, r->W, r->H, bs);
                        HBP_CUDA(cudaMemcpyAsync(r->ss->pinned, r->ddisp, sizeof(float) * n,
                                                 cudaMemcpyDeviceToHost, bs));
                        if (!r->ev_done)
                            HBP_CUDA(cudaEventCreateWithFlags(&r->ev_done, cudaEventDisableTiming));
                        HBP_CUDA(cudaEventRecord(r->ev_done, bs));
                        r->state = RQ_FINISHING;
                        finishing.push_back(r);
                    }
                }
                // completions (streams finish out of order: check each)
                const bool busy_bp = active();
                for (size_t i = 0; i < finishing.size();)
                {
                    ServerReq *r = finishing[i];
                    cudaError_t q = busy_bp || i > 0 ? cudaEventQuery(r->ev_done) : cudaEventSynchronize(r->ev_done);
                    if (q == cudaErrorNotReady)
                    {
                        ++i;
                        continue;
                    }
                    HBP_CUDA(q);
                    std::memcpy(r->out, r->ss->pinned, sizeof(float) * (size_t)r->W * r->H);
                    finishing.erase(finishing.begin() + (long)i);
                    std::lock_guard<std::mutex> lk(mu);
                    finish_locked(r, HBP_OK, "");
                }
            });
            if (st != HBP_OK)
            {
                // a CUDA failure on the scheduler stream ends the server: fail
                // everything in flight and every later request
                std::lock_guard<std::mutex> lk(mu);
                fatal = st;
                fatal_msg = g_err;
                fail_scheduled_locked(st, fatal_msg);
                return;
            }
        }
    }
};

extern "C" {

size_t hbp_request_bytes(int W, int H, int D)
{
    return W > 0 && H > 0 && D > 0 ? request_bytes(W, H, D) : 0;
}

hbp_status hbp_server_create(int device, size_t budget_bytes, int prep_lanes, const hbp_params *prm,
                             hbp_server **out)
{
    if (!out || budget_bytes == 0 || prep_lanes < 1 || prep_lanes > 64)
        return fail(HBP_ERR_INVALID_ARG, "need a budget > 0 and 1..64 preparation lanes");
    if (prm && (prm->post < 0 || prm->post > 1))
        return fail(HBP_ERR_INVALID_ARG, "the server runs post = 0 or 1 (driver median)");
    if (prm)
    {
        hbp_status st = guarded([&] { check_seg_config(seg_config(*prm)); });
        if (st != HBP_OK)
            return st;
    }
    *out = nullptr;
    auto s = std::make_unique<hbp_server>();
    s->device = device;
    s->budget = budget_bytes;
    hbp_default_params(&s->prm);
    if (prm)
        s->prm = *prm;
    hbp_status st = guarded([&] {
        lane_init(&s->sched, device);
        for (int i = 0; i < prep_lanes; ++i)
        {
            s->lanes.push_back(std::make_unique<Lane>());
            lane_init(s->lanes.back().get(), device);
        }
    });
    if (st != HBP_OK)
        return st;
    hbp_server *raw = s.get();
    for (auto &l : s->lanes)
        s->threads.emplace_back([raw, L = l.get()] { raw->prep_loop(L); });
    s->threads.emplace_back([raw] { raw->sched_loop(); });
    *out = s.release();
    return HBP_OK;
}

void hbp_server_destroy(hbp_server *s)
{
    if (!s)
        return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // finish what was admitted; drop what is still queued (nobody can
        // read their status: the server is freed below)
        for (ServerReq *r : s->queued)
        {
            r->st = HBP_ERR_CANCELLED;
            r->state = RQ_DONE;
        }
        s->queued.clear();
        s->stop = true;
        s->cv_done.notify_all();
        s->cv_prep.notify_all();
        s->cv_sched.notify_all();
    }
    for (auto &t : s->threads)
        t.join();
    for (auto &kv : s->reqs)
    {
        if (kv.second->ev_ready)
            cudaEventDestroy(kv.second->ev_ready);
        if (kv.second->ev_done)
            cudaEventDestroy(kv.second->ev_done);
    }
    s->pool.clear();
    s->busy.clear();
    for (auto &l : s->lanes)
        lane_release(l.get());
    lane_release(&s->sched);
    delete s;
}

hbp_status hbp_submit(hbp_server *s, const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D,
                      float *disp, long long *id)
{
    if (!s || !bgrL || !bgrR || !disp || !id)
        return fail(HBP_ERR_INVALID_ARG, "null pointer");
    return guarded([&] {
        check_dims(W, H, D);
        auto r = std::make_unique<ServerReq>();
        r->L = bgrL;
        r->R = bgrR;
        r->out = disp;
        r->W = W;
        r->H = H;
        r->D = D;
        r->need = request_bytes(W, H, D);
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->fatal != HBP_OK)
            throw StatusError{s->fatal, "the server stopped after a CUDA error"};
        if (r->need > s->budget)
            throw StatusError{HBP_ERR_ADMISSION_REJECTED, "the pair needs more device memory than the server's budget"};
        r->id = s->next_id++;
        r->t_submit = now_ms();
        *id = r->id;
        ServerReq *raw = r.get();
        s->reqs.emplace(r->id, std::move(r));
        s->queued.push_back(raw);
        s->admit_locked();
    });
}

hbp_status hbp_poll(hbp_server *s, long long id)
{
    if (!s)
        return fail(HBP_ERR_INVALID_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
        return fail(HBP_ERR_INVALID_ARG, "unknown request id");
    if (it->second->state != RQ_DONE)
        return HBP_ERR_NOT_READY;
    if (it->second->st != HBP_OK)
        return fail(it->second->st, it->second->err);
    return HBP_OK;
}

hbp_status hbp_wait(hbp_server *s, long long id, double timeout_ms, double *latency_ms)
{
    if (!s)
        return fail(HBP_ERR_INVALID_ARG, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
        return fail(HBP_ERR_INVALID_ARG, "unknown request id");
    ServerReq *r = it->second.get();
    auto done = [&] { return r->state == RQ_DONE; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done))
        return fail(HBP_ERR_TIMEOUT, "request still running");
    const hbp_status st = r->st;
    const std::string msg = r->err;
    if (latency_ms)
        *latency_ms = r->t_done - r->t_submit;
    if (r->ev_ready)
        cudaEventDestroy(r->ev_ready);
    if (r->ev_done)
        cudaEventDestroy(r->ev_done);
    s->reqs.erase(it);
    if (st != HBP_OK)
        return fail(st, msg);
    return HBP_OK;
}

} // extern "C"
