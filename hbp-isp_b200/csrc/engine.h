// Internal interfaces of the B200 HBP-ISP engine (not part of the C-ABI).
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "common.cuh"

namespace hbp
{

constexpr int P = 4, K = 12;       // particles per slot group, slots per node
constexpr int PC_CHUNK = 256;      // plane-cost chunk (32 slots x 8 deep)
constexpr float CENSUS_TAU = 25.0f; // stereo_cost.cu:433

// ---------------------------------------------------------------------------
// Device memory: one slab per pair, carved with a bump allocator (no
// cudaMalloc inside a request once the slab exists).
struct Arena
{
    char *base = nullptr;
    size_t cap = 0, off = 0;
    bool owned = false;

    Arena() = default;
    ~Arena() { release(); }
    Arena(const Arena &) = delete;
    Arena &operator=(const Arena &) = delete;

    void init(size_t bytes);
    void attach(void *p, size_t bytes);
    void release();
    void reset() { off = 0; }
    void *raw(size_t bytes, size_t align = 256);
    template <typename T>
    T *alloc(size_t n)
    {
        return static_cast<T *>(raw(sizeof(T) * (n ? n : 1)));
    }
    size_t mark() const { return off; }
    void rewind(size_t m) { off = m; }
};

// Temporary device memory for scans/sorts, reused across calls on one stream.
struct Scratch
{
    Arena *arena;
};

// ---------------------------------------------------------------------------
// cost.cu
// Cost volume layout: 8x4-pixel tiles in raster order, disparity-major inside
// a tile; byte (x, y, d) sits at vol_offset(x, y, d). Tiles that overhang the
// image hold 0 for the missing pixels.
constexpr int VT_W = 8, VT_H = 4, VT_BYTES = VT_W * VT_H;
__host__ __device__ __forceinline__ size_t vol_tile_base(int x, int y, int TX, int D)
{
    return ((size_t)(y >> 2) * TX + (x >> 3)) * (size_t)D * VT_BYTES + ((y & 3) << 3) + (x & 7);
}
__host__ __device__ __forceinline__ size_t vol_offset(int x, int y, int d, int TX, int D)
{
    return vol_tile_base(x, y, TX, D) + (size_t)d * VT_BYTES;
}
inline size_t volume_bytes(int W, int H, int D)
{
    return (size_t)((W + VT_W - 1) / VT_W) * ((H + VT_H - 1) / VT_H) * (size_t)D * VT_BYTES;
}
void launch_cost(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, uint32_t *cL,
                 uint32_t *cR, uint8_t *vol, float *wta, uint8_t *volR, float *wtaR,
                 cudaStream_t st);
// The MC-CNN path's volume: src [D][H][W] floats -> the tiled float layout
// (volume_f32_bytes), with the out-of-view fill and truncation at tau, and WTA;
// the left view into vol/wta and (each pair optional) the right view into volR/wtaR.
inline size_t volume_f32_bytes(int W, int H, int D) { return volume_bytes(W, H, D) * sizeof(float); }
void launch_ingest_f32(const float *src, int W, int H, int D, float tau, float *vol, float *wta, float *volR,
                       float *wtaR, cudaStream_t st);
// The AD cost (truncation tau = 30 in the reference): both views' float grey
// images, then the tiled float volume(s) and WTA as launch_ingest_f32.
constexpr float AD_TAU = 30.0f; // stereo_cost.cu:425
void launch_cost_ad(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, float tau, float *greyL,
                    float *greyR, float *vol, float *wta, float *volR, float *wtaR, cudaStream_t st);

// lab.cu
void launch_lab(const uint8_t *bgr, int n, float4 *lab, cudaStream_t st);
// LAB of the image blurred with sigma > 0 (tmp4: W*H float4 scratch)
constexpr int BLUR_MAX_S = 7; // the reference's filter buffer: 15 x 15 (segment.hpp:303-306)
int blur_radius(double sigma);
void launch_lab_blur(const uint8_t *bgr, int W, int H, double sigma, float4 *tmp4, float4 *lab, cudaStream_t st);

// scan_sort.cu
size_t scan_scratch_bytes(long n);
void exclusive_scan(const int *in, int *out, long n, int *total_dev, Arena &tmp, cudaStream_t st);
// Stable LSD radix sort of (key, value) pairs on the low `bits` bits of the
// keys; results land in keys/vals (ping-pong through alt buffers).
void radix_sort_pairs_u32(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt, uint32_t *vals_alt,
                          long n, int bits, Arena &tmp, cudaStream_t st);
void radix_sort_keys_u64(uint64_t *keys, uint64_t *keys_alt, long n, int bits, Arena &tmp,
                         cudaStream_t st);

// crtrees.cu: component labels (0..n-1 in label order); returns the count
// through num_dev (device int). err_dev receives DeviceErr codes.
void crtrees_labels(const int *nn, int N, int *clus, int *num_dev, int *err_dev, Arena &tmp,
                    cudaStream_t st);
// one block waiting at a grid barrier for a block that never comes, with the
// given poll limit (the bounded-wait check)
void launch_barrier_probe(unsigned int *count2, int *err, long spin_limit, cudaStream_t st);

// ---------------------------------------------------------------------------
// Segmentation pyramid in the reference's ISP layout (segment.cu:884-905),
// device resident.
struct Pyramid
{
    int W = 0, H = 0, L = 0;
    std::vector<int> N, E;                  // per level
    std::vector<size_t> node_off, edge_off; // offsets into the concatenated arrays
    std::vector<size_t> child_base, nb_base;
    int *clus = nullptr;   // sum N: node -> parent
    float *sums = nullptr; // 6 * sum N (per level channel-major: L, a, b, x, y, count)
    int2 *bd = nullptr;    // sum E: (source, target), sorted by source
    int *bdl = nullptr;    // sum E: boundary lengths
    // derived per level: children grouped by parent (increasing child index)
    // with offsets per parent, and CSR offsets of the edges by source
    uint32_t *child = nullptr; // sum N
    int *child_off = nullptr;  // per level N_{l+1} + 1 at child_base[l]
    int *nb_off = nullptr;     // per level N_l + 1 at nb_base[l]
};

// SegHAC's configuration (segment.hpp:248): linkage (segment.hpp:8-16),
// pixel neighbourhood and pre-blur. The path's default is CentroidLink, 4, 0.
enum SegLinkage
{
    LINK_MIN = 0,
    LINK_MAX = 1,
    LINK_CENTROID = 2,
    LINK_WARD = 3
};
struct SegConfig
{
    int link = LINK_CENTROID;
    int num_nb = 4;
    double sigma = 0.0;
    int target = 1; // target_clus: 1 = the whole pyramid; > 1 stops at that many superpixels
};
// Rejects configurations the reference cannot run (HBP_ERR_INVALID_ARG).
void check_seg_config(const SegConfig &cfg);
struct Pyramid;
// Each pixel's cluster after pyramid level `level` (LabelIntFormat, 0-based
// labels), and the number of those clusters.
void launch_level_labels(const Pyramid &pyr, int level, int *labels, Arena &tmp, cudaStream_t st);
int level_cluster_count(const Pyramid &pyr, int level, Arena &tmp, cudaStream_t st);
// draw_segmentation's pictures of that label image, in the reference's
// SegFormat numbering: W*H*3 bytes (label+1 as BGR bytes, or the boundaries
// in red over `bgr`) or W*H ints (label+1).
enum SegDraw
{
    SEG_DRAW_UCHAR3 = 0,
    SEG_DRAW_INT = 1,
    SEG_DRAW_BOUNDARY = 2
};
void launch_draw_segmentation(const Pyramid &pyr, int level, int format, const uint8_t *bgr, void *out,
                              Arena &tmp, cudaStream_t st);

// segment.cu: SegHAC::run_ms with LabelISPFormat and cfg.target. Uses `a` for
// the pyramid and `tmp` for temporaries; the host learns each level's size
// (one small device-to-host read per level).
void segment_image(const uint8_t *bgr, int W, int H, Pyramid &pyr, Arena &a, Arena &tmp,
                   int *err_dev, cudaStream_t st, const SegConfig &cfg = SegConfig{});

// ---------------------------------------------------------------------------
// hbp.cu
// Event timing for the roofline report: while enabled, the data-cost and the
// edge-message launches of every 16th BP tick of the first BP stream are
// bracketed by events.
struct EventTimer
{
    std::vector<cudaEvent_t> ev; // start/stop pairs, reused
    size_t used = 0;
    double bytes = 0; // algorithmic bytes of the timed launches
    double units = 0; // edges (or list positions) the timed launches covered
    long launches = 0;
    void reset()
    {
        used = 0;
        bytes = 0;
        units = 0;
        launches = 0;
    }
    void mark(cudaStream_t st)
    {
        if (used == ev.size())
        {
            cudaEvent_t e;
            HBP_CUDA(cudaEventCreate(&e));
            ev.push_back(e);
        }
        HBP_CUDA(cudaEventRecord(ev[used++], st));
    }
    double total_ms()
    {
        double t = 0;
        for (size_t i = 0; i + 1 < used; i += 2)
        {
            float ms = 0;
            HBP_CUDA(cudaEventSynchronize(ev[i + 1]));
            HBP_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
            t += ms;
        }
        return t;
    }
    EventTimer() = default;
    EventTimer(const EventTimer &) = delete;
    EventTimer &operator=(const EventTimer &) = delete;
    ~EventTimer()
    {
        for (cudaEvent_t e : ev)
            cudaEventDestroy(e);
    }
};

struct KernelProf
{
    EventTimer edges; // k_edges launches (units: directed edges)
    bool on = false;
    std::vector<cudaEvent_t> ev; // start/stop pairs, reused
    size_t used = 0;
    double bytes = 0;  // algorithmic bytes of the timed launches
    double pixels = 0; // list positions (pixels) the timed launches covered
    long launches = 0;
    // breakdown mode: every BP kernel of every 8th step timed, per (kind, level)
    static constexpr int KINDS = 10, LEVELS = 32;
    bool breakdown = false;
    std::vector<cudaEvent_t> evb;
    size_t usedb = 0;
    std::vector<int> tagb;           // kind * LEVELS + level of each timed pair
    long count[KINDS * LEVELS] = {}; // every launch, timed or not
    void reset()
    {
        used = 0;
        bytes = 0;
        pixels = 0;
        launches = 0;
        edges.reset();
        usedb = 0;
        tagb.clear();
        for (long &x : count)
            x = 0;
    }
    void markb(cudaStream_t st)
    {
        if (usedb == evb.size())
        {
            cudaEvent_t e;
            HBP_CUDA(cudaEventCreate(&e));
            evb.push_back(e);
        }
        HBP_CUDA(cudaEventRecord(evb[usedb++], st));
    }
    void read_breakdown(double *ms, long *timed, long *all)
    {
        for (int i = 0; i < KINDS * LEVELS; ++i)
        {
            ms[i] = 0;
            timed[i] = 0;
            all[i] = count[i];
        }
        for (size_t i = 0; i + 1 < usedb; i += 2)
        {
            float t = 0;
            HBP_CUDA(cudaEventSynchronize(evb[i + 1]));
            HBP_CUDA(cudaEventElapsedTime(&t, evb[i], evb[i + 1]));
            ms[tagb[i / 2]] += t;
            timed[tagb[i / 2]] += 1;
        }
    }
    void mark(cudaStream_t st)
    {
        if (used == ev.size())
        {
            cudaEvent_t e;
            HBP_CUDA(cudaEventCreate(&e));
            ev.push_back(e);
        }
        HBP_CUDA(cudaEventRecord(ev[used++], st));
    }
    double total_ms()
    {
        double t = 0;
        for (size_t i = 0; i + 1 < used; i += 2)
        {
            float ms = 0;
            HBP_CUDA(cudaEventSynchronize(ev[i + 1]));
            HBP_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
            t += ms;
        }
        return t;
    }
};

struct HbpParams
{
    float alpha = 1000.1f;
    float tau_smooth = 0.6f;
    int min_level = 2;
    int msg_fp16 = 0;
    int bp_streams = 0; // BP scheduler streams of a batch (0: automatic)
    KernelProf *prof = nullptr;
    // run_ms_vis: every level's map, top level L-1 first, down to min_level
    // (HW floats and HW x 3 floats per level; level_plane may be null)
    float *level_disp = nullptr, *level_plane = nullptr;
};



// One view ready for BP: per-level device data, BP buffers and its sizes.
struct ViewPlan
{
    struct Impl;
    Impl *impl;
    int L = 0, min_level = 0, D = 0, HW = 0;
    bool levels = false;                     // every level's map is kept (run_ms_vis)
    std::vector<int> levelN, levelE, levelC; // nodes, edges, data-cost chunks per level
    ViewPlan();
    ~ViewPlan();
    ViewPlan(const ViewPlan &) = delete;
    ViewPlan &operator=(const ViewPlan &) = delete;
};

// The data term's cost volume in the tiled layout: uint8 Census costs
// (truncation 25, stereo_cost.cu:433) or floats (MC-CNN, truncation 0.5,
// stereo_cost.cu:438). tau is also the cost of a disparity outside [0, D-1).
struct CostVolume
{
    const uint8_t *u8 = nullptr;
    const float *f32 = nullptr;
    float tau = CENSUS_TAU;
};

// Level setup of one view (persistent data in `persist`, temporaries in `tmp`);
// BP writes disparity (HW floats) and planes (HW x 3, may be null) there.
void hbp_prepare(const Pyramid &pyr, const CostVolume &cv, const float *wta, int D,
                 const HbpParams &prm, float *disp, float *plane, Arena &persist, Arena &tmp,
                 cudaStream_t st, ViewPlan &vp);
inline void hbp_prepare(const Pyramid &pyr, const uint8_t *vol, const float *wta, int D,
                        const HbpParams &prm, float *disp, float *plane, Arena &persist, Arena &tmp,
                        cudaStream_t st, ViewPlan &vp)
{
    CostVolume cv;
    cv.u8 = vol;
    hbp_prepare(pyr, cv, wta, D, prm, disp, plane, persist, tmp, st, vp);
}
// HBP_ISP::run_ms for prepared views, run together to completion.
void hbp_run_views(const std::vector<ViewPlan *> &views, const HbpParams &prm, Arena &tmp,
                   cudaStream_t st);

// Continuous BP over prepared views (HBP_ISP::run_ms per view). Each tick
// advances every active view by one action (level setup, one candidate/BP
// step, the level's final select, or MAP), with one launch per kernel kind
// serving all views (32 per launch descriptor). Views join with add() before
// any tick and leave after their MAP; a view's results do not depend on the
// others in flight. Launches go to `st`; the caller orders the views'
// preparation before their first tick (e.g. with an event).
class BpScheduler
{
  public:
    BpScheduler(const HbpParams &prm, cudaStream_t st);
    ~BpScheduler();
    BpScheduler(const BpScheduler &) = delete;
    BpScheduler &operator=(const BpScheduler &) = delete;
    void add(ViewPlan *vp, void *user);
    // One tick; appends the user tags of views whose MAP it launched.
    void tick(std::vector<void *> &finished);
    int active() const;

  private:
    struct View;
    struct Impl;
    Impl *impl;
};

// BpSchedulers on their own streams, ticked in turn from one host thread, so
// that kernels of different views share the GPU (a latency-bound data cost
// beside an issue-bound message pass). The caller picks a scheduler for a
// view (least_loaded(): fewest views in flight), orders the view's setup
// before that scheduler's stream, and adds it; tick() reports each finished
// view with its scheduler's index.
class BpPool
{
  public:
    BpPool(const HbpParams &prm, int streams);
    ~BpPool();
    BpPool(const BpPool &) = delete;
    BpPool &operator=(const BpPool &) = delete;
    int least_loaded() const;
    void add(int i, ViewPlan *vp, void *user);
    bool active() const;
    void tick(std::vector<std::pair<void *, int>> &finished);
    void sync();
    cudaStream_t stream(int i) const { return st_[(size_t)i]; }
    int size() const { return (int)st_.size(); }

  private:
    std::vector<cudaStream_t> st_;
    std::vector<std::unique_ptr<BpScheduler>> sc_;
};

// Streams a batch of `views` uses by default: two views per stream, at most 8.
int bp_default_streams(int views);

// ---------------------------------------------------------------------------
// post.cu
void launch_lr_check(const float *dispL, const float *dispR, float *planeL, uint8_t *fail,
                     uint8_t *fail2, int W, int H, cudaStream_t st);
void launch_plane_to_disp(const float *plane, float *disp, int W, int H, cudaStream_t st);
void median_weight_table(float *host766);
void launch_weighted_median(const uint8_t *bgr, const uint8_t *fail, const float *plane_in,
                            float *plane_out, int W, int H, const float *wtab, Arena &tmp,
                            cudaStream_t st);
void launch_driver_median(float *disp, float *tmp, int W, int H, cudaStream_t st);
// median_filter_gpu: the reference's GPU variant of the weighted median
// (device patch weights from launch_patch_weights, in lab.cu)
void launch_patch_weights(float *wtab766, cudaStream_t st);
void launch_weighted_median_gpu(const uint8_t *bgr, const uint8_t *fail, const float *plane_in,
                                float *plane_out, int W, int H, const float *wtab766, Arena &tmp,
                                cudaStream_t st);
// same filter with the file-scope static scratch of noalloc.cu (allocates nothing)
void launch_driver_median_noalloc(float *disp, int W, int H, cudaStream_t st);

} // namespace hbp
