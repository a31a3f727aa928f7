/*
 * hbp_b200.h - C ABI of the B200 HBP-ISP stereo engine.
 *
 * The engine takes a rectified BGR8 pair and produces a disparity map with the
 * method of HBP-ISP ("Hierarchical Belief Propagation on Image Segmentation
 * Pyramid"). Each entry point below replaces one step of the reference's C++
 * API (file:line into the reference tree) and keeps its meaning; the C++
 * classes in include/hbp_isp/ restore the reference's class interface on top
 * of these functions.
 *
 * Conventions: plain pointers and sizes only. Colour images are interleaved
 * BGR uint8 (the reference reads channel x as blue, imutil.cu:11-13);
 * disparity maps are H x W float32; plane maps are H x W x 3 float32 (a, b, c
 * with d = a*x + b*y + c). Functions whose names end in _d take device
 * pointers and an optional CUDA stream (cudaStream_t passed as void*, NULL =
 * the context's stream); all others take host pointers. A context is used by
 * one host thread at a time. Every call returns an hbp_status; on failure
 * hbp_last_error() describes the cause.
 */
#ifndef HBP_B200_H
#define HBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hbp_status
{
    HBP_OK = 0,
    HBP_ERR_INVALID_ARG = 1,        /* bad size, pointer or parameter */
    HBP_ERR_OUT_OF_MEMORY = 2,      /* device or pinned memory exhausted */
    HBP_ERR_ADMISSION_REJECTED = 3, /* request exceeds the server's memory budget */
    HBP_ERR_NO_CONVERGENCE = 4,     /* a bounded device loop gave up (CRTrees) */
    HBP_ERR_CUDA = 5,               /* CUDA runtime error */
    HBP_ERR_TIMEOUT = 6,            /* wait ended before the request finished */
    HBP_ERR_NOT_READY = 7,          /* poll: request still running */
    HBP_ERR_INTERNAL = 8,           /* invariant violated (capacity, ...) */
    HBP_ERR_CANCELLED = 9           /* request dropped by hbp_server_destroy */
} hbp_status;

typedef struct hbp_ctx hbp_ctx;

/* Parameters of one run. Defaults (hbp_default_params) are the reference's
 * Census run, test_stereo_hbp_isp.sh:4: alpha 1000.1, tau_smooth 0.6,
 * min_level 2 (CentroidLink, 4-grid, sigma 0 are fixed). */
typedef struct hbp_params
{
    float alpha;      /* data-term weight lambda (hbp_isp.hpp:353-363) */
    float tau_smooth; /* smoothness truncation (hbp_isp.cu:349) */
    int min_level;    /* finest pyramid level inferred (hbp_isp.cu:1328) */
    int msg_fp16;     /* 1: BP messages stored as FP16 (FP32 arithmetic) */
    int post;         /* 0: none; 1: driver 7-tap median (main_stereo_hbp_isp.cu:75);
                         2: right view + LR check/fill + weighted median + plane->disp
                            (main_bench_middv3.cu:189-219) */
    /* the segmentation's configuration, the drivers' argv link, num_nb, sigma
     * (main_stereo_hbp_isp.cu:15-29; SegHAC, segment.hpp:248) */
    int linkage;      /* 0 MinLink, 1 MaxLink, 2 CentoridLink (default), 3 WardLink */
    int num_nb;       /* pixel grid neighbours: 4 (default) or 8 */
    double sigma;     /* Gaussian pre-blur, 0 (default) or round(3 sigma) <= 7 */
} hbp_params;

void hbp_default_params(hbp_params *p);
/* sizeof(hbp_params) in this build, for bindings that declare the struct
 * themselves (ctypes, cgo) to check their layout (no reference counterpart). */
size_t hbp_params_size(void);
const char *hbp_status_string(hbp_status s);
const char *hbp_last_error(void);

/* Context: device, stream, device memory slab sized for images up to
 * max_pixels x max_disp (0 = sized lazily on first use). */
hbp_status hbp_ctx_create(int device, long max_pixels, int max_disp, hbp_ctx **out);
void hbp_ctx_destroy(hbp_ctx *ctx);
void *hbp_ctx_stream(hbp_ctx *ctx);

/* ---------------------------------------------------------------- stages */

/* StereoCost::compute_stereo_cost("Census") (stereo_cost.cu:421-445) with the
 * grey conversion of the constructor (stereo_cost.cu:290-297): census of both
 * views, the uint8 cost volume holding min(popcount, 25), and the WTA
 * disparity. With volR/wtaR non-NULL the right-view volume and WTA of
 * StereoCost::cost_to_right (stereo_cost.cu:488-516) are produced in the same
 * pass.
 * Volume layout (hbp_volume_bytes(W, H, D) bytes): 8 x 4-pixel tiles in
 * raster order, TX = ceil(W/8) tiles per row; inside a tile disparity-major
 * with 32 bytes per disparity. Cost(x, y, d) is at byte
 *   ((y/4 * TX + x/8) * D + d) * 32 + (y%4) * 8 + x%8;
 * overhanging tile entries are 0. */
size_t hbp_volume_bytes(int W, int H, int D);
hbp_status hbp_cost_census_d(hbp_ctx *ctx, const uint8_t *bgrL, const uint8_t *bgrR, int W, int H,
                             int D, uint32_t *censusL, uint32_t *censusR, uint8_t *vol,
                             float *wta, uint8_t *volR, float *wtaR, void *stream);

/* The MC-CNN cost path: StereoCost::compute_stereo_cost("MC-CNN")
 * (stereo_cost.cu:436-441, read_volume_from_file :396-418, WTA_D_k :249-266).
 * src is the network's device volume [D][H][W] (float, as in im0.acrt, which
 * the reference reads from disk). Columns x <= d take the value at x = d,
 * values are truncated at tau (the reference uses 0.5) and WTA keeps the
 * first minimum. vol (hbp_volume_f32_bytes) receives the volume in the tiled
 * layout above, in floats; wta the H x W WTA disparity. volR / wtaR receive
 * the volume after cost_to_right (stereo_cost.cu:488-516) and its WTA. Either
 * pair may be NULL, not both. */
size_t hbp_volume_f32_bytes(int W, int H, int D);
hbp_status hbp_cost_f32_d(hbp_ctx *ctx, const float *src, int W, int H, int D, float tau, float *vol,
                          float *wta, float *volR, float *wtaR, void *stream);

/* The AD cost: StereoCost::compute_stereo_cost("AD") (stereo_cost.cu:421-429,
 * ad_cost :9-43, grey img_BGR_to_grey imutil.cu:116-130, WTA_D_k :249-266).
 * greyL / greyR (H x W floats) receive the float grey images; vol / wta (and
 * volR / wtaR, the view after cost_to_right) as hbp_cost_f32_d, with
 * min(|gL(x) - gR(x - d)|, 30) for x >= D - 1 and 0 for every d where
 * x < D - 1 (the reference's border). HBP runs on it through hbp_infer_f32_d
 * with tau 30. */
hbp_status hbp_cost_ad_d(hbp_ctx *ctx, const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D,
                         float *greyL, float *greyR, float *vol, float *wta, float *volR, float *wtaR,
                         void *stream);

/* BGR -> CIELAB float4 (L, a, b, 1) (imutil.cu:4-40, segment.cu:795-809). */
hbp_status hbp_lab_d(hbp_ctx *ctx, const uint8_t *bgr, long n, float *lab4, void *stream);

/* CRTrees::get_clus + compact_clus_label (CRTrees.cu:315-354, :387-403):
 * connected components of the successor array nn (every entry in [0, N)),
 * labelled 0..n-1; *num_clusters receives n. Synchronous. */
hbp_status hbp_crtrees_d(hbp_ctx *ctx, const int *nn, int N, int *clus, int *num_clusters,
                         void *stream);

/* SegHAC(CentroidLink, 4, 0, LabelISPFormat, 1).run_ms() + ISPData
 * (segment.cu:1279-1321, hbp_isp.hpp:24-46): builds the image segmentation
 * pyramid of a device BGR image inside the context (replacing any previous
 * one) and returns its number of levels. hbp_pyramid_levels gives per level
 * (num_clus, num_bd); hbp_pyramid_copy copies the reference's ISP arrays
 * (clus, mean sums [6][N_l], bd pairs, bdl, concatenated over levels) to host
 * buffers of at least the summed sizes. */
hbp_status hbp_segment_d(hbp_ctx *ctx, const uint8_t *bgr, int W, int H, int *levels, void *stream);
/* The same for any SegHAC configuration of the reference's drivers (segment.hpp:
 * 248, segment.cu:1279-1321): linkage 0 MinLink, 1 MaxLink, 2 CentoridLink,
 * 3 WardLink; num_nb 4 or 8 (compute_1nn_grid_k, segment.cu:57-195); sigma >= 0
 * the Gaussian pre-blur (img_gauss_blur, imutil.cu:397-497; round(3 sigma)
 * <= 7, the reference's 15 x 15 filter buffer). hbp_segment_d is
 * (2, 4, 0.0). */
hbp_status hbp_segment_cfg_d(hbp_ctx *ctx, const uint8_t *bgr, int W, int H, int linkage, int num_nb,
                             double sigma, int *levels, void *stream);
/* The same with SegHAC's target_clus (segment.cu:1016-1041, :1279-1321):
 * 1 is hbp_segment_cfg_d; target_clus > 1 (below W * H) stops the pyramid at
 * the first level whose CRTrees pass leaves at most target_clus clusters,
 * after get_target_clus has broken the clusters with the largest summed
 * 1-NN distances into their children so that exactly target_clus remain (the
 * superpixel mode). The last level's clus then maps its nodes to the
 * superpixels 0 .. target_clus-1. Where the reference's order is unspecified
 * (float atomic distance sums, atomicSub label hand-out) children count in
 * increasing index. */
hbp_status hbp_segment_target_d(hbp_ctx *ctx, const uint8_t *bgr, int W, int H, int linkage, int num_nb,
                                double sigma, int target_clus, int *levels, void *stream);
/* SegHAC's LabelIntFormat output (update_image_label, segment.cu:871-883,
 * draw_segmentation :907-951) for the context's pyramid: every pixel's
 * cluster after pyramid level `level` (0 .. levels-1; -1 = the last level,
 * the superpixels of the target mode), W*H ints on the device, numbered from
 * 0 (the reference's image adds 1), and the number of those clusters in
 * *num_clusters (may be NULL). The reference draws one such image per level
 * with target_clus 1 and only the last otherwise. Synchronous. */
hbp_status hbp_segment_labels_d(hbp_ctx *ctx, int level, int *labels, int *num_clusters, void *stream);

/* SegHAC::draw_segmentation (segment.cu:907-951) for pyramid level `level`
 * (-1 = the last), with the reference's SegFormat numbers: format 0
 * (LabelUchar3Format) writes W*H*3 bytes, label+1 as B,G,R = bits 0-7, 8-15,
 * 16-23; format 1 (LabelIntFormat) writes W*H ints, label+1; format 2
 * (BoundaryFormat) writes W*H*3 bytes, the BGR image `bgr` (device, the one
 * segmented) with every pixel whose left or upper neighbour has another label
 * set to (0,0,255). `out` is device memory. Synchronous. */
hbp_status hbp_segment_draw_d(hbp_ctx *ctx, int level, int format, const uint8_t *bgr, void *out, void *stream);
/* SegHAC::img_CPU_to_GPU with sigma (segment.cu:795-809): CIELAB float4 of
 * the blurred image (the fourth channel is the blurred constant 1), into
 * lab4 (W*H float4). sigma = 0 gives hbp_lab_d's result. */
hbp_status hbp_lab_sigma_d(hbp_ctx *ctx, const uint8_t *bgr, int W, int H, double sigma, float *lab4,
                           void *stream);
hbp_status hbp_pyramid_levels(hbp_ctx *ctx, int *sizes, int max_levels);
hbp_status hbp_pyramid_copy(hbp_ctx *ctx, int *clus, float *mean, int *bd, int *bdl);
/* The same arrays in place on the device (SegHAC / ISPData g_isp_clus_d,
 * g_isp_mean_d, g_isp_bd_d (int pairs), g_isp_bdl_d; segment.hpp:131-150,
 * hbp_isp.hpp:18-21). Valid until the context's next segmentation. */
hbp_status hbp_pyramid_device(hbp_ctx *ctx, const int **clus, const float **mean, const int **bd,
                              const int **bdl);

/* HBP_ISP(ISPData, StereoData, alpha, tau_smooth).run_ms(min_level)
 * (hbp_isp.hpp:288-386, hbp_isp.cu:1313-1346) on the context's pyramid and a
 * device cost volume / WTA from hbp_cost_census_d. Writes disparity (H x W)
 * and plane labels (H x W x 3; may be NULL). */
hbp_status hbp_infer_d(hbp_ctx *ctx, const uint8_t *vol, const float *wta, int D,
                       const hbp_params *prm, float *disp, float *plane, void *stream);
/* The same on a float volume from hbp_cost_f32_d, with its truncation tau
 * (also the cost of a plane outside [0, D-1); hbp_isp.cu:205-227). The
 * reference's MC-CNN runs use alpha 1.3 (bench_MiddV3_train.sh:6). */
hbp_status hbp_infer_f32_d(hbp_ctx *ctx, const float *vol, const float *wta, int D, float tau,
                           const hbp_params *prm, float *disp, float *plane, void *stream);

/* HBP_ISP::run_ms_vis (hbp_isp.cu:1348-1383) without its superpixel drawing
 * (cvtColor, circles, lines: visualisation): every level's map from the top
 * level L-1 down to min_level. disp_levels receives (L - min_level) H x W
 * float disparities, top level first; plane_levels (may be NULL) the H x W x 3
 * planes in the same order; *num_levels (may be NULL) their count. Give
 * exactly one of vol (uint8, from hbp_cost_census_d) or volf (float, from
 * hbp_cost_f32_d / hbp_cost_ad_d, with its tau; tau is ignored for vol).
 * HBP_ERR_INVALID_ARG when L - min_level > max_levels. The last map equals
 * hbp_infer_d's result; the top level's is 0 everywhere (its planes are
 * never written; the reference maps uninitialised memory there). */
hbp_status hbp_infer_levels_d(hbp_ctx *ctx, const uint8_t *vol, const float *volf, const float *wta, int D,
                              float tau, const hbp_params *prm, int max_levels, float *disp_levels,
                              float *plane_levels, int *num_levels, void *stream);

/* PostProcess::left_right_check + plane_label_to_disp (post_process.cu:4-110,
 * :373-390): updates planeL in place, writes the failure mask (0/255) and the
 * disparity of the updated planes. */
hbp_status hbp_lr_check_d(hbp_ctx *ctx, const float *dispL, const float *dispR, float *planeL,
                          uint8_t *fail, float *disp_out, int W, int H, void *stream);
/* PostProcess::median_filter + plane_label_to_disp (post_process.cu:112-185). */
hbp_status hbp_weighted_median_d(hbp_ctx *ctx, const uint8_t *bgrL, const uint8_t *fail,
                                 float *plane, float *disp_out, int W, int H, void *stream);
/* PostProcess::median_filter_gpu (post_process.cu:188-371), the reference's
 * GPU variant: as hbp_weighted_median_d, but with the device's expf weights,
 * float weight sums, the disparity evaluated as fma(a, x, b * y) + c, and the
 * samples in bubble_sort's order (post_process.cu:216-229), whose ties can
 * differ from the CPU variant's. */
hbp_status hbp_weighted_median_gpu_d(hbp_ctx *ctx, const uint8_t *bgrL, const uint8_t *fail,
                                     float *plane, float *disp_out, int W, int H, void *stream);
/* A self-test with no counterpart in the reference: one block waits at the
 * engine's grid barrier for a block that is never launched. Every device wait
 * of the engine is bounded; this one runs out after ~50 ms, records a
 * time-out in the device error word and returns, and *timed_out is set to 1.
 * The context stays usable afterwards. */
hbp_status hbp_check_bounded_wait(hbp_ctx *ctx, int *timed_out);
/* The GPU variant's 766 patch weights expf(-k / 10), k = 0..765 (device
 * memory), as compute_patch_weight evaluates them (post_process.cu:199-213). */
hbp_status hbp_patch_weights_d(hbp_ctx *ctx, float *wtab766, void *stream);
/* PostProcess::plane_label_to_disp for one view (post_process.cu:373-390):
 * disp = a*x + b*y + c of each pixel's plane. */
hbp_status hbp_plane_to_disp_d(hbp_ctx *ctx, const float *plane, float *disp, int W, int H, void *stream);
/* medianFilter of the single-pair driver (main_stereo_hbp_isp.cu:120-192). */
hbp_status hbp_driver_median_d(hbp_ctx *ctx, float *disp, int W, int H, void *stream);

/* The same driver median with no context and no device allocation. This entry
 * point has no counterpart in the reference: it serves callers that may not
 * allocate device memory, e.g. a frame loop that reserved its whole device
 * budget up front (cudaMalloc/cudaFree synchronise the device and stall the
 * other streams) or a PyTorch process whose caching allocator already holds
 * the free memory, where creating a context could fail.
 *   - Scratch: a file-scope device array of HBP_NOALLOC_MAX_PIXELS floats
 *     (8 MiB); W*H above that is rejected with HBP_ERR_INVALID_ARG before
 *     anything is launched. No scratch contents need to start at zero: the
 *     first pass writes every entry the second pass reads.
 *   - Device: the calling thread's current CUDA device, which must own disp
 *     and stream (NULL = the legacy default stream).
 *   - Setup: the first call on each device looks up the scratch address
 *     (cudaGetSymbolAddress, which loads the module holding it); make that
 *     first call before any stream capture begins.
 *   - Asynchronous: enqueues two kernels on stream and returns; disp is
 *     updated in place when the stream reaches them.
 *   - One scratch per device: calls whose executions may overlap (different
 *     streams or host threads without ordering between them) race on it;
 *     order them on one stream or with events. */
#define HBP_NOALLOC_MAX_PIXELS 2097152L
hbp_status hbp_driver_median_noalloc_d(float *disp, int W, int H, void *stream);

/* Device memory for callers that hold no CUDA runtime of their own (the C++
 * classes in include/hbp_isp/ use these): allocation on a device, release,
 * and a synchronous copy in any direction (host or device pointers). */
hbp_status hbp_dev_alloc(int device, size_t bytes, void **ptr);
hbp_status hbp_dev_free(void *ptr);
hbp_status hbp_copy(void *dst, const void *src, size_t bytes);

/* ------------------------------------------------------------ whole pair */

/* The single-pair path of main_stereo_hbp_isp.cu:33-76 (post = 1) or of
 * MidV3_LR, main_bench_middv3.cu:169-219 (post = 2), on host buffers:
 * uploads the pair, runs every stage on the device and downloads the
 * disparity (and planes when plane != NULL). */
hbp_status hbp_run_pair(hbp_ctx *ctx, const uint8_t *bgrL, const uint8_t *bgrR, int W, int H,
                        int D, const hbp_params *prm, float *disp, float *plane);

/* A batch of same-size pairs whose images already sit in device memory
 * (arrays of npairs device pointers, held on the host); plane may be NULL or
 * hold NULL entries. Same path and outputs as hbp_run_pair per pair. Pairs run
 * concurrently on up to hbp_set_lanes() lanes (own stream and device slabs
 * each, default 8 or $HBP_LANES), one host thread per lane; the call returns
 * when every pair is done. */
hbp_status hbp_run_batch_d(hbp_ctx *ctx, int npairs, const uint8_t *const *bgrL,
                           const uint8_t *const *bgrR, int W, int H, int D, const hbp_params *prm,
                           float *const *disp, float *const *plane);

hbp_status hbp_set_lanes(hbp_ctx *ctx, int lanes);
/* BP of a batch runs on up to 8 streams (two pairs each) by default, so that
 * kernels of different pairs share the GPU; streams > 0 fixes the number
 * (1 = every BP kernel alone on the device). 0 restores the default. */
hbp_status hbp_set_bp_streams(hbp_ctx *ctx, int streams);
/* While the stream count is automatic (0), batches autotune it (no reference
 * counterpart): per class (W, H, D, msg_fp16, post, views per batch) the first
 * batches try 2, 4, 8, 12 and 16 streams (those not above the views), two
 * batches each in two rounds, timing the BP phase and keeping each count's
 * faster batch, and later batches use the fastest. The streams change no
 * result. on = 0 turns it off (the default 8 streams, two views each). The
 * table's rows hold each count's faster batch. */
hbp_status hbp_set_autotune(hbp_ctx *ctx, int on);
/* The autotuner's measurements: up to max_rows rows of 9 doubles (W, H, D,
 * msg_fp16, post, views, streams, BP ms per view, 1 if chosen); returns the
 * number of rows (or -1 for a null context). rows may be NULL to count. */
int hbp_autotune_table(hbp_ctx *ctx, double *rows, int max_rows);

/* ------------------------------------------------------------ serving */

/* A request server on one GPU (no reference counterpart: the reference runs
 * one pair per process). Pairs of any size and disparity range are submitted
 * from host buffers and run with continuous batching: a request is admitted
 * when its device footprint (hbp_request_bytes) fits in the budget beside the
 * requests in flight, prepared (upload, cost volume, pyramid, BP setup) by one
 * of prep_lanes host threads on its own stream, and joins the BP of the pairs
 * already running at the next BP step; it leaves after its MAP and the
 * driver's median. Each result equals hbp_run_pair's (post 1) bit for bit,
 * whatever runs beside it. prm applies to every request (post 0 or 1).
 * The budget counts the pairs' device slabs; the preparation lanes' scratch
 * (about 480 B per pixel of the largest pair, + 64 MB, per lane) comes on top.
 * A queued request that does not fit yet may be passed by later ones that
 * do, until it has waited 2 s; then nothing passes it and it is admitted as
 * soon as the pairs in flight free its memory.
 * All functions are thread safe. Input and output buffers must stay valid
 * until hbp_wait returns for the request. */
typedef struct hbp_server hbp_server;
size_t hbp_request_bytes(int W, int H, int D);
hbp_status hbp_server_create(int device, size_t budget_bytes, int prep_lanes, const hbp_params *prm,
                             hbp_server **out);
/* Finishes the admitted requests (writes their outputs), drops the ones
 * still queued for memory, joins the server's threads and frees everything.
 * The server and its request ids are invalid afterwards: hbp_poll and
 * hbp_wait must not be called on it, so a caller that needs every result
 * waits for its requests before destroying the server. */
void hbp_server_destroy(hbp_server *srv);
/* HBP_ERR_ADMISSION_REJECTED when the pair can never fit in the budget. */
hbp_status hbp_submit(hbp_server *srv, const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D,
                      float *disp, long long *request_id);
/* HBP_ERR_NOT_READY while running; otherwise the request's final status. */
hbp_status hbp_poll(hbp_server *srv, long long request_id);
/* Waits (timeout_ms < 0: without limit; HBP_ERR_TIMEOUT when it runs out),
 * reports submit-to-result latency, and forgets the request. */
hbp_status hbp_wait(hbp_server *srv, long long request_id, double timeout_ms, double *latency_ms);

/* -------------------------------------------------------- measurement */

/* Number of kernels the library has launched since it was loaded. */
long hbp_launch_count(void);
/* Host wall time (ms) of the last hbp_run_batch_d / hbp_run_pair call:
 * [0] preparation (cost volume, pyramid, BP setup; concurrent lanes),
 * [1] batched BP, [2] post stages, [3] whole call. */
hbp_status hbp_last_phase_ms(hbp_ctx *ctx, double *out4);
/* While enabled, launches of the data-cost kernel (the dominant kernel of the
 * path) of every 16th BP tick of the first BP stream are bracketed by CUDA
 * events (modes 1 and 2; 0 = off). Read returns the summed device time, the
 * launch count, the algorithmic bytes and the pixels (list positions) of the
 * timed launches (pixels may be NULL). Enabling resets the totals. */
hbp_status hbp_profile_enable(hbp_ctx *ctx, int on);
hbp_status hbp_profile_read(hbp_ctx *ctx, double *ms, long *launches, double *bytes, double *pixels);
/* The same per kernel: 0 the data cost (units: list positions), 1 the edge
 * messages, timed on the same ticks (units: directed edges; bytes per edge
 * 24 B of metadata and 12 message values read and written, plus per node its
 * planes, beliefs, RANSAC points and kept slots). */
hbp_status hbp_profile_read_kernel(hbp_ctx *ctx, int kernel, double *ms, long *launches, double *bytes,
                                   double *units);
/* Mode 3 additionally times every BP kernel of every 8th BP step. Breakdown
 * fills three arrays of 10 x 32 entries indexed [kind][level] (kinds: 0 node
 * select, 1 child candidates, 2 neighbour candidates, 3 set candidates,
 * 4 data cost, 5 edge messages, 6 prior data cost, 7 init nodes, 8 MAP):
 * summed device ms and count of the timed launches, and count of all launches. */
hbp_status hbp_profile_breakdown(hbp_ctx *ctx, double *ms, long *timed, long *all);

#ifdef __cplusplus
}
#endif
#endif /* HBP_B200_H */
