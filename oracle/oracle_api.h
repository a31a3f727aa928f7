// C-ABI of the CPU oracle (test infrastructure; see oracle_common.h). Images
// are row-major; colour images are interleaved BGR uint8; the cost volume is
// uint8 disparity-major ([D][H*W]); the segmentation pyramid uses the
// reference's ISP layout (segment.cu:884-905).
#pragma once
#include <cstdint>

extern "C" {
// matching cost and colour (oracle_cost.cpp)
void orc_grey_u8(const uint8_t *bgr, int n, uint8_t *out);
void orc_census(const uint8_t *img, int W, int H, uint32_t *out);
void orc_cost_volume(const uint32_t *cL, const uint32_t *cR, int W, int H, int D, uint8_t *vol,
                     float *wta);
void orc_cost_to_right(const uint8_t *volL, int W, int H, int D, uint8_t *volR, float *wta);
void orc_cost_f32(const float *src, int W, int H, int D, float tau, float *vol, float *wta);
void orc_cost_f32_right(const float *src, int W, int H, int D, float tau, float *volR, float *wta);
void orc_grey_f32(const uint8_t *bgr, int n, float *out);
void orc_cost_ad(const float *gL, const float *gR, int W, int H, int D, float tau, int right, float *vol,
                 float *wta);
void orc_lab_set_overrides(const uint32_t *keys, const float *vals, int n);
void orc_lab(const uint8_t *bgr, int n, float *lab4);
void orc_nn_grid(const float *lab4, int W, int H, int *nn, float *dist_min, int *bd);
void orc_nn_grid_nb(const float *lab4, int W, int H, int num_nb, int *nn, float *dist_min, int *bd, float *edist);
void orc_lab_sigma(const uint8_t *bgr, int W, int H, double sigma, float *lab4);

// segmentation (oracle_seg.cpp)
int orc_crtrees(const int *nn, int N, int *clus);
int orc_crtrees_literal(const int *nn, int N, int *clus);
int orc_segment(const float *lab4, int W, int H, int max_levels, int *level_sizes, int *clus,
                float *mean, int *bd, int *bdl);
int orc_segment_target(const float *lab4, int W, int H, int link, int num_nb, int target, int max_levels,
                       int *level_sizes, int *clus, float *mean, int *bd, int *bdl);
int orc_segment_cfg(const float *lab4, int W, int H, int link, int num_nb, int max_levels, int *level_sizes,
                    int *clus, float *mean, int *bd, int *bdl);

// belief propagation (oracle_hbp.cpp)
void orc_round_fp16(const float *in, float *out, long n);
int orc_hbp(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
            const int *bdl, const uint8_t *vol, const float *wta, int W, int H, int D,
            float alpha, float tau_smooth, int min_level, int mode, long max_steps, float *disp,
            float *plane, float *state_belief, float *state_plane);
int orc_hbp_lockstep(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
                     const int *bdl, const uint8_t *vol, const float *wta, int W, int H, int D, float alpha,
                     float tau_smooth, int min_level, int mode, int shadow_fp64, float *disp, double *stats);
int orc_hbp_levels(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
                   const int *bdl, const uint8_t *vol, const float *volf, const float *wta, int W, int H, int D,
                   float data_tau, float alpha, float tau_smooth, int min_level, int mode, float *disp_levels,
                   float *plane_levels);
int orc_hbp_f32(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
                const int *bdl, const float *volf, const float *wta, int W, int H, int D, float data_tau,
                float alpha, float tau_smooth, int min_level, int mode, long max_steps, float *disp,
                float *plane, float *state_belief, float *state_plane);

// post-processing (oracle_post.cpp)
void orc_lr_check(const float *dispL, const float *dispR, float *planeL, int W, int H,
                  uint8_t *failL);
void orc_plane_to_disp(const float *plane, int W, int H, float *disp);
void orc_weighted_median(const uint8_t *bgr, const uint8_t *fail, float *plane, int W, int H,
                         int stable);
void orc_driver_median(float *D, int W, int H);
void orc_weighted_median_gpu(const uint8_t *bgr, const uint8_t *fail, float *plane, int W, int H,
                             const float *wtab, int z_mode);
}
