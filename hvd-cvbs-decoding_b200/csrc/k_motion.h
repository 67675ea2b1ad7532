// k_motion.h -- launchers of the motion-estimation and warp kernels (k_motion.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hvdg {

// One luma plane taking part in motion estimation.
struct MeField {
  int h, w, pitch, dpitch;  // dpitch: row pitch of the 4x-decimated plane
  int64_t y_off;            // luma plane offset (floats) in MeBuffers::luma
  int64_t t_off;            // blur scratch offset in MeBuffers::tmp
  int64_t b_off;            // blurred plane offset in MeBuffers::blur
  int64_t d_off;            // decimated plane offset in MeBuffers::dec
};

// EstimateMotion(y_ref = field `ref`, y_cur = field `cur`).
struct MePair {
  int ref, cur;
};

struct MeArgs {
  int tile, search;
  int coarse_off;  // per-pair stride of the coarse tile arrays
  int tiles_off;   // per-pair stride of the full-resolution tile arrays
};

struct MeBuffers {
  const float* luma;
  float* tmp;
  float* blur;
  float* dec;
  float *cdy, *cdx;                  // coarse vectors
  float *mdy, *mdx, *sdy, *sdx, *best;
  float *dy, *dx, *conf;             // EstimateMotion outputs (per tile)
};

struct VecBuffers {
  const float *dy, *dx, *conf;       // per-tile motion
  float *snap_dy, *snap_dx;          // snapped tile vectors
  int2* src_idx;                     // per-pixel warp source (sy, sx), per pair
  const int64_t* pix_off;            // per-pair offset of the per-pixel planes
  float *c2, *c2_snap, *c2_snap2;    // fast-mode confidence tiles
  float* conf_tmp;                   // per-pixel scratch
  float* conf_px;                    // per-pixel confidence, per pair
  size_t conf_bytes;
};

// Integer-SAD mode (me_mode 1): block x block tiles, exhaustive +-range.
struct SadArgs {
  int block, range;
  int tiles_off;   // per-pair stride of the tile arrays
};

struct SadBuffers {
  const float* luma;               // per field at MeField::y_off
  int* vsum;                       // per field at MeField::t_off (vertical window sums)
  int* qblur;                      // per field at MeField::b_off (quantised, blurred luma)
  float *mdy, *mdx, *sdy, *sdx;    // per tile: integer vector, sub-pel offsets
  double *bestv, *s1, *s2, *npx;   // per tile: biased SSD (IRE^2), sums of A, pixel count
  float *dy, *dx, *conf;           // per tile outputs (as EstimateMotion's)
};

int sad_max_block();
int sad_max_range();
void launch_motion_sad(const MeField* d_fields, int nf, int max_h, int max_w,
                       const MePair* d_pairs, int npairs, const SadArgs& a, const SadBuffers& b,
                       cudaStream_t st);
void launch_motion(const MeField* d_fields, int nf, int max_h, int max_w, const MePair* d_pairs,
                   int npairs, const MeArgs& a, const MeBuffers& b, cudaStream_t st);
void launch_vectors(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                    int max_w, const MeArgs& a, const VecBuffers& v, bool fast_conf,
                    cudaStream_t st);

}  // namespace hvdg
