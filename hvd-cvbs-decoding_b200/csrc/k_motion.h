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

void launch_motion(const MeField* d_fields, int nf, int max_h, int max_w, const MePair* d_pairs,
                   int npairs, const MeArgs& a, const MeBuffers& b, cudaStream_t st);
void launch_vectors(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                    int max_w, const MeArgs& a, const VecBuffers& v, bool fast_conf,
                    cudaStream_t st);

}  // namespace hvdg
