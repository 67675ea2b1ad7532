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

// Trajectory consensus (motion.cpp:532-601) over the pairs of each field
// solved in one colour: pair index lists per field, offset and half-line
// parity shift per pair. Vectors are snapped in place.
constexpr int kTrajMaxPairs = 8;
struct TrajGroup {
  int count;
  int pair[kTrajMaxPairs];     // indices into the colour's pair list
};
struct TrajPair {
  int offset;                  // k - j
  float parity_shift;          // (p_k - p_j) / 2
};
void launch_traj_snap(const MeField* d_fields, const MePair* d_pairs, const TrajGroup* d_groups,
                      int ngroups, const TrajPair* d_tp, int max_h, int max_w, int tile,
                      int tiles_off, float* dy, float* dx, const float* conf, cudaStream_t st);
// Fast-mode predicted vectors audited by VerifyMotion (motion.cpp:490-530,
// sequence.cpp:714-763): for pair p (index base + i of the colour's list) of
// field group grp[i], the median velocity of the group's searched pairs
// predicts the vector; the SSD at its rounding competes with zero. Writes
// mdy / mdx (sdy = sdx = 0) and best at the pair's slot; confidences follow
// with launch_me_confidence.
void launch_traj_verify(const MeField* d_fields, const MePair* d_pairs, int base, int npred,
                        const int* d_grp, const TrajGroup* d_searched, const TrajPair* d_tp,
                        const float* blur, int max_h, int max_w, const MeArgs& a,
                        const float* dy_in, const float* dx_in, float* mdy, float* mdx,
                        float* sdy, float* sdx, float* best, cudaStream_t st,
                        const float* pred_dy = nullptr, const float* pred_dx = nullptr);
// BoxBlur(r = 2) of every field's luma into b.blur (motion.cpp:399-400), as
// launch_motion does first.
void launch_motion_blur(const MeField* d_fields, int nf, int max_h, int max_w, const MeBuffers& b,
                        cudaStream_t st);
// MotionConfidence + final vectors for `npairs` pairs whose tile arrays start
// at the given pointers (pair i at offset i * a.tiles_off).
void launch_me_confidence(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                          int max_w, const MeArgs& a, const float* blur, const float* mdy,
                          const float* mdx, const float* sdy, const float* sdx, const float* best,
                          float* dy, float* dx, float* conf, cudaStream_t st);
// Tile vectors / confidences of a colour's pairs to / from the window-wide
// motion cache (slot gid[i] per pair; fast mode reuses pass-0 motion).
void launch_motion_cache(const int* d_gid, int npairs, int nt, int tiles_off, float* dy, float* dx,
                         float* conf, float* cache, int64_t cache_stride, bool store,
                         cudaStream_t st);
// Coherence gate (sequence.cpp:946-998, ComplexCoherence temporal.cpp:172-202):
// conf_px *= (1 - a) + a gamma, gamma the |box-blurred cross term| over the
// blurred energies of chi_j and chi_k bilinearly warped by the snapped
// per-pixel vectors (radius 6).
struct CohBuffers {
  const float2* chi;           // per field at MeField::y_off (current chi)
  const float* snap_dy;        // snapped tile vectors (pair i at i * tiles_off)
  const float* snap_dx;
  float* terms;                // 4 planes per pair: re, im, |chi_j|^2, |cw|^2
  float* tmp;                  // one plane per pair
  float* conf_px;              // per-pixel confidence per pair (pix_off)
  const int64_t* pix_off;      // per-pair plane offset
  int64_t chan_stride;         // floats between the 4 channel blocks of terms
};
void launch_coherence_gate(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                           int max_w, const MeArgs& a, const CohBuffers& b, float gate,
                           cudaStream_t st);

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

// DrizzleFrame (sequence.cpp:283-421): deposits of every (source k, target
// jt) pair's samples onto the fine grid of frame j0, then the coverage
// blend with the plain woven decode.
struct DrizzlePair {
  int src, tgt;        // field indices (luma / chroma planes, parities)
  int me;              // motion pair index (tiles at me * tiles_off), -1 = self (zero motion, conf 1)
  int pad0;
};
struct DrizzleArgs {
  const float* Y;      // n luma planes, pitched (pitch, plane = h * pitch)
  const float2* C;     // n chroma planes, same layout
  const int* parity;   // n
  int h, w, pitch;
  int tile;
  const float* sdy;    // snapped tile vectors per motion pair
  const float* sdx;
  const float* conf;   // tile confidences per motion pair
  int tiles_off;
  float eps_b;
  int scale, j0;
  float* acc;          // 4 planes (Y, Re C, Im C, weight) of (2 h scale) x w
  float* out_y;        // (2 h scale) x w
  float2* out_c;
};
void launch_drizzle(const DrizzlePair* d_pairs, int npairs, const DrizzleArgs& a, cudaStream_t st);
// the snap of launch_vectors alone (sdy / sdx from dy / dx)
void launch_vec_snap(const MeField* d_fields, const MePair* d_pairs, int npairs, int max_h,
                     int max_w, const MeArgs& a, const float* dy, const float* dx, float* sdy,
                     float* sdx, cudaStream_t st);

}  // namespace hvdg
