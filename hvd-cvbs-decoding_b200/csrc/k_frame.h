// k_frame.h -- the frame-buffer ends of the woven-frame decode: de-weave of
// the field-sequential int16 frames into F32 IRE fields (SplitFrameFields,
// frame_bridge.cpp:61-99, and the chroma de-weave of DecodeYcFrameBuffer,
// frame_bridge.cpp:280-302) and the re-weave of the decoded woven planes into
// the 10-bit Y/C frame planes (DecodeFrameBuffer, frame_bridge.cpp:186-252;
// DecodeYcFrameBuffer, frame_bridge.cpp:313-376).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hvdg {

struct FrameSplitArgs {
  const int16_t* frames;     // n source frames, frame_stride samples apart
  int64_t frame_stride;
  const int64_t* line_off;   // FrameLineOffset of every flat line (fh entries)
  int fw, fh, f1;            // samples per line, flat lines, lines of field 1
  float center;              // blanking level (composite) or chroma_dc (C channel)
  float codes_per_ire;       // (white - blanking) / 100
  float* fields;             // 2 n planes of f1 x fw: slot 0 of frame t at 2 t, slot 1 at 2 t + 1
  int64_t field_stride;      // floats between consecutive planes
  // which flat block fills slot 0 (the field woven onto the even rows):
  // order 0 -> block 1, 1 -> block 2, 2 -> block 2 where vote[t] < 0
  int order;
  const int* vote;
};
// grid: 2 n x f1 rows
void launch_frame_split(const FrameSplitArgs& a, int n_frames, cudaStream_t st);

// The field-order vote of every frame (DetectFieldParity behind
// ResolveField1IsBottom, frame_bridge.cpp:152-160): +1 block 1 on top, -1
// block 2 on top, 0 undecided.
struct FrameVoteArgs {
  const int16_t* frames;     // as FrameSplitArgs
  int64_t frame_stride;
  const int64_t* line_off;
  int fh, f1;
  float blank, codes_per_ire;
  int r0, ystep, rows;       // field lines r0, r0 + ystep, ... (rows of them)
  int a0, cols;              // columns a0, a0 + 16, ... (cols of them)
  int blocks;                // CTAs per frame (frame_vote_blocks)
  double* partial;           // scratch: 2 doubles per CTA
  int* arrive;               // scratch: n counters (zeroed by the launch)
  int* vote;                 // n
};
int frame_vote_blocks(int terms);
// grid: n frames x blocks
void launch_frame_vote(const FrameVoteArgs& a, int n_frames, cudaStream_t st);

struct FrameOutArgs {
  // woven planes (one geometry): Y, chi, S at plane_stride apart
  const float* Y;
  const float2* chi;
  const float* S;
  int64_t plane_stride;      // pixels between consecutive planes
  int pitch, h, w;           // woven rows (2 x active lines), active width
  const float4* line_phasor; // h entries per plane, plane t at t * h
  const float2* col_phasor;  // w entries
  const float* amp;          // BurstAmplitudeIre per source field (2 per frame)
  // frames
  const int16_t* passthrough;  // luma source: the composite frames or the Y channel
  int64_t frame_stride;
  const int64_t* line_off;
  int fw, fh, f1, fal, a0;
  float blank, scale;        // blanking level, codes per IRE
  float chroma_gain, nominal_burst;
  int acc;                   // measure the ACC gain from the two bursts
  int yc;                    // 0: composite (chroma = S - Y), 1: Y/C (chroma = Re[chi c])
  int mono;                  // composite only: luma = S, chi = 0 (cfg.monochrome)
  int16_t* luma;             // n frames of fw x fh each
  int16_t* chroma;
  double* u;
  double* v;
};
// grid: n x fh rows
void launch_frame_out(const FrameOutArgs& a, int n_frames, cudaStream_t st);

}  // namespace hvdg
