/*
 * hvdg.h -- C ABI of the B200 (sm_100a) holographic-variational Y/C separator.
 *
 * Plain C: no C++ or torch types cross this boundary, only pointers, sizes
 * and POD structs. Every entry point returns an hvdg_status; none throws.
 *
 * Reference interfaces replaced (paths relative to the hvd-cvbs-decoding
 * project; each declaration below cites the one it stands in for):
 *
 *   hvd-core/src/frame_bridge.h:196-199   hvd::DecodeFrameSequenceWindow
 *   hvd-core/src/frame_bridge.h:149-150   hvd::DecodeFrameBuffer (engine.h:89 DecodeFrame)
 *   hvd-core/src/frame_bridge.h:223-226   hvd::DecodeYcFrameBuffer (engine.h:106 DecodeChromaOnly)
 *   hvd-core/src/engine/engine.h:112-114  HvdEngine::DecodeSequenceWindow
 *   hvd-core/src/engine/sequence.h:60-61  PrepareFieldObs
 *   hvd-core/src/engine/sequence.h:98-101 DecodeFieldWindow
 *   hvd-core/src/engine/lockin.h:31-59    BurstLockinPhase / BurstLockinPhasePal
 *   hvd-core/src/engine/lockin.h:36       BurstAmplitudeIre
 *   hvd-core/src/engine/holographic_init.h:221-223  HolographicInit
 *   hvd-core/src/engine/variational.h:76-78         VariationalRefine
 *   hvd-core/src/engine/motion.h:49-50              EstimateMotion
 *
 * Units and layouts follow the reference: planes are row-major float32,
 * index (y, x) -> y * width + x; complex planes are interleaved (re, im)
 * float pairs, chi = V - iU in IRE; composite samples are IRE referenced to
 * blanking (ntsc_geometry.h:225-228).
 *
 * Where the reference passes a carrier plane exp(i*phi) (FieldObs::carrier),
 * this ABI passes the per-line burst-locked phase theta[] plus the PAL
 * V-switch vswitch[] and rebuilds the carrier exactly as MakeCarrier /
 * MakeCarrierPal do (ntsc_geometry.cpp:29-47, 75-93): the device never
 * stores a carrier plane.
 *
 * Threading: one hvdg_ctx per host thread (same contract as one HvdEngine
 * per thread, frame_bridge.h:137-140). Calls on one context are serialised
 * on that context's CUDA stream and are synchronous unless named *_async.
 */
#ifndef HVDG_H_
#define HVDG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HVDG_ABI_VERSION 1

typedef enum hvdg_status {
  HVDG_OK = 0,
  HVDG_ERR_BAD_ARGUMENT = 1,    /* null pointer, n < 0, bad enum value */
  HVDG_ERR_BAD_GEOMETRY = 2,    /* active window / burst window out of range, h or w < 2 */
  HVDG_ERR_NONFINITE_INPUT = 3, /* NaN / Inf among the input samples */
  HVDG_ERR_DEVICE_TIMEOUT = 4,  /* a bounded device-side wait expired */
  HVDG_ERR_CUDA = 5,            /* a CUDA runtime call failed (see hvdg_last_error) */
  HVDG_ERR_OUT_OF_MEMORY = 6,   /* device or pinned allocation failed */
  HVDG_ERR_UNSUPPORTED = 7,     /* a configuration this build does not implement */
  HVDG_ERR_NO_DEVICE = 8        /* no CUDA device / wrong architecture */
} hvdg_status;

typedef enum hvdg_standard {
  HVDG_STD_NTSC = 0,  /* VideoStandard::kNtsc  (ntsc_geometry.h:137) */
  HVDG_STD_PAL = 1,   /* VideoStandard::kPal   */
  HVDG_STD_PAL_M = 2  /* VideoStandard::kPalM  */
} hvdg_standard;

typedef enum hvdg_sample_type {
  HVDG_SAMPLES_F32_IRE = 0, /* float, already IRE (FieldInput::samples) */
  HVDG_SAMPLES_U16 = 1,     /* uint16 codes; IRE = (s - blanking) / ((white - blanking) / 100) */
  HVDG_SAMPLES_S16 = 2      /* int16 codes (the plugin's 10-bit frame buffers), same level map */
} hvdg_sample_type;

/* Mirror of hvd::FieldGeometry (ntsc_geometry.h:66-191). */
typedef struct hvdg_geometry {
  int32_t field_width;             /* samples per line incl. blanking (910 NTSC, 1135 PAL) */
  int32_t field_height;            /* lines per field (263 NTSC, 313 PAL) */
  int32_t active_video_start;      /* first active sample (inclusive) */
  int32_t active_video_end;        /* one past the last active sample */
  int32_t colour_burst_start;      /* burst window start (inclusive) */
  int32_t colour_burst_end;        /* burst window end (exclusive) */
  int32_t first_active_field_line; /* first active line */
  int32_t last_active_field_line;  /* one past the last active line; 0 => field_height */
  double sample_rate;              /* Hz */
  int32_t standard;                /* hvdg_standard */
  int32_t reserved0;
  double subcarrier_hz;            /* 0 => the standard's nominal fsc */
} hvdg_geometry;

/* Mirror of hvd::HvdConfig (hvd_config.h:21-419), hot-path fields only, same
 * defaults (hvdg_config_default). */
typedef struct hvdg_config {
  float lambda_c;            /* 1.0  */
  float chroma_aniso;        /* 0.0 = auto (variational.cpp:130-196) */
  float charbonnier_eps;     /* 0.5  */
  float chroma_eps;          /* 1.0  */
  float structure_coupling;  /* 0.25 */
  float diag_prior;          /* 0.0; > 0 adds the oriented +-45 deg chroma prior (the adjoint refuses it) */
  int32_t cg_iterations;     /* 2    */
  int32_t irls_outer;        /* 4    */
  float cg_tol;              /* 0 = auto (0.02 slow / 0.10 fast) */
  int32_t fast;              /* 1    */
  int32_t parallel_across_fields; /* 1 (CPU-baseline knob; the device path always batches) */
  int32_t symmetry_variant;  /* 0; 1 adds the spectral-symmetry third init variant
                                (holographic_init.cpp:265-306); refused by the adjoint */
  int32_t acc;               /* 1    */
  float chroma_gain;         /* 1.0  */
  int32_t monochrome;        /* 0    */
  float chroma_phase_deg;    /* 0.0  */
  int32_t field_order;       /* 0 = auto, 1 = field 1 top, 2 = field 1 bottom */
  float temporal_strength;   /* 0 = adaptive, < 0 = 3-D off, > 0 = fixed */
  int32_t bidirectional;     /* 1    */
  int32_t passes;            /* 2    */
  float temporal_eps;        /* 0 = auto clip(7 sigma, 4, 20) */
  float nr_anchor;           /* 1.0  */
  float nr_eps;              /* 0 = auto clip(3 sigma, 3, 12) */
  int32_t nr_radius;         /* 2    */
  int32_t mc_tile;           /* 32   */
  int32_t mc_search;         /* 16   */
  int32_t trajectory_fit;    /* 1    */
  int32_t extended_temporal; /* 1    */
  float coherence_gate;      /* 0.6  */
  float odd_gate_floor;      /* 0.35 */
  int32_t output_fidelity;   /* 1    */
  int32_t psi_init;          /* 0    */
  int32_t selective_3d;      /* 0; full-window 2-D + 3-D on the ambiguous boxes
                                (hvd_config.h:405-416, frame_bridge.cpp:402-718) */
  float selective_max_area;  /* 0.45 */
  /* ---- B200 build extensions (no HvdConfig counterpart) ---- */
  int32_t me_mode;           /* 0 = reference float-SSD pyramid (motion.cpp:397-488),
                                1 = exhaustive integer SAD on uint16-quantised luma */
  int32_t me_block;          /* block size for me_mode 1 (16) */
  int32_t me_range;          /* +/- search range for me_mode 1 (16) */
  int32_t reserved[3];
} hvdg_config;

/* Mirror of hvd::FrameParams (frame_bridge.h:40-101). */
#define HVDG_MAX_EXTRA_SAMPLE_LINES 8
typedef struct hvdg_frame_params {
  int32_t standard;
  int32_t frame_width;
  int32_t frame_height;
  int32_t field1_lines;
  int32_t active_video_start;
  int32_t active_video_end;
  int32_t colour_burst_start;
  int32_t colour_burst_end;
  int32_t first_active_frame_line;
  int32_t last_active_frame_line;
  float black_level;
  float white_level;
  float blanking_level;
  float chroma_dc;
  double sample_rate;
  double subcarrier_hz;
  int32_t extra_sample_lines[HVDG_MAX_EXTRA_SAMPLE_LINES];
  int32_t extra_sample_line_count;
  int32_t reserved0;
} hvdg_frame_params;

/* One composite field in (FieldInput + the parity FieldObs carries). */
typedef struct hvdg_field_in {
  const void* samples;        /* field_height x field_width, see sample_type */
  int32_t sample_type;        /* hvdg_sample_type */
  int32_t parity;             /* 0 = top field, 1 = bottom (FieldObs::parity) */
  float blanking_level;       /* used for U16 / S16 samples */
  float white_level;          /* used for U16 / S16 samples */
  const hvdg_geometry* geometry; /* per-field geometry (mixed NTSC/PAL batches) */
  int32_t irls_outer;         /* <= 0: cfg->irls_outer   (per-field solver budget) */
  int32_t cg_iterations;      /* <  0: cfg->cg_iterations */
} hvdg_field_in;

/* One decoded field out (DecodedField, sequence.h:64-69). Caller-owned;
 * planes need only a float's alignment. Page-locked host planes (and device
 * planes on the _device entry points) are written by the solver directly as
 * each field finishes; pageable ones are copied after the launch. */
typedef struct hvdg_field_out {
  float* luma;     /* active_lines x active_width, IRE */
  float* chroma;   /* active_lines x active_width x 2 (re, im), chi = V - iU, IRE */
  float* theta;    /* optional (may be NULL): field_height carrier phases after the trim */
  int8_t* vswitch; /* optional (may be NULL): field_height V-switch senses (+1 / -1) */
} hvdg_field_out;

/* One decoded frame (YcFrameS16, frame_bridge.h:123-131). Caller-owned,
 * frame_width * frame_height elements each. */
typedef struct hvdg_yc_frame {
  int16_t* luma;
  int16_t* chroma;
  double* u_plane;
  double* v_plane;
} hvdg_yc_frame;

/* Per-call timing / diagnostics (SequenceDiagnostics, sequence.h:75-81, plus
 * device timings). Optional everywhere. */
typedef struct hvdg_diag {
  float resolved_strength;
  float ambiguity_ire;
  float sigma_ire;
  float temporal_eps;
  float nr_eps;
  float acc_gain;
  float ms_total;       /* device time of the whole call (CUDA events) */
  float ms_solver;      /* device time of the IRLS + CG persistent kernel(s) */
  float ms_init;        /* device time of lock-in + holographic init */
  float ms_motion;      /* device time of motion estimation + warps */
  int64_t cg_iterations_run;   /* sum over fields of CG iterations executed */
  int64_t solver_pixel_iters;  /* sum over fields of active px * CG iterations */
  int64_t solver_pixel_outers; /* sum over fields of active px * IRLS outers */
  int32_t kernel_launches;     /* kernels this call launched */
  int32_t reserved;
} hvdg_diag;

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */

int hvdg_abi_version(void);
const char* hvdg_status_string(hvdg_status s);
void hvdg_config_default(hvdg_config* cfg);
/* NTSC 4fsc / PAL 4fsc default geometries (ntsc_geometry.h:66-74;
 * research/reference-pal/hvd_pal/tbc.py:34-50). */
void hvdg_geometry_default(int standard, hvdg_geometry* g);

typedef struct hvdg_ctx hvdg_ctx;
/* Owns the device arena, the stream, the CUDA-graph cache and the tuning
 * table (HvdEngine, engine.h:70-128, owns the FFT plan cache). */
hvdg_status hvdg_create(int device, hvdg_ctx** out);
void hvdg_destroy(hvdg_ctx* ctx);
/* Last error text for this context (static storage, valid until next call). */
const char* hvdg_last_error(const hvdg_ctx* ctx);
/* 0 = plain path (one field per launch sequence), 1 = batched persistent
 * launch (default). Exists for the batched-vs-plain comparison. */
hvdg_status hvdg_set_batching(hvdg_ctx* ctx, int batched);
/* Solver tiling: band height (rows per work unit; 0 = autotuned). */
hvdg_status hvdg_set_tuning(hvdg_ctx* ctx, int band_rows, int ctas_per_sm);
/* Bound of the solver's device-side waits on a field's phase flag, in polls
 * (~0.5 us each; <= 0 restores the default 4,000,000, ~2 s). A wait that
 * runs out ends the launch and the call returns HVDG_ERR_DEVICE_TIMEOUT; the
 * context stays usable. No reference counterpart (the reference's CPU loops
 * have no waits to bound). */
hvdg_status hvdg_set_device_wait_limit(hvdg_ctx* ctx, int64_t polls);

/* ------------------------------------------------------------------------ */
/* Engine level                                                              */
/* ------------------------------------------------------------------------ */

/* PrepareFieldObs x n + DecodeFieldWindow (sequence.cpp:229-281, 423-1116):
 * burst lock-in, active crop, carrier, holographic init, (3-D neighbour
 * terms when cfg->temporal_strength > 0), IRLS + CG, output-fidelity luma.
 * All fields must share fields[0].geometry (the reference's window contract). */
hvdg_status hvdg_decode_field_window(hvdg_ctx* ctx, const hvdg_field_in* fields,
                                     int n_fields, const hvdg_config* cfg,
                                     hvdg_field_out* out, hvdg_diag* diag);

/* Independent 2-D fields of mixed geometry and per-field solver budgets in
 * one batched persistent launch (the reference decodes these one by one:
 * sequence.cpp:1076-1084 with temporal off). Host buffers in and out. */
hvdg_status hvdg_decode_fields(hvdg_ctx* ctx, const hvdg_field_in* fields,
                               int n_fields, const hvdg_config* cfg,
                               hvdg_field_out* out, hvdg_diag* diag);

/* Same as hvdg_decode_fields with every samples / luma / chroma / theta /
 * vswitch pointer a DEVICE pointer on the context's device; no host copies.
 * Returns after the work is enqueued on `stream` (0 = the context stream)
 * and completed (synchronous). */
hvdg_status hvdg_decode_fields_device(hvdg_ctx* ctx, const hvdg_field_in* fields,
                                      int n_fields, const hvdg_config* cfg,
                                      hvdg_field_out* out, hvdg_diag* diag);

/* Asynchronous form of hvdg_decode_fields_device: enqueues the decode (the
 * replay of the cached CUDA graph) and returns. `stream` (a cudaStream_t,
 * may be NULL) orders it: the decode starts after the work the caller's
 * stream enqueued before the call, and the caller's stream waits for the
 * decode's completion. The first call of a batch shape (tuning + capture)
 * completes before returning. hvdg_wait returns the call's status (device
 * timeouts, non-finite input) and diagnostics; any other call on the context
 * completes a call still in flight first, and hvdg_wait then reports it. */
hvdg_status hvdg_decode_fields_device_async(hvdg_ctx* ctx, const hvdg_field_in* fields,
                                            int n_fields, const hvdg_config* cfg,
                                            hvdg_field_out* out, void* stream);
/* Wait for the last asynchronous decode; its status and diag (optional).
 * HVDG_OK with zeroed diag when none is outstanding. */
hvdg_status hvdg_wait(hvdg_ctx* ctx, hvdg_diag* diag);

/* hvd::DecodeFrameSequenceWindow (frame_bridge.cpp:722-947): split each
 * int16 frame into fields, ACC, field-order vote, window decode, weave and
 * 10-bit requantise. `out` has core_end - core_begin entries. Returns
 * HVDG_ERR_BAD_ARGUMENT where the reference returns an empty vector. */
hvdg_status hvdg_decode_frame_sequence_window(
    hvdg_ctx* ctx, const int16_t* const* frames, int n_frames, int core_begin,
    int core_end, const hvdg_frame_params* fp, const hvdg_config* cfg,
    hvdg_yc_frame* out, hvdg_diag* diag);
/* The same with the reference's base_frame_id (frame_bridge.h:196-199),
 * which only numbers the diagnostic maps. */
hvdg_status hvdg_decode_frame_sequence_window_at(
    hvdg_ctx* ctx, const int16_t* const* frames, int n_frames, int core_begin,
    int core_end, int64_t base_frame_id, const hvdg_frame_params* fp,
    const hvdg_config* cfg, hvdg_yc_frame* out, hvdg_diag* diag);
/* HvdConfig::debug_dir (hvd_config.h:314): when non-empty (NULL or "" = off),
 * the sequence frame bridge appends its decision log to <dir>/diag.txt and
 * writes one rainbow_<frame id>.pgm map per core frame
 * (frame_bridge.cpp:807-865). Host-side file output; the decode is unchanged. */
hvdg_status hvdg_set_debug_dir(hvdg_ctx* ctx, const char* dir);

/* hvd::DecodeFrameBuffer (frame_bridge.h:149-150, frame_bridge.cpp:161-255) via HvdEngine::DecodeFrame
 * (engine.cpp:141-195): the 2-D frame-weave decode of one field-sequential
 * int16 composite frame -- split, field-order vote (cfg->field_order),
 * per-field lock-in, weave of the two fields' active pictures and carriers,
 * holographic init + IRLS / CG on the woven frame, lossless chroma S - Y,
 * ACC, re-weave and 10-bit requantisation into `out` (frame_width x
 * frame_height each). The source frame holds FrameLineOffset(fp,
 * frame_height - 1) + frame_width samples at least. */
hvdg_status hvdg_decode_frame_buffer(hvdg_ctx* ctx, const int16_t* frame,
                                     const hvdg_frame_params* fp, const hvdg_config* cfg,
                                     hvdg_yc_frame* out);
/* n independent frames of hvdg_decode_frame_buffer in one batched launch
 * sequence (no reference counterpart: the reference decodes frame by frame).
 * diag (optional) reports the first frame's ACC gain; its ms_total is the
 * device time of the kernels (frame split to re-weave), the host <-> device
 * copies of the frames excluded. Pinned host frames and planes copy at the
 * link's full rate. */
hvdg_status hvdg_decode_frame_buffers(hvdg_ctx* ctx, const int16_t* const* frames, int n_frames,
                                      const hvdg_frame_params* fp, const hvdg_config* cfg,
                                      hvdg_yc_frame* out, hvdg_diag* diag);
/* hvd::DecodeYcFrameBuffer (frame_bridge.h:223-226, frame_bridge.cpp:263-377) via
 * HvdEngine::DecodeChromaOnly (engine.cpp:197-237): Y/C-native input. The C
 * channel is de-woven around fp->chroma_dc, woven with its per-field
 * lock-in carriers and cropped by the holographic init alone (no IRLS / CG);
 * luma passes through from the Y channel. chroma = Re[chi c] requantised,
 * u / v from chi with ACC. Field order: cfg->field_order 2 puts field 1 on
 * the odd rows, anything else on the even rows (no vote on this path). */
hvdg_status hvdg_decode_yc_frame_buffer(hvdg_ctx* ctx, const int16_t* luma, const int16_t* chroma,
                                        const hvdg_frame_params* fp, const hvdg_config* cfg,
                                        hvdg_yc_frame* out);
/* n independent frames of hvdg_decode_yc_frame_buffer in one batch. */
hvdg_status hvdg_decode_yc_frame_buffers(hvdg_ctx* ctx, const int16_t* const* luma,
                                         const int16_t* const* chroma, int n_frames,
                                         const hvdg_frame_params* fp, const hvdg_config* cfg,
                                         hvdg_yc_frame* out, hvdg_diag* diag);

/* ------------------------------------------------------------------------ */
/* Kernel level (host buffers)                                               */
/* ------------------------------------------------------------------------ */

/* DrizzleFrame (sequence.h:123-130, sequence.cpp:283-421): the decoded
 * fields luma[i] (h x w, IRE) / chroma[i] (h x w x 2) with their parities,
 * motion-compensated and deposited onto the fine grid of the frame of fields
 * j0, j0 + 1 ((2 h scale) x w), blended by coverage with the plain weave.
 * Motion: the reference's float EstimateMotion (cfg->mc_tile,
 * cfg->mc_search); robust scale cfg->nr_eps (0: 3 IRE); sources within
 * 2 cfg->nr_radius fields. The deposits are float atomics: sums agree with
 * the reference to rounding, not bit for bit. */
hvdg_status hvdg_drizzle_frame(hvdg_ctx* ctx, const float* const* luma, const float* const* chroma,
                               const int32_t* parities, int n, int j0, int h, int w,
                               const hvdg_config* cfg, int scale, float* out_luma,
                               float* out_chroma);

/* DetectFieldParity (frame_bridge.h:170-171, frame_bridge.cpp:102-149) of
 * n field-sequential int16 frames, each split as SplitFrameFields splits it
 * (frame_bridge.cpp:61-99): votes[t] = +1 (field 1 is the top field), -1
 * (field 1 is the bottom field), 0 (no confident vote). The vote the
 * automatic field order (cfg->field_order 0) of hvdg_decode_frame_buffer(s)
 * takes, equal to the reference's for every input. */
hvdg_status hvdg_detect_field_parity(hvdg_ctx* ctx, const int16_t* const* frames, int n_frames,
                                     const hvdg_frame_params* fp, int32_t* votes);

/* AmbiguousBoxes (frame_bridge.cpp:402-580, the selective 3-D detector) on
 * one decoded field (luma h x w, chroma h x w x 2), host only. Writes up to
 * max_boxes boxes as (fy0, fy1, x0, x1) in active-picture coordinates and
 * sets *n_boxes to their count: 0 = stay 2-D, -1 = run the full 3-D window
 * (ambiguity everywhere). */
hvdg_status hvdg_ambiguous_boxes(const float* luma, const float* chroma, int h, int w,
                                 float max_area, int32_t* boxes, int max_boxes, int* n_boxes);


/* BurstLockinPhase (lockin.cpp:169-254) on NTSC, BurstLockinPhasePal
 * (lockin.cpp:325-417) on the PAL family. `field_ire` is field_height x
 * field_width IRE; theta/vswitch have field_height entries (vswitch is
 * filled with +1 on NTSC and may be NULL there). */
hvdg_status hvdg_burst_lockin(hvdg_ctx* ctx, const float* field_ire,
                              const hvdg_geometry* g, float* theta,
                              int8_t* vswitch);

/* BurstAmplitudeIre (lockin.cpp:256-323). */
hvdg_status hvdg_burst_amplitude(hvdg_ctx* ctx, const float* field_ire,
                                 const hvdg_geometry* g, float* amplitude_ire);

/* HolographicInit (holographic_init.cpp:427-544) on the active picture
 * `s` (active_lines x active_width); carrier from theta/vswitch (active
 * lines only). Outputs luma0 (h x w) and chi0 (h x w x 2). */
hvdg_status hvdg_holographic_init(hvdg_ctx* ctx, const float* s,
                                  const float* theta_active,
                                  const int8_t* vswitch_active,
                                  const hvdg_geometry* g, const hvdg_config* cfg,
                                  float* luma0, float* chi0);

/* VariationalRefine (variational.cpp:198-556), 2-D (no neighbours). */
hvdg_status hvdg_variational_refine(hvdg_ctx* ctx, const float* s,
                                    const float* theta_active,
                                    const int8_t* vswitch_active,
                                    const float* chi0, const hvdg_geometry* g,
                                    const hvdg_config* cfg, float* luma,
                                    float* chi);

/* EstimateMotion (motion.cpp:397-488): per-tile (dy, dx, confidence) from
 * y_ref to y_cur (both h x w); outputs are ceil(h/tile) x ceil(w/tile).
 * me_mode selects the cost (see hvdg_config::me_mode); for me_mode 1 the
 * block size and range come from `tile` and `search`. */
hvdg_status hvdg_estimate_motion(hvdg_ctx* ctx, const float* y_ref,
                                 const float* y_cur, int h, int w, int tile,
                                 int search, int me_mode, float* dy, float* dx,
                                 float* confidence);

/* VerifyMotion (motion.cpp:490-530, declared motion.h:74-75): the predicted
 * per-tile vectors pdy / pdx (ceil(h/tile) x ceil(w/tile), e.g. from a
 * trajectory fit) audited on the r = 2 box-blurred planes -- one SSD at the
 * rounded prediction, one at zero, the full prediction kept where it is
 * strictly better -- and MotionConfidence of the result; outputs per tile
 * like hvdg_estimate_motion. The fast 3-D window runs the same kernel on its
 * trajectory predictions. */
hvdg_status hvdg_verify_motion(hvdg_ctx* ctx, const float* y_ref, const float* y_cur, int h,
                               int w, int tile, const float* pdy, const float* pdx, float* dy,
                               float* dx, float* confidence);

/* ------------------------------------------------------------------------ */
/* Adjoint                                                                   */
/* ------------------------------------------------------------------------ */

/* No counterpart in the reference (it has no adjoint): gradients of a scalar
 * loss on the decoded planes, for research and training.
 * For each field of a 2-D decode (lock-in, HolographicInit, IRLS + CG
 * VariationalRefine, output luma; cfg->temporal_strength < 0), given the
 * loss cotangents y_bar[i] (active_lines x active_width floats) and
 * chi_bar[i] (active_lines x active_width x 2 floats) of the decoded Y and
 * chi, writes samples_bar[i] (field_height x field_width floats): d loss /
 * d sample value -- per code for integer samples, per IRE for float samples
 * -- and sets scalar_bar[0..3] to the gradients with respect to
 * cfg->lambda_c, charbonnier_eps, chroma_eps and structure_coupling, summed
 * over the fields.
 * The forward is recomputed with every IRLS iterate checkpointed. Each
 * outer's quadratic is differentiated as solved exactly (implicit function:
 * one adjoint CG solve of adjoint_cg_iterations, <= 0 = 300, on the same SPD
 * operator per outer), so the result is exact when the forward's CG budget
 * converges every outer. Held at their forward values (no gradient through
 * them): the lock-in carrier phase and the chroma-anisotropy split; samples
 * outside the active window therefore get zero gradient.
 * out (optional, may be NULL): the recomputed forward's luma / chroma. */
hvdg_status hvdg_decode_fields_adjoint(hvdg_ctx* ctx, const hvdg_field_in* fields, int n,
                                       const hvdg_config* cfg, const float* const* y_bar,
                                       const float* const* chi_bar, float* const* samples_bar,
                                       double* scalar_bar, int adjoint_cg_iterations,
                                       hvdg_field_out* out, hvdg_diag* diag);

/* ------------------------------------------------------------------------ */
/* Allocation-free entry point                                               */
/* ------------------------------------------------------------------------ */

/* No counterpart in the reference: this is an addition of this library.
 * HolographicInit (the same kernels and results as hvdg_holographic_init with
 * cfg->symmetry_variant = 0; the spectral-symmetry third variant is not run)
 * for callers that cannot allocate device memory -- e.g. a plugin inside a host
 * application that owns the CUDA allocator, or a real-time path that must
 * not risk a cudaMalloc stall. It takes no context and calls no cudaMalloc,
 * cudaFree or allocating library routine: its scratch is one file-scope
 * device array of HVDG_NOALLOC_SCRATCH_BYTES, which every GPU that loads this
 * library holds until the process exits. Inputs and outputs are host
 * buffers, as for hvdg_holographic_init; work runs on the legacy default
 * stream of the current device and the call returns when it is done.
 * Limits: geometry is checked as for hvdg_holographic_init (same statuses);
 * fields past the register transforms' lengths (more than 1024 active
 * samples, or more than 480 active lines), which hvdg_holographic_init takes
 * through its shared-memory transforms, are rejected here with
 * HVDG_ERR_UNSUPPORTED, and every field within them fits the array. The first call on each device
 * looks up the array's device address and keeps it for the life of the
 * process: make that first call before any stream capture, and do not
 * cudaDeviceReset that device between calls. All calls share the one array
 * and it keeps the last call's contents, so calls that overlap on the GPU
 * (from several host threads) race: serialise them. */
#define HVDG_NOALLOC_SCRATCH_BYTES (32u << 20)
hvdg_status hvdg_holographic_init_noalloc(const float* s, const float* theta_active,
                                          const int8_t* vswitch_active,
                                          const hvdg_geometry* g, float* luma0,
                                          float* chi0);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* HVDG_H_ */
