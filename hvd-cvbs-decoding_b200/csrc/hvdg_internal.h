// hvdg_internal.h -- host/device shared layouts of the batched field solver.
//
// Device memory holds a BATCH of fields. Every per-pixel plane of a field is
// stored row-major with a row pitch that is a multiple of 64 elements (one
// solver strip), at offset `px_off` (in pixels) inside one batch-wide array
// per plane kind. Per-line and per-column carrier phasors replace the
// reference's stored carrier plane (FieldObs::carrier, sequence.h:52-56):
//   c(y, x) = L[y] * P[x],  L[y] = exp(i theta[y]),  P[x] = exp(i w0 (a0 + x))
// and c -> -conj(c) on V-switched lines (MakeCarrierPal,
// ntsc_geometry.cpp:438-456).
#pragma once

#include <cstddef>
#include <cstdint>

namespace hvdg {

constexpr int kStrip = 64;        // solver strip width (columns per warp unit)
constexpr int kMaxLines = 1024;   // max field lines handled by the lock-in kernel
constexpr int kRowFft = 2048;     // init: row cyclic-convolution length (register FFT)
constexpr int kColFft = 1024;     // init: column cyclic-convolution length (field planes)
constexpr int kColFftWide = 2048; // init: column length of taller planes (woven frames)
constexpr int kFftLong = 4096;    // init: rows / columns past the register lengths (shared-memory FFT)
constexpr long long kSpinLimit = 4000000;  // bounded device waits: polls x ~0.5 us ~= 2 s
constexpr int kInitPad = 16;      // init: reflect-101 row pad (holographic_init.cpp:214-222)

// Per-field descriptor (device copy is read-only during a launch except the
// fields marked "written by").
struct FieldDesc {
  int h, w;            // active lines / active width
  int pitch;           // row pitch (elements), multiple of kStrip
  int fh, fw;          // full field height / width
  int64_t px_off;      // plane offset of this field (pixels)
  int line_off;        // offset into per-line tables (active lines)
  int col_off;         // offset into the column-phasor table (per geometry)
  int geom;            // geometry slot (init kernels, column phasors)
  int is_pal;          // V-switch family (aniso 4-line groups)
  int n_outer;         // IRLS outer passes (>= 1)
  int n_inner;         // CG iterations per outer (>= 1)
  float cg_tol;        // relative gradient-norm exit
  float eps, eps_c, k_coupling;  // Charbonnier scales, structure coupling
  float lambda_c, aniso_cfg;     // lambda_c, fixed aniso (> 0) or 0 = auto
  float diag_prior;    // oriented +-45 deg chroma prior weight (0 = off)
  float mu_h, mu_v;    // written by the aniso kernel
  float mu_d;          // oriented prior weight, written by the aniso kernel (0 = off)
  float aniso_p98[2];  // the aniso kernel's horizontal / vertical p98 (scratch)
  int aniso_arrive;    // the aniso kernel's per-field arrivals (two per run)
  float nu;            // temporal strength (0 = 2-D)
  float eps_t;         // temporal robust scale
  int has_nbr;         // 3-D neighbour terms present (M / b planes valid)
  int n_nbr;           // neighbour planes
  int64_t nbr_off;     // offset (float4) of this field's neighbour planes
  int64_t plane_px;    // h * pitch (one plane of this field)
  int unit_begin;      // first solver unit of this field
  int unit_count;      // number of solver units
  int n_phases;        // n_outer * (2 + n_inner) + 1
  int adj_flags;       // adjoint solves: kAdjFixedW | kAdjExtB (0 for decodes)
  // optional dense (row stride w) destinations the solver's final phase
  // writes the field's luma / chroma to, besides the planes: the caller's
  // device buffers, or its page-locked host buffers (mapped), so the copy
  // out overlaps the other fields' solves
  float* out_y;
  float2* out_c;
};

// FieldDesc::adj_flags. kAdjFixedW: the R phase keeps the weights already in
// W (the forward's lagged weights) instead of recomputing them from chi;
// kAdjExtB: the G phase adds the constant plane B (the adjoint right-hand
// side) to the gradient.
constexpr int kAdjFixedW = 1;
constexpr int kAdjExtB = 2;

// Per-geometry init tables.
struct GeomDesc {
  int w, h, hp;        // active width, active lines, padded lines (h + 2 pad)
  int pad;             // row pad
  int khat_row_off;    // offset (float2) of the 2 row kernels' spectra (2 * row_m)
  int khat_col_off;    // offset (float2) of the 2 column kernels' spectra (2 * col_m)
  int row_m;           // row convolution length: kRowFft or kFftLong
  int col_m;           // column convolution length: kColFft, kColFftWide or kFftLong
  // symmetry-variant tables (offsets into the same float2 table; -1 when
  // the batch runs without the variant): Bluestein chirps exp(-i pi n^2 / N)
  // and chirp-filter spectra (1/M folded in) of the exact-length row (w)
  // and column (hp) DFTs, and the {1.3 MHz, 60 c/ph} crop (gx, gy in .x)
  int sym_row_chirp, sym_row_hhat, sym_col_chirp, sym_col_hhat, sym_gx, sym_gy;
};

// Solver control block, one per field (written by the last arriver of each
// phase, read by every unit of the next phase).
struct FieldCtl {
  double gg;           // ||g_k||^2 (exact, of the stored residual)
  double gg0;          // ||g_0||^2 of the current outer pass
  double gg_next;      // ||g_{k+1}||^2 predicted by the recurrence
  float alpha;         // pending step to apply (chi += alpha d, g += alpha q)
  float beta;          // direction update factor for the next iteration
  int pending;         // 1 => alpha/beta pending from the previous I phase
  int cg_iters;        // CG iterations executed (stats)
  int sel;             // which of the double-buffered g / d / q planes is current
  int xsel;            // which of the double-buffered chi planes is current
};

// One solver work unit: a kStrip-wide strip x `band` rows of one field.
struct Unit {
  int field;
  int x0;
  int y0;
  int y1;
};

}  // namespace hvdg
