// hvdg_host.h -- host-side helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "hvdg.h"

struct hvdg_ctx;

namespace hvdg {

// Grow-only device arena (one allocation per context; zeroed when grown,
// in order on the context stream `st`).
struct DeviceArena {
  void* base = nullptr;
  size_t capacity = 0;
  hvdg_status reserve(size_t bytes, cudaStream_t st);
  ~DeviceArena();
};

// Grow-only pinned host staging buffer.
struct PinnedArena {
  void* base = nullptr;
  size_t capacity = 0;
  hvdg_status reserve(size_t bytes);
  ~PinnedArena();
};

// Host-side init tables of one geometry (kernel spectra, column phasors,
// FFT twiddles), as uploaded by the batched pipeline.
void init_tables_for(const hvdg_geometry& g, std::vector<float2>* khat_row_col,
                     std::vector<float2>* col_phasor, std::vector<float2>* tw_row,
                     std::vector<float2>* tw_col, int* hp, int* pad);

// The geometry checks every field entry point applies (arguments, ranges,
// device-path limits), as a status.
hvdg_status check_field_geometry(const hvdg_geometry* g);

// Records a CUDA failure in the context and maps it to a status.
hvdg_status cuda_fail(hvdg_ctx* ctx, cudaError_t e, const char* what);

}  // namespace hvdg
