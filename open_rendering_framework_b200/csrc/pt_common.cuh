// Shared host-side plumbing for the C ABI: status/error text, launch accounting, grid sizing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/orf_b200.h"

namespace pt {

// Sets the thread's error text and returns `s`.
pt_status fail(pt_status s, const std::string& msg);
// Maps a CUDA error to PT_CUDA_ERROR / PT_OOM with its text (PT_OK for cudaSuccess).
pt_status cuda_status(cudaError_t e, const char* what);
// Counts one kernel launch (pt_kernel_launch_count).
void count_launch(uint64_t n = 1);
// Number of SMs on the current device (cached per device).
int sm_count();
// Grid for a grid-stride kernel: a multiple of the SM count, no larger than the work needs.
int grid_for(uint64_t items, int block, int blocks_per_sm);

}  // namespace pt

#define PT_CHECK_CUDA(call, what)                              \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return ::pt::cuda_status(e_, what); \
  } while (0)
