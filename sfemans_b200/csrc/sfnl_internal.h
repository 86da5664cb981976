// sfnl_internal.h -- shared host-side helpers of the library (not installed).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/sfemans_nl.h"

namespace sfnl {

struct ProgArgs;

// Records the message for sfnl_last_error() on this thread and returns code.
int set_error(int code, const char *msg);
// Checks cudaGetLastError() after a launch; records "<what>: <cuda error>".
int check_launch(const char *what);
// Number of SMs of the current device (cached per device).
int num_sms();

// Kernel families.
int launch_grid(const ProgArgs &a, cudaStream_t st);   // sfnl_grid.cu
int launch_fast(const ProgArgs &a, cudaStream_t st);   // sfnl_fast.cu
bool fast_supported(int op, int m, int N_int);          // sfnl_fast.cu
int fast_grid_length(int m);                            // sfnl_fast.cu
void fast_release_tables();                             // sfnl_fast.cu
int launch_split(const ProgArgs &a, int split, cudaStream_t st);  // sfnl_split.cu
bool split_supported(int op, int m);                    // sfnl_split.cu

}  // namespace sfnl
