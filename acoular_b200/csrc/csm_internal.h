// Internal interfaces between the CSM sources (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace acb {

// Windowed rFFT of `num_windows` windows (FP64; FP32 for the operand tiles up to 8192 samples);
// out_form: 0 complex128 spectra, 1 complex64 spectra, 2 TF32 operand tiles, 3 split-BF16 operand tiles (R row tiles, KC window blocks, lo tiles
// `lo_elems` after the hi tiles).  Blocks above 16384 samples need `scratch` of
// fft_scratch_bytes(num_mics, block_size, num_windows) bytes (null otherwise).
int fft_launch(const void *samples, int sample_dtype, int out_form, int num_mics, int block_size, int hop,
               int64_t first_window, int64_t num_windows, const double *window, const double2 *tw, int bin_lo,
               int num_bins, void *out, int R, int KC, int64_t lo_elems, void *scratch, cudaStream_t s);
size_t fft_scratch_bytes(int num_mics, int block_size, int64_t num_windows);
// True when fft_launch writes every element of the operand tiles (padding windows and mics as zeros),
// which it does for the tile forms up to blocks of 8192 samples (the FP32 four-window transform).
bool fft_tiles_written_whole(int block_size);

// Tensor-core Welch accumulation into the complex128 upper triangle (csm_tc.cu).
int csm_tc_row_tiles(int num_mics);
size_t csm_tc_workspace_bytes(int num_mics, int num_bins, int64_t num_windows);
int csm_tc_accumulate(const void *samples, int sample_dtype, int num_mics, int block_size, int hop,
                      int64_t first_window, int64_t num_windows, const double *window, const double2 *tw,
                      int bin_lo, int num_bins, bool tf32, void *csm_upper, void *workspace, void *fft_scratch,
                      cudaStream_t s);

}  // namespace acb
