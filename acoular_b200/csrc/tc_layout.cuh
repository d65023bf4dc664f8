// Shared-memory operand tiles of the tensor-core kernels: 32 x 32 elements (row = M or N index,
// col = K index), K-major, no swizzle, stored in HBM in exactly the order the tcgen05 shared-memory
// descriptor reads so that a tile (or a run of tiles) is one bulk copy.
//   BF16: core matrices of 8 rows x 8 elements (16 bytes), 4 per 8-row group: LBO 128 B, SBO 512 B.
//   TF32: core matrices of 8 rows x 4 elements (16 bytes), 8 per 8-row group: LBO 128 B, SBO 1 KB.
// Consecutive tiles along the row index continue the 8-row groups, so n tiles in a row form an
// operand of 32 n rows with the same LBO/SBO.
#pragma once

#include <stdint.h>

namespace acb {

// Element offset inside a 32x32 BF16 tile.
__device__ __forceinline__ int tile_off(int row, int col)
{
    return (((row >> 3) * 4 + (col >> 3)) << 6) + ((row & 7) << 3) + (col & 7);
}

// Element offset inside a 32x32 TF32 (FP32 storage) tile.
__device__ __forceinline__ int tile_off_tf32(int row, int col)
{
    return (((row >> 3) * 8 + (col >> 2)) << 5) + ((row & 7) << 2) + (col & 3);
}

// Round an FP32 value to TF32 (nearest, ties away from zero), as the MMA reads only 19 bits.
__device__ __forceinline__ uint32_t tf32_bits(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

}  // namespace acb
