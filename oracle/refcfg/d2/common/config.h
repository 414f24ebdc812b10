// Compile-time index constants for building the reference with 2 dimensions.
// Same names and values as the reference's src/common/config.h:4-18 except the
// dimension count, which the reference fixes at compile time.
#pragma once

namespace ursus {
  __host__ __device__ constexpr unsigned int GetNumberOfDims() { return 2; }
  __host__ __device__ constexpr unsigned int GetNumberOfUpperTreeDegrees() { return 128; }
  __host__ __device__ constexpr unsigned int GetNumberOfLeafNodeDegrees() { return 192; }
  __host__ __device__ constexpr unsigned int GetNumberOfThreads() { return 192; }
  __host__ __device__ constexpr unsigned int GetNumberOfThreads2() { return 256; }
  __host__ __device__ constexpr unsigned int GetNumberOfMAXCPUThreads() { return 32; }
  __host__ __device__ constexpr unsigned int GetNumberOfMAXBlocks() { return 208; }
} // namespace ursus
