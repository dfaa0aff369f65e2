// Tensor maps for TMA (cp.async.bulk.tensor) copies of this GPU's own buffers.
//
// A map describes a row-major 2-D array of u32 (rows of `cols` words, `pitch`
// words apart) and the box one copy moves.  The driver's encoder is reached
// through the runtime's entry-point query, so the library links no libcuda.
// Encoding is host-only work (no device call, no allocation); a map is passed
// to kernels by value as a __grid_constant__ parameter.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace fpm {

enum class TmaSwizzle { kNone, k128B };

// rows x cols u32 words at `base` (16-byte aligned, pitch a multiple of 4
// words), box = box_rows x box_cols words.  Out-of-range parts of a box read
// as zero and are not written.  Throws CudaError-like std::runtime_error on a
// rejected map.
CUtensorMap make_tmap_u32(const void* base, uint64_t rows, uint64_t cols, uint64_t pitch, uint32_t box_rows,
                          uint32_t box_cols, TmaSwizzle swizzle);

}  // namespace fpm
