// Host side of the tensor-map (TMA) loads of the region kernels: a 2-D view
// of a row-strided byte matrix (rows = input slices) from which one
// `cp.async.bulk.tensor.2d` brings a box of several rows' byte ranges into
// shared memory.  Encoded with the driver's cuTensorMapEncodeTiled, reached
// through the runtime's driver entry point (no link against libcuda).
//
// Rules the callers meet (cuTensorMapEncodeTiled checks the first three):
// the base address 16-byte aligned, the row stride a multiple of 16 bytes,
// the box width a multiple of 16 bytes and at most 256 elements; and, checked
// by nobody before the copy runs, every box's x coordinate a multiple of 16
// bytes.  Elements outside the matrix (past the last row or column) arrive as
// zeros and still count toward the box's transaction bytes.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstddef>
#include <cstdint>

namespace pp {

inline PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// rows x row_bytes bytes at base, row r at base + r * stride; boxes of
// box_rows rows x box_bytes bytes, no swizzle (row-major in shared memory).
inline cudaError_t tma_encode_rows(CUtensorMap* map, const void* base, size_t row_bytes, uint32_t rows,
                                   size_t stride, uint32_t box_bytes, uint32_t box_rows) {
  auto enc = tma_encoder();
  if (!enc) return cudaErrorNotSupported;
  if (((uintptr_t)base % 16) || (stride % 16) || (box_bytes % 16) || box_bytes > 256 || box_rows > 256 ||
      !row_bytes || !rows)
    return cudaErrorInvalidValue;
  if (rows == 1 && stride < row_bytes) stride = (row_bytes + 15) & ~(size_t)15;  // one row: any valid stride
  const cuuint64_t dim[2] = {(cuuint64_t)row_bytes, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)stride};
  const cuuint32_t box[2] = {box_bytes, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dim, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace pp
