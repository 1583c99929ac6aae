// Tensor-core (TF32 mma.sync) variant of the affine FP32 cell operator (vmult_tc.cu).
#pragma once

#include "pmg_internal.hpp"

namespace pmg {
// dst += A_cells src with the operator's tensor-core mode (1: TF32, 3: three TF32 products);
// FP32 operators with affine geometry
void vmult_cells_tensor_cores(const pmg_operator &op, const void *src, void *dst, cudaStream_t s);
} // namespace pmg
