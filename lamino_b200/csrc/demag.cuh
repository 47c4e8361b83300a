// Demagnetizing field operator (include/demag.h:13-79) on the GPU.
#pragma once

#include "common.cuh"

namespace lamino {

// h3 = demagnetizing field of m3; both [3][n1][n2][n3] float32 on the device.
void demag(const float *m3, Dims3 d, float *h3, cudaStream_t s);

}  // namespace lamino
