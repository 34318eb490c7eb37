// Tight world-space instance boxes for the 8-wide instance hierarchy (see
// instance_boxes.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../trace/scene_types.hpp"

namespace mb {

// out[6 * i ..] = the box of instance i from its object hierarchy's top two
// 8-wide levels transformed by instToWorld (12 floats per instance),
// intersected with looseBoxes[6 * i ..] (the transformed object box); masked
// instances and objects without an 8-wide hierarchy keep the loose box.
cudaError_t tight_instance_boxes(const DLod* lods, const uint32_t* instLod, const float* instToWorld, uint32_t n,
                                 const float* looseBoxes, float* out, cudaStream_t stream);

} // namespace mb
