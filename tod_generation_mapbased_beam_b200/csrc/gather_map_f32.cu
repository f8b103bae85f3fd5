// gather_map_f32.cu -- instantiates the gather kernels for map element
// type float (compiled in parallel with the other map types).
#include "gather_impl.cuh"

namespace todgpu {
TODGPU_DEFINE_MAP_DISPATCH(f32, float)
}  // namespace todgpu
