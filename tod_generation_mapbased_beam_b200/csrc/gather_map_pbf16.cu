// gather_map_pbf16.cu -- instantiates the gather kernels for map element
// type PackBF16 (compiled in parallel with the other map types).
#include "gather_impl.cuh"

namespace todgpu {
TODGPU_DEFINE_MAP_DISPATCH(pbf16, PackBF16)
}  // namespace todgpu
