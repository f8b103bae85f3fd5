// gather_map_pf32.cu -- instantiates the gather kernels for map element
// type PackF32 (compiled in parallel with the other map types).
#include "gather_impl.cuh"

namespace todgpu {
TODGPU_DEFINE_MAP_DISPATCH(pf32, PackF32)
}  // namespace todgpu
