// gather_map_pf64.cu -- instantiates the gather kernels for map element
// type PackF64 (compiled in parallel with the other map types).
#include "gather_impl.cuh"

namespace todgpu {
TODGPU_DEFINE_MAP_DISPATCH(pf64, PackF64)
}  // namespace todgpu
