// gather_map_f64.cu -- instantiates the gather kernels for map element
// type double (compiled in parallel with the other map types).
#include "gather_impl.cuh"

namespace todgpu {
TODGPU_DEFINE_MAP_DISPATCH(f64, double)
}  // namespace todgpu
