// Launch variant 9: z-vectorised step kernel, 4 cells per lane, a 3-plane cp.async ring.
#include "vec_kernel.cuh"

namespace fdtdb200 {

FDTD_VEC_LAUNCHER(launch_vec_r4d3, 4, 3, 1)

}  // namespace fdtdb200
