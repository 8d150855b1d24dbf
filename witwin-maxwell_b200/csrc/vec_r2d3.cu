// Launch variant 8: z-vectorised step kernel, 2 cells per lane, a 3-plane cp.async ring.
#include "vec_kernel.cuh"

namespace fdtdb200 {

FDTD_VEC_LAUNCHER(launch_vec_r2d3, 2, 3, 2)

}  // namespace fdtdb200
