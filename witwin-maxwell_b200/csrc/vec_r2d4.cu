// Launch variant 7: z-vectorised step kernel, 2 cells per lane, a 4-plane cp.async ring.
#include "vec_kernel.cuh"

namespace fdtdb200 {

FDTD_VEC_LAUNCHER(launch_vec_r2d4, 2, 4, 2)

}  // namespace fdtdb200
