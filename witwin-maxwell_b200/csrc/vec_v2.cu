// Launch variant 6: z-vectorised step kernel, 2 cells per lane, direct loads.
#include "vec_kernel.cuh"

namespace fdtdb200 {

FDTD_VEC_LAUNCHER(launch_vec_v2, 2, 0, 2)

}  // namespace fdtdb200
