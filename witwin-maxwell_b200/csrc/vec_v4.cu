// Launch variant 5: z-vectorised step kernel, 4 cells per lane, direct loads;
// also the footprint classifier of every vectorised variant.
#include "vec_kernel.cuh"

namespace fdtdb200 {

FDTD_VEC_LAUNCHER(launch_vec_v4, 4, 0, 1)

int launch_classify_vec(const StepParams& p, int V, int n_kblocks, int n_chunks, unsigned char* out,
                        cudaStream_t stream) {
  const int64_t tasks = static_cast<int64_t>(n_chunks) * n_kblocks * p.NY;
  const int64_t blocks = (tasks + 7) / 8;
  if (V == 4) classify_vec_kernel<4><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(p, n_kblocks, n_chunks, out);
  else classify_vec_kernel<2><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(p, n_kblocks, n_chunks, out);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace fdtdb200
