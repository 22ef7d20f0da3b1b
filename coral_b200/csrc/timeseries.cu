// Timeseries reduction: the per-CTA partial sums of the timeseries objects
// (volume averages and horizontal averages at grid levels, computed by the z
// kernels on the first stage's physical fields) totalled over the grid, as
// output_global_quantities does with its loops over the local grid
// (src/plane_layer/PL_IMEX_timestepping_output.f90:30-127).
#include "device.hpp"

namespace coral {
namespace {

constexpr int kTsThreads = 256;

// one CTA per object; each thread sums a fixed strided subset, then a fixed
// tree: the result does not depend on scheduling
__global__ void __launch_bounds__(kTsThreads) k_ts_reduce(const double* part, size_t ncta, double scale,
                                                          double* out) {
  __shared__ double red[kTsThreads];
  const int o = blockIdx.x;
  double s = 0.0;
  for (size_t c = threadIdx.x; c < ncta; c += kTsThreads) s += part[c * kMaxTs + o];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kTsThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[o] = red[0] * scale;
}

}  // namespace

void launch_ts_reduce(const double* part, size_t ncta, int nobj, double scale, double* out, cudaStream_t s) {
  if (nobj <= 0) return;
  k_ts_reduce<<<nobj, kTsThreads, 0, s>>>(part, ncta, scale, out);
}

}  // namespace coral
