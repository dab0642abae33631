// The mixed-precision reciprocal and sincos (kt_physics.cuh: mx_rcp,
// mx_sincos) on the device against the division and against the
// renderer's libm.  Prints "max_rcp_ulp <u> max_sincos_abs <e> status <s>".
// Built and run by tests/test_gpu_mixed.py.
#include <cstdio>
#include <cstdint>
#include <cmath>
#include <random>
#include <vector>

#include "kt_physics.cuh"

using namespace kt;

__global__ void k_check(const double* x, double* o, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  o[4 * (size_t)i + 0] = mx_rcp<double>(x[i]);
  o[4 * (size_t)i + 1] = 1.0 / x[i];
  double s, c;
  // [-8, 8], and every 16th argument beyond the fast path's range
  mx_sincos((i % 16 == 15) ? ((i % 200001) - 100000) * 3e2 : ((i % 200001) - 100000) * 8e-5, &s, &c);
  o[4 * (size_t)i + 2] = s;
  o[4 * (size_t)i + 3] = c;
}

int main() {
  const int n = 1 << 22;
  std::vector<double> x(n);
  std::mt19937_64 rng(11);
  for (int i = 0; i < n; ++i) {
    const double m = 1.0 + (double)(rng() >> 11) * 0x1p-53;
    const int e = (int)(rng() % 2000) - 1000;  // beyond the fast range too
    x[i] = std::ldexp(m, e) * ((i & 1) ? -1.0 : 1.0);
  }
  x[0] = 0.0; x[1] = -0.0; x[2] = INFINITY; x[3] = 1e-300; x[4] = 1e300; x[5] = 3.0;
  double *dx = nullptr, *dout = nullptr;
  cudaMalloc(&dx, n * sizeof(double));
  cudaMalloc(&dout, 4 * (size_t)n * sizeof(double));
  cudaMemcpy(dx, x.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  k_check<<<(n + 255) / 256, 256>>>(dx, dout, n);
  std::vector<double> o(4 * (size_t)n);
  cudaMemcpy(o.data(), dout, 4 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  const cudaError_t err = cudaDeviceSynchronize();
  double max_ulp = 0.0, max_sc = 0.0;
  for (int i = 0; i < n; ++i) {
    const double got = o[4 * (size_t)i], want = o[4 * (size_t)i + 1];
    if (std::isinf(want) || want == 0.0) {
      if (got != want) max_ulp = INFINITY;
      continue;
    }
    int ex;
    std::frexp(want, &ex);
    const double ulp = std::ldexp(1.0, std::max(ex - 53, -1074));
    max_ulp = std::max(max_ulp, std::fabs(got - want) / ulp);
    const double a = (i % 16 == 15) ? ((i % 200001) - 100000) * 3e2 : ((i % 200001) - 100000) * 8e-5;
    double hs, hc;
    ktm_sincos(a, &hs, &hc);
    max_sc = std::max(max_sc, std::max(std::fabs(o[4 * (size_t)i + 2] - hs), std::fabs(o[4 * (size_t)i + 3] - hc)));
  }
  std::printf("max_rcp_ulp %.3g max_sincos_abs %.3g status %s\n", max_ulp, max_sc, cudaGetErrorString(err));
  return err == cudaSuccess ? 0 : 1;
}
