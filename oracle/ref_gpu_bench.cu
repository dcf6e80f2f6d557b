// ref_gpu_bench.cu -- times the reference's own single-GPU solver on the benchmark workload.
//
// MEASUREMENT INFRASTRUCTURE (oracle side): this driver is compiled with the reference's
// sources from where they lie (oracle/Makefile, target refgpu -> oracle/_ref/ref_gpu_bench)
// and is run only by the comparison workload of bench.py. Nothing in the product links it.
//
// It builds the reference's host solver sgn::SGN2D (src/solver/sgn2d.h:57-59) on the
// configuration-2 mesh with the elliptic-shoal still depth and the free surface of 8 sine
// waves (parameters on the command line, so that both sides use the same numbers), with
// the reference's only boundary (periodic), uploads it to sgn::SGN2DCuda
// (src/cuda/sgn2d_cuda.h:30-47), and times SGN2DCuda::integrateAdaptive over [0, tEnd]
// over [0, steps x dt0] (dt0 = the CFL-0.5 step, SGN2D::cflTimeStep) with CUDA events on
// the default stream the reference launches on, after one untimed warm-up integration of
// the same length; the median of reps runs. It prints one JSON line.
//
//   ref_gpu_bench Nx Ny Lx Ly steps reps H0 Hc xc yc ax ay a1..a8 l1..l8 t1..t8 p1..p8
#include "cuda/sgn2d_cuda.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char** argv) {
  if (argc != 7 + 6 + 32) {
    std::fprintf(stderr, "usage: ref_gpu_bench Nx Ny Lx Ly steps reps H0 Hc xc yc ax ay "
                         "amp[8] lam[8] theta[8] phase[8]\n");
    return 2;
  }
  const int Nx = std::atoi(argv[1]), Ny = std::atoi(argv[2]);
  const double Lx = std::atof(argv[3]), Ly = std::atof(argv[4]);
  const int steps = std::max(1, std::atoi(argv[5]));
  const int reps = std::max(1, std::atoi(argv[6]));
  double sh[6], wv[32];
  for (int i = 0; i < 6; ++i) sh[i] = std::atof(argv[7 + i]);
  for (int i = 0; i < 32; ++i) wv[i] = std::atof(argv[13 + i]);

  sgn2d::Params par;
  par.g = 9.81;
  par.c = 3.0 * std::sqrt(par.g * sh[0]);
  par.gamma = 1.5;
  // elliptic shoal: H0 - (H0 - Hc) (1 - r^2)^3 inside the ellipse, H0 outside
  auto depth = [sh](double x, double y) {
    const double dx = (x - sh[2]) / sh[4], dy = (y - sh[3]) / sh[5];
    const double r2 = dx * dx + dy * dy;
    if (r2 >= 1.0) return sh[0];
    const double q = 1.0 - r2;
    return sh[0] - (sh[0] - sh[1]) * (q * q * q);
  };
  sgn::SGN2D host(4, Nx, Ny, Lx, Ly, par, depth);
  std::vector<double> x, y;
  host.nodeCoords(x, y);
  const size_t Nd = x.size();
  std::vector<double> h(Nd), z(Nd, 0.0);
  const double kPi = 3.14159265358979323846;
  for (size_t i = 0; i < Nd; ++i) {
    double eta = 0.0;
    for (int j = 0; j < 8; ++j) {
      const double k = 2.0 * kPi / wv[8 + j];
      eta += wv[j] * std::sin(k * (x[i] * std::cos(wv[16 + j]) + y[i] * std::sin(wv[16 + j])) +
                              wv[24 + j]);
    }
    h[i] = depth(x[i], y[i]) + eta;
  }
  const sgn::State U = host.makeState(h, z, z, z, z);
  const double dt0 = host.cflTimeStep(U, 0.5);
  const double tEnd = steps * dt0;

  sgn::SGN2DCuda dev(host);
  dev.upload(U);
  dev.integrateAdaptive(0.0, tEnd, dt0);  // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  std::vector<double> ms(reps);
  sgn::AdaptiveRKStats st;
  for (int r = 0; r < reps; ++r) {
    dev.upload(U);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    st = dev.integrateAdaptive(0.0, tEnd, dt0);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float m = 0.f;
    cudaEventElapsedTime(&m, e0, e1);
    ms[r] = m;
  }
  std::sort(ms.begin(), ms.end());
  const double t = ms[reps / 2] / 1e3;
  const double dof = 5.0 * (double)Nd;
  std::printf("{\"impl\": \"reference-gpu\", \"solver\": \"sgn::SGN2DCuda::integrateAdaptive\", "
              "\"mesh\": [%d, %d], \"dof\": %.0f, \"tEnd\": %.17g, \"accepted\": %ld, "
              "\"rejected\": %ld, \"rhsEvals\": %ld, \"time_s\": %.9g, \"reps\": %d, "
              "\"value\": %.9g, \"unit\": \"DOF-updates/s\"}\n",
              Nx, Ny, dof, tEnd, (long)st.accepted, (long)st.rejected, (long)st.rhsEvals, t, reps,
              dof * (double)st.rhsEvals / t);
  return 0;
}
