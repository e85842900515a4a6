// wx3d_wind.cuh -- the userBoundary hook of the spherical-wind problems:
// imposeSphericalWind (winds.f90:123-240) re-imposes a steady r^-2 wind in
// every cell (physical and ghost) within a source's radius after each ghost
// exchange.  Here the ghosts are gathered on the fly from the physical
// cells, so wind_kernel imposes the wind on the physical cells of the stage's
// source array before the stage.  Inline functions only.
#pragma once

#include "wx3d_rates.cuh"

namespace wx {

constexpr double PI_REF = 3.14159265358979;  // source/constants.f90

// Conserved variables of the wind at cell (i, j, k) of block B (ghost
// indices allowed) if the cell centre lies inside a wind sphere; the last
// source that covers it wins, as in the reference's sequential calls.
template <int NEQ, bool MHD>
__device__ __forceinline__ bool wind_state(const PhysParams& ph, const DevBlock& B, int i, int j, int k, double* u) {
  // cellPos (amr.f90:1037-1065), then physical units
  const double x = ((B.bc[0] - 1) * NC + (i - 1) + 0.5) * B.dx * ph.l_sc;
  const double y = ((B.bc[1] - 1) * NC + (j - 1) + 0.5) * B.dy * ph.l_sc;
  const double z = ((B.bc[2] - 1) * NC + (k - 1) + 0.5) * B.dz * ph.l_sc;
  bool hit = false;
  for (int w = 0; w < ph.nwind; ++w) {
    const double* W = ph.wind + 12 * w;
    const double ddx = x - W[0], ddy = y - W[1], ddz = z - W[2];
    const double dist = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
    if (dist < W[6]) {
      const double dens = W[7] / W[8] / dist / dist / (4.0 * PI_REF);
      double p[NEQ];
#pragma unroll
      for (int e = 0; e < NEQ; ++e) p[e] = 0.0;
      p[0] = dens / ph.d_sc;
      p[1] = (W[8] * ddx / dist + W[3]) / ph.v_sc;
      p[2] = (W[8] * ddy / dist + W[4]) / ph.v_sc;
      p[3] = (W[8] * ddz / dist + W[5]) / ph.v_sc;
      p[4] = dens / (W[10] * AMU) * KB * W[9] / ph.p_sc;
      // the reference leaves the passive scalar undefined; a wind of neutral
      // fraction y0 carries neutral density y0 * rho
      if (!MHD && NEQ > 5) p[5] = W[11] * dens / ph.d_sc;
      prim2flow<NEQ, MHD>(p, u, ph.cv);
      hit = true;
    }
  }
  return hit;
}

}  // namespace wx
