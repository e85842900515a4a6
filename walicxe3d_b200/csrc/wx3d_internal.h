// wx3d_internal.h -- declarations shared by the translation units of
// libwx3d.so (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>

#include "wx3d_device.cuh"

struct wx_mlp;

namespace wx {

// Trust table of the surrogate: bins of log10(n_H * dt/yr), log10 T, x_HII.
constexpr int TRUST_ND = 48, TRUST_T = 48, TRUST_X = 8;
constexpr double TRUST_ND_LO = -5.0, TRUST_ND_W = 0.25;
constexpr double TRUST_T_LO = 2.0, TRUST_T_W = 0.125;
constexpr int TRUST_BYTES = TRUST_ND * TRUST_T * TRUST_X;

struct SurrLaunch {
  int neq;
  double* u;
  const DevBlock* blocks;
  const int32_t* work;
  int nwork;
  DevCtl* ctl;
  PhysParams ph;
  const wx_mlp* mlp;
  const uint8_t* trust;   // device [TRUST_ND][TRUST_T][TRUST_X], 1 = surrogate may be used
  int do_dt;
  int nsm;
  // table cooling that follows the hydrogen update when the cooling type is
  // not COOL_H (the layout of the plain source step's table)
  const double* cool_lt;
  const double* cool_lc;
  int ncool;
  int nZ;
};

// Fused updatePrims + surrogate (or plain) hrate, then cooling_h from the
// network (or plain) or table cooling (plain), + CFL minimum.
cudaError_t launch_surrogate_source(const SurrLaunch& L, cudaStream_t s);

}  // namespace wx
