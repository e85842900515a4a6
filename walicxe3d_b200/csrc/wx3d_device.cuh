// wx3d_device.cuh -- device-side physics and ghost gathering for the
// per-block Godunov update on sm_100a.
//
// Layout in HBM: every state array is [slot][eq][k][j][i] with the 16^3
// physical cells of each block only (no ghost storage).  Ghost cells are
// gathered on demand from the neighbour slots through the device neighbour
// table (DevBlock), following source/boundary.f90:74-686.  Cell coordinates
// in this file keep the reference's 1-based convention: physical cells
// 1..16, ghosts -1,0 and 17,18.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/wx3d.h"

namespace wx {

constexpr int NC = WX3D_NCELLS;
constexpr int PLANE = NC * NC;          // 256 cells per k-plane
constexpr int BCELLS = NC * NC * NC;    // 4096 cells per block

// One slot of the device neighbour table (built on the host from the
// reference's tree queries, source/amr.f90:439-1098).
struct __align__(16) DevBlock {
  int32_t level;
  int32_t bID;
  int32_t bc[3];       // block coordinates at its level (bcoords, amr.f90:972)
  int32_t sib[3];      // siblingCoords of this block (amr.f90:831), -1 for roots
  int32_t ftype[6];    // WX_NEIGH_* per face (LEFT..TOP), 0 = empty slot
  int32_t fnb[6][4];   // neighbour slots: [0] for SAME/COARSER, [0..3] for FINER;
                       // for BOUNDARY faces fnb[f][0] holds the BC type
  int32_t wind;        // 1: a wind sphere reaches the block or its ghost cells
  double dx, dy, dz;   // cell size at this level (init.f90:726-730)
};

// Device-resident step control: the simulation-state globals of
// source/globals.f90:52-56 plus the reduction targets of the step.
struct __align__(16) DevCtl {
  double time;
  double dt;
  unsigned long long dtmin_bits;  // min over cells of dx/(|u|+c), as ordered bits
  int32_t it;
  int32_t nextout;
  int32_t dumpout;
  int32_t dumps;                  // outputs that fell inside a batched run
  unsigned long long cnt[4];      // pressure floor, density floor, zero density, non-finite
  unsigned long long maxloss_bits;
  unsigned long long sur[2];      // cells updated by the surrogate / by the plain integrator
  unsigned work_next[2];          // next work item of the running first- and second-order stage
  unsigned pad_[2];
};

struct PhysParams {
  double gamma, cv, cfl, eta;
  double inv_cv;     // 1/cv: flow2prim multiplies by it instead of dividing by cv
  double mu0, mui, ion_thres;
  double d_sc, p_sc, e_sc, t_sc;
  double dtout;
  double cooling_limit;
  int32_t limiter;
  int32_t eight_wave;
  int32_t flux_cd;   // field-CD update of B (brio-wu/flux_cd.f90:52-86)
  int32_t bc[6];
  int32_t eos;
  int32_t cooling;
  int32_t fp;        // 0-based first passive
  int32_t npassive;
  double l_sc, v_sc;
  const double* wind;  // nwind x 12: xc yc zc vx vy vz radius mdot vinf temp mu y0 (cgs)
  int32_t nwind;
};

// ---------------------------------------------------------------------------
// Equation permutations: swapxy / swapxz (hydro_core.f90:448-496) as index maps.
template <int DIR, bool MHD>
__device__ __forceinline__ constexpr int perm(int e) {
  if (DIR == 1) {
    if (e == 1) return 2;
    if (e == 2) return 1;
    if (MHD && e == 5) return 6;
    if (MHD && e == 6) return 5;
  } else if (DIR == 2) {
    if (e == 1) return 3;
    if (e == 3) return 1;
    if (MHD && e == 5) return 7;
    if (MHD && e == 7) return 5;
  }
  return e;
}

__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// Reciprocal and square root for the hot flux path, without the special-case
// branches of IEEE division and sqrt.  The hardware estimate
// rcp.approx.ftz.f64 is refined by two Newton-Raphson steps (quadratic
// convergence: r <- r + r (1 - d r)); rsqrt.approx.ftz.f64 by one
// (y <- y + y (1 - x y^2) / 2), after which the square root x y takes the
// Newton correction s <- s + y (x - s^2) / 2, which squares its remaining
// error once more.  Both lie within 1 ulp of the correctly rounded results
// over 4e6 log-uniform arguments and every power of two and its neighbours
// (checked on the device by wx3d_check_fast_math).  Arguments must be positive and normal: the
// densities and pressures that reach them have passed the floors of
// flow2prim; zero, infinite or NaN arguments give a non-finite result.
__device__ __forceinline__ double rcp_nr(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  r = fma(r, fma(-d, r, 1.0), r);
  r = fma(r, fma(-d, r, 1.0), r);
  return r;
}
__device__ __forceinline__ double sqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = fma(0.5 * y, fma(-x * y, y, 1.0), y);
  const double s = x * y;
  return fma(0.5 * y, fma(-s, s, x), s);
}

// Brings the 128-byte line holding *p into L2 (no register result).
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// flow2prim (hydro_core.f90:323-378).  Returns istat: 0 ok, 1 pressure
// floor, 2 density floor, -1 zero density.  The divisions by rho and by cv
// of the reference are a Newton reciprocal of rho (IEEE division for zero,
// subnormal, infinite or NaN densities, which rcp_nr does not take) and a
// multiplication by inv_cv = 1/cv: the same values to within an ulp.
template <int NEQ, bool MHD>
__device__ __forceinline__ int flow2prim(const double* u, double* p, double inv_cv, double* rinv_out = nullptr) {
  int istat = 0;
  if (u[0] == 0.0) istat = -1;
  double rinv;
  if (fabs(u[0]) >= 2.2250738585072014e-308 && fabs(u[0]) <= 1.0e300) rinv = rcp_nr(u[0]);
  else rinv = 1.0 / u[0];
  if (rinv_out) *rinv_out = rinv;
  p[0] = u[0];
  p[1] = u[1] * rinv;
  p[2] = u[2] * rinv;
  p[3] = u[3] * rinv;
  double pr = (u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) * rinv) * inv_cv;
  if (MHD) pr = pr - 0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]) * inv_cv;
  if (pr < 1.0e-30) { pr = 1.0e-30; if (istat == 0) istat = 1; }
  p[4] = pr;
  if (p[0] < 1.0e-40) {
    p[0] = 1.0e-40;
    if (istat >= 0) istat = 2;
    if (rinv_out) *rinv_out = 1.0e40;
  }
#pragma unroll
  for (int e = 5; e < NEQ; ++e) p[e] = u[e];
  return istat;
}

// prim2flow (hydro_core.f90:278-313), x-oriented state.
template <int NEQ, bool MHD>
__device__ __forceinline__ void prim2flow(const double* p, double* u, double cv) {
  u[0] = p[0];
  u[1] = p[0] * p[1];
  u[2] = p[0] * p[2];
  u[3] = p[0] * p[3];
  u[4] = 0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]) + cv * p[4];
  if (MHD) u[4] = u[4] + 0.5 * (p[5] * p[5] + p[6] * p[6] + p[7] * p[7]);
#pragma unroll
  for (int e = 5; e < NEQ; ++e) u[e] = p[e];
}

// prim2fluxes along x (hydro_core.f90:387-442) of an already permuted state.
template <int NEQ, bool MHD>
__device__ __forceinline__ void xflux(const double* p, double* f, double cv) {
  const double ru = p[0] * p[1];
  f[0] = ru;
  f[1] = ru * p[1] + p[4];
  f[2] = ru * p[2];
  f[3] = ru * p[3];
  f[4] = p[1] * (0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]) + (cv + 1.) * p[4]);
  if (MHD) {
    f[5] = 0.;
    f[6] = p[1] * p[6] - p[2] * p[5];
    f[7] = p[1] * p[7] - p[3] * p[5];
    f[1] = f[1] + 0.5 * (p[6] * p[6] + p[7] * p[7] - p[5] * p[5]);
    f[2] = f[2] - p[5] * p[6];
    f[3] = f[3] - p[5] * p[7];
    f[4] = f[4] + p[1] * (p[5] * p[5] + p[6] * p[6] + p[7] * p[7]) - p[5] * (p[1] * p[5] + p[2] * p[6] + p[3] * p[7]);
  }
  constexpr int FP = MHD ? 8 : 5;
#pragma unroll
  for (int e = FP; e < NEQ; ++e) f[e] = p[1] * p[e];
}

// cfastX (hydro_core.f90:553-566)
__device__ __forceinline__ double cfastX(const double* p, double g) {
  const double b2 = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
  const double rinv = 1.0 / p[0];
  const double a = (g * p[4] + b2) * rinv;
  return sqrt(0.5 * (a + sqrt(a * a - 4. * g * p[4] * (p[5] * p[5]) * rinv * rinv)));
}

// average (hydro_core.f90:640-699)
__device__ __forceinline__ double average(double a, double b, int opt) {
  double s, c, d, r;
  switch (opt) {
    case WX_LIMITER_NO_AVERAGE: return 0.;
    case WX_LIMITER_NONE: return 0.5 * (a + b);
    case WX_LIMITER_VANLEER: return (a * b <= 0.0) ? 0.0 : a * b * (a + b) / (a * a + b * b);
    case WX_LIMITER_MINMOD: s = copysign(1.0, a); return s * dmax(0.0, dmin(fabs(a), s * b));
    case WX_LIMITER_ALBADA: return (a * (b * b + 1.0e-7) + b * (a * a + 1.0e-7)) / (a * a + b * b * 1.0e-7);
    case WX_LIMITER_UMIST:
      s = copysign(1.0, a);
      c = 0.25 * a + 0.75 * b;
      d = 0.75 * a + 0.25 * b;
      r = dmin(dmin(2.0 * fabs(a), 2.0 * s * b), dmin(s * c, s * d));
      return s * dmax(0.0, r);
    case WX_LIMITER_WOODWARD:
      s = copysign(1.0, a);
      c = 0.5 * (a + b);
      r = dmin(dmin(2.0 * fabs(a), 2.0 * s * b), s * c);
      return s * dmax(0.0, r);
    case WX_LIMITER_SUPERBEE:
      s = copysign(1.0, b);
      c = dmin(2.0 * fabs(b), s * a);
      d = dmin(fabs(b), 2.0 * s * a);
      return s * dmax(dmax(0.0, c), d);
    default: return 0.0;
  }
}

// average with the limiter fixed at compile time; LIM_RUNTIME dispatches on
// the run-time value instead.
constexpr int LIM_RUNTIME = -100;

template <int LIM>
__device__ __forceinline__ double average_t(double a, double b, int opt) {
  if constexpr (LIM == WX_LIMITER_MINMOD) {
    // s max(0, min(|a|, s b)) with s = sign(a) is the argument of smaller
    // magnitude when a and b share a sign and (signed) zero otherwise; the
    // product test differs only where a*b underflows (|a b| < 5e-324)
    const double m = fabs(a) < fabs(b) ? a : b;
    return a * b > 0.0 ? m : 0.0;
  } else if constexpr (LIM == WX_LIMITER_VANLEER) {
    const double ab = a * b;
    return (ab <= 0.0) ? 0.0 : ab * (a + b) / (a * a + b * b);
  } else if constexpr (LIM == WX_LIMITER_SUPERBEE) {
    const double s = copysign(1.0, b);
    const double c = dmin(2.0 * fabs(b), s * a);
    const double d = dmin(fabs(b), 2.0 * s * a);
    return s * dmax(dmax(0.0, c), d);
  } else {
    return average(a, b, opt);
  }
}

// ---------------------------------------------------------------------------
// Riemann solvers along x of permuted primitive states.

// HLL with the sound speeds supplied by the caller (hll.f90:175-260).
template <int NEQ>
__device__ __forceinline__ void riemann_hll_c(const double* pL, const double* pR, double cl, double cr, double* f,
                                              double cv) {
  const double sl = dmin(pL[1] - cl, pR[1] - cr);
  const double sr = dmax(pL[1] + cl, pR[1] + cr);
  if (sl >= 0.0) { xflux<NEQ, false>(pL, f, cv); return; }
  if (sr <= 0.0) { xflux<NEQ, false>(pR, f, cv); return; }
  double fL[NEQ], fR[NEQ], uL[NEQ], uR[NEQ];
  xflux<NEQ, false>(pL, fL, cv);
  xflux<NEQ, false>(pR, fR, cv);
  prim2flow<NEQ, false>(pL, uL, cv);
  prim2flow<NEQ, false>(pR, uR, cv);
  const double inv = rcp_nr(sr - sl);   // sl < 0 < sr here
  const double slsr = sl * sr;
#pragma unroll
  for (int e = 0; e < NEQ; ++e) f[e] = (sr * fL[e] - sl * fR[e] + slsr * (uR[e] - uL[e])) * inv;
}

// HLLC with sound speeds and 1/rho supplied by the caller (hllc.f90:209-357).
// The star state needs 1/(sk-sst) and 1/(sk-u_k); both come from one
// reciprocal of their product.
template <int NEQ>
__device__ __forceinline__ void riemann_hllc_c(const double* pL, const double* pR, double cl, double cr, double rl,
                                               double rr, double* f, double cv) {
  const double dl = pL[0], dr = pR[0], ul = pL[1], ur = pR[1];
  const double sl = dmin(ul - cl, ur - cr);
  const double sr = dmax(ul + cl, ur + cr);
  const double sst = (pR[4] - pL[4] + dl * ul * (sl - ul) - dr * ur * (sr - ur)) * rcp_nr(dl * (sl - ul) - dr * (sr - ur));
  const bool useL = (sl > 0.0) || (!(sr < 0.0) && (sst >= 0.0));
  double pk[NEQ];
#pragma unroll
  for (int e = 0; e < NEQ; ++e) pk[e] = useL ? pL[e] : pR[e];
  xflux<NEQ, false>(pk, f, cv);
  if (!(sl > 0.0) && !(sr < 0.0)) {
    const double sk = useL ? sl : sr;
    const double rinv = useL ? rl : rr;
    const double skmu = sk - pk[1];
    const double d1 = sk - sst;
    const double inv = rcp_nr(d1 * skmu);
    const double rhost = pk[0] * (skmu * skmu) * inv;          // rho (sk-u)/(sk-sst)
    const double q = pk[4] * rinv * (d1 * inv);                 // p / (rho (sk-u))
    const double E = 0.5 * pk[0] * (pk[1] * pk[1] + pk[2] * pk[2] + pk[3] * pk[3]) + cv * pk[4];
    double ust[NEQ], uk[NEQ];
    prim2flow<NEQ, false>(pk, uk, cv);
    ust[0] = rhost;
    ust[1] = rhost * sst;
    ust[2] = rhost * pk[2];
    ust[3] = rhost * pk[3];
    ust[4] = rhost * (E * rinv + (sst - pk[1]) * (sst + q));
#pragma unroll
    for (int e = 5; e < NEQ; ++e) ust[e] = rhost * pk[e] * rinv;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) f[e] = f[e] + sk * (ust[e] - uk[e]);
  }
}

// HLL (hll.f90:175-260): Davis wave speeds, branches sl>=0 / sr<=0.
template <int NEQ, bool MHD>
__device__ __forceinline__ void riemann_hll(const double* pL, const double* pR, double* f, double g, double cv) {
  const double cl = sqrt(g * pL[4] / pL[0]);
  const double cr = sqrt(g * pR[4] / pR[0]);
  const double sl = dmin(pL[1] - cl, pR[1] - cr);
  const double sr = dmax(pL[1] + cl, pR[1] + cr);
  if (sl >= 0.0) { xflux<NEQ, MHD>(pL, f, cv); return; }
  if (sr <= 0.0) { xflux<NEQ, MHD>(pR, f, cv); return; }
  double fL[NEQ], fR[NEQ], uL[NEQ], uR[NEQ];
  xflux<NEQ, MHD>(pL, fL, cv);
  xflux<NEQ, MHD>(pR, fR, cv);
  prim2flow<NEQ, MHD>(pL, uL, cv);
  prim2flow<NEQ, MHD>(pR, uR, cv);
  const double inv = 1.0 / (sr - sl);
  const double slsr = sl * sr;
#pragma unroll
  for (int e = 0; e < NEQ; ++e) f[e] = (sr * fL[e] - sl * fR[e] + slsr * (uR[e] - uL[e])) * inv;
}

// HLLE (hlle.f90:166-241): fast magnetosonic speeds, branches sl>0 / sr<0.
template <int NEQ>
__device__ __forceinline__ void riemann_hlle(const double* pL, const double* pR, double* f, double g, double cv) {
  const double cfL = cfastX(pL, g), cfR = cfastX(pR, g);
  const double sl = dmin(pL[1] - cfL, pR[1] - cfR);
  const double sr = dmax(pL[1] + cfL, pR[1] + cfR);
  if (sl > 0.0) { xflux<NEQ, true>(pL, f, cv); return; }
  if (sr < 0.0) { xflux<NEQ, true>(pR, f, cv); return; }
  double fL[NEQ], fR[NEQ], uL[NEQ], uR[NEQ];
  xflux<NEQ, true>(pL, fL, cv);
  xflux<NEQ, true>(pR, fR, cv);
  prim2flow<NEQ, true>(pL, uL, cv);
  prim2flow<NEQ, true>(pR, uR, cv);
  const double inv = 1.0 / (sr - sl);
  const double slsr = sl * sr;
#pragma unroll
  for (int e = 0; e < NEQ; ++e) f[e] = (sr * fL[e] - sl * fR[e] + slsr * (uR[e] - uL[e])) * inv;
}

// HLLC (hllc.f90:209-357).  The four regions of Toro 10.34 are folded into
// one selected side K (L when sl>0, or when sr>=0 and sst>=0; R otherwise)
// so the warp runs one flux evaluation and at most one star correction.
template <int NEQ>
__device__ __forceinline__ void riemann_hllc(const double* pL, const double* pR, double* f, double g, double cv) {
  const double dl = pL[0], dr = pR[0], ul = pL[1], ur = pR[1];
  const double cl = sqrt(g * pL[4] / dl);
  const double cr = sqrt(g * pR[4] / dr);
  const double sl = dmin(ul - cl, ur - cr);
  const double sr = dmax(ul + cl, ur + cr);
  const double sst = (pR[4] - pL[4] + dl * ul * (sl - ul) - dr * ur * (sr - ur)) * rcp_nr(dl * (sl - ul) - dr * (sr - ur));
  const bool useL = (sl > 0.0) || (!(sr < 0.0) && (sst >= 0.0));
  double pk[NEQ];
#pragma unroll
  for (int e = 0; e < NEQ; ++e) pk[e] = useL ? pL[e] : pR[e];
  xflux<NEQ, false>(pk, f, cv);
  if (!(sl > 0.0) && !(sr < 0.0)) {
    const double sk = useL ? sl : sr;
    const double rinv = 1.0 / pk[0];
    const double skmu = sk - pk[1];
    const double rhost = pk[0] * skmu / (sk - sst);
    const double E = 0.5 * pk[0] * (pk[1] * pk[1] + pk[2] * pk[2] + pk[3] * pk[3]) + cv * pk[4];
    double ust[NEQ], uk[NEQ];
    prim2flow<NEQ, false>(pk, uk, cv);
    ust[0] = rhost;
    ust[1] = rhost * sst;
    ust[2] = rhost * pk[2];
    ust[3] = rhost * pk[3];
    ust[4] = rhost * (E * rinv + (sst - pk[1]) * (sst + pk[4] / (pk[0] * skmu)));
#pragma unroll
    for (int e = 5; e < NEQ; ++e) ust[e] = rhost * pk[e] * rinv;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) f[e] = f[e] + sk * (ust[e] - uk[e]);
  }
}

// HLLD (hlld.f90:166-444), Miyoshi & Kusano five-state fan.  Passive
// scalars (NEQ>8) keep the caller's f values in the star regions, as the
// reference's intent(inout) ff does with PASSIVES undefined; the UR*
// region's denr==0 branch leaves the right star variables at 0.
template <int NEQ>
__device__ __forceinline__ void riemann_hlld(const double* pl, const double* pr, double* ff, double g, double cv) {
  const double csl = cfastX(pl, g), csr = cfastX(pr, g);
  const double sr = dmax(pl[1] + csl, pr[1] + csr);
  const double sl = dmin(pl[1] - csl, pr[1] - csr);
  if (sl > 0.0) { xflux<NEQ, true>(pl, ff, cv); return; }
  if (sr < 0.0) { xflux<NEQ, true>(pr, ff, cv); return; }
  const double bx = 0.5 * (pl[5] + pr[5]);
  const double signBx = copysign(1., bx);
  const double bx2 = bx * bx;
  const double pTL = pl[4] + 0.5 * (bx2 + pl[6] * pl[6] + pl[7] * pl[7]);
  const double pTR = pr[4] + 0.5 * (bx2 + pr[6] * pr[6] + pr[7] * pr[7]);
  const double slmul = sl - pl[1];
  const double srmur = sr - pr[1];
  const double den = srmur * pr[0] - slmul * pl[0];
  const double sM = (srmur * (pr[0] * pr[1]) - slmul * (pl[0] * pl[1]) - pTR + pTL) / den;
  const double srmsM = sr - sM;
  const double slmsM = sl - sM;
  const double rhostl = pl[0] * slmul / slmsM;
  const double rhostr = pr[0] * srmur / srmsM;
  const double sqrl = sqrt(rhostl), sqrr = sqrt(rhostr);
  const double sstl = sM - fabs(bx) / sqrl;
  const double sstr = sM + fabs(bx) / sqrr;
  const double pst = (srmur * pr[0] * pTL - slmul * pl[0] * pTR + pl[0] * pr[0] * srmur * slmul * (pr[1] - pl[1])) / den;
  const bool leftside = (sstl >= 0.0) || (!(sstr <= 0.0) && (sM >= 0.0));
  // star state of the left or right side
  double vstl = 0, wstl = 0, bystl = 0, bzstl = 0, vstr = 0, wstr = 0, bystr = 0, bzstr = 0;
  const double sMmul = sM - pl[1], sMmur = sM - pr[1];
  const double denl = pl[0] * slmul * slmsM - bx2;
  const double denr = pr[0] * srmur * srmsM - bx2;
  const bool needL = (sstl >= 0.0) || !(sstr <= 0.0);
  const bool needR = !(sstl >= 0.0);
  if (needL) {
    if (denl == 0) { vstl = pl[2]; wstl = pl[3]; bystl = 0.; bzstl = 0.; }
    else {
      const double q = 1.0 / denl;
      vstl = pl[2] - bx * pl[6] * sMmul * q;
      wstl = pl[3] - bx * pl[7] * sMmul * q;
      const double t = (pl[0] * (slmul * slmul) - bx2) * q;
      bystl = pl[6] * t;
      bzstl = pl[7] * t;
    }
  }
  if (needR) {
    if (denr == 0) {
      if (sstr <= 0.0) { vstl = pl[2]; wstl = pl[3]; bystl = 0.; bzstl = 0.; }
      else { vstr = pr[2]; wstr = pr[3]; bystr = 0.; bzstr = 0.; }
    } else {
      const double q = 1.0 / denr;
      vstr = pr[2] - bx * pr[6] * sMmur * q;
      wstr = pr[3] - bx * pr[7] * sMmur * q;
      const double t = (pr[0] * (srmur * srmur) - bx2) * q;
      bystr = pr[6] * t;
      bzstr = pr[7] * t;
    }
  }
  const double* pk = leftside ? pl : pr;
  const double skmu = leftside ? slmul : srmur;
  const double skms = leftside ? slmsM : srmsM;
  const double pTk = leftside ? pTL : pTR;
  const double rhost = leftside ? rhostl : rhostr;
  const double ek = 0.5 * pk[0] * (pk[1] * pk[1] + pk[2] * pk[2] + pk[3] * pk[3]) + cv * pk[4] +
                    0.5 * (bx2 + pk[6] * pk[6] + pk[7] * pk[7]);
  const double vdotb = pk[1] * bx + pk[2] * pk[6] + pk[3] * pk[7];
  const double vst = leftside ? vstl : vstr, wst = leftside ? wstl : wstr;
  const double byst = leftside ? bystl : bystr, bzst = leftside ? bzstl : bzstr;
  const double vstdotbst = sM * bx + vst * byst + wst * bzst;
  const double est = (skmu * ek - pTk * pk[1] + pst * sM + bx * (vdotb - vstdotbst)) / skms;
  if ((sstl >= 0.0) || (sstr <= 0.0)) {  // UL* or UR*
    ff[0] = rhost * sM;
    ff[1] = rhost * (sM * sM) + pst - bx2;
    ff[2] = rhost * sM * vst - bx * byst;
    ff[3] = rhost * sM * wst - bx * bzst;
    ff[4] = sM * (est + pst) - bx * vstdotbst;
    ff[5] = 0.;
    ff[6] = byst * sM - bx * vst;
    ff[7] = bzst * sM - bx * wst;
    return;
  }
  const double dd = sqrl + sqrr;
  const double ddi = 1.0 / dd;
  const double vstst = (sqrl * vstl + sqrr * vstr + (bystr - bystl) * signBx) * ddi;
  const double wstst = (sqrl * wstl + sqrr * wstr + (bzstr - bzstl) * signBx) * ddi;
  const double sqlr = sqrt(rhostl * rhostr);
  const double bystst = (sqrl * bystr + sqrr * bystl + sqlr * (vstr - vstl) * signBx) * ddi;
  const double bzstst = (sqrl * bzstr + sqrr * bzstl + sqlr * (wstr - wstl) * signBx) * ddi;
  const double vststdotbstst = sM * bx + vstst * bystst + wstst * bzstst;
  const double sq = leftside ? sqrl : sqrr;
  const double estst = leftside ? est - sq * (vstdotbst - vststdotbstst) * signBx
                                : est + sq * (vstdotbst - vststdotbstst) * signBx;
  ff[0] = rhost * sM;
  ff[1] = rhost * (sM * sM) + pst - bx2;
  ff[2] = rhost * sM * vstst - bx * bystst;
  ff[3] = rhost * sM * wstst - bx * bzstst;
  ff[4] = sM * (estst + pst) - bx * vststdotbstst;
  ff[5] = 0.;
  ff[6] = bystst * sM - bx * vstst;
  ff[7] = bzstst * sM - bx * wstst;
}

template <int NEQ, bool MHD, int SOLVER>
__device__ __forceinline__ void riemann(const double* pL, const double* pR, double* f, double g, double cv) {
  if constexpr (SOLVER == WX_SOLVER_HLLC) {
    riemann_hllc<NEQ>(pL, pR, f, g, cv);
  } else if constexpr (SOLVER == WX_SOLVER_HLLE) {
    riemann_hlle<NEQ>(pL, pR, f, g, cv);
  } else if constexpr (SOLVER == WX_SOLVER_HLLD) {
    riemann_hlld<NEQ>(pL, pR, f, g, cv);
  } else {
    riemann_hll<NEQ, MHD>(pL, pR, f, g, cv);
  }
}

// ---------------------------------------------------------------------------
// Ghost gathering (boundary.f90:74-686, single process).  (i,j,k) is a face
// ghost cell of the block described by `b` -- exactly one coordinate lies
// outside 1..16.  `a` is the array whose physical cells feed the fill.  The
// fill depth does not change the value of a given ghost cell, so one
// function serves boundary(1,.) and boundary(2,.).

__device__ __forceinline__ size_t cell_off(int slot, int neq, int e, int i, int j, int k) {
  return (((size_t)slot * neq + e) * NC + (k - 1)) * PLANE + (size_t)(j - 1) * NC + (i - 1);
}

template <int NEQ>
__device__ __forceinline__ void load_cell(const double* __restrict__ a, int slot, int i, int j, int k, double* u) {
  const double* p = a + cell_off(slot, NEQ, 0, i, j, k);
#pragma unroll
  for (int e = 0; e < NEQ; ++e) u[e] = __ldg(p + (size_t)e * BCELLS);
}

// Plain (coherent) loads for an array the same kernel writes.
template <int NEQ>
__device__ __forceinline__ void load_cell_rw(const double* a, int slot, int i, int j, int k, double* u) {
  const double* p = a + cell_off(slot, NEQ, 0, i, j, k);
#pragma unroll
  for (int e = 0; e < NEQ; ++e) u[e] = p[(size_t)e * BCELLS];
}

template <int NEQ>
__device__ void gather_ghost(const double* __restrict__ a, const DevBlock& b, int slot, int i, int j, int k,
                             double* u) {
  // face and axis of the ghost cell; coordinates are remapped per axis
  // without local arrays so nothing spills to the stack
  int f;
  if (i < 1) f = 0;
  else if (i > NC) f = 1;
  else if (j < 1) f = 2;
  else if (j > NC) f = 3;
  else if (k < 1) f = 4;
  else f = 5;
  const int ax = f >> 1, side = f & 1;
  const int type = b.ftype[f];
  if (type == WX_NEIGH_SAME) {  // boundary.f90:329-366
    const int sh = side ? -NC : NC;
    if (ax == 0) i += sh; else if (ax == 1) j += sh; else k += sh;
    load_cell<NEQ>(a, b.fnb[f][0], i, j, k, u);
  } else if (type == WX_NEIGH_COARSER) {  // boundary.f90:385-412
    const int fc = side ? 1 : NC;
    const int ci = ax == 0 ? fc : (i + 1) / 2 + b.sib[0] * (NC / 2);
    const int cj = ax == 1 ? fc : (j + 1) / 2 + b.sib[1] * (NC / 2);
    const int ck = ax == 2 ? fc : (k + 1) / 2 + b.sib[2] * (NC / 2);
    load_cell<NEQ>(a, b.fnb[f][0], ci, cj, ck, u);
  } else if (type == WX_NEIGH_FINER) {  // boundary.f90:494-540
    const int si = (i - 1) / (NC / 2), sj = (j - 1) / (NC / 2), sk = (k - 1) / (NC / 2);
    // child among the four: transverse sibling bits in x<y<z order
    const int q = ax == 0 ? sj + 2 * sk : (ax == 1 ? si + 2 * sk : si + 2 * sj);
    const int src = b.fnb[f][q];
    auto lo_n = [&](int g) { return side ? 2 * (g - NC) - 1 : NC + 2 * g - 1; };
    const int li = ax == 0 ? lo_n(i) : 2 * (i - si * (NC / 2)) - 1;
    const int lj = ax == 1 ? lo_n(j) : 2 * (j - sj * (NC / 2)) - 1;
    const int lk = ax == 2 ? lo_n(k) : 2 * (k - sk * (NC / 2)) - 1;
    const double* p = a + cell_off(src, NEQ, 0, li, lj, lk);
#pragma unroll
    for (int e = 0; e < NEQ; ++e) {
      const double* qq = p + (size_t)e * BCELLS;
      // x outer, y, z inner: the accumulation order of boundary.f90:516-536
      double s = 0.0;
      s += __ldg(qq);
      s += __ldg(qq + PLANE);
      s += __ldg(qq + NC);
      s += __ldg(qq + NC + PLANE);
      s += __ldg(qq + 1);
      s += __ldg(qq + 1 + PLANE);
      s += __ldg(qq + 1 + NC);
      s += __ldg(qq + 1 + NC + PLANE);
      u[e] = s * 0.125;
    }
  } else {  // domain boundary (boundary.f90:594-673); the BC type sits in fnb[f][0]
    const int bct = b.fnb[f][0];
    const int g = ax == 0 ? i : (ax == 1 ? j : k);
    const int src = bct == WX_BC_REFLECTIVE ? (side ? 2 * NC - g + 1 : 1 - g)
                                            : (side ? 2 * NC - g + 1 : 1);  // free flow: low copies cell 1
    if (ax == 0) i = src; else if (ax == 1) j = src; else k = src;
    load_cell<NEQ>(a, slot, i, j, k, u);
    if (bct == WX_BC_REFLECTIVE) {
      if (ax == 0) u[1] = -1.0 * u[1];
      else if (ax == 1) u[2] = -1.0 * u[2];
      else u[3] = -1.0 * u[3];
    }
  }
}

template <int NEQ>
__device__ __forceinline__ void get_cell(const double* __restrict__ a, const DevBlock& b, int slot, int i, int j,
                                         int k, double* u) {
  if (i >= 1 && i <= NC && j >= 1 && j <= NC && k >= 1 && k <= NC) load_cell<NEQ>(a, slot, i, j, k, u);
  else gather_ghost<NEQ>(a, b, slot, i, j, k, u);
}

// CFL time step of one cell (hydro_core.f90:503-543, hydro_solver.f90:441-455).
template <int NEQ, bool MHD>
__device__ __forceinline__ double cell_dt(const double* p, const DevBlock& B, double g) {
  if (MHD) {
    const double b2 = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
    const double a = g * p[4] + b2;
    const double cfx = sqrt(0.5 * (a + sqrt(a * a - 4. * g * p[4] * p[5] * p[5])) / p[0]);
    const double cfy = sqrt(0.5 * (a + sqrt(a * a - 4. * g * p[4] * p[6] * p[6])) / p[0]);
    const double cfz = sqrt(0.5 * (a + sqrt(a * a - 4. * g * p[4] * p[7] * p[7])) / p[0]);
    return dmin(dmin(B.dx / (fabs(p[1]) + cfx), B.dy / (fabs(p[2]) + cfy)), B.dz / (fabs(p[3]) + cfz));
  }
  const double cs = sqrt(g * p[4] / p[0]);
  return dmin(dmin(B.dx / (fabs(p[1]) + cs), B.dy / (fabs(p[2]) + cs)), B.dz / (fabs(p[3]) + cs));
}

// The CFL condition of a hydro cell as a signal speed over the cell size,
// max_d (|u_d| + c)/dx_d, whose reciprocal is cell_dt's
// min_d dx_d/(|u_d| + c).  A block's kernels keep the largest speed and take
// one reciprocal at the end, so the per-cell work has no division.  idx..idz
// are 1/dx..1/dz; rinv is 1/rho of flow2prim.
__device__ __forceinline__ double cell_cfl_speed(const double* p, double rinv, double idx, double idy, double idz,
                                                 double g) {
  const double cs = sqrt_nr(g * p[4] * rinv);
  return dmax(dmax((fabs(p[1]) + cs) * idx, (fabs(p[2]) + cs) * idy), (fabs(p[3]) + cs) * idz);
}

// One thread's running CFL reduction over the cells it visits: for hydro the
// largest cell_cfl_speed (one reciprocal at the end), for MHD the smallest
// cell_dt.  block() takes the inverse cell sizes of the block being walked.
template <int NEQ, bool MHD>
struct Cfl {
  double acc = MHD ? 1.0e300 : 0.0;
  double idx = 0.0, idy = 0.0, idz = 0.0;
  __device__ __forceinline__ void block(const DevBlock& B) {
    if (!MHD) { idx = 1.0 / B.dx; idy = 1.0 / B.dy; idz = 1.0 / B.dz; }
  }
  __device__ __forceinline__ void fold(const double* p, double rinv, const DevBlock& B, double g) {
    fold(p, rinv, B, idx, idy, idz, g);
  }
  // the same with the inverse cell sizes passed in (block() not used)
  __device__ __forceinline__ void fold(const double* p, double rinv, const DevBlock& B, double ix, double iy,
                                       double iz, double g) {
    if constexpr (MHD) acc = dmin(acc, cell_dt<NEQ, MHD>(p, B, g));
    else acc = dmax(acc, cell_cfl_speed(p, rinv, ix, iy, iz, g));
  }
  // the thread's time step (infinite when it saw no cell)
  __device__ __forceinline__ double dt() const { return MHD ? acc : 1.0 / acc; }
};

// Ordered bit patterns of positive doubles compare like the doubles.
__device__ __forceinline__ void atomic_min_pos(unsigned long long* t, double v) {
  atomicMin(t, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_pos(unsigned long long* t, double v) {
  atomicMax(t, (unsigned long long)__double_as_longlong(v));
}

}  // namespace wx
