// wx3d_rates.cuh -- device restatement of calcTemp (hydro_core.f90:231-270),
// the hydrogen rate solution (hrate.f90), the Biro et al. 1999 loss rate
// (cooling_h.f90) and the cooling-table lookup (cooling.f90).  Inline
// functions only, so several translation units can include it.
#pragma once

#include "wx3d_device.cuh"

namespace wx {

constexpr double AMU = 1.660538782e-24;  // source/constants.f90:37
constexpr double KB = 1.380650400e-16;   // source/constants.f90:38

// calcTemp (hydro_core.f90:231-270); EOS >= 0 fixes the equation of state
// at compile time, -1 reads it from ph.
template <int FP, int EOS = -1>
__device__ __forceinline__ double calc_temp(const double* p, const PhysParams& ph) {
  double temp = 0.0;
  switch (EOS >= 0 ? EOS : ph.eos) {
    case WX_EOS_ADIABATIC:
    case WX_EOS_SINGLE_SPECIE: temp = p[4] / p[0] * (ph.mu0 * AMU * ph.p_sc / ph.d_sc / KB); break;
    case WX_EOS_TWOTEMP:
      temp = p[4] / p[0] * (ph.mu0 * AMU * ph.p_sc / ph.d_sc / KB);
      if (temp > ph.ion_thres) temp = p[4] / p[0] * (ph.mui * AMU * ph.p_sc / ph.d_sc / KB);
      break;
    case WX_EOS_H_RATE:
      if (ph.npassive >= 1) temp = p[4] / (2.0 * p[0] / ph.mu0 - p[FP]) * ph.p_sc / KB;
      break;
  }
  return temp;
}

// solve_h_rate for one cell (hrate.f90:96-137); returns the new neutral
// fraction y1 for the cell's temperature T and H density dh.
__device__ __forceinline__ double h_rate_y1(double T, double dh, double y0, double dts) {
  const double xi = 1.e-4;
  const double col = 5.83e-11 * sqrt(T) * exp(-157828. / T);   // colf, hrate.f90:73
  const double rec = 2.55e-13 * exp(0.79 * log(1.e4 / T));    // alpha, hrate.f90:58: (1e4/T)^0.79
  const double a = rec + col;
  const double b = -((2.0 + xi) * rec + (1.0 + xi) * col + 0.0);
  const double c = (1.0 + xi) * rec;
  const double d = sqrt(b * b - 4.0 * a * c);
  const double g0 = (2.0 * a * y0 + b + d) / (2.0 * a * y0 + b - d);
  const double e = exp(-d * dh * dts);
  double y1 = (-b - d * (1.0 + g0 * e) / (1.0 - g0 * e)) / (2.0 * a);
  y1 = dmin(y1, 1.0 - xi);
  y1 = dmax(y1, 0.0);
  return y1;
}

// betah and aloss (cooling_h.f90:42-145), Biro et al. 1999 loss rate.
__device__ __forceinline__ double betah(double T) {
  const double a = 157890. / T;
  const double la = log(a);  // a^-0.33333 = exp(-0.33333 ln a)
  return 1.133e-24 / sqrt(a) * (-0.0713 + 0.5 * la + 0.640 * exp(-0.33333 * la));
}

__device__ __forceinline__ double aloss_h(double x1, double den, double dH0, double Te0) {
  const double XION = 2.179e-11, XO = 1.e-3;
  const double C0 = 0.5732, C1 = 1.8288e-5, C2 = -1.15822e-10, C3 = 9.4288e-16;
  const double D0 = 0.5856, D1 = 1.55083e-5, D2 = -9.669e-12, D3 = 5.716e-19;
  const double ENK = 118409., EN = 1.634E-11;
  const double Te = dmax(Te0, 10.);
  const double dHp = (1. - x1) * den;
  const double de = dHp + 1.E-4 * den;
  const double dOI = XO * dH0;
  const double dOII = XO * dHp;
  if (Te <= 1e4) return 1e-30;
  double omega;
  const double oL = C0 + Te * (C1 + Te * (C2 + Te * C3));
  const double oH = D0 + Te * (D1 + Te * (D2 + Te * D3));
  if (Te <= 55000.) omega = oL;
  else if (Te >= 72000.) omega = oH;
  else {
    const double frac = (Te - 55000.) / 17000.;
    omega = (1. - frac) * oL + frac * oH;
  }
  const double sTe = sqrt(Te);
  const double qla = 8.6287E-6 / (2. * sTe) * omega * exp(-ENK / Te);
  const double ecoll = dmax(de * dH0 * qla * EN, 0.);
  const double cion = 5.834E-11 * sTe * exp(-1.579E5 / Te);
  const double eion = de * dH0 * cion * XION;
  const double erec = dmax(de * dHp * betah(Te), 0.);
  const double Tm = 1. / Te;
  const double Tm2 = Tm * Tm;
  const double eOI = dmax(de * dOI * exp10(1381465 * Tm2 - 12328.69 * Tm - 19.82621), 0.);
  const double eOII = dmax(de * dOII * exp10(-2061075. * Tm2 - 14596.24 * Tm - 19.01402), 0.);
  const double betaf = 1.3 * 1.42E-27 * sTe;  // Te^0.5
  const double HIIcool = de * dHp * betaf;
  // Te^0.63 and (Te 1e-5)^1.63 as exp(a ln x)
  const double equil = (1.0455E-18 / exp(0.63 * log(Te))) * (1. - exp(-exp(1.63 * log(Te * 1.E-5)))) * de * den + HIIcool;
  double fr;
  if (Te <= 44770.) fr = 0.;
  else if (Te >= 54770.) fr = 1.;
  else {
    const double ex2 = exp(-2. * (Te - 49770.) / 500.);
    fr = 0.5 * (1. + (1. - ex2) / (1. + ex2));
  }
  return ecoll + eion + (erec + 7.033 * (eOI + eOII)) * (1. - fr) + equil * fr;
}

// find_coef (cooling.f90:378-419).  The reference scans for the first row
// whose logT exceeds the argument; on the (increasing) table this is the
// upper bound found here by bisection.
__device__ __forceinline__ double find_coef(const double* __restrict__ lt, const double* __restrict__ lc, int n,
                                            double logT) {
  if (logT < lt[0]) return 0.0;
  if (logT >= lt[n - 1]) return exp10(lc[n - 1] + 0.5 * (logT - lt[n - 1]));
  int lo = 0, hi = n - 1;  // lt[lo] <= logT < lt[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (lt[mid] > logT) hi = mid; else lo = mid;
  }
  const double T0 = lt[hi - 1], C0 = lc[hi - 1], T1 = lt[hi], C1 = lc[hi];
  return exp10((C1 - C0) / (T1 - T0) * (logT - T0) + C0);
}

// find_coef_metal (cooling.f90:435-519) on cooltable(nT+1, nZ+1) stored row
// by row: row 0 holds the metallicities, column 0 the log temperatures.
// Above the last temperature the reference extrapolates from row nptsT, one
// below the last data row; that row is used here as well.
__device__ __forceinline__ double find_coef_metal(const double* __restrict__ tab, int nT, int nZ, double logT,
                                                  double Z) {
  const int W = nZ + 1;
  auto ct = [&](int i, int j) { return tab[(i - 1) * W + (j - 1)]; };  // 1-based as the reference
  const double Tmin = ct(2, 1), Tmax = ct(nT + 1, 1);
  if (logT < Tmin) return 0.0;
  int Tlo = 2, Thi = nT + 1;
  double T0 = 0.0, T1 = 0.0;
  if (logT <= Tmax) {
    while (Thi - Tlo > 1) {
      const int Tmid = (Tlo + Thi) / 2;
      if (logT <= ct(Tmid, 1)) Thi = Tmid; else Tlo = Tmid;
    }
    T0 = ct(Tlo, 1);
    T1 = ct(Thi, 1);
  }
  int Zlo, Zhi;
  if (Z < ct(1, 2)) { Zlo = 2; Zhi = 3; }
  else if (Z > ct(1, nZ + 1)) { Zlo = nZ; Zhi = nZ + 1; }
  else {
    Zlo = 2; Zhi = nZ + 1;
    while (Zhi - Zlo > 1) {
      const int Zmid = (Zlo + Zhi) / 2;
      if (Z <= ct(1, Zmid)) Zhi = Zmid; else Zlo = Zmid;
    }
  }
  const double Z0 = ct(1, Zlo), Z1 = ct(1, Zhi);
  if (logT >= Tmax) {
    const double C0 = ct(nT, Zlo) + 0.5 * (logT - Tmax);
    const double C1 = ct(nT, Zhi) + 0.5 * (logT - Tmax);
    return exp10((C1 - C0) / (Z1 - Z0) * (Z - Z0) + C0);
  }
  const double TC = (logT - T0) / (T1 - T0);
  const double ZC = (Z - Z0) / (Z1 - Z0);
  const double coef = (1.0 - TC) * (1.0 - ZC) * ct(Tlo, Zlo) + (1.0 - TC) * ZC * ct(Tlo, Zhi) +
                      TC * (1.0 - ZC) * ct(Thi, Zlo) + TC * ZC * ct(Thi, Zhi);
  return exp10(coef);
}

// get_lambda (cooling_schure.f90:102-128): 180 rows of linear T and Lambda,
// rows 0.04 dex apart from log T = 1.
__device__ __forceinline__ double get_lambda_schure(const double* __restrict__ Tt, const double* __restrict__ Lt,
                                                    double T) {
  if (T > 1e8) return 0.21e-26 * sqrt(T);
  const int if1 = (int)((log10(T) - 1.0) / 0.04) + 1;
  if (if1 < 1) return Lt[0];
  const double T0 = Tt[if1 - 1], c0 = Lt[if1 - 1], T1 = Tt[if1], c1 = Lt[if1];
  return (c1 - c0) * (T - T0) / (T1 - T0) + c0;
}

// One plain step of updateNeutralFraction then apply_cooling_h_neq for a cell
// (hrate.f90:101-140, cooling_h.f90:175-246) on its conserved u and
// primitive p vectors -- the arithmetic of source_kernel's fused H_RATE +
// COOL_H path.  FP is the index of the neutral-H passive scalar.
template <int FP>
__device__ __forceinline__ void h_cool_step(double* u, double* p, double dts, const PhysParams& ph, double* mloss) {
  {
    const double T = calc_temp<FP, WX_EOS_H_RATE>(p, ph);
    const double dh = p[0] / ph.mu0;
    const double y0 = p[FP] / dh;
    const double y1 = h_rate_y1(T, dh, y0, dts);
    p[FP] = p[0] * y1 / ph.mu0;
  }
  const double dh = p[0] / ph.mu0;
  const double dh0 = p[FP];
  const double y0 = ph.mu0 * u[FP] / u[0];
  u[FP] = p[FP];
  const double Temp = calc_temp<FP, WX_EOS_H_RATE>(p, ph);
  if (Temp > 1.e4) {
    const double L0 = aloss_h(y0, dh, dh0, Temp);
    const double ce = (2.0 * L0) / (3.0 * KB * dh * Temp);
    const double T1 = 10.0 + (Temp - 10.0) * exp(-ce * dts);
    double cf = T1 / Temp;
    *mloss = dmax(*mloss, 1.0 - cf);
    if (cf < 1.0 - ph.cooling_limit) cf = 1.0 - ph.cooling_limit;
    if (Temp * cf < 10.0) cf = 10.0 / Temp;
    p[4] = p[4] * cf;
    const double EK = 0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
    u[4] = EK + ph.cv * p[4];
  }
}

// Table cooling of one cell after the hydrogen update: COOL_TABLE and
// COOL_TABLE_METAL (apply_cooling, cooling.f90:303-369) and COOL_SCHURE
// (cooling_schure.f90:134-228); updates p[4] and u[4] and folds the largest
// fractional loss into mloss.  No-op for other cooling types or an unloaded
// table.  COOL and EOS >= 0 fix the cooling type and the equation of state
// at compile time; -1 reads them from ph.
template <int NEQ, int FP, int COOL = -1, int EOS = -1>
__device__ __forceinline__ void table_cooling(double* u, double* p, double dts, const PhysParams& ph,
                                              const double* __restrict__ cool_lt, const double* __restrict__ cool_lc,
                                              int ncool, int nZ, double& mloss) {
  const int cooling = COOL >= 0 ? COOL : ph.cooling;
  if ((cooling == WX_COOL_TABLE || cooling == WX_COOL_TABLE_METAL) && ncool >= 2) {  // cooling.f90:303-369
    const bool metal_tab = cooling == WX_COOL_TABLE_METAL;
    const double temp = calc_temp<FP, EOS>(p, ph);
    const double logT = log10(temp);
    // metalpas = neqhydro + neqmhd + min(npassive, 1) (parameters.f90:318)
    const int mp = FP + (ph.npassive >= 1 ? 1 : 0) - 1;
    const double Tmin = metal_tab ? cool_lt[nZ + 1] : cool_lt[0];
    if (logT >= Tmin) {
      const double ETH = ph.cv * p[4];
      const double EK = 0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
      double al;
      if (metal_tab) {
        double metal = 0.0;
#pragma unroll
        for (int e = 0; e < NEQ; ++e)
          if (e == mp) metal = fabs(p[e] / p[0]);
        al = find_coef_metal(cool_lt, ncool, nZ, logT, metal);
      } else {
        al = find_coef(cool_lt, cool_lc, ncool, logT);
      }
      const double nd = p[0] * ph.d_sc / (ph.mui * AMU);
      const double ce = al * (nd * nd) / (ETH * ph.e_sc);
      double cf = exp(-ce * dts);
      mloss = dmax(mloss, 1.0 - cf);
      if (cf < 1.0 - ph.cooling_limit) cf = 1.0 - ph.cooling_limit;
      if (temp * cf < 10.0) cf = 10.0 / temp;
      p[4] = p[4] * cf;
      u[4] = EK + ph.cv * p[4];
    }
  } else if (cooling == WX_COOL_SCHURE && ncool == 180) {  // cooling_schure.f90:134-228
    const double T = calc_temp<FP, EOS>(p, ph);
    if (T > 10.0) {
      const double Lambda0 = get_lambda_schure(cool_lt, cool_lc, T);
      const double dens = p[0] / ph.mu0;
      const double emtauC = exp(-2.0 * dts * dens * Lambda0 / (3.0 * KB * T));
      double cf = (0.0 / (dens * dens * Lambda0)) * (1.0 - emtauC) + emtauC;  // gain = 0
      mloss = dmax(mloss, 1.0 - cf);
      if (cf < 1.0 - ph.cooling_limit) cf = 1.0 - ph.cooling_limit;
      p[4] = p[4] * cf;
      u[4] = ph.cv * p[4] + 0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
    }
  }
}

}  // namespace wx
