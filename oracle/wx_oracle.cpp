// wx_oracle.cpp -- CPU oracle for the Walicxe3D per-block Godunov update.
//
// TEST INFRASTRUCTURE ONLY.  This file is a literal FP64 restatement, in
// C++17, of the reference Fortran routines on the hot path.  It is used by
// tests/ (as the checker), by __graft_entry__.smoke() and by bench.py's CPU
// baseline leg.  The product path (walicxe3d_b200/, libwx3d.so) never links,
// loads or calls it.
//
// PARITY UNPINNED: the reference has no tests, fixtures or golden vectors,
// and no Fortran compiler exists on the build or GPU machines, so this
// restatement cannot be checked against the reference binary.  It is pinned
// instead by physics checks written for this project (exact Riemann solution
// of the Sod problem, FP64 conservation, octant symmetry of the blast wave,
// Brio-Wu wave structure).
//
// Restatement rules: Fortran arrays U/UP/PRIM(nbMaxProc,neq,-1:18,-1:18,-1:18)
// become per-slot arrays [slot][eq][k][j][i] with the same ghost ranges;
// indices i,j,k keep the Fortran (1-based, ghosts -1,0,17,18) values;
// equation numbers are 0-based (eq 1 -> 0).  Fortran x**2 is x*x, integer
// division truncates toward zero as in C, sign(1,a) is copysign(1,a), and
// expressions keep the Fortran evaluation order.  Compiled with
// -ffp-contract=off and without fast-math.

#include "../include/wx3d.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int NC = WX3D_NCELLS;       // ncells_x = ncells_y = ncells_z
constexpr int NGH = WX3D_NGHOST;      // nghost
constexpr int NT = NC + 2 * NGH;      // 20 cells with ghosts
constexpr int NCELL = NT * NT * NT;   // 8000
constexpr int MAXEQ = WX3D_MAX_NEQ;

inline int cidx(int i, int j, int k) { return (i + 1) + NT * ((j + 1) + NT * (k + 1)); }

// Physical constants (source/constants.f90:37-47).
constexpr double AMU = 1.660538782e-24;
constexpr double KB = 1.380650400e-16;
constexpr double PI = 3.14159265358979;

enum { CELLS_ALL = 0, CELLS_PHYS = 1, CELLS_GHOST = 2 };  // constants.f90:117-119
enum { DIM_X = 1, DIM_Y = 2, DIM_Z = 3 };

struct Wind {
  double xc, yc, zc, vx, vy, vz, radius, mdot, vinf, temp, mu, y0;
};

struct Ctx {
  wx_config cfg{};
  int neq = 5, nbMax = 0, fp = 5;  // fp: 0-based first passive (firstpas-1)
  double cv = 1.5, p_sc = 1, e_sc = 1, t_sc = 1;
  std::vector<double> U, UP, PRIM;
  std::vector<int> localBlocks;
  std::unordered_map<int, int> slotOf;  // stands in for find() over globalBlocks
  int nbx[WX3D_MAX_LEVELS + 2]{}, nby[WX3D_MAX_LEVELS + 2]{}, nbz[WX3D_MAX_LEVELS + 2]{};
  int minID[WX3D_MAX_LEVELS + 2]{}, maxID[WX3D_MAX_LEVELS + 2]{};
  double dx[WX3D_MAX_LEVELS + 2]{}, dy[WX3D_MAX_LEVELS + 2]{}, dz[WX3D_MAX_LEVELS + 2]{};
  double time = 0, dt = 0;
  int it = 0, nextout = 1;
  bool dumpout = false;
  std::vector<double> cooltable1, cooltable2;  // cooltable(1,:), cooltable(2,:)
  // COOL_TABLE_METAL: cooltable(nptsT+1, nptsZ+1), stored [i-1][j-1] row by row
  std::vector<double> ctab_metal;
  int nptsZ = 0;
  double cool_Zmin = 0, cool_Zmax = 0;
  // COOL_SCHURE: 180 rows of (T, Lambda), both linear
  std::vector<double> schureT, schureL;
  int nptsT = 0;
  double cool_Tmin = 0, cool_Tmax = 0;
  std::vector<Wind> winds;
  long long pressure_floor = 0, density_floor = 0, zero_density = 0;
  double maxloss = 0;
  int nthreads = 1;

  double* u(std::vector<double>& a, int nb, int eq) { return a.data() + ((size_t)nb * neq + eq) * NCELL; }
  const double* u(const std::vector<double>& a, int nb, int eq) const {
    return a.data() + ((size_t)nb * neq + eq) * NCELL;
  }
};

// ---------------------------------------------------------------------------
// Block tree queries (source/amr.f90:439-1098), geometry (init.f90:632-756)

int offsets(const Ctx& c, int level) {  // amr.f90:663-677
  int o = 0;
  for (int ilev = 2; ilev <= level; ++ilev) {
    int p = 1;
    for (int q = 0; q < ilev - 2; ++q) p *= 8;
    o += c.cfg.nbrootx * c.cfg.nbrooty * c.cfg.nbrootz * p;
  }
  return o;
}

int meshlevel(const Ctx& c, int bID) {  // amr.f90:637-656
  if (bID == -1) return -1;
  for (int level = 1; level <= c.cfg.maxlev; ++level)
    if (bID >= c.minID[level] && bID <= c.maxID[level]) return level;
  return c.cfg.maxlev + 1;  // Fortran loop exits with level = maxlev+1
}

void bcoords(const Ctx& c, int bID, int& x, int& y, int& z) {  // amr.f90:972-997
  int ilev = meshlevel(c, bID);
  int nx = c.nbx[ilev], ny = c.nby[ilev], nz = c.nbz[ilev];
  int localID = bID - offsets(c, ilev);
  x = localID % nx;
  if (x == 0) x = nx;
  y = (int)std::ceil(localID * 1.0 / nx) % ny;
  if (y == 0) y = ny;
  z = (int)std::ceil(localID * 1.0 / (nx * ny)) % nz;
  if (z == 0) z = nz;
}

int neighborLevel(const Ctx& c, int bID, int dir) {  // amr.f90:439-523
  int x, y, z;
  bcoords(c, bID, x, y, z);
  int ilev = meshlevel(c, bID);
  int nx = c.nbx[ilev], ny = c.nby[ilev], nz = c.nbz[ilev];
  int xp = x, yp = y, zp = z;
  switch (dir) {
    case WX_LEFT: if (x == 1) return -1; xp = x - 1; break;
    case WX_RIGHT: if (x == nx) return -1; xp = x + 1; break;
    case WX_FRONT: if (y == 1) return -1; yp = y - 1; break;
    case WX_BACK: if (y == ny) return -1; yp = y + 1; break;
    case WX_BOTTOM: if (z == 1) return -1; zp = z - 1; break;
    case WX_TOP: if (z == nz) return -1; zp = z + 1; break;
    default: return 0;
  }
  return 1 + (xp - 1) + (yp - 1) * nx + (zp - 1) * nx * ny + offsets(c, ilev);
}

int father(const Ctx& c, int bID) {  // amr.f90:916-961
  if (bID == -1) return -1;
  int ilev = meshlevel(c, bID);
  if (ilev == 1) return -1;
  int x, y, z;
  bcoords(c, bID, x, y, z);
  int xp = (int)std::floor((x + 1) / 2.0), yp = (int)std::floor((y + 1) / 2.0),
      zp = (int)std::floor((z + 1) / 2.0);
  int nx = c.nbx[ilev - 1], ny = c.nby[ilev - 1];
  return 1 + (xp - 1) + (yp - 1) * nx + (zp - 1) * nx * ny + offsets(c, ilev - 1);
}

int firstborn(const Ctx& c, int bID) {  // amr.f90:684-717
  int x, y, z;
  bcoords(c, bID, x, y, z);
  int ilev = meshlevel(c, bID);
  int nx = c.nbx[ilev + 1], ny = c.nby[ilev + 1];
  int xp = 2 * x - 1, yp = 2 * y - 1, zp = 2 * z - 1;
  return 1 + (xp - 1) + (yp - 1) * nx + (zp - 1) * nx * ny + offsets(c, ilev + 1);
}

void children(const Ctx& c, int bID, int out[8]) {  // amr.f90:882-909
  int fb = firstborn(c, bID);
  int ilev = meshlevel(c, bID);
  int nx = c.nbx[ilev + 1], ny = c.nby[ilev + 1];
  out[0] = fb; out[1] = fb + 1; out[2] = fb + nx; out[3] = fb + nx + 1;
  out[4] = fb + nx * ny; out[5] = fb + nx * ny + 1; out[6] = fb + nx * ny + nx; out[7] = fb + nx * ny + nx + 1;
}

void siblings(const Ctx& c, int bID, int out[8]) {  // amr.f90:739-775
  int f = father(c, bID);
  if (f == -1) { for (int i = 0; i < 8; ++i) out[i] = -1; return; }
  int fb = firstborn(c, f);
  int ilev = meshlevel(c, bID);
  int nx = c.nbx[ilev], ny = c.nby[ilev];
  out[0] = fb; out[1] = fb + 1; out[2] = fb + nx; out[3] = fb + nx + 1;
  out[4] = fb + nx * ny; out[5] = fb + nx * ny + 1; out[6] = fb + nx * ny + nx; out[7] = fb + nx * ny + nx + 1;
}

void siblingCoords(const Ctx& c, int bID, int& sx, int& sy, int& sz) {  // amr.f90:831-873
  if (father(c, bID) == -1) { sx = sy = sz = -1; return; }
  int sl[8];
  siblings(c, bID, sl);
  int sID = -1;
  for (int i = 0; i < 8; ++i) if (sl[i] == bID) { sID = i + 1; break; }
  sx = (sID % 2 == 0) ? 1 : 0;
  sy = (sID == 3 || sID == 4 || sID == 7 || sID == 8) ? 1 : 0;
  sz = (sID > 4) ? 1 : 0;
}

bool active(const Ctx& c, int bID) { return c.slotOf.count(bID) != 0; }

// neighbors (amr.f90:539-631).  The scan over globalBlocks returns on the
// first hit of either the same-level neighbour or its father; with a valid
// tree at most one of them is active.
void neighbors(const Ctx& c, int bID, int dir, int& ntype, int list[4]) {
  ntype = -1;
  for (int b = 0; b < 4; ++b) list[b] = -1;
  if (bID == -1) return;
  int nID = neighborLevel(c, bID, dir);
  int fID = father(c, nID);
  if (nID == -1) { ntype = WX_NEIGH_BOUNDARY; return; }
  if (active(c, nID)) { ntype = WX_NEIGH_SAME; list[0] = nID; return; }
  if (fID != -1 && active(c, fID)) { ntype = WX_NEIGH_COARSER; list[0] = fID; return; }
  ntype = WX_NEIGH_FINER;
  int ch[8];
  children(c, nID, ch);
  static const int pick[6][4] = {{2, 4, 6, 8}, {1, 3, 5, 7}, {3, 4, 7, 8},
                                 {1, 2, 5, 6}, {5, 6, 7, 8}, {1, 2, 3, 4}};
  for (int b = 0; b < 4; ++b) list[b] = ch[pick[dir - 1][b] - 1];
}

void cellPos(const Ctx& c, int bID, int i, int j, int k, double& x, double& y, double& z) {  // amr.f90:1037-1065
  int ilev = meshlevel(c, bID);
  int xb, yb, zb;
  bcoords(c, bID, xb, yb, zb);
  x = ((xb - 1) * NC + (i - 1) + 0.5) * c.dx[ilev];
  y = ((yb - 1) * NC + (j - 1) + 0.5) * c.dy[ilev];
  z = ((zb - 1) * NC + (k - 1) + 0.5) * c.dz[ilev];
}

// ---------------------------------------------------------------------------
// hydro_core.f90

// flow2prim (hydro_core.f90:323-378).  Returns istat; -1 = zero density.
int flow2prim(const Ctx& c, const double* uv, double* pv) {
  int istat = 0;
  if (uv[0] == 0.0) return -1;  // clean_abort(ERROR_DIVISION_BY_ZERO), :335-338
  pv[0] = uv[0];
  pv[1] = uv[1] / uv[0];
  pv[2] = uv[2] / uv[0];
  pv[3] = uv[3] / uv[0];
  pv[4] = (uv[4] - 0.5 * (uv[1] * uv[1] + uv[2] * uv[2] + uv[3] * uv[3]) / uv[0]) / c.cv;
  if (c.cfg.bfield && c.cfg.mhd) pv[4] = pv[4] - 0.5 * (uv[5] * uv[5] + uv[6] * uv[6] + uv[7] * uv[7]) / c.cv;
  if (pv[4] < 1.0e-30) { pv[4] = 1.0e-30; istat = 1; }
  if (pv[0] < 1.0e-40) { pv[0] = 1.0e-40; istat = 2; }
  if (c.cfg.bfield) { pv[5] = uv[5]; pv[6] = uv[6]; pv[7] = uv[7]; }
  if (c.cfg.npassive >= 1) for (int e = c.fp; e < c.neq; ++e) pv[e] = uv[e];
  return istat;
}

// prim2flow (hydro_core.f90:278-313).
void prim2flow(const Ctx& c, const double* pv, double* uv) {
  uv[0] = pv[0];
  uv[1] = pv[0] * pv[1];
  uv[2] = pv[0] * pv[2];
  uv[3] = pv[0] * pv[3];
  double v2 = pv[1] * pv[1] + pv[2] * pv[2] + pv[3] * pv[3];
  uv[4] = 0.5 * pv[0] * v2 + c.cv * pv[4];
  if (c.cfg.bfield) {
    if (c.cfg.mhd) uv[4] = uv[4] + 0.5 * (pv[5] * pv[5] + pv[6] * pv[6] + pv[7] * pv[7]);
    uv[5] = pv[5]; uv[6] = pv[6]; uv[7] = pv[7];
  }
  if (c.cfg.npassive >= 1) for (int e = c.fp; e < c.neq; ++e) uv[e] = pv[e];
}

void swapxy(const Ctx& c, double* v) {  // hydro_core.f90:448-469
  std::swap(v[1], v[2]);
  if (c.cfg.bfield) std::swap(v[5], v[6]);
}
void swapxz(const Ctx& c, double* v) {  // hydro_core.f90:475-496
  std::swap(v[1], v[3]);
  if (c.cfg.bfield) std::swap(v[5], v[7]);
}

// prim2fluxes (hydro_core.f90:387-442).
void prim2fluxes(const Ctx& c, const double* pvars, int dimens, double* flux) {
  double p[MAXEQ];
  for (int e = 0; e < c.neq; ++e) p[e] = pvars[e];
  if (dimens == DIM_Y) swapxy(c, p);
  else if (dimens == DIM_Z) swapxz(c, p);
  flux[0] = p[0] * p[1];
  flux[1] = p[0] * (p[1] * p[1]) + p[4];
  flux[2] = p[0] * p[1] * p[2];
  flux[3] = p[0] * p[1] * p[3];
  flux[4] = p[1] * (0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]) + (c.cv + 1.) * p[4]);
  if (c.cfg.bfield) {
    flux[5] = 0.;
    flux[6] = p[1] * p[6] - p[2] * p[5];
    flux[7] = p[1] * p[7] - p[3] * p[5];
    if (c.cfg.mhd) {
      flux[1] = flux[1] + 0.5 * (p[6] * p[6] + p[7] * p[7] - p[5] * p[5]);
      flux[2] = flux[2] - p[5] * p[6];
      flux[3] = flux[3] - p[5] * p[7];
      flux[4] = flux[4] + p[1] * (p[5] * p[5] + p[6] * p[6] + p[7] * p[7]) -
                p[5] * (p[1] * p[5] + p[2] * p[6] + p[3] * p[7]);
    }
  }
  if (c.cfg.npassive >= 1) for (int e = c.fp; e < c.neq; ++e) flux[e] = p[1] * p[e];
  if (dimens == DIM_Y) swapxy(c, flux);
  else if (dimens == DIM_Z) swapxz(c, flux);
}

double sound(const Ctx& c, const double* pv) { return std::sqrt(c.cfg.gamma * pv[4] / pv[0]); }  // :503-515

void cfast(const Ctx& c, double p, double d, double bx, double by, double bz, double& cfx, double& cfy,
           double& cfz) {  // hydro_core.f90:530-543
  double g = c.cfg.gamma;
  double b2 = bx * bx + by * by + bz * bz;
  double a = g * p + b2;
  cfx = std::sqrt(0.5 * (a + std::sqrt(a * a - 4. * g * p * bx * bx)) / d);
  cfy = std::sqrt(0.5 * (a + std::sqrt(a * a - 4. * g * p * by * by)) / d);
  cfz = std::sqrt(0.5 * (a + std::sqrt(a * a - 4. * g * p * bz * bz)) / d);
}

double cfastX(const Ctx& c, const double* pr) {  // hydro_core.f90:553-566
  double g = c.cfg.gamma;
  double b2 = pr[5] * pr[5] + pr[6] * pr[6] + pr[7] * pr[7];
  double cs2va2 = (g * pr[4] + b2) / pr[0];
  return std::sqrt(0.5 * (cs2va2 + std::sqrt(cs2va2 * cs2va2 - 4. * g * pr[4] * (pr[5] * pr[5]) / pr[0] / pr[0])));
}

// average (hydro_core.f90:640-699)
double average(double a, double b, int opt) {
  double s, cc, d, r;
  switch (opt) {
    case WX_LIMITER_NO_AVERAGE: return 0.;
    case WX_LIMITER_NONE: return 0.5 * (a + b);
    case WX_LIMITER_VANLEER:
      if (a * b <= 0.0) return 0.0;
      return a * b * (a + b) / (a * a + b * b);
    case WX_LIMITER_MINMOD:
      s = std::copysign(1.0, a);
      return s * std::max(0.0, std::min(std::fabs(a), s * b));
    case WX_LIMITER_ALBADA: {
      double eps = 1.0e-7;
      return (a * (b * b + eps) + b * (a * a + eps)) / (a * a + b * b * eps);
    }
    case WX_LIMITER_UMIST:
      s = std::copysign(1.0, a);
      cc = 0.25 * a + 0.75 * b;
      d = 0.75 * a + 0.25 * b;
      r = std::min(std::min(2.0 * std::fabs(a), 2.0 * s * b), std::min(s * cc, s * d));
      return s * std::max(0.0, r);
    case WX_LIMITER_WOODWARD:
      s = std::copysign(1.0, a);
      cc = 0.5 * (a + b);
      r = std::min(std::min(2.0 * std::fabs(a), 2 * s * b), s * cc);
      return s * std::max(0.0, r);
    case WX_LIMITER_SUPERBEE:
      s = std::copysign(1.0, b);
      cc = std::min(2.0 * std::fabs(b), s * a);
      d = std::min(std::fabs(b), 2.0 * s * a);
      return s * std::max(std::max(0.0, cc), d);
    default: return 0.0;
  }
}

// limiter (hydro_core.f90:613-636)
void limiter(const double* pll, double* pl, double* pr, const double* prr, int lim, int neqs) {
  for (int e = 0; e < neqs; ++e) {
    double dl = pl[e] - pll[e];
    double dm = pr[e] - pl[e];
    double dr = prr[e] - pr[e];
    double al = average(dl, dm, lim);
    double ar = average(dm, dr, lim);
    pl[e] = pl[e] + 0.5 * al;
    pr[e] = pr[e] - 0.5 * ar;
  }
}

// calcTemp (hydro_core.f90:231-270)
double calcTemp(const Ctx& c, const double* pv) {
  const wx_config& f = c.cfg;
  double temp = 0.0;
  switch (f.eos_type) {
    case WX_EOS_ADIABATIC:
    case WX_EOS_SINGLE_SPECIE: temp = pv[4] / pv[0] * (f.mu0 * AMU * c.p_sc / f.d_sc / KB); break;
    case WX_EOS_TWOTEMP:
      temp = pv[4] / pv[0] * (f.mu0 * AMU * c.p_sc / f.d_sc / KB);
      if (temp > f.ion_thres) temp = pv[4] / pv[0] * (f.mui * AMU * c.p_sc / f.d_sc / KB);
      break;
    case WX_EOS_H_RATE:
      if (f.npassive >= 1) temp = pv[4] / (2.0 * pv[0] / f.mu0 - pv[c.fp]) * c.p_sc / KB;
      break;
  }
  return temp;
}

// calcPrimsBlock (hydro_core.f90:108-223)
void calcPrimsBlock(Ctx& c, const std::vector<double>& uv, std::vector<double>& pv, int nb, int cells,
                    long long& pf, long long& df, long long& zd) {
  double ub[MAXEQ], pb[MAXEQ];
  auto one = [&](int i, int j, int k) {
    int id = cidx(i, j, k);
    for (int e = 0; e < c.neq; ++e) ub[e] = c.u(uv, nb, e)[id];
    int ist = flow2prim(c, ub, pb);
    if (ist < 0) { ++zd; return; }
    if (ist == 1) ++pf;
    if (ist == 2) ++df;
    for (int e = 0; e < c.neq; ++e) c.u(pv, nb, e)[id] = pb[e];
  };
  auto ghost = [&](int i, int j, int k) {
    if (c.u(uv, nb, 0)[cidx(i, j, k)] != 0.0) one(i, j, k);
  };
  if (cells == CELLS_ALL || cells == CELLS_PHYS)
    for (int k = 1; k <= NC; ++k)
      for (int j = 1; j <= NC; ++j)
        for (int i = 1; i <= NC; ++i) one(i, j, k);
  if (cells == CELLS_ALL || cells == CELLS_GHOST) {
    const int lo = 1 - NGH, hi = NC + NGH;
    for (int k = lo; k <= hi; ++k)
      for (int j = lo; j <= hi; ++j)
        for (int i = 1 - NGH; i <= 0; ++i) ghost(i, j, k);
    for (int k = lo; k <= hi; ++k)
      for (int j = lo; j <= hi; ++j)
        for (int i = NC + 1; i <= NC + 2; ++i) ghost(i, j, k);
    for (int k = lo; k <= hi; ++k)
      for (int j = 1 - NGH; j <= 0; ++j)
        for (int i = lo; i <= hi; ++i) ghost(i, j, k);
    for (int k = lo; k <= hi; ++k)
      for (int j = NC + 1; j <= NC + 2; ++j)
        for (int i = lo; i <= hi; ++i) ghost(i, j, k);
    for (int k = 1 - NGH; k <= 0; ++k)
      for (int j = lo; j <= hi; ++j)
        for (int i = lo; i <= hi; ++i) ghost(i, j, k);
    for (int k = NC + 1; k <= NC + 2; ++k)
      for (int j = lo; j <= hi; ++j)
        for (int i = lo; i <= hi; ++i) ghost(i, j, k);
  }
}

// calcPrimsAll (hydro_core.f90:67-95) over occupied slots.
void calcPrimsAll(Ctx& c, const std::vector<double>& uv, std::vector<double>& pv, int cells) {
  long long pf = 0, df = 0, zd = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : pf, df, zd) num_threads(c.nthreads)
  for (int nb = 0; nb < c.nbMax; ++nb)
    if (c.localBlocks[nb] != -1) calcPrimsBlock(c, uv, pv, nb, cells, pf, df, zd);
  c.pressure_floor += pf;
  c.density_floor += df;
  c.zero_density += zd;
}

// ---------------------------------------------------------------------------
// Riemann solvers

// wavespeedHLL / primfhll (hll.f90:175-260)
void primfhll(const Ctx& c, const double* pL, const double* pR, double* ff) {
  double cl = sound(c, pL), cr = sound(c, pR);
  double sl = std::min(pL[1] - cl, pR[1] - cr);
  double sr = std::max(pL[1] + cl, pR[1] + cr);
  double fL[MAXEQ], fR[MAXEQ], uL[MAXEQ], uR[MAXEQ];
  if (sl >= 0) { prim2fluxes(c, pL, DIM_X, ff); return; }
  if (sr <= 0) { prim2fluxes(c, pR, DIM_X, ff); return; }
  prim2fluxes(c, pL, DIM_X, fL);
  prim2fluxes(c, pR, DIM_X, fR);
  prim2flow(c, pL, uL);
  prim2flow(c, pR, uR);
  for (int e = 0; e < c.neq; ++e) ff[e] = (sr * fL[e] - sl * fR[e] + sl * sr * (uR[e] - uL[e])) / (sr - sl);
}

// wavespeedHLLC / primfhllc (hllc.f90:209-357).  The NaN fall-through of
// :290-296 leaves ff untouched, as in the reference.
void primfhllc(const Ctx& c, const double* pL, const double* pR, double* ff) {
  double dl1 = pL[0], dr1 = pR[0], ul1 = pL[1], ur1 = pR[1], pl1 = pL[4], pr1 = pR[4];
  double cl = sound(c, pL), cr = sound(c, pR);
  double sl = std::min(ul1 - cl, ur1 - cr);
  double sr = std::max(ul1 + cl, ur1 + cr);
  double sst = 0.0;
  if (c.cfg.solver_type == WX_SOLVER_HLLC)
    sst = (pr1 - pl1 + dl1 * ul1 * (sl - ul1) - dr1 * ur1 * (sr - ur1)) / (dl1 * (sl - ul1) - dr1 * (sr - ur1));
  double f[MAXEQ], u[MAXEQ], ust[MAXEQ];
  if (sl > 0) { prim2fluxes(c, pL, DIM_X, ff); return; }
  if (sr < 0) { prim2fluxes(c, pR, DIM_X, ff); return; }
  if (sst >= 0) {
    prim2fluxes(c, pL, DIM_X, f);
    prim2flow(c, pL, u);
    double rhost = pL[0] * (sl - pL[1]) / (sl - sst);
    double EL = 0.5 * pL[0] * (pL[1] * pL[1] + pL[2] * pL[2] + pL[3] * pL[3]) + c.cv * pL[4];
    ust[0] = rhost;
    ust[1] = rhost * sst;
    ust[2] = rhost * pL[2];
    ust[3] = rhost * pL[3];
    ust[4] = rhost * (EL / pL[0] + (sst - pL[1]) * (sst + pL[4] / (pL[0] * (sl - pL[1]))));
    if (c.cfg.npassive >= 1) for (int e = 5; e < c.neq; ++e) ust[e] = rhost * pL[e] / pL[0];
    for (int e = 0; e < c.neq; ++e) ff[e] = f[e] + sl * (ust[e] - u[e]);
    return;
  }
  if (sst <= 0) {
    prim2fluxes(c, pR, DIM_X, f);
    prim2flow(c, pR, u);
    double rhost = pR[0] * (sr - pR[1]) / (sr - sst);
    double ER = 0.5 * pR[0] * (pR[1] * pR[1] + pR[2] * pR[2] + pR[3] * pR[3]) + c.cv * pR[4];
    ust[0] = rhost;
    ust[1] = rhost * sst;
    ust[2] = rhost * pR[2];
    ust[3] = rhost * pR[3];
    ust[4] = rhost * (ER / pR[0] + (sst - pR[1]) * (sst + pR[4] / (pR[0] * (sr - pR[1]))));
    if (c.cfg.npassive >= 1) for (int e = 5; e < c.neq; ++e) ust[e] = rhost * pR[e] / pR[0];
    for (int e = 0; e < c.neq; ++e) ff[e] = f[e] + sr * (ust[e] - u[e]);
    return;
  }
}

// wavespeedHLLE / primfhlle (hlle.f90:166-241)
void primfhlle(const Ctx& c, const double* pL, const double* pR, double* ff) {
  double cfL = cfastX(c, pL), cfR = cfastX(c, pR);
  double sl = std::min(pL[1] - cfL, pR[1] - cfR);
  double sr = std::max(pL[1] + cfL, pR[1] + cfR);
  double fL[MAXEQ], fR[MAXEQ], uL[MAXEQ], uR[MAXEQ];
  if (sl > 0) { prim2fluxes(c, pL, DIM_X, ff); return; }
  if (sr < 0) { prim2fluxes(c, pR, DIM_X, ff); return; }
  prim2fluxes(c, pL, DIM_X, fL);
  prim2fluxes(c, pR, DIM_X, fR);
  prim2flow(c, pL, uL);
  prim2flow(c, pR, uR);
  for (int e = 0; e < c.neq; ++e) ff[e] = (sr * fL[e] - sl * fR[e] + sl * sr * (uR[e] - uL[e])) / (sr - sl);
}

// primfhlld (hlld.f90:166-444).  ff is intent(inout): passive components
// keep the caller's value in the star regions (PASSIVES undefined).  The
// denr==0 branch of the UR* region assigns the *left* star variables
// (:289-295) and leaves vstr..bzstr undefined; they are 0 here.
void primfhlld(const Ctx& c, const double* priml, const double* primr, double* ff) {
  const double cv = c.cv;
  double csl = cfastX(c, priml), csr = cfastX(c, primr);
  double sr = std::max(priml[1] + csl, primr[1] + csr);
  double sl = std::min(priml[1] - csl, primr[1] - csr);
  if (sl > 0) { prim2fluxes(c, priml, DIM_X, ff); return; }
  if (sr < 0) { prim2fluxes(c, primr, DIM_X, ff); return; }
  double bx = 0.5 * (priml[5] + primr[5]);
  double signBx = std::copysign(1., bx);
  double pTL = priml[4] + 0.5 * (bx * bx + priml[6] * priml[6] + priml[7] * priml[7]);
  double pTR = primr[4] + 0.5 * (bx * bx + primr[6] * primr[6] + primr[7] * primr[7]);
  double slmul = sl - priml[1];
  double srmur = sr - primr[1];
  double rholul = priml[0] * priml[1];
  double rhorur = primr[0] * primr[1];
  double sM = (srmur * rhorur - slmul * rholul - pTR + pTL) / (srmur * primr[0] - slmul * priml[0]);
  double srmsM = sr - sM;
  double slmsM = sl - sM;
  double rhostl = priml[0] * slmul / slmsM;
  double rhostr = primr[0] * srmur / srmsM;
  double sstl = sM - std::fabs(bx) / std::sqrt(rhostl);
  double sstr = sM + std::fabs(bx) / std::sqrt(rhostr);
  double pst = (srmur * primr[0] * pTL - slmul * priml[0] * pTR +
                priml[0] * primr[0] * srmur * slmul * (primr[1] - priml[1])) /
               (srmur * primr[0] - slmul * priml[0]);
  double vstl = 0, wstl = 0, bystl = 0, bzstl = 0, vstr = 0, wstr = 0, bystr = 0, bzstr = 0;
  double el, er, denl, denr, sMmul, sMmur, vdotbl, vstdotbstl, estl, vdotbr, vstdotbstr, estr;

  if (sstl >= 0) {  // UL*
    el = 0.5 * priml[0] * (priml[1] * priml[1] + priml[2] * priml[2] + priml[3] * priml[3]) + cv * priml[4] +
         0.5 * (bx * bx + priml[6] * priml[6] + priml[7] * priml[7]);
    sMmul = sM - priml[1];
    denl = priml[0] * slmul * slmsM - bx * bx;
    if (denl == 0) {
      vstl = priml[2]; wstl = priml[3]; bystl = 0.; bzstl = 0.;
    } else {
      vstl = priml[2] - bx * priml[6] * sMmul / denl;
      wstl = priml[3] - bx * priml[7] * sMmul / denl;
      bystl = priml[6] * (priml[0] * (slmul * slmul) - bx * bx) / denl;
      bzstl = priml[7] * (priml[0] * (slmul * slmul) - bx * bx) / denl;
    }
    vdotbl = priml[1] * bx + priml[2] * priml[6] + priml[3] * priml[7];
    vstdotbstl = sM * bx + vstl * bystl + wstl * bzstl;
    estl = (slmul * el - pTL * priml[1] + pst * sM + bx * (vdotbl - vstdotbstl)) / slmsM;
    ff[0] = rhostl * sM;
    ff[1] = rhostl * (sM * sM) + pst - bx * bx;
    ff[2] = rhostl * sM * vstl - bx * bystl;
    ff[3] = rhostl * sM * wstl - bx * bzstl;
    ff[4] = sM * (estl + pst) - bx * (vstdotbstl);
    ff[5] = 0.;
    ff[6] = bystl * sM - bx * vstl;
    ff[7] = bzstl * sM - bx * wstl;
    return;
  }
  if (sstr <= 0) {  // UR*
    er = 0.5 * primr[0] * (primr[1] * primr[1] + primr[2] * primr[2] + primr[3] * primr[3]) + cv * primr[4] +
         0.5 * (bx * bx + primr[6] * primr[6] + primr[7] * primr[7]);
    sMmur = sM - primr[1];
    denr = primr[0] * srmur * srmsM - bx * bx;
    if (denr == 0) {
      vstl = priml[2]; wstl = priml[3]; bystl = 0.; bzstl = 0.;
    } else {
      vstr = primr[2] - bx * primr[6] * sMmur / denr;
      wstr = primr[3] - bx * primr[7] * sMmur / denr;
      bystr = primr[6] * (primr[0] * (srmur * srmur) - bx * bx) / denr;
      bzstr = primr[7] * (primr[0] * (srmur * srmur) - bx * bx) / denr;
    }
    vdotbr = primr[1] * bx + primr[2] * primr[6] + primr[3] * primr[7];
    vstdotbstr = sM * bx + vstr * bystr + wstr * bzstr;
    estr = (srmur * er - pTR * primr[1] + pst * sM + bx * (vdotbr - vstdotbstr)) / srmsM;
    ff[0] = rhostr * sM;
    ff[1] = rhostr * (sM * sM) + pst - bx * bx;
    ff[2] = rhostr * sM * vstr - bx * bystr;
    ff[3] = rhostr * sM * wstr - bx * bzstr;
    ff[4] = sM * (estr + pst) - bx * (vstdotbstr);
    ff[5] = 0.;
    ff[6] = bystr * sM - bx * vstr;
    ff[7] = bzstr * sM - bx * wstr;
    return;
  }
  sMmul = sM - priml[1];
  sMmur = sM - primr[1];
  denl = priml[0] * slmul * slmsM - bx * bx;
  denr = primr[0] * srmur * srmsM - bx * bx;
  if (denl == 0) {
    vstl = priml[2]; wstl = priml[3]; bystl = 0.; bzstl = 0.;
  } else {
    vstl = priml[2] - bx * priml[6] * sMmul / denl;
    wstl = priml[3] - bx * priml[7] * sMmul / denl;
    bystl = priml[6] * (priml[0] * (slmul * slmul) - bx * bx) / denl;
    bzstl = priml[7] * (priml[0] * (slmul * slmul) - bx * bx) / denl;
  }
  if (denr == 0) {
    vstr = primr[2]; wstr = primr[3]; bystr = 0.; bzstr = 0.;
  } else {
    vstr = primr[2] - bx * primr[6] * sMmur / denr;
    wstr = primr[3] - bx * primr[7] * sMmur / denr;
    bystr = primr[6] * (primr[0] * (srmur * srmur) - bx * bx) / denr;
    bzstr = primr[7] * (primr[0] * (srmur * srmur) - bx * bx) / denr;
  }
  double dd = std::sqrt(rhostl) + std::sqrt(rhostr);
  double vstst = (std::sqrt(rhostl) * vstl + std::sqrt(rhostr) * vstr + (bystr - bystl) * signBx) / dd;
  double wstst = (std::sqrt(rhostl) * wstl + std::sqrt(rhostr) * wstr + (bzstr - bzstl) * signBx) / dd;
  double bystst =
      (std::sqrt(rhostl) * bystr + std::sqrt(rhostr) * bystl + std::sqrt(rhostl * rhostr) * (vstr - vstl) * signBx) / dd;
  double bzstst =
      (std::sqrt(rhostl) * bzstr + std::sqrt(rhostr) * bzstl + std::sqrt(rhostl * rhostr) * (wstr - wstl) * signBx) / dd;
  double vststdotbstst = sM * bx + vstst * bystst + wstst * bzstst;
  if (sM >= 0) {  // UL**
    el = 0.5 * priml[0] * (priml[1] * priml[1] + priml[2] * priml[2] + priml[3] * priml[3]) + cv * priml[4] +
         0.5 * (bx * bx + priml[6] * priml[6] + priml[7] * priml[7]);
    vdotbl = priml[1] * bx + priml[2] * priml[6] + priml[3] * priml[7];
    vstdotbstl = sM * bx + vstl * bystl + wstl * bzstl;
    estl = (slmul * el - pTL * priml[1] + pst * sM + bx * (vdotbl - vstdotbstl)) / slmsM;
    double eststl = estl - std::sqrt(rhostl) * (vstdotbstl - vststdotbstst) * signBx;
    ff[0] = rhostl * sM;
    ff[1] = rhostl * (sM * sM) + pst - bx * bx;
    ff[2] = rhostl * sM * vstst - bx * bystst;
    ff[3] = rhostl * sM * wstst - bx * bzstst;
    ff[4] = sM * (eststl + pst) - bx * (vststdotbstst);
    ff[5] = 0.;
    ff[6] = bystst * sM - bx * vstst;
    ff[7] = bzstst * sM - bx * wstst;
    return;
  }
  if (sM <= 0) {  // UR**
    er = 0.5 * primr[0] * (primr[1] * primr[1] + primr[2] * primr[2] + primr[3] * primr[3]) + cv * primr[4] +
         0.5 * (bx * bx + primr[6] * primr[6] + primr[7] * primr[7]);
    vdotbr = primr[1] * bx + primr[2] * primr[6] + primr[3] * primr[7];
    vstdotbstr = sM * bx + vstr * bystr + wstr * bzstr;
    estr = (srmur * er - pTR * primr[1] + pst * sM + bx * (vdotbr - vstdotbstr)) / srmsM;
    double eststr = estr + std::sqrt(rhostr) * (vstdotbstr - vststdotbstst) * signBx;
    ff[0] = rhostr * sM;
    ff[1] = rhostr * (sM * sM) + pst - bx * bx;
    ff[2] = rhostr * sM * vstst - bx * bystst;
    ff[3] = rhostr * sM * wstst - bx * bzstst;
    ff[4] = sM * (eststr + pst) - bx * (vststdotbstst);
    ff[5] = 0.;
    ff[6] = bystst * sM - bx * vstst;
    ff[7] = bzstst * sM - bx * wstst;
    return;
  }
}

void riemann(const Ctx& c, const double* pl, const double* pr, double* ff) {
  switch (c.cfg.solver_type) {
    case WX_SOLVER_HLL1:
    case WX_SOLVER_HLL: primfhll(c, pl, pr, ff); break;
    case WX_SOLVER_HLLC: primfhllc(c, pl, pr, ff); break;
    case WX_SOLVER_HLLE: primfhlle(c, pl, pr, ff); break;
    case WX_SOLVER_HLLD: primfhlld(c, pl, pr, ff); break;
  }
}

// validCell (amr.f90:1658-1687)
bool validCell(int i, int j, int k) {
  const int lo = 1 - NGH, hi = NC + NGH;
  if (i < lo || i > hi || j < lo || j > hi || k < lo || k > hi) return false;
  int counter = 0;
  if (i < 1 || i > NC) ++counter;
  if (j < 1 || j > NC) ++counter;
  if (k < 1 || k > NC) ++counter;
  return counter <= 1;
}

struct Fluxes {
  std::vector<double> FC, GC, HC;  // (neq, 20^3), same ghost ranges as U
  explicit Fluxes(int neq) : FC((size_t)neq * NCELL, 0.0), GC((size_t)neq * NCELL, 0.0), HC((size_t)neq * NCELL, 0.0) {}
};

// HLLfluxes / HLLCfluxes / HLLEfluxes / HLLDfluxes (hll.f90:52-167,
// hllc.f90:55-201, hlle.f90:54-158, hlld.f90:54-158).  HLL and HLLC loop
// i,j,k over 0..16 with validCell; HLLE and HLLD compute all 17^3 positions.
void blockFluxes(const Ctx& c, int nb, int order, Fluxes& F) {
  const int neq = c.neq, lim = c.cfg.limiter_type;
  const bool useValid = (c.cfg.solver_type == WX_SOLVER_HLL || c.cfg.solver_type == WX_SOLVER_HLL1 ||
                         c.cfg.solver_type == WX_SOLVER_HLLC);
  double pll[MAXEQ], pl[MAXEQ], pr[MAXEQ], prr[MAXEQ], ff[MAXEQ];
  for (int e = 0; e < neq; ++e) ff[e] = 0.0;
  auto P = [&](int e, int i, int j, int k) { return c.u(c.PRIM, nb, e)[cidx(i, j, k)]; };
  auto put = [&](std::vector<double>& A, int i, int j, int k) {
    for (int e = 0; e < neq; ++e) A[(size_t)e * NCELL + cidx(i, j, k)] = ff[e];
  };
  for (int i = 0; i <= NC; ++i)
    for (int j = 0; j <= NC; ++j)
      for (int k = 0; k <= NC; ++k) {
        if (useValid && !validCell(i, j, k)) continue;
        if (order == 1) {
          for (int e = 0; e < neq; ++e) { pl[e] = P(e, i, j, k); pr[e] = P(e, i + 1, j, k); }
          riemann(c, pl, pr, ff);
          put(F.FC, i, j, k);
          for (int e = 0; e < neq; ++e) { pl[e] = P(e, i, j, k); pr[e] = P(e, i, j + 1, k); }
          swapxy(c, pl); swapxy(c, pr);
          riemann(c, pl, pr, ff);
          swapxy(c, ff);
          put(F.GC, i, j, k);
          for (int e = 0; e < neq; ++e) { pl[e] = P(e, i, j, k); pr[e] = P(e, i, j, k + 1); }
          swapxz(c, pl); swapxz(c, pr);
          riemann(c, pl, pr, ff);
          swapxz(c, ff);
          put(F.HC, i, j, k);
        } else {
          for (int e = 0; e < neq; ++e) {
            pll[e] = P(e, i - 1, j, k); pl[e] = P(e, i, j, k); pr[e] = P(e, i + 1, j, k); prr[e] = P(e, i + 2, j, k);
          }
          limiter(pll, pl, pr, prr, lim, neq);
          riemann(c, pl, pr, ff);
          put(F.FC, i, j, k);
          for (int e = 0; e < neq; ++e) {
            pll[e] = P(e, i, j - 1, k); pl[e] = P(e, i, j, k); pr[e] = P(e, i, j + 1, k); prr[e] = P(e, i, j + 2, k);
          }
          swapxy(c, pll); swapxy(c, pl); swapxy(c, pr); swapxy(c, prr);
          limiter(pll, pl, pr, prr, lim, neq);
          riemann(c, pl, pr, ff);
          swapxy(c, ff);
          put(F.GC, i, j, k);
          for (int e = 0; e < neq; ++e) {
            pll[e] = P(e, i, j, k - 1); pl[e] = P(e, i, j, k); pr[e] = P(e, i, j, k + 1); prr[e] = P(e, i, j, k + 2);
          }
          swapxz(c, pll); swapxz(c, pl); swapxz(c, pr); swapxz(c, prr);
          limiter(pll, pl, pr, prr, lim, neq);
          riemann(c, pl, pr, ff);
          swapxz(c, ff);
          put(F.HC, i, j, k);
        }
      }
}

// sources.f90:38-133 (Powell 8-wave; user source terms are not supported)
void source_function(const Ctx& c, int nb, int lev, int i, int j, int k, double* s) {
  for (int e = 0; e < c.neq; ++e) s[e] = 0.;
  if (c.cfg.bfield && c.cfg.eight_wave) {
    auto P = [&](int e, int ii, int jj, int kk) { return c.u(c.PRIM, nb, e)[cidx(ii, jj, kk)]; };
    double divB = (P(5, i + 1, j, k) - P(5, i - 1, j, k)) / (2. * c.dx[lev]) +
                  (P(6, i, j + 1, k) - P(6, i, j - 1, k)) / (2. * c.dy[lev]) +
                  (P(7, i, j, k + 1) - P(7, i, j, k - 1)) / (2. * c.dz[lev]);
    double pp[MAXEQ];
    for (int e = 0; e < c.neq; ++e) pp[e] = P(e, i, j, k);
    s[1] = s[1] - divB * pp[5];
    s[2] = s[2] - divB * pp[6];
    s[3] = s[3] - divB * pp[7];
    s[4] = s[4] - divB * (pp[1] * pp[5] + pp[2] * pp[6] + pp[3] * pp[7]);
    s[5] = s[5] - divB * pp[1];
    s[6] = s[6] - divB * pp[2];
    s[7] = s[7] - divB * pp[3];
  }
}

// flux_cd_update (brio-wu/flux_cd.f90:52-86) for every physical cell of a
// block.  The reference declares efield(3,0:n+1,0:n+1,0:n+1) (flux_cd.f90:37)
// but never fills it and never calls flux_cd_update; the restatement fills
// efield with the field-interpolated electric field E = -v x B of the
// primitives the fluxes were computed from (Toth 2000, J. Comput. Phys. 161,
// 605, field-CD scheme).  As in flux_cd_update, no source term is added.
void flux_cd_update(Ctx& c, int nb, double dtdx, double dtdy, double dtdz, const Fluxes& F) {
  constexpr int NE = NC + 2;
  std::vector<double> ef(3 * NE * NE * NE);
  auto E = [&](int d, int i, int j, int k) -> double& { return ef[((size_t)(d * NE + k) * NE + j) * NE + i]; };
  auto P = [&](int e, int i, int j, int k) { return c.u(c.PRIM, nb, e)[cidx(i, j, k)]; };
  for (int k = 0; k <= NC + 1; ++k)
    for (int j = 0; j <= NC + 1; ++j)
      for (int i = 0; i <= NC + 1; ++i) {
        const double v1 = P(1, i, j, k), v2 = P(2, i, j, k), v3 = P(3, i, j, k);
        const double b1 = P(5, i, j, k), b2 = P(6, i, j, k), b3 = P(7, i, j, k);
        E(0, i, j, k) = v3 * b2 - v2 * b3;
        E(1, i, j, k) = v1 * b3 - v3 * b1;
        E(2, i, j, k) = v2 * b1 - v1 * b2;
      }
  for (int i = 1; i <= NC; ++i)
    for (int j = 1; j <= NC; ++j)
      for (int k = 1; k <= NC; ++k) {
        for (int e = 0; e < c.neq; ++e) {
          if (e >= 5 && e <= 7) continue;
          const double* fc = F.FC.data() + (size_t)e * NCELL;
          const double* gc = F.GC.data() + (size_t)e * NCELL;
          const double* hc = F.HC.data() + (size_t)e * NCELL;
          c.u(c.UP, nb, e)[cidx(i, j, k)] = c.u(c.U, nb, e)[cidx(i, j, k)] -
                                            dtdx * (fc[cidx(i, j, k)] - fc[cidx(i - 1, j, k)]) -
                                            dtdy * (gc[cidx(i, j, k)] - gc[cidx(i, j - 1, k)]) -
                                            dtdz * (hc[cidx(i, j, k)] - hc[cidx(i, j, k - 1)]);
        }
        auto U = [&](int e) { return c.u(c.U, nb, e)[cidx(i, j, k)]; };
        c.u(c.UP, nb, 5)[cidx(i, j, k)] = U(5) - 0.5 * dtdy * (E(2, i, j + 1, k) - E(2, i, j - 1, k)) -
                                          0.5 * dtdz * (-E(1, i, j, k + 1) + E(1, i, j, k - 1));
        c.u(c.UP, nb, 6)[cidx(i, j, k)] = U(6) - 0.5 * dtdx * (-E(2, i + 1, j, k) + E(2, i - 1, j, k)) -
                                          0.5 * dtdz * (E(0, i, j, k + 1) - E(0, i, j, k - 1));
        c.u(c.UP, nb, 7)[cidx(i, j, k)] = U(7) - 0.5 * dtdx * (E(1, i + 1, j, k) - E(1, i - 1, j, k)) -
                                          0.5 * dtdy * (-E(0, i, j + 1, k) + E(0, i, j - 1, k));
      }
}

// upwindStep (godunov.f90:199-277); with enable_flux_cd the update is
// flux_cd_update's
void upwindStep(Ctx& c, int nb, double dtp, const Fluxes& F) {
  int lev = meshlevel(c, c.localBlocks[nb]);
  double dtdx = dtp / c.dx[lev], dtdy = dtp / c.dy[lev], dtdz = dtp / c.dz[lev];
  if (c.cfg.enable_flux_cd) {
    flux_cd_update(c, nb, dtdx, dtdy, dtdz, F);
    return;
  }
  const bool src = c.cfg.eight_wave || c.cfg.user_source_terms;
  double s[MAXEQ];
  for (int i = 1; i <= NC; ++i)
    for (int j = 1; j <= NC; ++j)
      for (int k = 1; k <= NC; ++k) {
        if (src) source_function(c, nb, lev, i, j, k, s);
        for (int e = 0; e < c.neq; ++e) {
          const double* fc = F.FC.data() + (size_t)e * NCELL;
          const double* gc = F.GC.data() + (size_t)e * NCELL;
          const double* hc = F.HC.data() + (size_t)e * NCELL;
          double v = c.u(c.U, nb, e)[cidx(i, j, k)] + dtdx * (fc[cidx(i - 1, j, k)] - fc[cidx(i, j, k)]) +
                     dtdy * (gc[cidx(i, j - 1, k)] - gc[cidx(i, j, k)]) +
                     dtdz * (hc[cidx(i, j, k - 1)] - hc[cidx(i, j, k)]);
          if (src) v = v + dtp * s[e];
          c.u(c.UP, nb, e)[cidx(i, j, k)] = v;
        }
      }
}

// ---------------------------------------------------------------------------
// userBoundary hook: imposeSphericalWind (winds.f90:123-240), all cells of
// every block, after the standard ghost fill.  The reference leaves the
// passive scalar of primit undefined; it is set here to y0*dens/d_sc
// (neutral density of a wind with neutral fraction y0).
void userBoundary(Ctx& c, std::vector<double>& uv) {
  if (c.winds.empty()) return;
  const double d_sc = c.cfg.d_sc, v_sc = c.cfg.v_sc, l_sc = c.cfg.l_sc;
#pragma omp parallel for schedule(dynamic) num_threads(c.nthreads)
  for (int nb = 0; nb < c.nbMax; ++nb) {
    int bID = c.localBlocks[nb];
    if (bID == -1) continue;
    double primit[MAXEQ], fv[MAXEQ];
    for (const Wind& w : c.winds)
      for (int i = 1 - NGH; i <= NC + NGH; ++i)
        for (int j = 1 - NGH; j <= NC + NGH; ++j)
          for (int k = 1 - NGH; k <= NC + NGH; ++k) {
            double x, y, z;
            cellPos(c, bID, i, j, k, x, y, z);
            x = x * l_sc; y = y * l_sc; z = z * l_sc;
            double dist = std::sqrt((x - w.xc) * (x - w.xc) + (y - w.yc) * (y - w.yc) + (z - w.zc) * (z - w.zc));
            if (dist < w.radius) {
              double dens = w.mdot / w.vinf / dist / dist / (4.0 * PI);
              double vx = w.vinf * (x - w.xc) / dist + w.vx;
              double vy = w.vinf * (y - w.yc) / dist + w.vy;
              double vz = w.vinf * (z - w.zc) / dist + w.vz;
              double pres = dens / (w.mu * AMU) * KB * w.temp;
              for (int e = 0; e < c.neq; ++e) primit[e] = 0.0;
              primit[0] = dens / d_sc;
              primit[1] = vx / v_sc;
              primit[2] = vy / v_sc;
              primit[3] = vz / v_sc;
              primit[4] = pres / c.p_sc;
              if (c.cfg.npassive >= 1) primit[c.fp] = w.y0 * dens / d_sc;
              prim2flow(c, primit, fv);
              for (int e = 0; e < c.neq; ++e) c.u(uv, nb, e)[cidx(i, j, k)] = fv[e];
            }
          }
  }
}

// ---------------------------------------------------------------------------
// boundary / normalBoundary (boundary.f90:46-686), single process: every
// source block is local, so only the local-copy branches apply.

void layerLimits(int face, int depth, bool ghost, int& imin, int& imax, int& jmin, int& jmax, int& kmin,
                 int& kmax) {  // boundary.f90:700-764
  imin = 1; imax = NC; jmin = 1; jmax = NC; kmin = 1; kmax = NC;
  switch (face) {
    case WX_LEFT: imax = depth; break;
    case WX_RIGHT: imin = NC - depth + 1; break;
    case WX_FRONT: jmax = depth; break;
    case WX_BACK: jmin = NC - depth + 1; break;
    case WX_BOTTOM: kmax = depth; break;
    case WX_TOP: kmin = NC - depth + 1; break;
  }
  if (ghost) {
    switch (face) {
      case WX_LEFT: imin -= depth; imax -= depth; break;
      case WX_RIGHT: imin += depth; imax += depth; break;
      case WX_FRONT: jmin -= depth; jmax -= depth; break;
      case WX_BACK: jmin += depth; jmax += depth; break;
      case WX_BOTTOM: kmin -= depth; kmax -= depth; break;
      case WX_TOP: kmin += depth; kmax += depth; break;
    }
  }
}

int opposite(int d) {  // boundary.f90:857-884
  static const int o[7] = {0, WX_RIGHT, WX_LEFT, WX_BACK, WX_FRONT, WX_TOP, WX_BOTTOM};
  return o[d];
}

void normalBoundaryBlock(Ctx& c, int depth, std::vector<double>& uv, int direction, int destInd) {
  const int destID = c.localBlocks[destInd];
  const int neq = c.neq;
  int ntype, neighs[4];
  neighbors(c, destID, direction, ntype, neighs);
  int i1, i2, j1, j2, k1, k2, i3, i4, j3, j4, k3, k4;
  if (ntype == WX_NEIGH_SAME) {  // :329-368
    layerLimits(direction, depth, true, i1, i2, j1, j2, k1, k2);
    int srcInd = c.slotOf.at(neighs[0]);
    layerLimits(opposite(direction), depth, false, i3, i4, j3, j4, k3, k4);
    for (int e = 0; e < neq; ++e) {
      double* d = c.u(uv, destInd, e);
      const double* s = c.u(uv, srcInd, e);
      for (int k = k1; k <= k2; ++k)
        for (int j = j1; j <= j2; ++j)
          for (int i = i1; i <= i2; ++i) d[cidx(i, j, k)] = s[cidx(i - i1 + i3, j - j1 + j3, k - k1 + k3)];
    }
  }
  if (ntype == WX_NEIGH_COARSER) {  // :374-412
    layerLimits(direction, depth, true, i1, i2, j1, j2, k1, k2);
    int sx, sy, sz;
    siblingCoords(c, destID, sx, sy, sz);
    int srcInd = c.slotOf.at(neighs[0]);
    for (int e = 0; e < neq; ++e) {
      double* d = c.u(uv, destInd, e);
      const double* s = c.u(uv, srcInd, e);
      for (int i = i1; i <= i2; ++i)
        for (int j = j1; j <= j2; ++j)
          for (int k = k1; k <= k2; ++k) {
            int ip = (i + 1) / 2 + sx * NC / 2, jp = (j + 1) / 2 + sy * NC / 2, kp = (k + 1) / 2 + sz * NC / 2;
            switch (direction) {
              case WX_LEFT: ip = NC + (i + 1) / 2; break;
              case WX_RIGHT: ip = (i - NC + 1) / 2; break;
              case WX_FRONT: jp = NC + (j + 1) / 2; break;
              case WX_BACK: jp = (j - NC + 1) / 2; break;
              case WX_BOTTOM: kp = NC + (k + 1) / 2; break;
              case WX_TOP: kp = (k - NC + 1) / 2; break;
            }
            d[cidx(i, j, k)] = s[cidx(ip, jp, kp)];
          }
    }
  }
  if (ntype == WX_NEIGH_FINER) {  // :492-546
    layerLimits(direction, depth, true, i1, i2, j1, j2, k1, k2);
    for (int e = 0; e < neq; ++e) {
      double* d = c.u(uv, destInd, e);
      for (int k = k1; k <= k2; ++k)
        for (int j = j1; j <= j2; ++j)
          for (int i = i1; i <= i2; ++i) d[cidx(i, j, k)] = 0.0;
    }
    for (int b = 0; b < 4; ++b) {
      int srcID = neighs[b];
      int sx, sy, sz;
      siblingCoords(c, srcID, sx, sy, sz);
      layerLimits(opposite(direction), depth * 2, false, i3, i4, j3, j4, k3, k4);
      int srcInd = c.slotOf.at(srcID);
      for (int e = 0; e < neq; ++e) {
        double* d = c.u(uv, destInd, e);
        const double* s = c.u(uv, srcInd, e);
        for (int i = i3; i <= i4; ++i)
          for (int j = j3; j <= j4; ++j)
            for (int k = k3; k <= k4; ++k) {
              int ip = (i + 1) / 2 + sx * NC / 2, jp = (j + 1) / 2 + sy * NC / 2, kp = (k + 1) / 2 + sz * NC / 2;
              switch (direction) {
                case WX_LEFT: ip = (i - NC) / 2; break;
                case WX_RIGHT: ip = (i + 1) / 2 + NC; break;
                case WX_FRONT: jp = (j - NC) / 2; break;
                case WX_BACK: jp = (j + 1) / 2 + NC; break;
                case WX_BOTTOM: kp = (k - NC) / 2; break;
                case WX_TOP: kp = (k + 1) / 2 + NC; break;
              }
              d[cidx(ip, jp, kp)] = d[cidx(ip, jp, kp)] + s[cidx(i, j, k)] / 8.0;
            }
      }
    }
  }
  const int bc_type = c.cfg.bc[direction - 1];
  if (ntype == WX_NEIGH_BOUNDARY && bc_type != WX_BC_PERIODIC) {  // :594-673
    layerLimits(direction, depth, true, i1, i2, j1, j2, k1, k2);
    for (int i = i1; i <= i2; ++i)
      for (int j = j1; j <= j2; ++j)
        for (int k = k1; k <= k2; ++k) {
          int ip = i, jp = j, kp = k;
          if (bc_type == WX_BC_REFLECTIVE) {
            switch (direction) {
              case WX_LEFT: ip = 1 - i; break;
              case WX_RIGHT: ip = 2 * NC - i + 1; break;
              case WX_FRONT: jp = 1 - j; break;
              case WX_BACK: jp = 2 * NC - j + 1; break;
              case WX_BOTTOM: kp = 1 - k; break;
              case WX_TOP: kp = 2 * NC - k + 1; break;
            }
            for (int e = 0; e < neq; ++e) {
              double v = c.u(uv, destInd, e)[cidx(ip, jp, kp)];
              bool flip = ((direction == WX_LEFT || direction == WX_RIGHT) && e == 1) ||
                          ((direction == WX_FRONT || direction == WX_BACK) && e == 2) ||
                          ((direction == WX_BOTTOM || direction == WX_TOP) && e == 3);
              c.u(uv, destInd, e)[cidx(i, j, k)] = flip ? -1.0 * v : v;
            }
          } else if (bc_type == WX_BC_FREE_FLOW) {
            switch (direction) {
              case WX_LEFT: ip = 1; break;
              case WX_RIGHT: ip = 2 * NC - i + 1; break;
              case WX_FRONT: jp = 1; break;
              case WX_BACK: jp = 2 * NC - j + 1; break;
              case WX_BOTTOM: kp = 1; break;
              case WX_TOP: kp = 2 * NC - k + 1; break;
            }
            for (int e = 0; e < neq; ++e) c.u(uv, destInd, e)[cidx(i, j, k)] = c.u(uv, destInd, e)[cidx(ip, jp, kp)];
          }
        }
  }
}

void boundary(Ctx& c, int depth, std::vector<double>& uv) {  // boundary.f90:46-64
  for (int a = 1; a <= 6; ++a) {
#pragma omp parallel for schedule(dynamic) num_threads(c.nthreads)
    for (int nb = 0; nb < c.nbMax; ++nb)
      if (c.localBlocks[nb] != -1) normalBoundaryBlock(c, depth, uv, a, nb);
  }
  userBoundary(c, uv);
}

// ---------------------------------------------------------------------------
// godunov.f90, lax.f90, hydro_solver.f90

void Godunov(Ctx& c, int order) {  // godunov.f90:43-190
  double dtp = (order == 2) ? c.dt / 2.0 : c.dt;
  boundary(c, 1, c.U);
  calcPrimsAll(c, c.U, c.PRIM, CELLS_GHOST);
#pragma omp parallel num_threads(c.nthreads)
  {
    Fluxes F(c.neq);
#pragma omp for schedule(dynamic)
    for (int nb = 0; nb < c.nbMax; ++nb)
      if (c.localBlocks[nb] != -1) {
        blockFluxes(c, nb, 1, F);
        upwindStep(c, nb, dtp, F);
      }
  }
  if (order == 2) {
    boundary(c, 2, c.UP);
    calcPrimsAll(c, c.UP, c.PRIM, CELLS_ALL);
#pragma omp parallel num_threads(c.nthreads)
    {
      Fluxes F(c.neq);
#pragma omp for schedule(dynamic)
      for (int nb = 0; nb < c.nbMax; ++nb)
        if (c.localBlocks[nb] != -1) {
          blockFluxes(c, nb, 2, F);
          upwindStep(c, nb, c.dt, F);
        }
    }
  }
}

void LaxFriedrichs(Ctx& c) {  // lax.f90:39-99
  boundary(c, 1, c.U);
  calcPrimsAll(c, c.U, c.PRIM, CELLS_GHOST);
#pragma omp parallel num_threads(c.nthreads)
  {
    Fluxes F(c.neq);
    double pv[MAXEQ], f[MAXEQ];
#pragma omp for schedule(dynamic)
    for (int nb = 0; nb < c.nbMax; ++nb) {
      int bID = c.localBlocks[nb];
      if (bID == -1) continue;
      for (int i = 0; i <= NC + 1; ++i)
        for (int j = 0; j <= NC + 1; ++j)
          for (int k = 0; k <= NC + 1; ++k) {
            for (int e = 0; e < c.neq; ++e) pv[e] = c.u(c.PRIM, nb, e)[cidx(i, j, k)];
            prim2fluxes(c, pv, DIM_X, f);
            for (int e = 0; e < c.neq; ++e) F.FC[(size_t)e * NCELL + cidx(i, j, k)] = f[e];
            prim2fluxes(c, pv, DIM_Y, f);
            for (int e = 0; e < c.neq; ++e) F.GC[(size_t)e * NCELL + cidx(i, j, k)] = f[e];
            prim2fluxes(c, pv, DIM_Z, f);
            for (int e = 0; e < c.neq; ++e) F.HC[(size_t)e * NCELL + cidx(i, j, k)] = f[e];
          }
      int lev = meshlevel(c, bID);
      for (int i = 1; i <= NC; ++i)
        for (int j = 1; j <= NC; ++j)
          for (int k = 1; k <= NC; ++k)
            for (int e = 0; e < c.neq; ++e) {
              const double* u = c.u(c.U, nb, e);
              const double* fc = F.FC.data() + (size_t)e * NCELL;
              const double* gc = F.GC.data() + (size_t)e * NCELL;
              const double* hc = F.HC.data() + (size_t)e * NCELL;
              c.u(c.UP, nb, e)[cidx(i, j, k)] =
                  (u[cidx(i + 1, j, k)] + u[cidx(i - 1, j, k)] + u[cidx(i, j + 1, k)] + u[cidx(i, j - 1, k)] +
                   u[cidx(i, j, k + 1)] + u[cidx(i, j, k - 1)]) / 6.0 -
                  0.5 * c.dt / c.dx[lev] * (fc[cidx(i + 1, j, k)] - fc[cidx(i - 1, j, k)]) -
                  0.5 * c.dt / c.dy[lev] * (gc[cidx(i, j + 1, k)] - gc[cidx(i, j - 1, k)]) -
                  0.5 * c.dt / c.dz[lev] * (hc[cidx(i, j, k + 1)] - hc[cidx(i, j, k - 1)]);
            }
    }
  }
}

// getTimestep (hydro_solver.f90:129-211), single process.
double getTimestep(Ctx& c) {
  double dt_hydro = 1.0e30, dt_cool = 1.0e30;
#pragma omp parallel for schedule(dynamic) reduction(min : dt_hydro) num_threads(c.nthreads)
  for (int nb = 0; nb < c.nbMax; ++nb) {
    int bID = c.localBlocks[nb];
    if (bID == -1) continue;
    int ilev = meshlevel(c, bID);
    double pv[MAXEQ];
    for (int i = 1; i <= NC; ++i)
      for (int j = 1; j <= NC; ++j)
        for (int k = 1; k <= NC; ++k) {
          for (int e = 0; e < c.neq; ++e) pv[e] = c.u(c.PRIM, nb, e)[cidx(i, j, k)];
          if (c.cfg.mhd) {
            if (c.cfg.bfield) {
              double cfx, cfy, cfz;
              cfast(c, pv[4], pv[0], pv[5], pv[6], pv[7], cfx, cfy, cfz);
              dt_hydro = std::min(dt_hydro, c.dx[ilev] / (std::fabs(pv[1]) + cfx));
              dt_hydro = std::min(dt_hydro, c.dy[ilev] / (std::fabs(pv[2]) + cfy));
              dt_hydro = std::min(dt_hydro, c.dz[ilev] / (std::fabs(pv[3]) + cfz));
            }
          } else {
            double cs = sound(c, pv);
            dt_hydro = std::min(dt_hydro, c.dx[ilev] / (std::fabs(pv[1]) + cs));
            dt_hydro = std::min(dt_hydro, c.dy[ilev] / (std::fabs(pv[2]) + cs));
            dt_hydro = std::min(dt_hydro, c.dz[ilev] / (std::fabs(pv[3]) + cs));
          }
        }
  }
  double dt_loc;
  if (c.cfg.cooling_type == WX_COOL_NONE) dt_loc = dt_hydro * c.cfg.cfl;
  else dt_loc = std::min(dt_hydro, dt_cool) * c.cfg.cfl;
  if (c.it <= 10) dt_loc = std::pow(2., -(double)(11 - c.it)) * dt_loc;
  double dt_glob = dt_loc;
  double tnext = c.nextout * c.cfg.dtout / c.t_sc;
  if (c.time + dt_glob >= tnext) {
    dt_glob = tnext - c.time;
    c.dumpout = true;
  }
  return dt_glob;
}

void doViscousStep(Ctx& c) {  // hydro_solver.f90:217-250
  c.time = c.time + c.dt;
  const double eta = c.cfg.visc_eta;
#pragma omp parallel for schedule(dynamic) num_threads(c.nthreads)
  for (int nb = 0; nb < c.nbMax; ++nb) {
    if (c.localBlocks[nb] == -1) continue;
    for (int e = 0; e < c.neq; ++e) {
      const double* up = c.u(c.UP, nb, e);
      double* u = c.u(c.U, nb, e);
      for (int k = 1; k <= NC; ++k)
        for (int j = 1; j <= NC; ++j)
          for (int i = 1; i <= NC; ++i)
            u[cidx(i, j, k)] = up[cidx(i, j, k)] +
                               eta * (+up[cidx(i + 1, j, k)] + up[cidx(i - 1, j, k)] + up[cidx(i, j + 1, k)] +
                                      up[cidx(i, j - 1, k)] + up[cidx(i, j, k + 1)] + up[cidx(i, j, k - 1)] -
                                      6.0 * up[cidx(i, j, k)]);
    }
  }
}

void hydroSolver(Ctx& c) {  // hydro_solver.f90:39-121
  double dt_new = getTimestep(c);
  c.dt = dt_new;
  switch (c.cfg.solver_type) {
    case WX_SOLVER_LAX: LaxFriedrichs(c); break;
    case WX_SOLVER_HLL1: Godunov(c, 1); break;
    default: Godunov(c, 2); break;
  }
  doViscousStep(c);
}

// ---------------------------------------------------------------------------
// hrate.f90

double alpha_rec(double T) { return 2.55e-13 * std::pow(1.e4 / T, 0.79); }         // hrate.f90:51-60
double colf(double T) { return 5.83e-11 * std::sqrt(T) * std::exp(-157828. / T); }  // hrate.f90:66-75

void solve_h_rate(Ctx& c, int nb, double dt) {  // hrate.f90:82-142
  const int fp = c.fp;
  const double mu0 = c.cfg.mu0, xi = 1.e-4;
  double pv[MAXEQ];
  for (int k = 1; k <= NC; ++k)
    for (int j = 1; j <= NC; ++j)
      for (int i = 1; i <= NC; ++i) {
        int id = cidx(i, j, k);
        for (int e = 0; e < c.neq; ++e) pv[e] = c.u(c.PRIM, nb, e)[id];
        double T = calcTemp(c, pv);
        double col = colf(T);
        double rec = alpha_rec(T);
        double dh = pv[0] / mu0;
        double y0 = pv[fp] / dh;
        double fpn = 0.0;
        double a = rec + col;
        double b = -((2.0 + xi) * rec + (1.0 + xi) * col + fpn);
        double cc = (1.0 + xi) * rec;
        double d = std::sqrt(b * b - 4.0 * a * cc);
        double g0 = (2.0 * a * y0 + b + d) / (2.0 * a * y0 + b - d);
        double e = std::exp(-d * dh * dt);
        double y1 = (-b - d * (1.0 + g0 * e) / (1.0 - g0 * e)) / (2.0 * a);
        y1 = std::min(y1, 1.0 - xi);
        y1 = std::max(y1, 0.0);
        c.u(c.PRIM, nb, fp)[id] = pv[0] * y1 / mu0;
        if (c.cfg.cooling_type != WX_COOL_H) c.u(c.U, nb, fp)[id] = c.u(c.PRIM, nb, fp)[id];
      }
}

void updateNeutralFraction(Ctx& c) {  // hrate.f90:12-45
  double dts = c.dt * c.t_sc;
#pragma omp parallel for schedule(dynamic) num_threads(c.nthreads)
  for (int nb = 0; nb < c.nbMax; ++nb)
    if (c.localBlocks[nb] != -1) solve_h_rate(c, nb, dts);
}

// ---------------------------------------------------------------------------
// cooling.f90, cooling_h.f90

double find_coef(const Ctx& c, double logT) {  // cooling.f90:378-419
  if (logT < c.cool_Tmin) return 0.0;
  if (logT >= c.cool_Tmax) return std::pow(10., c.cooltable2[c.nptsT - 1] + 0.5 * (logT - c.cool_Tmax));
  for (int i = 2; i <= c.nptsT; ++i) {
    if (c.cooltable1[i - 1] > logT) {
      double T0 = c.cooltable1[i - 2], C0 = c.cooltable2[i - 2];
      double T1 = c.cooltable1[i - 1], C1 = c.cooltable2[i - 1];
      return std::pow(10., (C1 - C0) / (T1 - T0) * (logT - T0) + C0);
    }
  }
  return 0.0;  // NaN logT: the reference leaves coef unset
}

double find_coef_metal(const Ctx& c, double logT, double Z);

double apply_cooling(Ctx& c, int nb) {  // cooling.f90:285-371 (COOL_TABLE, COOL_TABLE_METAL)
  const double T_floor = 10.0;
  const wx_config& f = c.cfg;
  double maxloss = 0.0;
  double pv[MAXEQ];
  for (int i = 1; i <= NC; ++i)
    for (int j = 1; j <= NC; ++j)
      for (int k = 1; k <= NC; ++k) {
        int id = cidx(i, j, k);
        for (int e = 0; e < c.neq; ++e) pv[e] = c.u(c.PRIM, nb, e)[id];
        double temp = calcTemp(c, pv);
        double logT = std::log10(temp);
        double metal = 0.0;
        // metalpas = neqhydro + neqmhd + min(npassive, 1) (parameters.f90:318)
        const int metalpas = 5 + (c.cfg.bfield ? 3 : 0) + std::min(c.cfg.npassive, 1) - 1;
        if (f.cooling_type == WX_COOL_TABLE_METAL) metal = std::fabs(pv[metalpas] / pv[0]);
        if (logT >= c.cool_Tmin) {
          double ETH = c.cv * pv[4];
          double vel2 = pv[1] * pv[1] + pv[2] * pv[2] + pv[3] * pv[3];
          double EK = 0.5 * pv[0] * vel2;
          double aloss = f.cooling_type == WX_COOL_TABLE_METAL ? find_coef_metal(c, logT, metal) : find_coef(c, logT);
          double numdens = pv[0] * f.d_sc / (f.mui * AMU);
          double ce = aloss * (numdens * numdens) / (ETH * c.e_sc);
          double cool_factor = std::exp(-ce * (c.dt * c.t_sc));
          double frac_loss = 1.0 - cool_factor;
          maxloss = std::max(maxloss, frac_loss);
          if (cool_factor < 1.0 - f.cooling_limit) cool_factor = 1.0 - f.cooling_limit;
          double new_temp = temp * cool_factor;
          if (new_temp < T_floor) cool_factor = T_floor / temp;
          c.u(c.PRIM, nb, 4)[id] = pv[4] * cool_factor;
          ETH = c.cv * c.u(c.PRIM, nb, 4)[id];
          c.u(c.U, nb, 4)[id] = EK + ETH;
        }
      }
  return maxloss;
}

// cooltable(i, j) of loadcooldata_metal, 1-based (cooling.f90:193-265)
inline double ctm(const Ctx& c, int i, int j) { return c.ctab_metal[(size_t)(i - 1) * (c.nptsZ + 1) + (j - 1)]; }

double find_coef_metal(const Ctx& c, double logT, double Z) {  // cooling.f90:435-519
  if (logT < c.cool_Tmin) return 0.0;
  int Tlo = 2, Thi = c.nptsT + 1;
  double T0 = 0.0, T1 = 0.0;
  if (logT <= c.cool_Tmax) {  // binary search
    while (Thi - Tlo > 1) {
      int Tmid = (Tlo + Thi) / 2;
      if (logT <= ctm(c, Tmid, 1)) Thi = Tmid;
      else Tlo = Tmid;
    }
    T0 = ctm(c, Tlo, 1);
    T1 = ctm(c, Thi, 1);
  }
  int Zlo, Zhi;
  if (Z < c.cool_Zmin) { Zlo = 2; Zhi = 3; }
  else if (Z > c.cool_Zmax) { Zlo = c.nptsZ; Zhi = c.nptsZ + 1; }
  else {
    Zlo = 2; Zhi = c.nptsZ + 1;
    while (Zhi - Zlo > 1) {
      int Zmid = (Zlo + Zhi) / 2;
      if (Z <= ctm(c, 1, Zmid)) Zhi = Zmid;
      else Zlo = Zmid;
    }
  }
  const double Z0 = ctm(c, 1, Zlo), Z1 = ctm(c, 1, Zhi);
  if (logT >= c.cool_Tmax) {
    // row nptsT, one below the last data row, as the reference reads it
    const double C0 = ctm(c, c.nptsT, Zlo) + 0.5 * (logT - c.cool_Tmax);
    const double C1 = ctm(c, c.nptsT, Zhi) + 0.5 * (logT - c.cool_Tmax);
    return std::pow(10., (C1 - C0) / (Z1 - Z0) * (Z - Z0) + C0);
  }
  const double TC = (logT - T0) / (T1 - T0);
  const double ZC = (Z - Z0) / (Z1 - Z0);
  double coef = (1.0 - TC) * (1.0 - ZC) * ctm(c, Tlo, Zlo) + (1.0 - TC) * ZC * ctm(c, Tlo, Zhi) +
                TC * (1.0 - ZC) * ctm(c, Thi, Zlo) + TC * ZC * ctm(c, Thi, Zhi);
  return std::pow(10., coef);
}

double get_lambda(const Ctx& c, double T) {  // cooling_schure.f90:102-128
  const double deltaTemp = 0.04, logTmin = 1.0;
  if (T > 1e8) return 0.21e-26 * std::sqrt(T);
  const int if1 = (int)((std::log10(T) - logTmin) / deltaTemp) + 1;
  if (if1 < 1) return c.schureL[0];
  const double T0 = c.schureT[if1 - 1], c0 = c.schureL[if1 - 1];
  const double T1 = c.schureT[if1], c1 = c.schureL[if1];
  return (c1 - c0) * (T - T0) / (T1 - T0) + c0;
}

double apply_cooling_schure(Ctx& c, int nb) {  // cooling_schure.f90:134-228
  const double Tmin = 10.0;
  const wx_config& f = c.cfg;
  const double dt_seconds = c.dt * c.t_sc;
  double maxloss = 0.0;
  double pv[MAXEQ];
  for (int i = 1; i <= NC; ++i)
    for (int j = 1; j <= NC; ++j)
      for (int k = 1; k <= NC; ++k) {
        int id = cidx(i, j, k);
        for (int e = 0; e < c.neq; ++e) pv[e] = c.u(c.PRIM, nb, e)[id];
        double T = calcTemp(c, pv);
        if (T > Tmin) {
          double Lambda0 = get_lambda(c, T);
          double gain = 0.0;
          double dens = pv[0] / f.mu0;
          double emtauC = std::exp(-2.0 * dt_seconds * dens * Lambda0 / (3.0 * KB * T));
          double cool_factor = (gain / (dens * dens * Lambda0)) * (1.0 - emtauC) + emtauC;
          double frac_loss = 1.0 - cool_factor;
          maxloss = std::max(maxloss, frac_loss);
          if (cool_factor < 1.0 - f.cooling_limit) cool_factor = 1.0 - f.cooling_limit;
          c.u(c.PRIM, nb, 4)[id] = pv[4] * cool_factor;
          const double p4 = c.u(c.PRIM, nb, 4)[id];
          c.u(c.U, nb, 4)[id] = c.cv * p4 + 0.5 * pv[0] * (pv[1] * pv[1] + pv[2] * pv[2] + pv[3] * pv[3]);
        }
      }
  return maxloss;
}

double betah(double T) {  // cooling_h.f90:42-53
  double a = 157890. / T;
  return 1.133e-24 / std::sqrt(a) * (-0.0713 + 0.5 * std::log(a) + 0.640 * std::pow(a, -0.33333));
}

double aloss_h(double x1, double /*x2*/, double den, double dH0, double Te0) {  // cooling_h.f90:73-145
  const double XION = 2.179e-11, XO = 1.e-3;
  const double C0 = 0.5732, C1 = 1.8288e-5, C2 = -1.15822e-10, C3 = 9.4288e-16;
  const double D0 = 0.5856, D1 = 1.55083e-5, D2 = -9.669e-12, D3 = 5.716e-19;
  const double ENK = 118409., EN = 1.634E-11;
  double Te = std::max(Te0, 10.);
  double dHp = (1. - x1) * den;
  double de = dHp + 1.E-4 * den;
  double dOI = XO * dH0;
  double dOII = XO * dHp;
  if (Te <= 1e4) return 1e-30;
  double omega = 0.0;
  if (Te <= 55000.) omega = C0 + Te * (C1 + Te * (C2 + Te * C3));
  if (Te >= 72000.) omega = D0 + Te * (D1 + Te * (D2 + Te * D3));
  if (Te > 55000. && Te < 72000.) {
    double omegaL = C0 + Te * (C1 + Te * (C2 + Te * C3));
    double omegaH = D0 + Te * (D1 + Te * (D2 + Te * D3));
    double frac = (Te - 55000.) / 17000.;
    omega = (1. - frac) * omegaL + frac * omegaH;
  }
  double qla = 8.6287E-6 / (2. * std::sqrt(Te)) * omega * std::exp(-ENK / Te);
  double ecoll = de * dH0 * qla * EN;
  ecoll = std::max(ecoll, 0.);
  double cion = 5.834E-11 * std::sqrt(Te) * std::exp(-1.579E5 / Te);
  double eion = de * dH0 * cion * XION;
  double erec = de * dHp * (betah(Te));
  erec = std::max(erec, 0.);
  double Tm = 1. / Te;
  double Tm2 = Tm * Tm;
  double eOI = de * dOI * std::pow(10., 1381465 * Tm2 - 12328.69 * Tm - 19.82621);
  double eOII = de * dOII * std::pow(10., -2061075. * Tm2 - 14596.24 * Tm - 19.01402);
  eOI = std::max(eOI, 0.);
  eOII = std::max(eOII, 0.);
  double betaf = 1.3 * 1.42E-27 * std::pow(Te, 0.5);
  double HIIcool = de * dHp * betaf;
  double equil = (1.0455E-18 / std::pow(Te, 0.63)) * (1. - std::exp(-std::pow(Te * 1.E-5, 1.63))) * de * den + HIIcool;
  double fr = 0.0;
  if (Te <= 44770.) fr = 0.;
  if (Te >= 54770.) fr = 1.;
  if (Te > 44770. && Te < 54770.) {
    double ex2 = std::exp(-2. * (Te - 49770.) / 500.);
    double th = (1. - ex2) / (1. + ex2);
    fr = 0.5 * (1. + th);
  }
  return ecoll + eion + (erec + 7.033 * (eOI + eOII)) * (1. - fr) + equil * fr;
}

double apply_cooling_h_neq(Ctx& c, int nb) {  // cooling_h.f90:154-252
  const double T_floor = 10.0, Tmin_cool = 1.e4;
  const wx_config& f = c.cfg;
  const int fp = c.fp;
  double maxloss = 0.0;
  double dt_seconds = c.dt * c.t_sc;
  double pv[MAXEQ];
  for (int i = 1; i <= NC; ++i)
    for (int j = 1; j <= NC; ++j)
      for (int k = 1; k <= NC; ++k) {
        int id = cidx(i, j, k);
        double dh = c.u(c.PRIM, nb, 0)[id] / f.mu0;
        double dh0 = c.u(c.PRIM, nb, fp)[id];
        double y0 = f.mu0 * c.u(c.U, nb, fp)[id] / c.u(c.U, nb, 0)[id];
        double y1 = f.mu0 * c.u(c.PRIM, nb, fp)[id] / c.u(c.PRIM, nb, 0)[id];
        c.u(c.U, nb, fp)[id] = c.u(c.PRIM, nb, fp)[id];
        for (int e = 0; e < c.neq; ++e) pv[e] = c.u(c.PRIM, nb, e)[id];
        double Temp = calcTemp(c, pv);
        if (Temp > Tmin_cool) {
          double L0 = aloss_h(y0, y1, dh, dh0, Temp);
          double Tprime = T_floor;
          double ce = (2.0 * L0) / (3.0 * KB * dh * Temp);
          double T1 = Tprime + (Temp - Tprime) * std::exp(-ce * dt_seconds);
          double cool_factor = T1 / Temp;
          double frac_loss = 1.0 - cool_factor;
          maxloss = std::max(maxloss, frac_loss);
          if (cool_factor < 1.0 - f.cooling_limit) cool_factor = 1.0 - f.cooling_limit;
          T1 = Temp * cool_factor;
          if (T1 < T_floor) cool_factor = T_floor / Temp;
          c.u(c.PRIM, nb, 4)[id] = pv[4] * cool_factor;
          double ETH = c.cv * c.u(c.PRIM, nb, 4)[id];
          double vel2 = pv[1] * pv[1] + pv[2] * pv[2] + pv[3] * pv[3];
          double EK = 0.5 * pv[0] * vel2;
          c.u(c.U, nb, 4)[id] = EK + ETH;
        }
      }
  return maxloss;
}

double cooling(Ctx& c) {  // cooling.f90:37-118
  double ml = 0.0;
  if (c.cfg.cooling_type == WX_COOL_NONE) return ml;
#pragma omp parallel for schedule(dynamic) reduction(max : ml) num_threads(c.nthreads)
  for (int nb = 0; nb < c.nbMax; ++nb) {
    if (c.localBlocks[nb] == -1) continue;
    double m = 0.0;
    const int ct = c.cfg.cooling_type;
    if (ct == WX_COOL_TABLE || ct == WX_COOL_TABLE_METAL) m = apply_cooling(c, nb);
    else if (ct == WX_COOL_SCHURE) m = apply_cooling_schure(c, nb);
    else if (ct == WX_COOL_H) m = apply_cooling_h_neq(c, nb);
    ml = std::max(ml, m);
  }
  c.maxloss = ml;
  return ml;
}

// ---------------------------------------------------------------------------
// amr.f90 data operations

int markByPhysical(const Ctx& c, int nb) {  // amr.f90:142-230
  int bID = c.localBlocks[nb];
  int ilev = meshlevel(c, bID);
  double maxgrad = 0.0;
  const double dxl = c.dx[ilev];
  auto P = [&](int e, int i, int j, int k) { return c.u(c.PRIM, nb, e)[cidx(i, j, k)]; };
  for (int i = 1; i <= NC; ++i)
    for (int j = 1; j <= NC; ++j)
      for (int k = 1; k <= NC; ++k) {
        for (int e : {4, 0}) {
          double gx = std::fabs(P(e, i + 1, j, k) - P(e, i - 1, j, k)) / P(e, i, j, k) / (2 * dxl);
          double gy = std::fabs(P(e, i, j + 1, k) - P(e, i, j - 1, k)) / P(e, i, j, k) / (2 * dxl);
          double gz = std::fabs(P(e, i, j, k + 1) - P(e, i, j, k - 1)) / P(e, i, j, k) / (2 * dxl);
          double grad = std::max(std::max(gx, gy), gz);
          maxgrad = std::max(maxgrad, grad);
          if (grad >= c.cfg.refine_thres) {
            if (ilev == c.cfg.maxlev) return WX_FLAG_NONE;
            return WX_FLAG_REFINE;
          }
        }
      }
  if (maxgrad <= c.cfg.coarse_thres && ilev > 1) return WX_FLAG_COARSE;
  return WX_FLAG_NONE;
}

// Registry helpers (utils.f90:78-172): linear find, put into the first
// empty slot, pop.
int find(const std::vector<int>& list, int element) {
  for (int nb = 0; nb < (int)list.size(); ++nb)
    if (list[nb] == element) return nb;
  return -1;
}
int put(std::vector<int>& list, int element) {
  int nb = find(list, -1);
  if (nb != -1) list[nb] = element;
  return nb;
}
int pop(std::vector<int>& list, int element) {
  int nb = find(list, element);
  if (nb != -1) list[nb] = -1;
  return nb;
}

// checkProximity (amr.f90:1109-1254) with globalBlocks = localBlocks (one
// process); refineFlags change while the sweep goes.
void checkProximity(const Ctx& c, std::vector<int>& refineFlags, int finestLev) {
  const std::vector<int>& globalBlocks = c.localBlocks;
  for (int level = finestLev; level >= 1; --level)
    for (int nb = 0; nb < c.nbMax; ++nb) {
      int bID = globalBlocks[nb];
      if (bID == -1 || bID < c.minID[level] || bID > c.maxID[level]) continue;
      int bflag = refineFlags[nb];
      if (bflag == WX_FLAG_REFINE) {
        for (int dir = 1; dir <= 6; ++dir) {
          int ntype, list[4];
          neighbors(c, bID, dir, ntype, list);
          if (ntype == WX_NEIGH_SAME) {
            int nb1 = find(globalBlocks, list[0]);
            if (refineFlags[nb1] == WX_FLAG_COARSE) refineFlags[nb1] = WX_FLAG_NONE;
          } else if (ntype == WX_NEIGH_COARSER) {
            int nb2 = find(globalBlocks, list[0]);
            if (refineFlags[nb2] != WX_FLAG_REFINE) refineFlags[nb2] = WX_FLAG_REFINE;
          }
        }
      }
      if (bflag == WX_FLAG_COARSE) {
        bool inhibited = false;
        for (int dir = 1; dir <= 6; ++dir) {
          int ntype, list[4];
          neighbors(c, bID, dir, ntype, list);
          if (ntype == WX_NEIGH_FINER) {
            int sib[8];
            siblings(c, list[0], sib);
            for (int i = 0; i < 8; ++i) {
              int nb1 = find(globalBlocks, sib[i]);
              if (nb1 != -1 && refineFlags[nb1] != WX_FLAG_COARSE) {
                refineFlags[nb] = WX_FLAG_NONE;
                inhibited = true;
                break;
              }
            }
          }
          if (inhibited) break;
        }
      }
    }
}

// refineBlock (amr.f90:284-384): children into the first empty slots, U and
// PRIM injected from the father, the father's slot freed.
int refineBlock(Ctx& c, int fatherID, int& nbLocal) {
  int fatherIndex = find(c.localBlocks, fatherID);
  if (fatherIndex == -1) return 5;  // ERROR_LOCAL_BID_NOT_FOUND
  if (meshlevel(c, fatherID) == c.cfg.maxlev) return WX_ERR_ALREADY_MAX_LEV;
  if (nbLocal + 8 > c.nbMax) return WX_ERR_INSUFICIENT_NBMAXPROC;
  int childList[8];
  children(c, fatherID, childList);
  for (int ch = 0; ch < 8; ++ch) {
    int childIndex = put(c.localBlocks, childList[ch]);
    if (childIndex == -1) return 8;  // ERROR_REGISTER_CHILD
    int sx, sy, sz;
    siblingCoords(c, childList[ch], sx, sy, sz);
    for (int i = 1; i <= NC; ++i)
      for (int j = 1; j <= NC; ++j)
        for (int k = 1; k <= NC; ++k) {
          int ip = (NC / 2) * sx + (i + 1) / 2, jp = (NC / 2) * sy + (j + 1) / 2, kp = (NC / 2) * sz + (k + 1) / 2;
          for (int e = 0; e < c.neq; ++e) {
            c.u(c.U, childIndex, e)[cidx(i, j, k)] = c.u(c.U, fatherIndex, e)[cidx(ip, jp, kp)];
            c.u(c.PRIM, childIndex, e)[cidx(i, j, k)] = c.u(c.PRIM, fatherIndex, e)[cidx(ip, jp, kp)];
          }
        }
  }
  pop(c.localBlocks, fatherID);
  nbLocal = nbLocal + 7;
  return 0;
}

// coarseBlocks (amr.f90:1430-1650), single-process branch: families of
// marked blocks, then for each family of eight the father takes the first
// empty slot and receives the 8-cell sums / 8 of every sibling, whose slot
// is freed; calcPrimsBlock(CELLS_PHYS) of the father.
int coarseBlocks(Ctx& c, const std::vector<int>& refineFlags, int& ncoarse) {
  std::vector<std::pair<int, int>> family;
  for (int nb = 0; nb < c.nbMax; ++nb) {
    int flag = refineFlags[nb], bID = c.localBlocks[nb];
    if (bID != -1 && flag == WX_FLAG_COARSE) {
      int sib[8];
      siblings(c, bID, sib);
      int eID = sib[0];
      bool counted = false;
      for (auto& f : family)
        if (f.first == eID) { f.second += 1; counted = true; break; }
      if (!counted) family.push_back({eID, 1});
    }
  }
  ncoarse = 0;
  for (auto& f : family) {
    if (f.second != 8) continue;
    int eID = f.first, sib[8];
    siblings(c, eID, sib);
    int fID = father(c, eID);
    int fatherIndex = put(c.localBlocks, fID);
    if (fatherIndex == -1) return WX_ERR_REGISTER_FATHER;
    for (int s = 0; s < 8; ++s) {
      int sx, sy, sz;
      siblingCoords(c, sib[s], sx, sy, sz);
      int locIndx = find(c.localBlocks, sib[s]);
      for (int i = 1; i <= NC / 2; ++i)
        for (int j = 1; j <= NC / 2; ++j)
          for (int k = 1; k <= NC / 2; ++k) {
            int i1 = i * 2 - 1, j1 = j * 2 - 1, k1 = k * 2 - 1;
            int ip = i + sx * NC / 2, jp = j + sy * NC / 2, kp = k + sz * NC / 2;
            for (int e = 0; e < c.neq; ++e) {
              const double* src = c.u(c.U, locIndx, e);
              double sum = 0.0;
              for (int kk = k1; kk <= k1 + 1; ++kk)
                for (int jj = j1; jj <= j1 + 1; ++jj)
                  for (int ii = i1; ii <= i1 + 1; ++ii) sum += src[cidx(ii, jj, kk)];
              c.u(c.U, fatherIndex, e)[cidx(ip, jp, kp)] = sum / 8.0;
            }
          }
      pop(c.localBlocks, sib[s]);
    }
    long long pf = 0, df = 0, zd = 0;
    calcPrimsBlock(c, c.U, c.PRIM, fatherIndex, CELLS_PHYS, pf, df, zd);
    ++ncoarse;
  }
  return 0;
}

void setupGeometry(Ctx& c) {  // init.f90:632-756 (MESH_MANUAL)
  const wx_config& f = c.cfg;
  for (int ilev = 1; ilev <= f.maxlev; ++ilev) {
    double s = std::ldexp(1.0, ilev - 1);
    c.dx[ilev] = f.xphystot / ((double)(NC * f.nbrootx) * s) / f.l_sc;
    c.dy[ilev] = f.yphystot / ((double)(NC * f.nbrooty) * s) / f.l_sc;
    c.dz[ilev] = f.zphystot / ((double)(NC * f.nbrootz) * s) / f.l_sc;
    c.nbx[ilev] = f.nbrootx << (ilev - 1);
    c.nby[ilev] = f.nbrooty << (ilev - 1);
    c.nbz[ilev] = f.nbrootz << (ilev - 1);
  }
  c.minID[1] = 1;
  c.maxID[1] = f.nbrootx * f.nbrooty * f.nbrootz;
  for (int ilev = 2; ilev <= f.maxlev; ++ilev) {
    int nbl = f.nbrootx * f.nbrooty * f.nbrootz;
    for (int q = 0; q < ilev - 1; ++q) nbl *= 8;
    c.minID[ilev] = c.maxID[ilev - 1] + 1;
    c.maxID[ilev] = c.maxID[ilev - 1] + nbl;
  }
}

}  // namespace

// ===========================================================================
// extern "C" surface used by tests (ctypes) and bench.py's CPU leg.

extern "C" {

void* orc_create(const wx_config* cfg, int nbMax, int nthreads) {
  Ctx* c = new Ctx();
  c->cfg = *cfg;
  c->neq = cfg->neqtot;
  c->nbMax = nbMax;
  c->fp = 5 + 3 * (cfg->bfield ? 1 : 0);
  c->cv = 1.0 / (cfg->gamma - 1.0);                       // parameters.f90:373
  c->p_sc = cfg->d_sc * (cfg->v_sc * cfg->v_sc);            // parameters.f90:379
  c->e_sc = c->p_sc;                                        // :380
  c->t_sc = cfg->l_sc / cfg->v_sc;                          // :381
  size_t n = (size_t)nbMax * c->neq * NCELL;
  c->U.assign(n, 0.0);
  c->UP.assign(n, 0.0);
  c->PRIM.assign(n, 0.0);
  c->localBlocks.assign(nbMax, -1);
  c->nthreads = nthreads > 0 ? nthreads : 1;
  setupGeometry(*c);
  return c;
}

void orc_destroy(void* h) { delete static_cast<Ctx*>(h); }

void orc_set_threads(void* h, int n) { static_cast<Ctx*>(h)->nthreads = n > 0 ? n : 1; }

int orc_set_blocks(void* h, int n, const int* bids) {
  Ctx* c = static_cast<Ctx*>(h);
  if (n > c->nbMax) return WX_ERR_INVALID_ARG;
  c->slotOf.clear();
  for (int i = 0; i < c->nbMax; ++i) c->localBlocks[i] = (i < n) ? bids[i] : -1;
  for (int i = 0; i < c->nbMax; ++i)
    if (c->localBlocks[i] != -1) c->slotOf[c->localBlocks[i]] = i;
  return 0;
}

// Neighbour query (amr.f90:539) for the test of the device table.
void orc_neighbors(void* h, int bID, int dir, int* ntype, int* list4) {
  neighbors(*static_cast<Ctx*>(h), bID, dir, *ntype, list4);
}
void orc_sibling_coords(void* h, int bID, int* s3) { siblingCoords(*static_cast<Ctx*>(h), bID, s3[0], s3[1], s3[2]); }
int orc_meshlevel(void* h, int bID) { return meshlevel(*static_cast<Ctx*>(h), bID); }
void orc_children(void* h, int bID, int* out8) { children(*static_cast<Ctx*>(h), bID, out8); }
int orc_father(void* h, int bID) { return father(*static_cast<Ctx*>(h), bID); }
void orc_cell_pos(void* h, int bID, int i, int j, int k, double* xyz) {
  cellPos(*static_cast<Ctx*>(h), bID, i, j, k, xyz[0], xyz[1], xyz[2]);
}

// which: 0 = U, 1 = UP, 2 = PRIM.  full=1 copies all 20^3 cells, else the 16^3 interior.
static std::vector<double>& pick(Ctx* c, int which) { return which == 0 ? c->U : (which == 1 ? c->UP : c->PRIM); }

void orc_set_array(void* h, int which, int full, const double* src) {
  Ctx* c = static_cast<Ctx*>(h);
  std::vector<double>& a = pick(c, which);
  if (full) { std::memcpy(a.data(), src, a.size() * sizeof(double)); return; }
  size_t q = 0;
  for (int nb = 0; nb < c->nbMax; ++nb)
    for (int e = 0; e < c->neq; ++e) {
      double* d = c->u(a, nb, e);
      for (int k = 1; k <= NC; ++k)
        for (int j = 1; j <= NC; ++j)
          for (int i = 1; i <= NC; ++i) d[cidx(i, j, k)] = src[q++];
    }
}

void orc_get_array(void* h, int which, int full, double* dst) {
  Ctx* c = static_cast<Ctx*>(h);
  std::vector<double>& a = pick(c, which);
  if (full) { std::memcpy(dst, a.data(), a.size() * sizeof(double)); return; }
  size_t q = 0;
  for (int nb = 0; nb < c->nbMax; ++nb)
    for (int e = 0; e < c->neq; ++e) {
      const double* s = c->u(a, nb, e);
      for (int k = 1; k <= NC; ++k)
        for (int j = 1; j <= NC; ++j)
          for (int i = 1; i <= NC; ++i) dst[q++] = s[cidx(i, j, k)];
    }
}

void orc_set_state(void* h, const wx_state* s) {
  Ctx* c = static_cast<Ctx*>(h);
  c->time = s->time; c->dt = s->dt; c->it = s->it; c->nextout = s->nextout; c->dumpout = s->dumpout != 0;
}
void orc_get_state(void* h, wx_state* s) {
  Ctx* c = static_cast<Ctx*>(h);
  s->time = c->time; s->dt = c->dt; s->it = c->it; s->nextout = c->nextout; s->dumpout = c->dumpout ? 1 : 0; s->pad = 0;
}

void orc_get_counters(void* h, long long* out4) {
  Ctx* c = static_cast<Ctx*>(h);
  out4[0] = c->pressure_floor; out4[1] = c->density_floor; out4[2] = c->zero_density;
  out4[3] = 0;
}

void orc_update_prims(void* h) { Ctx* c = static_cast<Ctx*>(h); calcPrimsAll(*c, c->U, c->PRIM, CELLS_ALL); }
void orc_calc_prims(void* h, int which_src, int cells) {
  Ctx* c = static_cast<Ctx*>(h);
  calcPrimsAll(*c, pick(c, which_src), c->PRIM, cells);
}
void orc_boundary(void* h, int depth, int which) { Ctx* c = static_cast<Ctx*>(h); boundary(*c, depth, pick(c, which)); }
double orc_get_timestep(void* h) { return getTimestep(*static_cast<Ctx*>(h)); }
void orc_hydro_solver(void* h) { hydroSolver(*static_cast<Ctx*>(h)); }
void orc_update_neutral_fraction(void* h) { updateNeutralFraction(*static_cast<Ctx*>(h)); }
double orc_cooling(void* h) { return cooling(*static_cast<Ctx*>(h)); }

// One main-loop body without AMR/output (main.f90:81-100).
void orc_step(void* h) {
  Ctx* c = static_cast<Ctx*>(h);
  c->it = c->it + 1;
  hydroSolver(*c);
  calcPrimsAll(*c, c->U, c->PRIM, CELLS_ALL);
  if (c->cfg.eos_type == WX_EOS_H_RATE) updateNeutralFraction(*c);
  cooling(*c);
  if (c->dumpout) { c->nextout = c->nextout + 1; c->dumpout = false; }
}

// loadcooldata_metal (cooling.f90:193-265): tab[(nptsT+1)*(nptsZ+1)] row by
// row, tab[0][0] unused, tab[0][1..] metallicities, tab[1..][0] log T,
// the rest log Lambda.
int orc_set_cooltable_metal(void* h, int nptsT, int nptsZ, const double* tab) {
  Ctx* c = static_cast<Ctx*>(h);
  if (nptsT < 2 || nptsZ < 2) return WX_ERR_COOLING_LOAD_COEFS;
  c->nptsT = nptsT;
  c->nptsZ = nptsZ;
  c->ctab_metal.assign(tab, tab + (size_t)(nptsT + 1) * (nptsZ + 1));
  c->ctab_metal[0] = -1.0;
  c->cool_Tmin = ctm(*c, 2, 1);
  c->cool_Tmax = ctm(*c, nptsT + 1, 1);
  c->cool_Zmin = ctm(*c, 1, 2);
  c->cool_Zmax = ctm(*c, 1, nptsZ + 1);
  return 0;
}

// loadcooldata_schure (cooling_schure.f90:52-95): 180 rows of 5 columns as
// in the table file; column 1+dmc_f holds -log10 Lambda.
int orc_set_cooltable_schure(void* h, const double* data, int dmc_f) {
  Ctx* c = static_cast<Ctx*>(h);
  if (dmc_f < 1 || dmc_f > 4) return WX_ERR_COOLING_LOAD_COEFS;
  c->schureT.resize(180);
  c->schureL.resize(180);
  for (int i = 0; i < 180; ++i) {
    c->schureT[i] = std::pow(10.0, data[5 * i]);
    c->schureL[i] = std::pow(10.0, -data[5 * i + dmc_f]);
  }
  return 0;
}

int orc_set_cooltable(void* h, int npts, const double* logT, const double* b) {
  Ctx* c = static_cast<Ctx*>(h);
  if (npts < 2) return WX_ERR_COOLING_LOAD_COEFS;
  c->nptsT = npts;
  c->cooltable1.assign(logT, logT + npts);
  c->cooltable2.resize(npts);
  for (int i = 0; i < npts; ++i) c->cooltable2[i] = -b[i];
  c->cool_Tmin = c->cooltable1[0];
  c->cool_Tmax = c->cooltable1[npts - 1];
  return 0;
}

int orc_add_wind(void* h, const double* p12) {
  Ctx* c = static_cast<Ctx*>(h);
  Wind w{p12[0], p12[1], p12[2], p12[3], p12[4], p12[5], p12[6], p12[7], p12[8], p12[9], p12[10], p12[11]};
  c->winds.push_back(w);
  return 0;
}

void orc_mark(void* h, int* flags) {
  Ctx* c = static_cast<Ctx*>(h);
  for (int nb = 0; nb < c->nbMax; ++nb) flags[nb] = (c->localBlocks[nb] == -1) ? -1 : markByPhysical(*c, nb);
}

// refineBlock data part (amr.f90:355-367) for U and PRIM.
void orc_refine(void* h, int father_slot, const int* child_slots) {
  Ctx* c = static_cast<Ctx*>(h);
  for (int cc = 0; cc < 8; ++cc) {
    int sx = cc & 1, sy = (cc >> 1) & 1, sz = (cc >> 2) & 1;
    for (int i = 1; i <= NC; ++i)
      for (int j = 1; j <= NC; ++j)
        for (int k = 1; k <= NC; ++k) {
          int ip = (NC / 2) * sx + (i + 1) / 2, jp = (NC / 2) * sy + (j + 1) / 2, kp = (NC / 2) * sz + (k + 1) / 2;
          for (int e = 0; e < c->neq; ++e) {
            c->u(c->U, child_slots[cc], e)[cidx(i, j, k)] = c->u(c->U, father_slot, e)[cidx(ip, jp, kp)];
            c->u(c->PRIM, child_slots[cc], e)[cidx(i, j, k)] = c->u(c->PRIM, father_slot, e)[cidx(ip, jp, kp)];
          }
        }
  }
}

// admesh (amr.f90:44-133) with one process: markByPhysical, checkProximity
// (maxlev-1), refineBlock for the marked blocks in slot order, coarseBlocks.
// counts2 = blocks refined, families coarsened.  Returns the reference's
// abort code (0 = ok).
int orc_admesh(void* h, int* counts2) {
  Ctx* c = static_cast<Ctx*>(h);
  std::vector<int> refineFlags(c->nbMax, WX_FLAG_NONE);
  for (int nb = 0; nb < c->nbMax; ++nb)
    if (c->localBlocks[nb] != -1) refineFlags[nb] = markByPhysical(*c, nb);
  checkProximity(*c, refineFlags, c->cfg.maxlev - 1);
  const std::vector<int> globalBlocks = c->localBlocks;
  int nbLocal = 0;
  for (int b : c->localBlocks) nbLocal += (b != -1);
  int nref = 0;
  for (int nb = 0; nb < c->nbMax; ++nb) {
    if (refineFlags[nb] != WX_FLAG_REFINE) continue;
    int rc = refineBlock(*c, globalBlocks[nb], nbLocal);
    if (rc) return rc;
    ++nref;
  }
  int ncoarse = 0;
  int rc = coarseBlocks(*c, refineFlags, ncoarse);
  c->slotOf.clear();
  for (int i = 0; i < c->nbMax; ++i)
    if (c->localBlocks[i] != -1) c->slotOf[c->localBlocks[i]] = i;
  if (counts2) { counts2[0] = nref; counts2[1] = ncoarse; }
  return rc;
}

void orc_get_blocks(void* h, int* out) {
  Ctx* c = static_cast<Ctx*>(h);
  std::copy(c->localBlocks.begin(), c->localBlocks.end(), out);
}

// coarseBlocks local branch (amr.f90:1592-1625), then calcPrimsBlock(CELLS_PHYS).
void orc_coarsen(void* h, const int* child_slots, int father_slot) {
  Ctx* c = static_cast<Ctx*>(h);
  for (int sib = 0; sib < 8; ++sib) {
    int sx = sib & 1, sy = (sib >> 1) & 1, sz = (sib >> 2) & 1;
    int loc = child_slots[sib];
    for (int i = 1; i <= NC / 2; ++i)
      for (int j = 1; j <= NC / 2; ++j)
        for (int k = 1; k <= NC / 2; ++k) {
          int i1 = i * 2 - 1, j1 = j * 2 - 1, k1 = k * 2 - 1;
          int ip = i + sx * NC / 2, jp = j + sy * NC / 2, kp = k + sz * NC / 2;
          for (int e = 0; e < c->neq; ++e) {
            const double* s = c->u(c->U, loc, e);
            double sum = 0.0;  // Fortran SUM over the 2x2x2 section, array element order
            for (int kk = k1; kk <= k1 + 1; ++kk)
              for (int jj = j1; jj <= j1 + 1; ++jj)
                for (int ii = i1; ii <= i1 + 1; ++ii) sum += s[cidx(ii, jj, kk)];
            c->u(c->U, father_slot, e)[cidx(ip, jp, kp)] = sum / 8.0;
          }
        }
  }
  long long pf = 0, df = 0, zd = 0;
  calcPrimsBlock(*c, c->U, c->PRIM, father_slot, CELLS_PHYS, pf, df, zd);
}

}  // extern "C"
