// wx3d_kernels.cuh -- sm_100a kernels of the per-block Godunov update.
//
// Stage kernel: one CTA per (block, z-slab).  320 threads (10 warps) march
// through the slab's k-planes; a 4-plane shared-memory ring holds the
// primitives of each plane together with its two-deep x/y ghost frame, so
// every x-, y- and z-interface flux is computed exactly once and the
// conservative update (godunov.f90:259-271) reads the two fluxes of each
// face from shared memory (x, y) or from the thread's registers (z).
#pragma once

#include "wx3d_device.cuh"
#include "wx3d_wind.cuh"

namespace wx {


// 17*16 x- and y-interfaces per plane on the first 272 threads; the plane
// loads (320 cells at first order, 384 at second) spread over all 320, and
// two CTAs per SM put five warps on every sub-partition
constexpr int STAGE_THREADS = 320;
static_assert(STAGE_THREADS >= 17 * NC, "one thread per x- and y-interface of a plane");
static_assert(STAGE_THREADS >= PLANE + 4 * NC, "the viscous step's UP frame is gathered by threads PLANE..PLANE+63");
constexpr int RING = 4;             // planes p-1..p+2 of the second-order stencil

struct StageParams {
  const double* __restrict__ src;   // array whose primitives feed the fluxes (physical cells)
  const double* __restrict__ base;  // array the update starts from (U)
  double* __restrict__ out;         // result (UP for stage 1, W for stage 2)
  const DevBlock* __restrict__ blocks;
  const int32_t* __restrict__ work; // occupied slots
  int32_t nwork;                    // number of (block, slab) items
  int32_t zsplit;                   // slabs per block (1, 2, 4 or 8)
  DevCtl* ctl;
  double dt_factor;                 // 0.5 for the predictor, 1 otherwise
  PhysParams ph;
  int32_t do_dt;                    // fused viscous step: fold the CFL minimum of the result
  const double* __restrict__ gsrc;  // array the ghost cells are gathered from (src, or the
                                    // wind-imposed copy of U in the first stage of a wind run)
  double* __restrict__ gframe;      // first-order stage: where to leave the ghost primitives
                                    // markByPhysical reads (nullptr: not wanted)
};

// markByPhysical's ghost primitives (rho, p) of one block, left behind by the
// first-order stage, which gathers and converts exactly these cells anyway:
// entry (kk-1)*64 + h for entry h of the one-deep x/y frame of plane kk
// (1..16), 1024 + c for cell c of the bottom ghost plane (kk = 0) and
// 1280 + c for the top one (kk = 17).  Two doubles per entry.
constexpr int GFRAME = 16 * 64 + 2 * PLANE;

__device__ __forceinline__ int gframe_entry(int kk, int c) {
  if (c >= PLANE) return (kk >= 1 && kk <= NC) ? (kk - 1) * 64 + (c - PLANE) : -1;
  if (kk == 0) return 16 * 64 + c;
  if (kk == NC + 1) return 16 * 64 + PLANE + c;
  return -1;
}


// Ring plane geometry: 16x16 cells with the ORDER-deep x/y ghost frame.
template <int ORDER>
struct Geo {
  static constexpr int W = NC + 2 * ORDER;   // 20 for the corrector, 18 for the predictor
  static constexpr int PL = W * W;
};

// Ring channels per cell: the primitives, plus -- for the first-order hydro
// stage, whose interface states are the cell values -- the sound speed and
// 1/rho, computed once when the plane is loaded instead of at each of the
// six interfaces that use the cell.
template <int NEQ, bool MHD, int ORDER>
__host__ __device__ constexpr int ring_channels() {
  return NEQ + ((!MHD && ORDER == 1) ? 2 : 0);
}

constexpr int VPLANE = (NC + 2) * (NC + 2);  // a plane with its one-deep x/y frame

// Per-block constants and status counters of a stage CTA, kept in shared
// memory rather than in registers: dt/dx, dt/dy, dt/dz of the update, the
// inverse cell sizes of the CFL fold, and the counts of pressure floors,
// density floors, zero densities and non-finite results.
struct StageConsts {
  double dtdx, dtdy, dtdz, idx, idy, idz;
  unsigned cnt[4];
  int next;   // the CTA's next work item
  int pad_;
};

template <int NEQ, bool MHD, int ORDER, bool VISC = false>
__host__ __device__ constexpr size_t stage_smem_bytes() {
  return sizeof(double) * ((size_t)RING * ring_channels<NEQ, MHD, ORDER>() * Geo<ORDER>::PL + 2 * (size_t)NEQ * 17 * NC +
                           (VISC ? 2 * (size_t)NEQ * VPLANE : 0)) +
         sizeof(DevBlock) + sizeof(StageConsts);
}

template <int ORDER>
__device__ __forceinline__ int hidx(int i, int j) { return (i + ORDER - 1) + Geo<ORDER>::W * (j + ORDER - 1); }
__device__ __forceinline__ int ring_slot(int kk) { return (kk + 64) & (RING - 1); }

// Copies the (rho, p) just stored in ring plane pl at (i, j) to entry e of
// the block's ghost-primitive record.
template <int ORDER>
__device__ __forceinline__ void put_gframe(double* g, int slot, int e, const double* pl, int i, int j) {
  double2 v;
  v.x = pl[hidx<ORDER>(i, j)];
  v.y = pl[4 * Geo<ORDER>::PL + hidx<ORDER>(i, j)];
  reinterpret_cast<double2*>(g)[(size_t)slot * GFRAME + e] = v;
}

// Warp minimum of a positive time step folded into ctl->dtmin_bits.
__device__ __forceinline__ void block_min_dt(double v, DevCtl* ctl) {
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 16));
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 8));
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 4));
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 2));
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 1));
  if ((threadIdx.x & 31) == 0) atomic_min_pos(&ctl->dtmin_bits, v);
}

// Block-wide sum of four status counters into ctl->cnt.
__device__ __forceinline__ void flush_counts(DevCtl* ctl, unsigned pf, unsigned df, unsigned zd) {
  unsigned m = __activemask();
  pf = __reduce_add_sync(m, pf);
  df = __reduce_add_sync(m, df);
  zd = __reduce_add_sync(m, zd);
  if ((threadIdx.x & 31) == 0) {
    if (pf) atomicAdd(&ctl->cnt[0], (unsigned long long)pf);
    if (df) atomicAdd(&ctl->cnt[1], (unsigned long long)df);
    if (zd) atomicAdd(&ctl->cnt[2], (unsigned long long)zd);
  }
}

// One interface flux in direction DIR from ring cells c0..c3 (pointers to
// equation 0 of cells l-1, l, r, r+1; stride Geo<ORDER>::PL between channels).
// With CARRY (the z-interfaces, which a thread visits in order along its
// column) the limited slope of the lower cell is the upper cell's slope of
// the previous interface -- the limiter sees the same two differences -- and
// is taken from `carry` instead of being evaluated again, unless `first`;
// the upper cell's slope is left in `carry` for the next interface.
template <int NEQ, bool MHD, int SOLVER, int ORDER, int LIM, int DIR, bool CARRY = false>
__device__ __forceinline__ void iface_flux(const double* c0, const double* c1, const double* c2, const double* c3,
                                           const PhysParams& ph, double* f, double* carry = nullptr,
                                           bool first = true) {
  double pl[NEQ], pr[NEQ], fx[NEQ];
#pragma unroll
  for (int e = 0; e < NEQ; ++e) {
    const int q = perm<DIR, MHD>(e);
    pl[e] = c1[q * Geo<ORDER>::PL];
    pr[e] = c2[q * Geo<ORDER>::PL];
  }
  if (ORDER == 2) {  // limiter (hydro_core.f90:613-636) on permuted primitives
#pragma unroll
    for (int e = 0; e < NEQ; ++e) {
      const int q = perm<DIR, MHD>(e);
      const double prr = c3[q * Geo<ORDER>::PL];
      const double dm = pr[e] - pl[e], dr = prr - pr[e];
      double al;
      if (!CARRY || first) al = average_t<LIM>(pl[e] - c0[q * Geo<ORDER>::PL], dm, ph.limiter);
      else al = carry[e];
      const double ar = average_t<LIM>(dm, dr, ph.limiter);
      if (CARRY) carry[e] = ar;
      pl[e] = pl[e] + 0.5 * al;
      pr[e] = pr[e] - 0.5 * ar;
    }
  }
  if constexpr (!MHD && (SOLVER == WX_SOLVER_HLL || SOLVER == WX_SOLVER_HLLC)) {
    double cl, cr, rl, rr;
    if constexpr (ORDER == 1) {  // cell values: sound speed and 1/rho from the ring
      cl = c1[NEQ * Geo<ORDER>::PL];
      cr = c2[NEQ * Geo<ORDER>::PL];
      rl = c1[(NEQ + 1) * Geo<ORDER>::PL];
      rr = c2[(NEQ + 1) * Geo<ORDER>::PL];
    } else {
      rl = rcp_nr(pl[0]);
      rr = rcp_nr(pr[0]);
      cl = sqrt_nr(ph.gamma * pl[4] * rl);
      cr = sqrt_nr(ph.gamma * pr[4] * rr);
    }
    if constexpr (SOLVER == WX_SOLVER_HLLC) riemann_hllc_c<NEQ>(pl, pr, cl, cr, rl, rr, fx, ph.cv);
    else riemann_hll_c<NEQ>(pl, pr, cl, cr, fx, ph.cv);
  } else {
#pragma unroll
    for (int e = 0; e < NEQ; ++e) fx[e] = 0.0;
    riemann<NEQ, MHD, SOLVER>(pl, pr, fx, ph.gamma, ph.cv);
  }
#pragma unroll
  for (int e = 0; e < NEQ; ++e) f[perm<DIR, MHD>(e)] = fx[e];
}

// Stores the result of the fused viscous step for one cell, counts
// non-finite values and folds the cell's CFL time step.
template <int NEQ, bool MHD>
__device__ __forceinline__ void visc_store(const StageParams& P, const DevBlock& B, const double* un, size_t o,
                                           Cfl<NEQ, MHD>& cfl, StageConsts& K) {
  unsigned nonfinite = 0;
#pragma unroll
  for (int e = 0; e < NEQ; ++e) {
    P.out[o + (size_t)e * BCELLS] = un[e];
    nonfinite += !isfinite(un[e]);
  }
  if (nonfinite) atomicAdd(&K.cnt[3], nonfinite);
  if (P.do_dt) {
    double p[NEQ], rinv;
    flow2prim<NEQ, MHD>(un, p, P.ph.inv_cv, &rinv);
    cfl.fold(p, rinv, B, K.idx, K.idy, K.idz, P.ph.gamma);
  }
}

// Loads plane kk of the slab into its ring slot as primitives: the 16x16
// physical cells, plus -- for the planes that get x/y fluxes -- the x/y ghost
// frame (two deep for the second-order stage), gathered from the neighbours.
// Converts one cell's conserved variables to primitives (plus, for the
// first-order hydro stage, its sound speed and 1/rho) into ring plane pl,
// counting the flow2prim floors of physical cells when `count`.
template <int NEQ, bool MHD, int ORDER, int CH>
__device__ __forceinline__ void store_cell(const PhysParams& ph, double* pl, int i, int j, const double* u, bool count,
                                           unsigned* cnt) {
  double p[NEQ], rinv;
  const int st = flow2prim<NEQ, MHD>(u, p, ph.inv_cv, &rinv);
  if constexpr (CH > NEQ) {
    pl[NEQ * Geo<ORDER>::PL + hidx<ORDER>(i, j)] = sqrt_nr(ph.gamma * p[4] * rinv);
    pl[(NEQ + 1) * Geo<ORDER>::PL + hidx<ORDER>(i, j)] = rinv;
  }
  if (count && st != 0) atomicAdd(&cnt[st == 1 ? 0 : (st == 2 ? 1 : 2)], 1u);
#pragma unroll
  for (int e = 0; e < NEQ; ++e) pl[e * Geo<ORDER>::PL + hidx<ORDER>(i, j)] = p[e];
}

template <int NEQ, bool MHD, int ORDER, int CH>
__device__ __forceinline__ void load_plane(const StageParams& P, const DevBlock& B, int slot, int kk, int z0, int z1,
                                           double* ring, unsigned* cnt, bool skip_interior = false) {
  const int t = threadIdx.x;
  const PhysParams& ph = P.ph;
  double* pl = ring + ring_slot(kk) * CH * Geo<ORDER>::PL;
  const bool inner = (kk >= 1 && kk <= NC);
  const bool frame = (kk >= z0 && kk <= z1);  // plane gets x/y fluxes
  const int nframe = frame ? (ORDER == 2 ? 128 : 64) : 0;
  for (int c = skip_interior && t < PLANE ? t + STAGE_THREADS : t; c < PLANE + nframe; c += STAGE_THREADS) {
    int i, j;
    if (c < PLANE) { i = (c & 15) + 1; j = (c >> 4) + 1; }
    else {
      const int h = c - PLANE;
      const int per = ORDER == 2 ? 32 : 16;         // cells per side
      const int side = h / per, r = (h % 16) + 1;
      const int d = (ORDER == 2) ? ((h % 32) >> 4) : 1;   // 0: outer, 1: inner ghost layer
      if (side == 0) { i = d - 1; j = r; }
      else if (side == 1) { i = NC + 2 - d; j = r; }
      else if (side == 2) { i = r; j = d - 1; }
      else { i = r; j = NC + 2 - d; }
    }
    double u[NEQ];
    if (inner && c < PLANE) load_cell<NEQ>(P.src, slot, i, j, kk, u);
    else gather_ghost<NEQ>(P.gsrc ? P.gsrc : P.src, B, slot, i, j, kk, u);
    store_cell<NEQ, MHD, ORDER, CH>(ph, pl, i, j, u, c < PLANE && inner && frame, cnt);
    if (ORDER == 1 && P.gframe) {
      const int e = gframe_entry(kk, c);
      if (e >= 0) put_gframe<ORDER>(P.gframe, slot, e, pl, i, j);
    }
  }
}

// Per slab the planes are walked with two barriers each.  Phase A of update
// plane m loads plane m+ORDER+1 into the slot of plane m-1 (no longer read:
// the z-interface slope of plane m is carried in registers) while the same
// threads compute the z-flux m+1/2 and the x/y fluxes of plane m; phase B
// applies the update.  The loads of one warp overlap the flux arithmetic of
// the others.
//
// VISC (second stage, whole blocks) fuses doViscousStep
// (hydro_solver.f90:217-250): the stage result W of plane m goes to a
// two-plane shared buffer whose one-deep x/y frame holds the half-step UP
// ghosts, and phase B of plane m applies U = W + eta (sum of the six
// neighbours - 6 W) to plane m-1, whose z-neighbours are W(m-2) (still in
// the buffer slot that W(m) replaces, read first by the same thread) and
// W(m) (in registers).  The block-face z-neighbours are UP ghosts as well.
// Two CTAs per SM where the shared memory allows it; registers are then
// capped at 96 per thread (ten warps per CTA, five on each sub-partition).
template <int NEQ, bool MHD, int ORDER, bool VISC>
__host__ __device__ constexpr int stage_ctas_per_sm() {
  return (!MHD && 2 * (stage_smem_bytes<NEQ, MHD, ORDER, VISC>() + 1024) <= 228 * 1024) ? 2 : 1;
}

// Cell-centred electric field E = -v x B of the stage primitives at one ring
// cell: the field-interpolated E of the field-CD scheme (Toth 2000, J. Comput.
// Phys. 161, 605), which brio-wu/flux_cd.f90:37 declares as efield(3,...).
template <int ORDER>
__device__ __forceinline__ void efield(const double* c, double* E) {
  constexpr int PL = Geo<ORDER>::PL;
  const double v1 = c[1 * PL], v2 = c[2 * PL], v3 = c[3 * PL];
  const double b1 = c[5 * PL], b2 = c[6 * PL], b3 = c[7 * PL];
  E[0] = v3 * b2 - v2 * b3;
  E[1] = v1 * b3 - v3 * b1;
  E[2] = v2 * b1 - v1 * b2;
}

template <int NEQ, bool MHD, int SOLVER, int ORDER, int LIM, bool VISC = false>
__global__ void __launch_bounds__(STAGE_THREADS, (stage_ctas_per_sm<NEQ, MHD, ORDER, VISC>())) stage_kernel(StageParams P) {
  constexpr int CH = ring_channels<NEQ, MHD, ORDER>();
  extern __shared__ __align__(16) double smem[];
  double* ring = smem;                                   // [RING][CH][Geo<ORDER>::PL]
  double* fxs = ring + RING * CH * Geo<ORDER>::PL;               // [NEQ][16 rows][17]
  double* fys = fxs + NEQ * 17 * NC;                     // [NEQ][17][16 cols]
  double* wpl = fys + NEQ * 17 * NC;                     // VISC: [2][NEQ][VPLANE]
  DevBlock& B = *reinterpret_cast<DevBlock*>(wpl + (VISC ? 2 * NEQ * VPLANE : 0));
  StageConsts& K = *reinterpret_cast<StageConsts*>(&B + 1);
  auto vq = [](int i, int j) { return i + (NC + 2) * j; };
  Cfl<NEQ, MHD> cfl;
  const int t = threadIdx.x;
  const int planes = NC / P.zsplit;
  const PhysParams& ph = P.ph;
  if (t < 4) K.cnt[t] = 0;

  for (int w = blockIdx.x; w < P.nwork;) {
    const int slot = P.work[w / P.zsplit];
    const int z0 = 1 + (w % P.zsplit) * planes, z1 = z0 + planes - 1;
    __syncthreads();
    if (t < (int)(sizeof(DevBlock) / 4)) reinterpret_cast<int*>(&B)[t] = reinterpret_cast<const int*>(P.blocks + slot)[t];
    __syncthreads();
    if (t == 0) {  // read after the prologue's barriers
      const double dtp = P.ctl->dt * P.dt_factor;
      K.dtdx = dtp / B.dx;
      K.dtdy = dtp / B.dy;
      K.dtdz = dtp / B.dz;
      K.idx = 1.0 / B.dx;
      K.idy = 1.0 / B.dy;
      K.idz = 1.0 / B.dz;
    }
    const int ci = (t & (NC - 1)) + 1, cj = (t >> 4) + 1;   // column of threads t < 256
    const int hc = hidx<ORDER>(ci, cj);
    double zprev[NEQ], znew[NEQ], zslope[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { zprev[e] = 0.0; znew[e] = 0.0; zslope[e] = 0.0; }
    double bz_below = 0.0;  // B_z of plane m-1 in this thread's column (Powell source)
    double e_below[3] = {0.0, 0.0, 0.0};  // E of plane m-1 in this thread's column (field-CD)

    // ---- prologue: planes z0-ORDER .. z0+ORDER-1, the z-interface z0-1/2,
    // then plane z0+ORDER into the slot of plane z0-ORDER ------------------
    for (int kk = z0 - ORDER; kk <= z0 + ORDER - 1; ++kk) load_plane<NEQ, MHD, ORDER, CH>(P, B, slot, kk, z0, z1, ring, K.cnt);
    __syncthreads();
    if (t < PLANE) {
      const int m = z0 - 1;
      const double* c0 = ring + ring_slot(m - 1) * CH * Geo<ORDER>::PL + hc;
      const double* c1 = ring + ring_slot(m) * CH * Geo<ORDER>::PL + hc;
      const double* c2 = ring + ring_slot(m + 1) * CH * Geo<ORDER>::PL + hc;
      const double* c3 = ring + ring_slot(m + 2) * CH * Geo<ORDER>::PL + hc;
      iface_flux<NEQ, MHD, SOLVER, ORDER, LIM, 2, true>(c0, c1, c2, c3, ph, znew, zslope, true);
      if (MHD) bz_below = c1[7 * Geo<ORDER>::PL];
      if (MHD && ph.flux_cd) efield<ORDER>(c1, e_below);
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) zprev[e] = znew[e];
    if (VISC && t < PLANE) {  // W(z0-1) of the column: the bottom UP ghost
      double g[NEQ];
      gather_ghost<NEQ>(P.src, B, slot, ci, cj, z0 - 1, g);
#pragma unroll
      for (int e = 0; e < NEQ; ++e) wpl[((z0 - 1) & 1) * NEQ * VPLANE + e * VPLANE + vq(ci, cj)] = g[e];
    }
    __syncthreads();
    load_plane<NEQ, MHD, ORDER, CH>(P, B, slot, z0 + ORDER, z0, z1, ring, K.cnt);
    __syncthreads();

    for (int m = z0; m <= z1; ++m) {
      // ---- phase A: load plane m+ORDER+1; z-flux m+1/2; x/y fluxes of m ---
      {
        // L2 prefetch, one plane period ahead, of the physical cells of the
        // plane the next phase A loads and of the base plane the next phase B
        // reads (16 lines of 128 bytes per equation and plane)
        const int kq = t < 16 * NEQ ? m + ORDER + 2 : m + 1;
        const double* arr = t < 16 * NEQ ? P.src : P.base;
        const int r = t < 16 * NEQ ? t : t - 16 * NEQ;
        if (r < 16 * NEQ && kq >= 1 && kq <= NC && kq <= z1 + ORDER && (t < 16 * NEQ || kq <= z1))
          prefetch_l2(arr + cell_off(slot, NEQ, r >> 4, 1, 1, kq) + (size_t)(r & 15) * 16);
      }
      // the physical cell of each thread t < 256 is fetched here and
      // converted into the ring after the fluxes, so its load latency
      // overlaps them; the ghost frame is gathered and stored first
      const int kl = m + ORDER + 1;
      const bool late = t < PLANE && kl <= z1 + ORDER;
      double ul[NEQ];
      if (late) {
        if (kl >= 1 && kl <= NC) load_cell<NEQ>(P.src, slot, ci, cj, kl, ul);
        else gather_ghost<NEQ>(P.gsrc ? P.gsrc : P.src, B, slot, ci, cj, kl, ul);
      }
      if (kl <= z1 + ORDER) load_plane<NEQ, MHD, ORDER, CH>(P, B, slot, kl, z0, z1, ring, K.cnt, true);
      // one-deep x/y frame of W(m): UP ghosts of plane m, on threads 256..319,
      // which compute no z-flux and at most one x/y interface pair
      if (VISC && t >= PLANE && t < PLANE + 4 * NC) {
        {
          const int f = t - PLANE;
          const int side = f >> 4, r = (f & 15) + 1;
          const int gi = side == 0 ? 0 : (side == 1 ? NC + 1 : r);
          const int gj = side == 2 ? 0 : (side == 3 ? NC + 1 : r);
          double g[NEQ];
          gather_ghost<NEQ>(P.src, B, slot, gi, gj, m, g);
#pragma unroll
          for (int e = 0; e < NEQ; ++e) wpl[(m & 1) * NEQ * VPLANE + e * VPLANE + vq(gi, gj)] = g[e];
        }
      }
      if (t < 17 * NC) {
        const double* pp = ring + ring_slot(m) * CH * Geo<ORDER>::PL;
        // x-interface between ii and ii+1 in row jx: a half-warp takes 16
        // consecutive interfaces of one row (conflict-free shared loads),
        // threads 256..271 the last interface of each row; y-interface
        // between jj and jj+1 in column iy
        const int ii = t < PLANE ? (t & 15) : NC, jx = t < PLANE ? (t >> 4) + 1 : t - PLANE + 1;
        const int iy = (t & 15) + 1, jj = t >> 4;
        {
          double f[NEQ];
          iface_flux<NEQ, MHD, SOLVER, ORDER, LIM, 0>(pp + hidx<ORDER>(ii - 1, jx), pp + hidx<ORDER>(ii, jx), pp + hidx<ORDER>(ii + 1, jx),
                                                 pp + hidx<ORDER>(ii + 2, jx), ph, f);
#pragma unroll
          for (int e = 0; e < NEQ; ++e) fxs[(e * NC + (jx - 1)) * 17 + ii] = f[e];
        }
        {
          double f[NEQ];
          iface_flux<NEQ, MHD, SOLVER, ORDER, LIM, 1>(pp + hidx<ORDER>(iy, jj - 1), pp + hidx<ORDER>(iy, jj), pp + hidx<ORDER>(iy, jj + 1),
                                                 pp + hidx<ORDER>(iy, jj + 2), ph, f);
#pragma unroll
          for (int e = 0; e < NEQ; ++e) fys[(e * 17 + jj) * NC + (iy - 1)] = f[e];
        }
      }
      if (t < PLANE) {  // z-flux m+1/2 last: znew is live only from here to phase B
        const double* c1 = ring + ring_slot(m) * CH * Geo<ORDER>::PL + hc;
        const double* c2 = ring + ring_slot(m + 1) * CH * Geo<ORDER>::PL + hc;
        const double* c3 = ring + ring_slot(m + 2) * CH * Geo<ORDER>::PL + hc;
        iface_flux<NEQ, MHD, SOLVER, ORDER, LIM, 2, true>(nullptr, c1, c2, c3, ph, znew, zslope, false);
      }
      if (late) {
        double* pl = ring + ring_slot(kl) * CH * Geo<ORDER>::PL;
        store_cell<NEQ, MHD, ORDER, CH>(ph, pl, ci, cj, ul, kl >= 1 && kl <= NC && kl >= z0 && kl <= z1, K.cnt);
        if (ORDER == 1 && P.gframe && kl == NC + 1) put_gframe<ORDER>(P.gframe, slot, gframe_entry(kl, t), pl, ci, cj);
      }
      __syncthreads();
      // ---- phase B: conservative update of plane m (godunov.f90:259-271) --
      if (t < PLANE) {
        double s[NEQ];
#pragma unroll
        for (int e = 0; e < NEQ; ++e) s[e] = 0.0;
        if (MHD && ph.eight_wave) {  // Powell source (sources.f90:38-95) on the stage primitives
          const double* pm = ring + ring_slot(m) * CH * Geo<ORDER>::PL;
          const double* pu = ring + ring_slot(m + 1) * CH * Geo<ORDER>::PL;
          const int h = hc;
          const double divB = (pm[5 * Geo<ORDER>::PL + h + 1] - pm[5 * Geo<ORDER>::PL + h - 1]) / (2. * B.dx) +
                              (pm[6 * Geo<ORDER>::PL + h + Geo<ORDER>::W] - pm[6 * Geo<ORDER>::PL + h - Geo<ORDER>::W]) / (2. * B.dy) +
                              (pu[7 * Geo<ORDER>::PL + h] - bz_below) / (2. * B.dz);
          const double v1 = pm[1 * Geo<ORDER>::PL + h], v2 = pm[2 * Geo<ORDER>::PL + h], v3 = pm[3 * Geo<ORDER>::PL + h];
          const double b1 = pm[5 * Geo<ORDER>::PL + h], b2 = pm[6 * Geo<ORDER>::PL + h], b3 = pm[7 * Geo<ORDER>::PL + h];
          s[1] = -divB * b1;
          s[2] = -divB * b2;
          s[3] = -divB * b3;
          s[4] = -divB * (v1 * b1 + v2 * b2 + v3 * b3);
          s[5] = -divB * v1;
          s[6] = -divB * v2;
          s[7] = -divB * v3;
        }
        if (MHD) bz_below = ring[ring_slot(m) * CH * Geo<ORDER>::PL + 7 * Geo<ORDER>::PL + hc];
        const size_t o = cell_off(slot, NEQ, 0, ci, cj, m);
        // field-CD (brio-wu/flux_cd.f90:74-84): B from the central differences
        // of E over the six face neighbours; E of plane m-1 is carried
        double bcd[3] = {0.0, 0.0, 0.0};
        if (MHD && ph.flux_cd) {
          constexpr int PL = Geo<ORDER>::PL, W = Geo<ORDER>::W;
          const double* pm = ring + ring_slot(m) * CH * PL + hc;
          double xl[3], xr[3], yl[3], yr[3], zu[3], ec[3];
          efield<ORDER>(pm - 1, xl);
          efield<ORDER>(pm + 1, xr);
          efield<ORDER>(pm - W, yl);
          efield<ORDER>(pm + W, yr);
          efield<ORDER>(ring + ring_slot(m + 1) * CH * PL + hc, zu);
          efield<ORDER>(pm, ec);
          const double hx = 0.5 * K.dtdx, hy = 0.5 * K.dtdy, hz = 0.5 * K.dtdz;
          bcd[0] = __ldg(P.base + o + 5 * (size_t)BCELLS) - hy * (yr[2] - yl[2]) - hz * (-zu[1] + e_below[1]);
          bcd[1] = __ldg(P.base + o + 6 * (size_t)BCELLS) - hx * (-xr[2] + xl[2]) - hz * (zu[0] - e_below[0]);
          bcd[2] = __ldg(P.base + o + 7 * (size_t)BCELLS) - hx * (xr[1] - xl[1]) - hy * (-yr[0] + yl[0]);
#pragma unroll
          for (int d = 0; d < 3; ++d) e_below[d] = ec[d];
        }
        double wv[NEQ];
        const double dtdx = K.dtdx, dtdy = K.dtdy, dtdz = K.dtdz;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
          const double fxl = fxs[(e * NC + (cj - 1)) * 17 + ci - 1], fxr = fxs[(e * NC + (cj - 1)) * 17 + ci];
          const double fyl = fys[(e * 17 + cj - 1) * NC + ci - 1], fyr = fys[(e * 17 + cj) * NC + ci - 1];
          double v = __ldg(P.base + o + (size_t)e * BCELLS) + dtdx * (fxl - fxr) + dtdy * (fyl - fyr) +
                     dtdz * (zprev[e] - znew[e]);
          if (MHD && ph.eight_wave) v = v + P.ctl->dt * P.dt_factor * s[e];
          if (MHD && ph.flux_cd && e >= 5 && e <= 7) v = bcd[e - 5];
          if (VISC) wv[e] = v;
          else P.out[o + (size_t)e * BCELLS] = v;
        }
        if constexpr (VISC) {
          double* wb = wpl + (m & 1) * NEQ * VPLANE;          // W(m-2) of the column, then W(m)
          const double* wc = wpl + ((m - 1) & 1) * NEQ * VPLANE;  // W(m-1) with its frame
          if (m > z0) {
            double un[NEQ];
#pragma unroll
            for (int e = 0; e < NEQ; ++e) {
              const double* pe = wc + e * VPLANE;
              const double c = pe[vq(ci, cj)];
              un[e] = c + ph.eta * (+pe[vq(ci + 1, cj)] + pe[vq(ci - 1, cj)] + pe[vq(ci, cj + 1)] + pe[vq(ci, cj - 1)] +
                                    wv[e] + wb[e * VPLANE + vq(ci, cj)] - 6.0 * c);
            }
            visc_store<NEQ, MHD>(P, B, un, o - NC * NC, cfl, K);
          }
#pragma unroll
          for (int e = 0; e < NEQ; ++e) wb[e * VPLANE + vq(ci, cj)] = wv[e];
        }
      }
#pragma unroll
      for (int e = 0; e < NEQ; ++e) zprev[e] = znew[e];
      __syncthreads();
    }
    if (VISC && t < PLANE) {  // viscous step of plane z1: above it, the top UP ghost
      double g[NEQ], un[NEQ];
      gather_ghost<NEQ>(P.src, B, slot, ci, cj, z1 + 1, g);
      const double* wc = wpl + (z1 & 1) * NEQ * VPLANE;
      const double* wb = wpl + ((z1 - 1) & 1) * NEQ * VPLANE;
#pragma unroll
      for (int e = 0; e < NEQ; ++e) {
        const double* pe = wc + e * VPLANE;
        const double c = pe[vq(ci, cj)];
        un[e] = c + ph.eta * (+pe[vq(ci + 1, cj)] + pe[vq(ci - 1, cj)] + pe[vq(ci, cj + 1)] + pe[vq(ci, cj - 1)] + g[e] +
                              wb[e * VPLANE + vq(ci, cj)] - 6.0 * c);
      }
      visc_store<NEQ, MHD>(P, B, un, cell_off(slot, NEQ, 0, ci, cj, z1), cfl, K);
    }
    // items past the first wave go, in list order, to whichever CTA
    // finishes first (the counter is zeroed before each launch): blocks at
    // coarse/fine faces cost more, and a static stride left SMs idle
    if (t == 0) K.next = (int)gridDim.x + (int)atomicAdd(&P.ctl->work_next[ORDER - 1], 1u);
    __syncthreads();
    w = K.next;
  }
  if (VISC && P.do_dt) block_min_dt(cfl.dt(), P.ctl);
  __syncthreads();
  if (t < 4 && K.cnt[t]) atomicAdd(&P.ctl->cnt[t], (unsigned long long)K.cnt[t]);
}

// ---------------------------------------------------------------------------
// Lax-Friedrichs (lax.f90:39-99): first order, from U with one-deep ghosts.
struct LaxParams {
  const double* __restrict__ u;
  double* __restrict__ out;
  const DevBlock* __restrict__ blocks;
  const int32_t* __restrict__ work;
  int32_t nwork;
  DevCtl* ctl;
  PhysParams ph;
};

template <int NEQ, bool MHD>
__global__ void __launch_bounds__(256) lax_kernel(LaxParams P) {
  __shared__ DevBlock B;
  const int t = threadIdx.x;
  const int i = (t & 15) + 1, j = (t >> 4) + 1;
  for (int w = blockIdx.x; w < P.nwork; w += gridDim.x) {
    const int slot = P.work[w];
    __syncthreads();
    if (t < (int)(sizeof(DevBlock) / 4)) reinterpret_cast<int*>(&B)[t] = reinterpret_cast<const int*>(P.blocks + slot)[t];
    __syncthreads();
    const double dt = P.ctl->dt;
    const double cx = 0.5 * dt / B.dx, cy = 0.5 * dt / B.dy, cz = 0.5 * dt / B.dz;
    for (int k = 1; k <= NC; ++k) {
      double un[6][NEQ], fl[NEQ], fr[NEQ], pv[NEQ], tmp[NEQ];
      const int di[6] = {1, -1, 0, 0, 0, 0}, dj[6] = {0, 0, 1, -1, 0, 0}, dk[6] = {0, 0, 0, 0, 1, -1};
#pragma unroll
      for (int q = 0; q < 6; ++q) get_cell<NEQ>(P.u, B, slot, i + di[q], j + dj[q], k + dk[q], un[q]);
      double res[NEQ];
#pragma unroll
      for (int e = 0; e < NEQ; ++e)
        res[e] = (un[0][e] + un[1][e] + un[2][e] + un[3][e] + un[4][e] + un[5][e]) / 6.0;
      // physical fluxes of the neighbour primitives, direction by direction
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double cc = d == 0 ? cx : (d == 1 ? cy : cz);
        flow2prim<NEQ, MHD>(un[2 * d], pv, P.ph.inv_cv);
#pragma unroll
        for (int e = 0; e < NEQ; ++e) tmp[e] = pv[d == 0 ? e : (d == 1 ? perm<1, MHD>(e) : perm<2, MHD>(e))];
        xflux<NEQ, MHD>(tmp, fr, P.ph.cv);
        flow2prim<NEQ, MHD>(un[2 * d + 1], pv, P.ph.inv_cv);
#pragma unroll
        for (int e = 0; e < NEQ; ++e) tmp[e] = pv[d == 0 ? e : (d == 1 ? perm<1, MHD>(e) : perm<2, MHD>(e))];
        xflux<NEQ, MHD>(tmp, fl, P.ph.cv);
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
          const int q = d == 0 ? e : (d == 1 ? perm<1, MHD>(e) : perm<2, MHD>(e));
          res[q] = res[q] - cc * (fr[e] - fl[e]);
        }
      }
      const size_t o = cell_off(slot, NEQ, 0, i, j, k);
#pragma unroll
      for (int e = 0; e < NEQ; ++e) P.out[o + (size_t)e * BCELLS] = res[e];
    }
  }
}

// ---------------------------------------------------------------------------
// doViscousStep (hydro_solver.f90:217-250) with the next step's CFL minimum
// (hydro_solver.f90:150-182) of the new state fused into the epilogue.
struct ViscParams {
  double* __restrict__ w;              // stage result, overwritten in place by U^{n+1}
  const double* __restrict__ up;       // predictor state: source of the face ghosts
  const DevBlock* __restrict__ blocks;
  const int32_t* __restrict__ work;
  int32_t nwork;
  int32_t zero_ghost;                  // single-stage solvers: UP ghosts are never filled (0)
  int32_t do_dt;                       // fold the CFL minimum of the new state
  DevCtl* ctl;
  PhysParams ph;
};

// Four CTAs per SM (at most 64 registers): 2.87 instead of 3.05 ms per
// step on the 20,896-block winds mesh with three.
template <int NEQ, bool MHD>
__global__ void __launch_bounds__(256, 4) viscous_kernel(ViscParams P) {
  __shared__ DevBlock B;
  __shared__ double pl[NEQ][18 * 18];   // plane k of W with the one-deep ghost frame from UP
  const int t = threadIdx.x;
  const int i = (t & 15) + 1, j = (t >> 4) + 1;
  const double eta = P.ph.eta;
  Cfl<NEQ, MHD> cfl;
  unsigned nonfinite = 0;
  auto q = [](int ii, int jj) { return ii + 18 * jj; };
  for (int w = blockIdx.x; w < P.nwork; w += gridDim.x) {
    const int slot = P.work[w];
    __syncthreads();
    if (t < (int)(sizeof(DevBlock) / 4)) reinterpret_cast<int*>(&B)[t] = reinterpret_cast<const int*>(P.blocks + slot)[t];
    __syncthreads();
    cfl.block(B);
    double wm[NEQ], wc[NEQ], wp[NEQ];
    // W(k-1) for k=1 is the bottom ghost of UP
    if (P.zero_ghost) {
#pragma unroll
      for (int e = 0; e < NEQ; ++e) wm[e] = 0.0;
    } else {
      gather_ghost<NEQ>(P.up, B, slot, i, j, 0, wm);
    }
    load_cell_rw<NEQ>(P.w, slot, i, j, 1, wc);
    for (int k = 1; k <= NC; ++k) {
      if (k < NC) load_cell_rw<NEQ>(P.w, slot, i, j, k + 1, wp);
      else if (P.zero_ghost) {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) wp[e] = 0.0;
      } else {
        gather_ghost<NEQ>(P.up, B, slot, i, j, NC + 1, wp);
      }
      __syncthreads();
#pragma unroll
      for (int e = 0; e < NEQ; ++e) pl[e][q(i, j)] = wc[e];
      if (t < 64) {  // one-deep x/y ghost frame of plane k from UP
        const int side = t >> 4, r = (t & 15) + 1;
        int gi, gj;
        if (side == 0) { gi = 0; gj = r; }
        else if (side == 1) { gi = NC + 1; gj = r; }
        else if (side == 2) { gi = r; gj = 0; }
        else { gi = r; gj = NC + 1; }
        double g[NEQ];
        if (P.zero_ghost) {
#pragma unroll
          for (int e = 0; e < NEQ; ++e) g[e] = 0.0;
        } else {
          gather_ghost<NEQ>(P.up, B, slot, gi, gj, k, g);
        }
#pragma unroll
        for (int e = 0; e < NEQ; ++e) pl[e][q(gi, gj)] = g[e];
      }
      __syncthreads();
      double un[NEQ];
#pragma unroll
      for (int e = 0; e < NEQ; ++e) {
        const double c = wc[e];
        un[e] = c + eta * (+pl[e][q(i + 1, j)] + pl[e][q(i - 1, j)] + pl[e][q(i, j + 1)] + pl[e][q(i, j - 1)] + wp[e] +
                           wm[e] - 6.0 * c);
      }
      const size_t o = cell_off(slot, NEQ, 0, i, j, k);
#pragma unroll
      for (int e = 0; e < NEQ; ++e) {
        P.w[o + (size_t)e * BCELLS] = un[e];
        nonfinite += !isfinite(un[e]);
      }
      if (P.do_dt) {
        double p[NEQ], rinv;
        flow2prim<NEQ, MHD>(un, p, P.ph.inv_cv, &rinv);
        cfl.fold(p, rinv, B, P.ph.gamma);
      }
#pragma unroll
      for (int e = 0; e < NEQ; ++e) { wm[e] = wc[e]; wc[e] = wp[e]; }
    }
  }
  if (P.do_dt) block_min_dt(cfl.dt(), P.ctl);
  nonfinite = __reduce_add_sync(0xffffffffu, nonfinite);
  if ((t & 31) == 0 && nonfinite) atomicAdd(&P.ctl->cnt[3], (unsigned long long)nonfinite);
}

// CFL minimum of an arbitrary state (getTimestep's loop, hydro_solver.f90:150-182).
struct DtParams {
  const double* __restrict__ u;
  const DevBlock* __restrict__ blocks;
  const int32_t* __restrict__ work;
  int32_t nwork;
  DevCtl* ctl;
  PhysParams ph;
};

template <int NEQ, bool MHD>
__global__ void __launch_bounds__(256) dt_kernel(DtParams P) {
  const int t = threadIdx.x;
  Cfl<NEQ, MHD> cfl;
  for (int w = blockIdx.x; w < P.nwork; w += gridDim.x) {
    const int slot = P.work[w];
    const DevBlock& B = P.blocks[slot];
    cfl.block(B);
    for (int k = 1; k <= NC; ++k) {
      double u[NEQ], p[NEQ], rinv;
      load_cell<NEQ>(P.u, slot, (t & 15) + 1, (t >> 4) + 1, k, u);
      flow2prim<NEQ, MHD>(u, p, P.ph.inv_cv, &rinv);
      cfl.fold(p, rinv, B, P.ph.gamma);
    }
  }
  block_min_dt(cfl.dt(), P.ctl);
}

__global__ void ctl_reset_dtmin_kernel(DevCtl* ctl) {
  if (threadIdx.x == 0) ctl->dtmin_bits = (unsigned long long)__double_as_longlong(1.0e30);
}

// getTimestep's scalar tail (hydro_solver.f90:185-207) and the iteration
// counter of main.f90:81.  Single thread.
__global__ void step_begin_kernel(DevCtl* ctl, double cfl, int cooling_on, double dtout, double t_sc, int bump_it) {
  if (threadIdx.x != 0) return;
  if (bump_it) ctl->it = ctl->it + 1;
  const double dt_hydro = __longlong_as_double((long long)ctl->dtmin_bits);
  const double dt_cool = 1.0e30;
  double dt_loc = cooling_on ? dmin(dt_hydro, dt_cool) * cfl : dt_hydro * cfl;
  if (ctl->it <= 10) dt_loc = exp2(-(double)(11 - ctl->it)) * dt_loc;
  double dt_glob = dt_loc;
  const double tnext = (double)ctl->nextout * dtout / t_sc;
  if (ctl->time + dt_glob >= tnext) {
    dt_glob = tnext - ctl->time;
    ctl->dumpout = 1;
  }
  ctl->dt = dt_glob;
  ctl->dtmin_bits = (unsigned long long)__double_as_longlong(1.0e30);
}

// time += dt (hydro_solver.f90:225) and, when the call stands for a whole
// main-loop iteration, the output bookkeeping of main.f90:109-114 (the
// output itself belongs to the host).
__global__ void step_end_kernel(DevCtl* ctl, int finish_output) {
  if (threadIdx.x != 0) return;
  ctl->time = ctl->time + ctl->dt;
  if (finish_output && ctl->dumpout) {
    ctl->nextout = ctl->nextout + 1;
    ctl->dumpout = 0;
    ctl->dumps = ctl->dumps + 1;
  }
}

// ---------------------------------------------------------------------------
// userBoundary of the wind problems: imposes the wind on the physical cells
// of `u` inside the spheres (blocks flagged in the neighbour table only).
// A ghost in a sphere is then gathered from a same-level neighbour whose
// cell at the same position carries the same imposed value
// (wx3d_set_winds refuses meshes where a coarse/fine face's ghost layer
// meets a sphere).
struct WindParams {
  double* __restrict__ u;
  const DevBlock* __restrict__ blocks;
  const int32_t* __restrict__ work;
  int32_t nwork;
  PhysParams ph;
};

// Copies whole blocks within one array: slot pairs (from, to), one row of
// CTAs per pair.
__global__ void copy_slots_kernel(double* u, const int2* __restrict__ pairs, int neq) {
  const int2 pr = pairs[blockIdx.y];
  const size_t n = (size_t)neq * BCELLS;
  const double* from = u + (size_t)pr.x * n;
  double* to = u + (size_t)pr.y * n;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    to[c] = from[c];
}

template <int NEQ, bool MHD>
__global__ void __launch_bounds__(256) wind_kernel(WindParams P) {
  for (int w = blockIdx.x; w < P.nwork; w += gridDim.x) {
    const int slot = P.work[w];
    const DevBlock& B = P.blocks[slot];
    if (!B.wind) continue;
    for (int c = threadIdx.x; c < BCELLS; c += blockDim.x) {
      const int i = (c & 15) + 1, j = ((c >> 4) & 15) + 1, k = (c >> 8) + 1;
      double u[NEQ];
      if (wind_state<NEQ, MHD>(P.ph, B, i, j, k, u)) {
        const size_t o = cell_off(slot, NEQ, 0, i, j, k);
#pragma unroll
        for (int e = 0; e < NEQ; ++e) P.u[o + (size_t)e * BCELLS] = u[e];
      }
    }
  }
}

}  // namespace wx
