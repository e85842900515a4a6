// wx3d_source.cuh -- per-cell source terms (hrate.f90, cooling.f90,
// cooling_h.f90), markByPhysical and the AMR data copies, as sm_100a kernels.
#pragma once

#include "wx3d_rates.cuh"

namespace wx {

// mode bits: 1 = updateNeutralFraction, 2 = cooling, 4 = primitives come
// from and go to the PRIM buffer (separate calls, as the reference's PRIM
// array), otherwise they are recomputed from U (fused step); 8 = fold the
// CFL minimum of the resulting primitives.
struct SrcParams {
  double* __restrict__ u;
  double* __restrict__ prim;
  const DevBlock* __restrict__ blocks;
  const int32_t* __restrict__ work;
  int32_t nwork;
  int32_t mode;
  DevCtl* ctl;
  const double* __restrict__ cool_lt;   // cooltable(1,:); COOL_TABLE_METAL: the 2-D table;
                                        // COOL_SCHURE: the 180 temperatures
  const double* __restrict__ cool_lc;   // cooltable(2,:) (= -b); COOL_SCHURE: the 180 Lambdas
  int32_t ncool;                        // rows (COOL_TABLE, COOL_SCHURE) or nptsT (METAL)
  PhysParams ph;
  int32_t nZ;                           // COOL_TABLE_METAL: metallicity columns
};

// updatePrims + updateNeutralFraction + cooling for every physical cell
// (main.f90:94-100), followed by the CFL minimum of the resulting PRIM.
// Five CTAs per SM (at most 48 registers): the rate and loss formulas are
// chains of dependent FP64 operations, and 40 resident warps hide them
// better than the 24 that 80 registers allowed, spills included.  SPEC
// fixes the source terms at compile time for the two combinations of the
// radiative runs (1: EOS_H_RATE + COOL_H, 2: EOS_H_RATE + COOL_TABLE), which
// leaves the other branches out of the register allocation; 0 reads the
// equation of state and the cooling type from ph.
template <int NEQ, bool MHD, int SPEC = 0>
__global__ void __launch_bounds__(256, 5) source_kernel(SrcParams P) {
  constexpr int FP = MHD ? 8 : 5;
  constexpr bool HAS_PAS = NEQ > FP;
  constexpr int EOS_C = SPEC ? WX_EOS_H_RATE : -1;
  constexpr int COOL_C = SPEC == 1 ? WX_COOL_H : (SPEC == 2 ? WX_COOL_TABLE : -1);
  const PhysParams& ph = P.ph;
  const int eos = EOS_C >= 0 ? EOS_C : ph.eos;
  const int cooling = COOL_C >= 0 ? COOL_C : ph.cooling;
  const int t = threadIdx.x;
  const double dts = P.ctl->dt * ph.t_sc;
  const bool do_hrate = P.mode & 1, do_cool = P.mode & 2, use_prim = P.mode & 4, do_dt = P.mode & 8;
  double dtl = 1.0e300, mloss = 0.0;
  for (int w = blockIdx.x; w < P.nwork; w += gridDim.x) {
    const int slot = P.work[w];
    const DevBlock& B = P.blocks[slot];
    for (int c = t; c < BCELLS; c += 256) {
      const size_t o = ((size_t)slot * NEQ) * BCELLS + c;
      double u[NEQ], p[NEQ];
#pragma unroll
      for (int e = 0; e < NEQ; ++e) u[e] = P.u[o + (size_t)e * BCELLS];
      if (use_prim) {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) p[e] = P.prim[o + (size_t)e * BCELLS];
      } else {
        flow2prim<NEQ, MHD>(u, p, ph.inv_cv);
      }
      constexpr int fp = FP;
      if (HAS_PAS && do_hrate && do_cool && eos == WX_EOS_H_RATE && cooling == WX_COOL_H) {
        h_cool_step<FP>(u, p, dts, ph, &mloss);  // hrate.f90:101-140 then cooling_h.f90:175-246
      } else if (HAS_PAS && do_hrate && eos == WX_EOS_H_RATE) {  // hrate.f90:101-140
        const double T = calc_temp<FP, EOS_C>(p, ph);
        const double dh = p[0] / ph.mu0;
        const double y0 = p[fp] / dh;
        const double y1 = h_rate_y1(T, dh, y0, dts);
        p[fp] = p[0] * y1 / ph.mu0;
        if (cooling != WX_COOL_H) u[fp] = p[fp];
      }
      if (HAS_PAS && do_hrate && do_cool && eos == WX_EOS_H_RATE && cooling == WX_COOL_H) {
        // done above
      } else if (do_cool && cooling != WX_COOL_H) {  // cooling.f90:303-369, cooling_schure.f90:134-228
        table_cooling<NEQ, FP, COOL_C, EOS_C>(u, p, dts, ph, P.cool_lt, P.cool_lc, P.ncool, P.nZ, mloss);
      } else if (HAS_PAS && do_cool && cooling == WX_COOL_H) {  // cooling_h.f90:175-246
        const double dh = p[0] / ph.mu0;
        const double dh0 = p[fp];
        const double y0 = ph.mu0 * u[fp] / u[0];
        u[fp] = p[fp];
        const double Temp = calc_temp<FP, EOS_C>(p, ph);
        if (Temp > 1.e4) {
          const double L0 = aloss_h(y0, dh, dh0, Temp);
          const double ce = (2.0 * L0) / (3.0 * KB * dh * Temp);
          const double T1 = 10.0 + (Temp - 10.0) * exp(-ce * dts);
          double cf = T1 / Temp;
          mloss = dmax(mloss, 1.0 - cf);
          if (cf < 1.0 - ph.cooling_limit) cf = 1.0 - ph.cooling_limit;
          if (Temp * cf < 10.0) cf = 10.0 / Temp;
          p[4] = p[4] * cf;
          const double EK = 0.5 * p[0] * (p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
          u[4] = EK + ph.cv * p[4];
        }
      }
      P.u[o + 4 * (size_t)BCELLS] = u[4];
      if (HAS_PAS) P.u[o + (size_t)fp * BCELLS] = u[fp];
      if (use_prim) {
        P.prim[o + 4 * (size_t)BCELLS] = p[4];
        if (HAS_PAS) P.prim[o + (size_t)fp * BCELLS] = p[fp];
      }
      if (do_dt) dtl = dmin(dtl, cell_dt<NEQ, MHD>(p, B, ph.gamma));
    }
  }
  if (do_dt) {
    double v = dtl;
    for (int s = 16; s > 0; s >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, s));
    if ((t & 31) == 0) atomic_min_pos(&P.ctl->dtmin_bits, v);
  }
  double m = mloss;
  for (int s = 16; s > 0; s >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, s));
  if ((t & 31) == 0 && m > 0.0) atomic_max_pos(&P.ctl->maxloss_bits, m);
}

// ---------------------------------------------------------------------------
// markByPhysical (amr.f90:142-230).  Physical PRIM from `u`, the one-deep
// ghost frame from the depth-1 ghost fill of `g` (the state at the start of
// the last step, which is what the reference's PRIM ghosts hold).
struct MarkParams {
  const double* __restrict__ u;
  const double* __restrict__ g;
  const DevBlock* __restrict__ blocks;
  const int32_t* __restrict__ work;
  int32_t nwork;
  int32_t* __restrict__ flags;   // per slot
  int32_t maxlev;
  double refine_thres, coarse_thres;
  PhysParams ph;
  const double* __restrict__ gframe;  // ghost (rho, p) left by the last step's first-order stage
                                      // (GFRAME entries per block), or nullptr: gather from g
};

template <int NEQ, bool MHD>
__global__ void __launch_bounds__(256, 4) mark_kernel(MarkParams P) {
  __shared__ double pp[3][18 * 18], pr[3][18 * 18];  // pressure and density, planes k-1..k+1
  __shared__ double bmax;                             // largest |delta|/value of the block
  __shared__ __align__(16) DevBlock B;                // the block's neighbour-table entry
  const int t = threadIdx.x;
  const int i = (t & 15) + 1, j = (t >> 4) + 1;
  auto q = [](int ii, int jj) { return ii + 18 * jj; };
  for (int w = blockIdx.x; w < P.nwork; w += gridDim.x) {
    const int slot = P.work[w];
    __syncthreads();
    if (t < (int)(sizeof(DevBlock) / 4)) reinterpret_cast<int*>(&B)[t] = reinterpret_cast<const int*>(P.blocks + slot)[t];
    if (t == 0) bmax = 0.0;
    __syncthreads();
    double lmax = 0.0;
    // plane kk (0..17) is fetched into registers one plane ahead, then
    // converted into ring slot kk%3, so its loads overlap the gradients of
    // the plane before
    const int side = t >> 4, r = (t & 15) + 1;
    const int gi = side == 0 ? 0 : (side == 1 ? NC + 1 : r);
    const int gj = side == 2 ? 0 : (side == 3 ? NC + 1 : r);
    // with a ghost record (P.gframe) the ghost cells' (rho, p) are read from
    // it, coalesced, instead of being gathered from the neighbour slots;
    // they are the same values (the same gathers and flow2prim, done by the
    // step's first-order stage)
    const double2* G = P.gframe ? reinterpret_cast<const double2*>(P.gframe) + (size_t)slot * GFRAME : nullptr;
    double ua[NEQ], ug[NEQ];
    auto fetch = [&](int kk) {
      const bool inner = kk >= 1 && kk <= NC;
      if (inner || !G) {
        get_cell<NEQ>(inner ? P.u : P.g, B, slot, i, j, kk, ua);
      } else {
        const double2 v = G[kk == 0 ? 16 * 64 + t : 16 * 64 + PLANE + t];
        ua[0] = v.x;
        ua[1] = v.y;
      }
      if (inner && t < 64) {
        if (!G) {
          gather_ghost<NEQ>(P.g, B, slot, gi, gj, kk, ug);
        } else {
          const double2 v = G[(kk - 1) * 64 + t];
          ug[0] = v.x;
          ug[1] = v.y;
        }
      }
    };
    auto commit = [&](int kk) {
      const int s = kk % 3;
      const bool inner = kk >= 1 && kk <= NC;
      double p[NEQ];
      if (inner || !G) {
        flow2prim<NEQ, MHD>(ua, p, P.ph.inv_cv);
        pp[s][q(i, j)] = p[4];
        pr[s][q(i, j)] = p[0];
      } else {
        pp[s][q(i, j)] = ua[1];
        pr[s][q(i, j)] = ua[0];
      }
      if (inner && t < 64) {
        if (!G) {
          flow2prim<NEQ, MHD>(ug, p, P.ph.inv_cv);
          pp[s][q(gi, gj)] = p[4];
          pr[s][q(gi, gj)] = p[0];
        } else {
          pp[s][q(gi, gj)] = ug[1];
          pr[s][q(gi, gj)] = ug[0];
        }
      }
    };
    fetch(0);
    commit(0);
    fetch(1);
    commit(1);
    fetch(2);
    for (int k = 1; k <= NC; ++k) {
      commit(k + 1);
      if (k + 2 <= NC + 1) fetch(k + 2);
      __syncthreads();
      const int sm = (k - 1) % 3, sc = k % 3, sp = (k + 1) % 3;
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        double (*a)[18 * 18] = v == 0 ? pp : pr;
        // the reference's gradient of a cell is max over the axes of
        // |delta|/c/(2 dx); correctly rounded division by the same positive
        // c, and by the block's 2 dx, is monotonic, so the largest |delta|
        // divided by c here, and the block's maximum of those divided by
        // 2 dx once below, give its maximum gradient bit for bit
        const double c = a[sc][q(i, j)];
        const double dx_ = fabs(a[sc][q(i + 1, j)] - a[sc][q(i - 1, j)]);
        const double dy_ = fabs(a[sc][q(i, j + 1)] - a[sc][q(i, j - 1)]);
        const double dz_ = fabs(a[sp][q(i, j)] - a[sm][q(i, j)]);
        lmax = dmax(lmax, dmax(dmax(dx_, dy_), dz_) / c);
      }
      __syncthreads();
    }
    for (int s = 16; s > 0; s >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, s));
    if ((t & 31) == 0) atomic_max_pos(reinterpret_cast<unsigned long long*>(&bmax), lmax);
    __syncthreads();
    if (t == 0) {
      // the reference stops at the first cell whose gradient reaches
      // refineThres (amr.f90:142-230): refinement depends only on whether
      // the largest gradient does; coarsening on the largest gradient
      const double gmax = bmax / (2 * B.dx);
      int flag;
      if (gmax >= P.refine_thres) flag = (B.level == P.maxlev) ? WX_FLAG_NONE : WX_FLAG_REFINE;
      else flag = (gmax <= P.coarse_thres && B.level > 1) ? WX_FLAG_COARSE : WX_FLAG_NONE;
      P.flags[slot] = flag;
    }
  }
}

// refineBlock data copy (amr.f90:355-367): child c (natural order) cell
// (i,j,k) <- father cell ((n/2)s + (i+1)/2, ...).
struct Slots8 {
  int32_t s[8];
};

__global__ void refine_kernel(double* __restrict__ u, int neq, int father, Slots8 ch) {
  const int cc = blockIdx.y;
  const int child = ch.s[cc];
  const int sx = cc & 1, sy = (cc >> 1) & 1, sz = (cc >> 2) & 1;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < BCELLS * neq; c += gridDim.x * blockDim.x) {
    const int e = c / BCELLS, r = c % BCELLS;
    const int i = (r & 15) + 1, j = ((r >> 4) & 15) + 1, k = (r >> 8) + 1;
    const int ip = 8 * sx + (i + 1) / 2, jp = 8 * sy + (j + 1) / 2, kp = 8 * sz + (k + 1) / 2;
    u[cell_off(child, neq, e, i, j, k)] = u[cell_off(father, neq, e, ip, jp, kp)];
  }
}

// coarseBlocks local branch (amr.f90:1597-1625): father cell <- Fortran SUM
// of the sibling's 2x2x2 cells (i fastest) / 8.
__global__ void coarsen_kernel(double* __restrict__ u, int neq, int father, Slots8 ch) {
  const int sib = blockIdx.y;
  const int child = ch.s[sib];
  const int sx = sib & 1, sy = (sib >> 1) & 1, sz = (sib >> 2) & 1;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < 512 * neq; c += gridDim.x * blockDim.x) {
    const int e = c / 512, r = c % 512;
    const int i = (r & 7) + 1, j = ((r >> 3) & 7) + 1, k = (r >> 6) + 1;
    const int i1 = 2 * i - 1, j1 = 2 * j - 1, k1 = 2 * k - 1;
    double s = 0.0;
    for (int kk = k1; kk <= k1 + 1; ++kk)
      for (int jj = j1; jj <= j1 + 1; ++jj)
        for (int ii = i1; ii <= i1 + 1; ++ii) s += u[cell_off(child, neq, e, ii, jj, kk)];
    u[cell_off(father, neq, e, i + 8 * sx, j + 8 * sy, k + 8 * sz)] = s / 8.0;
  }
}

// Batched forms for admesh: op = [father, child0..child7] (9 slots), one
// CTA row per (op, child) or (op, sibling).  A slot freed by one op may be
// taken by a later one, so the blocks a pass reads are first copied (same
// slots) into a scratch array by stage_blocks_kernel, and the pass reads the
// scratch and writes the state: no op writes what another op reads.
//
// stage_blocks_kernel copies, for every op, the `per` slots starting at
// entry `off` (the father: per 1, off 0; the siblings: per 8, off 1).
__global__ void stage_blocks_kernel(const double* __restrict__ from, double* __restrict__ to, int neq,
                                    const int32_t* __restrict__ ops, int per, int off) {
  const int item = blockIdx.y;
  const int slot = ops[9 * (item / per) + off + item % per];
  const size_t base = (size_t)slot * neq * BCELLS;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < BCELLS * neq; c += gridDim.x * blockDim.x)
    to[base + c] = from[base + c];
}

__global__ void refine_batch_kernel(const double* __restrict__ from, double* __restrict__ u, int neq,
                                    const int32_t* __restrict__ ops) {
  const int op = blockIdx.y >> 3, cc = blockIdx.y & 7;
  const int father = ops[9 * op], child = ops[9 * op + 1 + cc];
  const int sx = cc & 1, sy = (cc >> 1) & 1, sz = (cc >> 2) & 1;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < BCELLS * neq; c += gridDim.x * blockDim.x) {
    const int e = c / BCELLS, r = c % BCELLS;
    const int i = (r & 15) + 1, j = ((r >> 4) & 15) + 1, k = (r >> 8) + 1;
    const int ip = 8 * sx + (i + 1) / 2, jp = 8 * sy + (j + 1) / 2, kp = 8 * sz + (k + 1) / 2;
    u[cell_off(child, neq, e, i, j, k)] = from[cell_off(father, neq, e, ip, jp, kp)];
  }
}

__global__ void coarsen_batch_kernel(const double* __restrict__ from, double* __restrict__ u, int neq,
                                     const int32_t* __restrict__ ops) {
  const int op = blockIdx.y >> 3, sib = blockIdx.y & 7;
  const int father = ops[9 * op], child = ops[9 * op + 1 + sib];
  const int sx = sib & 1, sy = (sib >> 1) & 1, sz = (sib >> 2) & 1;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < 512 * neq; c += gridDim.x * blockDim.x) {
    const int e = c / 512, r = c % 512;
    const int i = (r & 7) + 1, j = ((r >> 3) & 7) + 1, k = (r >> 6) + 1;
    const int i1 = 2 * i - 1, j1 = 2 * j - 1, k1 = 2 * k - 1;
    double s = 0.0;
    for (int kk = k1; kk <= k1 + 1; ++kk)
      for (int jj = j1; jj <= j1 + 1; ++jj)
        for (int ii = i1; ii <= i1 + 1; ++ii) s += from[cell_off(child, neq, e, ii, jj, kk)];
    u[cell_off(father, neq, e, i + 8 * sx, j + 8 * sy, k + 8 * sz)] = s / 8.0;
  }
}

// Primitive variables of the physical cells (calcPrimsBlock CELLS_PHYS).
template <int NEQ, bool MHD>
__global__ void prims_kernel(const double* __restrict__ u, double* __restrict__ prim, const int32_t* __restrict__ work,
                             int nwork, DevCtl* ctl, double inv_cv) {
  unsigned pf = 0, df = 0, zd = 0;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int slot = work[w];
    for (int c = threadIdx.x; c < BCELLS; c += blockDim.x) {
      const size_t o = (size_t)slot * NEQ * BCELLS + c;
      double uu[NEQ], p[NEQ];
#pragma unroll
      for (int e = 0; e < NEQ; ++e) uu[e] = u[o + (size_t)e * BCELLS];
      const int st = flow2prim<NEQ, MHD>(uu, p, inv_cv);
      pf += (st == 1); df += (st == 2); zd += (st < 0);
#pragma unroll
      for (int e = 0; e < NEQ; ++e) prim[o + (size_t)e * BCELLS] = p[e];
    }
  }
  unsigned m = 0xffffffffu;
  pf = __reduce_add_sync(m, pf); df = __reduce_add_sync(m, df); zd = __reduce_add_sync(m, zd);
  if ((threadIdx.x & 31) == 0) {
    if (pf) atomicAdd(&ctl->cnt[0], (unsigned long long)pf);
    if (df) atomicAdd(&ctl->cnt[1], (unsigned long long)df);
    if (zd) atomicAdd(&ctl->cnt[2], (unsigned long long)zd);
  }
}

// Fortran U(nbMax, neq, -1:18, -1:18, -1:18) slab at one k (physical k = kf)
// <-> native [slot][eq][k][j][i].  The slab holds nbMax*neq*20*20 values.
__global__ void fortran_to_native(const double* __restrict__ slab, double* __restrict__ u, int nbmax, int nslots,
                                  int neq, int kf) {
  const long long n = (long long)nslots * neq * PLANE;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int nb = (int)(c % nslots);
    const long long r = c / nslots;
    const int e = (int)(r % neq);
    const int ij = (int)(r / neq);
    const int i = (ij & 15) + 1, j = (ij >> 4) + 1;
    u[cell_off(nb, neq, e, i, j, kf)] = slab[nb + (size_t)nbmax * (e + (size_t)neq * ((i + 1) + 20 * (j + 1)))];
  }
}

__global__ void native_to_fortran(const double* __restrict__ u, double* __restrict__ slab, int nbmax, int nslots,
                                  int neq, int kf) {
  const long long n = (long long)nslots * neq * PLANE;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int nb = (int)(c % nslots);
    const long long r = c / nslots;
    const int e = (int)(r % neq);
    const int ij = (int)(r / neq);
    const int i = (ij & 15) + 1, j = (ij >> 4) + 1;
    slab[nb + (size_t)nbmax * (e + (size_t)neq * ((i + 1) + 20 * (j + 1)))] = u[cell_off(nb, neq, e, i, j, kf)];
  }
}

// writeBin / warmstart (output.f90:156-213, init.f90:527-623) store each
// block as U(nb, :, 1:16, 1:16, 1:16): the equation index fastest, then i,
// j, k.  pack: slots slot0.. of the native state -> nb consecutive blocks
// of that order; unpack: the reverse.
// The four cell layers of a block next to one of its faces (item = slot,
// face 0..5 = left, right, front, back, bottom, top), neq x 4 x 16 x 16
// doubles per item: per equation the layers in index order along the face
// normal, then the two transverse indices; pack copies them from `a` to
// `buf`, unpack back.
constexpr int FACE_LAYERS = 4;
__global__ void face_slab_kernel(double* __restrict__ a, const int32_t* __restrict__ items, int neq,
                                 double* __restrict__ buf, int pack) {
  const int item = blockIdx.y;
  const int slot = items[2 * item], f = items[2 * item + 1];
  const int ax = f >> 1, side = f & 1;
  const int per = neq * FACE_LAYERS * NC * NC;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < per; c += gridDim.x * blockDim.x) {
    const int e = c / (FACE_LAYERS * NC * NC), r = c % (FACE_LAYERS * NC * NC);
    const int l = r / (NC * NC), t2 = (r / NC) % NC + 1, t1 = r % NC + 1;
    const int g = side ? NC - FACE_LAYERS + 1 + l : 1 + l;
    const int i = ax == 0 ? g : t1, j = ax == 1 ? g : (ax == 0 ? t1 : t2), k = ax == 2 ? g : t2;
    double* cell = a + cell_off(slot, neq, e, i, j, k);
    double* b = buf + (size_t)item * per + c;
    if (pack) *b = *cell;
    else *cell = *b;
  }
}

__global__ void pack_bin_kernel(const double* __restrict__ u, const int32_t* __restrict__ slots, int nb, int neq,
                                double* __restrict__ out) {
  const long long n = (long long)nb * BCELLS * neq;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q % neq);
    const long long cell = q / neq;           // block-major, then k, j, i (i fastest)
    const int b = (int)(cell / BCELLS), c = (int)(cell % BCELLS);
    out[q] = u[((size_t)slots[b] * neq + e) * BCELLS + c];
  }
}

__global__ void unpack_bin_kernel(const double* __restrict__ in, int slot0, int nb, int neq, double* __restrict__ u) {
  const long long n = (long long)nb * BCELLS * neq;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q % neq);
    const long long cell = q / neq;
    const int b = (int)(cell / BCELLS), c = (int)(cell % BCELLS);
    u[((size_t)(slot0 + b) * neq + e) * BCELLS + c] = in[q];
  }
}

}  // namespace wx
