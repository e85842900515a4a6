// wx3d_api.cu -- C-ABI of the B200 per-block Godunov update (include/wx3d.h).
//
// Host side: context, neighbour-table construction from the localBlocks
// registry (restating the bID arithmetic of source/amr.f90:439-1098),
// uploads and downloads, and the step sequence of source/main.f90:81-100
// enqueued on one CUDA stream (replayed from a CUDA graph by wx3d_run).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <queue>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/wx3d.h"
#include "wx3d_internal.h"
#include "wx3d_kernels.cuh"
#include "wx3d_source.cuh"


using namespace wx;

namespace {

// ---------------------------------------------------------------------------
// Kernel table per (neq, mhd, solver)

struct Kern {
  void (*stage1)(StageParams) = nullptr;
  void (*stage2)(StageParams) = nullptr;
  void (*stage2v)(StageParams) = nullptr;  // corrector with the viscous step fused
  void (*lax)(LaxParams) = nullptr;
  void (*visc)(ViscParams) = nullptr;
  void (*dt)(DtParams) = nullptr;
  void (*wind)(WindParams) = nullptr;
  void (*src)(SrcParams) = nullptr;
  void (*mark)(MarkParams) = nullptr;
  void (*prims)(const double*, double*, const int32_t*, int, DevCtl*, double) = nullptr;
  size_t smem1 = 0;  // dynamic shared memory of the predictor and the corrector
  size_t smem2 = 0;
  size_t smem2v = 0;
};

template <int NEQ, bool MHD, int SOLVER, int LIM>
Kern make_kern() {
  Kern k;
  k.stage1 = stage_kernel<NEQ, MHD, SOLVER, 1, LIM_RUNTIME>;
  k.stage2 = stage_kernel<NEQ, MHD, SOLVER, 2, LIM>;
  k.stage2v = stage_kernel<NEQ, MHD, SOLVER, 2, LIM, true>;
  k.lax = lax_kernel<NEQ, MHD>;
  k.visc = viscous_kernel<NEQ, MHD>;
  k.dt = dt_kernel<NEQ, MHD>;
  k.wind = wind_kernel<NEQ, MHD>;
  k.src = source_kernel<NEQ, MHD>;
  k.mark = mark_kernel<NEQ, MHD>;
  k.prims = prims_kernel<NEQ, MHD>;
  k.smem1 = stage_smem_bytes<NEQ, MHD, 1>();
  k.smem2 = stage_smem_bytes<NEQ, MHD, 2>();
  k.smem2v = stage_smem_bytes<NEQ, MHD, 2, true>();
  return k;
}

// Limiters compiled into the corrector for the common cases; the others use
// the run-time switch.
template <int NEQ, bool MHD, int SOLVER>
Kern make_kern_lim(int lim) {
  if constexpr (NEQ == 5) {
    if (lim == WX_LIMITER_VANLEER) return make_kern<NEQ, MHD, SOLVER, WX_LIMITER_VANLEER>();
    if (lim == WX_LIMITER_SUPERBEE) return make_kern<NEQ, MHD, SOLVER, WX_LIMITER_SUPERBEE>();
  }
  if (lim == WX_LIMITER_MINMOD) return make_kern<NEQ, MHD, SOLVER, WX_LIMITER_MINMOD>();
  return make_kern<NEQ, MHD, SOLVER, LIM_RUNTIME>();
}

// The source kernel compiled for the radiative runs' source terms
// (EOS_H_RATE with COOL_H or COOL_TABLE) where the configuration has them.
template <int NEQ>
void pick_source_kernel(const wx_config& c, Kern& k) {
  if (c.eos_type != WX_EOS_H_RATE || c.npassive < 1) return;
  if (c.cooling_type == WX_COOL_H) k.src = source_kernel<NEQ, false, 1>;
  if (c.cooling_type == WX_COOL_TABLE) k.src = source_kernel<NEQ, false, 2>;
}

// Supported combinations: hydro with 0..2 passives (HLL/HLL1/HLLC/LAX) and
// ideal MHD without passives (HLL/HLL1/HLLE/HLLD/LAX).
bool select_kern(const wx_config& c, Kern& k) {
  const bool mhd = c.bfield != 0;
  const int s = c.solver_type;
  const int rs = (s == WX_SOLVER_HLL1 || s == WX_SOLVER_LAX) ? WX_SOLVER_HLL : s;
  const int lim = c.limiter_type;
  if (!mhd) {
    if (rs != WX_SOLVER_HLL && rs != WX_SOLVER_HLLC) return false;
    const bool c_ = rs == WX_SOLVER_HLLC;
    switch (c.neqtot) {
      case 5: k = c_ ? make_kern_lim<5, false, WX_SOLVER_HLLC>(lim) : make_kern_lim<5, false, WX_SOLVER_HLL>(lim); return true;
      case 6:
        k = c_ ? make_kern_lim<6, false, WX_SOLVER_HLLC>(lim) : make_kern_lim<6, false, WX_SOLVER_HLL>(lim);
        pick_source_kernel<6>(c, k);
        return true;
      case 7:
        k = c_ ? make_kern_lim<7, false, WX_SOLVER_HLLC>(lim) : make_kern_lim<7, false, WX_SOLVER_HLL>(lim);
        pick_source_kernel<7>(c, k);
        return true;
      default: return false;
    }
  }
  if (c.neqtot != 8) return false;
  switch (rs) {
    case WX_SOLVER_HLL: k = make_kern<8, true, WX_SOLVER_HLL, LIM_RUNTIME>(); return true;
    case WX_SOLVER_HLLE: k = make_kern<8, true, WX_SOLVER_HLLE, LIM_RUNTIME>(); return true;
    case WX_SOLVER_HLLD: k = make_kern<8, true, WX_SOLVER_HLLD, LIM_RUNTIME>(); return true;
    default: return false;
  }
}

// ---------------------------------------------------------------------------
// Block tree arithmetic (source/amr.f90), independent of the process layout.

struct Tree {
  int nbroot[3] = {1, 1, 1};
  int maxlev = 1;
  int nb[WX3D_MAX_LEVELS + 2][3] = {};
  long long minID[WX3D_MAX_LEVELS + 2] = {}, maxID[WX3D_MAX_LEVELS + 2] = {};

  void init(const wx_config& c) {  // init.f90:733-756
    nbroot[0] = c.nbrootx; nbroot[1] = c.nbrooty; nbroot[2] = c.nbrootz;
    maxlev = c.maxlev;
    long long acc = 0;
    for (int l = 1; l <= maxlev; ++l) {
      for (int d = 0; d < 3; ++d) nb[l][d] = nbroot[d] << (l - 1);
      long long n = (long long)nb[l][0] * nb[l][1] * nb[l][2];
      minID[l] = acc + 1;
      maxID[l] = acc + n;
      acc += n;
    }
  }
  __host__ __device__ int level(long long bID) const {  // meshlevel, amr.f90:637
    for (int l = 1; l <= maxlev; ++l) if (bID >= minID[l] && bID <= maxID[l]) return l;
    return -1;
  }
  __host__ __device__ void coords(long long bID, int l, int x[3]) const {  // bcoords, amr.f90:972 (0-based here)
    long long loc = bID - minID[l];
    x[0] = (int)(loc % nb[l][0]);
    x[1] = (int)((loc / nb[l][0]) % nb[l][1]);
    x[2] = (int)(loc / ((long long)nb[l][0] * nb[l][1]));
  }
  __host__ __device__ long long id(int l, const int x[3]) const {
    return minID[l] + x[0] + (long long)nb[l][0] * (x[1] + (long long)nb[l][1] * x[2]);
  }
};

// bID -> slot for the neighbour-table build and admesh's slot registry: open
// addressing with linear probing in a power-of-two table at most half full,
// deletion by backward shift (no tombstones), so every lookup is a short
// scan of one cache line or two.
class SlotMap {
 public:
  explicit SlotMap(size_t n) {
    int bits = 4;
    while ((size_t(1) << bits) < 2 * n + 16) ++bits;
    shift_ = 64 - bits;
    mask_ = (size_t(1) << bits) - 1;
    key_.assign(mask_ + 1, -1);
    val_.assign(mask_ + 1, -1);
  }
  int find(long long k) const {  // -1 if absent; keys are bIDs >= 1
    if (k < 0) return -1;
    for (size_t i = home(k);; i = (i + 1) & mask_) {
      if (key_[i] == k) return val_[i];
      if (key_[i] == -1) return -1;
    }
  }
  bool insert(long long k, int v) {  // false if k is present
    for (size_t i = home(k);; i = (i + 1) & mask_) {
      if (key_[i] == k) return false;
      if (key_[i] == -1) {
        key_[i] = k;
        val_[i] = v;
        ++n_;
        return true;
      }
    }
  }
  void erase(long long k) {
    size_t i = home(k);
    while (key_[i] != k) {
      if (key_[i] == -1) return;
      i = (i + 1) & mask_;
    }
    for (size_t j = i;;) {  // shift back the entries of the run that may fill the hole
      j = (j + 1) & mask_;
      if (key_[j] == -1) break;
      if (((j - home(key_[j])) & mask_) >= ((j - i) & mask_)) {
        key_[i] = key_[j];
        val_[i] = val_[j];
        i = j;
      }
    }
    key_[i] = -1;
    val_[i] = -1;
    --n_;
  }
  size_t size() const { return n_; }

 private:
  size_t home(long long k) const { return (size_t)(((unsigned long long)k * 0x9E3779B97F4A7C15ull) >> shift_); }
  std::vector<long long> key_;
  std::vector<int> val_;
  size_t mask_ = 0, n_ = 0;
  int shift_ = 60;
};

}  // namespace

// ---------------------------------------------------------------------------

struct wx_ctx {
  wx_config cfg{};
  PhysParams ph{};
  Kern k;
  int neq = 5;
  int max_blocks = 0;
  int dev = 0, nsm = 148;
  cudaStream_t own = nullptr, stream = nullptr;
  double* dU = nullptr;
  double* dUP = nullptr;
  double* dW = nullptr;
  double* dPrim = nullptr;
  double* dStage = nullptr;  // staging slab for the Fortran layout
  size_t stage_bytes = 0;
  DevBlock* dBlocks = nullptr;
  // neighbour-table build on the device (meshes without halo slots or wind
  // sources): the new table goes to dBlocksNext and is swapped in on commit
  DevBlock* dBlocksNext = nullptr;
  int2* dHash = nullptr;          // bID -> slot, open addressing, hash_size entries
  unsigned hash_size = 0;
  int32_t* dLbBuf = nullptr;      // the slot list being built
  int32_t* dMeshErr = nullptr;    // [3] first failing slots, then max_blocks face codes
  bool next_on_device = false;    // the next table was built on the device
  bool host_table_stale = false;  // hblocks lags dBlocks (built on the device)
  int32_t* dWork = nullptr;
  int32_t* dFlags = nullptr;
  int32_t* dOps = nullptr;   // admesh: refine/coarsen operations, 9 slots each
  int32_t* dItems = nullptr; // face-slab exchange: (slot, face) pairs
  DevCtl* dCtl = nullptr;
  DevCtl* hCtl = nullptr;   // pinned mirror
  double* dCool = nullptr;  // COOL_TABLE [2][ncool]; METAL [ncool+1][nZ+1]; SCHURE [2][180]
  int ncool = 0;
  int nZ = 0;
  Tree tree;
  std::vector<int32_t> local;     // localBlocks
  std::vector<int32_t> work;      // occupied slots
  DevBlock* hblocks = nullptr;       // host copy of the device neighbour table (pinned)
  DevBlock* hblocks_next = nullptr;  // pinned buffer the next table is built in, then swapped in
  std::vector<double> hwind;      // wind sources, 12 doubles each (wx_wind)
  double* dWind = nullptr;
  // Wind runs: the blocks a sphere reaches get a copy with the wind imposed
  // in slots past max_blocks of dU, and the first stage gathers its ghosts
  // through dBlocksWind, a neighbour table that points there.
  int slot_cap = 0;                 // slots allocated in dU and dW
  bool wind_ready = false;          // dBlocksWind and the lists match the mesh and the winds
  int nwslot = 0;                   // reached blocks, copied each step
  int wind_cap = 0;                 // entries allocated in the three arrays below
  DevBlock* dBlocksWind = nullptr;  // [max_blocks + wind_cap]
  int2* dWindPairs = nullptr;       // (slot, extra slot) of each reached block
  int32_t* dWindWork = nullptr;     // the extra slots
  int nwork = 0;
  bool mesh_set = false;  // a mesh was set; it may hold no blocks (localBlocks all -1)
  int zsplit = 1;
  bool fuse = true;   // corrector carries the viscous step when zsplit == 1
  int zero_ghost = 0; // single-stage solver: the viscous step sees zero UP ghosts
  int nhalo = 0;      // slots that hold copies of other processes' blocks
  int grid_stage = 0, grid_256 = 0;
  bool dt_valid = false;
  bool prestep = false;           // dW holds the state at the start of the last step
  // ghost primitives for markByPhysical, left by the first-order stage once
  // admesh is in use (GFRAME x (rho, p) per slot)
  double* dG = nullptr;
  bool mark_ghosts = false;       // the first-order stage writes dG
  bool g_step = false;            // the step being enqueued writes dG
  bool g_valid = false;           // dG holds the ghosts of the state in dW (with prestep)
  cudaGraphExec_t graph = nullptr;
  bool graph_valid = false;
  long long launches = 0;
  // learned surrogate of hrate + cooling_h (wx3d_set_surrogate)
  const wx_mlp* mlp = nullptr;
  uint8_t* dTrust = nullptr;
  bool use_surrogate = false;
  // per-kernel timing: event pairs around the launches of one step sequence
  bool timing = false;
  bool timing_mute = false;
  cudaEvent_t ev[64] = {};
  int ev_kind[32] = {};
  int nev = 0;
  std::string err;
};

namespace {

int fail(wx_ctx* c, int code, const char* fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

#define WX_CUDA(call)                                                                           \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return fail(c, WX_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

#define WX_LAUNCHED()                                                                     \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) return fail(c, WX_ERR_CUDA, "launch: %s", cudaGetErrorString(e_)); \
    ++c->launches;                                                                        \
  } while (0)

int validate(const wx_config& f, std::string& why) {
  if (f.neqtot != 5 + 3 * (f.bfield ? 1 : 0) + f.npassive) { why = "neqtot != 5 + 3*bfield + npassive"; return WX_ERR_INVALID_ARG; }
  if (f.neqtot > WX3D_MAX_NEQ) { why = "neqtot too large"; return WX_ERR_INVALID_ARG; }
  if (f.maxlev < 1 || f.maxlev > WX3D_MAX_LEVELS) { why = "maxlev out of 1..10"; return WX_ERR_TOO_MANY_LEVS; }
  if (f.nbrootx < 1 || f.nbrooty < 1 || f.nbrootz < 1) { why = "root block counts must be >= 1"; return WX_ERR_INVALID_ARG; }
  if (f.mhd && !f.bfield) { why = "mhd without bfield computes no time step in the reference"; return WX_ERR_UNSUPPORTED; }
  if (f.bfield && !f.mhd) { why = "passive magnetic field (bfield without mhd) is not supported"; return WX_ERR_UNSUPPORTED; }
  if (f.user_source_terms) { why = "user source terms are not part of this ABI"; return WX_ERR_UNSUPPORTED; }
  if (f.enable_flux_cd) {
    if (!(f.bfield && f.mhd)) { why = "enable_flux_cd needs an active magnetic field (bfield and mhd)"; return WX_ERR_UNSUPPORTED; }
    if (f.eight_wave) { why = "enable_flux_cd and eight_wave are alternative div(B) controls (init.f90:264-270): pick one"; return WX_ERR_UNSUPPORTED; }
    if (f.solver_type == WX_SOLVER_LAX) { why = "the field-CD update replaces upwindStep, which the Lax-Friedrichs solver does not use"; return WX_ERR_UNSUPPORTED; }
  }
  for (int i = 0; i < 6; ++i) {
    if (f.bc[i] == WX_BC_PERIODIC) { why = "BC_PERIODIC is not implemented by the reference (ghosts stay stale)"; return WX_ERR_UNSUPPORTED; }
    if (f.bc[i] != WX_BC_REFLECTIVE && f.bc[i] != WX_BC_FREE_FLOW) { why = "unknown boundary condition"; return WX_ERR_INVALID_ARG; }
  }
  if ((f.eos_type == WX_EOS_H_RATE || f.cooling_type == WX_COOL_H) && f.npassive < 1) { why = "H-rate EOS / COOL_H need a passive scalar"; return WX_ERR_NOT_ENOUGH_PASSIVES; }
  if (f.cooling_type < WX_COOL_NONE || f.cooling_type > WX_COOL_SCHURE) { why = "unknown cooling type"; return WX_ERR_INVALID_ARG; }
  if (f.gamma <= 1.0) { why = "gamma must exceed 1"; return WX_ERR_INVALID_ARG; }
  return WX_OK;
}

void fill_phys(wx_ctx* c) {
  const wx_config& f = c->cfg;
  PhysParams& p = c->ph;
  p.gamma = f.gamma;
  p.cv = 1.0 / (f.gamma - 1.0);           // parameters.f90:373
  p.inv_cv = 1.0 / p.cv;
  p.cfl = f.cfl;
  p.eta = f.visc_eta;
  p.mu0 = f.mu0; p.mui = f.mui; p.ion_thres = f.ion_thres;
  p.d_sc = f.d_sc;
  p.p_sc = f.d_sc * (f.v_sc * f.v_sc);    // parameters.f90:379
  p.e_sc = p.p_sc;                        // :380
  p.t_sc = f.l_sc / f.v_sc;               // :381
  p.dtout = f.dtout;
  p.cooling_limit = f.cooling_limit;
  p.limiter = f.limiter_type;
  p.eight_wave = f.eight_wave;
  p.flux_cd = f.enable_flux_cd;
  for (int i = 0; i < 6; ++i) p.bc[i] = f.bc[i];
  p.eos = f.eos_type;
  p.cooling = f.cooling_type;
  p.fp = 5 + 3 * (f.bfield ? 1 : 0);
  p.npassive = f.npassive;
  p.l_sc = f.l_sc;
  p.v_sc = f.v_sc;
  p.wind = c->dWind;
  p.nwind = (int32_t)(c->hwind.size() / 12);
}

// Flags the blocks whose cells, ghost layers included, a wind sphere
// reaches (cell centres from cellPos, amr.f90:1037-1065).  Returns false
// (with the slot in *bad) if a sphere reaches the ghost layer of a face
// with a coarser or finer neighbour, or of the domain boundary: those
// ghosts would need the wind at their own positions (or their sources the
// values before it), which only a same-level neighbour provides.
bool flag_wind_blocks(const wx_ctx* c, DevBlock* hb, size_t n, int* bad) {
  const size_t nw = c->hwind.size() / 12;
  const double l_sc = c->cfg.l_sc;
  auto reach = [&](const double* W, const double* lo, const double* hi) {
    double s = 0.0;
    for (int ax = 0; ax < 3; ++ax) {
      const double q = W[ax] < lo[ax] ? lo[ax] - W[ax] : (W[ax] > hi[ax] ? W[ax] - hi[ax] : 0.0);
      s += q * q;
    }
    return std::sqrt(s) <= W[6] * (1.0 + 1e-12);
  };
  for (size_t s = 0; s < n; ++s) {
    DevBlock& b = hb[s];
    b.wind = 0;
    if (b.level < 1 || nw == 0) continue;
    const double d[3] = {b.dx, b.dy, b.dz};
    double lo[3], hi[3];
    for (int ax = 0; ax < 3; ++ax) {   // cells -1 .. 18 (their volumes)
      lo[ax] = ((b.bc[ax] - 1) * NC - 2) * d[ax] * l_sc;
      hi[ax] = ((b.bc[ax] - 1) * NC + 18) * d[ax] * l_sc;
    }
    for (size_t w = 0; w < nw; ++w) {
      const double* W = &c->hwind[12 * w];
      if (!reach(W, lo, hi)) continue;
      b.wind = 1;
      for (int f = 0; f < 6; ++f) {
        if (b.ftype[f] != WX_NEIGH_COARSER && b.ftype[f] != WX_NEIGH_FINER && b.ftype[f] != WX_NEIGH_BOUNDARY) continue;
        const int ax = f / 2, side = f & 1;
        double glo[3], ghi[3];
        // the volume of the face's two ghost layers: it holds the ghost
        // centres and every neighbour cell a coarse/fine ghost is made from
        for (int a2 = 0; a2 < 3; ++a2) {
          const double base = (b.bc[a2] - 1) * NC;
          if (a2 == ax) {
            glo[a2] = (side ? base + 16 : base - 2) * d[a2] * l_sc;
            ghi[a2] = (side ? base + 18 : base) * d[a2] * l_sc;
          } else {
            glo[a2] = base * d[a2] * l_sc;
            ghi[a2] = (base + 16) * d[a2] * l_sc;
          }
        }
        if (reach(W, glo, ghi)) {
          if (bad) *bad = (int)s;
          return false;
        }
      }
    }
  }
  return true;
}

bool sources_on(const wx_ctx* c) { return c->cfg.eos_type == WX_EOS_H_RATE || c->cfg.cooling_type != WX_COOL_NONE; }

// kinds: 0 stage1, 1 stage2 (or the single stage), 2 viscous, 3 sources
void tick(wx_ctx* c, int kind, bool begin) {
  if (!c->timing || c->timing_mute || c->nev >= 64) return;
  if (begin) c->ev_kind[c->nev / 2] = kind;
  // external record: inside a stream capture this becomes an event-record
  // node of the graph, so the replay itself stamps the event; outside a
  // capture the flag is not allowed and a plain record is used
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(c->stream, &cs);
  cudaEventRecordWithFlags(c->ev[c->nev], c->stream,
                           cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault);
  ++c->nev;
}

int grid_for(wx_ctx* c, const void* fn, int threads, size_t smem, int items) {
  int per = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem);
  per = std::max(per, 1);
  return std::max(1, std::min(items, per * c->nsm));
}

int set_stage_attrs(wx_ctx* c) {
  WX_CUDA(cudaFuncSetAttribute(c->k.stage1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->k.smem1));
  WX_CUDA(cudaFuncSetAttribute(c->k.stage2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->k.smem2));
  WX_CUDA(cudaFuncSetAttribute(c->k.stage2v, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->k.smem2v));
  return WX_OK;
}

// ---- step pieces -------------------------------------------------------------

int launch_dt(wx_ctx* c, const double* u) {
  ctl_reset_dtmin_kernel<<<1, 1, 0, c->stream>>>(c->dCtl);
  WX_LAUNCHED();
  DtParams P{u, c->dBlocks, c->dWork, c->nwork, c->dCtl, c->ph};
  c->k.dt<<<grid_for(c, (const void*)c->k.dt, 256, 0, c->nwork), 256, 0, c->stream>>>(P);
  WX_LAUNCHED();
  return WX_OK;
}

int launch_wind(wx_ctx* c, double* u, const DevBlock* blocks = nullptr, const int32_t* work = nullptr, int nwork = -1) {
  if (c->hwind.empty()) return WX_OK;
  if (nwork < 0) nwork = c->nwork;
  WindParams P{u, blocks ? blocks : c->dBlocks, work ? work : c->dWork, nwork, c->ph};
  c->k.wind<<<grid_for(c, (const void*)c->k.wind, 256, 0, nwork), 256, 0, c->stream>>>(P);
  WX_LAUNCHED();
  return WX_OK;
}

// fused: the corrector that also applies doViscousStep (whole blocks only)
int launch_stage(wx_ctx* c, int order, const double* src, const double* base, double* out, double factor,
                 bool fused = false, const double* gsrc = nullptr, const DevBlock* blocks = nullptr) {
  StageParams P{src, base, out, blocks ? blocks : c->dBlocks, c->dWork, c->nwork * c->zsplit, c->zsplit, c->dCtl, factor, c->ph,
                sources_on(c) ? 0 : 1, gsrc ? gsrc : src, order == 1 && c->g_step ? c->dG : nullptr};
  auto fn = order == 1 ? c->k.stage1 : (fused ? c->k.stage2v : c->k.stage2);
  const size_t smem = order == 1 ? c->k.smem1 : (fused ? c->k.smem2v : c->k.smem2);
  const int grid = grid_for(c, (const void*)fn, STAGE_THREADS, smem, c->nwork * c->zsplit);
  const int kind = (order == 2 || factor == 1.0) ? 1 : 0;
  WX_CUDA(cudaMemsetAsync(&c->dCtl->work_next[order - 1], 0, sizeof(unsigned), c->stream));
  tick(c, kind, true);
  fn<<<grid, STAGE_THREADS, smem, c->stream>>>(P);
  WX_LAUNCHED();
  tick(c, kind, false);
  return WX_OK;
}

// doViscousStep in place on w (the stage result), UP ghosts (zero for
// single-stage solvers)
int launch_visc(wx_ctx* c, int zero_ghost, double* w = nullptr) {
  ViscParams V{w ? w : c->dW, c->dUP, c->dBlocks, c->dWork, c->nwork, zero_ghost, sources_on(c) ? 0 : 1, c->dCtl, c->ph};
  tick(c, 2, true);
  c->k.visc<<<grid_for(c, (const void*)c->k.visc, 256, 0, c->nwork), 256, 0, c->stream>>>(V);
  WX_LAUNCHED();
  tick(c, 2, false);
  return WX_OK;
}

// The corrector carries the viscous step when every block is one slab.
bool fuse_visc(const wx_ctx* c) {
  const int s = c->cfg.solver_type;
  return c->fuse && c->zsplit == 1 && s != WX_SOLVER_LAX && s != WX_SOLVER_HLL1;
}

// The first stage: Godunov's predictor (dt/2), or the single stage of HLL1
// and Lax-Friedrichs (result in W).
int solver_first(wx_ctx* c) {
  const int solver = c->cfg.solver_type;
  int rc;
  c->zero_ghost = 0;
  if (solver == WX_SOLVER_LAX) {
    LaxParams P{c->dU, c->dW, c->dBlocks, c->dWork, c->nwork, c->dCtl, c->ph};
    tick(c, 1, true);
    c->k.lax<<<grid_for(c, (const void*)c->k.lax, 256, 0, c->nwork), 256, 0, c->stream>>>(P);
    WX_LAUNCHED();
    tick(c, 1, false);
    c->zero_ghost = 1;
  } else if (solver == WX_SOLVER_HLL1) {
    if ((rc = launch_stage(c, 1, c->dU, c->dU, c->dW, 1.0))) return rc;
    c->zero_ghost = 1;
  } else {
    if ((rc = launch_stage(c, 1, c->dU, c->dU, c->dUP, 0.5))) return rc;
  }
  return WX_OK;
}

// The corrector (two-stage solvers), doViscousStep, time += dt, and the
// U/W swap: on return dU holds U^{n+1}.
int solver_second(wx_ctx* c, bool finish_output) {
  const int solver = c->cfg.solver_type;
  int rc;
  if (solver != WX_SOLVER_LAX && solver != WX_SOLVER_HLL1 &&
      (rc = launch_stage(c, 2, c->dUP, c->dU, c->dW, 1.0, fuse_visc(c))))
    return rc;
  if (!fuse_visc(c) && (rc = launch_visc(c, c->zero_ghost))) return rc;
  step_end_kernel<<<1, 1, 0, c->stream>>>(c->dCtl, finish_output ? 1 : 0);
  WX_LAUNCHED();
  std::swap(c->dU, c->dW);
  c->prestep = true;
  c->g_valid = c->g_step;
  c->g_step = false;   // other first-order launches (the autotuner's) leave the record alone
  c->dt_valid = !sources_on(c);
  return WX_OK;
}

// Godunov(order)/LaxFriedrichs + doViscousStep; on return dU holds U^{n+1}.
int enqueue_solver(wx_ctx* c, bool bump_it, bool finish_output) {
  const bool src = sources_on(c);
  c->g_step = c->mark_ghosts && c->dG && c->hwind.empty() && c->cfg.solver_type != WX_SOLVER_LAX;
  step_begin_kernel<<<1, 1, 0, c->stream>>>(c->dCtl, c->ph.cfl, c->cfg.cooling_type != WX_COOL_NONE, c->ph.dtout,
                                            c->ph.t_sc, bump_it ? 1 : 0);
  WX_LAUNCHED();
  int rc;
  if (!c->hwind.empty()) {
    if (!c->wind_ready) return fail(c, WX_ERR_GENERIC, "wind sources without their redirected neighbour table");
    // Wind run (userBoundary after every ghost fill, winds.f90:123-240).
    // Stage 1 of godunov.f90 refreshes only the ghost primitives after
    // boundary(1, U): the physical cells feed their fluxes with the
    // primitives of U before the wind, the ghosts see it.  The blocks a
    // sphere reaches are copied into extra slots and take the wind there;
    // stage 1 reads its own cells from U and gathers its ghosts through
    // dBlocksWind, which points at those copies.  Then U takes the wind in
    // place and is the base of stage 2; boundary(2, UP) imposes the wind on
    // UP's physical cells.  The result goes to W and the buffers swap.
    if (c->nwslot > 0) {
      for (int r = 0; r < c->nwslot; r += 65535) {  // grid y limit
        copy_slots_kernel<<<dim3(16, std::min(65535, c->nwslot - r)), 256, 0, c->stream>>>(c->dU, c->dWindPairs + r,
                                                                                          c->neq);
        WX_LAUNCHED();
      }
      if ((rc = launch_wind(c, c->dU, c->dBlocksWind, c->dWindWork, c->nwslot))) return rc;
    }
    if ((rc = launch_stage(c, 1, c->dU, c->dU, c->dUP, 0.5, false, nullptr, c->nwslot > 0 ? c->dBlocksWind : nullptr)))
      return rc;
    if ((rc = launch_wind(c, c->dUP))) return rc;
    if ((rc = launch_wind(c, c->dU))) return rc;
    if ((rc = launch_stage(c, 2, c->dUP, c->dU, c->dW, 1.0, fuse_visc(c)))) return rc;
    if (!fuse_visc(c) && (rc = launch_visc(c, 0, c->dW))) return rc;
    step_end_kernel<<<1, 1, 0, c->stream>>>(c->dCtl, finish_output ? 1 : 0);
    WX_LAUNCHED();
    std::swap(c->dU, c->dW);
    c->prestep = true;
    c->g_valid = false;
    c->dt_valid = !src;
    return WX_OK;
  }
  if ((rc = solver_first(c))) return rc;
  return solver_second(c, finish_output);
}

// mode bits: 1 = hrate, 2 = cooling, 4 = read/write the PRIM buffer, 8 = CFL minimum
int enqueue_sources(wx_ctx* c, int mode) {
  if (mode & 8) {
    ctl_reset_dtmin_kernel<<<1, 1, 0, c->stream>>>(c->dCtl);
    WX_LAUNCHED();
  }
  SrcParams P{c->dU, (mode & 4) ? c->dPrim : nullptr, c->dBlocks, c->dWork, c->nwork, mode, c->dCtl,
              c->dCool, c->dCool ? c->dCool + c->ncool : nullptr, c->ncool, c->ph, c->nZ};
  tick(c, 3, true);
  // one CTA per block: the hardware hands blocks to SMs as CTAs finish, and
  // blocks of hot cells (the full Biro et al. loss) cost more than cold ones
  c->k.src<<<std::max(1, c->nwork), 256, 0, c->stream>>>(P);
  WX_LAUNCHED();
  tick(c, 3, false);
  if (mode & 8) c->dt_valid = true;
  return WX_OK;
}

int enqueue_surrogate(wx_ctx* c) {
  ctl_reset_dtmin_kernel<<<1, 1, 0, c->stream>>>(c->dCtl);
  WX_LAUNCHED();
  SurrLaunch L{c->neq, c->dU, c->dBlocks, c->dWork, c->nwork, c->dCtl, c->ph, c->mlp, c->dTrust, 1, c->nsm,
               c->dCool, c->dCool ? c->dCool + c->ncool : nullptr, c->ncool, c->nZ};
  tick(c, 3, true);
  const cudaError_t e = launch_surrogate_source(L, c->stream);
  if (e != cudaSuccess) return fail(c, WX_ERR_CUDA, "surrogate launch: %s", cudaGetErrorString(e));
  ++c->launches;
  tick(c, 3, false);
  c->dt_valid = true;
  return WX_OK;
}

int enqueue_step(wx_ctx* c) {
  int rc;
  if (!c->dt_valid) {
    if ((rc = launch_dt(c, c->dU))) return rc;
    c->dt_valid = true;
  }
  if ((rc = enqueue_solver(c, true, true))) return rc;
  if (c->use_surrogate) return enqueue_surrogate(c);
  if (sources_on(c)) {
    int mode = 8;
    if (c->cfg.eos_type == WX_EOS_H_RATE) mode |= 1;
    if (c->cfg.cooling_type != WX_COOL_NONE) mode |= 2;
    if ((rc = enqueue_sources(c, mode))) return rc;
  }
  return WX_OK;
}

int sync_check(wx_ctx* c) {
  WX_CUDA(cudaMemcpyAsync(c->hCtl, c->dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  if (c->hCtl->cnt[2]) return fail(c, WX_ERR_DIVISION_BY_ZERO, "zero density in flow2prim (%llu cells)", c->hCtl->cnt[2]);
  if (c->hCtl->cnt[3]) return fail(c, WX_ERR_NAN, "non-finite state after the step (%llu values)", c->hCtl->cnt[3]);
  return WX_OK;
}

void invalidate_graph(wx_ctx* c) {
  if (c->graph) cudaGraphExecDestroy(c->graph);
  c->graph = nullptr;
  c->graph_valid = false;
}

// A process whose localBlocks are all -1 still steps: its loops find no
// block, its local dt is 1e30*CFL and time advances with the others
// (getTimestep, hydro_solver.f90:145-205).
bool ready(wx_ctx* c) { return c && c->mesh_set; }

// FP64 FMA throughput: 8 independent chains per thread, 4096 steps each.
__global__ void __launch_bounds__(256) fp64_peak_kernel(double* out, double a, double b) {
  double x[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) x[i] = threadIdx.x * 1e-3 + i;
  for (int s = 0; s < 4096; ++s) {
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = fma(x[i], a, b);
  }
  double r = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) r += x[i];
  if (r == 12345.678) out[0] = r;  // keeps the chains live
}

__device__ __forceinline__ unsigned long long ulp_dist(double a, double b) {
  const long long x = __double_as_longlong(a), y = __double_as_longlong(b);
  return (unsigned long long)(x > y ? x - y : y - x);
}

__global__ void fast_math_check_kernel(const double* __restrict__ x, int n, unsigned long long* ulp) {
  unsigned long long m0 = 0, m1 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = x[i];
    m0 = max(m0, ulp_dist(rcp_nr(v), 1.0 / v));
    m1 = max(m1, ulp_dist(sqrt_nr(v), sqrt(v)));
  }
  atomicMax(&ulp[0], m0);
  atomicMax(&ulp[1], m1);
}

}  // namespace

// =============================================================================
extern "C" {

int wx3d_config_defaults(wx_config* f) {
  if (!f) return WX_ERR_INVALID_ARG;
  std::memset(f, 0, sizeof *f);
  f->neqtot = 5;
  f->solver_type = WX_SOLVER_HLLC;
  f->limiter_type = WX_LIMITER_VANLEER;
  f->eos_type = WX_EOS_ADIABATIC;
  f->cooling_type = WX_COOL_NONE;
  for (int i = 0; i < 6; ++i) f->bc[i] = WX_BC_FREE_FLOW;
  f->nbrootx = f->nbrooty = f->nbrootz = 1;
  f->maxlev = 1;
  f->gamma = 5.0 / 3.0;
  f->cfl = 0.4;
  f->visc_eta = 5.0e-3;
  f->cooling_limit = 0.5;
  f->mu0 = 1.3; f->mui = 0.61; f->ion_thres = 1.0e4;
  f->l_sc = f->d_sc = f->v_sc = 1.0;
  f->xphystot = f->yphystot = f->zphystot = 1.0;
  f->tfin = 1.0e30; f->dtout = 1.0e30;
  f->refine_thres = 0.3; f->coarse_thres = 0.03;
  return WX_OK;
}

const char* wx3d_error_string(int32_t code) {
  switch (code) {
    case WX_OK: return "ok";
    case WX_ERR_ALREADY_MAX_LEV: return "block already at the finest level";
    case WX_ERR_INSUFICIENT_NBMAXPROC: return "not enough block slots";
    case WX_ERR_REGISTER_FATHER: return "no free slot for a coarsened father block";
    case WX_ERR_TOO_MANY_LEVS: return "too many refinement levels";
    case WX_ERR_COOLING_LOAD_COEFS: return "bad cooling table";
    case WX_ERR_OUTPUT_FILE_OPEN: return "could not write an output file";
    case WX_ERR_WARM_FILE_OPEN: return "could not read a warm-start file";
    case WX_ERR_WARM_READ_BLOCKS: return "warm-start block file is short or malformed";
    case WX_ERR_DIVISION_BY_ZERO: return "zero density";
    case WX_ERR_NOT_ENOUGH_PASSIVES: return "not enough passive scalars";
    case WX_ERR_NAN_IN_FLUXES: return "NaN in fluxes";
    case WX_ERR_CUDA: return "CUDA error";
    case WX_ERR_TIMEOUT: return "device wait timed out";
    case WX_ERR_NAN: return "non-finite state";
    case WX_ERR_INVALID_ARG: return "invalid argument";
    case WX_ERR_UNSUPPORTED: return "unsupported configuration";
    case WX_ERR_NO_DEVICE: return "no CUDA device";
    case WX_ERR_MESH: return "invalid mesh";
    default: return "generic error";
  }
}

int wx3d_last_error(wx_ctx* c, char* buf, int32_t len) {
  if (!c || !buf || len <= 0) return WX_ERR_INVALID_ARG;
  std::snprintf(buf, (size_t)len, "%s", c->err.c_str());
  return WX_OK;
}

int wx3d_init(const wx_config* cfg, int32_t max_blocks, wx_ctx** out) {
  if (!cfg || !out || max_blocks <= 0) return WX_ERR_INVALID_ARG;
  *out = nullptr;
  std::string why;
  int rc = validate(*cfg, why);
  if (rc) { std::fprintf(stderr, "wx3d_init: %s\n", why.c_str()); return rc; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return WX_ERR_NO_DEVICE;
  wx_ctx* c = new wx_ctx();
  c->cfg = *cfg;
  c->neq = cfg->neqtot;
  c->max_blocks = max_blocks;
  if (!select_kern(*cfg, c->k)) { delete c; std::fprintf(stderr, "wx3d_init: solver/equation set not supported\n"); return WX_ERR_UNSUPPORTED; }
  fill_phys(c);
  c->tree.init(*cfg);
  cudaGetDevice(&c->dev);
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev);
  auto cleanup = [&](int code) { wx3d_finalize(c); return code; };
  if ((rc = set_stage_attrs(c))) return cleanup(rc);
  const size_t n = (size_t)max_blocks * c->neq * BCELLS;
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) return cleanup(WX_ERR_CUDA);
  c->stream = c->own;
  if (cudaMalloc(&c->dU, n * 8) || cudaMalloc(&c->dUP, n * 8) || cudaMalloc(&c->dW, n * 8)) return cleanup(WX_ERR_CUDA);
  c->slot_cap = max_blocks;
  cudaMemset(c->dU, 0, n * 8);
  cudaMemset(c->dUP, 0, n * 8);
  cudaMemset(c->dW, 0, n * 8);
  if (cudaMalloc(&c->dBlocks, sizeof(DevBlock) * max_blocks) || cudaMalloc(&c->dWork, 4 * (size_t)max_blocks) ||
      cudaMalloc(&c->dFlags, 4 * (size_t)max_blocks) || cudaMalloc(&c->dCtl, sizeof(DevCtl)) ||
      cudaMallocHost(&c->hCtl, sizeof(DevCtl)))
    return cleanup(WX_ERR_CUDA);
  std::memset(c->hCtl, 0, sizeof(DevCtl));
  c->hCtl->nextout = 1;
  {
    const double big = 1.0e30;
    std::memcpy(&c->hCtl->dtmin_bits, &big, 8);
  }
  if (cudaMemcpy(c->dCtl, c->hCtl, sizeof(DevCtl), cudaMemcpyHostToDevice)) return cleanup(WX_ERR_CUDA);
  c->local.assign(max_blocks, -1);
  if (cudaMallocHost(&c->hblocks, sizeof(DevBlock) * (size_t)max_blocks) ||
      cudaMallocHost(&c->hblocks_next, sizeof(DevBlock) * (size_t)max_blocks))
    return cleanup(WX_ERR_CUDA);
  std::memset(c->hblocks, 0, sizeof(DevBlock) * (size_t)max_blocks);
  *out = c;
  return WX_OK;
}

int wx3d_finalize(wx_ctx* c) {
  if (!c) return WX_ERR_INVALID_ARG;
  if (c->stream) cudaStreamSynchronize(c->stream);
  invalidate_graph(c);
  cudaFree(c->dU); cudaFree(c->dUP); cudaFree(c->dW); cudaFree(c->dPrim); cudaFree(c->dStage);
  cudaFree(c->dBlocks); cudaFree(c->dWork); cudaFree(c->dFlags); cudaFree(c->dCtl); cudaFree(c->dCool);
  cudaFree(c->dTrust);
  cudaFree(c->dWind);
  cudaFree(c->dBlocksWind); cudaFree(c->dWindPairs); cudaFree(c->dWindWork);
  cudaFree(c->dOps);
  cudaFree(c->dItems);
  cudaFree(c->dG);
  cudaFree(c->dBlocksNext);
  cudaFree(c->dHash);
  cudaFree(c->dLbBuf);
  cudaFree(c->dMeshErr);
  if (c->hCtl) cudaFreeHost(c->hCtl);
  if (c->hblocks) cudaFreeHost(c->hblocks);
  if (c->hblocks_next) cudaFreeHost(c->hblocks_next);
  for (int i = 0; i < 64; ++i)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return WX_OK;
}

int wx3d_set_stream(wx_ctx* c, void* s) {
  if (!c) return WX_ERR_INVALID_ARG;
  cudaStreamSynchronize(c->stream);
  c->stream = s ? (cudaStream_t)s : c->own;
  invalidate_graph(c);
  return WX_OK;
}

// Neighbour table from the localBlocks registry (amr.f90:539-631 neighbors,
// :831 siblingCoords, :916 father, :882 children).
int wx3d_set_mesh(wx_ctx* c, int32_t nslots, const int32_t* lb) { return wx3d_set_mesh_halo(c, nslots, lb, 0, nullptr); }

// As wx3d_set_mesh, with nhalo slots holding copies of blocks another
// process owns: they are read as neighbours but never updated, and their
// own faces may lead out of the local block set.
// Builds the neighbour table of a mesh into hblocks_next and its work list,
// refusing what the tree queries cannot resolve and wind spheres on a
// coarse/fine face; the context's mesh and state are left as they are.
static int build_mesh(wx_ctx* c, int32_t nslots, const int32_t* lb, int32_t nhalo, const int32_t* halo,
                      std::vector<int32_t>& work) {
  if (!c || !lb || nslots < 0 || nhalo < 0 || (nhalo > 0 && !halo)) return WX_ERR_INVALID_ARG;
  std::vector<char> is_halo(c->max_blocks, 0);
  for (int h = 0; h < nhalo; ++h) {
    if (halo[h] < 0 || halo[h] >= nslots || lb[halo[h]] == -1) return fail(c, WX_ERR_INVALID_ARG, "halo slot %d is not an occupied slot", halo[h]);
    is_halo[halo[h]] = 1;
  }
  if (nhalo > 0 && !c->hwind.empty()) return fail(c, WX_ERR_UNSUPPORTED, "wind sources in a partitioned run");
  if (nslots > c->max_blocks) return fail(c, WX_ERR_INSUFICIENT_NBMAXPROC, "%d slots > max_blocks %d", nslots, c->max_blocks);
  const Tree& T = c->tree;
  SlotMap slot((size_t)nslots);
  for (int s = 0; s < nslots; ++s) {
    if (lb[s] == -1) continue;
    if (T.level(lb[s]) < 1) return fail(c, WX_ERR_MESH, "slot %d: bID %d outside the tree", s, lb[s]);
    if (!slot.insert(lb[s], s)) return fail(c, WX_ERR_MESH, "bID %d registered twice", lb[s]);
  }
  // the table entry of every slot, independent per slot (over the host
  // cores); a face without a valid neighbour is reported as 1 + 2*face +
  // (0: no active neighbour at the finest level, 1: not one level apart)
  DevBlock* hb = c->hblocks_next;
  for (int s = nslots; s < c->max_blocks; ++s) hb[s] = DevBlock{};
  std::vector<int> face_err(nslots, 0);
  auto entry = [&](int s) -> int {
    DevBlock b{};
    const long long id = lb[s];
    if (id == -1) { hb[s] = b; return 0; }
    const int l = T.level(id);
    int x[3];
    T.coords(id, l, x);
    b.level = l;
    b.bID = (int32_t)id;
    for (int d = 0; d < 3; ++d) {
      b.bc[d] = x[d] + 1;
      b.sib[d] = l > 1 ? (x[d] & 1) : -1;
    }
    const double s2 = std::ldexp(1.0, l - 1);
    b.dx = c->cfg.xphystot / ((double)(NC * c->cfg.nbrootx) * s2) / c->cfg.l_sc;
    b.dy = c->cfg.yphystot / ((double)(NC * c->cfg.nbrooty) * s2) / c->cfg.l_sc;
    b.dz = c->cfg.zphystot / ((double)(NC * c->cfg.nbrootz) * s2) / c->cfg.l_sc;
    for (int f = 0; f < 6; ++f) {
      const int ax = f / 2, side = f & 1;
      for (int q = 0; q < 4; ++q) b.fnb[f][q] = -1;
      int y[3] = {x[0], x[1], x[2]};
      y[ax] += side ? 1 : -1;
      if (y[ax] < 0 || y[ax] >= T.nb[l][ax]) {
        b.ftype[f] = WX_NEIGH_BOUNDARY;
        b.fnb[f][0] = c->cfg.bc[f];
        continue;
      }
      const long long nID = T.id(l, y);
      const int sn = slot.find(nID);
      if (sn >= 0) { b.ftype[f] = WX_NEIGH_SAME; b.fnb[f][0] = sn; continue; }
      if (l > 1) {
        int z[3] = {y[0] / 2, y[1] / 2, y[2] / 2};
        const int sf = slot.find(T.id(l - 1, z));
        if (sf >= 0) { b.ftype[f] = WX_NEIGH_COARSER; b.fnb[f][0] = sf; continue; }
      }
      // finer: the four children of nID adjacent to this face, transverse
      // axes in x<y<z order (amr.f90:590-628)
      if (l >= T.maxlev) {
        if (is_halo[s]) { b.ftype[f] = 0; continue; }   // outside the local set
        return 1 + 2 * f;
      }
      const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
      b.ftype[f] = WX_NEIGH_FINER;
      for (int q = 0; q < 4; ++q) {
        int ch[3];
        ch[ax] = 2 * y[ax] + (side ? 0 : 1);
        ch[t1] = 2 * y[t1] + (q & 1);
        ch[t2] = 2 * y[t2] + (q >> 1);
        const int sc = slot.find(T.id(l + 1, ch));
        if (sc < 0) {
          if (is_halo[s]) { b.ftype[f] = 0; break; }
          return 2 + 2 * f;
        }
        b.fnb[f][q] = sc;
      }
    }
    hb[s] = b;
    return 0;
  };
#pragma omp parallel for schedule(dynamic, 512) if (nslots > 4096)
  for (int s = 0; s < nslots; ++s) face_err[s] = entry(s);
  work.clear();
  work.reserve(nslots);
  for (int s = 0; s < nslots; ++s) {
    if (face_err[s]) {
      const int f = (face_err[s] - 1) / 2;
      if ((face_err[s] - 1) % 2 == 0) return fail(c, WX_ERR_MESH, "bID %d face %d: no active neighbour", lb[s], f + 1);
      return fail(c, WX_ERR_MESH, "bID %d face %d: neighbour region is neither same, coarser nor finer by one", lb[s], f + 1);
    }
    if (lb[s] != -1 && !is_halo[s]) work.push_back(s);
  }
  int bad = -1;
  if (!flag_wind_blocks(c, hb, c->max_blocks, &bad))
    return fail(c, WX_ERR_UNSUPPORTED, "slot %d: a wind sphere reaches the ghost layer of a coarse/fine face or of the domain "
                "boundary; refine the zone around the source (refineZone) further", bad);
  return WX_OK;
}

// ---------------------------------------------------------------------------
// The same neighbour table built on the device, for meshes without halo slots
// or wind sources (the host build above stays for those): a bID -> slot hash
// table filled by one thread per slot, then one thread per slot resolving its
// six faces with the tree queries of amr.f90:439-1098, into dBlocksNext.  The
// errors the host build reports are recorded as the smallest failing slot.

__device__ __forceinline__ unsigned bid_hash(int id, unsigned mask) { return ((unsigned)id * 2654435761u) & mask; }

__device__ __forceinline__ int hash_find(const int2* __restrict__ h, unsigned mask, long long id) {
  if (id < 1 || id > 0x7fffffffLL) return -1;
  unsigned k = bid_hash((int)id, mask);
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const int2 e = h[k];
    if (e.x == (int)id) return e.y;
    if (e.x == -1) return -1;
    k = (k + 1) & mask;
  }
  return -1;
}

// err[0]: first slot whose bID lies outside the tree; err[1]: a slot whose
// bID another slot holds too
__global__ void mesh_insert_kernel(const int32_t* __restrict__ lb, int n, Tree T, int2* h, unsigned mask, int* err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int id = lb[s];
  if (id == -1) return;
  if (T.level(id) < 1) { atomicMin(&err[0], s); return; }
  unsigned k = bid_hash(id, mask);
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const int prev = atomicCAS(&h[k].x, -1, id);
    if (prev == -1) { h[k].y = s; return; }
    if (prev == id) { atomicMin(&err[1], s); return; }
    k = (k + 1) & mask;
  }
  atomicMin(&err[1], s);
}

struct MeshGeom {
  double xphystot, yphystot, zphystot, l_sc;
  int nbroot[3];
  int bc[6];
};

// err[2]: first slot with a face the tree queries cannot resolve; its code
// (1 + 2 face: no active neighbour at the finest level, 2 + 2 face: not one
// level apart) in code[slot]
__global__ void mesh_table_kernel(const int32_t* __restrict__ lb, int n, int max_blocks, Tree T, MeshGeom G,
                                  const int2* __restrict__ h, unsigned mask, DevBlock* out, int* err, int* code) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= max_blocks) return;
  DevBlock b{};
  const long long id = s < n ? lb[s] : -1;
  const int l = id == -1 ? -1 : T.level(id);
  if (l < 1) { out[s] = b; return; }   // empty slot, or outside the tree (reported by the insertion)
  int x[3];
  T.coords(id, l, x);
  b.level = l;
  b.bID = (int32_t)id;
  for (int d = 0; d < 3; ++d) {
    b.bc[d] = x[d] + 1;
    b.sib[d] = l > 1 ? (x[d] & 1) : -1;
  }
  const double s2 = ldexp(1.0, l - 1);
  b.dx = G.xphystot / ((double)(NC * G.nbroot[0]) * s2) / G.l_sc;
  b.dy = G.yphystot / ((double)(NC * G.nbroot[1]) * s2) / G.l_sc;
  b.dz = G.zphystot / ((double)(NC * G.nbroot[2]) * s2) / G.l_sc;
  int bad = 0;
  for (int f = 0; f < 6 && !bad; ++f) {
    const int ax = f / 2, side = f & 1;
    for (int q = 0; q < 4; ++q) b.fnb[f][q] = -1;
    int y[3] = {x[0], x[1], x[2]};
    y[ax] += side ? 1 : -1;
    if (y[ax] < 0 || y[ax] >= T.nb[l][ax]) {
      b.ftype[f] = WX_NEIGH_BOUNDARY;
      b.fnb[f][0] = G.bc[f];
      continue;
    }
    const int sn = hash_find(h, mask, T.id(l, y));
    if (sn >= 0) { b.ftype[f] = WX_NEIGH_SAME; b.fnb[f][0] = sn; continue; }
    if (l > 1) {
      const int z[3] = {y[0] / 2, y[1] / 2, y[2] / 2};
      const int sf = hash_find(h, mask, T.id(l - 1, z));
      if (sf >= 0) { b.ftype[f] = WX_NEIGH_COARSER; b.fnb[f][0] = sf; continue; }
    }
    if (l >= T.maxlev) { bad = 1 + 2 * f; break; }
    const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
    b.ftype[f] = WX_NEIGH_FINER;
    for (int q = 0; q < 4; ++q) {
      int ch[3];
      ch[ax] = 2 * y[ax] + (side ? 0 : 1);
      ch[t1] = 2 * y[t1] + (q & 1);
      ch[t2] = 2 * y[t2] + (q >> 1);
      const int sc = hash_find(h, mask, T.id(l + 1, ch));
      if (sc < 0) { bad = 2 + 2 * f; break; }
      b.fnb[f][q] = sc;
    }
  }
  if (bad) {
    code[s] = bad;
    atomicMin(&err[2], s);
    out[s] = DevBlock{};
    return;
  }
  out[s] = b;
}

// build_mesh on the device (no halo slots, no wind sources); on success the
// new table is in dBlocksNext and next_on_device is set.
static int build_mesh_gpu(wx_ctx* c, int32_t nslots, const int32_t* lb, std::vector<int32_t>& work) {
  if (!c || !lb || nslots < 0) return WX_ERR_INVALID_ARG;
  if (nslots > c->max_blocks) return fail(c, WX_ERR_INSUFICIENT_NBMAXPROC, "%d slots > max_blocks %d", nslots, c->max_blocks);
  if (!c->dBlocksNext) {
    unsigned hs = 16;
    while (hs < 2u * (unsigned)c->max_blocks) hs <<= 1;
    c->hash_size = hs;
    if (cudaMalloc(&c->dBlocksNext, sizeof(DevBlock) * (size_t)c->max_blocks) != cudaSuccess ||
        cudaMalloc(&c->dHash, sizeof(int2) * (size_t)hs) != cudaSuccess ||
        cudaMalloc(&c->dLbBuf, 4 * (size_t)c->max_blocks) != cudaSuccess ||
        cudaMalloc(&c->dMeshErr, 4 * (3 + (size_t)c->max_blocks)) != cudaSuccess)
      return fail(c, WX_ERR_CUDA, "device neighbour-table buffers");
  }
  work.clear();
  work.reserve(nslots);
  for (int s = 0; s < nslots; ++s)
    if (lb[s] != -1) work.push_back(s);
  const int big = 0x7fffffff;
  const int init[3] = {big, big, big};
  if (nslots > 0) WX_CUDA(cudaMemcpyAsync(c->dLbBuf, lb, 4 * (size_t)nslots, cudaMemcpyHostToDevice, c->stream));
  WX_CUDA(cudaMemcpyAsync(c->dMeshErr, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  WX_CUDA(cudaMemsetAsync(c->dHash, 0xff, sizeof(int2) * (size_t)c->hash_size, c->stream));
  const unsigned mask = c->hash_size - 1;
  if (nslots > 0) {
    mesh_insert_kernel<<<(nslots + 255) / 256, 256, 0, c->stream>>>(c->dLbBuf, nslots, c->tree, c->dHash, mask, c->dMeshErr);
    WX_LAUNCHED();
  }
  MeshGeom G;
  G.xphystot = c->cfg.xphystot; G.yphystot = c->cfg.yphystot; G.zphystot = c->cfg.zphystot; G.l_sc = c->cfg.l_sc;
  G.nbroot[0] = c->cfg.nbrootx; G.nbroot[1] = c->cfg.nbrooty; G.nbroot[2] = c->cfg.nbrootz;
  for (int f = 0; f < 6; ++f) G.bc[f] = c->cfg.bc[f];
  mesh_table_kernel<<<(c->max_blocks + 255) / 256, 256, 0, c->stream>>>(c->dLbBuf, nslots, c->max_blocks, c->tree, G,
                                                                        c->dHash, mask, c->dBlocksNext, c->dMeshErr,
                                                                        c->dMeshErr + 3);
  WX_LAUNCHED();
  int herr[3];
  WX_CUDA(cudaMemcpyAsync(herr, c->dMeshErr, sizeof(herr), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  if (herr[0] != big || herr[1] != big) {
    if (herr[0] < herr[1]) return fail(c, WX_ERR_MESH, "slot %d: bID %d outside the tree", herr[0], lb[herr[0]]);
    return fail(c, WX_ERR_MESH, "bID %d registered twice", lb[herr[1]]);
  }
  if (herr[2] != big) {
    int code = 0;
    WX_CUDA(cudaMemcpy(&code, c->dMeshErr + 3 + herr[2], 4, cudaMemcpyDeviceToHost));
    const int f = (code - 1) / 2;
    if ((code - 1) % 2 == 0) return fail(c, WX_ERR_MESH, "bID %d face %d: no active neighbour", lb[herr[2]], f + 1);
    return fail(c, WX_ERR_MESH, "bID %d face %d: neighbour region is neither same, coarser nor finer by one", lb[herr[2]], f + 1);
  }
  c->next_on_device = true;
  return WX_OK;
}

// The host copy of the table, for the host readers (neighbour queries, the
// wind-sphere flags), after a build on the device.
static int sync_host_table(wx_ctx* c) {
  if (!c->host_table_stale) return WX_OK;
  WX_CUDA(cudaMemcpyAsync(c->hblocks, c->dBlocks, sizeof(DevBlock) * (size_t)c->max_blocks, cudaMemcpyDeviceToHost,
                          c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  c->host_table_stale = false;
  return WX_OK;
}

// Wind runs: lists the occupied blocks a sphere reaches, gives each an
// extra slot past max_blocks in dU and dW (growing both when needed), and
// builds dBlocksWind, the neighbour table whose same-level, coarser and
// finer entries point at the extra slot of a reached block.  Domain-boundary
// ghosts keep mirroring the block's own cells before the wind, as the
// reference's fill does before userBoundary (spheres that reach those
// ghosts are refused by flag_wind_blocks).
static int prepare_wind_redirect(wx_ctx* c) {
  c->wind_ready = false;
  c->nwslot = 0;
  if (c->hwind.empty() || !c->mesh_set) return WX_OK;
  int rc = sync_host_table(c);
  if (rc) return rc;
  const DevBlock* hb = c->hblocks;
  std::vector<int32_t> reached;
  for (int s : c->work)
    if (hb[s].wind) reached.push_back(s);
  const int nr = (int)reached.size();
  const int mb = c->max_blocks;
  if (mb + nr > c->slot_cap) {
    const int cap = mb + std::max(nr, 64);
    const size_t per = (size_t)c->neq * BCELLS * 8;
    double *u = nullptr, *w = nullptr;
    WX_CUDA(cudaStreamSynchronize(c->stream));
    if (cudaMalloc(&u, per * cap) != cudaSuccess || cudaMalloc(&w, per * cap) != cudaSuccess) {
      cudaFree(u);
      return fail(c, WX_ERR_CUDA, "wind: no device memory for %d extra slots", cap - mb);
    }
    WX_CUDA(cudaMemcpy(u, c->dU, per * mb, cudaMemcpyDeviceToDevice));
    WX_CUDA(cudaMemset(w, 0, per * cap));
    cudaFree(c->dU);
    cudaFree(c->dW);
    c->dU = u;
    c->dW = w;
    c->slot_cap = cap;
    c->prestep = false;
    c->g_valid = false;
    invalidate_graph(c);
  }
  if (nr > c->wind_cap) {
    const int cap = std::max(nr, 64);
    cudaFree(c->dBlocksWind);
    cudaFree(c->dWindPairs);
    cudaFree(c->dWindWork);
    c->dBlocksWind = nullptr;
    c->dWindPairs = nullptr;
    c->dWindWork = nullptr;
    c->wind_cap = 0;
    if (cudaMalloc(&c->dBlocksWind, sizeof(DevBlock) * (size_t)(mb + cap)) != cudaSuccess ||
        cudaMalloc(&c->dWindPairs, sizeof(int2) * (size_t)cap) != cudaSuccess ||
        cudaMalloc(&c->dWindWork, sizeof(int32_t) * (size_t)cap) != cudaSuccess)
      return fail(c, WX_ERR_CUDA, "wind: no device memory for the redirected table");
    c->wind_cap = cap;
  }
  std::vector<int32_t> extra(mb, -1);
  std::vector<int2> pairs(nr);
  std::vector<int32_t> ework(nr);
  for (int r = 0; r < nr; ++r) {
    extra[reached[r]] = mb + r;
    pairs[r] = make_int2(reached[r], mb + r);
    ework[r] = mb + r;
  }
  std::vector<DevBlock> tab(hb, hb + mb);
  tab.resize((size_t)mb + nr);
  for (int s = 0; s < mb; ++s) {
    DevBlock& b = tab[s];
    if (b.level < 1) continue;
    for (int f = 0; f < 6; ++f) {
      const int t = b.ftype[f];
      const int nq = t == WX_NEIGH_FINER ? 4 : ((t == WX_NEIGH_SAME || t == WX_NEIGH_COARSER) ? 1 : 0);
      for (int q = 0; q < nq; ++q) {
        const int nbs = b.fnb[f][q];
        if (nbs >= 0 && nbs < mb && extra[nbs] >= 0) b.fnb[f][q] = extra[nbs];
      }
    }
  }
  for (int r = 0; r < nr; ++r) tab[(size_t)mb + r] = hb[reached[r]];
  WX_CUDA(cudaMemcpy(c->dBlocksWind, tab.data(), sizeof(DevBlock) * tab.size(), cudaMemcpyHostToDevice));
  if (nr > 0) {
    WX_CUDA(cudaMemcpy(c->dWindPairs, pairs.data(), sizeof(int2) * nr, cudaMemcpyHostToDevice));
    WX_CUDA(cudaMemcpy(c->dWindWork, ework.data(), sizeof(int32_t) * nr, cudaMemcpyHostToDevice));
  }
  c->nwslot = nr;
  c->wind_ready = true;
  invalidate_graph(c);
  return WX_OK;
}

// Makes the mesh that build_mesh left in hblocks_next the context's.
static int commit_mesh(wx_ctx* c, int32_t nslots, const int32_t* lb, int32_t nhalo, std::vector<int32_t>& work) {
  c->local.assign(c->max_blocks, -1);
  std::copy(lb, lb + nslots, c->local.begin());
  c->nhalo = nhalo;
  c->work = std::move(work);
  c->nwork = (int)c->work.size();
  c->mesh_set = true;
  if (c->next_on_device) {
    std::swap(c->dBlocks, c->dBlocksNext);
    c->next_on_device = false;
    c->host_table_stale = true;
  } else {
    std::swap(c->hblocks, c->hblocks_next);
    WX_CUDA(cudaMemcpyAsync(c->dBlocks, c->hblocks, sizeof(DevBlock) * c->max_blocks, cudaMemcpyHostToDevice, c->stream));
    c->host_table_stale = false;
  }
  if (!c->work.empty())
    WX_CUDA(cudaMemcpyAsync(c->dWork, c->work.data(), 4 * c->work.size(), cudaMemcpyHostToDevice, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  // small meshes split every block into z-slabs so all SMs get work
  c->zsplit = 1;
  while (c->zsplit < 8 && c->nwork * c->zsplit < 2 * c->nsm) c->zsplit *= 2;
  c->dt_valid = false;
  c->prestep = false;
  c->g_valid = false;
  invalidate_graph(c);
  return prepare_wind_redirect(c);
}

// The device build serves meshes without halo slots or wind sources.
static int build_any(wx_ctx* c, int32_t nslots, const int32_t* lb, int32_t nhalo, const int32_t* halo,
                     std::vector<int32_t>& work) {
  if (c && nhalo == 0 && c->hwind.empty()) return build_mesh_gpu(c, nslots, lb, work);
  if (c) c->next_on_device = false;
  return build_mesh(c, nslots, lb, nhalo, halo, work);
}

int wx3d_set_mesh_halo(wx_ctx* c, int32_t nslots, const int32_t* lb, int32_t nhalo, const int32_t* halo) {
  std::vector<int32_t> work;
  const int rc = build_any(c, nslots, lb, nhalo, halo, work);
  return rc ? rc : commit_mesh(c, nslots, lb, nhalo, work);
}

int wx3d_set_zsplit(wx_ctx* c, int32_t zsplit) {
  if (!c || (zsplit != 1 && zsplit != 2 && zsplit != 4 && zsplit != 8)) return WX_ERR_INVALID_ARG;
  c->zsplit = zsplit;
  invalidate_graph(c);
  return WX_OK;
}

// Measured choice of the z-slab split: times the predictor and corrector
// stages (which write only the UP and W scratch arrays, so U and the
// simulation state are untouched) for every split and keeps the fastest.
// userBoundary hook of the wind problems (imposeSphericalWind,
// winds.f90:123-240): nwind sources in physical (cgs) units; 0 removes them.
int wx3d_set_winds(wx_ctx* c, int32_t nwind, const wx_wind* winds) {
  if (!c || nwind < 0 || (nwind > 0 && !winds)) return WX_ERR_INVALID_ARG;
  if (nwind > 0 && (c->cfg.solver_type == WX_SOLVER_LAX || c->cfg.solver_type == WX_SOLVER_HLL1))
    return fail(c, WX_ERR_UNSUPPORTED, "wind sources with a single-stage solver");
  if (nwind > 0 && c->cfg.npassive > 1)
    return fail(c, WX_ERR_UNSUPPORTED, "wind sources with more than one passive scalar (the reference leaves them undefined)");
  std::vector<double> h((size_t)nwind * 12);
  for (int w = 0; w < nwind; ++w) {
    const wx_wind& s = winds[w];
    const double v[12] = {s.xc, s.yc, s.zc, s.vx, s.vy, s.vz, s.radius, s.mdot, s.vinf, s.temp, s.mu, s.y0};
    if (!(s.radius > 0.0) || !(s.vinf > 0.0) || !(s.mdot > 0.0) || !(s.mu > 0.0))
      return fail(c, WX_ERR_INVALID_ARG, "wind %d: radius, vinf, mdot and mu must be positive", w);
    std::copy(v, v + 12, h.begin() + 12 * w);
  }
  const int rs = sync_host_table(c);
  if (rs) return rs;
  std::vector<double> prev = c->hwind;
  c->hwind = h;
  int bad = -1;
  DevBlock* hb = c->hblocks_next;
  std::memcpy(hb, c->hblocks, sizeof(DevBlock) * (size_t)c->max_blocks);
  if (!flag_wind_blocks(c, hb, c->max_blocks, &bad)) {
    c->hwind = prev;
    return fail(c, WX_ERR_UNSUPPORTED, "slot %d: a wind sphere reaches the ghost layer of a coarse/fine face or of the domain "
                "boundary; refine the zone around the source (refineZone) further", bad);
  }
  WX_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(c->dWind);
  c->dWind = nullptr;
  if (nwind > 0) {
    WX_CUDA(cudaMalloc(&c->dWind, sizeof(double) * h.size()));
    WX_CUDA(cudaMemcpy(c->dWind, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
  }
  std::swap(c->hblocks, c->hblocks_next);
  fill_phys(c);
  WX_CUDA(cudaMemcpyAsync(c->dBlocks, c->hblocks, sizeof(DevBlock) * c->max_blocks, cudaMemcpyHostToDevice,
                          c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  invalidate_graph(c);
  return prepare_wind_redirect(c);
}

int wx3d_step_part(wx_ctx* c, int32_t part) {
  if (!ready(c) || part < 0 || part > 3) return WX_ERR_INVALID_ARG;
  if (!c->hwind.empty()) return fail(c, WX_ERR_UNSUPPORTED, "the step in parts does not run wind sources");
  int rc;
  c->nev = 0;
  switch (part) {
    case 0:
      if (!c->dt_valid) {
        if ((rc = launch_dt(c, c->dU))) return rc;
        c->dt_valid = true;
      }
      step_begin_kernel<<<1, 1, 0, c->stream>>>(c->dCtl, c->ph.cfl, c->cfg.cooling_type != WX_COOL_NONE, c->ph.dtout,
                                                c->ph.t_sc, 1);
      WX_LAUNCHED();
      return WX_OK;
    case 1: return solver_first(c);
    case 2: return solver_second(c, true);
    default:
      if (sources_on(c)) {
        int mode = 8;
        if (c->cfg.eos_type == WX_EOS_H_RATE) mode |= 1;
        if (c->cfg.cooling_type != WX_COOL_NONE) mode |= 2;
        if ((rc = enqueue_sources(c, mode))) return rc;
      }
      return sync_check(c);
  }
}

int wx3d_get_dtmin(wx_ctx* c, double* v) {
  if (!ready(c) || !v) return WX_ERR_INVALID_ARG;
  int rc;
  if (!c->dt_valid) {
    if ((rc = launch_dt(c, c->dU))) return rc;
    c->dt_valid = true;
  }
  WX_CUDA(cudaMemcpyAsync(c->hCtl, c->dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  std::memcpy(v, &c->hCtl->dtmin_bits, 8);
  return WX_OK;
}

int wx3d_set_dtmin(wx_ctx* c, double v) {
  if (!c || !(v > 0.0)) return WX_ERR_INVALID_ARG;
  unsigned long long bits;
  std::memcpy(&bits, &v, 8);   // positive doubles order like their bit patterns
  WX_CUDA(cudaMemcpyAsync(&c->dCtl->dtmin_bits, &bits, 8, cudaMemcpyHostToDevice, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  c->dt_valid = true;
  return WX_OK;
}

static int copy_blocks(wx_ctx* c, int32_t array, int32_t n, const int32_t* slots, double* buf, bool pack) {
  if (!c || n < 0 || (n > 0 && (!slots || !buf)) || (array != 0 && array != 1)) return WX_ERR_INVALID_ARG;
  double* a = array == 0 ? c->dU : c->dUP;
  const size_t per = (size_t)c->neq * BCELLS * 8;
  for (int b = 0; b < n; ++b) {
    if (slots[b] < 0 || slots[b] >= c->max_blocks) return fail(c, WX_ERR_INVALID_ARG, "slot %d out of range", slots[b]);
    double* s = a + (size_t)slots[b] * c->neq * BCELLS;
    double* d = buf + (size_t)b * c->neq * BCELLS;
    WX_CUDA(cudaMemcpyAsync(pack ? d : s, pack ? s : d, per, cudaMemcpyDeviceToDevice, c->stream));
  }
  WX_CUDA(cudaStreamSynchronize(c->stream));
  return WX_OK;
}

int wx3d_pack_blocks(wx_ctx* c, int32_t array, int32_t n, const int32_t* slots, double* d_buf) {
  return copy_blocks(c, array, n, slots, d_buf, true);
}

int wx3d_unpack_blocks(wx_ctx* c, int32_t array, int32_t n, const int32_t* slots, const double* d_buf) {
  return copy_blocks(c, array, n, slots, const_cast<double*>(d_buf), false);
}

static int copy_faces(wx_ctx* c, int32_t array, int32_t n, const int32_t* slots, const int32_t* faces, double* buf,
                      bool pack) {
  if (!c || n < 0 || (n > 0 && (!slots || !faces || !buf)) || (array != 0 && array != 1)) return WX_ERR_INVALID_ARG;
  if (n == 0) return WX_OK;
  if (n > 6 * c->max_blocks) return fail(c, WX_ERR_INVALID_ARG, "%d face slabs > 6 x max_blocks", n);
  std::vector<int32_t> items(2 * (size_t)n);
  for (int b = 0; b < n; ++b) {
    if (slots[b] < 0 || slots[b] >= c->max_blocks) return fail(c, WX_ERR_INVALID_ARG, "slot %d out of range", slots[b]);
    if (faces[b] < 0 || faces[b] > 5) return fail(c, WX_ERR_INVALID_ARG, "face %d out of 0..5", faces[b]);
    items[2 * b] = slots[b];
    items[2 * b + 1] = faces[b];
  }
  if (!c->dItems) WX_CUDA(cudaMalloc(&c->dItems, sizeof(int32_t) * 12 * (size_t)c->max_blocks));
  WX_CUDA(cudaMemcpyAsync(c->dItems, items.data(), 4 * items.size(), cudaMemcpyHostToDevice, c->stream));
  double* a = array == 0 ? c->dU : c->dUP;
  for (int o = 0; o < n; o += 60000) {
    const int m = std::min(60000, n - o);
    face_slab_kernel<<<dim3(4, m), 256, 0, c->stream>>>(a, c->dItems + 2 * o, c->neq,
                                                        buf + (size_t)o * c->neq * FACE_LAYERS * NC * NC, pack ? 1 : 0);
    WX_LAUNCHED();
  }
  WX_CUDA(cudaStreamSynchronize(c->stream));
  return WX_OK;
}

int wx3d_pack_faces(wx_ctx* c, int32_t array, int32_t n, const int32_t* slots, const int32_t* faces, double* d_buf) {
  return copy_faces(c, array, n, slots, faces, d_buf, true);
}

int wx3d_unpack_faces(wx_ctx* c, int32_t array, int32_t n, const int32_t* slots, const int32_t* faces,
                      const double* d_buf) {
  return copy_faces(c, array, n, slots, faces, const_cast<double*>(d_buf), false);
}

int wx3d_set_fusion(wx_ctx* c, int32_t on) {
  if (!c) return WX_ERR_INVALID_ARG;
  c->fuse = on != 0;
  invalidate_graph(c);
  return WX_OK;
}

int wx3d_autotune(wx_ctx* c, int32_t reps, double* ms5, int32_t* best) {
  if (!ready(c) || c->nwork == 0 || reps <= 0) return WX_ERR_INVALID_ARG;
  if (c->cfg.solver_type == WX_SOLVER_LAX) {
    if (best) { best[0] = 1; best[1] = 0; }
    return WX_OK;
  }
  int rc;
  if (!c->dt_valid) {
    if ((rc = launch_dt(c, c->dU))) return rc;
    c->dt_valid = true;
  }
  // The timed passes fold their CFL minima and status counts into the
  // control block; it is saved here and put back after them, so that the
  // next step takes the time step of U, as the reference does.
  DevCtl saved;
  WX_CUDA(cudaMemcpyAsync(c->hCtl, c->dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  saved = *c->hCtl;
  cudaEvent_t e0, e1;
  WX_CUDA(cudaEventCreate(&e0));
  WX_CUDA(cudaEventCreate(&e1));
  const bool timing = c->timing;
  c->timing = false;
  // launch shapes: whole blocks with the fused corrector, whole blocks with
  // a separate viscous kernel, then 2, 4 and 8 slabs per block
  const int splits[5] = {1, 1, 2, 4, 8};
  const bool fused[5] = {true, false, false, false, false};
  double bestms = 1e300;
  int bz = c->zsplit;
  bool bf = c->fuse;
  const bool hll1 = c->cfg.solver_type == WX_SOLVER_HLL1;
  for (int s = 0; s < 5; ++s) {
    c->zsplit = splits[s];
    c->fuse = fused[s];
    // one untimed pass, then reps timed passes of both stages and the
    // viscous step
    for (int r = 0; r <= reps; ++r) {
      if (r == 1) cudaEventRecord(e0, c->stream);
      if ((rc = launch_stage(c, 1, c->dU, c->dU, hll1 ? c->dW : c->dUP, hll1 ? 1.0 : 0.5))) break;
      if (!hll1 && (rc = launch_stage(c, 2, c->dUP, c->dU, c->dW, 1.0, fuse_visc(c)))) break;
      if (!fuse_visc(c) && (rc = launch_visc(c, hll1 ? 1 : 0))) break;
    }
    if (rc) break;
    cudaEventRecord(e1, c->stream);
    WX_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    WX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double per = ms / reps;
    if (ms5) ms5[s] = per;
    if (per < bestms) { bestms = per; bz = splits[s]; bf = fused[s]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->timing = timing;
  c->zsplit = bz;
  c->fuse = bf;
  if (rc) return rc;
  *c->hCtl = saved;
  WX_CUDA(cudaMemcpyAsync(c->dCtl, c->hCtl, sizeof(DevCtl), cudaMemcpyHostToDevice, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  if (best) { best[0] = bz; best[1] = bf ? 1 : 0; }
  invalidate_graph(c);
  return WX_OK;
}

int wx3d_get_neighbours(wx_ctx* c, int32_t nslots, int32_t* ft, int32_t* fs) {
  if (!c || !ft || !fs || nslots > c->max_blocks) return WX_ERR_INVALID_ARG;
  const int rc = sync_host_table(c);
  if (rc) return rc;
  for (int s = 0; s < nslots; ++s)
    for (int f = 0; f < 6; ++f) {
      ft[s * 6 + f] = c->hblocks[s].ftype[f];
      for (int q = 0; q < 4; ++q) fs[(s * 6 + f) * 4 + q] = c->hblocks[s].fnb[f][q];
    }
  return WX_OK;
}

int wx3d_upload_blocks(wx_ctx* c, int32_t nslots, const double* u) {
  if (!c || !u || nslots < 0 || nslots > c->max_blocks) return WX_ERR_INVALID_ARG;
  if (nslots > 0)
    WX_CUDA(cudaMemcpyAsync(c->dU, u, (size_t)nslots * c->neq * BCELLS * 8, cudaMemcpyHostToDevice, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  c->dt_valid = false;
  c->prestep = false;
  c->g_valid = false;
  return WX_OK;
}

int wx3d_download_blocks(wx_ctx* c, int32_t nslots, double* u) {
  if (!c || !u || nslots < 0 || nslots > c->max_blocks) return WX_ERR_INVALID_ARG;
  if (nslots > 0)
    WX_CUDA(cudaMemcpyAsync(u, c->dU, (size_t)nslots * c->neq * BCELLS * 8, cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  return WX_OK;
}

static int ensure_stage(wx_ctx* c, size_t bytes) {
  if (c->stage_bytes >= bytes) return WX_OK;
  cudaFree(c->dStage);
  c->dStage = nullptr;
  c->stage_bytes = 0;
  WX_CUDA(cudaMalloc(&c->dStage, bytes));
  c->stage_bytes = bytes;
  return WX_OK;
}

// ---- checkpoints: writeBin / writeState / warmstart --------------------------

// writeBin (output.f90:156-213): stream file of int32 nbLocal, then per
// occupied slot in slot order int32 bID and U(nb,:,1:16,1:16,1:16) (FP64,
// equation index fastest), written from device memory in chunks.
int wx3d_write_bin(wx_ctx* c, const char* path) {
  if (!c || !path) return WX_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(c, WX_ERR_OUTPUT_FILE_OPEN, "could not open %s", path);
  const int32_t nloc = c->nwork;
  int rc = WX_OK;
  const int chunk = 256;
  const size_t per = (size_t)c->neq * BCELLS;
  double* host = nullptr;
  int32_t* dslots = nullptr;
  if (std::fwrite(&nloc, 4, 1, f) != 1) rc = fail(c, WX_ERR_OUTPUT_FILE_OPEN, "write failed: %s", path);
  if (!rc) rc = ensure_stage(c, chunk * per * 8);
  if (!rc && (cudaMallocHost(&host, chunk * per * 8) != cudaSuccess || cudaMalloc(&dslots, 4 * chunk) != cudaSuccess))
    rc = fail(c, WX_ERR_CUDA, "checkpoint buffers");
  for (int b0 = 0; !rc && b0 < nloc; b0 += chunk) {
    const int nb = std::min(chunk, nloc - b0);
    cudaMemcpyAsync(dslots, c->work.data() + b0, 4 * nb, cudaMemcpyHostToDevice, c->stream);
    pack_bin_kernel<<<1184, 256, 0, c->stream>>>(c->dU, dslots, nb, c->neq, c->dStage);
    cudaMemcpyAsync(host, c->dStage, nb * per * 8, cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) { rc = fail(c, WX_ERR_CUDA, "checkpoint copy"); break; }
    for (int b = 0; b < nb; ++b) {
      const int32_t bid = c->local[c->work[b0 + b]];
      if (std::fwrite(&bid, 4, 1, f) != 1 || std::fwrite(host + b * per, 8, per, f) != per) {
        rc = fail(c, WX_ERR_OUTPUT_FILE_OPEN, "write failed: %s", path);
        break;
      }
    }
  }
  if (std::fclose(f) != 0 && !rc) rc = fail(c, WX_ERR_OUTPUT_FILE_OPEN, "close failed: %s", path);
  cudaFreeHost(host);
  cudaFree(dslots);
  return rc;
}

// warmstart's block read (init.f90:589-612): the file's blocks go to slots
// 0..nbLocal-1 in file order (localBlocks(nb) = bID), the neighbour table is
// rebuilt for them, and local_blocks (max_slots entries, -1 beyond nbLocal)
// receives the registry for the host's block tree.
int wx3d_read_bin(wx_ctx* c, const char* path, int32_t max_slots, int32_t* local_blocks, int32_t* nblocks) {
  if (!c || !path || !local_blocks || max_slots <= 0) return WX_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(c, WX_ERR_WARM_FILE_OPEN, "could not open %s", path);
  int32_t nloc = 0;
  if (std::fread(&nloc, 4, 1, f) != 1 || nloc < 0) { std::fclose(f); return fail(c, WX_ERR_WARM_READ_BLOCKS, "bad header in %s", path); }
  if (nloc > c->max_blocks || nloc > max_slots) {
    std::fclose(f);
    return fail(c, WX_ERR_INSUFICIENT_NBMAXPROC, "%d blocks in %s exceed the %d slots", nloc, path, std::min(c->max_blocks, max_slots));
  }
  const size_t per = (size_t)c->neq * BCELLS;
  const int chunk = 256;
  int rc = ensure_stage(c, chunk * per * 8);
  double* host = nullptr;
  if (!rc && cudaMallocHost(&host, chunk * per * 8) != cudaSuccess) rc = fail(c, WX_ERR_CUDA, "checkpoint buffers");
  std::vector<int32_t> lb(max_slots, -1);
  for (int b0 = 0; !rc && b0 < nloc; b0 += chunk) {
    const int nb = std::min(chunk, nloc - b0);
    for (int b = 0; b < nb; ++b) {
      if (std::fread(&lb[b0 + b], 4, 1, f) != 1 || std::fread(host + b * per, 8, per, f) != per) {
        rc = fail(c, WX_ERR_WARM_READ_BLOCKS, "read %d of %d blocks from %s", b0 + b, nloc, path);
        break;
      }
    }
    if (rc) break;
    cudaMemcpyAsync(c->dStage, host, nb * per * 8, cudaMemcpyHostToDevice, c->stream);
    unpack_bin_kernel<<<1184, 256, 0, c->stream>>>(c->dStage, b0, nb, c->neq, c->dU);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = fail(c, WX_ERR_CUDA, "checkpoint copy");
  }
  std::fclose(f);
  cudaFreeHost(host);
  if (rc) return rc;
  if ((rc = wx3d_set_mesh(c, std::min(max_slots, c->max_blocks), lb.data()))) return rc;
  std::copy(lb.begin(), lb.end(), local_blocks);
  if (nblocks) *nblocks = nloc;
  c->dt_valid = false;
  c->prestep = false;
  c->g_valid = false;
  return WX_OK;
}

// Fortran ES22.15 of x: the exponent letter is dropped when three exponent
// digits are needed.
static void fortran_es22_15(double x, char* out) {   // out: at least 64 bytes
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.15E", x);
  char* e = std::strchr(buf, 'E');
  if (e) {
    const int ex = std::atoi(e + 1);
    if (ex >= 100 || ex <= -100) std::snprintf(e, sizeof buf - (e - buf), "%+04d", ex);
  }
  const size_t n = std::strlen(buf);
  std::memset(out, ' ', 22 > n ? 22 - n : 0);
  std::memcpy(out + (22 > n ? 22 - n : 0), buf, n + 1);
}

// writeState (output.f90:219-263): '(es22.15,i8,i5)' time*t_sc, it, noutput,
// then the data directory.
int wx3d_write_state(wx_ctx* c, const char* path, int32_t noutput, const char* datadir) {
  if (!c || !path) return WX_ERR_INVALID_ARG;
  WX_CUDA(cudaMemcpyAsync(c->hCtl, c->dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(c, WX_ERR_OUTPUT_FILE_OPEN, "could not open %s", path);
  char t[64];
  fortran_es22_15(c->hCtl->time * c->ph.t_sc, t);
  std::fprintf(f, "%s%8d%5d\n%s\n", t, c->hCtl->it, noutput, datadir ? datadir : "");
  return std::fclose(f) == 0 ? WX_OK : fail(c, WX_ERR_OUTPUT_FILE_OPEN, "close failed: %s", path);
}

// warmstart's state read (init.f90:549-573): time (cgs), it and noutput;
// the context takes time/t_sc, it and nextout = noutput + 1.  datadir
// (nbytes, may be NULL) receives the second line.
int wx3d_read_state(wx_ctx* c, const char* path, int32_t* noutput, char* datadir, int32_t nbytes) {
  if (!c || !path) return WX_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "r");
  if (!f) return fail(c, WX_ERR_WARM_FILE_OPEN, "could not open %s", path);
  char line[512] = {0}, dir[512] = {0};
  const bool ok = std::fgets(line, sizeof line, f) != nullptr;
  if (std::fgets(dir, sizeof dir, f)) dir[std::strcspn(dir, "\r\n")] = 0;
  std::fclose(f);
  if (!ok || std::strlen(line) < 35) return fail(c, WX_ERR_WARM_FILE_OPEN, "bad state line in %s", path);
  // fixed columns: 22 for the time, 8 for it, 5 for noutput
  char tt[23] = {0}, ti[9] = {0}, tn[6] = {0};
  std::memcpy(tt, line, 22);
  std::memcpy(ti, line + 22, 8);
  std::memcpy(tn, line + 30, 5);
  // a three-digit exponent without its letter: put the E back
  std::string ts(tt);
  const size_t pos = ts.find_last_of("+-");
  if (ts.find_first_of("Ee") == std::string::npos && pos != std::string::npos && pos > ts.find_first_not_of(' ') + 1)
    ts.insert(pos, "E");
  wx_state st{};
  st.time = std::strtod(ts.c_str(), nullptr) / c->ph.t_sc;
  st.it = std::atoi(ti);
  const int nout = std::atoi(tn);
  st.nextout = nout + 1;
  st.dt = 0.0;
  int rc = wx3d_set_state(c, &st);
  if (rc) return rc;
  if (noutput) *noutput = nout;
  if (datadir && nbytes > 0) {
    std::strncpy(datadir, dir, nbytes - 1);
    datadir[nbytes - 1] = 0;
  }
  return WX_OK;
}

int wx3d_upload_U_fortran(wx_ctx* c, int32_t nbmax, const double* U) {
  if (!c || !U || nbmax <= 0) return WX_ERR_INVALID_ARG;
  const int ns = std::min(nbmax, c->max_blocks);
  const size_t slab = (size_t)nbmax * c->neq * 400;  // U(:,:,:,:,k) for one k
  int rc;
  if ((rc = ensure_stage(c, slab * 8))) return rc;
  for (int kf = 1; kf <= NC; ++kf) {
    WX_CUDA(cudaMemcpyAsync(c->dStage, U + slab * (size_t)(kf + 1), slab * 8, cudaMemcpyHostToDevice, c->stream));
    fortran_to_native<<<c->nsm * 4, 256, 0, c->stream>>>(c->dStage, c->dU, nbmax, ns, c->neq, kf);
    WX_LAUNCHED();
  }
  WX_CUDA(cudaStreamSynchronize(c->stream));
  c->dt_valid = false;
  c->prestep = false;
  c->g_valid = false;
  return WX_OK;
}

int wx3d_download_U_fortran(wx_ctx* c, int32_t nbmax, double* U) {
  if (!c || !U || nbmax <= 0) return WX_ERR_INVALID_ARG;
  const int ns = std::min(nbmax, c->max_blocks);
  const size_t slab = (size_t)nbmax * c->neq * 400;
  int rc;
  if ((rc = ensure_stage(c, slab * 8))) return rc;
  for (int kf = 1; kf <= NC; ++kf) {
    // keep the ghost and unused entries of the caller's slab
    WX_CUDA(cudaMemcpyAsync(c->dStage, U + slab * (size_t)(kf + 1), slab * 8, cudaMemcpyHostToDevice, c->stream));
    native_to_fortran<<<c->nsm * 4, 256, 0, c->stream>>>(c->dU, c->dStage, nbmax, ns, c->neq, kf);
    WX_LAUNCHED();
    WX_CUDA(cudaMemcpyAsync(U + slab * (size_t)(kf + 1), c->dStage, slab * 8, cudaMemcpyDeviceToHost, c->stream));
  }
  WX_CUDA(cudaStreamSynchronize(c->stream));
  return WX_OK;
}

int wx3d_update_prims(wx_ctx* c) {
  if (!ready(c)) return fail(c, WX_ERR_MESH, "no mesh");
  if (!c->dPrim) WX_CUDA(cudaMalloc(&c->dPrim, (size_t)c->max_blocks * c->neq * BCELLS * 8));
  c->k.prims<<<grid_for(c, (const void*)c->k.prims, 256, 0, c->nwork), 256, 0, c->stream>>>(c->dU, c->dPrim, c->dWork,
                                                                                              c->nwork, c->dCtl, c->ph.inv_cv);
  WX_LAUNCHED();
  return sync_check(c);
}

int wx3d_download_prims(wx_ctx* c, int32_t nslots, double* prim) {
  if (!c || !prim || nslots < 0 || nslots > c->max_blocks || !c->dPrim) return WX_ERR_INVALID_ARG;
  WX_CUDA(cudaMemcpyAsync(prim, c->dPrim, (size_t)nslots * c->neq * BCELLS * 8, cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  return WX_OK;
}

int wx3d_set_state(wx_ctx* c, const wx_state* s) {
  if (!c || !s) return WX_ERR_INVALID_ARG;
  WX_CUDA(cudaMemcpyAsync(c->hCtl, c->dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  c->hCtl->time = s->time;
  c->hCtl->dt = s->dt;
  c->hCtl->it = s->it;
  c->hCtl->nextout = s->nextout;
  c->hCtl->dumpout = s->dumpout;
  WX_CUDA(cudaMemcpyAsync(c->dCtl, c->hCtl, sizeof(DevCtl), cudaMemcpyHostToDevice, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  return WX_OK;
}

int wx3d_get_state(wx_ctx* c, wx_state* s) {
  if (!c || !s) return WX_ERR_INVALID_ARG;
  WX_CUDA(cudaMemcpyAsync(c->hCtl, c->dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  s->time = c->hCtl->time;
  s->dt = c->hCtl->dt;
  s->it = c->hCtl->it;
  s->nextout = c->hCtl->nextout;
  s->dumpout = c->hCtl->dumpout;
  s->pad = c->hCtl->dumps;
  return WX_OK;
}

int wx3d_get_timestep(wx_ctx* c, double* dt_glob) {
  if (!ready(c) || !dt_glob) return WX_ERR_INVALID_ARG;
  int rc;
  if (!c->dt_valid) {
    if ((rc = launch_dt(c, c->dU))) return rc;
    c->dt_valid = true;
  }
  WX_CUDA(cudaMemcpyAsync(c->hCtl, c->dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  const DevCtl& h = *c->hCtl;
  double dt_hydro;
  std::memcpy(&dt_hydro, &h.dtmin_bits, 8);
  double dt_loc = c->cfg.cooling_type == WX_COOL_NONE ? dt_hydro * c->cfg.cfl : std::min(dt_hydro, 1.0e30) * c->cfg.cfl;
  if (h.it <= 10) dt_loc = std::ldexp(1.0, -(11 - h.it)) * dt_loc;
  const double tnext = (double)h.nextout * c->cfg.dtout / c->ph.t_sc;
  if (h.time + dt_loc >= tnext) dt_loc = tnext - h.time;
  *dt_glob = dt_loc;
  return WX_OK;
}

int wx3d_hydro_solver(wx_ctx* c) {
  if (!ready(c)) return fail(c, WX_ERR_MESH, "no mesh");
  int rc;
  if (!c->dt_valid) {
    if ((rc = launch_dt(c, c->dU))) return rc;
    c->dt_valid = true;
  }
  if ((rc = enqueue_solver(c, false, false))) return rc;
  return sync_check(c);
}

int wx3d_update_neutral_fraction(wx_ctx* c) {
  if (!ready(c)) return fail(c, WX_ERR_MESH, "no mesh");
  if (c->cfg.eos_type != WX_EOS_H_RATE) return WX_OK;
  int rc;
  if (!c->dPrim && (rc = wx3d_update_prims(c))) return rc;
  if ((rc = enqueue_sources(c, 1 | 4 | (c->cfg.cooling_type == WX_COOL_NONE ? 8 : 0)))) return rc;
  return sync_check(c);
}

int wx3d_cooling(wx_ctx* c, double* maxloss) {
  if (!ready(c)) return fail(c, WX_ERR_MESH, "no mesh");
  int rc;
  if (c->cfg.cooling_type != WX_COOL_NONE) {
    if (!c->dPrim && (rc = wx3d_update_prims(c))) return rc;
    WX_CUDA(cudaMemsetAsync(&c->dCtl->maxloss_bits, 0, 8, c->stream));
    if ((rc = enqueue_sources(c, 2 | 4 | 8))) return rc;
  }
  if ((rc = sync_check(c))) return rc;
  if (maxloss) std::memcpy(maxloss, &c->hCtl->maxloss_bits, 8);
  return WX_OK;
}

// updatePrims + updateNeutralFraction + cooling fused in one pass over U (the
// source part of wx3d_step), with the surrogate when one is attached.
int wx3d_sources(wx_ctx* c, double* maxloss) {
  if (!ready(c)) return fail(c, WX_ERR_MESH, "no mesh");
  int rc;
  c->nev = 0;
  WX_CUDA(cudaMemsetAsync(&c->dCtl->maxloss_bits, 0, 8, c->stream));
  if (c->use_surrogate) {
    if ((rc = enqueue_surrogate(c))) return rc;
  } else if (sources_on(c)) {
    int mode = 8;
    if (c->cfg.eos_type == WX_EOS_H_RATE) mode |= 1;
    if (c->cfg.cooling_type != WX_COOL_NONE) mode |= 2;
    if ((rc = enqueue_sources(c, mode))) return rc;
  }
  if ((rc = sync_check(c))) return rc;
  if (maxloss) std::memcpy(maxloss, &c->hCtl->maxloss_bits, 8);
  return WX_OK;
}

int wx3d_step(wx_ctx* c, wx_state* out) {
  if (!ready(c)) return fail(c, WX_ERR_MESH, "no mesh");
  const int dumps0 = c->hCtl->dumps;
  int rc;
  c->nev = 0;
  if ((rc = enqueue_step(c))) return rc;
  if ((rc = sync_check(c))) return rc;
  if (out) {
    const DevCtl& h = *c->hCtl;
    out->time = h.time; out->dt = h.dt; out->it = h.it; out->nextout = h.nextout;
    out->dumpout = h.dumps != dumps0; out->pad = h.dumps;
  }
  return WX_OK;
}

int wx3d_run_async(wx_ctx* c, int32_t nsteps) {
  if (!ready(c) || nsteps < 0) return WX_ERR_INVALID_ARG;
  int rc;
  if (!c->dt_valid) {
    if ((rc = launch_dt(c, c->dU))) return rc;
    c->dt_valid = true;
  }
  int done = 0;
  if (nsteps >= 2) {
    if (!c->graph_valid) {
      // two steps bring U back to the same buffer, so one graph serves every replay
      double* u0 = c->dU;
      cudaGraph_t g;
      const long long l0 = c->launches;
      c->nev = 0;
      WX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int r1 = enqueue_step(c);
      int r2 = r1 ? r1 : enqueue_step(c);
      cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
      c->launches = l0;
      if (r2) return r2;
      if (ce != cudaSuccess) return fail(c, WX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      if (c->dU != u0) return fail(c, WX_ERR_GENERIC, "graph capture did not return U to its buffer");
      ce = cudaGraphInstantiate(&c->graph, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return fail(c, WX_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      c->graph_valid = true;
    }
    // kernels per step: step_begin, stage(s), viscous, step_end, [dt reset, sources]
    const long long per2 = 2 * (3 + (c->cfg.solver_type == WX_SOLVER_LAX || c->cfg.solver_type == WX_SOLVER_HLL1 ? 1 : 2) +
                                (sources_on(c) ? 2 : 0));
    for (; done + 2 <= nsteps; done += 2) {
      WX_CUDA(cudaGraphLaunch(c->graph, c->stream));
      c->launches += per2;
    }
    c->prestep = true;
    c->dt_valid = true;
  }
  // an odd remainder runs eagerly; its kernels are not timed so the event
  // pairs keep describing the last graph replay
  c->timing_mute = done > 0;
  if (done == 0) c->nev = 0;
  for (; done < nsteps; ++done)
    if ((rc = enqueue_step(c))) { c->timing_mute = false; return rc; }
  c->timing_mute = false;
  return WX_OK;
}

int wx3d_run(wx_ctx* c, int32_t nsteps, wx_state* out) {
  int rc;
  if ((rc = wx3d_run_async(c, nsteps))) return rc;
  if ((rc = sync_check(c))) return rc;
  if (out) {
    const DevCtl& h = *c->hCtl;
    out->time = h.time; out->dt = h.dt; out->it = h.it; out->nextout = h.nextout;
    out->dumpout = 0; out->pad = h.dumps;
  }
  return WX_OK;
}

int wx3d_set_cooltable(wx_ctx* c, int32_t npts, const double* logT, const double* b) {
  if (!c || !logT || !b) return WX_ERR_INVALID_ARG;
  if (npts < 2) return fail(c, WX_ERR_COOLING_LOAD_COEFS, "cooling table needs at least two rows");
  std::vector<double> h(2 * (size_t)npts);
  for (int i = 0; i < npts; ++i) {
    if (i && !(logT[i] > logT[i - 1])) return fail(c, WX_ERR_COOLING_LOAD_COEFS, "cooling table temperatures must increase");
    h[i] = logT[i];
    h[npts + i] = -b[i];  // cooltable(2,i) = -b (cooling.f90:163)
  }
  cudaFree(c->dCool);
  c->dCool = nullptr;
  WX_CUDA(cudaMalloc(&c->dCool, h.size() * 8));
  WX_CUDA(cudaMemcpy(c->dCool, h.data(), h.size() * 8, cudaMemcpyHostToDevice));
  c->ncool = npts;
  c->nZ = 0;
  invalidate_graph(c);
  return WX_OK;
}

// loadcooldata_metal (cooling.f90:193-265): table[(nptsT+1)*(nptsZ+1)] row
// by row as the file lists it (first row: metallicities after an unused
// entry; then per row log T followed by log Lambda per metallicity).
int wx3d_set_cooltable_metal(wx_ctx* c, int32_t nptsT, int32_t nptsZ, const double* table) {
  if (!c || !table) return WX_ERR_INVALID_ARG;
  if (nptsT < 2 || nptsZ < 2) return fail(c, WX_ERR_COOLING_LOAD_COEFS, "metal cooling table needs 2 x 2 values");
  const int W = nptsZ + 1;
  std::vector<double> h(table, table + (size_t)(nptsT + 1) * W);
  h[0] = -1.0;
  for (int i = 2; i <= nptsT; ++i)
    if (!(h[(size_t)i * W] > h[(size_t)(i - 1) * W])) return fail(c, WX_ERR_COOLING_LOAD_COEFS, "temperatures must increase");
  for (int j = 2; j <= nptsZ; ++j)
    if (!(h[j] > h[j - 1])) return fail(c, WX_ERR_COOLING_LOAD_COEFS, "metallicities must increase");
  cudaFree(c->dCool);
  c->dCool = nullptr;
  WX_CUDA(cudaMalloc(&c->dCool, h.size() * 8));
  WX_CUDA(cudaMemcpy(c->dCool, h.data(), h.size() * 8, cudaMemcpyHostToDevice));
  c->ncool = nptsT;
  c->nZ = nptsZ;
  invalidate_graph(c);
  return WX_OK;
}

// loadcooldata_schure (cooling_schure.f90:52-95): 180 rows of five columns
// as in the table file; column 1+dmc_f (1..4) holds -log10 Lambda.
int wx3d_set_cooltable_schure(wx_ctx* c, const double* data, int32_t dmc_f) {
  if (!c || !data) return WX_ERR_INVALID_ARG;
  if (dmc_f < 1 || dmc_f > 4) return fail(c, WX_ERR_COOLING_LOAD_COEFS, "dmc_f selects column 2..5 (1..4)");
  std::vector<double> h(360);
  for (int i = 0; i < 180; ++i) {
    h[i] = std::pow(10.0, data[5 * i]);
    h[180 + i] = std::pow(10.0, -data[5 * i + dmc_f]);
  }
  cudaFree(c->dCool);
  c->dCool = nullptr;
  WX_CUDA(cudaMalloc(&c->dCool, h.size() * 8));
  WX_CUDA(cudaMemcpy(c->dCool, h.data(), h.size() * 8, cudaMemcpyHostToDevice));
  c->ncool = 180;
  c->nZ = 0;
  invalidate_graph(c);
  return WX_OK;
}

int wx3d_mark(wx_ctx* c, int32_t nslots, int32_t* flags) {
  if (!ready(c) || !flags || nslots > c->max_blocks) return WX_ERR_INVALID_ARG;
  WX_CUDA(cudaMemsetAsync(c->dFlags, 0xff, 4 * (size_t)c->max_blocks, c->stream));
  MarkParams P{c->dU, c->prestep ? c->dW : c->dU, c->dBlocks, c->dWork, c->nwork, c->dFlags, c->cfg.maxlev,
               c->cfg.refine_thres, c->cfg.coarse_thres, c->ph, c->prestep && c->g_valid ? c->dG : nullptr};
  c->k.mark<<<grid_for(c, (const void*)c->k.mark, 256, 0, c->nwork), 256, 0, c->stream>>>(P);
  WX_LAUNCHED();
  WX_CUDA(cudaMemcpyAsync(flags, c->dFlags, 4 * (size_t)nslots, cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  return WX_OK;
}

int wx3d_refine(wx_ctx* c, int32_t father, const int32_t* ch) {
  if (!c || !ch || father < 0 || father >= c->max_blocks) return WX_ERR_INVALID_ARG;
  Slots8 s;
  for (int i = 0; i < 8; ++i) {
    if (ch[i] < 0 || ch[i] >= c->max_blocks || ch[i] == father) return WX_ERR_INVALID_ARG;
    s.s[i] = ch[i];
  }
  refine_kernel<<<dim3(16, 8), 256, 0, c->stream>>>(c->dU, c->neq, father, s);
  WX_LAUNCHED();
  WX_CUDA(cudaStreamSynchronize(c->stream));
  c->dt_valid = false;
  c->prestep = false;
  c->g_valid = false;
  invalidate_graph(c);
  return WX_OK;
}

// ---------------------------------------------------------------------------
// admesh (amr.f90:44-133) of one process.
namespace {

// localBlocks with the reference's registry operations (utils.f90:78-172):
// find by bID, put into the first empty slot, pop (free) a block's slot;
// a hash table and a min-heap of the empty slots instead of linear scans.
struct SlotList {
  std::vector<int32_t> lb;
  SlotMap at;
  std::priority_queue<int, std::vector<int>, std::greater<int>> empty;
  explicit SlotList(const std::vector<int32_t>& l) : lb(l), at(l.size()) {
    std::vector<int> e;
    for (int s = 0; s < (int)lb.size(); ++s) {
      if (lb[s] == -1) e.push_back(s);
      else at.insert(lb[s], s);
    }
    empty = decltype(empty)(std::greater<int>(), std::move(e));
  }
  int find(long long id) const { return at.find(id); }
  int put(long long id) {
    if (empty.empty()) return -1;
    const int s = empty.top();
    empty.pop();
    lb[s] = (int32_t)id;
    at.insert(id, s);
    return s;
  }
  void pop(long long id) {
    const int s = at.find(id);
    if (s < 0) return;
    lb[s] = -1;
    empty.push(s);
    at.erase(id);
  }
};

long long tree_father(const Tree& T, long long id) {  // amr.f90:916-961
  const int l = T.level(id);
  if (l <= 1) return -1;
  int x[3];
  T.coords(id, l, x);
  const int y[3] = {x[0] / 2, x[1] / 2, x[2] / 2};
  return T.id(l - 1, y);
}

void tree_children(const Tree& T, long long id, long long out[8]) {  // amr.f90:882-909, x fastest
  const int l = T.level(id);
  int x[3];
  T.coords(id, l, x);
  for (int c = 0; c < 8; ++c) {
    const int y[3] = {2 * x[0] + (c & 1), 2 * x[1] + ((c >> 1) & 1), 2 * x[2] + (c >> 2)};
    out[c] = T.id(l + 1, y);
  }
}

// Same-level region across face f (0..5 = left..top), -1 at the domain edge
// (neighborLevel, amr.f90:439-523).
long long tree_region(const Tree& T, long long id, int f) {
  const int l = T.level(id);
  int x[3];
  T.coords(id, l, x);
  const int ax = f / 2;
  x[ax] += (f & 1) ? 1 : -1;
  if (x[ax] < 0 || x[ax] >= T.nb[l][ax]) return -1;
  return T.id(l, x);
}

// checkProximity (amr.f90:1109-1254) over the synchronised flags, level
// finest down to 1, blocks in slot order; flags change as the sweep goes.
void check_proximity(const Tree& T, const SlotList& L, std::vector<int>& flags, int finest) {
  const std::vector<int32_t>& glob = L.lb;
  std::vector<std::vector<int>> by_level(T.maxlev + 1);  // occupied slots per level, ascending
  for (int nb = 0; nb < (int)glob.size(); ++nb)
    if (glob[nb] != -1) by_level[T.level(glob[nb])].push_back(nb);
  for (int level = finest; level >= 1; --level)
    for (const int nb : by_level[level]) {
      const long long id = glob[nb];
      const int bflag = flags[nb];
      if (bflag == WX_FLAG_REFINE) {
        for (int f = 0; f < 6; ++f) {
          const long long n = tree_region(T, id, f);
          if (n < 0) continue;
          const int s = L.find(n);
          if (s >= 0) {  // same level: its coarsening is inhibited
            if (flags[s] == WX_FLAG_COARSE) flags[s] = WX_FLAG_NONE;
            continue;
          }
          const int sf = L.find(tree_father(T, n));
          if (sf >= 0 && flags[sf] != WX_FLAG_REFINE) flags[sf] = WX_FLAG_REFINE;  // coarser: refined too
        }
      }
      if (bflag == WX_FLAG_COARSE) {
        bool inhibited = false;
        for (int f = 0; f < 6 && !inhibited; ++f) {
          const long long n = tree_region(T, id, f);
          if (n < 0 || L.find(n) >= 0 || L.find(tree_father(T, n)) >= 0 || level >= T.maxlev) continue;
          long long sib[8];  // finer neighbour: all eight children of the region
          tree_children(T, n, sib);
          for (int i = 0; i < 8; ++i) {
            const int s = L.find(sib[i]);
            if (s >= 0 && flags[s] != WX_FLAG_COARSE) {
              flags[nb] = WX_FLAG_NONE;
              inhibited = true;
              break;
            }
          }
        }
      }
    }
}

}  // namespace

int wx3d_admesh(wx_ctx* c, int32_t nbmax, int32_t* lb, int32_t* counts) {
  if (!ready(c) || !lb) return WX_ERR_INVALID_ARG;
  if (nbmax != c->max_blocks) return fail(c, WX_ERR_INVALID_ARG, "local_blocks must have max_blocks (%d) entries", c->max_blocks);
  if (c->nhalo > 0) return fail(c, WX_ERR_UNSUPPORTED, "admesh of a partitioned mesh");
  for (int s = 0; s < nbmax; ++s)
    if (lb[s] != c->local[s]) return fail(c, WX_ERR_MESH, "slot %d: local_blocks differs from the mesh last set", s);
  const Tree& T = c->tree;
  // From now on the steps' first-order stage leaves the ghost primitives the
  // marking reads (the record is allocated once; without it the marking
  // gathers them from the neighbour slots).
  if (!c->mark_ghosts) {
    if (!c->dG && cudaMalloc(&c->dG, sizeof(double) * 2 * GFRAME * (size_t)c->max_blocks) != cudaSuccess) {
      cudaGetLastError();
      c->dG = nullptr;
    }
    c->mark_ghosts = c->dG != nullptr;
    invalidate_graph(c);
  }
  // markByPhysical on the device; empty slots keep FLAG_NONE
  std::vector<int32_t> mk(nbmax);
  int rc = wx3d_mark(c, nbmax, mk.data());
  if (rc) return rc;
  std::vector<int> flags(nbmax, WX_FLAG_NONE);
  for (int s = 0; s < nbmax; ++s)
    if (lb[s] != -1) flags[s] = mk[s];
  SlotList L(c->local);
  check_proximity(T, L, flags, c->cfg.maxlev - 1);
  // refineBlock for the marked blocks, in slot order of the list before it
  const std::vector<int32_t> glob = c->local;
  int nbLocal = (int)L.at.size();
  std::vector<int32_t> rops, cops;
  for (int nb = 0; nb < nbmax; ++nb) {
    const long long id = glob[nb];
    if (id == -1 || flags[nb] != WX_FLAG_REFINE) continue;
    const int fi = L.find(id);
    if (T.level(id) == c->cfg.maxlev) return fail(c, WX_ERR_ALREADY_MAX_LEV, "bID %lld is at the finest level", id);
    if (nbLocal + 8 > nbmax)
      return fail(c, WX_ERR_INSUFICIENT_NBMAXPROC, "refining bID %lld needs 8 slots; %d of %d are used", id, nbLocal, nbmax);
    long long ch[8];
    tree_children(T, id, ch);
    rops.push_back(fi);
    for (int k = 0; k < 8; ++k) rops.push_back(L.put(ch[k]));
    L.pop(id);
    nbLocal += 7;
  }
  // coarseBlocks: families in the order their first marked member appears
  // (flags stay indexed by the slots before refinement; a new child only
  // takes an empty or a refined father's slot, never a COARSE one)
  std::vector<long long> fam;
  std::unordered_map<long long, int> count;
  for (int nb = 0; nb < nbmax; ++nb) {
    const long long id = L.lb[nb];
    if (id == -1 || flags[nb] != WX_FLAG_COARSE) continue;
    long long sib[8];
    tree_children(T, tree_father(T, id), sib);
    if (count[sib[0]]++ == 0) fam.push_back(sib[0]);
  }
  int ncoarse = 0;
  for (long long e : fam) {
    if (count[e] != 8) continue;
    const long long fid = tree_father(T, e);
    long long sib[8];
    tree_children(T, fid, sib);
    const int fslot = L.put(fid);
    if (fslot < 0) return fail(c, WX_ERR_REGISTER_FATHER, "no free slot for father bID %lld", fid);
    cops.push_back(fslot);
    for (int k = 0; k < 8; ++k) {
      cops.push_back(L.find(sib[k]));
      L.pop(sib[k]);
    }
    ++ncoarse;
  }
  if (counts) {
    counts[0] = (int32_t)(rops.size() / 9);
    counts[1] = ncoarse;
  }
  if (rops.empty() && cops.empty()) return WX_OK;  // the mesh and the state stay as they are
  // the new mesh is checked before any data moves, so a refused mesh
  // leaves the state and the slot registry as they were
  std::vector<int32_t> work;
  if ((rc = build_any(c, nbmax, L.lb.data(), 0, nullptr, work))) return rc;
  // data: refinements, then coarsenings.  Each pass first copies the blocks
  // it reads (fathers, or siblings) from U into UP at the same slots -- UP
  // holds nothing between steps, the next predictor overwrites it -- then
  // reads them there, so slots freed and taken again within the pass need no
  // ordering.
  {
    if (!c->dOps) WX_CUDA(cudaMalloc(&c->dOps, sizeof(int32_t) * 9 * (size_t)c->max_blocks));
    for (int pass = 0; pass < 2; ++pass) {
      const std::vector<int32_t>& ops = pass == 0 ? rops : cops;
      if (ops.empty()) continue;
      WX_CUDA(cudaMemcpyAsync(c->dOps, ops.data(), 4 * ops.size(), cudaMemcpyHostToDevice, c->stream));
      const int nops = (int)(ops.size() / 9), per = pass == 0 ? 1 : 8, off = pass == 0 ? 0 : 1;
      for (int o = 0; o < nops; o += 8000) {
        const int n = std::min(8000, nops - o);
        stage_blocks_kernel<<<dim3(8, per * n), 256, 0, c->stream>>>(c->dU, c->dUP, c->neq, c->dOps + 9 * o, per, off);
        WX_LAUNCHED();
      }
      for (int o = 0; o < nops; o += 8000) {
        const int n = std::min(8000, nops - o);
        if (pass == 0) refine_batch_kernel<<<dim3(16, 8 * n), 256, 0, c->stream>>>(c->dUP, c->dU, c->neq, c->dOps + 9 * o);
        else coarsen_batch_kernel<<<dim3(4, 8 * n), 256, 0, c->stream>>>(c->dUP, c->dU, c->neq, c->dOps + 9 * o);
        WX_LAUNCHED();
      }
      WX_CUDA(cudaStreamSynchronize(c->stream));  // dOps is refilled by the next pass
    }
  }
  const int zsplit = c->zsplit;  // the launch shape chosen for the context stays
  if ((rc = commit_mesh(c, nbmax, L.lb.data(), 0, work))) return rc;
  c->zsplit = zsplit;
  std::copy(L.lb.begin(), L.lb.end(), lb);
  return WX_OK;
}

int wx3d_coarsen(wx_ctx* c, const int32_t* ch, int32_t father) {
  if (!c || !ch || father < 0 || father >= c->max_blocks) return WX_ERR_INVALID_ARG;
  Slots8 s;
  for (int i = 0; i < 8; ++i) {
    if (ch[i] < 0 || ch[i] >= c->max_blocks || ch[i] == father) return WX_ERR_INVALID_ARG;
    s.s[i] = ch[i];
  }
  coarsen_kernel<<<dim3(4, 8), 256, 0, c->stream>>>(c->dU, c->neq, father, s);
  WX_LAUNCHED();
  WX_CUDA(cudaStreamSynchronize(c->stream));
  c->dt_valid = false;
  c->prestep = false;
  c->g_valid = false;
  invalidate_graph(c);
  return WX_OK;
}

int wx3d_set_timing(wx_ctx* c, int32_t on) {
  if (!c) return WX_ERR_INVALID_ARG;
  if (on && !c->ev[0])
    for (int i = 0; i < 64; ++i) WX_CUDA(cudaEventCreate(&c->ev[i]));
  c->timing = on != 0;
  c->nev = 0;
  invalidate_graph(c);
  return WX_OK;
}

int wx3d_kernel_times(wx_ctx* c, double* ms4, int32_t* count4) {
  if (!c || !ms4) return WX_ERR_INVALID_ARG;
  WX_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 4; ++k) { ms4[k] = 0.0; if (count4) count4[k] = 0; }
  for (int p = 0; p + 1 < c->nev; p += 2) {
    float ms = 0.f;
    WX_CUDA(cudaEventElapsedTime(&ms, c->ev[p], c->ev[p + 1]));
    const int k = c->ev_kind[p / 2];
    ms4[k] += ms;
    if (count4) ++count4[k];
  }
  return WX_OK;
}

// Measured FP64 FMA throughput of the device (GFLOP/s, one FMA = 2 flops):
// the compute roofline of the stage kernels, which are bound by FP64 issue.
int wx3d_measure_fp64_peak(double* gflops) {
  if (!gflops) return WX_ERR_INVALID_ARG;
  int ndev = 0, dev = 0, nsm = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return WX_ERR_NO_DEVICE;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  double* d = nullptr;
  if (cudaMalloc(&d, 8) != cudaSuccess) return WX_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int grid = nsm * 8;
  float best = 1e30f;
  for (int r = 0; r < 6; ++r) {
    cudaEventRecord(e0);
    fp64_peak_kernel<<<grid, 256>>>(d, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;
  }
  const cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  if (e != cudaSuccess) return WX_ERR_CUDA;
  *gflops = 2.0 * 8.0 * 4096.0 * 256.0 * grid / (best * 1e-3) / 1e9;
  return WX_OK;
}

// Largest distance in ulp of rcp_nr / sqrt_nr from the device's IEEE 1/x and
// sqrt(x) over n host arguments.
int wx3d_check_fast_math(int32_t n, const double* host_x, int64_t* max_ulp2) {
  if (n <= 0 || !host_x || !max_ulp2) return WX_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return WX_ERR_NO_DEVICE;
  double* dx = nullptr;
  unsigned long long* du = nullptr;
  if (cudaMalloc(&dx, sizeof(double) * n) != cudaSuccess) return WX_ERR_CUDA;
  if (cudaMalloc(&du, 16) != cudaSuccess) { cudaFree(dx); return WX_ERR_CUDA; }
  cudaMemcpy(dx, host_x, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaMemset(du, 0, 16);
  fast_math_check_kernel<<<256, 256>>>(dx, n, du);
  unsigned long long h[2] = {0, 0};
  const cudaError_t e = cudaMemcpy(h, du, 16, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(du);
  if (e != cudaSuccess) return WX_ERR_CUDA;
  max_ulp2[0] = (int64_t)h[0];
  max_ulp2[1] = (int64_t)h[1];
  return WX_OK;
}

// Attaches (enable=1) or detaches the learned surrogate of hrate + cooling_h.
int wx3d_set_surrogate(wx_ctx* c, wx_mlp* mlp, const uint8_t* trust, int32_t nbytes, int32_t enable) {
  if (!c) return WX_ERR_INVALID_ARG;
  if (!enable) {
    c->use_surrogate = false;
    invalidate_graph(c);
    return WX_OK;
  }
  if (!mlp || !trust || nbytes != TRUST_BYTES) return fail(c, WX_ERR_INVALID_ARG, "surrogate needs a %d-byte trust table", TRUST_BYTES);
  const wx_config& f = c->cfg;
  if (f.eos_type != WX_EOS_H_RATE || f.bfield || f.npassive < 1 || f.neqtot > 7)
    return fail(c, WX_ERR_UNSUPPORTED, "the surrogate replaces the EOS_H_RATE update in hydro runs with 1-2 passives");
  if (f.cooling_type == WX_COOL_H && f.cooling_limit != 0.5)
    return fail(c, WX_ERR_UNSUPPORTED, "the surrogate's cooling_h output was trained with cooling_limit = 0.5");
  if (!c->dTrust) WX_CUDA(cudaMalloc(&c->dTrust, TRUST_BYTES));
  WX_CUDA(cudaMemcpy(c->dTrust, trust, TRUST_BYTES, cudaMemcpyHostToDevice));
  c->mlp = mlp;
  c->use_surrogate = true;
  invalidate_graph(c);
  return WX_OK;
}

int wx3d_get_status(wx_ctx* c, wx_status* st) {
  if (!c || !st) return WX_ERR_INVALID_ARG;
  WX_CUDA(cudaMemcpyAsync(c->hCtl, c->dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  st->pressure_floor = (int64_t)c->hCtl->cnt[0];
  st->density_floor = (int64_t)c->hCtl->cnt[1];
  st->zero_density = (int64_t)c->hCtl->cnt[2];
  st->nan_cells = (int64_t)c->hCtl->cnt[3];
  std::memcpy(&st->max_cool_loss, &c->hCtl->maxloss_bits, 8);
  st->kernels_launched = c->launches;
  st->surrogate_cells = (int64_t)c->hCtl->sur[0];
  st->fallback_cells = (int64_t)c->hCtl->sur[1];
  return WX_OK;
}

int wx3d_reset_status(wx_ctx* c) {
  if (!c) return WX_ERR_INVALID_ARG;
  WX_CUDA(cudaMemsetAsync(&c->dCtl->cnt[0], 0, sizeof(c->hCtl->cnt) + 8, c->stream));
  WX_CUDA(cudaMemsetAsync(&c->dCtl->sur[0], 0, sizeof(c->hCtl->sur), c->stream));
  WX_CUDA(cudaStreamSynchronize(c->stream));
  return WX_OK;
}

}  // extern "C"

// =============================================================================
// Allocation-free hydro step.
//
// Some callers cannot call cudaMalloc: a host whose device memory is owned by
// its own pool or framework allocator (foreign allocations are forbidden or
// invisible to its accounting), code that must not grow its footprint after
// start-up, and embedded drivers that only hand out pointers into buffers
// they already own.  wx3d_hydro_step_noalloc serves them: the caller passes
// the input and output state in its own device memory, and everything else
// the step needs lives in one file-scope device array of fixed size.
//
// The scratch holds the predictor state UP of up to WX3D_NOALLOC_MAX_BLOCK_EQS
// block-equations (blocks x neqtot <= 320, i.e. 10 MiB), the neighbour table,
// the work list and the step-control block.  Every GPU that loads this
// library reserves the array until the process exits.  All calls share it
// and it keeps the last call's contents: the control block (time, dt, CFL
// minimum, counters) is rewritten from the host at the start of every call,
// and the predictor stage rewrites every UP cell the later kernels read.
// Calls whose work overlaps on the GPU (two streams, or two host threads)
// race on the array and must be serialised by the caller.

namespace {

constexpr int NOALLOC_MAX_BLOCK_EQS = WX3D_NOALLOC_MAX_BLOCK_EQS;
constexpr int NOALLOC_MAX_BLOCKS = WX3D_NOALLOC_MAX_BLOCK_EQS / 5;  // neqtot >= 5
constexpr size_t NOALLOC_UP_BYTES = (size_t)NOALLOC_MAX_BLOCK_EQS * BCELLS * sizeof(double);
constexpr size_t NOALLOC_TABLE_OFF = NOALLOC_UP_BYTES;
constexpr size_t NOALLOC_WORK_OFF = NOALLOC_TABLE_OFF + ((sizeof(DevBlock) * NOALLOC_MAX_BLOCKS + 255) / 256) * 256;
constexpr size_t NOALLOC_CTL_OFF = NOALLOC_WORK_OFF + ((4 * NOALLOC_MAX_BLOCKS + 255) / 256) * 256;
constexpr size_t NOALLOC_BYTES = NOALLOC_CTL_OFF + ((sizeof(DevCtl) + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Device address of g_noalloc_scratch (the symbol is a host-side stand-in in
// host code).  It is looked up with cudaGetSymbolAddress, with the device
// current, on the first call on a device, and again whenever the current
// driver context differs from the one the cached address belongs to: a
// primary context that was reset and recreated, or a caller's own driver-API
// context, loads the module at another address.  The cache is guarded by a
// mutex, so host threads making their first calls together are safe (their
// GPU work still shares the array, see above).
constexpr int NOALLOC_MAX_DEVICES = 64;
struct NoallocAddr {
  void* ctx = nullptr;          // driver context the address belongs to (nullptr: unknown)
  unsigned char* ptr = nullptr;
};
std::mutex g_noalloc_mu;
NoallocAddr g_noalloc_addr[NOALLOC_MAX_DEVICES];

// The current driver context (CUcontext), through the runtime's driver entry
// point so the library needs no link against libcuda; nullptr when it cannot
// be told, in which case the address is looked up on every call.
void* noalloc_current_context() {
  using CtxGetCurrent = int (*)(void**);
  static const CtxGetCurrent fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<CtxGetCurrent>(p);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

int noalloc_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return WX_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoallocAddr& a = g_noalloc_addr[dev];
  void* ctx = noalloc_current_context();
  if (!a.ptr || !ctx || ctx != a.ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      a = NoallocAddr{};
      std::fprintf(stderr, "wx3d_hydro_step_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return WX_ERR_CUDA;
    }
    a.ptr = static_cast<unsigned char*>(p);
    a.ctx = noalloc_current_context();  // the lookup may have made the primary context current
  }
  *out = a.ptr;
  return WX_OK;
}

// Neighbour table of one registry (same construction as wx3d_set_mesh, kept
// separate so that entry point is unchanged).  Fixed-size arrays and a linear
// bID lookup: at most NOALLOC_MAX_BLOCKS slots, and no heap use.
int noalloc_find(const int32_t* lb, int n, long long id) {
  for (int s = 0; s < n; ++s)
    if (lb[s] == id) return s;
  return -1;
}

int noalloc_table(const wx_config& cfg, int n, const int32_t* lb, DevBlock* hb, int32_t* work, int* nwork) {
  Tree T;
  T.init(cfg);
  for (int s = 0; s < n; ++s) {
    if (lb[s] == -1) continue;
    if (T.level(lb[s]) < 1 || noalloc_find(lb, s, lb[s]) >= 0) return WX_ERR_MESH;
  }
  *nwork = 0;
  for (int s = 0; s < n; ++s) {
    hb[s] = DevBlock{};
    if (lb[s] == -1) continue;
    DevBlock b{};
    const long long id = lb[s];
    const int l = T.level(id);
    int x[3];
    T.coords(id, l, x);
    b.level = l;
    b.bID = (int32_t)id;
    for (int d = 0; d < 3; ++d) {
      b.bc[d] = x[d] + 1;
      b.sib[d] = l > 1 ? (x[d] & 1) : -1;
    }
    const double s2 = std::ldexp(1.0, l - 1);
    b.dx = cfg.xphystot / ((double)(NC * cfg.nbrootx) * s2) / cfg.l_sc;
    b.dy = cfg.yphystot / ((double)(NC * cfg.nbrooty) * s2) / cfg.l_sc;
    b.dz = cfg.zphystot / ((double)(NC * cfg.nbrootz) * s2) / cfg.l_sc;
    for (int f = 0; f < 6; ++f) {
      const int ax = f / 2, side = f & 1;
      for (int q = 0; q < 4; ++q) b.fnb[f][q] = -1;
      int y[3] = {x[0], x[1], x[2]};
      y[ax] += side ? 1 : -1;
      if (y[ax] < 0 || y[ax] >= T.nb[l][ax]) {
        b.ftype[f] = WX_NEIGH_BOUNDARY;
        b.fnb[f][0] = cfg.bc[f];
        continue;
      }
      int ns = noalloc_find(lb, n, T.id(l, y));
      if (ns >= 0) { b.ftype[f] = WX_NEIGH_SAME; b.fnb[f][0] = ns; continue; }
      if (l > 1) {
        int z[3] = {y[0] / 2, y[1] / 2, y[2] / 2};
        ns = noalloc_find(lb, n, T.id(l - 1, z));
        if (ns >= 0) { b.ftype[f] = WX_NEIGH_COARSER; b.fnb[f][0] = ns; continue; }
      }
      if (l >= T.maxlev) return WX_ERR_MESH;
      const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
      b.ftype[f] = WX_NEIGH_FINER;
      for (int q = 0; q < 4; ++q) {
        int ch[3];
        ch[ax] = 2 * y[ax] + (side ? 0 : 1);
        ch[t1] = 2 * y[t1] + (q & 1);
        ch[t2] = 2 * y[t2] + (q >> 1);
        ns = noalloc_find(lb, n, T.id(l + 1, ch));
        if (ns < 0) return WX_ERR_MESH;
        b.fnb[f][q] = ns;
      }
    }
    hb[s] = b;
    work[(*nwork)++] = s;
  }
  return WX_OK;
}

// Physical parameters of a bare config (as fill_phys does for a context).
void noalloc_phys(const wx_config& f, PhysParams& p) {
  p.gamma = f.gamma;
  p.cv = 1.0 / (f.gamma - 1.0);
  p.inv_cv = 1.0 / p.cv;
  p.cfl = f.cfl;
  p.eta = f.visc_eta;
  p.mu0 = f.mu0; p.mui = f.mui; p.ion_thres = f.ion_thres;
  p.d_sc = f.d_sc;
  p.p_sc = f.d_sc * (f.v_sc * f.v_sc);
  p.e_sc = p.p_sc;
  p.t_sc = f.l_sc / f.v_sc;
  p.dtout = f.dtout;
  p.cooling_limit = f.cooling_limit;
  p.limiter = f.limiter_type;
  p.eight_wave = f.eight_wave;
  p.flux_cd = f.enable_flux_cd;
  for (int i = 0; i < 6; ++i) p.bc[i] = f.bc[i];
  p.eos = f.eos_type;
  p.cooling = f.cooling_type;
  p.fp = 5 + 3 * (f.bfield ? 1 : 0);
  p.npassive = f.npassive;
  p.l_sc = f.l_sc;
  p.v_sc = f.v_sc;
}

int noalloc_grid(const void* fn, int threads, size_t smem, int items, int nsm) {
  int per = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem);
  per = std::max(per, 1);
  return std::max(1, std::min(items, per * nsm));
}

}  // namespace

extern "C" int wx3d_hydro_step_noalloc(const wx_config* cfg, int32_t nslots, const int32_t* local_blocks,
                                       const double* u_in, double* u_out, wx_state* state, void* cuda_stream) {
  if (!cfg || !local_blocks || !u_in || !u_out || !state || nslots <= 0) return WX_ERR_INVALID_ARG;
  std::string why;
  int rc = validate(*cfg, why);
  if (rc) { std::fprintf(stderr, "wx3d_hydro_step_noalloc: %s\n", why.c_str()); return rc; }
  if (cfg->eos_type == WX_EOS_H_RATE || cfg->cooling_type != WX_COOL_NONE) {
    std::fprintf(stderr, "wx3d_hydro_step_noalloc: source terms are not part of the allocation-free step\n");
    return WX_ERR_UNSUPPORTED;
  }
  if ((long long)nslots * cfg->neqtot > NOALLOC_MAX_BLOCK_EQS || nslots > NOALLOC_MAX_BLOCKS) {
    std::fprintf(stderr,
                 "wx3d_hydro_step_noalloc: %d slots x %d equations exceeds the fixed scratch of %d block-equations "
                 "(%d blocks); use wx3d_init/wx3d_step for larger meshes\n",
                 nslots, cfg->neqtot, NOALLOC_MAX_BLOCK_EQS, NOALLOC_MAX_BLOCKS);
    return WX_ERR_INSUFICIENT_NBMAXPROC;
  }
  {
    // u_in is read by every stage while u_out is written: the two ranges must
    // be disjoint (an aliased Lax-Friedrichs or HLL1 step would race)
    const size_t bytes = (size_t)nslots * cfg->neqtot * BCELLS * sizeof(double);
    const uintptr_t a0 = reinterpret_cast<uintptr_t>(u_in), b0 = reinterpret_cast<uintptr_t>(u_out);
    if (a0 < b0 + bytes && b0 < a0 + bytes) {
      std::fprintf(stderr, "wx3d_hydro_step_noalloc: u_in and u_out overlap\n");
      return WX_ERR_INVALID_ARG;
    }
  }
  Kern k;
  if (!select_kern(*cfg, k)) return WX_ERR_UNSUPPORTED;
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) != cudaSuccess) return WX_ERR_NO_DEVICE;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  unsigned char* base = nullptr;
  if ((rc = noalloc_scratch(dev, &base))) return rc;
  double* dUP = reinterpret_cast<double*>(base);
  DevBlock* dBlocks = reinterpret_cast<DevBlock*>(base + NOALLOC_TABLE_OFF);
  int32_t* dWork = reinterpret_cast<int32_t*>(base + NOALLOC_WORK_OFF);
  DevCtl* dCtl = reinterpret_cast<DevCtl*>(base + NOALLOC_CTL_OFF);

  DevBlock hb[NOALLOC_MAX_BLOCKS];
  int32_t work[NOALLOC_MAX_BLOCKS];
  int nwork = 0;
  if ((rc = noalloc_table(*cfg, nslots, local_blocks, hb, work, &nwork))) {
    std::fprintf(stderr, "wx3d_hydro_step_noalloc: invalid mesh\n");
    return rc;
  }
  // An empty registry steps like wx3d_step on an empty mesh: no block is
  // updated, the local dt is 1e30*CFL (clamped to the next output time) and
  // time advances.
  int zsplit = 1;
  while (zsplit < 8 && nwork * zsplit < 2 * nsm) zsplit *= 2;

  PhysParams ph{};
  noalloc_phys(*cfg, ph);
  DevCtl h{};
  h.time = state->time;
  h.dt = state->dt;
  h.it = state->it;
  h.nextout = state->nextout;
  // The output bookkeeping of a crossed output time finishes inside the call
  // (step_end_kernel advances nextout), so no pending flag carries over:
  // state->dumpout on entry is ignored, on return it reports a crossing.
  h.dumpout = 0;
  const double big = 1.0e30;
  std::memcpy(&h.dtmin_bits, &big, 8);

  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  auto ck = [](cudaError_t e) { return e == cudaSuccess ? WX_OK : WX_ERR_CUDA; };
  if ((rc = ck(cudaFuncSetAttribute(k.stage1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem1)))) return rc;
  if ((rc = ck(cudaFuncSetAttribute(k.stage2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem2)))) return rc;
  if ((rc = ck(cudaMemcpyAsync(dBlocks, hb, sizeof(DevBlock) * nslots, cudaMemcpyHostToDevice, s)))) return rc;
  if ((rc = ck(cudaMemcpyAsync(dWork, work, 4 * (size_t)nwork, cudaMemcpyHostToDevice, s)))) return rc;
  if ((rc = ck(cudaMemcpyAsync(dCtl, &h, sizeof(DevCtl), cudaMemcpyHostToDevice, s)))) return rc;

  // getTimestep on u_in, then the step sequence of enqueue_solver
  DtParams D{u_in, dBlocks, dWork, nwork, dCtl, ph};
  k.dt<<<noalloc_grid((const void*)k.dt, 256, 0, nwork, nsm), 256, 0, s>>>(D);
  step_begin_kernel<<<1, 1, 0, s>>>(dCtl, ph.cfl, 0, ph.dtout, ph.t_sc, 1);
  const int solver = cfg->solver_type;
  int zero_ghost = 0;
  auto stage = [&](void (*fn)(StageParams), size_t smem, const double* src, double* out, double factor) {
    StageParams P{src, u_in, out, dBlocks, dWork, nwork * zsplit, zsplit, dCtl, factor, ph, 0, src};
    fn<<<noalloc_grid((const void*)fn, STAGE_THREADS, smem, nwork * zsplit, nsm), STAGE_THREADS, smem, s>>>(P);
  };
  if (solver == WX_SOLVER_LAX) {
    LaxParams L{u_in, u_out, dBlocks, dWork, nwork, dCtl, ph};
    k.lax<<<noalloc_grid((const void*)k.lax, 256, 0, nwork, nsm), 256, 0, s>>>(L);
    zero_ghost = 1;
  } else if (solver == WX_SOLVER_HLL1) {
    stage(k.stage1, k.smem1, u_in, u_out, 1.0);
    zero_ghost = 1;
  } else {
    stage(k.stage1, k.smem1, u_in, dUP, 0.5);
    stage(k.stage2, k.smem2, dUP, u_out, 1.0);
  }
  ViscParams V{u_out, dUP, dBlocks, dWork, nwork, zero_ghost, 1, dCtl, ph};
  k.visc<<<noalloc_grid((const void*)k.visc, 256, 0, nwork, nsm), 256, 0, s>>>(V);
  step_end_kernel<<<1, 1, 0, s>>>(dCtl, 1);
  if ((rc = ck(cudaGetLastError()))) return rc;
  if ((rc = ck(cudaMemcpyAsync(&h, dCtl, sizeof(DevCtl), cudaMemcpyDeviceToHost, s)))) return rc;
  if ((rc = ck(cudaStreamSynchronize(s)))) return rc;
  state->time = h.time;
  state->dt = h.dt;
  state->it = h.it;
  state->nextout = h.nextout;
  state->dumpout = h.dumps != 0;
  if (h.cnt[2]) return WX_ERR_DIVISION_BY_ZERO;
  if (h.cnt[3]) return WX_ERR_NAN;
  return WX_OK;
}
