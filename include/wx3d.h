/*
 * wx3d.h -- C-ABI of the B200 (sm_100a) per-block Godunov update for
 * Walicxe3D-style block-structured AMR hydro/MHD.
 *
 * The entry points replace the argument-less Fortran module subroutines of
 * the reference that act on module globals (U, UP, PRIM, dt, time, it):
 *
 *   hydroSolver()            source/hydro_solver.f90:39   -> wx3d_hydro_solver
 *   getTimestep(dt)          source/hydro_solver.f90:129  -> wx3d_get_timestep
 *   updatePrims()            source/hydro_core.f90:43     -> wx3d_update_prims
 *   updateNeutralFraction()  source/hrate.f90:12          -> wx3d_update_neutral_fraction
 *   cooling()                source/cooling.f90:37        -> wx3d_cooling
 *   loadcooldata()           source/cooling.f90:135       -> wx3d_set_cooltable
 *   boundary(depth, uvars)   source/boundary.f90:46       -> fused into the stage kernels
 *   markByPhysical(...)      source/amr.f90:142           -> wx3d_mark
 *   refineBlock(fatherID)    source/amr.f90:284 (data)    -> wx3d_refine
 *   coarseBlocks()           source/amr.f90:1430 (data)   -> wx3d_coarsen
 *   admesh()                 source/amr.f90:44            -> wx3d_admesh
 *   main-loop body           source/main.f90:81-100       -> wx3d_step / wx3d_run
 *
 * Memory: the library owns the device copies of every block's conserved
 * variables (and primitives on request).  The host keeps the block tree
 * (localBlocks, bIDs) and passes it with wx3d_set_mesh after every mesh
 * change, exactly like the reference's localBlocks registry
 * (source/globals.f90:125).
 *
 * Conventions: every call returns an int status (0 = OK).  Codes 1..27 and
 * 255 mirror the reference's error codes (source/constants.f90:135-162);
 * codes >= 100 are added by this library.  Calls are synchronous from the
 * host's point of view unless the name ends in _async, are not thread safe,
 * and use one CUDA stream per context (settable with wx3d_set_stream).
 * Signatures carry plain pointers and sizes only.
 */
#ifndef WX3D_H
#define WX3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Block geometry: ncells_block and nghost (source/parameters.f90:113,209). */
#define WX3D_NCELLS 16
#define WX3D_NGHOST 2
#define WX3D_BLOCK_CELLS (WX3D_NCELLS * WX3D_NCELLS * WX3D_NCELLS)
#define WX3D_MAX_LEVELS 10 /* basegrid limit, source/init.f90:694-700 */
#define WX3D_MAX_NEQ 12

/* Directions (source/constants.f90:52-57). */
enum { WX_LEFT = 1, WX_RIGHT = 2, WX_FRONT = 3, WX_BACK = 4, WX_BOTTOM = 5, WX_TOP = 6 };
/* Boundary conditions (source/constants.f90:65-67). */
enum { WX_BC_REFLECTIVE = 1, WX_BC_FREE_FLOW = 2, WX_BC_PERIODIC = 3 };
/* Neighbour types (source/constants.f90:70-73). */
enum { WX_NEIGH_SAME = 1, WX_NEIGH_COARSER = 2, WX_NEIGH_FINER = 3, WX_NEIGH_BOUNDARY = 4 };
/* Refinement flags (source/constants.f90:76-78). */
enum { WX_FLAG_NONE = 0, WX_FLAG_REFINE = 1, WX_FLAG_COARSE = 2 };
/* Solvers (source/constants.f90:81-86). */
enum {
  WX_SOLVER_LAX = 1, WX_SOLVER_HLL1 = 2, WX_SOLVER_HLL = 3,
  WX_SOLVER_HLLC = 4, WX_SOLVER_HLLE = 5, WX_SOLVER_HLLD = 6
};
/* Slope limiters (source/constants.f90:89-96). */
enum {
  WX_LIMITER_NO_AVERAGE = -1, WX_LIMITER_NONE = 0, WX_LIMITER_MINMOD = 1,
  WX_LIMITER_VANLEER = 2, WX_LIMITER_ALBADA = 3, WX_LIMITER_UMIST = 4,
  WX_LIMITER_WOODWARD = 5, WX_LIMITER_SUPERBEE = 6
};
/* Equations of state (source/constants.f90:99-102). */
enum { WX_EOS_ADIABATIC = 0, WX_EOS_SINGLE_SPECIE = 1, WX_EOS_TWOTEMP = 2, WX_EOS_H_RATE = 3 };
/* Cooling (source/constants.f90:106-110). */
enum { WX_COOL_NONE = 0, WX_COOL_TABLE = 1, WX_COOL_TABLE_METAL = 2, WX_COOL_H = 3, WX_COOL_SCHURE = 4 };

/* Status codes.  1..27 and 255 are the reference's (source/constants.f90:135-162). */
enum {
  WX_OK = 0,
  WX_ERR_GENERIC = 255,
  WX_ERR_ALREADY_MAX_LEV = 6,
  WX_ERR_INSUFICIENT_NBMAXPROC = 7,
  WX_ERR_REGISTER_FATHER = 10,
  WX_ERR_TOO_MANY_LEVS = 12,
  WX_ERR_COOLING_LOAD_COEFS = 14,
  WX_ERR_OUTPUT_FILE_OPEN = 18,
  WX_ERR_WARM_FILE_OPEN = 20,
  WX_ERR_WARM_READ_BLOCKS = 21,
  WX_ERR_DIVISION_BY_ZERO = 23,
  WX_ERR_NOT_ENOUGH_PASSIVES = 26,
  WX_ERR_NAN_IN_FLUXES = 27,
  WX_ERR_CUDA = 100,
  WX_ERR_TIMEOUT = 101,
  WX_ERR_NAN = 102,
  WX_ERR_INVALID_ARG = 103,
  WX_ERR_UNSUPPORTED = 104,
  WX_ERR_NO_DEVICE = 105,
  WX_ERR_MESH = 106
};

/*
 * Run-time mirror of the compile-time parameters the hot path reads
 * (source/parameters.f90 and the per-problem copies).  BFIELD, a Makefile
 * switch in the reference (Makefile:34-128), is the field `bfield`.
 */
typedef struct wx_config {
  int32_t neqtot;            /* neqtot = 5 + 3*bfield + npassive        */
  int32_t npassive;          /* npassive                                 */
  int32_t bfield;            /* -DBFIELD                                 */
  int32_t mhd;               /* mhd                                      */
  int32_t solver_type;       /* WX_SOLVER_*                              */
  int32_t limiter_type;      /* WX_LIMITER_*                             */
  int32_t eos_type;          /* WX_EOS_*                                 */
  int32_t cooling_type;      /* WX_COOL_*                                */
  int32_t bc[6];             /* bc_left, bc_right, bc_front, bc_back, bc_bottom, bc_top */
  int32_t eight_wave;        /* Powell 8-wave source (brio-wu/parameters.f90:198) */
  int32_t user_source_terms; /* must be 0: get_user_source_terms is not part of this ABI */
  int32_t enable_flux_cd;    /* field-CD update of B (brio-wu/parameters.f90:200, brio-wu/flux_cd.f90:52-86) */
  int32_t pad0;              /* keeps the doubles 8-byte aligned; set to 0 */
  int32_t nbrootx, nbrooty, nbrootz; /* root blocks (MESH_MANUAL)        */
  int32_t maxlev;            /* number of refinement levels              */
  double gamma;              /* heat capacity ratio                      */
  double cfl;                /* CFL                                      */
  double visc_eta;           /* artificial viscosity                     */
  double cooling_limit;      /* max fractional thermal loss per step     */
  double mu0, mui, ion_thres;
  double l_sc, d_sc, v_sc;   /* unit scalings; p_sc, e_sc, t_sc derived  */
  double xphystot, yphystot, zphystot; /* box size (cgs)                 */
  double tfin, dtout;        /* final time and output cadence (cgs)      */
  double refine_thres, coarse_thres; /* markByPhysical thresholds        */
} wx_config;

/* Simulation state globals (source/globals.f90:52-56). */
typedef struct wx_state {
  double time;      /* code units */
  double dt;        /* code units */
  int32_t it;
  int32_t nextout;
  int32_t dumpout;  /* set when getTimestep clipped dt to an output time */
  int32_t pad;
} wx_state;

/* Device-side health counters, read after a step (never a trap). */
typedef struct wx_status {
  int64_t pressure_floor;  /* flow2prim istat=1 (source/hydro_core.f90:355-358) */
  int64_t density_floor;   /* flow2prim istat=2 (source/hydro_core.f90:361-364) */
  int64_t zero_density;    /* flow2prim abort case (source/hydro_core.f90:335-338) */
  int64_t nan_cells;       /* non-finite state after a step                     */
  double max_cool_loss;    /* max fractional thermal loss before limiting       */
  int64_t kernels_launched;/* running count of kernels this context launched    */
  int64_t surrogate_cells; /* cells whose hrate + cooling_h step came from the MLP */
  int64_t fallback_cells;  /* cells of surrogate steps that used the plain integrator */
} wx_status;

typedef struct wx_ctx wx_ctx;
typedef struct wx_mlp wx_mlp;

/* Fills *cfg with the defaults of source/parameters.f90 (HD, HLLC, van Leer,
 * free-flow, CFL 0.4, eta 5e-3) in code units (all scalings 1). */
int wx3d_config_defaults(wx_config* cfg);

/* Allocates HBM for max_blocks block slots.  Replaces the big-array
 * allocation of initmain (source/init.f90:375-423). */
int wx3d_init(const wx_config* cfg, int32_t max_blocks, wx_ctx** out);
int wx3d_finalize(wx_ctx* ctx);

/* Use an external cudaStream_t (NULL selects the context's own stream). */
int wx3d_set_stream(wx_ctx* ctx, void* cuda_stream);

/* localBlocks registry: bID of the block held in each slot, -1 if empty
 * (source/globals.f90:125, source/init.f90:431-437).  Rebuilds the device
 * neighbour table with the reference's tree queries (source/amr.f90:439-631).
 * Every slot may be -1 (a process that holds no block): the steps then run
 * no block and the local dt is 1e30*CFL, as getTimestep gives such a
 * process (source/hydro_solver.f90:145-192); wx3d_autotune needs a block. */
int wx3d_set_mesh(wx_ctx* ctx, int32_t nslots, const int32_t* local_blocks);

/* A process's share of a partitioned mesh: as wx3d_set_mesh, with nhalo of
 * the slots (halo_slots) holding copies of blocks other processes own --
 * read as neighbours by the stages, never updated, their own faces allowed
 * to lead out of the local set.  The host refreshes them with
 * wx3d_pack_blocks/wx3d_unpack_blocks before each stage (the MPI halo
 * exchange of boundary.f90:174-291 and :357-555).  Wind sources are not
 * supported in this mode. */
int wx3d_set_mesh_halo(wx_ctx* ctx, int32_t nslots, const int32_t* local_blocks, int32_t nhalo,
                       const int32_t* halo_slots);

/* Device neighbour table as built by wx3d_set_mesh, for inspection:
 * per slot and face (6): type, 4 neighbour slots.  face_type[nslots*6],
 * face_slot[nslots*24]; empty slots report type 0. */
int wx3d_get_neighbours(wx_ctx* ctx, int32_t nslots, int32_t* face_type, int32_t* face_slot);

/* Slabs per block of the stage kernels (1, 2, 4 or 8 CTAs per block along z).
 * wx3d_set_mesh picks a default; the autotuner overrides it. */
int wx3d_set_zsplit(wx_ctx* ctx, int32_t zsplit);

/* A spherical wind source (spherical_wind_type, winds.f90), physical cgs
 * units: centre, bulk velocity of the source, radius, mass-loss rate,
 * terminal speed, temperature, mean molecular mass.  y0 is the neutral
 * fraction of the wind's passive scalar (EOS_H_RATE runs), a value the
 * reference leaves undefined. */
typedef struct wx_wind {
  double xc, yc, zc, vx, vy, vz, radius, mdot, vinf, temp, mu, y0;
} wx_wind;

/* userBoundary hook of the wind problems (imposeSphericalWind,
 * winds.f90:123-240): after every ghost exchange the reference re-imposes
 * the r^-2 wind in all cells, ghosts included, within a source's radius.
 * The library applies it where the stages read those cells.  nwind = 0
 * removes the sources.  The zone refinement the reference does at it = 0
 * (refineZone) is the host's, like the rest of the mesh.  A sphere that
 * reaches the ghost layer of a coarse/fine face or of the domain boundary
 * is refused (WX_ERR_UNSUPPORTED, the previous sources stay), here and in
 * wx3d_set_mesh / wx3d_admesh. */
int wx3d_set_winds(wx_ctx* ctx, int32_t nwind, const wx_wind* winds);

/* With fusion on (the default) and whole blocks per CTA (zsplit 1), the
 * corrector stage also applies doViscousStep; otherwise a separate viscous
 * kernel runs after it.  The autotuner overrides the choice. */
int wx3d_set_fusion(wx_ctx* ctx, int32_t fuse_viscous);

/* Autotuner of the stage launch shape for the current mesh: times the
 * predictor, the corrector and the viscous step (reps passes each) -- on
 * the live state, without changing it -- for five shapes: whole blocks with
 * the viscous step fused into the corrector, whole blocks with a separate
 * viscous kernel, and 2, 4, 8 z-slabs per block; keeps the fastest.  The
 * state, the next time step and the status counters are left as they were,
 * so a run may be tuned between any two steps.
 * ms5 (may be NULL) receives the time per pass of each shape in that
 * order, best (may be NULL) two values: the chosen split and the fusion
 * flag. */
int wx3d_autotune(wx_ctx* ctx, int32_t reps, double* ms5, int32_t* best);

/* Checkpoints in the reference's formats, written from and read into HBM.
 * wx3d_write_bin: writeBin (source/output.f90:156-213), a stream file of
 * int32 nbLocal then, per occupied slot in slot order, int32 bID and
 * U(nb,:,1:16,1:16,1:16) in FP64 with the equation index fastest.
 * wx3d_read_bin: warmstart's block read (source/init.f90:589-612): blocks go
 * to slots 0..nbLocal-1 in file order, the neighbour table is rebuilt, and
 * local_blocks[max_slots] receives the registry (-1 beyond nbLocal).
 * wx3d_write_state / wx3d_read_state: writeState (output.f90:219-263) and
 * warmstart's state read (init.f90:549-573), '(es22.15,i8,i5)' with
 * time*t_sc, it, noutput, then the data directory; reading sets time, it
 * and nextout = noutput + 1. */
int wx3d_write_bin(wx_ctx* ctx, const char* path);
int wx3d_read_bin(wx_ctx* ctx, const char* path, int32_t max_slots, int32_t* local_blocks, int32_t* nblocks);
int wx3d_write_state(wx_ctx* ctx, const char* path, int32_t noutput, const char* datadir);
int wx3d_read_state(wx_ctx* ctx, const char* path, int32_t* noutput, char* datadir, int32_t nbytes);

/* Conserved variables, native layout: u[slot][eq][k][j][i], 16^3 physical
 * cells per block, host memory (pinned or pageable). */
int wx3d_upload_blocks(wx_ctx* ctx, int32_t nslots, const double* u);
int wx3d_download_blocks(wx_ctx* ctx, int32_t nslots, double* u);

/* Conserved variables in the reference's own array layout
 * U(nbMaxProc, neqtot, -1:18, -1:18, -1:18), block index fastest
 * (source/globals.f90:97).  Only physical cells are read / written. */
int wx3d_upload_U_fortran(wx_ctx* ctx, int32_t nbMaxProc, const double* U);
int wx3d_download_U_fortran(wx_ctx* ctx, int32_t nbMaxProc, double* U);

/* updatePrims (source/hydro_core.f90:43) on physical cells, then download
 * PRIM in the native layout. */
int wx3d_update_prims(wx_ctx* ctx);
int wx3d_download_prims(wx_ctx* ctx, int32_t nslots, double* prim);

int wx3d_set_state(wx_ctx* ctx, const wx_state* st);
int wx3d_get_state(wx_ctx* ctx, wx_state* st);

/* getTimestep (source/hydro_solver.f90:129) on the current primitives,
 * using st.it as already incremented by the caller (source/main.f90:81).
 * Does not change the stored dt. */
int wx3d_get_timestep(wx_ctx* ctx, double* dt_glob);

/* hydroSolver (source/hydro_solver.f90:39): dt, Godunov(order) or
 * LaxFriedrichs, doViscousStep.  Updates state.dt and state.time. */
int wx3d_hydro_solver(wx_ctx* ctx);

/* updateNeutralFraction (source/hrate.f90:12) and cooling
 * (source/cooling.f90:37).  maxloss may be NULL. */
int wx3d_update_neutral_fraction(wx_ctx* ctx);
int wx3d_cooling(wx_ctx* ctx, double* maxloss);

/* updatePrims + updateNeutralFraction + cooling (source/main.f90:94-100)
 * fused in one pass over U with the current dt, the source part of
 * wx3d_step; uses the surrogate when one is attached.  Also folds the CFL
 * minimum for the next step.  maxloss as for wx3d_cooling.  No reference
 * counterpart as one call. */
int wx3d_sources(wx_ctx* ctx, double* maxloss);

/* One main-loop iteration without AMR and output (source/main.f90:81-100):
 * it += 1, hydroSolver, updatePrims, updateNeutralFraction (EOS_H_RATE),
 * cooling.  *out (may be NULL) receives the state after the step. */
int wx3d_step(wx_ctx* ctx, wx_state* out);

/* nsteps iterations of wx3d_step with no host synchronisation in between
 * (the step sequence is captured once in a CUDA graph and replayed). */
int wx3d_run(wx_ctx* ctx, int32_t nsteps, wx_state* out);
/* Same, enqueued on the context stream without a final synchronisation. */
int wx3d_run_async(wx_ctx* ctx, int32_t nsteps);

/* loadcooldata (source/cooling.f90:135-184): npts rows (logT, b) with the
 * cooling rate stored as -b (cooltable(2,i) = -b). */
int wx3d_set_cooltable(wx_ctx* ctx, int32_t npts, const double* logT, const double* b);

/* loadcooldata_metal (source/cooling.f90:193-265), COOL_TABLE_METAL: the
 * (nptsT+1) x (nptsZ+1) table row by row as the file lists it -- first row
 * an unused entry then the metallicities, each further row log10 T then
 * log10 Lambda per metallicity.  The metallicity scalar is passive
 * metalpas = 5 + 3*bfield + min(npassive, 1) (parameters.f90:318). */
int wx3d_set_cooltable_metal(wx_ctx* ctx, int32_t nptsT, int32_t nptsZ, const double* table);

/* loadcooldata_schure (source/cooling_schure.f90:52-95), COOL_SCHURE: the
 * 180 rows of five columns of the Schure et al. table file (log10 T, then
 * -log10 Lambda for four ionisation fractions); dmc_f (1..4) picks the
 * column. */
int wx3d_set_cooltable_schure(wx_ctx* ctx, const double* data, int32_t dmc_f);

/* markByPhysical (source/amr.f90:142-230) for every occupied slot:
 * flags[slot] = WX_FLAG_*; empty slots get -1. */
int wx3d_mark(wx_ctx* ctx, int32_t nslots, int32_t* flags);

/* Data part of refineBlock (source/amr.f90:355-367): injection of the
 * father's octants into 8 child slots (children in x,y,z natural order). */
int wx3d_refine(wx_ctx* ctx, int32_t father_slot, const int32_t* child_slots8);

/* Data part of coarseBlocks (source/amr.f90:1597-1625): 8-cell averages of
 * the 8 siblings (natural order) into the father slot. */
int wx3d_coarsen(wx_ctx* ctx, const int32_t* child_slots8, int32_t father_slot);

/* admesh (source/amr.f90:44-133) of one process, in place of the whole
 * subroutine: markByPhysical on the device, checkProximity(maxlev-1)
 * (amr.f90:1109-1254) on the flags, refineBlock (:284-384) for every block
 * still marked REFINE in slot order, then coarseBlocks (:1430-1650) for
 * every family whose eight siblings are marked COARSE.  Slots follow the
 * reference's registry: a new block takes the first empty slot (put,
 * utils.f90:112) and a removed block frees its own (pop, :157); with one
 * process loadBalance moves no block, so the slot order is the reference's.
 * local_blocks (nbmax = the context's max_blocks entries, -1 = empty) must
 * hold the list last passed to wx3d_set_mesh, padded with -1; on return it
 * holds the new list.  When a block changed, the device neighbour table is
 * rebuilt from it (the context's z-slab split is kept); otherwise nothing
 * but the marking runs.
 * counts2 (may be NULL): blocks refined, families coarsened.  Capacity
 * errors (WX_ERR_INSUFICIENT_NBMAXPROC, WX_ERR_REGISTER_FATHER) and a new
 * mesh that wx3d_set_mesh would refuse (WX_ERR_MESH, or WX_ERR_UNSUPPORTED
 * for a wind sphere on a coarse/fine face) are found before any data moves
 * and leave the mesh and the state unchanged. */
int wx3d_admesh(wx_ctx* ctx, int32_t nbmax, int32_t* local_blocks, int32_t* counts2);

/* Per-kernel device timing with CUDA events recorded around each launch of
 * the step sequence (inside the CUDA graph of wx3d_run).  wx3d_kernel_times
 * returns, for the last step(s) executed, the summed milliseconds and the
 * launch counts of: [0] predictor stage, [1] corrector (or single) stage,
 * [2] viscous step + CFL reduction, [3] source terms. */
int wx3d_set_timing(wx_ctx* ctx, int32_t on);
int wx3d_kernel_times(wx_ctx* ctx, double* ms4, int32_t* count4);

int wx3d_get_status(wx_ctx* ctx, wx_status* st);
int wx3d_reset_status(wx_ctx* ctx);

/* Allocation-free hydro step.  No counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc -- hosts whose device memory
 * belongs to their own pool or framework allocator, or that must not grow
 * their footprint after start-up.  The caller passes the state in its own
 * device memory: u_in and u_out are [slot][eq][k][j][i] arrays of nslots
 * blocks whose byte ranges must not overlap (an overlap returns
 * WX_ERR_INVALID_ARG), local_blocks is the host-side bID registry, and
 * *state (host) carries time, dt, it and nextout in and out like
 * wx3d_step's: on return dumpout reports whether this step crossed an
 * output time (nextout has then been advanced); its value on entry is
 * ignored.  One main-loop step without source terms is run (it += 1,
 * getTimestep, Godunov / Lax-Friedrichs, viscous step) on cuda_stream
 * (NULL = default stream) and the call returns after the stream is
 * synchronised.  A registry with no block (all -1) steps like wx3d_step on
 * an empty mesh: dt = 1e30*CFL clamped to the next output time.
 * Scratch (predictor state, neighbour table, control block) lives in one
 * fixed device array of the library: nslots x neqtot must not exceed
 * WX3D_NOALLOC_MAX_BLOCK_EQS (10 MiB of predictor state), otherwise the call
 * returns WX_ERR_INSUFICIENT_NBMAXPROC.  The array's device address is
 * looked up (cudaGetSymbolAddress) on the first call on each device and
 * again whenever the current CUDA context changes, so the first call, and
 * the first after a context change, should come before any stream capture.
 * All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  Source terms (EOS_H_RATE, cooling) return
 * WX_ERR_UNSUPPORTED. */
#define WX3D_NOALLOC_MAX_BLOCK_EQS 320
int wx3d_hydro_step_noalloc(const wx_config* cfg, int32_t nslots, const int32_t* local_blocks,
                            const double* u_in, double* u_out, wx_state* state, void* cuda_stream);

/*
 * Learned surrogate of the hydrogen-rate + cooling_h update (one step of
 * updateNeutralFraction, hrate.f90:82-142, then apply_cooling_h_neq,
 * cooling_h.f90:154-252): a 4-64-64-2 SiLU MLP with BF16 operands and FP32
 * accumulation, trained and run by tcgen05 tensor-core kernels (forward
 * hidden layers as BF16 head + tail products, FP32 output layer).  Inputs
 * are (log10 n_H dt/yr, log10 T, x_HII, log10 dt/yr) normalised to [-1,1]
 * over the box n_H in [1e-3,1e4] cm^-3, T in [1e2,1e8] K, dt in
 * [1e-2,1e3] yr; outputs are (delta x_HII / 0.125, log10(P1/P0) / log10 2).
 * Device pointers are caller-owned; calls are synchronous.
 */
int wx3d_mlp_create(uint64_t seed, wx_mlp** out);
int wx3d_mlp_destroy(wx_mlp* mlp);
int wx3d_mlp_nparams(void);
/* parameters, FP32: W1[4][64], b1[64], W2[64][64], b2[64], W3[64][2], b3[2] */
int wx3d_mlp_get_params(wx_mlp* mlp, float* host_params);
int wx3d_mlp_set_params(wx_mlp* mlp, const float* host_params);
/* n samples drawn log-uniformly in the box (x_HII uniform), targets from the
 * plain FP64 integrator with the rates and scalings of *cfg.  d_in [n][4],
 * d_target [n][2], d_raw [n][4] = (n_H, T, x_HII, dt in s) or NULL. */
int wx3d_mlp_samples(const wx_config* cfg, int64_t n, uint64_t seed, float* d_in, float* d_target, double* d_raw,
                     void* cuda_stream);
int wx3d_mlp_forward(wx_mlp* mlp, int64_t n, const float* d_in, float* d_out, void* cuda_stream);
/* loss = mean over samples of the summed squared error; gradient in host_grad */
int wx3d_mlp_gradient(wx_mlp* mlp, int64_t n, const float* d_in, const float* d_target, float* loss,
                      float* host_grad);
int wx3d_mlp_train(wx_mlp* mlp, int64_t n, const float* d_in, const float* d_target, int32_t epochs, int32_t batch,
                   float lr, float* loss_per_epoch);

/* Attaches (enable = 1) the surrogate to a context whose config is
 * EOS_H_RATE (hydro, 1-2 passive scalars): the source step of wx3d_step /
 * wx3d_run then uses the MLP for the cells in the trust box whose bin of
 * `trust` is non-zero, and the plain integrator elsewhere.  With COOL_H
 * both outputs are used (x_HII and the cooling factor; cooling_limit must
 * be 0.5, as in training); with the table coolings (COOL_TABLE,
 * COOL_TABLE_METAL, COOL_SCHURE) only the x_HII output replaces the hrate
 * update and the plain table cooling follows.  trust[48][48][8]
 * (nbytes = 18432) bins log10(n_H dt/yr) in [-5,7) by 0.25, log10 T in
 * [2,8) by 0.125 and x_HII in eighths.  enable = 0 detaches it. */
int wx3d_set_surrogate(wx_ctx* ctx, wx_mlp* mlp, const uint8_t* trust, int32_t nbytes, int32_t enable);

/* Self-check of the Newton-refined reciprocal and square root that the flux
 * kernels use in place of IEEE division and sqrt: max_ulp2[0] and [1]
 * receive their largest distance in ulp from the device's 1/x and sqrt(x)
 * over the n positive normal arguments host_x. */
int wx3d_check_fast_math(int32_t n, const double* host_x, int64_t* max_ulp2);

/* Self-check of the bounded waits of the tensor-core kernels (no
 * counterpart in the reference): one CTA waits, giving up after `limit`
 * tries (1 .. 2^22), on an mbarrier that nothing arrives at, and records the
 * timeout as the MLP kernels do.  Returns WX_ERR_TIMEOUT, the expected
 * outcome; the device stays usable. */
int wx3d_check_wait_timeout(int32_t limit);

/* Measured FP64 FMA throughput of the current device in GFLOP/s (an FMA
 * counts two flops): the compute roofline of the stage kernels. */
int wx3d_measure_fp64_peak(double* gflops);

/* The main-loop iteration in parts, for partitioned runs that exchange
 * halo blocks between the stages:
 *   part 0: getTimestep's tail (dt from the CFL minimum, it += 1);
 *   part 1: the first stage (predictor, or the single stage) -- exchange U
 *           halos before it;
 *   part 2: the corrector, doViscousStep, time += dt -- exchange UP halos
 *           before it;
 *   part 3: updatePrims + hrate + cooling, and the CFL minimum of the new
 *           state.
 * wx3d_get_dtmin returns this process's CFL minimum (dx/(|v|+c) over its
 * blocks, computed if needed); wx3d_set_dtmin replaces it with the global
 * minimum (MPI_ALLREDUCE, hydro_solver.f90:198) before part 0. */
int wx3d_step_part(wx_ctx* ctx, int32_t part);
int wx3d_get_dtmin(wx_ctx* ctx, double* dtmin);
int wx3d_set_dtmin(wx_ctx* ctx, double dtmin);

/* Copies n whole blocks (slots, host array) of the current state (array 0)
 * or of the predictor state UP (array 1) to a device buffer of
 * n*neqtot*4096 doubles, block after block in native layout, or back. */
int wx3d_pack_blocks(wx_ctx* ctx, int32_t array, int32_t n, const int32_t* slots, double* d_buf);
int wx3d_unpack_blocks(wx_ctx* ctx, int32_t array, int32_t n, const int32_t* slots, const double* d_buf);

/* As wx3d_pack_blocks/wx3d_unpack_blocks for the four cell layers of each
 * block next to one of its faces (faces[i]: 0..5 = left, right, front,
 * back, bottom, top): n*neqtot*1024 doubles, item after item.  Whatever a
 * neighbouring process reads of a halo block lies within those layers
 * across the faces it shares with the halo block: two layers for a
 * same-level ghost fill, one coarse layer for injection, four fine layers
 * for the averages of a coarser block's ghosts (boundary.f90:329-540).  The
 * same halo refresh as whole blocks, at a quarter of the bytes per face. */
int wx3d_pack_faces(wx_ctx* ctx, int32_t array, int32_t n, const int32_t* slots, const int32_t* faces, double* d_buf);
int wx3d_unpack_faces(wx_ctx* ctx, int32_t array, int32_t n, const int32_t* slots, const int32_t* faces,
                      const double* d_buf);

/* Human-readable text of a status code and of the context's last error. */
const char* wx3d_error_string(int32_t code);
int wx3d_last_error(wx_ctx* ctx, char* buf, int32_t len);

#ifdef __cplusplus
}
#endif

#endif /* WX3D_H */
