/* pmp_spray.h -- C ABI of the B200 Lagrangian spray particle update.
 *
 * Drop-in for PeleMP's SprayParticleContainer::updateParticles /
 * calculateSpraySource path (Source/PP_Spray/SprayParticles.cpp:142-502,
 * Source/PP_Spray/Drag.H:138-441).  Plain C types only: a host program (the
 * C++ container shim in pelemp_b200/csrc/host, a ctypes binding, an AMReX
 * build) calls these functions; the library owns the device copy of the
 * droplets and launches the sm_100a kernels.
 *
 * Conventions
 *  - 3D, AMReX index space; mesh arrays use the AMReX Array4 layout:
 *    element (i,j,k,n) of a view sits at
 *      p[(i-lo0) + (j-lo1)*jstride + (k-lo2)*kstride + n*nstride].
 *  - Units follow the PeleLMeX coupling of the reference (MKS at the mesh
 *    and droplet interface; PELELM_USE_SPRAY in Source/PP_Spray/SprayFuelData.H:44-54).
 *  - Every function returns PMP_OK (0) or a PMP_ERR_* code; the library never
 *    aborts the process (the reference calls amrex::Abort at
 *    SprayParticles.cpp:350,422 and SprayInterpolation.H:122).
 *  - One handle must not be used from two host threads at once; separate
 *    handles are independent.  Kernels run on the stream passed in (NULL =
 *    the legacy default stream).
 *  - The update entry points (pmp_spray_update, _update_host, _move_kick,
 *    _move_kick_drift) are stream-ordered: they check their arguments,
 *    enqueue the device work on the stream and return without waiting for
 *    it (the reference instead synchronises after every box,
 *    SprayParticles.cpp:499).  Their return value reports argument and
 *    host-side errors, and a device error of an earlier call that the host
 *    can already see.  Device errors (the reference's amrex::Abort sites)
 *    are reported by pmp_spray_sync; after one, later calls leave the
 *    droplets untouched until pmp_spray_sync has reported it.  A handle's
 *    calls go on one stream, or the caller orders its streams.  The other
 *    entry points (droplet hand-over and read-back, the operations around
 *    the update, learning, tuning) first wait for the handle's enqueued
 *    updates.  Update calls may be captured into a CUDA graph by the caller
 *    once the same call has run outside the capture (so that its buffers
 *    exist); a captured call's box table stays in the handle (up to 8
 *    distinct tables captured per handle).
 */
#ifndef PMP_SPRAY_H
#define PMP_SPRAY_H

#ifdef __cplusplus
extern "C" {
#endif

#define PMP_MAX_FUEL 4
#ifndef PMP_MAX_SPEC
#define PMP_MAX_SPEC 8
#endif
#define PMP_NAME_LEN 32

/* Particle real components of one droplet, SprayComps at
 * Source/PP_Spray/SprayFuelData.H:10-19, for F fuels. */
#define PMP_PSTATE_VEL 0
#define PMP_PSTATE_T 3
#define PMP_PSTATE_DIA 4
#define PMP_PSTATE_Y 5
#define PMP_PSTATE_NUMDENS(F) (5 + (F))
#define PMP_PSTATE_N0(F) (6 + (F))
#define PMP_PSTATE_BM1(F) (7 + (F))
#define PMP_PSTATE_BM2(F) (8 + (F))
#define PMP_PSTATE_FILMHGHT(F) (9 + (F))
#define PMP_PSTATE_NUM(F) (10 + (F))
#define PMP_MAX_RCOMP PMP_PSTATE_NUM(PMP_MAX_FUEL)

enum pmp_status {
  PMP_OK = 0,
  PMP_ERR_LEFT_DOMAIN = 1,  /* droplet outside a non-periodic, non-reflective domain at entry */
  PMP_ERR_STATE_BOX = 2,    /* interpolation stencil outside the grown state box */
  PMP_ERR_SOURCE_BOX = 3,   /* deposit cell outside the grown source box */
  PMP_ERR_UNSUPPORTED = 4,  /* breakup, splash, wall film or EB requested */
  PMP_ERR_TIMEOUT = 5,      /* a bounded device wait gave up */
  PMP_ERR_CUDA = 6,         /* a CUDA runtime call failed */
  PMP_ERR_INVALID = 7,      /* bad argument */
  PMP_ERR_NO_DEVICE = 8     /* no usable sm_100 device */
};

/* Precision / method forms of the update (pmp_spray_set_mode). */
enum pmp_mode {
  PMP_MODE_FP64 = 0,    /* plain method, FP64 throughout */
  PMP_MODE_MIXED = 1,   /* FP32 bulk physics, FP64 near d->0 and for deposits */
  PMP_MODE_LEARNED = 2  /* MLP surrogate for the evaporation sub-step + gate */
};

/* Boundary designation per face, as updateParticles computes it
 * (SprayParticles.cpp:200-218): 0 periodic, 1 reflective, -1 outflow. */
typedef struct pmp_geometry {
  double plo[3];
  double phi[3];
  double dx[3];
  int domain_lo[3];
  int domain_hi[3];
  int bndry_lo[3];
  int bndry_hi[3];
} pmp_geometry;

/* Index box, inclusive bounds (amrex::Box, cell-centred). */
typedef struct pmp_box {
  int lo[3];
  int hi[3];
} pmp_box;

/* View of one box of a multi-component mesh array (amrex::Array4). lo/hi are
 * the bounds of the allocated (grown) box. */
typedef struct pmp_box_view {
  double* p;
  int lo[3];
  int hi[3];
  long long jstride;
  long long kstride;
  long long nstride;
  int ncomp;
} pmp_box_view;

/* Mirror of SprayComps' mesh component indices (SprayFuelData.H:20-28),
 * assigned by the caller (SprayParticles.H:386). */
typedef struct pmp_spray_comps {
  int rhoIndx;
  int momIndx;
  int engIndx;
  int utempIndx;
  int specIndx;
  int rhoSrcIndx;
  int momSrcIndx;
  int engSrcIndx;
  int specSrcIndx;
} pmp_spray_comps;

/* Mirror of SprayData (SprayFuelData.H:115-143), F = nfuel entries used. */
typedef struct pmp_spray_data {
  int nfuel;
  int mass_trans;
  int mom_trans;
  int fixed_parts;
  int do_splash;
  int do_breakup;
  double min_eb_vfrac;
  double ref_T;
  double sigma;
  double wall_T;
  double theta_c;
  double dtmod;
  double body_force[3];
  double critT[PMP_MAX_FUEL];
  double boilT[PMP_MAX_FUEL];
  double cp[PMP_MAX_FUEL];
  double latent[PMP_MAX_FUEL];
  double ref_latent[PMP_MAX_FUEL];
  double psat_coef[4 * PMP_MAX_FUEL];
  double rho_coef[4 * PMP_MAX_FUEL];
  double lambda_coef[4 * PMP_MAX_FUEL];
  double mu_coef[4 * PMP_MAX_FUEL];
  int indx[PMP_MAX_FUEL];
  int dep_indx[PMP_MAX_FUEL];
} pmp_spray_data;

/* The "particles.*" inputs readSprayParams parses
 * (Source/PP_Spray/SpraySetup.cpp:73-253).  A coefficient array with
 * ncoef_X[f] == 1 is a constant, == 4 a fit (getInpCoef, SpraySetup.cpp:22-58),
 * == 0 absent. */
typedef struct pmp_spray_inputs {
  int nfuel;
  char fuel_species[PMP_MAX_FUEL][PMP_NAME_LEN];
  char dep_fuel_species[PMP_MAX_FUEL][PMP_NAME_LEN]; /* "" = same as fuel */
  int mass_transfer;
  int mom_transfer;
  int fixed_parts;
  int use_splash_model;
  int use_breakup_model; /* 0 None, 1 TAB, 2 KHRT */
  double cfl;            /* particles.cfl, <= 2 */
  double fuel_ref_temp;
  double crit_temp[PMP_MAX_FUEL];
  double boil_temp[PMP_MAX_FUEL];
  double cp[PMP_MAX_FUEL];
  double latent[PMP_MAX_FUEL];
  int ncoef_lambda[PMP_MAX_FUEL];
  int ncoef_psat[PMP_MAX_FUEL];
  int ncoef_rho[PMP_MAX_FUEL];
  int ncoef_mu[PMP_MAX_FUEL];
  double lambda[PMP_MAX_FUEL][4];
  double psat[PMP_MAX_FUEL][4];
  double rho[PMP_MAX_FUEL][4];
  double mu[PMP_MAX_FUEL][4];
  double body_force[3];
} pmp_spray_inputs;

/* Droplets of one box.  layout PMP_LAYOUT_AOS: aos points to n records of
 *   { double pos[3]; double rdata[10+F]; int id; int cpu; }
 * (amrex::Particle<NSR_SPR,0> with separate id/cpu words).
 * layout PMP_LAYOUT_SOA: pos[d] and rdata[c] point to n doubles each, id to
 * n ints.  id > 0 marks a live droplet (the reference kills with id = -1). */
enum { PMP_LAYOUT_AOS = 0, PMP_LAYOUT_SOA = 1 };
enum { PMP_WHERE_HOST = 0, PMP_WHERE_DEVICE = 1 };
typedef struct pmp_particles {
  int layout;
  int where;
  long long n;
  void* aos;
  double* pos[3];
  double* rdata[PMP_MAX_RCOMP];
  int* id;
} pmp_particles;

typedef struct pmp_spray_config {
  int nfuel;                          /* SPRAY_FUEL_NUM */
  int nspec;                          /* NUM_SPECIES */
  char species[PMP_MAX_SPEC][PMP_NAME_LEN]; /* gas species, mechanism order */
  int device;                         /* CUDA device ordinal */
} pmp_spray_config;

typedef struct pmp_error_info {
  int code;
  int box;
  long long particle;   /* index within the box, caller order; -1 if none */
  double pos[3];
  char message[160];
} pmp_error_info;

/* Counters of the update calls between the last two pmp_spray_sync calls
 * (summed over those calls), as of the last pmp_spray_sync. */
typedef struct pmp_stats {
  long long substeps;        /* droplet-substeps executed (live droplets x sub-cycles) */
  long long killed;          /* droplets that evaporated or left the domain */
  long long inner_steps;     /* sum over droplet-substeps of the inner nsub */
  long long fallback;        /* mixed / learned forms: droplets handed to the
                                plain FP64 kernel (small, out of range) */
  double kernel_ms;          /* device time of the last call's update kernels
                                (host views: from the first copy in to the
                                last copy out) */
  int graph;                 /* last call: 1 replayed the batched form's
                                CUDA graph, 2 captured a new one, 0 direct launches */
} pmp_stats;

typedef struct pmp_spray pmp_spray;

/* Create a handle on cfg->device.  Replaces the static state of
 * SprayParticleContainer (SprayParticles.H:388-405). */
int pmp_spray_create(const pmp_spray_config* cfg, pmp_spray** out);
int pmp_spray_destroy(pmp_spray* h);

/* readSprayParams + spraySetup (SpraySetup.cpp:73-297): builds SprayData,
 * maps fuel names to species indices, subtracts h_fuel(ref_T) from the
 * latent heat (SpraySetup.cpp:284-290) and uploads it.  Rejects breakup and
 * splash models with PMP_ERR_UNSUPPORTED. */
int pmp_spray_setup(pmp_spray* h, const pmp_spray_inputs* in);
/* Install an already built SprayData (the H2D copy at SpraySetup.cpp:294). */
int pmp_spray_set_data(pmp_spray* h, const pmp_spray_data* data);
int pmp_spray_get_data(const pmp_spray* h, pmp_spray_data* data);

/* AssignSprayComps (SprayParticles.H:386). */
int pmp_spray_set_comps(pmp_spray* h, const pmp_spray_comps* comps);
/* Level geometry and boundary designation (SprayParticles.cpp:183-218). */
int pmp_spray_set_geometry(pmp_spray* h, const pmp_geometry* geom);
/* Valid boxes of the level's BoxArray, in ParIter order. */
int pmp_spray_set_grids(pmp_spray* h, int nboxes, const pmp_box* boxes);

/* Hand the droplets of box `box` to the library (copied; the library keeps
 * them on the device, sorted by cell, and remembers the caller's order). */
int pmp_spray_set_particles(pmp_spray* h, int box, const pmp_particles* p);
/* Copy the droplets of box `box` back in the caller's order; out->n must be
 * the count given to set_particles and out's arrays sized for it. */
int pmp_spray_get_particles(pmp_spray* h, int box, pmp_particles* out);
int pmp_spray_num_particles(const pmp_spray* h, int box, long long* n);

/* SprayParticleContainer::updateParticles (SprayParticles.cpp:142-502) for
 * all boxes in one call, stream-ordered (see the conventions above).
 * state[b] / source[b] are DEVICE views of box b's state and source fabs;
 * deposits are added to source (callers zero it, as transferSource does at
 * SprayParticles.H:294).  ltransparm is not needed: the transport model is
 * built into the handle. */
int pmp_spray_update(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source,
  int nboxes, double flow_dt, double time, int state_ghosts,
  int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, void* stream);

/* Same call with HOST views: the state is copied to the device, the source
 * deposits are added into the host source arrays after the update.  The
 * copies overlap the update: the boxes go in up to 8 groups, each group's
 * update starting once its views are on the device and its sources copied
 * back while later groups run (page-locked host memory lets all three
 * proceed at once).  The FP64 form with a non-default launch shape or CUDA
 * graph, and the learned form with its audit on, copy, update and copy back
 * in sequence.  Stream-ordered like pmp_spray_update: with page-locked host
 * views the call returns before the copies run, so the caller synchronises
 * the stream (or calls pmp_spray_sync) before it reads the host source or
 * writes the host state. */
int pmp_spray_update_host(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source,
  int nboxes, double flow_dt, double time, int state_ghosts,
  int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, void* stream);

/* What pmp_spray_update_host does with the host source arrays on entry.
 * copy_in = 1 (default): they are copied to the device and the deposits are
 * added to them.  copy_in = 0: they are taken to be zero, as the temporary
 * source is in the reference's workflow (transferSource,
 * SprayParticles.H:250-292, folds it into the flow's source and ends with
 * tmpSource.setVal(0)); the device mirror is cleared instead of copied in
 * and the call writes the deposits over the host arrays' source
 * components, which saves one host-to-device copy of the source per call. */
int pmp_spray_set_host_source_in(pmp_spray* h, int copy_in);

/* moveKickDrift / moveKick (SprayParticles.cpp:37-87). */
int pmp_spray_move_kick_drift(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source,
  int nboxes, double dt, double time, int is_virt, int is_ghost,
  int state_ghosts, int source_ghosts, int do_move, double spray_cfl_lev,
  void* stream);
int pmp_spray_move_kick(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source,
  int nboxes, double dt, double time, int is_virt, int is_ghost,
  int state_ghosts, int source_ghosts, double spray_cfl_lev, void* stream);

/* Method form (enum pmp_mode), default PMP_MODE_FP64. */
int pmp_spray_set_mode(pmp_spray* h, int mode);

/* Flow solver the update couples to (replaces the compile-time choice
 * PELELM_USE_SPRAY: the units of Source/PP_Spray/SprayFuelData.H:41-70, the
 * gas state of SprayInterpolation.H:111-146, the energy terms of
 * Drag.H:282-286 and 418-421).
 *   PMP_COUPLING_LMEX  (default): MKS units; the state holds rho, rho*u,
 *                      rho*Y and T; the energy source is the enthalpy source.
 *   PMP_COUPLING_PELEC: CGS units; the state holds rho, rho*u, rho*E, rho*Y
 *                      and T (the guess for the gas temperature, which is
 *                      found from e = E - |u|^2/2 and Y, EOS::EY2T); the
 *                      energy source adds the drag work and the kinetic
 *                      energy the evaporated mass carries.
 * Call before pmp_spray_setup / pmp_spray_set_data (the latent heat is
 * shifted by the fuel enthalpy in the coupling's units there); PMP_ERR_INVALID
 * after.  The PeleC coupling runs the FP64 form (default launch:
 * pmp_spray_set_launch does not apply) and the mixed form; the learned form
 * returns PMP_ERR_UNSUPPORTED in it, and pmp_spray_update_static couples to
 * PeleLMeX only. */
enum pmp_coupling { PMP_COUPLING_LMEX = 0, PMP_COUPLING_PELEC = 1 };
int pmp_spray_set_coupling(pmp_spray* h, int coupling);
int pmp_spray_get_coupling(const pmp_spray* h, int* coupling);

/* Wait for the device work of the handle's update calls (the stream of the
 * last call), report and clear their status: returns the first device error
 * of the calls since the previous pmp_spray_sync (PMP_OK if none), with the
 * box, the droplet (caller's index) and its position in pmp_spray_last_error,
 * and sets pmp_spray_get_stats to those calls' summed counters.  The
 * synchronising point of the update, where the reference's device code would
 * have aborted (SprayParticles.cpp:350,422, SprayInterpolation.H:122).
 * After graph replays on another stream, synchronise that stream first. */
int pmp_spray_sync(pmp_spray* h);
int pmp_spray_last_error(const pmp_spray* h, pmp_error_info* info);
int pmp_spray_get_stats(const pmp_spray* h, pmp_stats* stats);

/* Library version string. */
const char* pmp_spray_version(void);

/* Allocation-free update.  No counterpart in the reference: PeleMP relies on
 * AMReX allocating as it goes.  For hosts that cannot call cudaMalloc when the
 * update runs: every byte of device memory is already handed to their own
 * pre-sized pool (an arena sized at start-up), or their solver forbids device
 * allocations after initialisation.  The caller passes everything: the gas species
 * (cfg; cfg->device is ignored, the current device is used), a built SprayData,
 * the component indices, geometry and boxes, the droplets of each box as
 * DEVICE SoA arrays (updated in place, caller's order, not sorted), and
 * device state/source views.  The plain FP64 kernel runs with its working
 * data in one fixed device array inside the library (about 90 KB per device,
 * held until the process exits); nothing is allocated or freed.
 *  - nboxes <= PMP_STATIC_MAX_BOXES, else PMP_ERR_INVALID;
 *  - the first call on a device looks up that array's address (with the
 *    device current) and loads this entry point's kernels.  Under CUDA's
 *    default lazy module loading that is when the array and the kernels'
 *    code take device memory: make the first call at initialisation, before
 *    the pool reserves the device's memory, or run with
 *    CUDA_MODULE_LOADING=EAGER;
 *  - synchronous: the call waits for its kernel and reads the status back,
 *    so it cannot be captured into a CUDA graph (PMP_ERR_INVALID under an
 *    active capture);
 *  - all calls share the array: calls whose GPU work overlaps race, so
 *    serialise them;
 *  - err (may be NULL) receives the status, box and droplet index; on a
 *    nonzero return the droplet arrays and the sources may be partly updated
 *    (restore or discard them). */
#define PMP_STATIC_MAX_BOXES 256
int pmp_spray_update_static(
  const pmp_spray_config* cfg, const pmp_spray_data* data,
  const pmp_spray_comps* comps, const pmp_geometry* geom, int nboxes,
  const pmp_box* boxes, const pmp_particles* parts,
  const pmp_box_view* state, const pmp_box_view* source, double flow_dt,
  double time, int state_ghosts, int source_ghosts, int is_virt,
  int is_ghost, int do_move, double spray_cfl_lev, void* stream,
  pmp_error_info* err);

/* ---------------------------------------------------------------------------
 * The operations on either side of the update, on the device. */

/* SprayParticleContainer::estTimestep (SprayParticles.cpp:89-140): min over
 * the droplets of cfl / max_d(|u_d| / dx_d) (1e50 for a droplet at rest), -1
 * for any dead droplet still held (the reference's reduction gives dead
 * droplets -1 too; pmp_spray_redistribute drops them), then
 * min(dt, cfl dx_0 / max_jet_vel) when max_jet_vel > 0 (the injection jets'
 * bound).  -1 with fixed_parts; DBL_MAX with no droplets.  cfl is
 * particles.cfl. */
int pmp_spray_est_timestep(pmp_spray* h, double cfl, double max_jet_vel,
                           double* dt, void* stream);

/* computeDerivedVars (SprayDerive.cpp:9-155): adds into vars[b] components
 * start_indx + (0 spray_mass, 1 spray_density, 2 spray_num, 3 spray_vol,
 * 4 spray_surf_area, 5 spray_vol_frac, 6 d10, 7 d32, 8 wall_film_hght,
 * 9 wall_film_mass, 10 spray_temp, 11 num_parcels, 12-14 spray_x/y/z_vel,
 * then 15.. spray_mass_<fuel> per fuel when with_species and F > 1) from the
 * droplets of box b at the cell holding each, then divides d10 by the number,
 * d32 by the surface, temperature and velocity by the mass where the divisor
 * is non-zero, over every cell of the view.  The caller zeroes vars first, as
 * the reference's callers do.  PMP_ERR_SOURCE_BOX if a view does not hold a
 * droplet's cell. */
int pmp_spray_derive(pmp_spray* h, const pmp_box_view* vars, int nboxes,
                     int start_indx, int with_species, void* stream);

/* transferSource (SprayParticles.H:250-295) on level 0: SumBoundary of the
 * temporary source with the domain's periodicity (each ghost cell adds into
 * the valid cell of the box owning its wrapped location; ghost cells keep
 * their values), then act += tmp over each box grown by
 * min(act_ghosts, source_ghosts): all components when tmp and act have the
 * same count, else addSpraySrc's mapping (momentum, density, energy, and
 * fuel f's source into species dep_indx[f]); finally tmp = 0 everywhere.
 * tmp views cover each box grown by source_ghosts. */
int pmp_spray_transfer_source(pmp_spray* h, const pmp_box_view* tmp_source,
                              const pmp_box_view* act_source, int nboxes,
                              int source_ghosts, int act_ghosts, void* stream);

/* Re-bin the droplets after a move, what AMReX's Redistribute does for this
 * container (AMReX is not in the reference tree; the rule is restated here):
 * positions are wrapped across periodic faces (while x >= phi: x -= L; while
 * x < plo: x += L), each droplet goes to the box whose valid region holds its
 * cell floor((x - plo)/dx), and droplets with id <= 0 or in no box are
 * dropped (*removed, may be NULL, receives their count).  Afterwards every
 * box's droplets are in cell order (x fastest) and that order is the box's
 * caller order
 * for pmp_spray_get_particles. */
int pmp_spray_redistribute(pmp_spray* h, long long* removed, void* stream);

/* ---------------------------------------------------------------------------
 * Launch shape of the FP64 form (the batched form).  No counterpart in the
 * reference, which launches one kernel per box and synchronises after each
 * (SprayParticles.cpp:244-248,499).  Here all boxes go in one launch; the
 * shape only changes speed: droplet results are bit-identical for every
 * shape (deposits differ by the order of the atomic additions).
 *  - PMP_LAUNCH_GRID: one CTA per `block` droplet slots of a box;
 *  - PMP_LAUNCH_PERSISTENT: resident CTAs only (ctas_per_sm per SM, 0 = the
 *    occupancy limit) taking chunks of `chunk` slots from a device counter;
 *  - PMP_LAUNCH_PER_BOX: the reference's pattern, one launch per box with a
 *    stream synchronisation after each (the baseline of the batched form).
 * block is 64, 128 or 256 threads; regs the register cap, 96 (64 or 128
 * threads) or 128 (128 or 256 threads).  use_graph = 1 captures the device
 * work of an update (box table upload, status reset, kernels, status
 * read-back) in a CUDA graph on an internal stream and replays it while the
 * call's arguments repeat (PMP_MODE_FP64 and PMP_MODE_MIXED, not with
 * PMP_LAUNCH_PER_BOX).  The default is GRID, 128 threads, 96 registers, no
 * graph.  PMP_MODE_MIXED and PMP_MODE_LEARNED use their own launch. */
enum { PMP_LAUNCH_GRID = 0, PMP_LAUNCH_PERSISTENT = 1, PMP_LAUNCH_PER_BOX = 2 };
typedef struct pmp_launch_config {
  int kind;
  int block;
  int regs;
  int chunk;
  int ctas_per_sm;
  int use_graph;
} pmp_launch_config;

typedef struct pmp_tune_report {
  int cached;                /* 1: taken from the cache file, nothing timed */
  int ncandidates;           /* launch shapes timed */
  double best_ms;            /* device time of one update with the chosen shape */
  double default_ms;         /* with the default shape */
  double per_box_ms;         /* one launch per box, synchronised after each */
  pmp_launch_config best;    /* the chosen shape (use_graph as it was set) */
} pmp_tune_report;

int pmp_spray_set_launch(pmp_spray* h, const pmp_launch_config* cfg);
int pmp_spray_get_launch(const pmp_spray* h, pmp_launch_config* cfg);
/* The autotuner: times the FP64 update with each candidate launch shape on
 * the given views (arguments as pmp_spray_update), keeps the fastest in the
 * handle and, when cache_path is not NULL, records it in that text file
 * under a key of device name, species and fuel counts, droplet count (to a
 * power of two), box count, do_move and sub-cycle count; a later call with
 * the same key reads it back without timing.  Droplets are restored after
 * every trial and deposits go to scratch arrays: the handle's droplets and
 * the caller's source are left as they were. */
int pmp_spray_autotune(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source,
  int nboxes, double flow_dt, int state_ghosts, int source_ghosts,
  int is_ghost, int do_move, double spray_cfl_lev, const char* cache_path,
  pmp_tune_report* report, void* stream);

/* ---------------------------------------------------------------------------
 * Learned form (PMP_MODE_LEARNED).  No counterpart in the reference.  A
 * 10-64-64-64-5 SiLU network replaces the film-property and heat/mass
 * transfer evaluation of each inner sub-step of calculateSpraySource
 * (Drag.H:212-360); the drag law, sub-step count, explicit FP64 update,
 * deposits and move stay exact.  Droplets whose inputs fall outside the
 * training range (widened by gate_margin), or whose predicted outputs are
 * not sane, and droplets below 2 um, run the plain FP64 kernel instead.
 * Workflow: set grids and droplets, call pmp_spray_learn_generate on one or
 * more representative states (the FP64 teacher labels the droplets there),
 * pmp_spray_learn_train, then pmp_spray_set_mode(h, PMP_MODE_LEARNED). */
typedef struct pmp_learn_config {
  int epochs;              /* passes over the training tuples (0: 20) */
  int batch;               /* rows per Adam step (0: 8192) */
  double lr;               /* initial learning rate (0: 2e-3), decays x0.01 */
  double gate_margin;      /* accepted input range = training range widened
                              by this fraction of its span (0: 0.05) */
  double audit_fraction;   /* share of droplets re-labelled by the teacher in
                              every learned update to measure the error (0: none) */
  int no_quant;            /* 1: train without bf16 rounding (diagnostics) */
  unsigned long long seed; /* initialisation / batch order (0: 1) */
} pmp_learn_config;

typedef struct pmp_learn_report {
  long long tuples;        /* training + validation rows */
  long long steps;         /* Adam steps */
  double loss_first;       /* normalised MSE of the first / last batch */
  double loss_last;
  double val_rel_rms[5];   /* held-out RMS error per output; the outputs are
                              logarithms (fuel mass fluxes, heat transfer,
                              film viscosity, film density), so this is
                              their relative error */
  double train_ms;         /* wall time of pmp_spray_learn_train */
  double base_resid_frac[5]; /* spread (std) of each output's residual about
                              the fitted quadratic baseline over the spread
                              of the output: the network predicts the
                              residual, so its error scales with this */
} pmp_learn_report;

/* Label droplets for training: every sample_stride-th droplet (offset from
 * seed) at the given device state, plus `augment` perturbed copies of each
 * (temperature towards boiling, diameter, slip and composition).  Tuples
 * accumulate over calls.  Views and arguments as for pmp_spray_update; no
 * droplet or state is modified. */
int pmp_spray_learn_generate(
  pmp_spray* h, const pmp_box_view* state, int nboxes, double flow_dt,
  int state_ghosts, int do_move, double spray_cfl_lev,
  long long sample_stride, int augment, unsigned long long seed,
  void* stream);
int pmp_spray_learn_count(const pmp_spray* h, long long* n);
/* Copy up to *n tuples to buf (16 floats each: the 10 raw inputs, the 5
 * targets, one pad); *n receives the number copied.  With buf NULL, *n
 * receives the number held. */
int pmp_spray_learn_tuples(const pmp_spray* h, float* buf, long long* n);
/* Train the network on the GPU (own forward / backward / Adam kernels; the
 * forward pass rounds weights and activations to bf16 as inference does).
 * The network learns each output's residual about a quadratic polynomial in
 * the normalised inputs, fitted first by least squares (FP64) over the
 * tuples; inference adds the polynomial (FP32) back. */
int pmp_spray_learn_train(pmp_spray* h, const pmp_learn_config* cfg,
                          pmp_learn_report* report);
/* get = 1: copy the trained parameters, normalisation and baseline
 * coefficients to buf; get = 0: install them from buf.  With buf NULL,
 * *count receives the length. */
int pmp_spray_learn_weights(pmp_spray* h, int get, float* buf,
                            long long* count);
/* Share of droplets audited by the teacher in each learned update. */
int pmp_spray_learn_set_audit(pmp_spray* h, double audit_fraction);
/* Result of the audit of the last learned update: droplets audited and the
 * RMS error of each of the 5 surrogate outputs, measured as val_rel_rms. */
int pmp_spray_learn_audit(const pmp_spray* h, long long* audited,
                          double rel_rms[5]);
/* Check of the training kernels: MSE loss and its gradient for n rows of
 * normalised inputs x[n][10] and targets y[n][5] at the flat parameter
 * vector params[pmp_learn_param_count()] (quant = 1 rounds to bf16 as the
 * training forward pass does).  Runs on the current device. */
int pmp_learn_debug_grad(const float* params, const float* x, const float* y,
                         int n, int quant, float* grads, double* loss);
/* Check of the inference: the network evaluated with warp-level mma.sync
 * tiles (the cross-check of the tcgen05 path) on n rows of normalised inputs
 * xn[n][10] at params; outputs y[n][5]. */
int pmp_learn_debug_infer(const float* params, const float* xn, int n,
                          float* y);
/* The same with the CTA-level tcgen05 network of the learned update kernel
 * (tensor-memory accumulators, 128-row tiles, 256 rows per CTA here);
 * PMP_ERR_TIMEOUT if an MMA completion wait timed out. */
int pmp_learn_debug_infer_tc(const float* params, const float* xn, int n,
                             float* y);
/* Check of the tcgen05 timeout path: one CTA waits on an mbarrier that
 * nothing arrives on.  Returns PMP_ERR_TIMEOUT when the bounded wait gave up
 * (as it must), with the cycles it waited; the device stays usable. */
int pmp_learn_debug_wait_timeout(long long* cycles);
int pmp_learn_param_count(void);
/* Number of terms of the targets' baseline polynomial (per output). */
int pmp_learn_base_terms(void);
/* Host evaluation of the baseline (no GPU): its terms feats[base_terms] for
 * normalised inputs xn[10] and the derived variables ell = ln(1 + B_M) and
 * g = (1 + c Re)^(1/3) - 2, and the polynomial with coefficients
 * coef[base_terms] in FP32 as the kernels evaluate it. */
int pmp_learn_debug_base(const float* xn, float ell, float g, const float* coef,
                         double* feats, float* value);
/* Host solve of the baseline fit (no GPU): acc holds the normal equations
 * (the upper triangle of F^T F row by row, then F^T Y row by row, F the
 * terms, Y the 5 targets); coef[5][base_terms] receives the ridge least
 * squares coefficients. */
int pmp_learn_debug_solve_baseline(const double* acc, float* coef);

/* ---------------------------------------------------------------------------
 * Measured compute peaks of a device (no counterpart in the reference): the
 * rates of loop kernels of independent FP64 FMAs, FP32 FMAs and SFU base-2
 * exponentials over the whole GPU, best of three timed launches, at the
 * clocks the device runs at (no setting is changed).  The denominators of
 * the update kernels' compute roofline: fp64 and fp32 in TFLOP/s (an FMA is
 * 2 FLOP), sfu in G operations/s. */
int pmp_measure_peaks(int device, double* fp64_tflops, double* fp32_tflops,
                      double* sfu_gops);

#ifdef __cplusplus
}
#endif

#endif /* PMP_SPRAY_H */
