/* spray_oracle.h -- CPU FP64 oracle of the spray particle update.
 *
 * TEST INFRASTRUCTURE.  Only the tests, the smoke check and the bench's CPU
 * baseline load this code, to compare against; the product (libpmpspray) never
 * links it.
 *
 * A plain-C restatement of PeleMP's non-EB, no-breakup, no-splash
 * updateParticles path in PeleLMeX units:
 *   Source/PP_Spray/SprayParticles.cpp:142-502   (driver, gather/scatter/move)
 *   Source/PP_Spray/Drag.H:6-441                 (calcHeatCoeff, calcVaporState,
 *                                                 calculateSpraySource)
 *   Source/PP_Spray/SprayInterpolation.H:64-199  (check_bounds, InterpolateGasPhase,
 *                                                 trilinear_interp)
 *   Source/PP_Spray/SprayFuelData.H:42-212       (SprayUnits, GasPhaseVals, SprayData)
 *   Source/PP_Spray/WallFunctions.H:8-35,89-234  (tile_at_bndry, check_wall, impose_wall)
 *   Source/PP_Spray/SpraySetup.cpp:73-297        (SprayData build, latent adjustment)
 * The arithmetic follows the reference expression by expression, so that
 * when it is built with the C library's math (PMP_USE_LIBM) it reproduces,
 * bit for bit, the reference headers compiled against the same thermo model
 * (oracle/ref_driver.cpp).  The default build uses the project's math
 * library (pmp_math.h), the same functions the CUDA kernels call.
 *
 * Parity pin: the reference ships no numeric results for this path; the pin
 * is the bitwise comparison with the reference's own Drag.H, SprayFuelData.H
 * and SprayInterpolation.H compiled in this repository's build, plus the
 * known-answer checks in tests/.  The gas thermo/transport under both is the
 * project's model (PelePhysics is not part of PeleMP): parity unpinned
 * against PelePhysics itself.
 */
#ifndef PMP_SPRAY_ORACLE_H
#define PMP_SPRAY_ORACLE_H

#include "../include/pmp_spray.h"
#include "../pelemp_b200/csrc/phys/pmp_thermo.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Coupling of every following call: 0 = PeleLMeX (PELELM_USE_SPRAY, the
 * default), 1 = PeleC (CGS units, energy-based gas temperature, kinetic
 * energy and drag-work energy sources). */
void pmp_oracle_set_coupling(int pelec);

/* Build a mechanism from species names; returns 0 or -1. */
int pmp_oracle_mech(pmp_mech* mech, int nspec, const char (*names)[PMP_NAME_LEN]);

/* readSprayParams + spraySetup; returns PMP_OK or an error code. */
int pmp_oracle_setup(
  const pmp_mech* mech, const char (*names)[PMP_NAME_LEN],
  const pmp_spray_inputs* in, pmp_spray_data* out);

/* updateParticles for every box.  parts[b] are HOST SoA droplets of box b,
 * updated in place; state/source are HOST views.  nthreads == 1 runs the
 * droplets of a box in order (deterministic deposits); nthreads > 1 runs
 * them with OpenMP and atomic deposits.  substeps (may be NULL) receives the
 * number of droplet-substeps executed. */
int pmp_oracle_update(
  const pmp_mech* mech, const pmp_spray_data* fdat,
  const pmp_spray_comps* comps, const pmp_geometry* geom, int nboxes,
  const pmp_box* boxes, pmp_particles* parts, const pmp_box_view* state,
  const pmp_box_view* source, double flow_dt, int state_ghosts,
  int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, int nthreads, pmp_error_info* err,
  long long* substeps);

/* Energy identity of the explicit scheme (PeleLMeX coupling): when per_box
 * is not NULL, every following pmp_oracle_update adds to per_box[b][i] the
 * parcel's residual of  (liquid enthalpy change) + (enthalpy received by the
 * gas)  for droplet i of box b, summed over the call's sub-cycles, as the
 * named terms of calculateSpraySource's comment in spray_oracle.c (the
 * explicit update, the composition clip, the latent heat taken below the
 * boiling temperature, the vapour enthalpy taken at the last sub-step, a
 * droplet's death, the average over the sub-steps).  NULL
 * switches it off. */
void pmp_oracle_set_energy_out(double** per_box);

/* One evaluation of calculateSpraySource for a single droplet against a
 * given interpolated gas state (unit-level hook for the tests).
 * rdata: the droplet's real components (updated in place); gas: rho, T,
 * vel[3], Y[nspec] in MKS; returns the Reynolds number.  src receives
 * fluid_mom_src[3], fluid_mass_src, fluid_eng_src, fluid_Y_dot[F]. */
double pmp_oracle_droplet_source(
  const pmp_mech* mech, const pmp_spray_data* fdat, double flow_dt,
  const double* gas, double* rdata, int* id, double* src);

#ifdef __cplusplus
}
#endif

#endif
