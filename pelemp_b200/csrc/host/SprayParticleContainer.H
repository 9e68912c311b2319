// SprayParticleContainer.H -- C++ host-side mirror of PeleMP's spray
// container update surface, over the C ABI of include/pmp_spray.h.
//
// Method names, argument order and meaning follow
// Source/PP_Spray/SprayParticles.H:195-243 (moveKick, moveKickDrift,
// updateParticles), SprayParticles.H:386 (AssignSprayComps) and
// SpraySetup.cpp:73-297 (readSprayParams, spraySetup).  Where the reference
// calls amrex::Abort this class throws pmp::SprayAbort with the reference's
// message text; the process is never terminated.
//
// Mesh data are passed as one pmp_box_view per box (the Array4 of the box's
// fab: data pointer, allocated bounds, strides), in ParIter order, on the
// device (pmp_spray_update) or on the host (updateParticlesHost).
//
// The update methods are stream-ordered, as the C ABI is: they return once
// the work is enqueued.  synchronize() is where a device-side error of the
// enqueued updates surfaces as SprayAbort (the reference's device abort
// surfaces at its stream synchronisation, SprayParticles.cpp:499); call it
// before reading host-view sources or the stats.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "pmp_spray.h"

namespace pmp {

class SprayAbort : public std::runtime_error
{
public:
  SprayAbort(int code, const std::string& msg, const pmp_error_info& info)
    : std::runtime_error(msg), code_(code), info_(info)
  {
  }
  int code() const { return code_; }
  const pmp_error_info& info() const { return info_; }

private:
  int code_;
  pmp_error_info info_;
};

class SprayParticleContainer
{
public:
  using Real = double;

  SprayParticleContainer(const std::vector<std::string>& species, int nfuel, int device = 0)
  {
    pmp_spray_config cfg{};
    cfg.nfuel = nfuel;
    cfg.nspec = static_cast<int>(species.size());
    cfg.device = device;
    for (size_t k = 0; k < species.size() && k < PMP_MAX_SPEC; ++k) {
      species[k].copy(cfg.species[k], PMP_NAME_LEN - 1);
    }
    const int rc = pmp_spray_create(&cfg, &h_);
    if (rc != PMP_OK) {
      pmp_error_info none{};
      throw SprayAbort(rc, "SprayParticleContainer: no usable sm_100 device or bad species", none);
    }
  }
  ~SprayParticleContainer() { pmp_spray_destroy(h_); }
  SprayParticleContainer(const SprayParticleContainer&) = delete;
  SprayParticleContainer& operator=(const SprayParticleContainer&) = delete;

  /// readSprayParams + spraySetup (SpraySetup.cpp:73-297)
  void readSprayParams(const pmp_spray_inputs& inputs) { check(pmp_spray_setup(h_, &inputs)); }

  /// AssignSprayComps (SprayParticles.H:386)
  void AssignSprayComps(const pmp_spray_comps& comps) { check(pmp_spray_set_comps(h_, &comps)); }

  /// Geom(level) and the boundary designation (SprayParticles.cpp:183-218)
  void setGeometry(const pmp_geometry& geom) { check(pmp_spray_set_geometry(h_, &geom)); }

  /// the level's BoxArray, ParIter order
  void setGrids(const std::vector<pmp_box>& boxes)
  {
    nboxes_ = static_cast<int>(boxes.size());
    check(pmp_spray_set_grids(h_, nboxes_, boxes.data()));
  }

  void setParticles(int box, const pmp_particles& p) { check(pmp_spray_set_particles(h_, box, &p)); }
  void getParticles(int box, pmp_particles& p) { check(pmp_spray_get_particles(h_, box, &p)); }
  long long numParticles(int box) const
  {
    long long n = 0;
    pmp_spray_num_particles(h_, box, &n);
    return n;
  }
  void setMode(int mode) { check(pmp_spray_set_mode(h_, mode)); }
  /// the flow solver (PMP_COUPLING_LMEX / PMP_COUPLING_PELEC), before readSprayParams
  void setCoupling(int coupling) { check(pmp_spray_set_coupling(h_, coupling)); }

  /// Update but do not move particles (SprayParticles.cpp:37-57)
  void moveKick(
    const std::vector<pmp_box_view>& state, const std::vector<pmp_box_view>& source,
    const int level, const Real& dt, const Real time, const bool isVirtualPart,
    const bool isGhostPart, const int state_ghosts, const int source_ghosts,
    const void* ltransparm = nullptr, const Real spray_cfl_lev = -1., void* stream = nullptr)
  {
    moveKickDrift(
      state, source, level, dt, time, isVirtualPart, isGhostPart, state_ghosts, source_ghosts,
      false, ltransparm, spray_cfl_lev, stream);
  }

  /// Update and move particles (SprayParticles.cpp:59-87)
  void moveKickDrift(
    const std::vector<pmp_box_view>& state, const std::vector<pmp_box_view>& source,
    const int level, const Real& dt, const Real time, const bool isVirtualPart,
    const bool isGhostPart, const int state_ghosts, const int source_ghosts, const bool do_move,
    const void* ltransparm = nullptr, const Real spray_cfl_lev = -1., void* stream = nullptr)
  {
    updateParticles(
      level, state, source, dt, time, state_ghosts, source_ghosts, isVirtualPart, isGhostPart,
      do_move, ltransparm, spray_cfl_lev, stream);
  }

  /// Where the mesh views passed to updateParticles / moveKick /
  /// moveKickDrift live: device memory (default, as in an AMReX GPU build) or
  /// host memory (the library stages them to the device inside the call).
  void setViewsOnHost(bool on_host) { views_on_host_ = on_host; }

  /// Update particle data and solve gas-phase source terms
  /// (SprayParticles.cpp:142-502).  The transport parameters are built into
  /// the handle, so ltransparm is ignored.
  void updateParticles(
    const int& level, const std::vector<pmp_box_view>& state,
    const std::vector<pmp_box_view>& source, const Real& flow_dt, const Real& time,
    const int state_ghosts, const int source_ghosts, const bool isVirt, const bool isGhost,
    const bool do_move, const void* ltransparm, const Real spray_cfl_lev,
    void* stream = nullptr)
  {
    if (views_on_host_) {
      updateParticlesHost(level, state, source, flow_dt, time, state_ghosts, source_ghosts, isVirt,
                          isGhost, do_move, ltransparm, spray_cfl_lev, stream);
      return;
    }
    (void)level;
    check(pmp_spray_update(
      h_, state.data(), source.data(), static_cast<int>(state.size()), flow_dt, time,
      state_ghosts, source_ghosts, isVirt, isGhost, do_move, spray_cfl_lev, stream));
  }

  /// updateParticles with host views (copies inside)
  void updateParticlesHost(
    const int& level, const std::vector<pmp_box_view>& state,
    const std::vector<pmp_box_view>& source, const Real& flow_dt, const Real& time,
    const int state_ghosts, const int source_ghosts, const bool isVirt, const bool isGhost,
    const bool do_move, const void* /*ltransparm*/, const Real spray_cfl_lev,
    void* stream = nullptr)
  {
    (void)level;
    check(pmp_spray_update_host(
      h_, state.data(), source.data(), static_cast<int>(state.size()), flow_dt, time,
      state_ghosts, source_ghosts, isVirt, isGhost, do_move, spray_cfl_lev, stream));
  }

  /// Wait for the enqueued updates; throws SprayAbort with the reference's
  /// abort message if one of them failed on the device.
  void synchronize() { check(pmp_spray_sync(h_)); }

  /// counters of the updates between the last two synchronize() calls
  pmp_stats stats() const
  {
    pmp_stats s{};
    pmp_spray_get_stats(h_, &s);
    return s;
  }

  /// estTimestep (SprayParticles.cpp:89-140); cfl is particles.cfl, max_jet_vel
  /// the fastest injection jet (0 without jets).  Single process: the
  /// ReduceRealMin over ranks is the caller's.
  Real estTimestep(int /*level*/, Real cfl, Real max_jet_vel = 0., void* stream = nullptr)
  {
    double dt = 0.;
    check(pmp_spray_est_timestep(h_, cfl, max_jet_vel, &dt, stream));
    return dt;
  }

  /// computeDerivedVars (SprayDerive.cpp:9-155): one view of mf_var per box.
  void computeDerivedVars(
    const std::vector<pmp_box_view>& mf_var, int /*level*/, int start_indx, bool derive_plot_species = true,
    void* stream = nullptr)
  {
    check(pmp_spray_derive(h_, mf_var.data(), static_cast<int>(mf_var.size()), start_indx,
                           derive_plot_species ? 1 : 0, stream));
  }

  /// transferSource (SprayParticles.H:250-295), level 0: fold the ghost
  /// deposits of tmpSource, add into actSource, zero tmpSource.
  void transferSource(
    int source_ghosts, int level, const std::vector<pmp_box_view>& tmpSource,
    const std::vector<pmp_box_view>& actSource, int act_ghosts, void* stream = nullptr)
  {
    if (level != 0) {
      throw SprayAbort(PMP_ERR_UNSUPPORTED, "SprayParticleContainer::transferSource: level 0 only", {});
    }
    check(pmp_spray_transfer_source(h_, tmpSource.data(), actSource.data(), static_cast<int>(tmpSource.size()),
                                    source_ghosts, act_ghosts, stream));
  }

  /// Redistribute for this container: re-bin moved droplets to their boxes
  /// (periodic wrap), drop dead ones; returns how many were dropped.
  long long Redistribute(void* stream = nullptr)
  {
    long long removed = 0;
    check(pmp_spray_redistribute(h_, &removed, stream));
    return removed;
  }

  pmp_spray* handle() { return h_; }

private:
  void check(int rc)
  {
    if (rc == PMP_OK) {
      return;
    }
    pmp_error_info info{};
    pmp_spray_last_error(h_, &info);
    // the reference's amrex::Abort messages (SprayParticles.cpp:350,422;
    // SprayInterpolation.H:122)
    std::string msg;
    switch (rc) {
      case PMP_ERR_LEFT_DOMAIN: msg = "Particle has incorrectly left the domain"; break;
      case PMP_ERR_SOURCE_BOX: msg = "SprayParticleContainer::updateParticles() -- source box too small"; break;
      case PMP_ERR_STATE_BOX: msg = "SprayParticleContainer::updateParticles() -- state box too small"; break;
      default: msg = std::string("SprayParticleContainer: ") + info.message; break;
    }
    throw SprayAbort(rc, msg, info);
  }

  pmp_spray* h_ = nullptr;
  int nboxes_ = 0;
  bool views_on_host_ = false;
};

}  // namespace pmp
