// ref_driver.cpp -- runs PeleMP's own spray physics headers on the host.
//
// TEST INFRASTRUCTURE.  Compiled (by oracle/Makefile) directly against the
// reference sources Source/PP_Spray/{SprayFuelData.H, Drag.H,
// SprayInterpolation.H, WallFunctions.H} and BreakupSplash/{SBData.H,
// AhamedSplash.H}, with the stand-in AMReX/PelePhysics headers of
// oracle/ref_shim and PELELM_USE_SPRAY defined; output goes to oracle/_ref.
// The per-droplet loop below restates the device lambda of
// SprayParticleContainer::updateParticles (SprayParticles.cpp:324-481)
// around those functions (the lambda's own file needs the full AMReX
// particle container and is not compiled); breakup and splash branches are
// not taken (their inputs are rejected).  Abort() is turned into a status.
//
// Its purpose: the C oracle (spray_oracle.c) built with the C library's math
// must reproduce this program bit for bit.
#include <AMReX_RealVect.H>

#include "PelePhysics.H"

#include "SprayFuelData.H"

struct RefParticle {
  amrex::Real m_pos[3];
  amrex::Real m_rdata[SprayComps::pstateNum];
  int m_id;
  int m_cpu;
  amrex::RealVect pos() const { return amrex::RealVect(m_pos[0], m_pos[1], m_pos[2]); }
  amrex::Real& pos(int d) { return m_pos[d]; }
  amrex::Real& rdata(int i) { return m_rdata[i]; }
  const amrex::Real& rdata(int i) const { return m_rdata[i]; }
  int& id() { return m_id; }
};

struct SprayParticleContainer {
  using ParticleType = RefParticle;
};

#include "SBData.H"

#include "Drag.H"
#include "SprayInterpolation.H"
#include "WallFunctions.H"

#include "../include/pmp_spray.h"

#include <cstring>
#include <cstdio>

using namespace amrex;

static SprayData to_spray_data(const pmp_spray_data* f)
{
  SprayData s{};
  s.mass_trans = f->mass_trans != 0;
  s.mom_trans = f->mom_trans != 0;
  s.fixed_parts = f->fixed_parts != 0;
  s.do_splash = f->do_splash != 0;
  s.do_breakup = f->do_breakup;
  s.min_eb_vfrac = f->min_eb_vfrac;
  s.ref_T = f->ref_T;
  s.sigma = f->sigma;
  s.wall_T = f->wall_T;
  s.theta_c = f->theta_c;
  s.dtmod = f->dtmod;
  for (int d = 0; d < 3; ++d) {
    s.body_force[d] = f->body_force[d];
  }
  for (int i = 0; i < SPRAY_FUEL_NUM; ++i) {
    s.critT[i] = f->critT[i];
    s.boilT[i] = f->boilT[i];
    s.cp[i] = f->cp[i];
    s.latent[i] = f->latent[i];
    s.ref_latent[i] = f->ref_latent[i];
    s.indx[i] = f->indx[i];
    s.dep_indx[i] = f->dep_indx[i];
    for (int c = 0; c < 4; ++c) {
      s.psat_coef[4 * i + c] = f->psat_coef[4 * i + c];
      s.rho_coef[4 * i + c] = f->rho_coef[4 * i + c];
      s.lambda_coef[4 * i + c] = f->lambda_coef[4 * i + c];
      s.mu_coef[4 * i + c] = f->mu_coef[4 * i + c];
    }
  }
  return s;
}

static Array4<Real> view_comp(const pmp_box_view& v, int comp)
{
  Array4<Real> a;
  a.p = v.p + static_cast<long long>(comp) * v.nstride;
  for (int d = 0; d < 3; ++d) {
    a.lo[d] = v.lo[d];
  }
  a.jstride = v.jstride;
  a.kstride = v.kstride;
  a.nstride = v.nstride;
  return a;
}

static Box to_box(const pmp_box& b)
{
  return Box(IntVect(b.lo[0], b.lo[1], b.lo[2]), IntVect(b.hi[0], b.hi[1], b.hi[2]));
}

extern "C" int pmp_ref_update(
  const pmp_mech* mech, const pmp_spray_data* fdat_in,
  const pmp_spray_comps* comps, const pmp_geometry* geom, int nboxes,
  const pmp_box* boxes, pmp_particles* parts, const pmp_box_view* state,
  const pmp_box_view* source, double flow_dt, int state_ghosts,
  int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, int nthreads, pmp_error_info* err,
  long long* substeps)
{
  (void)nthreads;
  if (mech->nspec != NUM_SPECIES || fdat_in->nfuel != SPRAY_FUEL_NUM) {
    return PMP_ERR_INVALID;
  }
  if (fdat_in->do_breakup != 0 || fdat_in->do_splash) {
    return PMP_ERR_UNSUPPORTED;
  }
  pele::physics::ref_mech() = *mech;
  const SprayData fdat_v = to_spray_data(fdat_in);
  const SprayData* fdat = &fdat_v;
  const SprayComps SPI{
    comps->rhoIndx,    comps->momIndx,    comps->engIndx,
    comps->utempIndx,  comps->specIndx,   comps->rhoSrcIndx,
    comps->momSrcIndx, comps->engSrcIndx, comps->specSrcIndx};
  pele::physics::transport::TransParm<pele::physics::EosType, pele::physics::TransportType> tp;
  const auto* ltransparm = &tp;
  const bool isGhost = is_ghost != 0;
  const bool isActive = !(is_virt || is_ghost);
  (void)isActive;
  // SprayParticles.cpp:183-229
  RealVect dx(geom->dx[0], geom->dx[1], geom->dx[2]);
  RealVect dxi(1. / dx[0], 1. / dx[1], 1. / dx[2]);
  RealVect plo(geom->plo[0], geom->plo[1], geom->plo[2]);
  RealVect phi(geom->phi[0], geom->phi[1], geom->phi[2]);
  const Box domain(
    IntVect(geom->domain_lo[0], geom->domain_lo[1], geom->domain_lo[2]),
    IntVect(geom->domain_hi[0], geom->domain_hi[1], geom->domain_hi[2]));
  IntVect bndry_lo(geom->bndry_lo[0], geom->bndry_lo[1], geom->bndry_lo[2]);
  IntVect bndry_hi(geom->bndry_hi[0], geom->bndry_hi[1], geom->bndry_hi[2]);
  const Real vol = AMREX_D_TERM(dx[0], *dx[1], *dx[2]);
  const Real inv_vol = 1. / vol;
  Real sub_cfl = 0.5;
  Real sub_dt = flow_dt;
  int num_iter = 1;
  if (do_move && spray_cfl_lev > sub_cfl) {
    num_iter = static_cast<int>(std::ceil(spray_cfl_lev / sub_cfl));
    sub_dt = flow_dt / static_cast<Real>(num_iter);
  }
  long long nsubs = 0;
  if (err) {
    std::memset(err, 0, sizeof(*err));
    err->particle = -1;
  }
  for (int b = 0; b < nboxes; ++b) {
    Box tile_box = to_box(boxes[b]);
    Box src_box = tile_box;
    src_box.grow(source_ghosts);
    Box state_box = tile_box;
    state_box.grow(state_ghosts);
    const bool at_bounds = tile_at_bndry(tile_box, bndry_lo, bndry_hi, domain);
    pmp_particles& P = parts[b];
    const long long Np = P.n;
    const int nr = SprayComps::pstateNum;
    std::vector<RefParticle> aos(static_cast<size_t>(Np));
    for (long long i = 0; i < Np; ++i) {
      for (int d = 0; d < 3; ++d) {
        aos[i].m_pos[d] = P.pos[d][i];
      }
      for (int r = 0; r < nr; ++r) {
        aos[i].m_rdata[r] = P.rdata[r][i];
      }
      aos[i].m_id = P.id[i];
      aos[i].m_cpu = 0;
    }
    Array4<const Real> Tarr, rhoYarr, rhoarr, momarr, engarr;
    {
      auto c = [&](int comp) {
        Array4<Real> a = view_comp(state[b], comp);
        Array4<const Real> r;
        r.p = a.p;
        for (int d = 0; d < 3; ++d) {
          r.lo[d] = a.lo[d];
        }
        r.jstride = a.jstride;
        r.kstride = a.kstride;
        r.nstride = a.nstride;
        return r;
      };
      Tarr = c(SPI.utempIndx);
      rhoYarr = c(SPI.specIndx);
      rhoarr = c(SPI.rhoIndx);
      momarr = c(SPI.momIndx);
      engarr = c(SPI.engIndx);
    }
    Array4<Real> rhoYSrcarr = view_comp(source[b], SPI.specSrcIndx);
    Array4<Real> rhoSrcarr = view_comp(source[b], SPI.rhoSrcIndx);
    Array4<Real> momSrcarr = view_comp(source[b], SPI.momSrcIndx);
    Array4<Real> engSrcarr = view_comp(source[b], SPI.engSrcIndx);
    SBPtrs rf_d;
    splash_breakup* N_SB = nullptr;
    const bool do_splash_box = false;
    const bool eb_in_box = false;
    // Gpu::Atomic::Add: an OpenMP atomic when droplets run on several threads
    const bool atomic = nthreads > 1;
    auto atomic_add = [atomic](Real& dst, Real v) {
      if (atomic) {
#pragma omp atomic
        dst += v;
      } else {
        dst += v;
      }
    };
    long long first_bad = -1;
    int bad_code = 0;
    long long box_subs = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 1 ? nthreads : 1) reduction(+ : box_subs)
    for (long long pid = 0; pid < Np; ++pid) {
      RefParticle& p = aos[pid];
      try {
        // ---- SprayParticles.cpp:326-480 ----
        if (p.id() > 0) {
          auto eos = pele::physics::PhysicsType::eos();
          SprayUnits SPU;
          GasPhaseVals gpv;
          GpuArray<Real, SPRAY_FUEL_NUM> cBoilT;
          eos.molecular_weight(gpv.mw.data());
          for (int n = 0; n < NUM_SPECIES; ++n) {
            gpv.mw[n] *= SPU.mass_conv;
          }
          GpuArray<IntVect, AMREX_D_PICK(2, 4, 8)> indx_array;
          GpuArray<Real, AMREX_D_PICK(2, 4, 8)> weights;
          RealVect lx = (p.pos() - plo) * dxi + 0.5;
          IntVect ijk = lx.floor();
          RealVect lxc = (p.pos() - plo) * dxi;
          IntVect ijkc = lxc.floor();
          IntVect bflags(IntVect::TheZeroVector());
          if (at_bounds) {
            bool left_dom = check_bounds(p.pos(), plo, phi, dx, bndry_lo, bndry_hi, bflags);
            if (left_dom) {
              throw std::pair<int, long long>(PMP_ERR_LEFT_DOMAIN, pid);
            }
          }
          for (int cur_iter = 0; cur_iter < num_iter && p.id() > 0; ++cur_iter) {
            if (p.rdata(SprayComps::pstateFilmHght) > 0.) {
              throw std::pair<int, long long>(PMP_ERR_UNSUPPORTED, pid);
            }
            trilinear_interp(ijk, lx, indx_array.data(), weights.data(), bflags);
            gpv.reset();
            try {
              InterpolateGasPhase(
                gpv, state_box, rhoarr, rhoYarr, Tarr, momarr, engarr, indx_array.data(),
                weights.data());
            } catch (const RefAbort&) {
              throw std::pair<int, long long>(PMP_ERR_STATE_BOX, pid);
            }
            gpv.define();
            fdat->calcBoilT(gpv, cBoilT.data());
            calculateSpraySource(sub_dt, gpv, *fdat, p, cBoilT.data(), ltransparm);
            ++box_subs;
            IntVect cur_indx = ijkc;
            Real cvol = inv_vol;
            Real cur_coef = -cvol * sub_dt / flow_dt;
            if (!src_box.contains(cur_indx)) {
              if (!isGhost) {
                throw std::pair<int, long long>(PMP_ERR_SOURCE_BOX, pid);
              }
            }
            if (fdat->mom_trans) {
              for (int dir = 0; dir < AMREX_SPACEDIM; ++dir) {
                atomic_add(momSrcarr(cur_indx, dir), cur_coef * gpv.fluid_mom_src[dir]);
              }
            }
            if (fdat->mass_trans) {
              atomic_add(rhoSrcarr(cur_indx), cur_coef * gpv.fluid_mass_src);
              for (int spf = 0; spf < SPRAY_FUEL_NUM; ++spf) {
                atomic_add(rhoYSrcarr(cur_indx, spf), cur_coef * gpv.fluid_Y_dot[spf]);
              }
            }
            atomic_add(engSrcarr(cur_indx), cur_coef * gpv.fluid_eng_src);
            if (do_move && !fdat->fixed_parts && p.id() > 0) {
              for (int dir = 0; dir < AMREX_SPACEDIM; ++dir) {
                const Real cvel = p.rdata(SprayComps::pstateVel + dir);
                p.pos(dir) += sub_dt * cvel;
              }
              if (at_bounds) {
                bool left_dom =
                  check_bounds(p.pos(), plo, phi, dx, bndry_lo, bndry_hi, bflags);
                if (left_dom) {
                  p.id() = -1;
                } else {
                  Real film_h = 0.;
                  impose_wall(
                    do_splash_box, static_cast<int>(pid), p, *fdat, dx, plo, phi, bflags,
                    cBoilT.data(), gpv.p_fluid, eb_in_box, ijkc, N_SB, rf_d, film_h);
                }
              }
              lx = (p.pos() - plo) * dxi + 0.5;
              ijk = lx.floor();
              lxc = (p.pos() - plo) * dxi;
              ijkc = lxc.floor();
            }
            if (isGhost && !src_box.contains(ijkc)) {
              p.id() = -1;
            }
          }
        }
      } catch (const std::pair<int, long long>& e) {
#pragma omp critical
        {
          if (first_bad < 0 || e.second < first_bad) {
            first_bad = e.second;
            bad_code = e.first;
          }
        }
      }
    }
    nsubs += box_subs;
    if (first_bad >= 0) {
      if (err) {
        err->code = bad_code;
        err->box = b;
        err->particle = first_bad;
        std::snprintf(err->message, sizeof(err->message), "reference: error %d", bad_code);
      }
      if (substeps) {
        *substeps = nsubs;
      }
      return bad_code;
    }
    for (long long i = 0; i < Np; ++i) {
      for (int d = 0; d < 3; ++d) {
        P.pos[d][i] = aos[i].m_pos[d];
      }
      for (int r = 0; r < nr; ++r) {
        P.rdata[r][i] = aos[i].m_rdata[r];
      }
      P.id[i] = aos[i].m_id;
    }
  }
  if (substeps) {
    *substeps = nsubs;
  }
  return PMP_OK;
}
