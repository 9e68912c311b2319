// Stand-in for the PelePhysics interface the spray headers call
// (eos.molecular_weight / T2Cpi / T2Hi, trans.transport, Constants::RU/PATM),
// backed by the project's thermo/transport model (pmp_thermo.h) evaluated
// with the C library's math.  TEST INFRASTRUCTURE for the oracle's reference
// build; PelePhysics itself is not part of PeleMP.
#ifndef PMP_REF_SHIM_PELEPHYSICS_H
#define PMP_REF_SHIM_PELEPHYSICS_H

#include <AMReX_RealVect.H>

#ifndef PMP_USE_LIBM
#define PMP_USE_LIBM 1
#endif
#include "../../pelemp_b200/csrc/phys/pmp_thermo.h"

namespace pele {
namespace physics {

/* the active mechanism of the reference build (set by the driver) */
inline pmp_mech& ref_mech()
{
  static pmp_mech m;
  return m;
}

namespace Constants {
constexpr amrex::Real RU = 8.31446261815324e7;
constexpr amrex::Real PATM = 1013250.0;
} // namespace Constants

struct EosType {};
struct TransportType {};

namespace transport {
template <class E, class T>
struct TransParm {
  int unused = 0;
};
} // namespace transport

struct RefEos {
  void molecular_weight(amrex::Real* mw) const { pmp_eos_molecular_weight(&ref_mech(), mw); }
  void T2Cpi(amrex::Real T, amrex::Real* cp) const { pmp_eos_T2Cpi(&ref_mech(), T, cp); }
  void T2Hi(amrex::Real T, amrex::Real* h) const { pmp_eos_T2Hi(&ref_mech(), T, h); }
  void EY2T(const amrex::Real e, const amrex::Real* Y, amrex::Real& T) const
  {
    pmp_eos_EY2T(&ref_mech(), e, Y, &T);
  }
};

struct RefTransport {
  void transport(
    bool get_xi, bool get_mu, bool get_lam, bool get_Ddiag, bool get_chi,
    amrex::Real T, amrex::Real rho, amrex::Real* Y, amrex::Real* Ddiag,
    amrex::Real* chi, amrex::Real& mu, amrex::Real& xi, amrex::Real& lam,
    transport::TransParm<EosType, TransportType> const* /*tparm*/) const
  {
    (void)get_xi;
    (void)get_chi;
    (void)chi;
    (void)xi;
    pmp_transport(&ref_mech(), get_mu, get_lam, get_Ddiag, T, rho, Y, Ddiag, &mu, &lam);
  }
};

struct PhysicsType {
  static RefEos eos() { return RefEos{}; }
  static RefTransport transport() { return RefTransport{}; }
};

} // namespace physics
} // namespace pele

#endif
