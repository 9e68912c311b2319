// pmp_device.cuh -- device-side data structures of the spray update.
//
// KParams is the single __grid_constant__ argument of every update kernel:
// the handle's mechanism (species reordered so that fuel f is species f),
// the SprayData constants, the level geometry and the per-call settings.
// BoxEntry describes one AMReX box: its state and source Array4 views and its
// droplet range in the library's cell-sorted SoA.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pmp_spray.h"

namespace pmp {

constexpr int kMaxSpec = PMP_MAX_SPEC;
constexpr int kMaxFuel = PMP_MAX_FUEL;

// SprayUnits, PeleLMeX branch (Source/PP_Spray/SprayFuelData.H:44-54,66)
constexpr double kRuConv = 1.E-7;
constexpr double kEngConv = 1.E-4;
constexpr double kRhoConv = 1.E3;
constexpr double kMassConv = 1.E-3;
constexpr double kRhodConv = 0.1;
constexpr double kMuConv = 0.1;
constexpr double kLambdaConv = 1.E-5;
constexpr double kPresConv = 0.1;
// SprayUnits of either coupling, for the FP64 kernels: PELEC = false is the
// PeleLMeX branch above (MKS at the interface), PELEC = true the PeleC branch
// (CGS throughout, every factor 1; SprayFuelData.H:55-64)
template <bool PELEC>
struct Units {
  static constexpr double ru = PELEC ? 1. : kRuConv;
  static constexpr double eng = PELEC ? 1. : kEngConv;
  static constexpr double mass = PELEC ? 1. : kMassConv;
  static constexpr double rhod = PELEC ? 1. : kRhodConv;
  static constexpr double mu = PELEC ? 1. : kMuConv;
  static constexpr double lambda = PELEC ? 1. : kLambdaConv;
  static constexpr double pres = PELEC ? 1. : kPresConv;
};
constexpr double kRuCgs = 8.31446261815324e7;
constexpr double kPatmCgs = 1013250.0;

// Species in the caller's (mechanism) order.
struct DevMech {
  double mw_kg[kMaxSpec];            // kg/mol (gpv.mw after mass_conv)
  double mw_g[kMaxSpec];             // g/mol (the transport model's W)
  double ru_w[kMaxSpec];             // RU_cgs / W_gmol
  double cp[kMaxSpec][5];            // cp/R polynomial
  double hc[kMaxSpec][6];            // h/(RT) polynomial + a5
  double mu[kMaxSpec][4];            // ln mu(lnT), CGS
  double lam[kMaxSpec][4];           // ln lambda(lnT), CGS
  double dbin[kMaxFuel][kMaxSpec][4];// ln(P D_{indx[f],j})(lnT), fuel rows
};

struct DevFuel {
  double critT[kMaxFuel];
  double boilT[kMaxFuel];
  double cp[kMaxFuel];
  double latent[kMaxFuel];
  double ref_latent[kMaxFuel];
  double psat_coef[4 * kMaxFuel];
  double rho_coef[4 * kMaxFuel];
  double hboil_ref[kMaxFuel];  // ref_latent * ((critT-ref_T)/(critT-boilT))^-0.38
  int indx[kMaxFuel];          // gas species of fuel f
  int dep[kMaxFuel];           // deposit species of fuel f
  double ln10;                 // pmp_log(10.), as pmp_pow(10., y) uses it
  double ref_T;
  double dtmod;
  double body_force[3];
  int mass_trans;
  int mom_trans;
  int fixed_parts;
};

// FP32 copies of the tables for the mixed-precision and learned forms
// (converted once on the host; scaled where the physics always scales them)
// FP32 tables of the mixed and learned forms.  Species are stored in the
// order spec_perm of KParams: when every fuel deposits into its own gas
// species (dep_indx == indx), the fuels' gas species come first (fuel f is
// species f), so that the kernels index them at compile time (fuel_first).
struct DevMechF {
  float mw_kg[kMaxSpec];
  float inv_mw_kg[kMaxSpec];
  float inv_mw_g[kMaxSpec];
  float mw_g[kMaxSpec];
  float ru_w_eng[kMaxSpec];          // RU/W * eng_conv
  float cp[kMaxSpec][5];
  float hc[kMaxSpec][6];
  float mu6[kMaxSpec][4];            // 6 ln mu(lnT)
  float lam4[kMaxSpec][4];           // ln lambda(lnT) / 4
  float dbinm[kMaxFuel][kMaxSpec][4];// -ln(P D)(lnT)
};

struct DevFuelF {
  float cp[kMaxFuel];
  float latent[kMaxFuel];
  float boilT[kMaxFuel];
  float inv_boilT[kMaxFuel];
  float critT[kMaxFuel];
  float hb[kMaxFuel];        // RU / (Hboil_ref * W_fuel)
  float psat_a[kMaxFuel];
  float psat_b[kMaxFuel];
  float psat_c[kMaxFuel];
  float psat_d[kMaxFuel];
  float ref_T;
  float body_force[3];
};

struct BoxEntry {
  const double* st;          // state fab, component 0
  double* sr;                // source fab, component 0
  int st_lo[3];
  int sr_lo[3];
  long long st_js, st_ks, st_ns;
  long long sr_js, sr_ks, sr_ns;
  int state_lo[3], state_hi[3];   // tilebox grown by state_ghosts
  int src_lo[3], src_hi[3];       // tilebox grown by source_ghosts
  int sr_alo[3], sr_ahi[3];       // allocated bounds of the source view
  int at_bounds;
  int pad;
  long long p_begin, p_end;       // droplet slots of this box
  // the strides again as 32-bit ints (every view is checked to span fewer
  // than 2^31 elements), for cheaper index arithmetic in the update kernels
  int st_j32, st_k32, st_n32;
  int sr_j32, sr_k32, sr_n32;
  // FP32 gas records of the grown box (mixed and learned forms, written by
  // k_gas_records before the update): gas_rec4<NS>() float4 per cell,
  // {rho, T, u, v}, {w, Y_0, Y_1, Y_2}, {Y_3, ...}, mass fractions in the
  // FP32 tables' species order; cell (i, j, k) is record
  // (k - state_lo[2]) * gr_k + (j - state_lo[1]) * gr_j + (i - state_lo[0])
  float4* gr;
  int gr_j, gr_k;
  // FP64 gas records of the grown box (FP64 form; same cell order): per cell
  // gas_rec2<NS>() double2 {rho, T}, {u, v}, {w, Y_0}, ... (mechanism order),
  // holding exactly the per-cell terms the gather weights: rho, the cell's T
  // (PeleC: from its energy), the velocity and Y = (rho Y) * (1 / rho); null
  // when the FP64 kernel gathers the state planes itself (fallback list,
  // allocation-free entry point)
  double2* gr64;
};

// Place of cell (c0, c1, c2) (>= 0, relative to a corner of a region ex x ey
// x .. cells wide) in the droplets' sort order: x-fastest cells by default;
// with PMP_SORT_BRICKS, bricks of 2 x 2 x 2 cells, bricks x fastest, cells
// within a brick x fastest.  In the brick order the 128 consecutive droplets
// a CTA takes (about 17 cells at 7-8 droplets per cell) cover a compact
// block of cells whose 8-cell stencils fit the shared-memory gather tile;
// the row order spreads them along a row (and a quarter of the CTAs over two
// rows).
// The brick order goes with the gather tile (a build option): measured alone,
// the row order is 2 % faster for the mixed form on config 2 (7.49e9 vs
// 7.34e9 droplet-substeps/s), its gathers hitting L1 more often.
#ifndef PMP_SORT_BRICKS
#define PMP_SORT_BRICKS PMP_GATHER_TILE
#endif
__host__ __device__ inline unsigned long long brick_key(int c0, int c1, int c2, int ex, int ey)
{
#if !PMP_SORT_BRICKS
  // the plain x-fastest cell order (build option)
  return ((unsigned long long)c2 * (unsigned long long)ey + (unsigned long long)c1) * (unsigned long long)ex +
         (unsigned long long)c0;
#endif
  const unsigned long long nbx = (unsigned long long)((ex + 1) >> 1);
  const unsigned long long nby = (unsigned long long)((ey + 1) >> 1);
  const unsigned long long brick = ((unsigned long long)(c2 >> 1) * nby + (unsigned long long)(c1 >> 1)) * nbx +
                                   (unsigned long long)(c0 >> 1);
  return brick * 8ULL + (unsigned long long)(((c2 & 1) * 2 + (c1 & 1)) * 2 + (c0 & 1));
}
// keys brick_key can return for a region of ex x ey x ez cells
__host__ __device__ inline unsigned long long brick_key_count(int ex, int ey, int ez)
{
  return (unsigned long long)((ex + 1) >> 1) * (unsigned long long)((ey + 1) >> 1) *
         (unsigned long long)((ez + 1) >> 1) * 8ULL;
}

// float4 records per cell of the FP32 gas records: rho, T, velocity, Y
__host__ __device__ constexpr int gas_rec4(int ns) { return (8 + ns) / 4; }
// double2 records per cell of the FP64 gas records
__host__ __device__ constexpr int gas_rec2(int ns) { return (6 + ns) / 2; }

#ifdef __CUDACC__
// Deposit into a source cell: a relaxed device-scope FP64 add with no return
// value (red), so the issuing warp never waits for it.
__device__ __forceinline__ void red_add(double* p, double v)
{
  asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// FP64 gas record of cell (i, j, k) of box B (inside its grown box), as 2 * R2 doubles.
template <int R2>
__device__ __forceinline__ void load_gas_rec64(const BoxEntry& B, int i, int j, int k, double* rec)
{
  const double2* r = B.gr64 + ((k - B.state_lo[2]) * B.gr_k + (j - B.state_lo[1]) * B.gr_j + (i - B.state_lo[0])) * R2;
#pragma unroll
  for (int m = 0; m < R2; ++m) {
    const double2 v = __ldg(r + m);
    rec[2 * m] = v.x;
    rec[2 * m + 1] = v.y;
  }
}

// Gas record of cell (i, j, k) of box B (inside its grown box), as 4 * R4 floats.
template <int R4>
__device__ __forceinline__ void load_gas_rec(const BoxEntry& B, int i, int j, int k, float* rec)
{
  const float4* r = B.gr + ((k - B.state_lo[2]) * B.gr_k + (j - B.state_lo[1]) * B.gr_j + (i - B.state_lo[0])) * R4;
#pragma unroll
  for (int m = 0; m < R4; ++m) {
    const float4 v = __ldg(r + m);
    rec[4 * m] = v.x;
    rec[4 * m + 1] = v.y;
    rec[4 * m + 2] = v.z;
    rec[4 * m + 3] = v.w;
  }
}
#endif

// Device status block of a handle.  Update calls are stream-ordered and do
// not wait for one another: code/box/slot (the first error, sticky) and the
// counters accumulate over every call since the host last read and cleared
// the block (pmp_spray_sync); fb_count alone is per call (the length of the
// call's FP64 fallback list, reset by each call before its kernels).
// The update kernels' counters (droplet-substeps, kills, inner sub-steps),
// spread over PMP_CTR_SLOTS 32-byte slots: each warp adds its sums to the
// slot of its CTA, so that the ~3 adds per warp of a 16M-droplet launch do
// not all queue at one L2 address; the host adds the slots up.
#ifndef PMP_CTR_SLOTS
#define PMP_CTR_SLOTS 64
#endif
struct alignas(32) CtrSlot {
  unsigned long long substeps;
  unsigned long long killed;
  unsigned long long inner;
  unsigned long long pad;
};

struct DevStatus {
  int code;
  int box;
  long long slot;
  // the fallback lists' counters (adds from the gate and the selection of
  // small droplets) on a line apart from the error word as well
  alignas(128) unsigned long long fallback;
  unsigned long long fb_count;
  // learned form: droplets its gate rejects, listed from the end of the
  // fallback list (per call, reset with fb_count)
  unsigned long long fb_gate;
  // the counters start on a cache line of their own: every CTA reads `code`
  // when it starts, which must not queue behind the warps' adds
  alignas(128) CtrSlot ctr[PMP_CTR_SLOTS];
};

// The counters of a status read back to the host, summed over the slots.
inline void status_counters(const DevStatus& st, long long& substeps, long long& killed, long long& inner)
{
  substeps = killed = inner = 0;
  for (int i = 0; i < PMP_CTR_SLOTS; ++i) {
    substeps += (long long)st.ctr[i].substeps;
    killed += (long long)st.ctr[i].killed;
    inner += (long long)st.ctr[i].inner;
  }
}

// SoA droplet store: ncomp double arrays of length cap, then ids.
struct DevParts {
  double* pos[3];
  double* rd[PMP_MAX_RCOMP];
  int* id;
};

struct KParams {
  DevMech m;
  DevFuel f;
  DevMechF mf;
  DevFuelF ff;
  DevParts parts;
  // geometry
  double plo[3], phi[3], dx[3], dxi[3];
  double inv_vol;
  int bndry_lo[3], bndry_hi[3];
  // state / source component offsets (caller's mesh layout)
  int c_rho, c_mom, c_T, c_spec;
  int s_rho, s_mom, s_eng, s_spec;
  // call settings
  double flow_dt, sub_dt;
  double cur_coef;  // deposit factor -(1/V) sub_dt / flow_dt (SprayParticles.cpp:419-421), set on the host
  double inv_dtf;   // 1 / (dtmod sub_dt): the FP32 forms' mass-source factor, set on the host
  int num_iter, do_move, is_ghost, nboxes;
  long long nslots;  // droplet slots in the store (bound of the start-of-CTA prefetch; 0: none)
  const BoxEntry* boxes;
  const int* cta_box;
  const long long* cta_start;
  const long long* box_begin;  // nboxes + 1 slot offsets
  long long* fb_list;          // slots handed to the FP64 fallback kernel
  DevStatus* status;
  // page-locked, device-mapped host word: the first error code is also
  // written here, so the host sees a failed call without synchronising
  int* err_host;
  // PeleC coupling (FP64 form only): energy component of the state
  int pelec, c_eng;
  // fallback-list kernel: when list_nbox > 0, only the entries of boxes
  // [list_box0, list_box0 + list_nbox) (one stage of the host-view pipeline)
  int list_box0, list_nbox;
  // mixed and learned forms: the droplets below 2 um were listed before the
  // launch (k_select_small); the update kernel skips them without listing them
  int fb_pre;
  // fallback-list kernel: list_back = 1 runs the learned form's gate
  // rejections, fb_list[fb_cap - 1 - i] for i < fb_gate, instead of
  // fb_list[i] for i < fb_count
  int list_back;
  long long fb_cap;
  // mixed form: the diameter below which a droplet takes the FP64 path, 2 um
  // in the coupling's length unit
  double mixed_min_dia;
  // mixed / learned forms: species k of DevMechF (and of their gas-state
  // gather) is mechanism species spec_perm[k]; fuel_first as in DevMechF
  int spec_perm[kMaxSpec];
  int fuel_first;
};

}  // namespace pmp
