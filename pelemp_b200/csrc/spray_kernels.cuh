// spray_kernels.cuh -- the droplet driver loop and the update kernels.
//
// update_one<NS, NF, FORM> is the body of the device lambda of
// SprayParticleContainer::updateParticles (SprayParticles.cpp:324-481) for
// one droplet slot: cell location, bounds check, and per sub-cycle the
// trilinear gather (SprayInterpolation.H:99-199), GasPhaseVals::define,
// calcBoilT (SprayFuelData.H:178-200), the droplet physics of the chosen form
// (spray_source_fp64 or spray_source_mixed), the atomic scatter into the cell
// holding the droplet (SprayParticles.cpp:419-441) and the move with wall
// handling (SprayParticles.cpp:444-479).
//
// Cell indices and positions are formed with explicit round-to-nearest
// intrinsics, so they are bit-exact whatever the translation unit's
// contraction setting.
//
// Kernels
//  - spray_update_fp64<NS,NF,BLOCK>: plain FP64, one thread per droplet, CTA
//    -> (box, first slot) from the work map;
//  - spray_update_mixed<NS,NF,BLOCK,FF>: mixed precision; droplets entering the
//    call with d < 2 um are appended to the fallback list instead;
//  - spray_update_fp64_list<NS,NF,BLOCK>: plain FP64 over the fallback list
//    (grid-stride; the list length is read on the device).
#pragma once

#include "spray_fp64.cuh"
#include "spray_mixed.cuh"

namespace pmp {

enum class Form { FP64 = 0, MIXED = 1 };

// per-thread counts (32-bit: a thread's own counts stay far below 2^32)
struct Counters {
  unsigned sub = 0;
  unsigned killed = 0;
  unsigned inner = 0;
};

// Off by default: on config 2 the staging (the CTA's stencil box, about 9x
// the cells its droplets hold) and its barriers add more instructions than
// the L1/L2 gather latency it removes in these issue-bound kernels (mixed
// form 7.40e9 -> 7.05e9 droplet-substeps/s, FP64 2.26e9 -> 2.13e9).
#ifndef PMP_GATHER_TILE
#define PMP_GATHER_TILE 0
#endif

// The gas records (BoxEntry::gr or gr64, R 16-byte words per cell) of the
// cells that a CTA's 8-cell stencils cover when the call starts, copied into
// shared memory once per call: the state does not change during a call, so
// every sub-cycle's gather whose stencil lies inside the tile reads it there
// (cell-sorted droplets share their stencils) instead of through L1/L2.
// Stencils that leave it (a droplet that moved across a cell face) read the
// records in global memory as before.
template <typename Rec>
struct CellTile {
  int lo[3], hi[3];  // cells covered, inclusive (state index space)
  int nx, nxy;
  int on;            // 0: the CTA's stencils span more than the tile's capacity
  Rec* rec;          // R records per cell, x fastest
};

// Stage the tile: every thread of the CTA calls it (BLOCK threads), with its
// droplet slot s when it holds one.  CAP: capacity in cells.
template <int R, int CAP, int BLOCK, typename Rec>
__device__ __forceinline__ void stage_tile(const KParams& P, const DevParts& D, const BoxEntry& B, long long s,
                                           bool holds, const Rec* grec, CellTile<Rec>& T, Rec* buf)
{
  __shared__ int wred[6][BLOCK / 32];
  int v[6];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    v[d] = 0x7fffffff;
    v[3 + d] = 0x7fffffff;
  }
  if (holds && D.id[s] > 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double l = __dadd_rn(__dmul_rn(__dsub_rn(D.pos[d][s], P.plo[d]), P.dxi[d]), 0.5);
      // stencil cells ijk - 1 and ijk (upper cell centre); clamped so that
      // a droplet far outside cannot overflow the arithmetic
      const int ijk = max(-(1 << 24), min(1 << 24, static_cast<int>(floor(l))));
      v[d] = ijk - 1;
      v[3 + d] = -ijk;
    }
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    v[i] = __reduce_min_sync(0xffffffffu, v[i]);
  }
  const int warp = threadIdx.x / 32;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      wred[i][warp] = v[i];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int m[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      m[i] = wred[i][0];
      for (int w = 1; w < BLOCK / 32; ++w) {
        m[i] = min(m[i], wred[i][w]);
      }
    }
    long long vol = 1;
    for (int d = 0; d < 3; ++d) {
      T.lo[d] = max(m[d], B.state_lo[d]);
      T.hi[d] = m[3 + d] == 0x7fffffff ? T.lo[d] - 1 : min(-m[3 + d], B.state_hi[d]);
      vol *= (long long)max(T.hi[d] - T.lo[d] + 1, 0);
    }
    T.nx = T.hi[0] - T.lo[0] + 1;
    T.nxy = T.nx * (T.hi[1] - T.lo[1] + 1);
    T.on = vol > 0 && vol <= CAP;
    T.rec = buf;
  }
  __syncthreads();
  if (T.on) {
    const int nx = T.nx;
    const int ny = T.nxy / nx;
    const int n = T.nxy * (T.hi[2] - T.lo[2] + 1) * R;
    for (int c = threadIdx.x; c < n; c += BLOCK) {
      const int cell = c / R;
      const int w = c - cell * R;
      const int i = cell % nx;
      const int t = cell / nx;
      const int j = t % ny;
      const int k = t / ny;
      const int g = (k + T.lo[2] - B.state_lo[2]) * B.gr_k + (j + T.lo[1] - B.state_lo[1]) * B.gr_j +
                    (i + T.lo[0] - B.state_lo[0]);
      buf[c] = grec[g * R + w];
    }
  }
  __syncthreads();
}

// Index in the tile of stencil corner (ijk - 1), or -1 when the stencil
// ijk - 1 .. ijk is not inside it.
template <typename Rec>
__device__ __forceinline__ int tile_base(const CellTile<Rec>* T, const int* ijk)
{
  if (!T || !T->on) {
    return -1;
  }
  bool in = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    in = in && ijk[d] - 1 >= T->lo[d] && ijk[d] <= T->hi[d];
  }
  return in ? (ijk[2] - 1 - T->lo[2]) * T->nxy + (ijk[1] - 1 - T->lo[1]) * T->nx + (ijk[0] - 1 - T->lo[0]) : -1;
}

__device__ __forceinline__ void cell_of(const KParams& P, const double* pos, double* lx, int* ijk, int* ijkc)
{
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double l = __dmul_rn(__dsub_rn(pos[d], P.plo[d]), P.dxi[d]);
    lx[d] = __dadd_rn(l, 0.5);
    ijk[d] = static_cast<int>(floor(lx[d]));
    ijkc[d] = static_cast<int>(floor(l));
  }
}

// One droplet slot s of box b through the whole call.  D holds the droplet
// arrays (the library's packed SoA, or a caller's per-box arrays in the
// allocation-free entry point).  B is box b's entry: the kernel passes a copy
// in shared memory when the CTA works on one box (read at low latency,
// without re-deriving addresses), or the global entry otherwise.  A mixed-form
// droplet below 2 um is left to the fallback list.
// Droplet loads and stores of update_one: cache-streaming (evict-first: each
// droplet is read and written once per call), so that the mesh's gas records
// and source lines stay in L2 longer (measured +0.2-0.3 % on configs 2 and 5;
// PMP_STREAM_DROPLETS=0 for plain loads and stores).
#ifndef PMP_STREAM_DROPLETS
#define PMP_STREAM_DROPLETS 1
#endif
#if PMP_STREAM_DROPLETS
#define PMP_LDD(p) __ldcs(p)
#define PMP_STD(p, v) __stcs((p), (v))
#else
#define PMP_LDD(p) (*(p))
#define PMP_STD(p, v) (*(p) = (v))
#endif

template <int NS, int NF, Form FORM, bool FF = false, bool PELEC = false>
__device__ __forceinline__ void update_one(const KParams& P, const DevParts& D, const BoxEntry& B, int b,
                                           long long s, Counters& c, double* sx = nullptr, int sxs = 0,
                                           const CellTile<double2>* tile64 = nullptr,
                                           const CellTile<float4>* tile32 = nullptr)
{
  int id = PMP_LDD(&D.id[s]);
  if (!(id > 0)) {
    return;
  }
  double dia = PMP_LDD(&D.rd[PMP_PSTATE_DIA][s]);
  if (FORM == Form::MIXED && dia < P.mixed_min_dia) {
    if (!P.fb_pre) {
      push_fallback(P, s);
    }
    return;
  }
  double pos[3], vel[3], Y[NF];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pos[d] = PMP_LDD(&D.pos[d][s]);
    vel[d] = PMP_LDD(&D.rd[PMP_PSTATE_VEL + d][s]);
  }
  double T = PMP_LDD(&D.rd[PMP_PSTATE_T][s]);
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    Y[spf] = PMP_LDD(&D.rd[PMP_PSTATE_Y + spf][s]);
  }
  const double num_ppp = PMP_LDD(&D.rd[PMP_PSTATE_NUMDENS(NF)][s]);
  const double film = PMP_LDD(&D.rd[PMP_PSTATE_FILMHGHT(NF)][s]);
  int bflags[3] = {0, 0, 0};
  bool ok = true;
  if (B.at_bounds) {
    if (check_bounds(P, pos, bflags)) {
      set_error(P, PMP_ERR_LEFT_DOMAIN, b, s);
      ok = false;
    }
  }
  // a wall-film droplet stops the first sub-cycle (the film height never
  // changes here, so the check is made once)
  if (ok && P.num_iter > 0 && id > 0 && film > 0.) {
    set_error(P, PMP_ERR_UNSUPPORTED, b, s);
    ok = false;
  }
  for (int cur_iter = 0; ok && cur_iter < P.num_iter && id > 0; ++cur_iter) {
    // cell of the droplet, from its position at the start of the sub-cycle
    // (recomputed rather than carried, so that it is not live across the physics)
    double lx[3];
    int ijk[3], ijkc[3];
    cell_of(P, pos, lx, ijk, ijkc);
    if (sx) {
      // the position waits in shared memory across the droplet physics (sx:
      // this thread's slots, stride sxs), which does not read it: fewer
      // registers live there, fewer spills
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        sx[d * sxs] = pos[d];
      }
    }
    // trilinear_interp (SprayInterpolation.H:158-199)
    double ssv[2][3];
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      const double sx_hi = __dsub_rn(lx[dir], static_cast<double>(ijk[dir]));
      const double sx_lo = __dsub_rn(1., sx_hi);
      if (bflags[dir] > 1) {
        ssv[0][dir] = 1.;
        ssv[1][dir] = 0.;
      } else if (bflags[dir] < -1) {
        ssv[0][dir] = 0.;
        ssv[1][dir] = 1.;
      } else {
        ssv[0][dir] = sx_lo;
        ssv[1][dir] = sx_hi;
      }
    }
    // InterpolateGasPhase (SprayInterpolation.H:99-150), PeleLMeX branch, then
    // GasPhaseVals::define, calcBoilT and the droplet physics of the form
    SrcD<NF> src;
    int nsub = 0;
    bool state_ok = true;
    if (FORM == Form::FP64) {
      GasVals<NS, NF> gpv;
      gpv.rho = 0.;
      gpv.T = 0.;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        gpv.vel[d] = 0.;
        gpv.mom_src[d] = 0.;
      }
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        gpv.Y[n] = 0.;
      }
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        gpv.Ydot[spf] = 0.;
      }
      gpv.eng_src = 0.;
      gpv.mass_src = 0.;
      const int tb = tile_base(tile64, ijk);
#pragma unroll
      for (int kk = -1; kk < 1; ++kk) {
#pragma unroll
        for (int jj = -1; jj < 1; ++jj) {
#pragma unroll
          for (int ii = -1; ii < 1; ++ii) {
            const double cw = __dmul_rn(__dmul_rn(ssv[ii + 1][0], ssv[jj + 1][1]), ssv[kk + 1][2]);
            if (cw > 0.) {
              const int ci = ijk[0] + ii;
              const int cj = ijk[1] + jj;
              const int ck = ijk[2] + kk;
              if (!in_box(B.state_lo, B.state_hi, ci, cj, ck)) {
                state_ok = false;
              } else if (B.gr64) {
                // the cell's record holds the same per-cell terms the plane
                // gather below forms (k_gas_records64), so the sums are equal
                constexpr int R2 = gas_rec2(NS);
                double rec[2 * R2];
                if (tb >= 0) {
                  const double2* r = tile64->rec + (tb + (kk + 1) * tile64->nxy + (jj + 1) * tile64->nx + (ii + 1)) * R2;
#pragma unroll
                  for (int m = 0; m < R2; ++m) {
                    const double2 v = r[m];
                    rec[2 * m] = v.x;
                    rec[2 * m + 1] = v.y;
                  }
                } else {
                  load_gas_rec64<R2>(B, ci, cj, ck, rec);
                }
                gpv.rho = __dadd_rn(gpv.rho, __dmul_rn(cw, rec[0]));
#pragma unroll
                for (int n = 0; n < NS; ++n) {
                  gpv.Y[n] = __dadd_rn(gpv.Y[n], __dmul_rn(cw, rec[5 + n]));
                }
#pragma unroll
                for (int dir = 0; dir < 3; ++dir) {
                  gpv.vel[dir] = __dadd_rn(gpv.vel[dir], __dmul_rn(cw, rec[2 + dir]));
                }
                gpv.T = __dadd_rn(gpv.T, __dmul_rn(cw, rec[1]));
              } else {
                const double* q = B.st + ((ci - B.st_lo[0]) + (cj - B.st_lo[1]) * B.st_j32 + (ck - B.st_lo[2]) * B.st_k32);
                const double cur_rho = __ldg(q + P.c_rho * B.st_n32);
                gpv.rho = __dadd_rn(gpv.rho, __dmul_rn(cw, cur_rho));
                const double inv_rho = 1. / cur_rho;
                if (!PELEC) {
#pragma unroll
                  for (int n = 0; n < NS; ++n) {
                    const double cur_mf = __dmul_rn(__ldg(q + (P.c_spec + n) * B.st_n32), inv_rho);
                    gpv.Y[n] = __dadd_rn(gpv.Y[n], __dmul_rn(cw, cur_mf));
                  }
#pragma unroll
                  for (int dir = 0; dir < 3; ++dir) {
                    gpv.vel[dir] =
                      __dadd_rn(gpv.vel[dir], __dmul_rn(cw, __ldg(q + (P.c_mom + dir) * B.st_n32)));
                  }
                  gpv.T = __dadd_rn(gpv.T, __dmul_rn(cw, __ldg(q + P.c_T * B.st_n32)));
                } else {
                  // PeleC branch (SprayInterpolation.H:111-146): velocity from
                  // momentum, T from the internal energy (eos.EY2T, the cell's
                  // T as the guess)
                  double mass_frac[NS];
#pragma unroll
                  for (int n = 0; n < NS; ++n) {
                    const double cur_mf = __dmul_rn(__ldg(q + (P.c_spec + n) * B.st_n32), inv_rho);
                    gpv.Y[n] = __dadd_rn(gpv.Y[n], __dmul_rn(cw, cur_mf));
                    mass_frac[n] = cur_mf;
                  }
                  double ke = 0.;
#pragma unroll
                  for (int dir = 0; dir < 3; ++dir) {
                    const double vel = __dmul_rn(__ldg(q + (P.c_mom + dir) * B.st_n32), inv_rho);
                    gpv.vel[dir] = __dadd_rn(gpv.vel[dir], __dmul_rn(cw, vel));
                    ke = __dadd_rn(ke, __dmul_rn(vel, vel) / 2.);
                  }
                  const double intEng = __dsub_rn(__dmul_rn(__ldg(q + P.c_eng * B.st_n32), inv_rho), ke);
                  const double T_i = ey2t<NS>(P.m, intEng, mass_frac, __ldg(q + P.c_T * B.st_n32));
                  gpv.T = __dadd_rn(gpv.T, __dmul_rn(cw, T_i));
                }
              }
            }
          }
        }
      }
      if (!state_ok) {
        set_error(P, PMP_ERR_STATE_BOX, b, s);
        ok = false;
        break;
      }
      double mw_mix = 0.;
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        mw_mix = __dadd_rn(mw_mix, gpv.Y[n] / P.m.mw_kg[n]);
      }
      gpv.p = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(gpv.rho, kRuCgs), mw_mix), gpv.T), Units<PELEC>::ru);
      gpv.mw_mix = 1. / mw_mix;
      double cBoilT[NF];
      {
        const double RU = kRuCgs * Units<PELEC>::ru;
        const double PATM = kPatmCgs * Units<PELEC>::pres;
        const double lp = pmp_log(PATM / gpv.p);
#pragma unroll
        for (int spf = 0; spf < NF; ++spf) {
          const double mw_fuel = P.m.mw_kg[P.f.indx[spf]];
          const double cc = 1. / __dadd_rn(__dmul_rn(lp, RU) / (P.f.hboil_ref[spf] * mw_fuel), 1. / P.f.boilT[spf]);
          cBoilT[spf] = dmin(P.f.critT[spf], cc);
        }
      }
      nsub = spray_source_fp64<NS, NF, PELEC>(P, P.sub_dt, gpv, vel, T, dia, Y, num_ppp, id, cBoilT, sx, sxs);
      if (sx) {
        // the position and the cell it gives, back from shared memory
        const volatile double* vx = sx;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          pos[d] = vx[d * sxs];
        }
        cell_of(P, pos, lx, ijk, ijkc);
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        src.mom[d] = gpv.mom_src[d];
      }
      src.mass = gpv.mass_src;
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        src.Ydot[spf] = gpv.Ydot[spf];
      }
      src.eng = gpv.eng_src;
    } else {
      // FP32 gather of the cells' gas records (weights from the FP64 position)
      constexpr int R4 = gas_rec4(NS);
      float rho = 0.f, Tg = 0.f, vel_g[3] = {0.f, 0.f, 0.f}, Yg[NS];
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        Yg[n] = 0.f;
      }
      const int tb = tile_base(tile32, ijk);
      // FP32 weights from the FP64 factors; a corner is gathered when all
      // three factors are positive (the FP64 product's test, which FP32
      // products could underflow); one bounds check for the whole stencil,
      // per corner only when the stencil crosses the grown state box
      float wf[2][3];
#pragma unroll
      for (int dir = 0; dir < 3; ++dir) {
        wf[0][dir] = (float)ssv[0][dir];
        wf[1][dir] = (float)ssv[1][dir];
      }
      const bool stencil_in = in_box(B.state_lo, B.state_hi, ijk[0] - 1, ijk[1] - 1, ijk[2] - 1) &&
                              in_box(B.state_lo, B.state_hi, ijk[0], ijk[1], ijk[2]);
#pragma unroll
      for (int kk = -1; kk < 1; ++kk) {
#pragma unroll
        for (int jj = -1; jj < 1; ++jj) {
#pragma unroll
          for (int ii = -1; ii < 1; ++ii) {
            if (ssv[ii + 1][0] > 0. && ssv[jj + 1][1] > 0. && ssv[kk + 1][2] > 0.) {
              const int ci = ijk[0] + ii;
              const int cj = ijk[1] + jj;
              const int ck = ijk[2] + kk;
              if (!stencil_in && !in_box(B.state_lo, B.state_hi, ci, cj, ck)) {
                state_ok = false;
              } else {
                float rec[4 * R4];
                if (tb >= 0) {
                  const float4* r = tile32->rec + (tb + (kk + 1) * tile32->nxy + (jj + 1) * tile32->nx + (ii + 1)) * R4;
#pragma unroll
                  for (int m = 0; m < R4; ++m) {
                    const float4 v = r[m];
                    rec[4 * m] = v.x;
                    rec[4 * m + 1] = v.y;
                    rec[4 * m + 2] = v.z;
                    rec[4 * m + 3] = v.w;
                  }
                } else {
                  load_gas_rec<R4>(B, ci, cj, ck, rec);
                }
                const float w = wf[ii + 1][0] * wf[jj + 1][1] * wf[kk + 1][2];
                rho = fmaf(w, rec[0], rho);
                Tg = fmaf(w, rec[1], Tg);
#pragma unroll
                for (int dir = 0; dir < 3; ++dir) {
                  vel_g[dir] = fmaf(w, rec[2 + dir], vel_g[dir]);
                }
#pragma unroll
                for (int n = 0; n < NS; ++n) {
                  Yg[n] = fmaf(w, rec[5 + n], Yg[n]);
                }
              }
            }
          }
        }
      }
      if (!state_ok) {
        set_error(P, PMP_ERR_STATE_BOX, b, s);
        ok = false;
        break;
      }
      GasF<NS> g;
      g.rho = rho;
      g.T = Tg;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        g.vel[d] = vel_g[d];
      }
      float mwinv = 0.f;
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        g.Y[n] = Yg[n];
        mwinv = fmaf(g.Y[n], P.mf.inv_mw_kg[n], mwinv);
      }
      g.p = g.rho * (float)(kRuCgs * Units<PELEC>::ru) * mwinv * g.T;
      g.mw_mix = fdiv(1.f, mwinv);
      float cBoilT[NF];
      const float lp = flog(fdiv((float)(kPatmCgs * Units<PELEC>::pres), g.p));
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        cBoilT[spf] = fminf(P.ff.critT[spf], fdiv(1.f, fmaf(lp, P.ff.hb[spf], P.ff.inv_boilT[spf])));
      }
      nsub = spray_source_mixed<NS, NF, FF, PELEC>(P, P.sub_dt, g, cBoilT, vel, T, dia, Y, num_ppp, id, src, sx, sxs);
      {
        // the position and the cell it gives, back from shared memory
        const volatile double* vx = sx;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          pos[d] = vx[d * sxs];
        }
        cell_of(P, pos, lx, ijk, ijkc);
      }
    }
    c.sub += 1;
    c.inner += static_cast<unsigned>(nsub);
    // source scatter into the cell holding the droplet (SprayParticles.cpp:419-441)
    const double cur_coef = P.cur_coef;  // -(1/V) sub_dt / flow_dt, computed on the host
    if (!in_box(B.src_lo, B.src_hi, ijkc[0], ijkc[1], ijkc[2])) {
      if (!P.is_ghost || !in_box(B.sr_alo, B.sr_ahi, ijkc[0], ijkc[1], ijkc[2])) {
        set_error(P, PMP_ERR_SOURCE_BOX, b, s);
        ok = false;
        break;
      }
    }
    double* q = B.sr + ((ijkc[0] - B.sr_lo[0]) + (ijkc[1] - B.sr_lo[1]) * B.sr_j32 + (ijkc[2] - B.sr_lo[2]) * B.sr_k32);
    deposit<NF>(P, q, B.sr_n32, cur_coef, src.mom, src.mass, src.Ydot, src.eng);
    // move (SprayParticles.cpp:444-476)
    if (P.do_move && !P.f.fixed_parts && id > 0) {
#pragma unroll
      for (int dir = 0; dir < 3; ++dir) {
        pos[dir] = __dadd_rn(pos[dir], __dmul_rn(P.sub_dt, vel[dir]));
      }
      if (B.at_bounds) {
        if (check_bounds(P, pos, bflags)) {
          id = -1;
        } else {
          impose_wall(P, pos, vel, bflags);
        }
      }
    }
    if (P.is_ghost) {
      cell_of(P, pos, lx, ijk, ijkc);
      if (!in_box(B.src_lo, B.src_hi, ijkc[0], ijkc[1], ijkc[2])) {
        id = -1;
      }
    }
  }
  if (ok) {
    if (P.do_move) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        PMP_STD(&D.pos[d][s], pos[d]);
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      PMP_STD(&D.rd[PMP_PSTATE_VEL + d][s], vel[d]);
    }
    PMP_STD(&D.rd[PMP_PSTATE_T][s], T);
    PMP_STD(&D.rd[PMP_PSTATE_DIA][s], dia);
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      PMP_STD(&D.rd[PMP_PSTATE_Y + spf][s], Y[spf]);
    }
    if (id <= 0) {
      PMP_STD(&D.id[s], id);
      c.killed += 1;
    }
  }
}

// update_one over the library's packed droplet arrays
template <int NS, int NF, Form FORM, bool FF = false, bool PELEC = false>
__device__ __forceinline__ void update_one(const KParams& P, const BoxEntry& B, int b, long long s, Counters& c,
                                           double* sx = nullptr, int sxs = 0,
                                           const CellTile<double2>* tile64 = nullptr,
                                           const CellTile<float4>* tile32 = nullptr)
{
  update_one<NS, NF, FORM, FF, PELEC>(P, P.parts, B, b, s, c, sx, sxs, tile64, tile32);
}

__device__ __forceinline__ void flush_counters(const KParams& P, Counters& c)
{
  const unsigned mask = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    c.sub += __shfl_down_sync(mask, c.sub, o);
    c.killed += __shfl_down_sync(mask, c.killed, o);
    c.inner += __shfl_down_sync(mask, c.inner, o);
  }
  if ((threadIdx.x & 31) == 0 && (c.sub | c.killed | c.inner)) {
    CtrSlot& k = P.status->ctr[blockIdx.x % PMP_CTR_SLOTS];
    atomicAdd(&k.substeps, (unsigned long long)c.sub);
    if (c.killed) {
      atomicAdd(&k.killed, (unsigned long long)c.killed);
    }
    atomicAdd(&k.inner, (unsigned long long)c.inner);
  }
}

#ifndef PMP_FP64_MIN_BLOCKS
#define PMP_FP64_MIN_BLOCKS 5  /* 96 registers: 5 CTAs of 128 per SM (measured best) */
#endif
#ifndef PMP_MIXED_MIN_BLOCKS
#define PMP_MIXED_MIN_BLOCKS 7  /* 72 registers: 7 CTAs of 128 per SM (measured best against 6 and 8
                                   with the FP32 gas records and the shared-memory stash) */
#endif
#ifndef PMP_MIXED_MIN_BLOCKS_SMALL
#define PMP_MIXED_MIN_BLOCKS_SMALL 8  /* one fuel, <= 3 species: 64 registers, 8 CTAs per SM (config 5:
                                         +3 % against 7; the 5-species, 2-fuel kernel loses 7 % at 8) */
#endif
__host__ __device__ constexpr int mixed_min_blocks(int ns, int nf)
{
  return (nf == 1 && ns <= 3) ? PMP_MIXED_MIN_BLOCKS_SMALL : PMP_MIXED_MIN_BLOCKS;
}

// Copy box b's entry into shared memory (all threads of the CTA call it).
// Returns true, for the whole CTA, when a call of the handle failed since the
// host last cleared the status (cta_call_failed): the CTA then does nothing.
__device__ __forceinline__ bool stage_box(const KParams& P, int b, BoxEntry& sB)
{
  static_assert(sizeof(BoxEntry) % 4 == 0, "box entry copied as words");
  __shared__ int s_failed;
  if (threadIdx.x == 0) {
    s_failed = *reinterpret_cast<volatile const int*>(&P.status->code);
  }
  const int* src = reinterpret_cast<const int*>(P.boxes + b);
  int* dst = reinterpret_cast<int*>(&sB);
  for (int i = threadIdx.x; i < (int)(sizeof(BoxEntry) / 4); i += blockDim.x) {
    dst[i] = src[i];
  }
  __syncthreads();
  return s_failed != 0;
}

// Ask for the lines of slot s's droplet (L1) before the CTA waits for its
// box entry: their DRAM latency then overlaps the start of the CTA, whose
// droplet loads come after the barrier.
#ifndef PMP_PREFETCH_DROPLETS
#define PMP_PREFETCH_DROPLETS 1
#endif
__device__ __forceinline__ void prefetch_l1(const void* p)
{
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
template <int NF>
__device__ __forceinline__ void prefetch_droplet(const KParams& P, long long s)
{
#if PMP_PREFETCH_DROPLETS
  if (s < P.nslots) {
    const DevParts& D = P.parts;
    prefetch_l1(D.id + s);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      prefetch_l1(D.pos[d] + s);
      prefetch_l1(D.rd[PMP_PSTATE_VEL + d] + s);
    }
    prefetch_l1(D.rd[PMP_PSTATE_T] + s);
    prefetch_l1(D.rd[PMP_PSTATE_DIA] + s);
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      prefetch_l1(D.rd[PMP_PSTATE_Y + spf] + s);
    }
    prefetch_l1(D.rd[PMP_PSTATE_NUMDENS(NF)] + s);
    prefetch_l1(D.rd[PMP_PSTATE_FILMHGHT(NF)] + s);
  }
#endif
}

// capacities of the gather tiles, in cells: FP64 records (the FP64 forms,
// 5 CTAs per SM) and FP32 records (the mixed form, 7 CTAs per SM)
#ifndef PMP_TILE64_CELLS
#define PMP_TILE64_CELLS 192
#endif
#ifndef PMP_TILE32_CELLS
#define PMP_TILE32_CELLS 192
#endif

template <int NS, int NF, int BLOCK, bool PELEC>
__device__ __forceinline__ void fp64_cta(const KParams& P)
{
  __shared__ BoxEntry sB;
  const int b = P.cta_box[blockIdx.x];
  const long long s = P.cta_start[blockIdx.x] + threadIdx.x;
  prefetch_droplet<NF>(P, s);
  if (stage_box(P, b, sB)) {
    return;
  }
  Counters c;
  // per thread: position, parcel count, start mass, composition, across the
  // droplet physics (update_one, spray_source_fp64)
  __shared__ double stash[(5 + NF) * BLOCK];
  double* sx = stash + threadIdx.x;
#if PMP_GATHER_TILE
  constexpr int R2 = gas_rec2(NS);
  __shared__ CellTile<double2> tile;
  __shared__ double2 tile_rec[PMP_TILE64_CELLS * R2];
  const bool tiled = sB.gr64 != nullptr;
  if (tiled) {
    stage_tile<R2, PMP_TILE64_CELLS, BLOCK>(P, P.parts, sB, s, s < sB.p_end, sB.gr64, tile, tile_rec);
  }
  if (s < sB.p_end) {
    update_one<NS, NF, Form::FP64, false, PELEC>(P, sB, b, s, c, sx, BLOCK, tiled ? &tile : nullptr);
  }
#else
  if (s < sB.p_end) {
    update_one<NS, NF, Form::FP64, false, PELEC>(P, sB, b, s, c, sx, BLOCK);
  }
#endif
  flush_counters(P, c);
}

template <int NS, int NF, int BLOCK>
__global__ void __launch_bounds__(BLOCK, PMP_FP64_MIN_BLOCKS) spray_update_fp64(const __grid_constant__ KParams P)
{
  fp64_cta<NS, NF, BLOCK, false>(P);
}

// the PeleC coupling of the FP64 form
template <int NS, int NF, int BLOCK>
__global__ void __launch_bounds__(BLOCK, PMP_FP64_MIN_BLOCKS) spray_update_fp64_pelec(const __grid_constant__ KParams P)
{
  fp64_cta<NS, NF, BLOCK, true>(P);
}

template <int NS, int NF, int BLOCK, bool FF, bool PELEC = false>
__global__ void __launch_bounds__(BLOCK, mixed_min_blocks(NS, NF)) spray_update_mixed(const __grid_constant__ KParams P)
{
  __shared__ BoxEntry sB;
  const int b = P.cta_box[blockIdx.x];
  const long long s = P.cta_start[blockIdx.x] + threadIdx.x;
  prefetch_droplet<NF>(P, s);
  if (stage_box(P, b, sB)) {
    return;
  }
  Counters c;
  // per thread: position, parcel count, start mass, composition (update_one,
  // spray_source_mixed)
  __shared__ double stash[(5 + NF) * BLOCK];
  double* sx = stash + threadIdx.x;
#if PMP_GATHER_TILE
  constexpr int R4 = gas_rec4(NS);
  __shared__ CellTile<float4> tile;
  __shared__ float4 tile_rec[PMP_TILE32_CELLS * R4];
  stage_tile<R4, PMP_TILE32_CELLS, BLOCK>(P, P.parts, sB, s, s < sB.p_end, sB.gr, tile, tile_rec);
  if (s < sB.p_end) {
    update_one<NS, NF, Form::MIXED, FF, PELEC>(P, sB, b, s, c, sx, BLOCK, nullptr, &tile);
  }
#else
  if (s < sB.p_end) {
    update_one<NS, NF, Form::MIXED, FF, PELEC>(P, sB, b, s, c, sx, BLOCK);
  }
#endif
  flush_counters(P, c);
}

// box holding slot s (box_begin has nboxes + 1 entries)
__device__ __forceinline__ int box_of_slot(const KParams& P, long long s)
{
  int lo = 0;
  int hi = P.nboxes;
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (P.box_begin[mid] <= s) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  return lo;
}

// The droplets of slots [s0, s1) that the mixed kernel leaves to the FP64
// kernel (alive, d < 2 um at the call's start), appended to the fallback list
// before the mixed kernel runs, so that the FP64 list kernel can run beside it.
static __global__ void __launch_bounds__(256) k_select_small(const __grid_constant__ KParams P, long long s0, long long s1)
{
  for (long long s = s0 + (long long)blockIdx.x * 256 + threadIdx.x; s < s1; s += (long long)gridDim.x * 256) {
    if (P.parts.id[s] > 0 && P.parts.rd[PMP_PSTATE_DIA][s] < P.mixed_min_dia) {
      push_fallback(P, s);
    }
  }
}

// The FP32 gas records of boxes [b0, b0 + gridDim.y) (BoxEntry::gr), one
// thread per cell of the grown box, from the FP64 state: the mixed and
// learned updates then gather 2-3 16-byte records per stencil cell instead of
// 5 + NS FP64 planes, with rho*Y / rho divided once per cell.
template <int NS, bool PELEC = false>
__global__ void __launch_bounds__(256) k_gas_records(const __grid_constant__ KParams P, int b0)
{
  constexpr int R4 = gas_rec4(NS);
  const BoxEntry& B = P.boxes[b0 + blockIdx.y];
  const int nx = B.state_hi[0] - B.state_lo[0] + 1;
  const int ny = B.state_hi[1] - B.state_lo[1] + 1;
  const int nz = B.state_hi[2] - B.state_lo[2] + 1;
  const int n = nx * ny * nz;
  for (int c = blockIdx.x * 256 + threadIdx.x; c < n; c += gridDim.x * 256) {
    const int i = c % nx;
    const int t = c / nx;
    const int j = t % ny;
    const int k = t / ny;
    const double* q = B.st + ((i + B.state_lo[0] - B.st_lo[0]) + (j + B.state_lo[1] - B.st_lo[1]) * B.st_j32 +
                              (k + B.state_lo[2] - B.st_lo[2]) * B.st_k32);
    const double rho = __ldg(q + P.c_rho * B.st_n32);
    float v[4 * R4];
    v[0] = (float)rho;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      v[5 + s] = (float)(__ldg(q + (P.c_spec + P.spec_perm[s]) * B.st_n32) / rho);
    }
    if (!PELEC) {
      v[1] = (float)__ldg(q + P.c_T * B.st_n32);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        v[2 + d] = (float)__ldg(q + (P.c_mom + d) * B.st_n32);
      }
    } else {
      // velocity from momentum, T from the internal energy (FP64, as the
      // FP64 records), mass fractions in mechanism order for the inversion
      const double inv_rho = 1. / rho;
      double Yc[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        Yc[s] = __ldg(q + (P.c_spec + s) * B.st_n32) * inv_rho;
      }
      double ke = 0.;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double u = __ldg(q + (P.c_mom + d) * B.st_n32) * inv_rho;
        v[2 + d] = (float)u;
        ke += 0.5 * u * u;
      }
      const double e = __ldg(q + P.c_eng * B.st_n32) * inv_rho - ke;
      v[1] = (float)ey2t<NS>(P.m, e, Yc, __ldg(q + P.c_T * B.st_n32));
    }
#pragma unroll
    for (int s = 5 + NS; s < 4 * R4; ++s) {
      v[s] = 0.f;
    }
    float4* r = B.gr + (long long)c * R4;
#pragma unroll
    for (int m = 0; m < R4; ++m) {
      r[m] = make_float4(v[4 * m], v[4 * m + 1], v[4 * m + 2], v[4 * m + 3]);
    }
  }
}

// The FP64 gas records of boxes [b0, b0 + gridDim.y) (BoxEntry::gr64): per
// cell of the grown box, rho, T, the velocity and the mass fractions formed
// with exactly the operations of update_one's plane gather (PeleC: velocity
// from momentum, T by EY2T from the cell's energy with its T as the guess),
// so that the gathered sums are bit-identical.  Each cell is then converted
// once per call instead of once per droplet and stencil corner (the PeleC
// EOS inversion and the 1 / rho division included).
template <int NS, bool PELEC>
__global__ void __launch_bounds__(256) k_gas_records64(const __grid_constant__ KParams P, int b0)
{
  constexpr int R2 = gas_rec2(NS);
  const BoxEntry& B = P.boxes[b0 + blockIdx.y];
  const int nx = B.state_hi[0] - B.state_lo[0] + 1;
  const int ny = B.state_hi[1] - B.state_lo[1] + 1;
  const int nz = B.state_hi[2] - B.state_lo[2] + 1;
  const int n = nx * ny * nz;
  for (int c = blockIdx.x * 256 + threadIdx.x; c < n; c += gridDim.x * 256) {
    const int i = c % nx;
    const int t = c / nx;
    const int j = t % ny;
    const int k = t / ny;
    const double* q = B.st + ((i + B.state_lo[0] - B.st_lo[0]) + (j + B.state_lo[1] - B.st_lo[1]) * B.st_j32 +
                              (k + B.state_lo[2] - B.st_lo[2]) * B.st_k32);
    const double cur_rho = __ldg(q + P.c_rho * B.st_n32);
    const double inv_rho = 1. / cur_rho;
    double v[2 * R2];
    v[0] = cur_rho;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      v[5 + s] = __dmul_rn(__ldg(q + (P.c_spec + s) * B.st_n32), inv_rho);
    }
    if (!PELEC) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        v[2 + d] = __ldg(q + (P.c_mom + d) * B.st_n32);
      }
      v[1] = __ldg(q + P.c_T * B.st_n32);
    } else {
      double ke = 0.;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double vel = __dmul_rn(__ldg(q + (P.c_mom + d) * B.st_n32), inv_rho);
        v[2 + d] = vel;
        ke = __dadd_rn(ke, __dmul_rn(vel, vel) / 2.);
      }
      const double intEng = __dsub_rn(__dmul_rn(__ldg(q + P.c_eng * B.st_n32), inv_rho), ke);
      v[1] = ey2t<NS>(P.m, intEng, v + 5, __ldg(q + P.c_T * B.st_n32));
    }
#pragma unroll
    for (int s = 5 + NS; s < 2 * R2; ++s) {
      v[s] = 0.;
    }
    double2* r = B.gr64 + (long long)c * R2;
#pragma unroll
    for (int m = 0; m < R2; ++m) {
      r[m] = make_double2(v[2 * m], v[2 * m + 1]);
    }
  }
}

template <int NS, int NF, int BLOCK, bool PELEC = false>
__global__ void __launch_bounds__(BLOCK, PMP_FP64_MIN_BLOCKS) spray_update_fp64_list(const __grid_constant__ KParams P)
{
  if (cta_call_failed(P)) {
    return;
  }
  const unsigned long long n =
    *reinterpret_cast<volatile unsigned long long*>(P.list_back ? &P.status->fb_gate : &P.status->fb_count);
  Counters c;
  for (unsigned long long i = blockIdx.x * (unsigned long long)BLOCK + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * BLOCK) {
    const long long s = P.list_back ? P.fb_list[P.fb_cap - 1 - (long long)i] : P.fb_list[i];
    const int b = box_of_slot(P, s);
    if (P.list_nbox > 0 && (b < P.list_box0 || b >= P.list_box0 + P.list_nbox)) {
      continue;
    }
    update_one<NS, NF, Form::FP64, false, PELEC>(P, P.boxes[b], b, s, c);
  }
  flush_counters(P, c);
}

}  // namespace pmp
