// pmp_static.cu -- pmp_spray_update_static: the plain FP64 update with no
// device allocation at all.
//
// Who needs it: hosts that hand every byte of device memory to their own
// pre-sized pool (an AMReX arena sized at start-up) or run a solver that
// forbids device allocations after initialisation, so that a cudaMalloc
// during the step would fail or is not allowed.  Such
// callers own the droplet arrays and the mesh views; this entry point runs
// the update on them in place and keeps its own working data (the per-box
// table, the CTA-to-box prefix and the status/counter block) in one
// file-scope device array of fixed size.
//
// Limits and rules
//  - at most PMP_STATIC_MAX_BOXES boxes per call (larger counts are
//    rejected with PMP_ERR_INVALID); the array is sizeof(StaticScratch)
//    (about 90 KB) and stays resident on every device that loads the
//    library until the process exits;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current and loads every kernel
//    of this entry point: with CUDA's lazy module loading (the default) that
//    first call is when the array and the kernels' code take device memory,
//    so make it at initialisation, before the host's pool reserves the
//    device's memory (or run with CUDA_MODULE_LOADING=EAGER);
//  - the call is synchronous (it waits for its kernel and reads the status
//    back) and cannot be captured into a CUDA graph: under an active stream
//    capture it returns PMP_ERR_INVALID;
//  - on a nonzero return the droplet arrays and the sources may be partly
//    updated (every droplet whose thread ran to the end was): restore or
//    discard them;
//  - every call reuses the same array: calls whose GPU work overlaps (two
//    streams, two host threads) race on it and must be serialised by the
//    caller;
//  - droplets are processed in the caller's order (no sort), so results per
//    droplet are the same bits as pmp_spray_update's, deposits differ only by
//    atomic ordering.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "phys/pmp_thermo.h"
#include "pmp_device.cuh"
#include "spray_kernels.cuh"

namespace {

constexpr int kStaticBlock = 128;

struct StaticBox {
  pmp::BoxEntry e;        // views and grown boxes (p_begin/p_end unused)
  pmp::DevParts parts;    // the caller's device arrays of this box
  long long n;            // droplets in the box
};

struct StaticScratch {
  pmp::DevStatus status;                      // zeroed before every launch
  int cta_prefix[PMP_STATIC_MAX_BOXES + 1];   // first CTA of each box
  StaticBox boxes[PMP_STATIC_MAX_BOXES];
};

constexpr size_t kScratchWords = (sizeof(StaticScratch) + 7) / 8;

// The working array shared by every call of pmp_spray_update_static.
static __device__ __align__(256) unsigned long long g_static_scratch[kScratchWords];

// Device address of g_static_scratch, looked up once per device.
constexpr int kMaxDevices = 64;
StaticScratch* g_scratch_ptr[kMaxDevices] = {nullptr};

int fail(pmp_error_info* err, int code, const char* msg, int box = -1, long long particle = -1)
{
  if (err) {
    memset(err, 0, sizeof(*err));
    err->code = code;
    err->box = box;
    err->particle = particle;
    snprintf(err->message, sizeof(err->message), "%s", msg);
  }
  return code;
}

// The FP64 update over per-box caller arrays: CTA -> box by a search of the
// prefix table in the scratch array, the box's entry and array pointers
// staged in shared memory, then the droplet body every FP64 launch of the
// library runs (update_one), so each droplet's result is the same bits as
// pmp_spray_update's.
template <int NS, int NF>
__global__ void __launch_bounds__(kStaticBlock, PMP_FP64_MIN_BLOCKS)
  spray_update_fp64_static(const __grid_constant__ pmp::KParams P, const StaticScratch* scr)
{
  using namespace pmp;
  __shared__ BoxEntry sB;
  __shared__ DevParts sD;
  __shared__ int s_box;
  __shared__ long long s_n;
  if (threadIdx.x == 0) {
    int lo = 0;
    int hi = P.nboxes;  // cta_prefix[lo] <= blockIdx.x < cta_prefix[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) / 2;
      if (scr->cta_prefix[mid] <= (int)blockIdx.x) {
        lo = mid;
      } else {
        hi = mid;
      }
    }
    s_box = lo;
    s_n = scr->boxes[lo].n;
  }
  __syncthreads();
  const int b = s_box;
  {
    static_assert(sizeof(BoxEntry) % 4 == 0 && sizeof(DevParts) % 4 == 0, "copied as words");
    const int* src_e = reinterpret_cast<const int*>(&scr->boxes[b].e);
    const int* src_d = reinterpret_cast<const int*>(&scr->boxes[b].parts);
    int* dst_e = reinterpret_cast<int*>(&sB);
    int* dst_d = reinterpret_cast<int*>(&sD);
    for (int i = threadIdx.x; i < (int)(sizeof(BoxEntry) / 4); i += kStaticBlock) {
      dst_e[i] = src_e[i];
    }
    for (int i = threadIdx.x; i < (int)(sizeof(DevParts) / 4); i += kStaticBlock) {
      dst_d[i] = src_d[i];
    }
  }
  __syncthreads();
  const long long s = (long long)(blockIdx.x - scr->cta_prefix[b]) * kStaticBlock + threadIdx.x;
  Counters c;
  if (s < s_n) {
    update_one<NS, NF, Form::FP64>(P, sD, sB, b, s, c);
  }
  flush_counters(P, c);
}

// Loads every instantiation of the kernel (CUDA loads a kernel's code on its
// first use when modules load lazily, and that load allocates device memory).
bool load_static_kernels()
{
  cudaFuncAttributes a;
  return cudaFuncGetAttributes(&a, spray_update_fp64_static<3, 1>) == cudaSuccess &&
         cudaFuncGetAttributes(&a, spray_update_fp64_static<5, 1>) == cudaSuccess &&
         cudaFuncGetAttributes(&a, spray_update_fp64_static<5, 2>) == cudaSuccess &&
         cudaFuncGetAttributes(&a, spray_update_fp64_static<4, 1>) == cudaSuccess &&
         cudaFuncGetAttributes(&a, spray_update_fp64_static<4, 2>) == cudaSuccess;
}

// elements a view spans, first to last
long long extent(const pmp_box_view& v)
{
  return (long long)(v.hi[0] - v.lo[0]) + (long long)(v.hi[1] - v.lo[1]) * v.jstride +
         (long long)(v.hi[2] - v.lo[2]) * v.kstride + (long long)(v.ncomp - 1) * v.nstride + 1;
}

bool covers(const pmp_box_view& v, const int* lo, const int* hi, int need)
{
  if (!v.p || v.ncomp < need) {
    return false;
  }
  for (int d = 0; d < 3; ++d) {
    if (lo[d] < v.lo[d] || hi[d] > v.hi[d]) {
      return false;
    }
  }
  return true;
}

int at_boundary(const pmp_box& b, const pmp_geometry& g)
{
  bool inside = true;
  for (int d = 0; d < 3; ++d) {
    if (b.lo[d] - 1 < g.domain_lo[d] || b.hi[d] + 1 > g.domain_hi[d]) {
      inside = false;
    }
  }
  if (inside) {
    return 0;
  }
  for (int d = 0; d < 3; ++d) {
    const bool lo_out = b.lo[d] - 1 < g.domain_lo[d];
    const bool hi_out = b.hi[d] + 1 > g.domain_hi[d];
    if ((lo_out && g.bndry_lo[d] != 0) || (hi_out && g.bndry_hi[d] != 0)) {
      return 1;
    }
  }
  return 0;
}

}  // namespace

extern "C" int pmp_spray_update_static(
  const pmp_spray_config* cfg, const pmp_spray_data* data, const pmp_spray_comps* comps,
  const pmp_geometry* geom, int nboxes, const pmp_box* boxes, const pmp_particles* parts,
  const pmp_box_view* state, const pmp_box_view* source, double flow_dt, double time,
  int state_ghosts, int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, void* stream, pmp_error_info* err)
{
  (void)time;
  (void)is_virt;
  if (!cfg || !data || !comps || !geom || nboxes < 0 || (nboxes > 0 && (!boxes || !parts || !state || !source))) {
    return fail(err, PMP_ERR_INVALID, "null argument");
  }
  if (nboxes > PMP_STATIC_MAX_BOXES) {
    return fail(err, PMP_ERR_INVALID, "pmp_spray_update_static takes at most PMP_STATIC_MAX_BOXES boxes");
  }
  if (cfg->nfuel < 1 || cfg->nfuel > PMP_MAX_FUEL || cfg->nspec < 1 || cfg->nspec > PMP_MAX_SPEC ||
      data->nfuel != cfg->nfuel || !(flow_dt > 0.)) {
    return fail(err, PMP_ERR_INVALID, "bad configuration");
  }
  if (data->do_breakup != 0 || data->do_splash) {
    return fail(err, PMP_ERR_UNSUPPORTED, "breakup and splash models are not supported");
  }
  const int NS = cfg->nspec;
  const int NF = cfg->nfuel;
  if (!((NS == 3 && NF == 1) || (NS == 5 && NF == 1) || (NS == 5 && NF == 2) || (NS == 4 && NF == 1) ||
        (NS == 4 && NF == 2))) {
    return fail(err, PMP_ERR_UNSUPPORTED, "no kernel for this species / fuel count");
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    return fail(err, PMP_ERR_NO_DEVICE, "no current CUDA device");
  }
  cudaStream_t st = (cudaStream_t)stream;
  {
    // synchronous (the status is read back before returning): not capturable
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
      return fail(err, PMP_ERR_INVALID, "pmp_spray_update_static is synchronous and cannot be captured");
    }
  }
  // one-time set-up on this device: the array's device address, and every
  // kernel instantiation loaded now (with lazy module loading both would
  // otherwise allocate device memory at their first use)
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) {
      return fail(err, PMP_ERR_CUDA, "cudaGetSymbolAddress of the static scratch array failed");
    }
    if (!load_static_kernels()) {
      return fail(err, PMP_ERR_CUDA, "loading the allocation-free kernels failed");
    }
    g_scratch_ptr[dev] = static_cast<StaticScratch*>(p);
  }
  StaticScratch* scr = g_scratch_ptr[dev];
  // mechanism and fuel tables (host only)
  int idx[PMP_MAX_SPEC];
  for (int k = 0; k < NS; ++k) {
    char name[PMP_NAME_LEN];
    memcpy(name, cfg->species[k], PMP_NAME_LEN);
    name[PMP_NAME_LEN - 1] = 0;
    idx[k] = pmp_db_lookup(name);
    if (idx[k] < 0) {
      return fail(err, PMP_ERR_INVALID, "unknown species");
    }
  }
  pmp_mech mech;
  if (pmp_mech_build(&mech, NS, idx) != 0) {
    return fail(err, PMP_ERR_INVALID, "bad mechanism");
  }
  pmp::KParams P;
  memset(&P, 0, sizeof(P));
  for (int f = 0; f < NF; ++f) {
    if (data->indx[f] < 0 || data->indx[f] >= NS || data->dep_indx[f] < 0 || data->dep_indx[f] >= NS) {
      return fail(err, PMP_ERR_INVALID, "fuel species index out of range");
    }
  }
  for (int k = 0; k < NS; ++k) {
    P.m.mw_g[k] = mech.mw[k];
    P.m.mw_kg[k] = mech.mw[k] * pmp::kMassConv;
    P.m.ru_w[k] = PMP_RU_CGS / mech.mw[k];
    for (int n = 0; n < 5; ++n) {
      P.m.cp[k][n] = mech.cp[k][n];
    }
    for (int n = 0; n < 6; ++n) {
      P.m.hc[k][n] = mech.hc[k][n];
    }
    for (int n = 0; n < 4; ++n) {
      P.m.mu[k][n] = mech.mu[k][n];
      P.m.lam[k][n] = mech.lam[k][n];
    }
  }
  for (int f = 0; f < NF; ++f) {
    for (int j = 0; j < NS; ++j) {
      for (int n = 0; n < 4; ++n) {
        P.m.dbin[f][j][n] = mech.dbin[data->indx[f]][j][n];
      }
    }
    P.f.critT[f] = data->critT[f];
    P.f.boilT[f] = data->boilT[f];
    P.f.cp[f] = data->cp[f];
    P.f.latent[f] = data->latent[f];
    P.f.ref_latent[f] = data->ref_latent[f];
    for (int c = 0; c < 4; ++c) {
      P.f.psat_coef[4 * f + c] = data->psat_coef[4 * f + c];
      P.f.rho_coef[4 * f + c] = data->rho_coef[4 * f + c];
    }
    P.f.hboil_ref[f] =
      data->ref_latent[f] * pmp_pow((data->critT[f] - data->ref_T) / (data->critT[f] - data->boilT[f]), -0.38);
    P.f.indx[f] = data->indx[f];
    P.f.dep[f] = data->dep_indx[f];
  }
  P.f.ln10 = pmp_log(10.);
  P.f.ref_T = data->ref_T;
  P.f.dtmod = data->dtmod;
  for (int i = 0; i < 3; ++i) {
    P.f.body_force[i] = data->body_force[i];
  }
  P.f.mass_trans = data->mass_trans;
  P.f.mom_trans = data->mom_trans;
  P.f.fixed_parts = data->fixed_parts;
  for (int d = 0; d < 3; ++d) {
    if (!(geom->dx[d] > 0.)) {
      return fail(err, PMP_ERR_INVALID, "bad geometry");
    }
    P.plo[d] = geom->plo[d];
    P.phi[d] = geom->phi[d];
    P.dx[d] = geom->dx[d];
    P.dxi[d] = 1. / geom->dx[d];
    P.bndry_lo[d] = geom->bndry_lo[d];
    P.bndry_hi[d] = geom->bndry_hi[d];
  }
  const double vol = geom->dx[0] * geom->dx[1] * geom->dx[2];
  P.inv_vol = 1. / vol;
  P.c_rho = comps->rhoIndx;
  P.c_mom = comps->momIndx;
  P.c_T = comps->utempIndx;
  P.c_spec = comps->specIndx;
  P.s_rho = comps->rhoSrcIndx;
  P.s_mom = comps->momSrcIndx;
  P.s_eng = comps->engSrcIndx;
  P.s_spec = comps->specSrcIndx;
  P.flow_dt = flow_dt;
  P.sub_dt = flow_dt;
  P.num_iter = 1;
  if (do_move && spray_cfl_lev > 0.5) {
    P.num_iter = static_cast<int>(std::ceil(spray_cfl_lev / 0.5));
    P.sub_dt = flow_dt / static_cast<double>(P.num_iter);
  }
  {
    // launch constants, the same IEEE operations the kernels did per droplet
    const double t = -P.inv_vol * P.sub_dt;
    P.cur_coef = t / P.flow_dt;
    P.inv_dtf = 1. / (P.f.dtmod * P.sub_dt);
  }
  P.do_move = do_move;
  P.is_ghost = is_ghost;
  P.nboxes = nboxes;
  P.status = &scr->status;  // device address inside the scratch array
  // per-box table, built on the host stack and copied into the array
  const int need_state = 1 + std::max(std::max(comps->rhoIndx, comps->momIndx + 2),
                                      std::max(comps->utempIndx, comps->specIndx + NS - 1));
  const int need_src = 1 + std::max(std::max(comps->rhoSrcIndx, comps->momSrcIndx + 2),
                                    std::max(comps->engSrcIndx, comps->specSrcIndx + NF - 1));
  static thread_local StaticBox h_boxes[PMP_STATIC_MAX_BOXES];
  static thread_local int h_prefix[PMP_STATIC_MAX_BOXES + 1];
  int ncta = 0;
  for (int b = 0; b < nboxes; ++b) {
    StaticBox& sb = h_boxes[b];
    memset(&sb, 0, sizeof(sb));
    pmp::BoxEntry& e = sb.e;
    for (int d = 0; d < 3; ++d) {
      e.state_lo[d] = boxes[b].lo[d] - state_ghosts;
      e.state_hi[d] = boxes[b].hi[d] + state_ghosts;
      e.src_lo[d] = boxes[b].lo[d] - source_ghosts;
      e.src_hi[d] = boxes[b].hi[d] + source_ghosts;
    }
    if (!covers(state[b], e.state_lo, e.state_hi, need_state)) {
      return fail(err, PMP_ERR_INVALID, "state view does not cover the grown box", b);
    }
    if (!covers(source[b], e.src_lo, e.src_hi, need_src)) {
      return fail(err, PMP_ERR_INVALID, "source view does not cover the grown box", b);
    }
    const pmp_particles& pp = parts[b];
    if (pp.layout != PMP_LAYOUT_SOA || pp.where != PMP_WHERE_DEVICE || pp.n < 0) {
      return fail(err, PMP_ERR_INVALID, "droplets must be device SoA arrays", b);
    }
    if (pp.n > 0) {
      for (int d = 0; d < 3; ++d) {
        if (!pp.pos[d]) {
          return fail(err, PMP_ERR_INVALID, "missing position array", b);
        }
      }
      for (int r = 0; r < PMP_PSTATE_NUM(NF); ++r) {
        if (!pp.rdata[r]) {
          return fail(err, PMP_ERR_INVALID, "missing real component array", b);
        }
      }
      if (!pp.id) {
        return fail(err, PMP_ERR_INVALID, "missing id array", b);
      }
    }
    e.st = state[b].p;
    e.sr = source[b].p;
    for (int d = 0; d < 3; ++d) {
      e.st_lo[d] = state[b].lo[d];
      e.sr_lo[d] = source[b].lo[d];
      e.sr_alo[d] = source[b].lo[d];
      e.sr_ahi[d] = source[b].hi[d];
    }
    e.st_js = state[b].jstride;
    e.st_ks = state[b].kstride;
    e.st_ns = state[b].nstride;
    e.sr_js = source[b].jstride;
    e.sr_ks = source[b].kstride;
    e.sr_ns = source[b].nstride;
    if (extent(state[b]) >= (1LL << 31) || extent(source[b]) >= (1LL << 31)) {
      return fail(err, PMP_ERR_INVALID, "a state or source view spans 2^31 elements or more", b);
    }
    e.st_j32 = (int)state[b].jstride;
    e.st_k32 = (int)state[b].kstride;
    e.st_n32 = (int)state[b].nstride;
    e.sr_j32 = (int)source[b].jstride;
    e.sr_k32 = (int)source[b].kstride;
    e.sr_n32 = (int)source[b].nstride;
    e.at_bounds = at_boundary(boxes[b], *geom);
    for (int d = 0; d < 3; ++d) {
      sb.parts.pos[d] = pp.pos[d];
    }
    for (int r = 0; r < PMP_PSTATE_NUM(NF); ++r) {
      sb.parts.rd[r] = pp.rdata[r];
    }
    sb.parts.id = pp.id;
    sb.n = pp.n;
    h_prefix[b] = ncta;
    const long long nb = (pp.n + kStaticBlock - 1) / kStaticBlock;
    if ((long long)ncta + nb > 0x7fffffffLL) {
      return fail(err, PMP_ERR_INVALID, "too many droplets for one launch", b);
    }
    ncta += (int)nb;
  }
  h_prefix[nboxes] = ncta;
  if (cudaMemcpyAsync(scr->boxes, h_boxes, sizeof(StaticBox) * nboxes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(scr->cta_prefix, h_prefix, sizeof(int) * (nboxes + 1), cudaMemcpyHostToDevice, st) !=
        cudaSuccess ||
      cudaMemsetAsync(&scr->status, 0, sizeof(pmp::DevStatus), st) != cudaSuccess) {
    return fail(err, PMP_ERR_CUDA, "copy into the static scratch array failed");
  }
  if (ncta > 0) {
#define PMP_STATIC_CASE(S, F)                                                   \
  if (NS == S && NF == F) {                                                     \
    spray_update_fp64_static<S, F><<<ncta, kStaticBlock, 0, st>>>(P, scr);      \
  }
    PMP_STATIC_CASE(3, 1)
    PMP_STATIC_CASE(5, 1)
    PMP_STATIC_CASE(5, 2)
    PMP_STATIC_CASE(4, 1)
    PMP_STATIC_CASE(4, 2)
#undef PMP_STATIC_CASE
    if (cudaGetLastError() != cudaSuccess) {
      return fail(err, PMP_ERR_CUDA, "launch failed");
    }
  }
  pmp::DevStatus hs;
  if (cudaMemcpyAsync(&hs, &scr->status, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    return fail(err, PMP_ERR_CUDA, "status read-back failed");
  }
  if (hs.code != 0) {
    static const char* names[] = {"ok", "droplet left the domain", "state box too small",
                                  "source box too small", "unsupported droplet state", "timeout"};
    return fail(err, hs.code, hs.code < 6 ? names[hs.code] : "error", hs.box, hs.slot);
  }
  if (err) {
    memset(err, 0, sizeof(*err));
    err->particle = -1;
  }
  return PMP_OK;
}
