// pmp_spray.cu -- implementation of the C ABI in include/pmp_spray.h.
//
// The handle replaces SprayParticleContainer's static state
// (Source/PP_Spray/SprayParticles.H:388-405) and its particle tiles.  Droplets
// handed in per box are copied to the device, sorted by the cell that holds
// them, and packed into one structure-of-arrays; the permutation back to the
// caller's order is kept.  pmp_spray_update is updateParticles
// (SprayParticles.cpp:142-502) for all boxes in one launch.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "phys/pmp_thermo.h"
#include "pmp_device.cuh"
#include "spray_kernels.cuh"

namespace pmp {
// pmp_mixed.cu
int launch_mixed(int ns, int nf, const KParams& P, int ncta, int block, cudaStream_t st);
// the mixed form's droplets below 2 um of slots [s0, s1) onto the fallback list
int launch_select_small(const KParams& P, long long s0, long long s1, cudaStream_t st);
// FP32 gas records (BoxEntry::gr) of boxes [b0, b0 + nb); max_cells = the
// largest grown box's cell count
int launch_gas_records(int ns, const KParams& P, int b0, int nb, int max_cells, cudaStream_t st);
}  // namespace pmp

using pmp::BoxEntry;
using pmp::DevStatus;
using pmp::KParams;

#include "pmp_handle.h"

using pmp::BoxStore;
using pmp::kBlock;
using pmp::kSortPad;

int pmp::set_err(pmp_spray* h, int code, const char* msg, int box, long long particle)
{
  if (h) {
    memset(&h->last_err, 0, sizeof(h->last_err));
    h->last_err.code = code;
    h->last_err.box = box;
    h->last_err.particle = particle;
    snprintf(h->last_err.message, sizeof(h->last_err.message), "%s", msg);
  }
  return code;
}

namespace {

using pmp::set_err;

#define PMP_CUDA(h, call)                                                   \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      char b_[160];                                                         \
      snprintf(b_, sizeof(b_), "%s: %s", #call, cudaGetErrorString(e_));    \
      return set_err((h), PMP_ERR_CUDA, b_);                                \
    }                                                                       \
  } while (0)

// --------------------------------------------------------------------------
// small data-movement kernels

__global__ void k_aos_to_soa(const char* aos, long long n, int nr, double* soa, int* ids)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const size_t rec = sizeof(double) * (3 + nr) + 2 * sizeof(int);
  const double* r = reinterpret_cast<const double*>(aos + i * rec);
  for (int c = 0; c < 3 + nr; ++c) {
    soa[c * n + i] = r[c];
  }
  ids[i] = *reinterpret_cast<const int*>(r + 3 + nr);
}

__global__ void k_soa_to_aos(const double* soa, const int* ids, long long n, int nr, char* aos)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const size_t rec = sizeof(double) * (3 + nr) + 2 * sizeof(int);
  double* r = reinterpret_cast<double*>(aos + i * rec);
  for (int c = 0; c < 3 + nr; ++c) {
    r[c] = soa[c * n + i];
  }
  int* ip = reinterpret_cast<int*>(r + 3 + nr);
  ip[0] = ids[i];
  ip[1] = 0;
}

__global__ void k_cell_keys(
  const double* x, const double* y, const double* z, long long n, double plo0, double plo1,
  double plo2, double dxi0, double dxi1, double dxi2, int lo0, int lo1, int lo2, int nx, int ny,
  int nz, unsigned* keys, long long* idx)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  int c[3];
  const double p[3] = {x[i], y[i], z[i]};
  const double pl[3] = {plo0, plo1, plo2};
  const double di[3] = {dxi0, dxi1, dxi2};
  const int lo[3] = {lo0, lo1, lo2};
  const int ext[3] = {nx, ny, nz};
  for (int d = 0; d < 3; ++d) {
    const double l = __dmul_rn(__dsub_rn(p[d], pl[d]), di[d]);
    int v = static_cast<int>(floor(l)) - lo[d] + kSortPad;
    v = v < 0 ? 0 : (v >= ext[d] ? ext[d] - 1 : v);
    c[d] = v;
  }
  keys[i] = (unsigned)pmp::brick_key(c[0], c[1], c[2], ext[0], ext[1]);
  idx[i] = i;
}

// dst[c][s] = src[c][perm[s]] for every component; ids likewise
__global__ void k_gather(
  const double* src, const int* sid, const long long* perm, long long n, int ncomp, double* dst,
  int* did)
{
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) {
    return;
  }
  const long long j = perm[s];
  for (int c = 0; c < ncomp; ++c) {
    dst[c * n + s] = src[c * n + j];
  }
  did[s] = sid[j];
}

// dst[c][perm[s]] = src[c * stride + s]: back to the caller's order
__global__ void k_unsort(
  const double* src, long long stride, const int* sid, const long long* perm, long long n, int ncomp,
  double* dst, int* did)
{
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) {
    return;
  }
  const long long j = perm[s];
  for (int c = 0; c < ncomp; ++c) {
    dst[c * n + j] = src[c * stride + s];
  }
  did[j] = sid[s];
}

inline unsigned nblk(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

// --------------------------------------------------------------------------
// handle helpers

void free_store(BoxStore& s)
{
  cudaFree(s.d);
  cudaFree(s.id);
  cudaFree(s.perm);
  s = BoxStore{};
}

void free_packed(pmp_spray* h)
{
  cudaFree(h->soa);
  cudaFree(h->ids);
  cudaFree(h->perm);
  cudaFree(h->d_cta_box);
  cudaFree(h->d_cta_start);
  cudaFree(h->d_box_begin);
  cudaFree(h->fb_list);
  cudaFree(h->soa_spare);
  cudaFree(h->ids_spare);
  h->soa_spare = nullptr;
  h->ids_spare = nullptr;
  h->spare_cap = 0;
  h->soa = nullptr;
  h->ids = nullptr;
  h->perm = nullptr;
  h->d_cta_box = nullptr;
  h->d_cta_start = nullptr;
  h->d_box_begin = nullptr;
  h->fb_list = nullptr;
  h->cta_cap = 0;
  h->packed = false;
  h->ncta = 0;
  pmp::batch_reset(h);
}

// DevMech (species in mechanism order) and DevFuel from the mechanism and
// SprayData.
int build_device_tables(pmp_spray* h)
{
  const pmp_spray_data& d = h->data;
  const int NF = h->nfuel;
  const int NS = h->nspec;
  for (int f = 0; f < NF; ++f) {
    if (d.indx[f] < 0 || d.indx[f] >= NS || d.dep_indx[f] < 0 || d.dep_indx[f] >= NS) {
      return set_err(h, PMP_ERR_INVALID, "fuel species index out of range");
    }
    for (int g = 0; g < f; ++g) {
      if (d.indx[g] == d.indx[f]) {
        return set_err(h, PMP_ERR_INVALID, "two fuels map to the same gas species");
      }
    }
  }
  pmp::DevMech& m = h->dmech;
  memset(&m, 0, sizeof(m));
  for (int k = 0; k < NS; ++k) {
    m.mw_g[k] = h->mech.mw[k];
    m.mw_kg[k] = h->mech.mw[k] * (h->pelec ? 1. : pmp::kMassConv);
    m.ru_w[k] = PMP_RU_CGS / h->mech.mw[k];
    for (int n = 0; n < 5; ++n) {
      m.cp[k][n] = h->mech.cp[k][n];
    }
    for (int n = 0; n < 6; ++n) {
      m.hc[k][n] = h->mech.hc[k][n];
    }
    for (int n = 0; n < 4; ++n) {
      m.mu[k][n] = h->mech.mu[k][n];
      m.lam[k][n] = h->mech.lam[k][n];
    }
  }
  for (int f = 0; f < NF; ++f) {
    for (int j = 0; j < NS; ++j) {
      for (int n = 0; n < 4; ++n) {
        m.dbin[f][j][n] = h->mech.dbin[d.indx[f]][j][n];
      }
    }
  }
  pmp::DevFuel& F = h->dfuel;
  memset(&F, 0, sizeof(F));
  for (int f = 0; f < NF; ++f) {
    F.critT[f] = d.critT[f];
    F.boilT[f] = d.boilT[f];
    F.cp[f] = d.cp[f];
    F.latent[f] = d.latent[f];
    F.ref_latent[f] = d.ref_latent[f];
    for (int c = 0; c < 4; ++c) {
      F.psat_coef[4 * f + c] = d.psat_coef[4 * f + c];
      F.rho_coef[4 * f + c] = d.rho_coef[4 * f + c];
    }
    // Hboil_ref of SprayData::calcBoilT (SprayFuelData.H:190-192): constant per fuel
    F.hboil_ref[f] =
      d.ref_latent[f] * pmp_pow((d.critT[f] - d.ref_T) / (d.critT[f] - d.boilT[f]), -0.38);
    F.indx[f] = d.indx[f];
    F.dep[f] = d.dep_indx[f];
  }
  F.ln10 = pmp_log(10.);
  F.ref_T = d.ref_T;
  F.dtmod = d.dtmod;
  for (int i = 0; i < 3; ++i) {
    F.body_force[i] = d.body_force[i];
  }
  F.mass_trans = d.mass_trans;
  F.mom_trans = d.mom_trans;
  F.fixed_parts = d.fixed_parts;
  // FP32 tables of the mixed / learned forms, fuels' species first when
  // every fuel deposits into its own species
  h->fuel_first = 1;
  for (int f = 0; f < NF; ++f) {
    h->fuel_first = h->fuel_first && d.dep_indx[f] == d.indx[f];
  }
  {
    int k = 0;
    if (h->fuel_first) {
      for (int f = 0; f < NF; ++f) {
        h->spec_perm[k++] = d.indx[f];
      }
    }
    for (int n = 0; n < NS; ++n) {
      bool fuel = false;
      for (int f = 0; f < NF; ++f) {
        fuel = fuel || (h->fuel_first && d.indx[f] == n);
      }
      if (!fuel) {
        h->spec_perm[k++] = n;
      }
    }
  }
  pmp::DevMechF& mf = h->dmechf;
  pmp::DevFuelF& ff = h->dfuelf;
  memset(&mf, 0, sizeof(mf));
  memset(&ff, 0, sizeof(ff));
  for (int k = 0; k < NS; ++k) {
    const int s = h->spec_perm[k];
    mf.mw_kg[k] = (float)m.mw_kg[s];
    mf.inv_mw_kg[k] = (float)(1. / m.mw_kg[s]);
    mf.inv_mw_g[k] = (float)(1. / m.mw_g[s]);
    mf.mw_g[k] = (float)m.mw_g[s];
    mf.ru_w_eng[k] = (float)(m.ru_w[s] * (h->pelec ? 1. : pmp::kEngConv));
    for (int n = 0; n < 5; ++n) {
      mf.cp[k][n] = (float)m.cp[s][n];
    }
    for (int n = 0; n < 6; ++n) {
      mf.hc[k][n] = (float)m.hc[s][n];
    }
    for (int n = 0; n < 4; ++n) {
      mf.mu6[k][n] = (float)(6. * m.mu[s][n]);
      mf.lam4[k][n] = (float)(0.25 * m.lam[s][n]);
    }
  }
  for (int f = 0; f < NF; ++f) {
    for (int j = 0; j < NS; ++j) {
      for (int n = 0; n < 4; ++n) {
        mf.dbinm[f][j][n] = (float)(-m.dbin[f][h->spec_perm[j]][n]);
      }
    }
    ff.cp[f] = (float)d.cp[f];
    ff.latent[f] = (float)d.latent[f];
    ff.boilT[f] = (float)d.boilT[f];
    ff.inv_boilT[f] = (float)(1. / d.boilT[f]);
    ff.critT[f] = (float)d.critT[f];
    ff.hb[f] = (float)(pmp::kRuCgs * (h->pelec ? 1. : pmp::kRuConv) / (F.hboil_ref[f] * m.mw_kg[d.indx[f]]));
    ff.psat_a[f] = (float)d.psat_coef[4 * f];
    ff.psat_b[f] = (float)d.psat_coef[4 * f + 1];
    ff.psat_c[f] = (float)d.psat_coef[4 * f + 2];
    ff.psat_d[f] = (float)d.psat_coef[4 * f + 3];
  }
  ff.ref_T = (float)d.ref_T;
  for (int i = 0; i < 3; ++i) {
    ff.body_force[i] = (float)d.body_force[i];
  }
  return PMP_OK;
}

int ensure_boxes_cap(pmp_spray* h, int n)
{
  if (n <= h->boxes_cap) {
    return PMP_OK;
  }
  delete[] h->h_boxes;
  h->h_boxes = new BoxEntry[n];
  h->boxes_cap = n;
  return PMP_OK;
}

// The device box table of the call being prepared (h->h_boxes[0, nboxes)):
// the slot already holding that content, or else the least recently used
// slot that no captured graph holds, uploaded on st.  Under stream capture
// the slot is held from then on: the graph reads it (and, if the capture
// uploaded it, copies from its staging) at every replay.
int acquire_table(pmp_spray* h, int nboxes, cudaStream_t st, const BoxEntry** out)
{
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PMP_CUDA(h, cudaStreamIsCapturing(st, &cap));
  const bool capturing = cap == cudaStreamCaptureStatusActive;
  const size_t bytes = sizeof(BoxEntry) * (size_t)nboxes;
  int pick = -1;
  for (int i = 0; i < pmp::kTableSlots; ++i) {
    pmp::TableSlot& t = h->tables[i];
    if (t.d && (int)t.host.size() == nboxes && memcmp(t.host.data(), h->h_boxes, bytes) == 0) {
      if (!capturing && t.stream != st) {
        PMP_CUDA(h, cudaStreamWaitEvent(st, t.uploaded, 0));
      }
      pick = i;
      break;
    }
  }
  if (pick < 0) {
    for (int i = 0; i < pmp::kTableSlots; ++i) {
      const pmp::TableSlot& t = h->tables[i];
      if (t.holds == 0 && (pick < 0 || t.last_use < h->tables[pick].last_use)) {
        pick = i;
      }
    }
    if (pick < 0) {
      return set_err(h, PMP_ERR_INVALID, "every box-table slot is held by a captured CUDA graph");
    }
    pmp::TableSlot& t = h->tables[pick];
    const int need = std::max(nboxes, 1);
    if (t.cap < need) {
      // kernels of earlier calls may still read the slot's table
      pmp::quiesce(h);
      cudaFree(t.d);
      cudaFreeHost(t.stage);
      t.d = nullptr;
      t.stage = nullptr;
      t.cap = 0;
      t.host.clear();
      const int n = std::max(need, 8);
      PMP_CUDA(h, cudaMalloc(&t.d, sizeof(BoxEntry) * n));
      PMP_CUDA(h, cudaMallocHost(&t.stage, sizeof(BoxEntry) * n));
      t.cap = n;
    }
    if (!t.uploaded) {
      PMP_CUDA(h, cudaEventCreateWithFlags(&t.uploaded, cudaEventDisableTiming));
    } else {
      // the slot's previous upload has read its staging
      PMP_CUDA(h, cudaEventSynchronize(t.uploaded));
    }
    memcpy(t.stage, h->h_boxes, bytes);
    t.host.assign(h->h_boxes, h->h_boxes + nboxes);
    if (nboxes > 0) {
      PMP_CUDA(h, cudaMemcpyAsync(t.d, t.stage, bytes, cudaMemcpyHostToDevice, st));
    }
    if (!capturing) {
      PMP_CUDA(h, cudaEventRecord(t.uploaded, st));
      t.stream = st;
    }
  }
  pmp::TableSlot& t = h->tables[pick];
  t.last_use = ++h->table_clock;
  if (capturing) {
    t.holds += 1;
  }
  h->cur_table = pick;
  *out = t.d;
  return PMP_OK;
}

int build_cta_map(pmp_spray* h);

int pack(pmp_spray* h)
{
  if (h->packed) {
    return PMP_OK;
  }
  const int nb = (int)h->boxes.size();
  for (int b = 0; b < nb; ++b) {
    if (!h->box_set[b]) {
      return set_err(h, PMP_ERR_INVALID, "set_particles was not called for every box", b);
    }
  }
  free_packed(h);
  const int nc = h->ncomp();
  long long total = 0;
  h->box_begin.assign(nb + 1, 0);
  for (int b = 0; b < nb; ++b) {
    h->box_begin[b] = total;
    total += h->staged[b].n;
  }
  h->box_begin[nb] = total;
  h->total = total;
  const long long cap = total > 0 ? total : 1;
  PMP_CUDA(h, cudaMalloc(&h->soa, sizeof(double) * nc * cap));
  PMP_CUDA(h, cudaMalloc(&h->ids, sizeof(int) * cap));
  PMP_CUDA(h, cudaMalloc(&h->perm, sizeof(long long) * cap));
  for (int b = 0; b < nb; ++b) {
    BoxStore& s = h->staged[b];
    const long long o = h->box_begin[b];
    if (s.n > 0) {
      PMP_CUDA(h, cudaMemcpy2D(h->soa + o, sizeof(double) * cap, s.d, sizeof(double) * s.n,
                               sizeof(double) * s.n, nc, cudaMemcpyDeviceToDevice));
      PMP_CUDA(h, cudaMemcpy(h->ids + o, s.id, sizeof(int) * s.n, cudaMemcpyDeviceToDevice));
      PMP_CUDA(h, cudaMemcpy(h->perm + o, s.perm, sizeof(long long) * s.n, cudaMemcpyDeviceToDevice));
    }
    free_store(s);
  }
  return build_cta_map(h);
}

// CTA -> (box, first slot) map, box offsets and fallback list of the packed droplets
int build_cta_map(pmp_spray* h)
{
  const int nb = (int)h->boxes.size();
  const long long cap = h->total > 0 ? h->total : 1;
  std::vector<int> cb;
  std::vector<long long> cs;
  for (int b = 0; b < nb; ++b) {
    for (long long o = h->box_begin[b]; o < h->box_begin[b + 1]; o += kBlock) {
      cb.push_back(b);
      cs.push_back(o);
    }
  }
  h->ncta = (int)cb.size();
  if (h->ncta > h->cta_cap) {  // kept by a re-binning while large enough
    cudaFree(h->d_cta_box);
    cudaFree(h->d_cta_start);
    h->d_cta_box = nullptr;
    h->d_cta_start = nullptr;
    h->cta_cap = 0;
    PMP_CUDA(h, cudaMalloc(&h->d_cta_box, sizeof(int) * h->ncta));
    PMP_CUDA(h, cudaMalloc(&h->d_cta_start, sizeof(long long) * h->ncta));
    h->cta_cap = h->ncta;
  }
  if (h->ncta > 0) {
    PMP_CUDA(h, cudaMemcpy(h->d_cta_box, cb.data(), sizeof(int) * h->ncta, cudaMemcpyHostToDevice));
    PMP_CUDA(h, cudaMemcpy(h->d_cta_start, cs.data(), sizeof(long long) * h->ncta, cudaMemcpyHostToDevice));
  }
  if (!h->d_box_begin) {
    PMP_CUDA(h, cudaMalloc(&h->d_box_begin, sizeof(long long) * (nb + 1)));
  }
  PMP_CUDA(h, cudaMemcpy(h->d_box_begin, h->box_begin.data(), sizeof(long long) * (nb + 1),
                         cudaMemcpyHostToDevice));
  if (!h->fb_list) {  // kept by a re-binning, whose droplet count only falls
    PMP_CUDA(h, cudaMalloc(&h->fb_list, sizeof(long long) * cap));
  }
  h->packed = true;
  return PMP_OK;
}

// Copy the droplets of box b (packed or staged) back into a device SoA of
// caller order: out_d (nc * n doubles), out_id (n ints).
int unsort_box(pmp_spray* h, int b, double* out_d, int* out_id, long long n)
{
  const int nc = h->ncomp();
  if (n == 0) {
    return PMP_OK;
  }
  if (h->packed) {
    const long long o = h->box_begin[b];
    k_unsort<<<nblk(n), 256>>>(h->soa + o, h->total, h->ids + o, h->perm + o, n, nc, out_d, out_id);
  } else {
    BoxStore& s = h->staged[b];
    k_unsort<<<nblk(n), 256>>>(s.d, s.n, s.id, s.perm, n, nc, out_d, out_id);
  }
  PMP_CUDA(h, cudaGetLastError());
  return PMP_OK;
}

// Device memory, managed memory or pinned (mapped) host memory; a plain host
// pointer would fault in the kernel.
bool device_accessible(const void* p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged ||
         a.type == cudaMemoryTypeHost;
}

bool view_covers(const pmp_box_view& v, const int* lo, const int* hi, int ncomp_needed)
{
  if (v.p == nullptr || v.ncomp < ncomp_needed) {
    return false;
  }
  for (int d = 0; d < 3; ++d) {
    if (lo[d] < v.lo[d] || hi[d] > v.hi[d]) {
      return false;
    }
  }
  return true;
}

size_t view_extent(const pmp_box_view& v)
{
  const long long nx = v.hi[0] - v.lo[0] + 1;
  const long long ny = v.hi[1] - v.lo[1] + 1;
  const long long nz = v.hi[2] - v.lo[2] + 1;
  return (size_t)((v.ncomp - 1) * v.nstride + (nz - 1) * v.kstride + (ny - 1) * v.jstride + nx);
}

// The components an update reads of the state (rho, momentum or velocity,
// T, species; PeleC: energy) or reads and writes of the source, as runs
// [first, last) of consecutive components: the host-view update copies only
// these.
std::vector<std::pair<int, int>> comp_runs(const pmp_spray* h, bool state)
{
  const pmp_spray_comps& c = h->comps;
  std::vector<int> need;
  if (state) {
    need = {c.rhoIndx, c.momIndx, c.momIndx + 1, c.momIndx + 2, c.utempIndx};
    for (int n = 0; n < h->nspec; ++n) {
      need.push_back(c.specIndx + n);
    }
    if (h->pelec) {
      need.push_back(c.engIndx);
    }
  } else {
    need = {c.rhoSrcIndx, c.momSrcIndx, c.momSrcIndx + 1, c.momSrcIndx + 2, c.engSrcIndx};
    for (int n = 0; n < h->nfuel; ++n) {
      need.push_back(c.specSrcIndx + n);
    }
  }
  std::sort(need.begin(), need.end());
  need.erase(std::unique(need.begin(), need.end()), need.end());
  std::vector<std::pair<int, int>> runs;
  for (int n : need) {
    if (!runs.empty() && runs.back().second == n) {
      runs.back().second = n + 1;
    } else {
      runs.push_back({n, n + 1});
    }
  }
  return runs;
}

// Copies components runs of view v (same layout at dst and src).
cudaError_t copy_runs(double* dst, const double* src, const pmp_box_view& v,
                      const std::vector<std::pair<int, int>>& runs, cudaMemcpyKind kind, cudaStream_t st)
{
  const size_t one = view_extent(v) - (size_t)(v.ncomp - 1) * v.nstride;  // one component's extent
  for (const auto& r : runs) {
    const size_t off = (size_t)r.first * v.nstride;
    const size_t n = (size_t)(r.second - 1 - r.first) * v.nstride + one;
    const cudaError_t e = cudaMemcpyAsync(dst + off, src + off, sizeof(double) * n, kind, st);
    if (e != cudaSuccess) {
      return e;
    }
  }
  return cudaSuccess;
}

// The source mirror's components on entry to a host-view update: the host
// arrays copied in (copy_in), or zeros (the host source is zero on entry).
cudaError_t source_in(double* dst, const double* src, const pmp_box_view& v,
                      const std::vector<std::pair<int, int>>& runs, int copy_in, cudaStream_t st)
{
  if (copy_in) {
    return copy_runs(dst, src, v, runs, cudaMemcpyHostToDevice, st);
  }
  const size_t one = view_extent(v) - (size_t)(v.ncomp - 1) * v.nstride;
  for (const auto& r : runs) {
    const size_t off = (size_t)r.first * v.nstride;
    const size_t n = (size_t)(r.second - 1 - r.first) * v.nstride + one;
    const cudaError_t e = cudaMemsetAsync(dst + off, 0, sizeof(double) * n, st);
    if (e != cudaSuccess) {
      return e;
    }
  }
  return cudaSuccess;
}

// tile_at_bndry (Source/PP_Spray/WallFunctions.H:8-35)
int tile_at_bndry(const pmp_box& b, const pmp_geometry& g)
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
  int at = 0;
  for (int d = 0; d < 3; ++d) {
    const bool lo_out = b.lo[d] - 1 < g.domain_lo[d];
    const bool hi_out = b.hi[d] + 1 > g.domain_hi[d];
    if ((lo_out && g.bndry_lo[d] != 0) || (hi_out && g.bndry_hi[d] != 0)) {
      at = 1;
    }
  }
  return at;
}

template <int NS, int NF>
void launch_fp64(const KParams& P, int ncta, cudaStream_t st)
{
  pmp::spray_update_fp64<NS, NF, kBlock><<<ncta, kBlock, 0, st>>>(P);
}

int dispatch_fp64(int ns, int nf, const KParams& P, int ncta, cudaStream_t st)
{
#define PMP_CASE(S, F)          \
  if (ns == S && nf == F) {     \
    launch_fp64<S, F>(P, ncta, st); \
    return PMP_OK;              \
  }
  PMP_CASE(3, 1)
  PMP_CASE(5, 1)
  PMP_CASE(5, 2)
  PMP_CASE(4, 1)
  PMP_CASE(4, 2)
#undef PMP_CASE
  return PMP_ERR_UNSUPPORTED;
}

int dispatch_fp64_pelec(int ns, int nf, const KParams& P, int ncta, cudaStream_t st)
{
#define PMP_CASE(S, F)                                                  \
  if (ns == S && nf == F) {                                             \
    pmp::spray_update_fp64_pelec<S, F, kBlock><<<ncta, kBlock, 0, st>>>(P); \
    return PMP_OK;                                                      \
  }
  PMP_CASE(3, 1)
  PMP_CASE(5, 1)
  PMP_CASE(5, 2)
  PMP_CASE(4, 1)
  PMP_CASE(4, 2)
#undef PMP_CASE
  return PMP_ERR_UNSUPPORTED;
}

// the FP64 kernel over the fallback list filled by the mixed / learned kernels
int dispatch_fp64_list(int ns, int nf, const KParams& P, long long total, cudaStream_t st)
{
  const long long need = (total + kBlock - 1) / kBlock;
  const int grid = (int)std::max(1LL, std::min(need, 148LL * 4));
#define PMP_CASE(S, F)                                                              \
  if (ns == S && nf == F) {                                                         \
    if (P.pelec) {                                                                  \
      pmp::spray_update_fp64_list<S, F, kBlock, true><<<grid, kBlock, 0, st>>>(P);  \
    } else {                                                                        \
      pmp::spray_update_fp64_list<S, F, kBlock><<<grid, kBlock, 0, st>>>(P);        \
    }                                                                               \
    return PMP_OK;                                                                  \
  }
  PMP_CASE(3, 1)
  PMP_CASE(5, 1)
  PMP_CASE(5, 2)
  PMP_CASE(4, 1)
  PMP_CASE(4, 2)
#undef PMP_CASE
  return PMP_ERR_UNSUPPORTED;
}

int prepare_update_impl(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes,
  double flow_dt, int state_ghosts, int source_ghosts, int is_ghost, int do_move,
  double spray_cfl_lev, cudaStream_t st, KParams& P)
{
  if (!h->have_data || !h->have_comps || !h->have_geom) {
    return set_err(h, PMP_ERR_INVALID, "setup, comps and geometry must be set before update");
  }
  if (nboxes != (int)h->boxes.size()) {
    return set_err(h, PMP_ERR_INVALID, "nboxes differs from the grids given to set_grids");
  }
  if (h->pelec && h->mode == PMP_MODE_LEARNED) {
    return set_err(h, PMP_ERR_UNSUPPORTED, "the PeleC coupling runs the FP64 and mixed forms");
  }
  if (h->mode == PMP_MODE_LEARNED && !pmp::learn_ready(h)) {
    return set_err(h, PMP_ERR_INVALID, "the learned form needs a trained surrogate (pmp_spray_learn_train)");
  }
  if (h->data.do_breakup != 0 || h->data.do_splash) {
    return set_err(h, PMP_ERR_UNSUPPORTED, "breakup and splash models are not supported");
  }
  if (!(flow_dt > 0.)) {
    return set_err(h, PMP_ERR_INVALID, "flow_dt must be positive");
  }
  int rc = pack(h);
  if (rc != PMP_OK) {
    return rc;
  }
  rc = ensure_boxes_cap(h, nboxes);
  if (rc != PMP_OK) {
    return rc;
  }
  const pmp_spray_comps& c = h->comps;
  const int NS = h->nspec;
  const int NF = h->nfuel;
  const int need_state = 1 + std::max({c.rhoIndx, c.momIndx + 2, c.utempIndx, c.specIndx + NS - 1,
                                       h->pelec ? c.engIndx : 0});
  const int need_src = 1 + std::max({c.rhoSrcIndx, c.momSrcIndx + 2, c.engSrcIndx, c.specSrcIndx + NF - 1});
  // gas records of the grown boxes: FP32 for the mixed and learned forms, FP64
  // for the FP64 form (16-byte units per cell: R)
  const bool rec32 = h->mode == PMP_MODE_MIXED || h->mode == PMP_MODE_LEARNED;
  const int R = rec32 ? pmp::gas_rec4(NS) : pmp::gas_rec2(NS);
  size_t rec_total = 0;
  h->gas_rec_max_cells = 0;
  for (int b = 0; b < nboxes; ++b) {
    long long cells = 1;
    for (int d = 0; d < 3; ++d) {
      cells *= (long long)(h->boxes[b].hi[d] - h->boxes[b].lo[d] + 1 + 2 * state_ghosts);
    }
    if (cells * R >= (1LL << 31)) {
      return set_err(h, PMP_ERR_INVALID, "a grown box holds 2^31 gas-record words or more", b);
    }
    h->gas_rec_max_cells = std::max(h->gas_rec_max_cells, (int)cells);
    rec_total += (size_t)cells * R;
  }
  if (16 * rec_total > h->gas_rec_bytes) {
    pmp::quiesce(h);  // kernels of earlier calls may still read the records
    cudaFree(h->gas_rec);
    h->gas_rec = nullptr;
    h->gas_rec_bytes = 0;
    PMP_CUDA(h, cudaMalloc(&h->gas_rec, 16 * rec_total));
    h->gas_rec_bytes = 16 * rec_total;
  }
  size_t rec_off = 0;
  for (int b = 0; b < nboxes; ++b) {
    const pmp_box& bx = h->boxes[b];
    BoxEntry& e = h->h_boxes[b];
    memset(&e, 0, sizeof(e));
    for (int d = 0; d < 3; ++d) {
      e.state_lo[d] = bx.lo[d] - state_ghosts;
      e.state_hi[d] = bx.hi[d] + state_ghosts;
      e.src_lo[d] = bx.lo[d] - source_ghosts;
      e.src_hi[d] = bx.hi[d] + source_ghosts;
    }
    if (!view_covers(state[b], e.state_lo, e.state_hi, need_state)) {
      return set_err(h, PMP_ERR_INVALID, "state view does not cover the grown box", b);
    }
    if (!view_covers(source[b], e.src_lo, e.src_hi, need_src)) {
      return set_err(h, PMP_ERR_INVALID, "source view does not cover the grown box", b);
    }
    if ((int)h->checked_state.size() != nboxes) {
      h->checked_state.assign(nboxes, nullptr);
      h->checked_src.assign(nboxes, nullptr);
    }
    if (h->checked_state[b] != state[b].p) {
      if (!device_accessible(state[b].p)) {
        return set_err(h, PMP_ERR_INVALID, "state view is not device memory (use pmp_spray_update_host)", b);
      }
      h->checked_state[b] = state[b].p;
    }
    if (h->checked_src[b] != source[b].p) {
      if (!device_accessible(source[b].p)) {
        return set_err(h, PMP_ERR_INVALID, "source view is not device memory (use pmp_spray_update_host)", b);
      }
      h->checked_src[b] = source[b].p;
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
    if (view_extent(state[b]) >= (1LL << 31) || view_extent(source[b]) >= (1LL << 31)) {
      return set_err(h, PMP_ERR_INVALID, "a state or source view spans 2^31 elements or more", b);
    }
    e.st_j32 = (int)state[b].jstride;
    e.st_k32 = (int)state[b].kstride;
    e.st_n32 = (int)state[b].nstride;
    e.sr_j32 = (int)source[b].jstride;
    e.sr_k32 = (int)source[b].kstride;
    e.sr_n32 = (int)source[b].nstride;
    {
      const int nx = e.state_hi[0] - e.state_lo[0] + 1;
      const int ny = e.state_hi[1] - e.state_lo[1] + 1;
      const int nz = e.state_hi[2] - e.state_lo[2] + 1;
      if (rec32) {
        e.gr = static_cast<float4*>(h->gas_rec) + rec_off;
      } else {
        e.gr64 = static_cast<double2*>(h->gas_rec) + rec_off;
      }
      e.gr_j = nx;
      e.gr_k = nx * ny;
      rec_off += (size_t)nx * ny * nz * R;
    }
    e.at_bounds = tile_at_bndry(bx, h->geom);
    e.p_begin = h->box_begin[b];
    e.p_end = h->box_begin[b + 1];
  }
  const BoxEntry* dtab = nullptr;
  rc = acquire_table(h, nboxes, st, &dtab);
  if (rc != PMP_OK) {
    return rc;
  }
  memset(&P, 0, sizeof(P));
  P.m = h->dmech;
  P.f = h->dfuel;
  P.mf = h->dmechf;
  for (int k = 0; k < PMP_MAX_SPEC; ++k) {
    P.spec_perm[k] = k < h->nspec ? h->spec_perm[k] : k;
  }
  P.fuel_first = h->fuel_first;
  P.ff = h->dfuelf;
  const long long T = h->total;
  for (int d = 0; d < 3; ++d) {
    P.parts.pos[d] = h->soa + (long long)d * T;
  }
  for (int r = 0; r < h->nr(); ++r) {
    P.parts.rd[r] = h->soa + (long long)(3 + r) * T;
  }
  P.parts.id = h->ids;
  const pmp_geometry& g = h->geom;
  for (int d = 0; d < 3; ++d) {
    P.plo[d] = g.plo[d];
    P.phi[d] = g.phi[d];
    P.dx[d] = g.dx[d];
    P.dxi[d] = 1. / g.dx[d];
    P.bndry_lo[d] = g.bndry_lo[d];
    P.bndry_hi[d] = g.bndry_hi[d];
  }
  const double vol = g.dx[0] * g.dx[1] * g.dx[2];
  P.inv_vol = 1. / vol;
  P.c_rho = c.rhoIndx;
  P.c_mom = c.momIndx;
  P.c_T = c.utempIndx;
  P.c_eng = c.engIndx;
  P.pelec = h->pelec;
  P.mixed_min_dia = h->pelec ? 100. * pmp::kMixedMinDia : pmp::kMixedMinDia;  // cm or m
  if (h->mode == PMP_MODE_LEARNED) {
    P.mixed_min_dia = pmp::kLearnMinDia;  // PeleLMeX only
  }
  P.c_spec = c.specIndx;
  P.s_rho = c.rhoSrcIndx;
  P.s_mom = c.momSrcIndx;
  P.s_eng = c.engSrcIndx;
  P.s_spec = c.specSrcIndx;
  // sub-cycling (SprayParticles.cpp:221-229)
  const double sub_cfl = 0.5;
  P.flow_dt = flow_dt;
  P.sub_dt = flow_dt;
  P.num_iter = 1;
  if (do_move && spray_cfl_lev > sub_cfl) {
    P.num_iter = static_cast<int>(std::ceil(spray_cfl_lev / sub_cfl));
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
  P.boxes = dtab;
  P.cta_box = h->d_cta_box;
  P.cta_start = h->d_cta_start;
  P.status = h->d_status;
  P.err_host = h->err_dev;
  P.box_begin = h->d_box_begin;
  P.fb_list = h->fb_list;
  P.fb_cap = h->total > 0 ? h->total : 1;
  P.nslots = h->total;
  return PMP_OK;
}

// After a call's device work is enqueued on st: remember the stream and mark
// the point (nothing is recorded while st is being captured into a graph;
// the caller then orders the replays).
int mark_enqueued(pmp_spray* h, cudaStream_t st)
{
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PMP_CUDA(h, cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    return PMP_OK;
  }
  PMP_CUDA(h, cudaEventRecord(h->ev_done, st));
  h->last_stream = st;
  h->pending = true;
  return PMP_OK;
}

// A device error of an earlier call that the host can already see (the
// kernels also write the code into mapped host memory): report it at once.
bool earlier_call_failed(const pmp_spray* h)
{
  return h->err_host && *reinterpret_cast<volatile const int*>(h->err_host) != 0;
}

// updateParticles for all boxes, stream-ordered: validates, enqueues the
// device work on st and returns without waiting for it.
int do_update(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes,
  double flow_dt, int state_ghosts, int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, cudaStream_t st)
{
  (void)is_virt;
  if (earlier_call_failed(h)) {
    return pmp::sync_status(h);
  }
  KParams P;
  int rc = prepare_update_impl(h, state, source, nboxes, flow_dt, state_ghosts, source_ghosts,
                               is_ghost, do_move, spray_cfl_lev, st, P);
  if (rc != PMP_OK) {
    return rc;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PMP_CUDA(h, cudaStreamIsCapturing(st, &cap));
  // the internal graph of the batched form is not nested in a caller's capture
  const bool graph = h->batch.cfg.use_graph && h->mode != PMP_MODE_LEARNED &&
                     h->batch.cfg.kind != PMP_LAUNCH_PER_BOX && cap == cudaStreamCaptureStatusNone;
  int graph_state = 0;
  rc = graph ? pmp::graph_update(h, P, nboxes, st, &graph_state) : pmp::enqueue_update(h, P, nboxes, st);
  if (rc != PMP_OK) {
    return rc;
  }
  h->stats.graph = graph_state;
  return mark_enqueued(h, st);
}

// The mixed form over CTA-map items [c0, c0 + n) (Q's map already offset),
// droplet slots [s0, s1) and boxes [b0, b0 + nb): the droplets it leaves to
// the FP64 kernel (d < 2 um at the call's start) are listed on the handle's
// high-priority side stream while the FP32 gas records are built on the
// caller's stream; the mixed kernel (which skips those droplets itself)
// starts once both are done, and the FP64 list kernel runs beside it on the
// side stream (it gathers the FP64 state, not the records).  The list kernel
// is one thread per listed droplet, so it costs the latency of one droplet's
// FP64 sub-cycles; beside the mixed kernel that latency is hidden.  The
// caller's stream waits for both.
int enqueue_mixed(pmp_spray* h, const KParams& Q, int n, long long s0, long long s1, int b0, int nb,
                  cudaStream_t st)
{
  KParams R = Q;
  R.fb_pre = 1;
  PMP_CUDA(h, cudaEventRecord(h->ev_fork, st));
  PMP_CUDA(h, cudaStreamWaitEvent(h->side, h->ev_fork, 0));
  int rc = pmp::launch_select_small(R, s0, s1, h->side);
  // the selection must read the droplets before the mixed kernel changes them
  const cudaError_t es = rc == PMP_OK ? cudaEventRecord(h->ev_sel, h->side) : cudaSuccess;
  if (rc == PMP_OK && es == cudaSuccess) {
    rc = dispatch_fp64_list(h->nspec, h->nfuel, R, h->total, h->side);
  }
  if (rc == PMP_OK && es == cudaSuccess) {
    rc = pmp::launch_gas_records(h->nspec, Q, b0, nb, h->gas_rec_max_cells, st);
    if (rc != PMP_OK) {
      rc = set_err(h, rc, "no gas-record kernel for this species count");
    }
  }
  const cudaError_t ew = rc == PMP_OK && es == cudaSuccess ? cudaStreamWaitEvent(st, h->ev_sel, 0) : cudaSuccess;
  if (rc == PMP_OK && es == cudaSuccess && ew == cudaSuccess) {
    rc = pmp::launch_mixed(h->nspec, h->nfuel, R, n, kBlock, st);
  }
  // join the side stream whatever happened (a capture must not end with
  // unjoined work, and a failing launch keeps its own code)
  const cudaError_t e1 = cudaEventRecord(h->ev_join, h->side);
  const cudaError_t e2 = cudaStreamWaitEvent(st, h->ev_join, 0);
  if (rc != PMP_OK) {
    return rc;
  }
  PMP_CUDA(h, es);
  PMP_CUDA(h, ew);
  PMP_CUDA(h, e1);
  PMP_CUDA(h, e2);
  return PMP_OK;
}

// The learned form over CTA-map items [c0, c0 + n) and droplet slots
// [s0, s1), arranged as the mixed form's: the droplets below 2 um are listed
// first and their FP64 kernel runs on the side stream beside the learned
// kernel; the droplets the learned kernel's gate rejects (listed from the end
// of the fallback list) are updated by the FP64 kernel after it.  Q's box
// filter (list_box0 / list_nbox) applies to both lists.
int enqueue_learned(pmp_spray* h, const KParams& Q, int c0, int n, long long s0, long long s1, cudaStream_t st)
{
  KParams R = Q;
  R.fb_pre = 1;
  int rc = pmp::launch_select_small(R, s0, s1, st);
  if (rc != PMP_OK) {
    return rc;
  }
  PMP_CUDA(h, cudaEventRecord(h->ev_fork, st));
  PMP_CUDA(h, cudaStreamWaitEvent(h->side, h->ev_fork, 0));
  rc = dispatch_fp64_list(h->nspec, h->nfuel, R, h->total, h->side);
  if (rc == PMP_OK) {
    rc = pmp::launch_learned(h, R, st, c0, n);
  }
  if (rc == PMP_OK) {
    KParams G = R;
    G.list_back = 1;
    rc = dispatch_fp64_list(h->nspec, h->nfuel, G, h->total, st);
  }
  const cudaError_t e1 = cudaEventRecord(h->ev_join, h->side);
  const cudaError_t e2 = cudaStreamWaitEvent(st, h->ev_join, 0);
  if (rc != PMP_OK) {
    return rc;
  }
  PMP_CUDA(h, e1);
  PMP_CUDA(h, e2);
  return PMP_OK;
}

// The overlapped form of pmp_spray_update_host.  The boxes are split into up
// to kHostStages consecutive groups of about equal bytes; group g's state and
// source are copied in on one stream while the update of the groups before
// it runs on the caller's stream, and its sources are copied back on a third
// stream while later groups run.  A droplet reads and deposits only its own
// box's views, and the CTA map is box-contiguous, so group g's launch (the
// map's CTA range of its boxes, then the fallback list filtered to its boxes)
// needs group g's copies only.  hst/hsr are the caller's host views, dst/dsr
// their device mirrors.
int update_host_overlapped_impl(
  pmp_spray* h, const pmp_box_view* hst, const pmp_box_view* hsr, const pmp_box_view* dst,
  const pmp_box_view* dsr, int nboxes, double flow_dt, int state_ghosts, int source_ghosts,
  int is_ghost, int do_move, double spray_cfl_lev, cudaStream_t st)
{
  KParams P;
  int rc = prepare_update_impl(h, dst, dsr, nboxes, flow_dt, state_ghosts, source_ghosts,
                               is_ghost, do_move, spray_cfl_lev, st, P);
  if (rc != PMP_OK) {
    return rc;
  }
  if (!h->hs_in) {
    PMP_CUDA(h, cudaStreamCreateWithFlags(&h->hs_in, cudaStreamNonBlocking));
    PMP_CUDA(h, cudaStreamCreateWithFlags(&h->hs_out, cudaStreamNonBlocking));
    for (int g = 0; g < pmp_spray::kHostStages; ++g) {
      PMP_CUDA(h, cudaEventCreateWithFlags(&h->hev_in[g], cudaEventDisableTiming));
      PMP_CUDA(h, cudaEventCreateWithFlags(&h->hev_done[g], cudaEventDisableTiming));
    }
    PMP_CUDA(h, cudaEventCreateWithFlags(&h->hev_start, cudaEventDisableTiming));
    PMP_CUDA(h, cudaEventCreateWithFlags(&h->hev_out, cudaEventDisableTiming));
  }
  // groups of consecutive boxes of about equal bytes
  std::vector<size_t> bytes(nboxes);
  size_t total_bytes = 0;
  for (int b = 0; b < nboxes; ++b) {
    bytes[b] = sizeof(double) * (view_extent(hst[b]) + 2 * view_extent(hsr[b]));
    total_bytes += bytes[b];
  }
  const int G = std::max(1, std::min(nboxes, (int)pmp_spray::kHostStages));
  std::vector<int> gfirst(1, 0);
  {
    size_t acc = 0;
    for (int b = 0; b < nboxes; ++b) {
      acc += bytes[b];
      const int made = (int)gfirst.size();
      if (b + 1 < nboxes && made < G && acc * G >= total_bytes * made) {
        gfirst.push_back(b + 1);
      }
    }
    gfirst.push_back(nboxes);
  }
  const int ngroups = (int)gfirst.size() - 1;
  // first CTA-map item of each box (build_cta_map: ceil(n_b / kBlock) items per box, in box order)
  std::vector<int> cta_first(nboxes + 1, 0);
  for (int b = 0; b < nboxes; ++b) {
    const long long n = h->box_begin[b + 1] - h->box_begin[b];
    cta_first[b + 1] = cta_first[b] + (int)((n + kBlock - 1) / kBlock);
  }
  if (cta_first[nboxes] != h->ncta) {
    return set_err(h, PMP_ERR_INVALID, "CTA map does not match the boxes");
  }
  const int NS = h->nspec;
  const int NF = h->nfuel;
  PMP_CUDA(h, cudaMemsetAsync(&h->d_status->fb_count, 0, 2 * sizeof(unsigned long long), st));
  PMP_CUDA(h, cudaEventRecord(h->ev0, st));
  PMP_CUDA(h, cudaEventRecord(h->hev_start, st));
  PMP_CUDA(h, cudaStreamWaitEvent(h->hs_in, h->hev_start, 0));
  PMP_CUDA(h, cudaStreamWaitEvent(h->hs_out, h->hev_start, 0));
  const auto st_runs = comp_runs(h, true);
  const auto sr_runs = comp_runs(h, false);
  auto copy_in = [&](int g) -> int {
    for (int b = gfirst[g]; b < gfirst[g + 1]; ++b) {
      PMP_CUDA(h, copy_runs(dst[b].p, hst[b].p, hst[b], st_runs, cudaMemcpyHostToDevice, h->hs_in));
      PMP_CUDA(h, source_in(dsr[b].p, hsr[b].p, hsr[b], sr_runs, h->host_src_in, h->hs_in));
    }
    PMP_CUDA(h, cudaEventRecord(h->hev_in[g], h->hs_in));
    return PMP_OK;
  };
  rc = copy_in(0);
  if (rc != PMP_OK) {
    return rc;
  }
  for (int g = 0; g < ngroups; ++g) {
    PMP_CUDA(h, cudaStreamWaitEvent(st, h->hev_in[g], 0));
    const int b0 = gfirst[g], b1 = gfirst[g + 1];
    const int c0 = cta_first[b0], n = cta_first[b1] - c0;
    KParams Q = P;
    Q.cta_box = P.cta_box + c0;
    Q.cta_start = P.cta_start + c0;
    Q.list_box0 = b0;
    Q.list_nbox = b1 - b0;
    if (n > 0) {
      // the mixed form builds its gas records inside enqueue_mixed
      if (h->mode != PMP_MODE_MIXED) {
        rc = h->mode == PMP_MODE_LEARNED ? pmp::launch_gas_records(NS, P, b0, b1 - b0, h->gas_rec_max_cells, st)
                                         : pmp::launch_gas_records64(h, P, b0, b1 - b0, st);
        if (rc != PMP_OK) {
          return set_err(h, rc, "no gas-record kernel for this species count");
        }
      }
      if (h->mode == PMP_MODE_LEARNED) {
        // the learned kernel takes the whole map and an item range; the
        // fallback lists are filtered to the group's boxes
        KParams Lq = P;
        Lq.list_box0 = b0;
        Lq.list_nbox = b1 - b0;
        rc = enqueue_learned(h, Lq, c0, n, h->box_begin[b0], h->box_begin[b1], st);
      } else if (h->mode == PMP_MODE_MIXED) {
        rc = enqueue_mixed(h, Q, n, h->box_begin[b0], h->box_begin[b1], b0, b1 - b0, st);
      } else if (P.pelec) {
        rc = dispatch_fp64_pelec(NS, NF, Q, n, st);
      } else {
        rc = dispatch_fp64(NS, NF, Q, n, st);
      }
      if (rc == PMP_ERR_UNSUPPORTED) {
        return set_err(h, rc, "no kernel for this species / fuel count");
      }
      if (rc != PMP_OK) {
        return rc;
      }
      PMP_CUDA(h, cudaGetLastError());
    }
    PMP_CUDA(h, cudaEventRecord(h->hev_done[g], st));
    if (g + 1 < ngroups) {
      rc = copy_in(g + 1);
      if (rc != PMP_OK) {
        return rc;
      }
    }
  }
  for (int g = 0; g < ngroups; ++g) {
    PMP_CUDA(h, cudaStreamWaitEvent(h->hs_out, h->hev_done[g], 0));
    for (int b = gfirst[g]; b < gfirst[g + 1]; ++b) {
      PMP_CUDA(h, copy_runs(hsr[b].p, dsr[b].p, hsr[b], sr_runs, cudaMemcpyDeviceToHost, h->hs_out));
    }
  }
  PMP_CUDA(h, cudaEventRecord(h->hev_out, h->hs_out));
  PMP_CUDA(h, cudaStreamWaitEvent(st, h->hev_out, 0));
  PMP_CUDA(h, cudaEventRecord(h->ev1, st));
  h->stats.graph = 0;
  return mark_enqueued(h, st);
}

int update_host_overlapped(
  pmp_spray* h, const pmp_box_view* hst, const pmp_box_view* hsr, const pmp_box_view* dst,
  const pmp_box_view* dsr, int nboxes, double flow_dt, int state_ghosts, int source_ghosts,
  int is_ghost, int do_move, double spray_cfl_lev, cudaStream_t st)
{
  if (earlier_call_failed(h)) {
    return pmp::sync_status(h);
  }
  const int rc = update_host_overlapped_impl(h, hst, hsr, dst, dsr, nboxes, flow_dt, state_ghosts,
                                             source_ghosts, is_ghost, do_move, spray_cfl_lev, st);
  if (rc != PMP_OK && h->hs_in) {
    // no copy of the caller's host memory may still be in flight on return
    cudaStreamSynchronize(h->hs_in);
    cudaStreamSynchronize(h->hs_out);
    cudaStreamSynchronize(st);
  }
  return rc;
}

}  // namespace

void pmp::quiesce(pmp_spray* h)
{
  if (h->pending && h->ev_done) {
    cudaEventSynchronize(h->ev_done);
  }
}

void pmp::release_table(pmp_spray* h, int slot)
{
  if (slot >= 0 && slot < pmp::kTableSlots && h->tables[slot].holds > 0) {
    h->tables[slot].holds -= 1;
  }
}

// The status the handle's calls accumulated since the last read: copied back
// after the last call's work on its stream, reported (stats, error record)
// and cleared.
int pmp::sync_status(pmp_spray* h)
{
  cudaStream_t st = h->last_stream;
  PMP_CUDA(h, cudaMemcpyAsync(h->h_status, h->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
  PMP_CUDA(h, cudaStreamSynchronize(st));
  h->pending = false;
  const long long T = h->total;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) {
    h->stats.kernel_ms = ms;
  } else {
    h->stats.kernel_ms = -1.;
    cudaGetLastError();  // not sticky: clear it so that the next call does not report it
  }
  pmp::status_counters(*h->h_status, h->stats.substeps, h->stats.killed, h->stats.inner_steps);
  h->stats.fallback = (long long)h->h_status->fallback;
  if (h->h_status->code != 0) {
    const int b = h->h_status->box;
    long long caller = -1;
    const long long slot = h->h_status->slot;
    if (slot >= 0 && slot < h->total) {
      cudaMemcpy(&caller, h->perm + slot, sizeof(long long), cudaMemcpyDeviceToHost);
    }
    double pos[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d) {
      cudaMemcpy(&pos[d], h->soa + (long long)d * T + slot, sizeof(double), cudaMemcpyDeviceToHost);
    }
    static const char* names[] = {"ok", "droplet left the domain", "state box too small",
                                  "source box too small", "unsupported droplet state", "timeout"};
    const int code = h->h_status->code;
    // clear the status (the error is reported once; later calls run again)
    PMP_CUDA(h, cudaMemsetAsync(h->d_status, 0, sizeof(DevStatus), st));
    PMP_CUDA(h, cudaStreamSynchronize(st));
    *reinterpret_cast<volatile int*>(h->err_host) = 0;
    set_err(h, code, code < 6 ? names[code] : "error", b, caller);
    for (int d = 0; d < 3; ++d) {
      h->last_err.pos[d] = pos[d];
    }
    return code;
  }
  PMP_CUDA(h, cudaMemsetAsync(h->d_status, 0, sizeof(DevStatus), st));
  PMP_CUDA(h, cudaStreamSynchronize(st));
  memset(&h->last_err, 0, sizeof(h->last_err));
  h->last_err.particle = -1;
  return PMP_OK;
}

int pmp::prepare_update(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes,
  double flow_dt, int state_ghosts, int source_ghosts, int is_ghost, int do_move,
  double spray_cfl_lev, cudaStream_t st, KParams& P)
{
  const int rc = prepare_update_impl(h, state, source, nboxes, flow_dt, state_ghosts, source_ghosts,
                                     is_ghost, do_move, spray_cfl_lev, st, P);
  if (rc != PMP_OK) {
    return rc;
  }
  PMP_CUDA(h, cudaMemsetAsync(&h->d_status->fb_count, 0, 2 * sizeof(unsigned long long), st));
  return PMP_OK;
}

int pmp::ensure_packed(pmp_spray* h) { return pack(h); }

int pmp::install_rebinned(pmp_spray* h, const std::vector<long long>& box_begin)
{
  const int nb = (int)h->boxes.size();
  h->box_begin = box_begin;
  h->total = box_begin[nb];
  for (int b = 0; b < nb; ++b) {
    free_store(h->staged[b]);
    h->staged[b].n = box_begin[b + 1] - box_begin[b];
    h->box_set[b] = true;
  }
  // the CTA map and the box bounds of the new counts (their arrays, perm and
  // the fallback list keep their capacity: the droplet count only falls)
  h->ncta = 0;
  pmp::batch_reset(h);
  return build_cta_map(h);
}

int pmp::enqueue_update(pmp_spray* h, const KParams& P, int nboxes, cudaStream_t st)
{
  // under stream capture the timing events become event-record nodes of the graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PMP_CUDA(h, cudaStreamIsCapturing(st, &cap));
  const unsigned ev_flags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0u;
  PMP_CUDA(h, cudaMemsetAsync(&h->d_status->fb_count, 0, 2 * sizeof(unsigned long long), st));
  PMP_CUDA(h, cudaEventRecordWithFlags(h->ev0, st, ev_flags));
  if (h->ncta > 0) {
    const int NS = h->nspec;
    const int NF = h->nfuel;
    int rc = PMP_OK;
    if (h->mode == PMP_MODE_LEARNED) {
      rc = pmp::launch_gas_records(NS, P, 0, nboxes, h->gas_rec_max_cells, st);
      if (rc == PMP_OK) {
        rc = enqueue_learned(h, P, 0, h->ncta, 0, h->total, st);
      }
    } else if (h->mode == PMP_MODE_MIXED) {
      rc = enqueue_mixed(h, P, h->ncta, 0, h->total, 0, nboxes, st);
    } else if (P.pelec) {
      rc = pmp::launch_gas_records64(h, P, 0, nboxes, st);
      if (rc == PMP_OK) {
        rc = dispatch_fp64_pelec(NS, NF, P, h->ncta, st);
      }
    } else {
      rc = pmp::batch_enqueue_fp64(h, P, nboxes, st);
    }
    if (rc == PMP_ERR_UNSUPPORTED) {
      return set_err(h, rc, "no kernel for this species / fuel count");
    }
    if (rc != PMP_OK) {
      return rc;
    }
    PMP_CUDA(h, cudaGetLastError());
  }
  PMP_CUDA(h, cudaEventRecordWithFlags(h->ev1, st, ev_flags));
  return PMP_OK;
}

int pmp::run_update(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes,
  double flow_dt, int state_ghosts, int source_ghosts, int is_ghost, int do_move,
  double spray_cfl_lev, cudaStream_t st)
{
  const int rc = do_update(h, state, source, nboxes, flow_dt, state_ghosts, source_ghosts, 0, is_ghost,
                           do_move, spray_cfl_lev, st);
  if (rc != PMP_OK) {
    return rc;
  }
  return sync_status(h);
}

int pmp::launch_gas_records64(const pmp_spray* h, const KParams& P, int b0, int nb, cudaStream_t st)
{
  const int max_cells = h->gas_rec_max_cells;
  if (nb <= 0 || max_cells <= 0 || h->mode != PMP_MODE_FP64) {
    return PMP_OK;
  }
  const dim3 grid((unsigned)std::min((max_cells + 255) / 256, 128), (unsigned)nb);
#define PMP_REC_CASE(S)                                                  \
  if (h->nspec == S) {                                                   \
    if (h->pelec) {                                                      \
      pmp::k_gas_records64<S, true><<<grid, 256, 0, st>>>(P, b0);        \
    } else {                                                             \
      pmp::k_gas_records64<S, false><<<grid, 256, 0, st>>>(P, b0);       \
    }                                                                    \
    return PMP_OK;                                                       \
  }
  PMP_REC_CASE(3)
  PMP_REC_CASE(4)
  PMP_REC_CASE(5)
#undef PMP_REC_CASE
  return PMP_ERR_UNSUPPORTED;
}

int pmp::dispatch_fp64_default(int ns, int nf, const KParams& P, int ncta, cudaStream_t st)
{
  return dispatch_fp64(ns, nf, P, ncta, st);
}

int pmp::run_fp64_list(int ns, int nf, const KParams& P, long long total, cudaStream_t st)
{
  return ::dispatch_fp64_list(ns, nf, P, total, st);
}

// ===========================================================================
// C ABI

extern "C" {

const char* pmp_spray_version(void) { return "pmp-spray-b200 0.1 (sm_100a)"; }

int pmp_spray_create(const pmp_spray_config* cfg, pmp_spray** out)
{
  if (!cfg || !out) {
    return PMP_ERR_INVALID;
  }
  *out = nullptr;
  if (cfg->nfuel < 1 || cfg->nfuel > PMP_MAX_FUEL || cfg->nspec < 1 || cfg->nspec > PMP_MAX_SPEC) {
    return PMP_ERR_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
    cudaGetLastError();
    return PMP_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major != 10) {
    return PMP_ERR_NO_DEVICE;
  }
  pmp_spray* h = new pmp_spray();
  h->device = cfg->device;
  h->nfuel = cfg->nfuel;
  h->nspec = cfg->nspec;
  int idx[PMP_MAX_SPEC];
  for (int k = 0; k < cfg->nspec; ++k) {
    memcpy(h->species[k], cfg->species[k], PMP_NAME_LEN);
    h->species[k][PMP_NAME_LEN - 1] = 0;
    idx[k] = pmp_db_lookup(h->species[k]);
    if (idx[k] < 0) {
      delete h;
      return PMP_ERR_INVALID;
    }
  }
  if (pmp_mech_build(&h->mech, cfg->nspec, idx) != 0) {
    delete h;
    return PMP_ERR_INVALID;
  }
  memset(&h->last_err, 0, sizeof(h->last_err));
  memset(&h->stats, 0, sizeof(h->stats));
  if (cudaSetDevice(h->device) != cudaSuccess ||
      cudaMalloc(&h->d_status, sizeof(DevStatus)) != cudaSuccess ||
      cudaMemset(h->d_status, 0, sizeof(DevStatus)) != cudaSuccess ||
      cudaMallocHost(&h->h_status, sizeof(DevStatus)) != cudaSuccess ||
      cudaHostAlloc(&h->err_host, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(&h->err_dev, h->err_host, 0) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_done, cudaEventDisableTiming) != cudaSuccess) {
    pmp_spray_destroy(h);
    return PMP_ERR_CUDA;
  }
  *h->err_host = 0;
  {
    int lo = 0, hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_sel, cudaEventDisableTiming) != cudaSuccess) {
      pmp_spray_destroy(h);
      return PMP_ERR_CUDA;
    }
  }
  *out = h;
  return PMP_OK;
}

int pmp_spray_destroy(pmp_spray* h)
{
  if (!h) {
    return PMP_OK;
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  for (auto& s : h->staged) {
    free_store(s);
  }
  free_packed(h);
  pmp::learn_free(h);
  pmp::batch_free(h);
  pmp::mesh_free(h);
  for (double* p : h->stage_state) {
    cudaFree(p);
  }
  for (double* p : h->stage_src) {
    cudaFree(p);
  }
  cudaFree(h->gas_rec);
  delete[] h->h_boxes;
  for (pmp::TableSlot& t : h->tables) {
    cudaFree(t.d);
    cudaFreeHost(t.stage);
    if (t.uploaded) {
      cudaEventDestroy(t.uploaded);
    }
  }
  cudaFree(h->d_status);
  cudaFreeHost(h->h_status);
  cudaFreeHost(h->err_host);
  if (h->ev_done) {
    cudaEventDestroy(h->ev_done);
  }
  if (h->ev0) {
    cudaEventDestroy(h->ev0);
  }
  if (h->ev1) {
    cudaEventDestroy(h->ev1);
  }
  if (h->side) {
    cudaStreamDestroy(h->side);
  }
  if (h->ev_fork) {
    cudaEventDestroy(h->ev_fork);
  }
  if (h->ev_join) {
    cudaEventDestroy(h->ev_join);
  }
  if (h->ev_sel) {
    cudaEventDestroy(h->ev_sel);
  }
  if (h->hs_in) {
    cudaStreamDestroy(h->hs_in);
    cudaStreamDestroy(h->hs_out);
    for (int g = 0; g < pmp_spray::kHostStages; ++g) {
      cudaEventDestroy(h->hev_in[g]);
      cudaEventDestroy(h->hev_done[g]);
    }
    cudaEventDestroy(h->hev_start);
    cudaEventDestroy(h->hev_out);
  }
  delete h;
  return PMP_OK;
}

int pmp_spray_setup(pmp_spray* h, const pmp_spray_inputs* in)
{
  if (!h || !in) {
    return PMP_ERR_INVALID;
  }
  // readSprayParams (SpraySetup.cpp:73-253)
  if (in->nfuel != h->nfuel) {
    return set_err(h, PMP_ERR_INVALID, "Number of fuel species in input file must match SPRAY_FUEL_NUM");
  }
  if (in->cfl > 2.) {
    return set_err(h, PMP_ERR_INVALID, "particles.cfl must be <= 2");
  }
  if (in->use_breakup_model != 0 || in->use_splash_model) {
    return set_err(h, PMP_ERR_UNSUPPORTED, "breakup and splash models are not supported");
  }
  pmp_spray_data d;
  memset(&d, 0, sizeof(d));
  d.nfuel = in->nfuel;
  d.mass_trans = in->mass_transfer;
  d.mom_trans = in->mom_transfer;
  d.fixed_parts = in->fixed_parts;
  d.min_eb_vfrac = 0.05;
  d.sigma = -1.;
  d.wall_T = -1.;
  d.theta_c = -1.;
  d.dtmod = 0.5;
  const int NF = in->nfuel;
  for (int f = 0; f < NF; ++f) {
    d.critT[f] = in->crit_temp[f];
    d.boilT[f] = in->boil_temp[f];
    d.cp[f] = in->cp[f];
    d.ref_latent[f] = in->latent[f];
    const int* nc[4] = {in->ncoef_lambda, in->ncoef_psat, in->ncoef_rho, in->ncoef_mu};
    const double(*src[4])[4] = {in->lambda, in->psat, in->rho, in->mu};
    double* dst[4] = {d.lambda_coef, d.psat_coef, d.rho_coef, d.mu_coef};
    for (int q = 0; q < 4; ++q) {
      if (nc[q][f] == 4) {
        for (int i = 0; i < 4; ++i) {
          dst[q][4 * f + i] = src[q][f][i];
        }
      } else if (nc[q][f] == 1) {
        for (int i = 0; i < 4; ++i) {
          dst[q][4 * f + i] = 0.;
        }
        dst[q][4 * f] = src[q][f][0];
      } else if (q == 2) {
        return set_err(h, PMP_ERR_INVALID, "particles.<fuel>_rho is required");
      }
    }
    d.latent[f] = d.ref_latent[f];
  }
  d.ref_T = in->fuel_ref_temp;
  // spraySetup (SpraySetup.cpp:255-297)
  for (int f = 0; f < NF; ++f) {
    d.indx[f] = -1;
    d.dep_indx[f] = -1;
    const char* dep = in->dep_fuel_species[f][0] ? in->dep_fuel_species[f] : in->fuel_species[f];
    for (int ns = 0; ns < h->nspec; ++ns) {
      if (strncmp(h->species[ns], in->fuel_species[f], PMP_NAME_LEN) == 0) {
        d.indx[f] = ns;
      }
      if (strncmp(h->species[ns], dep, PMP_NAME_LEN) == 0) {
        d.dep_indx[f] = ns;
      }
    }
    if (d.indx[f] < 0 || d.dep_indx[f] < 0) {
      return set_err(h, PMP_ERR_INVALID, "Fuel not found in species list");
    }
  }
  double fuelEnth[PMP_MAX_SPEC];
  pmp_eos_T2Hi(&h->mech, d.ref_T, fuelEnth);
  for (int ns = 0; ns < NF; ++ns) {
    d.latent[ns] -= fuelEnth[d.indx[ns]] * (h->pelec ? 1. : pmp::kEngConv);
  }
  for (int i = 0; i < 3; ++i) {
    d.body_force[i] = in->body_force[i];
  }
  return pmp_spray_set_data(h, &d);
}

int pmp_spray_set_data(pmp_spray* h, const pmp_spray_data* data)
{
  if (!h || !data) {
    return PMP_ERR_INVALID;
  }
  if (data->nfuel != h->nfuel) {
    return set_err(h, PMP_ERR_INVALID, "SprayData fuel count differs from the handle's");
  }
  if (data->do_breakup != 0 || data->do_splash) {
    return set_err(h, PMP_ERR_UNSUPPORTED, "breakup and splash models are not supported");
  }
  h->data = *data;
  const int rc = build_device_tables(h);
  h->have_data = rc == PMP_OK;
  return rc;
}

int pmp_spray_get_data(const pmp_spray* h, pmp_spray_data* data)
{
  if (!h || !data || !h->have_data) {
    return PMP_ERR_INVALID;
  }
  *data = h->data;
  return PMP_OK;
}

int pmp_spray_set_comps(pmp_spray* h, const pmp_spray_comps* comps)
{
  if (!h || !comps) {
    return PMP_ERR_INVALID;
  }
  const int idx[] = {comps->rhoIndx,    comps->momIndx,    comps->engIndx,
                     comps->utempIndx,  comps->specIndx,   comps->rhoSrcIndx,
                     comps->momSrcIndx, comps->engSrcIndx, comps->specSrcIndx};
  for (int i : idx) {
    if (i < 0) {
      return set_err(h, PMP_ERR_INVALID, "negative component index");
    }
  }
  h->comps = *comps;
  h->have_comps = true;
  return PMP_OK;
}

int pmp_spray_set_geometry(pmp_spray* h, const pmp_geometry* geom)
{
  if (!h || !geom) {
    return PMP_ERR_INVALID;
  }
  for (int d = 0; d < 3; ++d) {
    if (!(geom->dx[d] > 0.) || geom->domain_hi[d] < geom->domain_lo[d]) {
      return set_err(h, PMP_ERR_INVALID, "bad geometry");
    }
    const int bl = geom->bndry_lo[d];
    const int bh = geom->bndry_hi[d];
    if (bl < -1 || bl > 1 || bh < -1 || bh > 1 || ((bl == 0) != (bh == 0))) {
      return set_err(h, PMP_ERR_INVALID, "bad boundary designation");
    }
  }
  h->geom = *geom;
  h->have_geom = true;
  h->grids_version += 1;
  return PMP_OK;
}

int pmp_spray_set_grids(pmp_spray* h, int nboxes, const pmp_box* boxes)
{
  if (!h || nboxes < 0 || (nboxes > 0 && !boxes)) {
    return PMP_ERR_INVALID;
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  for (auto& s : h->staged) {
    free_store(s);
  }
  free_packed(h);
  h->boxes.assign(boxes, boxes + nboxes);
  h->grids_version += 1;
  h->staged.assign(nboxes, BoxStore{});
  h->box_set.assign(nboxes, false);
  return PMP_OK;
}

int pmp_spray_set_particles(pmp_spray* h, int box, const pmp_particles* p)
{
  if (!h || !p || box < 0 || box >= (int)h->boxes.size() || p->n < 0) {
    return PMP_ERR_INVALID;
  }
  if (!h->have_geom) {
    return set_err(h, PMP_ERR_INVALID, "set_geometry must precede set_particles");
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  // unpack the other boxes first if the layout changes
  if (h->packed) {
    const int nb = (int)h->boxes.size();
    const int nc = h->ncomp();
    for (int b = 0; b < nb; ++b) {
      const long long n = h->box_begin[b + 1] - h->box_begin[b];
      BoxStore s;
      s.n = n;
      if (n > 0) {
        PMP_CUDA(h, cudaMalloc(&s.d, sizeof(double) * nc * n));
        PMP_CUDA(h, cudaMalloc(&s.id, sizeof(int) * n));
        PMP_CUDA(h, cudaMalloc(&s.perm, sizeof(long long) * n));
        const long long o = h->box_begin[b];
        PMP_CUDA(h, cudaMemcpy2D(s.d, sizeof(double) * n, h->soa + o, sizeof(double) * h->total,
                                 sizeof(double) * n, nc, cudaMemcpyDeviceToDevice));
        PMP_CUDA(h, cudaMemcpy(s.id, h->ids + o, sizeof(int) * n, cudaMemcpyDeviceToDevice));
        PMP_CUDA(h, cudaMemcpy(s.perm, h->perm + o, sizeof(long long) * n, cudaMemcpyDeviceToDevice));
      }
      h->staged[b] = s;
    }
    free_packed(h);
  }
  BoxStore& s = h->staged[box];
  free_store(s);
  const long long n = p->n;
  const int nc = h->ncomp();
  const int nr = h->nr();
  s.n = n;
  h->box_set[box] = true;
  if (n == 0) {
    return PMP_OK;
  }
  double* raw = nullptr;
  int* rid = nullptr;
  PMP_CUDA(h, cudaMalloc(&raw, sizeof(double) * nc * n));
  PMP_CUDA(h, cudaMalloc(&rid, sizeof(int) * n));
  const cudaMemcpyKind kind =
    p->where == PMP_WHERE_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  if (p->layout == PMP_LAYOUT_SOA) {
    for (int d = 0; d < 3; ++d) {
      if (!p->pos[d]) {
        cudaFree(raw);
        cudaFree(rid);
        return set_err(h, PMP_ERR_INVALID, "missing position array");
      }
      PMP_CUDA(h, cudaMemcpy(raw + (long long)d * n, p->pos[d], sizeof(double) * n, kind));
    }
    for (int r = 0; r < nr; ++r) {
      if (p->rdata[r]) {
        PMP_CUDA(h, cudaMemcpy(raw + (long long)(3 + r) * n, p->rdata[r], sizeof(double) * n, kind));
      } else {
        PMP_CUDA(h, cudaMemset(raw + (long long)(3 + r) * n, 0, sizeof(double) * n));
      }
    }
    if (!p->id) {
      cudaFree(raw);
      cudaFree(rid);
      return set_err(h, PMP_ERR_INVALID, "missing id array");
    }
    PMP_CUDA(h, cudaMemcpy(rid, p->id, sizeof(int) * n, kind));
  } else if (p->layout == PMP_LAYOUT_AOS) {
    const size_t rec = sizeof(double) * nc + 2 * sizeof(int);
    char* tmp = nullptr;
    PMP_CUDA(h, cudaMalloc(&tmp, rec * n));
    PMP_CUDA(h, cudaMemcpy(tmp, p->aos, rec * n, kind));
    k_aos_to_soa<<<nblk(n), 256>>>(tmp, n, nr, raw, rid);
    PMP_CUDA(h, cudaGetLastError());
    PMP_CUDA(h, cudaDeviceSynchronize());
    cudaFree(tmp);
  } else {
    cudaFree(raw);
    cudaFree(rid);
    return set_err(h, PMP_ERR_INVALID, "unknown particle layout");
  }
  // sort by the cell holding the droplet, in brick order (margin kSortPad
  // around the box)
  const pmp_box& bx = h->boxes[box];
  const int ext[3] = {bx.hi[0] - bx.lo[0] + 1 + 2 * kSortPad, bx.hi[1] - bx.lo[1] + 1 + 2 * kSortPad,
                      bx.hi[2] - bx.lo[2] + 1 + 2 * kSortPad};
  unsigned *keys = nullptr, *keys2 = nullptr;
  long long* idx = nullptr;
  PMP_CUDA(h, cudaMalloc(&keys, sizeof(unsigned) * n));
  PMP_CUDA(h, cudaMalloc(&keys2, sizeof(unsigned) * n));
  PMP_CUDA(h, cudaMalloc(&idx, sizeof(long long) * n));
  PMP_CUDA(h, cudaMalloc(&s.perm, sizeof(long long) * n));
  const pmp_geometry& g = h->geom;
  k_cell_keys<<<nblk(n), 256>>>(raw, raw + n, raw + 2 * n, n, g.plo[0], g.plo[1], g.plo[2],
                                1. / g.dx[0], 1. / g.dx[1], 1. / g.dx[2], bx.lo[0], bx.lo[1],
                                bx.lo[2], ext[0], ext[1], ext[2], keys, idx);
  PMP_CUDA(h, cudaGetLastError());
  size_t tbytes = 0;
  const long long maxkey = (long long)pmp::brick_key_count(ext[0], ext[1], ext[2]);
  if (maxkey >= (1LL << 32)) {
    cudaFree(raw);
    cudaFree(rid);
    cudaFree(keys);
    cudaFree(keys2);
    cudaFree(idx);
    return set_err(h, PMP_ERR_INVALID, "box too large for the droplet sort key", box);
  }
  int end_bit = 1;
  while ((1LL << end_bit) < maxkey && end_bit < 32) {
    ++end_bit;
  }
  PMP_CUDA(h, cub::DeviceRadixSort::SortPairs(nullptr, tbytes, keys, keys2, idx, s.perm, (int)n, 0, end_bit));
  void* tmp = nullptr;
  PMP_CUDA(h, cudaMalloc(&tmp, tbytes));
  PMP_CUDA(h, cub::DeviceRadixSort::SortPairs(tmp, tbytes, keys, keys2, idx, s.perm, (int)n, 0, end_bit));
  PMP_CUDA(h, cudaMalloc(&s.d, sizeof(double) * nc * n));
  PMP_CUDA(h, cudaMalloc(&s.id, sizeof(int) * n));
  k_gather<<<nblk(n), 256>>>(raw, rid, s.perm, n, nc, s.d, s.id);
  PMP_CUDA(h, cudaGetLastError());
  PMP_CUDA(h, cudaDeviceSynchronize());
  cudaFree(tmp);
  cudaFree(keys);
  cudaFree(keys2);
  cudaFree(idx);
  cudaFree(raw);
  cudaFree(rid);
  return PMP_OK;
}

int pmp_spray_num_particles(const pmp_spray* h, int box, long long* n)
{
  if (!h || !n || box < 0 || box >= (int)h->boxes.size()) {
    return PMP_ERR_INVALID;
  }
  *n = h->packed ? h->box_begin[box + 1] - h->box_begin[box] : h->staged[box].n;
  return PMP_OK;
}

int pmp_spray_get_particles(pmp_spray* h, int box, pmp_particles* out)
{
  if (!h || !out || box < 0 || box >= (int)h->boxes.size()) {
    return PMP_ERR_INVALID;
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  long long n = 0;
  pmp_spray_num_particles(h, box, &n);
  if (out->n != n) {
    return set_err(h, PMP_ERR_INVALID, "output count differs from the box's droplet count", box);
  }
  if (n == 0) {
    return PMP_OK;
  }
  const int nc = h->ncomp();
  const int nr = h->nr();
  double* d = nullptr;
  int* id = nullptr;
  PMP_CUDA(h, cudaMalloc(&d, sizeof(double) * nc * n));
  PMP_CUDA(h, cudaMalloc(&id, sizeof(int) * n));
  int rc = unsort_box(h, box, d, id, n);
  if (rc == PMP_OK) {
    const cudaMemcpyKind kind =
      out->where == PMP_WHERE_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (out->layout == PMP_LAYOUT_SOA) {
      for (int dd = 0; dd < 3; ++dd) {
        if (out->pos[dd]) {
          PMP_CUDA(h, cudaMemcpy(out->pos[dd], d + (long long)dd * n, sizeof(double) * n, kind));
        }
      }
      for (int r = 0; r < nr; ++r) {
        if (out->rdata[r]) {
          PMP_CUDA(h, cudaMemcpy(out->rdata[r], d + (long long)(3 + r) * n, sizeof(double) * n, kind));
        }
      }
      if (out->id) {
        PMP_CUDA(h, cudaMemcpy(out->id, id, sizeof(int) * n, kind));
      }
    } else {
      const size_t rec = sizeof(double) * nc + 2 * sizeof(int);
      char* tmp = nullptr;
      PMP_CUDA(h, cudaMalloc(&tmp, rec * n));
      k_soa_to_aos<<<nblk(n), 256>>>(d, id, n, nr, tmp);
      PMP_CUDA(h, cudaGetLastError());
      PMP_CUDA(h, cudaMemcpy(out->aos, tmp, rec * n, kind));
      cudaFree(tmp);
    }
  }
  cudaFree(d);
  cudaFree(id);
  return rc;
}

int pmp_spray_update(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes, double flow_dt,
  double time, int state_ghosts, int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, void* stream)
{
  (void)time;
  if (!h || (nboxes > 0 && (!state || !source))) {
    return PMP_ERR_INVALID;
  }
  cudaSetDevice(h->device);
  return do_update(h, state, source, nboxes, flow_dt, state_ghosts, source_ghosts, is_virt, is_ghost,
                   do_move, spray_cfl_lev, (cudaStream_t)stream);
}

int pmp_spray_update_host(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes, double flow_dt,
  double time, int state_ghosts, int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, void* stream)
{
  (void)time;
  if (!h || nboxes < 0 || (nboxes > 0 && (!state || !source))) {
    return PMP_ERR_INVALID;
  }
  cudaSetDevice(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (earlier_call_failed(h)) {
    return pmp::sync_status(h);
  }
  if ((int)h->stage_state.size() < nboxes) {
    h->stage_state.resize(nboxes, nullptr);
    h->stage_src.resize(nboxes, nullptr);
    h->stage_state_n.resize(nboxes, 0);
    h->stage_src_n.resize(nboxes, 0);
  }
  std::vector<pmp_box_view> dst(nboxes), dsr(nboxes);
  for (int b = 0; b < nboxes; ++b) {
    if (!state[b].p || !source[b].p || state[b].ncomp < 1 || source[b].ncomp < 1) {
      return set_err(h, PMP_ERR_INVALID, "null host view", b);
    }
    const size_t ns = view_extent(state[b]);
    const size_t nsr = view_extent(source[b]);
    if (h->stage_state_n[b] < ns || h->stage_src_n[b] < nsr) {
      pmp::quiesce(h);  // earlier calls' kernels may still read the staged views
    }
    if (h->stage_state_n[b] < ns) {
      cudaFree(h->stage_state[b]);
      h->stage_state[b] = nullptr;
      PMP_CUDA(h, cudaMalloc(&h->stage_state[b], sizeof(double) * ns));
      h->stage_state_n[b] = ns;
    }
    if (h->stage_src_n[b] < nsr) {
      cudaFree(h->stage_src[b]);
      h->stage_src[b] = nullptr;
      PMP_CUDA(h, cudaMalloc(&h->stage_src[b], sizeof(double) * nsr));
      h->stage_src_n[b] = nsr;
    }
    dst[b] = state[b];
    dst[b].p = h->stage_state[b];
    dsr[b] = source[b];
    dsr[b].p = h->stage_src[b];
  }
  // copies overlapped with the update, except for the FP64 form's launch
  // shapes and graphs and the learned form's audit (whole-map launches)
  const pmp_launch_config& lc = h->batch.cfg;
  const bool default_fp64 = lc.kind == PMP_LAUNCH_GRID && lc.block == 128 && lc.regs == 96 && !lc.use_graph;
  const bool overlapped = h->mode == PMP_MODE_MIXED ||
                          (h->mode == PMP_MODE_LEARNED && !pmp::learn_audit_on(h)) ||
                          (h->mode == PMP_MODE_FP64 && (h->pelec || default_fp64));
  if (overlapped) {
    return update_host_overlapped(h, state, source, dst.data(), dsr.data(), nboxes, flow_dt,
                                  state_ghosts, source_ghosts, is_ghost, do_move, spray_cfl_lev, st);
  }
  const auto st_runs = comp_runs(h, true);
  const auto sr_runs = comp_runs(h, false);
  for (int b = 0; b < nboxes; ++b) {
    if (st_runs.back().second > state[b].ncomp || sr_runs.back().second > source[b].ncomp ||
        st_runs.front().first < 0 || sr_runs.front().first < 0) {
      return set_err(h, PMP_ERR_INVALID, "a view has fewer components than the update reads", b);
    }
  }
  for (int b = 0; b < nboxes; ++b) {
    PMP_CUDA(h, copy_runs(dst[b].p, state[b].p, state[b], st_runs, cudaMemcpyHostToDevice, st));
    PMP_CUDA(h, source_in(dsr[b].p, source[b].p, source[b], sr_runs, h->host_src_in, st));
  }
  const int rc = do_update(h, dst.data(), dsr.data(), nboxes, flow_dt, state_ghosts, source_ghosts,
                           is_virt, is_ghost, do_move, spray_cfl_lev, st);
  if (rc != PMP_OK) {
    cudaStreamSynchronize(st);  // no copy of the caller's memory in flight on return
    return rc;
  }
  for (int b = 0; b < nboxes; ++b) {
    PMP_CUDA(h, copy_runs(source[b].p, h->stage_src[b], source[b], sr_runs, cudaMemcpyDeviceToHost, st));
  }
  return mark_enqueued(h, st);
}

int pmp_spray_set_host_source_in(pmp_spray* h, int copy_in)
{
  if (!h || (copy_in != 0 && copy_in != 1)) {
    return PMP_ERR_INVALID;
  }
  h->host_src_in = copy_in;
  return PMP_OK;
}

int pmp_spray_move_kick_drift(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes, double dt,
  double time, int is_virt, int is_ghost, int state_ghosts, int source_ghosts, int do_move,
  double spray_cfl_lev, void* stream)
{
  return pmp_spray_update(h, state, source, nboxes, dt, time, state_ghosts, source_ghosts, is_virt,
                          is_ghost, do_move, spray_cfl_lev, stream);
}

int pmp_spray_move_kick(
  pmp_spray* h, const pmp_box_view* state, const pmp_box_view* source, int nboxes, double dt,
  double time, int is_virt, int is_ghost, int state_ghosts, int source_ghosts, double spray_cfl_lev,
  void* stream)
{
  return pmp_spray_update(h, state, source, nboxes, dt, time, state_ghosts, source_ghosts, is_virt,
                          is_ghost, 0, spray_cfl_lev, stream);
}

int pmp_spray_set_mode(pmp_spray* h, int mode)
{
  if (!h || mode < PMP_MODE_FP64 || mode > PMP_MODE_LEARNED) {
    return PMP_ERR_INVALID;
  }
  h->mode = mode;
  return PMP_OK;
}

int pmp_spray_set_coupling(pmp_spray* h, int coupling)
{
  if (!h || (coupling != PMP_COUPLING_LMEX && coupling != PMP_COUPLING_PELEC)) {
    return PMP_ERR_INVALID;
  }
  if (h->have_data && coupling != h->pelec) {
    return set_err(h, PMP_ERR_INVALID, "set the coupling before the spray data");
  }
  h->pelec = coupling;
  return PMP_OK;
}

int pmp_spray_get_coupling(const pmp_spray* h, int* coupling)
{
  if (!h || !coupling) {
    return PMP_ERR_INVALID;
  }
  *coupling = h->pelec;
  return PMP_OK;
}

int pmp_spray_sync(pmp_spray* h)
{
  if (!h) {
    return PMP_ERR_INVALID;
  }
  cudaSetDevice(h->device);
  return pmp::sync_status(h);
}

int pmp_spray_last_error(const pmp_spray* h, pmp_error_info* info)
{
  if (!h || !info) {
    return PMP_ERR_INVALID;
  }
  *info = h->last_err;
  return PMP_OK;
}

int pmp_spray_get_stats(const pmp_spray* h, pmp_stats* stats)
{
  if (!h || !stats) {
    return PMP_ERR_INVALID;
  }
  *stats = h->stats;
  return PMP_OK;
}

}  // extern "C"
