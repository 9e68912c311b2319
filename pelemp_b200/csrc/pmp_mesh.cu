// pmp_mesh.cu -- the operations on either side of the update that a time step
// of the host code needs every step, on the device:
//  * estTimestep (SprayParticles.cpp:89-140): particle CFL time step, a min
//    reduction over the droplets;
//  * computeDerivedVars (SprayDerive.cpp:9-155): droplet mass, number,
//    volume, surface, d10, d32, temperature and velocity fields by atomic
//    deposition into the cell holding each droplet, then the protected
//    divisions;
//  * transferSource (SprayParticles.H:250-319), level 0: the source ghost
//    fold (SumBoundary with periodicity), the add into the caller's state
//    source (MultiFab::Add or addSpraySrc), and the reset of the temporary;
//  * redistribute: after a move, droplets are re-binned to the box whose
//    valid region holds their cell, positions wrapped across periodic faces,
//    and dead droplets (id <= 0) dropped -- what AMReX's Redistribute does for
//    this container.  AMReX is not in the reference tree, so its periodic
//    shift is restated here as: while x >= phi, x -= L; while x < plo, x += L
//    (periodic directions only); a droplet whose cell lies in no box is dropped.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pmp_handle.h"
#include "spray_fp64.cuh"

namespace pmp {

namespace {

struct View32 {
  double* p;
  int lo[3], hi[3];
  int js, ks, ns;
  int ncomp;
};

int check(pmp_spray* h, cudaError_t e, const char* what)
{
  if (e != cudaSuccess) {
    char b[160];
    snprintf(b, sizeof(b), "%s: %s", what, cudaGetErrorString(e));
    return set_err(h, PMP_ERR_CUDA, b);
  }
  return PMP_OK;
}

#define PMP_TRY(h, call)                        \
  do {                                          \
    const int rc_ = check((h), (call), #call);  \
    if (rc_ != PMP_OK) {                        \
      return rc_;                               \
    }                                           \
  } while (0)

inline unsigned nblk(long long n, int b = 256) { return (unsigned)std::max(1LL, (n + b - 1) / b); }

long long view_elems(const pmp_box_view& v)
{
  return (long long)(v.hi[0] - v.lo[0]) + (long long)(v.hi[1] - v.lo[1]) * v.jstride +
         (long long)(v.hi[2] - v.lo[2]) * v.kstride + (long long)(v.ncomp - 1) * v.nstride + 1;
}

int to_view32(pmp_spray* h, const pmp_box_view& v, View32& o)
{
  if (!v.p || v.ncomp < 1 || view_elems(v) >= (1LL << 31)) {
    return set_err(h, PMP_ERR_INVALID, "view is empty or spans 2^31 elements or more");
  }
  o.p = v.p;
  for (int d = 0; d < 3; ++d) {
    o.lo[d] = v.lo[d];
    o.hi[d] = v.hi[d];
  }
  o.js = (int)v.jstride;
  o.ks = (int)v.kstride;
  o.ns = (int)v.nstride;
  o.ncomp = v.ncomp;
  return PMP_OK;
}

__device__ __forceinline__ bool inside(const View32& v, int i, int j, int k)
{
  return i >= v.lo[0] && i <= v.hi[0] && j >= v.lo[1] && j <= v.hi[1] && k >= v.lo[2] && k <= v.hi[2];
}

__device__ __forceinline__ double* at(const View32& v, int i, int j, int k, int n)
{
  return v.p + ((i - v.lo[0]) + (j - v.lo[1]) * v.js + (k - v.lo[2]) * v.ks + n * v.ns);
}

// item -> (box, local index) over a prefix of per-box counts
__device__ __forceinline__ int find_box(const long long* prefix, int nb, long long i)
{
  int lo = 0, hi = nb;
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (prefix[mid] <= i) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  return lo;
}

// the handle's scratch for the small per-call tables of this file
int scratch(pmp_spray* h, size_t bytes, void** out)
{
  if (h->mesh_scratch_bytes < bytes) {
    cudaFree(h->mesh_scratch);
    h->mesh_scratch = nullptr;
    h->mesh_scratch_bytes = 0;
    PMP_TRY(h, cudaMalloc(&h->mesh_scratch, bytes));
    h->mesh_scratch_bytes = bytes;
  }
  *out = h->mesh_scratch;
  return PMP_OK;
}

// --------------------------------------------------------------------------
// cell -> box map over the domain

__global__ void k_fill_box_map(int* map, int b, int lo0, int lo1, int lo2, int nx, int ny, int nz, int dlo0, int dlo1,
                               int dlo2, int dnx, int dny)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nx * ny * nz) {
    return;
  }
  const int i = lo0 + (int)(t % nx);
  const int j = lo1 + (int)((t / nx) % ny);
  const int k = lo2 + (int)(t / ((long long)nx * ny));
  map[(long long)(k - dlo2) * dny * dnx + (long long)(j - dlo1) * dnx + (i - dlo0)] = b;
}

int ensure_box_map(pmp_spray* h, cudaStream_t st)
{
  if (h->box_map_version == h->grids_version && h->d_box_map) {
    return PMP_OK;
  }
  const pmp_geometry& g = h->geom;
  const long long dnx = g.domain_hi[0] - g.domain_lo[0] + 1;
  const long long dny = g.domain_hi[1] - g.domain_lo[1] + 1;
  const long long dnz = g.domain_hi[2] - g.domain_lo[2] + 1;
  const long long ncell = dnx * dny * dnz;
  cudaFree(h->d_box_map);
  h->d_box_map = nullptr;
  PMP_TRY(h, cudaMalloc(&h->d_box_map, sizeof(int) * ncell));
  PMP_TRY(h, cudaMemsetAsync(h->d_box_map, 0xff, sizeof(int) * ncell, st));  // -1: no box
  for (int b = 0; b < (int)h->boxes.size(); ++b) {
    const pmp_box& bx = h->boxes[b];
    for (int d = 0; d < 3; ++d) {
      if (bx.lo[d] < g.domain_lo[d] || bx.hi[d] > g.domain_hi[d]) {
        return set_err(h, PMP_ERR_INVALID, "box outside the domain", b);
      }
    }
    const int nx = bx.hi[0] - bx.lo[0] + 1, ny = bx.hi[1] - bx.lo[1] + 1, nz = bx.hi[2] - bx.lo[2] + 1;
    k_fill_box_map<<<nblk((long long)nx * ny * nz), 256, 0, st>>>(h->d_box_map, b, bx.lo[0], bx.lo[1], bx.lo[2], nx,
                                                                    ny, nz, g.domain_lo[0], g.domain_lo[1],
                                                                    g.domain_lo[2], (int)dnx, (int)dny);
  }
  PMP_TRY(h, cudaGetLastError());
  h->box_map_version = h->grids_version;
  return PMP_OK;
}

struct Domain {
  int lo[3], n[3];
  int periodic[3];
};

Domain domain_of(const pmp_spray* h)
{
  Domain D;
  for (int d = 0; d < 3; ++d) {
    D.lo[d] = h->geom.domain_lo[d];
    D.n[d] = h->geom.domain_hi[d] - h->geom.domain_lo[d] + 1;
    D.periodic[d] = h->geom.bndry_lo[d] == 0;
  }
  return D;
}

// box whose valid region holds cell (i,j,k) after periodic wrap; -1 if none
__device__ __forceinline__ int owner(const int* map, const Domain& D, int* c)
{
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int r = c[d] - D.lo[d];
    if (D.periodic[d]) {
      r %= D.n[d];
      r += r < 0 ? D.n[d] : 0;
    } else if (r < 0 || r >= D.n[d]) {
      return -1;
    }
    c[d] = D.lo[d] + r;
  }
  return map[((long long)(c[2] - D.lo[2]) * D.n[1] + (c[1] - D.lo[1])) * D.n[0] + (c[0] - D.lo[0])];
}

// --------------------------------------------------------------------------
// estTimestep

__global__ void k_est_dt(const double* vx, const double* vy, const double* vz, const int* id, long long n,
                         double dxi0, double dxi1, double dxi2, double cfl, double* partial)
{
  double m = DBL_MAX;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = -1.;
    if (id[i] > 0) {
      const double mv = fmax(fmax(fabs(vx[i]) * dxi0, fabs(vy[i]) * dxi1), fabs(vz[i]) * dxi2);
      v = mv > 0. ? cfl / mv : 1.E50;
    }
    m = fmin(m, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
  }
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      r = fmin(r, red[w]);
    }
    partial[blockIdx.x] = r;
  }
}

// --------------------------------------------------------------------------
// computeDerivedVars

struct DeriveArgs {
  const double* pos[3];
  const double* vel[3];
  const double* T;
  const double* dia;
  const double* Y[PMP_MAX_FUEL];
  const double* numdens;
  const double* film;
  const int* id;
  long long n;
  const long long* box_begin;
  int nboxes;
  const View32* views;
  int start;
  int species;  // deposit the per-fuel liquid masses
  int nf;
  double rho_coef[4 * PMP_MAX_FUEL];
  double plo[3], dx[3], dxi[3];
  double cell_vol;
  int* error;  // first slot whose cell the view does not hold (+1), 0 if none
};

// component offsets (relative to start) in the reference's order
enum { kMass = 0, kDens, kNum, kVol, kSurf, kVolf, kD10, kD32, kWfh, kWfm, kTemp, kNump, kVel, kSpec = kVel + 3 };

__global__ void k_derive(const DeriveArgs A)
{
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= A.n || !(A.id[s] > 0)) {
    return;
  }
  const int b = find_box(A.box_begin, A.nboxes, s);
  const View32& V = A.views[b];
  int c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c[d] = static_cast<int>(floor(__dmul_rn(__dsub_rn(A.pos[d][s], A.plo[d]), A.dxi[d])));
  }
  if (!inside(V, c[0], c[1], c[2])) {
    atomicCAS(A.error, 0, (int)min(s + 1, 0x7fffffffLL));
    return;
  }
  const double T_part = A.T[s];
  const double dia_part = A.dia[s];
  double rho_part = 0.;
  for (int spf = 0; spf < A.nf; ++spf) {
    const double* rc = A.rho_coef + 4 * spf;
    rho_part += A.Y[spf][s] / (rc[0] + T_part * (rc[1] + T_part * (rc[2] + T_part * rc[3])));
  }
  rho_part = 1. / rho_part;
  const double surf = PMP_PI * dia_part * dia_part;
  const double vol = PMP_PI / 6. * (dia_part * dia_part * dia_part);
  const double pmass = vol * rho_part;
  const double num_ppp = A.numdens[s];
  const double curvol = A.cell_vol;
  const double face_area = A.dx[0] * A.dx[0];
  const double film = A.film[s];
  auto add = [&](int comp, double v) { atomicAdd(at(V, c[0], c[1], c[2], A.start + comp), v); };
  if (film == 0.) {
    add(kMass, num_ppp * pmass);
    add(kDens, num_ppp * pmass / curvol);
    add(kNum, num_ppp);
    add(kVol, num_ppp * vol);
    add(kSurf, num_ppp * surf);
    add(kVolf, num_ppp * vol / curvol);
    add(kD10, num_ppp * dia_part);
    add(kD32, num_ppp * vol * 6.);
    add(kTemp, num_ppp * pmass * T_part);
    add(kNump, 1.);
    for (int d = 0; d < 3; ++d) {
      add(kVel + d, num_ppp * pmass * A.vel[d][s]);
    }
    if (A.species) {
      for (int spf = 0; spf < A.nf; ++spf) {
        add(kSpec + spf, A.Y[spf][s] * pmass);  // no parcel count, as the reference
      }
    }
  } else {
    const double rad2 = (0.5 * dia_part) * (0.5 * dia_part);
    const double cur_vol = PMP_PI / 6. * film * (3. * rad2 + film * film);
    add(kWfh, cur_vol / face_area);
    add(kWfm, rho_part * cur_vol);
  }
}

// FArrayBox::protected_divide over every cell of each view (ghost cells too)
__global__ void k_protected_divide(const View32* views, const long long* prefix, int nb, long long total, int start)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= total) {
    return;
  }
  const int b = find_box(prefix, nb, t);
  const View32& V = views[b];
  const long long l = t - prefix[b];
  const int nx = V.hi[0] - V.lo[0] + 1, ny = V.hi[1] - V.lo[1] + 1;
  const int i = V.lo[0] + (int)(l % nx);
  const int j = V.lo[1] + (int)((l / nx) % ny);
  const int k = V.lo[2] + (int)(l / ((long long)nx * ny));
  const int pairs[6][2] = {{kNum, kD10}, {kSurf, kD32}, {kMass, kTemp}, {kMass, kVel}, {kMass, kVel + 1}, {kMass, kVel + 2}};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const double den = *at(V, i, j, k, start + pairs[q][0]);
    if (den != 0.) {
      double* num = at(V, i, j, k, start + pairs[q][1]);
      *num = *num / den;
    }
  }
}

// --------------------------------------------------------------------------
// transferSource

// SumBoundary: every ghost cell of every box adds into the valid cell that
// owns its (periodically wrapped) location
__global__ void k_sum_boundary(const View32* tmp, const pmp_box* boxes, const long long* prefix, int nb,
                               long long total, int g, const int* map, Domain D, int ncomp)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= total) {
    return;
  }
  const int b = find_box(prefix, nb, t);
  const pmp_box& bx = boxes[b];
  const long long l = t - prefix[b];
  const int nx = bx.hi[0] - bx.lo[0] + 1 + 2 * g, ny = bx.hi[1] - bx.lo[1] + 1 + 2 * g;
  const int i = bx.lo[0] - g + (int)(l % nx);
  const int j = bx.lo[1] - g + (int)((l / nx) % ny);
  const int k = bx.lo[2] - g + (int)(l / ((long long)nx * ny));
  if (i >= bx.lo[0] && i <= bx.hi[0] && j >= bx.lo[1] && j <= bx.hi[1] && k >= bx.lo[2] && k <= bx.hi[2]) {
    return;  // valid cell: a destination, not a source
  }
  int c[3] = {i, j, k};
  const int o = owner(map, D, c);
  if (o < 0) {
    return;
  }
  const View32& S = tmp[b];
  const View32& T = tmp[o];
  for (int n = 0; n < ncomp; ++n) {
    const double v = *at(S, i, j, k, n);
    if (v != 0.) {
      atomicAdd(at(T, c[0], c[1], c[2], n), v);
    }
  }
}

struct AddMap {
  int same;  // add every component
  int mom_src, rho_src, eng_src, spec_src;
  int mom, rho, eng, spec;
  int nf;
  int dep[PMP_MAX_FUEL];
};

// MultiFab::Add or addSpraySrc over each box grown by nghost
__global__ void k_add_source(const View32* tmp, const View32* act, const pmp_box* boxes, const long long* prefix, int nb,
                             long long total, int ng, const AddMap M)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= total) {
    return;
  }
  const int b = find_box(prefix, nb, t);
  const pmp_box& bx = boxes[b];
  const long long l = t - prefix[b];
  const int nx = bx.hi[0] - bx.lo[0] + 1 + 2 * ng, ny = bx.hi[1] - bx.lo[1] + 1 + 2 * ng;
  const int i = bx.lo[0] - ng + (int)(l % nx);
  const int j = bx.lo[1] - ng + (int)((l / nx) % ny);
  const int k = bx.lo[2] - ng + (int)(l / ((long long)nx * ny));
  const View32& S = tmp[b];
  const View32& A = act[b];
  if (M.same) {
    for (int n = 0; n < A.ncomp; ++n) {
      *at(A, i, j, k, n) += *at(S, i, j, k, n);
    }
    return;
  }
  for (int d = 0; d < 3; ++d) {
    *at(A, i, j, k, M.mom + d) += *at(S, i, j, k, M.mom_src + d);
  }
  *at(A, i, j, k, M.rho) += *at(S, i, j, k, M.rho_src);
  *at(A, i, j, k, M.eng) += *at(S, i, j, k, M.eng_src);
  for (int sp = 0; sp < M.nf; ++sp) {
    *at(A, i, j, k, M.spec + M.dep[sp]) += *at(S, i, j, k, M.spec_src + sp);
  }
}

__global__ void k_zero_views(const View32* v, const long long* prefix, int nb, long long total)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= total) {
    return;
  }
  const int b = find_box(prefix, nb, t);
  const View32& V = v[b];
  const long long l = t - prefix[b];
  const int nx = V.hi[0] - V.lo[0] + 1, ny = V.hi[1] - V.lo[1] + 1, nz = V.hi[2] - V.lo[2] + 1;
  const long long cells = (long long)nx * ny * nz;
  const int n = (int)(l / cells);
  const long long r = l % cells;
  *at(V, V.lo[0] + (int)(r % nx), V.lo[1] + (int)((r / nx) % ny), V.lo[2] + (int)(r / ((long long)nx * ny)), n) = 0.;
}

// --------------------------------------------------------------------------
// redistribute

// Sort key of a droplet: its new box o above `shift` bits of its cell's
// place in the box's sort order (pmp::brick_key); dead droplets and droplets
// in no box get box nb, so that they sort last.  K / V: 32-bit keys and slot
// indices when the key fits 32 bits and the count 2^31, else 64-bit.
template <typename K, typename V>
__global__ void k_rebin_keys(double* px, double* py, double* pz, const int* id, long long n, const int* map, Domain D,
                             double plo0, double plo1, double plo2, double phi0, double phi1, double phi2, double dxi0,
                             double dxi1, double dxi2, const pmp_box* boxes, int nb, int shift, K* keys, V* idx)
{
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) {
    return;
  }
  idx[s] = (V)s;
  const K dead = (K)nb << shift;
  if (!(id[s] > 0)) {
    keys[s] = dead;
    return;
  }
  double* p[3] = {px, py, pz};
  const double plo[3] = {plo0, plo1, plo2}, phi[3] = {phi0, phi1, phi2}, dxi[3] = {dxi0, dxi1, dxi2};
  int c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double x = p[d][s];
    if (D.periodic[d]) {
      const double L = phi[d] - plo[d];
      const double x0 = x;
      for (int it = 0; it < 64 && x >= phi[d]; ++it) {
        x -= L;
      }
      for (int it = 0; it < 64 && x < plo[d]; ++it) {
        x += L;
      }
      if (x != x0) {
        p[d][s] = x;
      }
    }
    c[d] = static_cast<int>(floor(__dmul_rn(__dsub_rn(x, plo[d]), dxi[d])));
  }
  const int o = owner(map, D, c);
  if (o < 0) {
    keys[s] = dead;
    return;
  }
  const pmp_box& bx = boxes[o];
  const int ex = bx.hi[0] - bx.lo[0] + 1, ey = bx.hi[1] - bx.lo[1] + 1;
  const unsigned long long local = pmp::brick_key(c[0] - bx.lo[0], c[1] - bx.lo[1], c[2] - bx.lo[2], ex, ey);
  keys[s] = ((K)o << shift) | (K)local;
}

// begin[b]: the first sorted position of box b (b = nb: the dead)
template <typename K>
__global__ void k_box_bounds(const K* keys, long long n, int nb, int shift, long long* begin)
{
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > nb) {
    return;
  }
  const K key = (K)b << shift;
  long long lo = 0, hi = n;  // first index with keys[i] >= key
  while (lo < hi) {
    const long long mid = (lo + hi) / 2;
    if (keys[mid] < key) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  begin[b] = lo;
}

template <typename V>
__global__ void k_gather_soa(const double* src, long long stride_src, const int* sid, const V* perm, long long n,
                             int ncomp, double* dst, int* did)
{
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) {
    return;
  }
  const long long j = (long long)perm[s];
  for (int c = 0; c < ncomp; ++c) {
    dst[c * n + s] = src[c * stride_src + j];
  }
  did[s] = sid[j];
}

// perm[s] = s - begin[b] for the slots s of box b (the re-binned order is
// each box's caller order)
__global__ void k_rebin_perm(long long* perm, const long long* begin, int nb, long long n)
{
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) {
    return;
  }
  int lo = 0, hi = nb;  // the box b with begin[b] <= s < begin[b + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (begin[mid] <= s) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  perm[s] = s - begin[lo];
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Offsets of the re-binning's working arrays in the handle's rebin_scratch:
// keys, sorted keys, slot indices, sorted indices (the gather order), box
// bounds, the box list, CUB's temporary storage.
struct RebinLayout {
  size_t keys2, idx, perm, begin, boxes, tmp, total;
};
RebinLayout rebin_layout(long long n, int nb, size_t kbytes, size_t vbytes, size_t tbytes)
{
  const size_t cap = (size_t)std::max(n, 1LL);
  RebinLayout L;
  L.keys2 = align256(kbytes * cap);
  L.idx = L.keys2 + align256(kbytes * cap);
  L.perm = L.idx + align256(vbytes * cap);
  L.begin = L.perm + align256(vbytes * cap);
  L.boxes = L.begin + align256(sizeof(long long) * (nb + 1));
  L.tmp = L.boxes + align256(sizeof(pmp_box) * std::max(nb, 1));
  L.total = L.tmp + align256(std::max(tbytes, (size_t)1));
  return L;
}

}  // namespace

void mesh_free(pmp_spray* h)
{
  cudaFree(h->d_box_map);
  h->d_box_map = nullptr;
  h->box_map_version = -1;
  cudaFree(h->mesh_scratch);
  h->mesh_scratch = nullptr;
  h->mesh_scratch_bytes = 0;
  cudaFree(h->rebin_scratch);
  h->rebin_scratch = nullptr;
  h->rebin_scratch_bytes = 0;
}

}  // namespace pmp

using namespace pmp;

extern "C" int pmp_spray_est_timestep(pmp_spray* h, double cfl, double max_jet_vel, double* dt, void* stream)
{
  if (!h || !dt) {
    return PMP_ERR_INVALID;
  }
  if (!h->have_data || !h->have_geom) {
    return set_err(h, PMP_ERR_INVALID, "setup and geometry must be set first");
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  cudaStream_t st = (cudaStream_t)stream;
  if (h->data.fixed_parts) {
    *dt = -1.;
    return PMP_OK;
  }
  int rc = ensure_packed(h);
  if (rc != PMP_OK) {
    return rc;
  }
  const pmp_geometry& g = h->geom;
  double r = DBL_MAX;
  const long long n = h->total;
  if (n > 0) {
    const int nblocks = (int)std::min<long long>(nblk(n, 256), 148 * 8);
    void* sp = nullptr;
    rc = scratch(h, sizeof(double) * nblocks, &sp);
    if (rc != PMP_OK) {
      return rc;
    }
    double* partial = static_cast<double*>(sp);
    const double* vel = h->soa + 3 * n;  // rdata component 0 follows the positions
    k_est_dt<<<nblocks, 256, 0, st>>>(vel, vel + n, vel + 2 * n, h->ids, n, 1. / g.dx[0], 1. / g.dx[1], 1. / g.dx[2],
                                      cfl, partial);
    std::vector<double> hp(nblocks);
    PMP_TRY(h, cudaMemcpyAsync(hp.data(), partial, sizeof(double) * nblocks, cudaMemcpyDeviceToHost, st));
    PMP_TRY(h, cudaStreamSynchronize(st));
    for (double v : hp) {
      r = std::min(r, v);
    }
  }
  if (max_jet_vel > 0.) {
    r = std::min(r, cfl * g.dx[0] / max_jet_vel);
  }
  *dt = r;
  return PMP_OK;
}

extern "C" int pmp_spray_derive(pmp_spray* h, const pmp_box_view* vars, int nboxes, int start_indx, int with_species,
                                void* stream)
{
  if (!h || !vars || nboxes != (int)h->boxes.size() || start_indx < 0) {
    return set_err(h, PMP_ERR_INVALID, "bad arguments to pmp_spray_derive");
  }
  if (!h->have_data || !h->have_geom) {
    return set_err(h, PMP_ERR_INVALID, "setup and geometry must be set first");
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_packed(h);
  if (rc != PMP_OK) {
    return rc;
  }
  const int nf = h->nfuel;
  const int nvar = kSpec + ((with_species && nf > 1) ? nf : 0);
  std::vector<View32> hv(nboxes);
  std::vector<long long> prefix(nboxes + 1, 0);
  for (int b = 0; b < nboxes; ++b) {
    rc = to_view32(h, vars[b], hv[b]);
    if (rc != PMP_OK) {
      return rc;
    }
    if (vars[b].ncomp < start_indx + nvar) {
      return set_err(h, PMP_ERR_INVALID, "derive view has too few components", b);
    }
    const long long cells = (long long)(vars[b].hi[0] - vars[b].lo[0] + 1) * (vars[b].hi[1] - vars[b].lo[1] + 1) *
                            (vars[b].hi[2] - vars[b].lo[2] + 1);
    prefix[b + 1] = prefix[b] + cells;
  }
  const size_t need = sizeof(View32) * nboxes + sizeof(long long) * (nboxes + 1) + 16;
  void* sp = nullptr;
  rc = scratch(h, need, &sp);
  if (rc != PMP_OK) {
    return rc;
  }
  int* d_err = static_cast<int*>(sp);
  View32* d_views = reinterpret_cast<View32*>(static_cast<char*>(sp) + 16);
  long long* d_prefix = reinterpret_cast<long long*>(d_views + nboxes);
  PMP_TRY(h, cudaMemsetAsync(d_err, 0, sizeof(int), st));
  PMP_TRY(h, cudaMemcpyAsync(d_views, hv.data(), sizeof(View32) * nboxes, cudaMemcpyHostToDevice, st));
  PMP_TRY(h, cudaMemcpyAsync(d_prefix, prefix.data(), sizeof(long long) * (nboxes + 1), cudaMemcpyHostToDevice, st));
  const long long n = h->total;
  const pmp_geometry& g = h->geom;
  DeriveArgs A;
  memset(&A, 0, sizeof(A));
  for (int d = 0; d < 3; ++d) {
    A.pos[d] = h->soa + (long long)d * n;
    A.vel[d] = h->soa + (long long)(3 + PMP_PSTATE_VEL + d) * n;
    A.plo[d] = g.plo[d];
    A.dx[d] = g.dx[d];
    A.dxi[d] = 1. / g.dx[d];
  }
  A.T = h->soa + (long long)(3 + PMP_PSTATE_T) * n;
  A.dia = h->soa + (long long)(3 + PMP_PSTATE_DIA) * n;
  for (int f = 0; f < nf; ++f) {
    A.Y[f] = h->soa + (long long)(3 + PMP_PSTATE_Y + f) * n;
  }
  A.numdens = h->soa + (long long)(3 + PMP_PSTATE_NUMDENS(nf)) * n;
  A.film = h->soa + (long long)(3 + PMP_PSTATE_FILMHGHT(nf)) * n;
  A.id = h->ids;
  A.n = n;
  A.box_begin = h->d_box_begin;
  A.nboxes = nboxes;
  A.views = d_views;
  A.start = start_indx;
  A.species = with_species && nf > 1;
  A.nf = nf;
  for (int i = 0; i < 4 * nf; ++i) {
    A.rho_coef[i] = h->data.rho_coef[i];
  }
  A.cell_vol = g.dx[0] * g.dx[1] * g.dx[2];
  A.error = d_err;
  if (n > 0) {
    k_derive<<<nblk(n, 128), 128, 0, st>>>(A);
  }
  if (prefix[nboxes] > 0) {
    k_protected_divide<<<nblk(prefix[nboxes]), 256, 0, st>>>(d_views, d_prefix, nboxes, prefix[nboxes], start_indx);
  }
  int herr = 0;
  PMP_TRY(h, cudaGetLastError());
  PMP_TRY(h, cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  PMP_TRY(h, cudaStreamSynchronize(st));
  if (herr != 0) {
    return set_err(h, PMP_ERR_SOURCE_BOX, "derive view does not hold a droplet's cell", -1, herr - 1);
  }
  return PMP_OK;
}

extern "C" int pmp_spray_transfer_source(pmp_spray* h, const pmp_box_view* tmp_source, const pmp_box_view* act_source,
                                         int nboxes, int source_ghosts, int act_ghosts, void* stream)
{
  if (!h || !tmp_source || !act_source || nboxes != (int)h->boxes.size() || source_ghosts < 0 || act_ghosts < 0) {
    return set_err(h, PMP_ERR_INVALID, "bad arguments to pmp_spray_transfer_source");
  }
  if (!h->have_geom || !h->have_comps || !h->have_data) {
    return set_err(h, PMP_ERR_INVALID, "setup, comps and geometry must be set first");
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_box_map(h, st);
  if (rc != PMP_OK) {
    return rc;
  }
  const int g = source_ghosts;
  const int ng = std::min(act_ghosts, source_ghosts);
  std::vector<View32> ht(nboxes), ha(nboxes);
  std::vector<long long> pg(nboxes + 1, 0), pa(nboxes + 1, 0), pz(nboxes + 1, 0);
  int ncomp = -1;
  for (int b = 0; b < nboxes; ++b) {
    const pmp_box& bx = h->boxes[b];
    if ((rc = to_view32(h, tmp_source[b], ht[b])) != PMP_OK || (rc = to_view32(h, act_source[b], ha[b])) != PMP_OK) {
      return rc;
    }
    for (int d = 0; d < 3; ++d) {
      if (tmp_source[b].lo[d] > bx.lo[d] - g || tmp_source[b].hi[d] < bx.hi[d] + g) {
        return set_err(h, PMP_ERR_INVALID, "source view does not cover the box grown by source_ghosts", b);
      }
      if (act_source[b].lo[d] > bx.lo[d] - ng || act_source[b].hi[d] < bx.hi[d] + ng) {
        return set_err(h, PMP_ERR_INVALID, "destination view does not cover the box grown by its ghosts", b);
      }
    }
    if (ncomp < 0) {
      ncomp = tmp_source[b].ncomp;
    } else if (ncomp != tmp_source[b].ncomp) {
      return set_err(h, PMP_ERR_INVALID, "source views differ in component count", b);
    }
    auto cells = [&](int grow) {
      return (long long)(bx.hi[0] - bx.lo[0] + 1 + 2 * grow) * (bx.hi[1] - bx.lo[1] + 1 + 2 * grow) *
             (bx.hi[2] - bx.lo[2] + 1 + 2 * grow);
    };
    pg[b + 1] = pg[b] + cells(g);
    pa[b + 1] = pa[b] + cells(ng);
    const pmp_box_view& v = tmp_source[b];
    pz[b + 1] = pz[b] + (long long)(v.hi[0] - v.lo[0] + 1) * (v.hi[1] - v.lo[1] + 1) * (v.hi[2] - v.lo[2] + 1) * v.ncomp;
  }
  const pmp_spray_comps& c = h->comps;
  AddMap M;
  memset(&M, 0, sizeof(M));
  M.same = 1;
  for (int b = 0; b < nboxes; ++b) {
    M.same = M.same && act_source[b].ncomp == tmp_source[b].ncomp;
  }
  M.mom_src = c.momSrcIndx;
  M.rho_src = c.rhoSrcIndx;
  M.eng_src = c.engSrcIndx;
  M.spec_src = c.specSrcIndx;
  M.mom = c.momIndx;
  M.rho = c.rhoIndx;
  M.eng = c.engIndx;
  M.spec = c.specIndx;
  M.nf = h->nfuel;
  for (int f = 0; f < h->nfuel; ++f) {
    M.dep[f] = h->data.dep_indx[f];
  }
  if (!M.same) {
    const int need_src = 1 + std::max({c.momSrcIndx + 2, c.rhoSrcIndx, c.engSrcIndx, c.specSrcIndx + h->nfuel - 1});
    int need_act = 1 + std::max({c.momIndx + 2, c.rhoIndx, c.engIndx});
    for (int f = 0; f < h->nfuel; ++f) {
      need_act = std::max(need_act, c.specIndx + h->data.dep_indx[f] + 1);
    }
    for (int b = 0; b < nboxes; ++b) {
      if (tmp_source[b].ncomp < need_src || act_source[b].ncomp < need_act) {
        return set_err(h, PMP_ERR_INVALID, "views lack the source or state components", b);
      }
    }
  }
  const size_t need = 2 * sizeof(View32) * nboxes + 3 * sizeof(long long) * (nboxes + 1) + sizeof(pmp_box) * nboxes;
  void* sp = nullptr;
  if ((rc = scratch(h, need, &sp)) != PMP_OK) {
    return rc;
  }
  View32* d_t = static_cast<View32*>(sp);
  View32* d_a = d_t + nboxes;
  long long* d_pg = reinterpret_cast<long long*>(d_a + nboxes);
  long long* d_pa = d_pg + nboxes + 1;
  long long* d_pz = d_pa + nboxes + 1;
  pmp_box* d_boxes = reinterpret_cast<pmp_box*>(d_pz + nboxes + 1);
  PMP_TRY(h, cudaMemcpyAsync(d_t, ht.data(), sizeof(View32) * nboxes, cudaMemcpyHostToDevice, st));
  PMP_TRY(h, cudaMemcpyAsync(d_a, ha.data(), sizeof(View32) * nboxes, cudaMemcpyHostToDevice, st));
  PMP_TRY(h, cudaMemcpyAsync(d_pg, pg.data(), sizeof(long long) * (nboxes + 1), cudaMemcpyHostToDevice, st));
  PMP_TRY(h, cudaMemcpyAsync(d_pa, pa.data(), sizeof(long long) * (nboxes + 1), cudaMemcpyHostToDevice, st));
  PMP_TRY(h, cudaMemcpyAsync(d_pz, pz.data(), sizeof(long long) * (nboxes + 1), cudaMemcpyHostToDevice, st));
  PMP_TRY(h, cudaMemcpyAsync(d_boxes, h->boxes.data(), sizeof(pmp_box) * nboxes, cudaMemcpyHostToDevice, st));
  const Domain D = domain_of(h);
  if (g > 0 && pg[nboxes] > 0) {
    k_sum_boundary<<<nblk(pg[nboxes]), 256, 0, st>>>(d_t, d_boxes, d_pg, nboxes, pg[nboxes], g, h->d_box_map, D, ncomp);
  }
  if (pa[nboxes] > 0) {
    k_add_source<<<nblk(pa[nboxes]), 256, 0, st>>>(d_t, d_a, d_boxes, d_pa, nboxes, pa[nboxes], ng, M);
  }
  if (pz[nboxes] > 0) {
    k_zero_views<<<nblk(pz[nboxes]), 256, 0, st>>>(d_t, d_pz, nboxes, pz[nboxes]);
  }
  PMP_TRY(h, cudaGetLastError());
  PMP_TRY(h, cudaStreamSynchronize(st));
  return PMP_OK;
}

// The re-binning's keys, their sort and the box bounds (begin, host copy),
// with K-bit keys over bits [0, end_bit) and V-bit slot indices; the sorted
// indices (the gather order) stay in rebin_scratch at RebinLayout::perm.
template <typename K, typename V>
static int rebin_sort(pmp_spray* h, cudaStream_t st, long long n, int nb, int shift, int end_bit,
                      std::vector<long long>& begin)
{
  size_t tbytes = 0;
  if (n > 0) {
    cub::DeviceRadixSort::SortPairs(nullptr, tbytes, (const K*)nullptr, (K*)nullptr, (const V*)nullptr, (V*)nullptr,
                                    (int)n, 0, end_bit, st);
  }
  const RebinLayout L = rebin_layout(n, nb, sizeof(K), sizeof(V), tbytes);
  if (h->rebin_scratch_bytes < L.total) {
    cudaFree(h->rebin_scratch);
    h->rebin_scratch = nullptr;
    h->rebin_scratch_bytes = 0;
    if (cudaMalloc(&h->rebin_scratch, L.total) != cudaSuccess) {
      return set_err(h, PMP_ERR_CUDA, "redistribute: allocation failed");
    }
    h->rebin_scratch_bytes = L.total;
  }
  char* base = static_cast<char*>(h->rebin_scratch);
  K* keys = reinterpret_cast<K*>(base);
  K* keys2 = reinterpret_cast<K*>(base + L.keys2);
  V* idx = reinterpret_cast<V*>(base + L.idx);
  V* perm = reinterpret_cast<V*>(base + L.perm);
  long long* d_begin = reinterpret_cast<long long*>(base + L.begin);
  pmp_box* d_boxes = reinterpret_cast<pmp_box*>(base + L.boxes);
  const pmp_geometry& g = h->geom;
  PMP_TRY(h, cudaMemcpyAsync(d_boxes, h->boxes.data(), sizeof(pmp_box) * nb, cudaMemcpyHostToDevice, st));
  const Domain D = domain_of(h);
  if (n > 0) {
    k_rebin_keys<K, V><<<nblk(n), 256, 0, st>>>(h->soa, h->soa + n, h->soa + 2 * n, h->ids, n, h->d_box_map, D,
                                                g.plo[0], g.plo[1], g.plo[2], g.phi[0], g.phi[1], g.phi[2],
                                                1. / g.dx[0], 1. / g.dx[1], 1. / g.dx[2], d_boxes, nb, shift, keys,
                                                idx);
    cub::DeviceRadixSort::SortPairs(base + L.tmp, tbytes, keys, keys2, idx, perm, (int)n, 0, end_bit, st);
    k_box_bounds<K><<<nblk(nb + 1, 64), 64, 0, st>>>(keys2, n, nb, shift, d_begin);
  } else {
    PMP_TRY(h, cudaMemsetAsync(d_begin, 0, sizeof(long long) * (nb + 1), st));
  }
  PMP_TRY(h, cudaMemcpyAsync(begin.data(), d_begin, sizeof(long long) * (nb + 1), cudaMemcpyDeviceToHost, st));
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    return set_err(h, PMP_ERR_CUDA, "redistribute: kernel failed");
  }
  return PMP_OK;
}

extern "C" int pmp_spray_redistribute(pmp_spray* h, long long* removed, void* stream)
{
  if (!h) {
    return PMP_ERR_INVALID;
  }
  if (!h->have_geom) {
    return set_err(h, PMP_ERR_INVALID, "geometry must be set first");
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_packed(h);
  if (rc == PMP_OK) {
    rc = ensure_box_map(h, st);
  }
  if (rc != PMP_OK) {
    return rc;
  }
  const int nb = (int)h->boxes.size();
  const long long n = h->total;
  const int nc = h->ncomp();
  // key bits: the largest box's cell count, then the box index (nb: dead)
  int shift = 0;
  for (const pmp_box& bx : h->boxes) {
    const unsigned long long cells =
      pmp::brick_key_count(bx.hi[0] - bx.lo[0] + 1, bx.hi[1] - bx.lo[1] + 1, bx.hi[2] - bx.lo[2] + 1);
    while (shift < 63 && (1ULL << shift) < cells) {
      ++shift;
    }
  }
  int end_bit = shift + 1;
  while (end_bit < 64 && (1LL << (end_bit - shift)) <= nb) {
    ++end_bit;
  }
  if (end_bit > 62 || nb >= (1 << 22)) {
    return set_err(h, PMP_ERR_INVALID, "box too large for the re-binning key");
  }
  std::vector<long long> begin(nb + 1, 0);
  const bool narrow = end_bit <= 32 && n < (1LL << 31);
  const int rc2 = narrow ? rebin_sort<unsigned, int>(h, st, n, nb, shift, end_bit, begin)
                         : rebin_sort<unsigned long long, long long>(h, st, n, nb, shift, end_bit, begin);
  if (rc2 != PMP_OK) {
    return rc2;
  }
  const long long live = begin[nb];
  // gather into the spare store (grown when too small), which then becomes
  // the store; the old store becomes the spare
  if (h->spare_cap < live || !h->soa_spare) {
    cudaFree(h->soa_spare);
    cudaFree(h->ids_spare);
    h->soa_spare = nullptr;
    h->ids_spare = nullptr;
    h->spare_cap = 0;
    const long long lcap = std::max(live, 1LL);
    if (cudaMalloc(&h->soa_spare, sizeof(double) * nc * lcap) != cudaSuccess ||
        cudaMalloc(&h->ids_spare, sizeof(int) * lcap) != cudaSuccess) {
      return set_err(h, PMP_ERR_CUDA, "redistribute: allocation failed");
    }
    h->spare_cap = lcap;
  }
  if (live > 0) {
    const RebinLayout Lr = rebin_layout(n, nb, narrow ? 4 : 8, narrow ? 4 : 8, 0);
    const void* perm = static_cast<char*>(h->rebin_scratch) + Lr.perm;
    const long long* d_begin = reinterpret_cast<const long long*>(static_cast<char*>(h->rebin_scratch) + Lr.begin);
    if (narrow) {
      k_gather_soa<<<nblk(live), 256, 0, st>>>(h->soa, n, h->ids, static_cast<const int*>(perm), live, nc,
                                               h->soa_spare, h->ids_spare);
    } else {
      k_gather_soa<<<nblk(live), 256, 0, st>>>(h->soa, n, h->ids, static_cast<const long long*>(perm), live, nc,
                                               h->soa_spare, h->ids_spare);
    }
    // each box's new order is its caller order (h->perm holds >= n >= live slots)
    k_rebin_perm<<<nblk(live), 256, 0, st>>>(h->perm, d_begin, nb, live);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    return set_err(h, PMP_ERR_CUDA, "redistribute: gather failed");
  }
  const long long cap = std::max(n, 1LL);
  std::swap(h->soa, h->soa_spare);
  std::swap(h->ids, h->ids_spare);
  h->spare_cap = cap;  // the old store
  if (removed) {
    *removed = n - live;
  }
  return install_rebinned(h, begin);
}
