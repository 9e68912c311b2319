// mlp_tc.cuh -- CTA-level tcgen05 inference of the 10-64-64-64-5 SiLU
// surrogate: 128 droplets per M tile, one thread per droplet.
//
// Per layer, the CTA's threads write their rows of the bf16 A operand into
// shared memory, one elected thread issues tcgen05.mma (kind::f16, bf16 x
// bf16 -> f32, M = 128, N = 64 or 16, K = 16 per instruction) with A and the
// layer's weights (B) read from shared memory through matrix descriptors and
// the accumulator D in tensor memory, tcgen05.commit signals an mbarrier, and
// every thread then reads its own accumulator row back with tcgen05.ld
// (TMEM lane = row), adds the bias, applies SiLU and writes the next layer's
// A row in place.  Accumulators never occupy registers; a thread holds 16
// values of its row at a time.
//
// Operand layout in shared memory: the canonical K-major layout without
// swizzle.  A core matrix is 8 rows x 8 bf16 (16 bytes per row, 128 bytes
// contiguous); element (row, k) of a K-column matrix is at byte
//   (row / 8) * (16 K) + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,
// so the descriptor's leading-dimension byte offset (next core matrix along
// K) is 128 and its stride byte offset (next 8-row group) is 16 K; the
// K-step s of an MMA starts 256 s bytes in.
//
// Numerics as the warp-level path it replaces (mlp_mma.cuh): the hidden
// layers' weights and biases are stored halved, a layer yields h = x / 2 in
// FP32 and SiLU(x) = fma(h, tanh h, h) in packed bf16x2; the input row is a
// hi/lo bf16 pair (K = 32: hi in k 0-9, lo in k 16-25).
//
// Waits are bounded: an mbarrier wait gives up after about half a second of
// clock cycles; the CTA then agrees (syncthreads_and) to stop, waits once more
// with the same bound for its MMAs in flight, frees its tensor memory and
// reports the timeout.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace pmp {
namespace tc {

constexpr int kTile = 128;             // rows (droplets) per MMA tile
constexpr int kHid = 64;               // hidden width
constexpr int kK1 = 32;                // layer-1 K (hi | lo input halves)
constexpr int kN4 = 16;                // output layer N (5 used)
constexpr int kCols = 64;              // TMEM columns per tile (the 64-wide accumulator)

// weights and biases, canonical layout (bf16 operands, FP32 biases)
struct __align__(128) TcMlp {
  __nv_bfloat16 w1[kHid * kK1];
  __nv_bfloat16 w2[kHid * kHid];
  __nv_bfloat16 w3[kHid * kHid];
  __nv_bfloat16 w4[kN4 * kHid];
  float b1[kHid];
  float b2[kHid];
  float b3[kHid];
  float b4[kN4];
};
static_assert(sizeof(TcMlp) % 16 == 0, "copied as 16-byte words");

// per-tile A operand: 128 rows x 64 bf16 (layer 1 uses the first 128 x 32)
struct __align__(128) TcTileA {
  __nv_bfloat16 a[kTile * kHid];
};

// element offset of (row, k) in a K-column canonical operand
__host__ __device__ constexpr int tc_off(int row, int k, int K)
{
  return (row >> 3) * (8 * K) + (k >> 3) * 64 + (row & 7) * 8 + (k & 7);
}

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor, K-major, no swizzle: LBO 128 B, SBO 16 K B
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, int K)
{
  const uint64_t sbo = (uint64_t)(16 * K) >> 4;
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((sbo & 0x3FFFu) << 32) |
         (1ull << 46);  // descriptor version 1 (sm_100); base offset 0, SWIZZLE_NONE
}

// instruction descriptor: kind::f16, A = B = bf16, D = f32, both K-major, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "setp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
    :
    : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v)
{
  uint32_t r[16];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
    : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    v[i] = __uint_as_float(r[i]);
  }
}

__device__ __forceinline__ void mbar_init(uint32_t mbar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for the mbarrier phase with the given parity (about 0.5 s)
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(mbar), "r"(parity)
      : "memory");
    if (done) {
      return true;
    }
    if (clock64() - t0 > (1LL << 30)) {
      return false;
    }
  }
}

// One thread: a bulk (TMA, no tensor map) copy of `bytes` (a multiple of 16,
// both addresses 16-byte aligned) from global to shared memory, completing
// the mbarrier's current phase when the bytes have landed.
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gsrc, uint32_t bytes, uint32_t mbar)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                 smem_u32(smem_dst)),
               "l"(gsrc), "r"(bytes), "r"(mbar)
               : "memory");
}

__device__ __forceinline__ unsigned silu2(float h0, float h1)
{
  const __nv_bfloat162 p2 = __floats2bfloat162_rn(h0, h1);
  const unsigned p = *reinterpret_cast<const unsigned*>(&p2);
  unsigned t, r;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(p));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(r) : "r"(p), "r"(t));
  return r;
}

__device__ __forceinline__ unsigned pack2(float lo, float hi)
{
  const __nv_bfloat162 p2 = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&p2);
}

// The tensor-memory and barrier state of one CTA.
struct TcCta {
  uint32_t tmem;    // base address of the CTA's columns (tiles x kCols)
  uint32_t mbar;    // shared address of the MMA-completion mbarrier
  uint32_t phase;   // parity of the next completion
};

// Warp 0 allocates ncols TMEM columns (a power of 2, 32 to 512) and the
// thread 0 initialises the mbarrier; every thread of the CTA calls it.
__device__ __forceinline__ TcCta tc_setup(uint32_t* tmem_slot, unsigned long long* mbar_slot, int ncols)
{
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(mbar_slot));
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  TcCta c;
  c.tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
  c.mbar = smem_u32(mbar_slot);
  c.phase = 0;
  return c;
}

// All TMEM reads are complete in every thread: warp 0 frees the columns.
__device__ __forceinline__ void tc_teardown(const TcCta& c, int ncols)
{
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(c.tmem), "r"(ncols) : "memory");
  }
}

// The A rows of every tile are written: one thread issues the layer's MMAs
// for all tiles and commits; every thread waits.  Returns false (uniformly
// over the CTA) if the wait timed out.
template <int TILES>
__device__ __forceinline__ bool tc_layer(TcCta& c, TcTileA* A, const __nv_bfloat16* w, int K, int N)
{
  proxy_fence();      // this thread's A writes -> visible to the tensor core's reads
  tc_fence_before();  // this thread's earlier TMEM reads -> ordered before the next MMA
  __syncthreads();
  if (threadIdx.x == 0) {
    tc_fence_after();
    const uint32_t idesc = tc_idesc(N);
    const uint32_t wb = smem_u32(w);
#pragma unroll
    for (int t = 0; t < TILES; ++t) {
      const uint32_t ab = smem_u32(A[t].a);
      for (int s = 0; s < K / 16; ++s) {
        tc_mma(c.tmem + (uint32_t)(t * kCols), tc_desc(ab + 256u * s, K), tc_desc(wb + 256u * s, K), idesc,
               s > 0 ? 1u : 0u);
      }
    }
    tc_commit(c.mbar);
  }
  const bool ok = mbar_wait(c.mbar, c.phase);
  c.phase ^= 1u;
  tc_fence_after();
  return __syncthreads_and(ok) != 0;
}

// The network for the CTA's TILES x 128 rows: each thread passes its row's
// 10 normalised inputs (zeros for an idle row) and gets the 5 normalised
// outputs.  All threads of the CTA call it.  Returns false on a timed-out
// wait (the outputs are then undefined).
template <int TILES>
__device__ __forceinline__ bool mlp_cta_tc(const TcMlp& S, TcTileA* A, TcCta& c, const float* xin, float* yout)
{
  const int t = threadIdx.x / kTile;
  const int row = threadIdx.x % kTile;
  const uint32_t lane_off = (uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16;
  const uint32_t dcol = c.tmem + lane_off + (uint32_t)(t * kCols);
  __nv_bfloat16* arow = A[t].a;
  // layer-1 input: hi in k 0-9, lo in k 16-25
  {
    unsigned hi[8], lo[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float x0 = 2 * j < 10 ? xin[2 * j] : 0.f;
      const float x1 = 2 * j + 1 < 10 ? xin[2 * j + 1] : 0.f;
      const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
      const float2 hf = __bfloat1622float2(h);
      hi[j] = *reinterpret_cast<const unsigned*>(&h);
      lo[j] = pack2(x0 - hf.x, x1 - hf.y);
    }
    uint4* base = reinterpret_cast<uint4*>(arow + tc_off(row, 0, kK1));  // chunk kc at +8 uint4
    base[0] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    base[8] = make_uint4(hi[4], hi[5], hi[6], hi[7]);
    base[16] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    base[24] = make_uint4(lo[4], lo[5], lo[6], lo[7]);
  }
  if (!tc_layer<TILES>(c, A, S.w1, kK1, kHid)) {
    return false;
  }
  const float* bias[3] = {S.b1, S.b2, S.b3};
  const __nv_bfloat16* wnext[3] = {S.w2, S.w3, S.w4};
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    // accumulator row -> bias, SiLU -> this row of the next A (K = 64)
    uint4* base = reinterpret_cast<uint4*>(arow + tc_off(row, 0, kHid));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float v[16];
      tc_ld16(dcol + 16 * q, v);
      unsigned p[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        p[j] = silu2(v[2 * j] + bias[l][16 * q + 2 * j], v[2 * j + 1] + bias[l][16 * q + 2 * j + 1]);
      }
      base[8 * (2 * q)] = make_uint4(p[0], p[1], p[2], p[3]);
      base[8 * (2 * q + 1)] = make_uint4(p[4], p[5], p[6], p[7]);
    }
    if (!tc_layer<TILES>(c, A, wnext[l], kHid, l < 2 ? kHid : kN4)) {
      return false;
    }
  }
  float v[16];
  tc_ld16(dcol, v);
#pragma unroll
  for (int o = 0; o < 5; ++o) {
    yout[o] = v[o] + S.b4[o];
  }
  return true;
}

#endif  // __CUDACC__

}  // namespace tc
}  // namespace pmp
