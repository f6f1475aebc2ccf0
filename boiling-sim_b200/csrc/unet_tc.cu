// unet_tc.cu -- inference path of the warm-start U-Net on the fifth-generation
// tensor cores: tcgen05.mma with the accumulator in tensor memory (TMEM),
// operand tiles staged in shared memory by TMA (cp.async.bulk.tensor, never
// with cluster multicast), one elected thread issuing the MMAs, warp-
// specialised producer / MMA / epilogue roles.
//
// Padded activation layout.  A level of interior size (nx, ny, nz) is stored
// with a one-cell zero halo: row q = ((i+1)(ny+2) + (j+1))(nz+2) + (k+1) for
// interior cell (i, j, k), act[q][c] BF16, channels innermost.  A 3x3x3 tap
// (di, dj, dk) is then a constant shift of the row index, so every operand
// tile of the implicit GEMM is a run of consecutive rows -- one TMA box, no
// gather, and the zero halo supplies the convolution's zero padding.
//
// The GEMM.  A tile is a window of 128 consecutive rows w = 0..127 (rows
// q0 - 1 + w); it produces outputs q0 + m, m = 0..125.  The three dk taps of
// each (di, dj) pair are stacked along N: B = [W(dk=-1); W(dk=0); W(dk=+1)]
// (N = 3 cout), so one MMA per (di, dj) and 16-channel chunk computes
// D[w][dk block] = sum_ci in(q0 - 1 + w + di P + dj R)[ci] W[di,dj,dk][co][ci]
// (P = (ny+2)(nz+2), R = nz+2), and the epilogue forms
// out[m] = D[m][dk=-1] + D[m+1][dk=0] + D[m+2][dk=+1]
// by exchanging neighbouring TMEM lanes through warp shuffles.  Stacking the
// dk taps makes N three times larger than cout, so each byte of activation
// read from shared memory by the tensor core feeds 3x the multiply-adds.
//
// Roles (one CTA per SM, persistent over work items = (row tile, cout tile)):
//   warp 0   TMA producer: per 16-channel chunk, 9 (di, dj) slabs, each a
//            {16 channels x 128 rows} box (32-byte rows, one sector each) with
//            the 32-byte swizzle, into a ring of shared-memory stages (full /
//            empty mbarriers); streams the chunk's weights too when they do
//            not stay resident;
//   warp 1   TMEM allocator and MMA issuer (one thread): 9 MMAs
//            (M = 128, N = 3 cout_tile, K = 16) per chunk into one of 8, 4 or 2
//            TMEM accumulators (as many as 512 columns hold), tcgen05.commit to release
//            stages and to hand the accumulator to the epilogue;
//   warps 2-17 epilogue, four warpgroups taking work items in turn (as many
//            as there are accumulators):
//            tcgen05.ld of their 32 TMEM lanes, dk combination, bias, ReLU,
//            optional skip add, BF16 store (halo rows get zeros).
// Row indices stay in 32 bits (padded rows < 2^30) and the stage ring is
// walked with running counters: no 64-bit division on the critical path of
// the single-thread roles.
// Every mbarrier wait is bounded; on a timeout the kernel records
// BSP_ERR_TIMEOUT in a device flag, drains its outstanding copies and MMAs
// (bounded), frees its TMEM and returns.
//
// Shared-memory operand layouts (K-major).  Activations: a slab is 128 rows
// x 32 bytes (16 channels), written by TMA with the 32-byte swizzle and read
// by the MMA through a 32-byte-swizzle descriptor (8-row groups 256 bytes
// apart).  Weights (no swizzle): a "core matrix" is 8 rows x 16 bytes (8 BF16
// of K) stored as 128 contiguous bytes; each 8-channel half of a (di, dj,
// chunk) block is N rows x 16 B, so its descriptor uses stride-byte-offset 128
// and leading-byte-offset = the distance between the two K halves.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "bsp_common.cuh"
#include "profile.cuh"
#include "tma.cuh"

namespace bsp {
namespace utc {

constexpr int M = 128;          // window rows per tile (TMEM lanes)
constexpr int MOUT = 126;       // outputs per tile
constexpr int NEPI_MAX = 4;     // epilogue warpgroups (take work items in turn), at most
// producer warp, MMA warp, epilogue warpgroups
__host__ __device__ constexpr int conv_threads(int nepi) { return 64 + nepi * 128; }
constexpr int SLAB = M * 32;               // one (di, dj) slab: 128 rows x 16 channels
constexpr int A_STAGE = 9 * SLAB;          // 36,864 bytes per 16-channel chunk
constexpr int SMEM_MAX = 232448;           // dynamic shared memory per CTA (227 KB)
constexpr int SMEM_MIN = 120 * 1024;       // keep one CTA per SM (TMEM is not shared)
constexpr int WRES_MAX = 112 * 1024;       // weights stay resident up to this size
constexpr int SMEM_PAIR = 112 * 1024;      // per CTA with two CTAs per SM
constexpr int ROWS_MAX = 1 << 30;          // padded rows: row arithmetic stays in 32 bits
__host__ __device__ constexpr int round1k(int b) { return (b + 1023) / 1024 * 1024; }

__device__ int g_utc_err;  // BSP_ERR_TIMEOUT once any wait of this kernel gave up
// Optional cycle accounting (bsp_unet_tc_trace), summed over CTAs:
// 0 producer waiting for a free stage, 1 MMA issuer waiting for a full stage,
// 2 MMA issuer waiting for a free accumulator, 3 epilogue waiting for a
// complete accumulator, 4 epilogue busy (per warpgroup, from the accumulator
// to its release), 5 CTA lifetime, 6 work items, 7 MMA issuer busy.
__device__ unsigned long long g_utc_trace[8];

struct Params {
  __nv_bfloat16 *out;          // padded output rows x cout
  const __nv_bfloat16 *wimg;   // weight image (bsp_unet_tc_weights)
  const float *bias;           // cout or NULL (16-byte aligned)
  const __nv_bfloat16 *skip;   // padded rows x cout, added after ReLU, or NULL
  int nx, ny, nz, cin, cout;
  int ct;        // cout per CTA tile (16, 32 or 64); N = 3 ct
  int nct;       // cout tiles
  int relu;
  int r0;        // first interior row
  int rows;      // total padded rows (< ROWS_MAX)
  int nwork;     // work items = row tiles x cout tiles
  int resident;  // weights resident in shared memory
  int nst;       // A stages
  int w_bytes_chunk;  // bytes of one chunk's weights (9 x 2 x N x 16)
  int trace;     // accumulate g_utc_trace
};

// ---- PTX wrappers --------------------------------------------------------------------
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tma_load2(void *dst, const CUtensorMap *map, int x, int y,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// The same with the shared-memory addresses already in the shared window.
__device__ __forceinline__ void tma_load2u(uint32_t dst, const CUtensorMap *map, int x, int y,
                                           uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
// 1-D bulk copy global -> shared (no multicast); size a multiple of 16
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// 16 consecutive TMEM columns of this thread's lane from each of three column
// offsets, then wait::ld -- in one asm statement, so no use of the registers
// can be scheduled before the wait.
__device__ __forceinline__ void tmem_ld3x16(uint32_t a0, uint32_t a1, uint32_t a2,
                                           float (&x0)[16], float (&x1)[16], float (&x2)[16]) {
  uint32_t r[48];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%48];\n"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16, %17, %18, %19, %20, %21, %22, %23, %24, "
      "%25, %26, %27, %28, %29, %30, %31}, [%49];\n"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32, %33, %34, %35, %36, %37, %38, %39, %40, "
      "%41, %42, %43, %44, %45, %46, %47}, [%50];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]),
        "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]),
        "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47])
      : "r"(a0), "r"(a1), "r"(a2)
      : "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    x0[q] = __uint_as_float(r[q]);
    x1[q] = __uint_as_float(r[16 + q]);
    x2[q] = __uint_as_float(r[32 + q]);
  }
}
// 16 columns of this thread's lane from each of two column offsets, then wait::ld.
__device__ __forceinline__ void tmem_ld2x16(uint32_t a0, uint32_t a1, float (&x0)[16],
                                           float (&x1)[16]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%32];\n"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16, %17, %18, %19, %20, %21, %22, %23, %24, "
      "%25, %26, %27, %28, %29, %30, %31}, [%33];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(a0), "r"(a1)
      : "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    x0[q] = __uint_as_float(r[q]);
    x1[q] = __uint_as_float(r[16 + q]);
  }
}
// 16 columns of this thread's lane, then wait::ld.
__device__ __forceinline__ void tmem_ld1x16(uint32_t a0, float (&x0)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(a0)
      : "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) x0[q] = __uint_as_float(r[q]);
}
// Two floats rounded to BF16 (round to nearest even) in one 32-bit word, lo
// in the low half (the lower address).
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
__device__ __forceinline__ void named_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// descriptor version 1: start >> 4 in bits 0-13, leading-byte-offset >> 4 in
// 16-29, stride-byte-offset >> 4 in 32-45, version in 46-47.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// The same for the activation slabs, written by TMA with the 32-byte swizzle:
// rows of 32 bytes (the 16 channels of one K step), 8-row groups 256 bytes
// apart, layout type 6 (32-byte swizzle) in bits 61-63; the leading byte
// offset is not used by swizzled K-major layouts (encoded as 1).  The slab
// base is 1024-byte aligned so the swizzle pattern starts with it.
__device__ __forceinline__ uint64_t sdesc_sw32(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)6 << 61);
}
// Instruction descriptor of kind::f16: FP32 accumulate (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 in bits 17-22,
// M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, int m) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

struct Ctl {
  // lane-31 dk=-1 block and lane-0 dk=+1 block of each epilogue quarter, per
  // warpgroup, double-buffered over the 16-channel blocks
  __align__(16) float xch0[NEPI_MAX][2][4][16];
  __align__(16) float xch2[NEPI_MAX][2][4][16];
  uint64_t full[8], empty[8], acc_full[8], acc_empty[8], wbar, drain;
  uint32_t tmem_base;
  int abort;
  int ep_ok[NEPI_MAX][2];   // accumulator-ready vote of each epilogue warpgroup
};

__device__ __forceinline__ bool wait_or_abort(uint64_t *bar, uint32_t parity, Ctl *c) {
  if (mbar_wait(bar, parity)) return true;
  *(volatile int *)&c->abort = 1;
  atomicExch(&g_utc_err, BSP_ERR_TIMEOUT);
  return false;
}
// wait_or_abort that adds the cycles spent to `acc` when tracing
__device__ __forceinline__ bool timed_wait(uint64_t *bar, uint32_t parity, Ctl *c, bool tr,
                                           unsigned long long &acc) {
  const long long t0 = tr ? clock64() : 0;
  const bool ok = wait_or_abort(bar, parity, c);
  if (tr) acc += (unsigned long long)(clock64() - t0);
  return ok;
}

// NEPI epilogue warpgroups.  The register file is split over the four SM
// sub-partitions (16 K registers each): 18 warps (NEPI = 4) put five warps on
// two of them and allow 96 registers a thread, 14 warps (NEPI = 3) 128.
// NEPI = 1 runs two CTAs per SM (each its own producer, MMA issuer and
// epilogue warpgroup, half the shared memory and 256 TMEM columns): two
// independent single-thread issue streams per SM.
template <int NEPI>
__global__ void __launch_bounds__(conv_threads(NEPI), NEPI == 1 ? 2 : 1) conv_tc_kernel(
    const __grid_constant__ CUtensorMap amap, const Params p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int N = 3 * p.ct;
  const int ncol = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  // accumulators in TMEM: as many as fit in this CTA's columns (512, or 256
  // with two CTAs per SM), at most 8; epilogue warpgroups in use: at most one
  // per accumulator
  const int tmem_max = NEPI == 1 ? 256 : 512;
  int lgacc = 0;
  while (lgacc < 3 && (ncol << (lgacc + 1)) <= tmem_max) ++lgacc;
  const int nacc = 1 << lgacc;
  const int nwg = nacc < NEPI ? nacc : NEPI;
  const uint32_t tcols = (uint32_t)(nacc * ncol);
  const int nchunk = p.cin >> 4;
  const int wchunk = p.w_bytes_chunk;
  const bool tr = p.trace != 0;
  const long long t_start = tr ? clock64() : 0;
  // layout (from a 1024-byte aligned base): [weights (resident: all chunks;
  // else none)] [stages] [Ctl]; weights and stages padded to 1024 bytes
  unsigned char *base0 = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem) + 1023) & ~(uintptr_t)1023);
  unsigned char *wres = base0;
  const int wres_bytes = p.resident ? round1k(wchunk * nchunk) : 0;
  const int stage_bytes = round1k(A_STAGE + (p.resident ? 0 : wchunk));
  const uint32_t stage_tx = (uint32_t)(A_STAGE + (p.resident ? 0 : wchunk));  // bytes landing
  unsigned char *stages = base0 + wres_bytes;
  Ctl *c = reinterpret_cast<Ctl *>(stages + (size_t)p.nst * stage_bytes);
  const int nwork = p.nwork;

  if (threadIdx.x == 0) {
    for (int s = 0; s < p.nst; ++s) {
      mbar_init(&c->full[s], 1);
      mbar_init(&c->empty[s], 1);
    }
    for (int b = 0; b < nacc; ++b) {
      mbar_init(&c->acc_full[b], 1);
      mbar_init(&c->acc_empty[b], 4);
    }
    mbar_init(&c->wbar, 1);
    mbar_init(&c->drain, 1);
    c->abort = 0;
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&c->tmem_base)),
                 "r"(tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_shared();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = c->tmem_base;
  const int R = p.nz + 2, P = (p.ny + 2) * R;

  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      unsigned long long t_wait = 0;
      if (p.resident) {
        const uint32_t total = (uint32_t)(wchunk * nchunk);
        mbar_expect_tx(&c->wbar, total);
        for (uint32_t off = 0; off < total; off += 16384) {
          const uint32_t nb = total - off < 16384 ? total - off : 16384;
          bulk_load(wres + off, reinterpret_cast<const unsigned char *>(p.wimg) + off, nb,
                    &c->wbar);
        }
      }
      // The issue loop is one thread's dependent instruction stream: the
      // slabs' row offsets and the shared-memory addresses are formed once,
      // the nine loads unrolled.
      int yoff[9];
#pragma unroll
      for (int sl = 0; sl < 9; ++sl) yoff[sl] = (sl / 3 - 1) * P + (sl % 3 - 1) * R;
      const uint32_t stages_u = smem_u32(stages), full_u = smem_u32(&c->full[0]);
      int it = 0, s = 0;  // stage fills issued; current stage
      uint32_t ph = 0;    // its phase
      for (int wk = blockIdx.x; wk < nwork && !*(volatile int *)&c->abort; wk += gridDim.x) {
        const int t = wk / p.nct;
        const int ctile = wk - t * p.nct;
        const int base = p.r0 + t * MOUT - 1;
        for (int kc = 0; kc < nchunk; ++kc, ++it) {
          if (!timed_wait(&c->empty[s], ph ^ 1u, c, tr, t_wait)) break;
          unsigned char *st = stages + (size_t)s * stage_bytes;
          const uint32_t st_u = stages_u + (uint32_t)(s * stage_bytes);
          const uint32_t bar_u = full_u + 8u * (uint32_t)s;
          mbar_expect_tx(&c->full[s], stage_tx);
#pragma unroll
          for (int sl = 0; sl < 9; ++sl)
            tma_load2u(st_u + (uint32_t)(sl * SLAB), &amap, kc * 16, base + yoff[sl], bar_u);
          if (!p.resident)
            bulk_load(st + A_STAGE,
                      reinterpret_cast<const unsigned char *>(p.wimg) +
                          ((size_t)ctile * nchunk + kc) * wchunk,
                      (uint32_t)wchunk, &c->full[s]);
          if (++s == p.nst) {
            s = 0;
            ph ^= 1u;
          }
        }
        if (*(volatile int *)&c->abort) break;
      }
      // drain: every fill issued has landed (or the wait gives up)
      if (*(volatile int *)&c->abort && it > 0) {
        for (int q = it > p.nst ? it - p.nst : 0; q < it; ++q)
          mbar_wait(&c->full[q % p.nst], (uint32_t)((q / p.nst) & 1));
      }
      if (tr) atomicAdd(&g_utc_trace[0], t_wait);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      unsigned long long t_full = 0, t_acc = 0, t_busy = 0;
      const uint32_t idesc = idesc_bf16(N, M);
      const uint32_t stages_u = smem_u32(stages), wres_u = smem_u32(wres);
      bool ok = true;
      if (p.resident) ok = wait_or_abort(&c->wbar, 0, c);
      int s = 0, li = 0;
      uint32_t ph = 0;
      for (int wk = blockIdx.x; ok && wk < nwork; wk += gridDim.x, ++li) {
        const int b = li & (nacc - 1);
        if (!timed_wait(&c->acc_empty[b], (uint32_t)(((li >> lgacc) & 1) ^ 1), c, tr, t_acc)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t dt = tbase + (uint32_t)(b * ncol);
        for (int kc = 0; kc < nchunk; ++kc) {
          if (!timed_wait(&c->full[s], ph, c, tr, t_full)) {
            ok = false;
            break;
          }
          const long long t0 = tr ? clock64() : 0;
          tc_fence_after();
          // descriptors of slab 0; slab sl starts sl SLAB bytes (A) and
          // sl 2 N 16 bytes (B) further, i.e. + (offset >> 4) in the start
          // field (shared addresses stay below 2^18, so no carry leaves it)
          const uint32_t abase = stages_u + (uint32_t)(s * stage_bytes);
          const uint32_t bbase = p.resident ? wres_u + (uint32_t)(kc * wchunk) : abase + A_STAGE;
          const uint64_t ad0 = sdesc_sw32(abase), bd0 = sdesc(bbase, N * 16, 128);
          const uint64_t bstep = (uint64_t)(2 * N);
          tc_mma(dt, ad0, bd0, idesc, kc > 0 ? 1u : 0u);
#pragma unroll
          for (int sl = 1; sl < 9; ++sl)
            tc_mma(dt, ad0 + (uint64_t)(sl * (SLAB >> 4)), bd0 + (uint64_t)sl * bstep, idesc, 1u);
          tc_commit(&c->empty[s]);  // stage free once these MMAs have read it
          if (++s == p.nst) {
            s = 0;
            ph ^= 1u;
          }
          if (tr) t_busy += (unsigned long long)(clock64() - t0);
        }
        if (!ok) break;
        tc_commit(&c->acc_full[b]);  // accumulator complete
      }
      // drain: every MMA issued has completed before TMEM is freed
      tc_commit(&c->drain);
      mbar_wait(&c->drain, 0);
      if (tr) {
        atomicAdd(&g_utc_trace[1], t_full);
        atomicAdd(&g_utc_trace[2], t_acc);
        atomicAdd(&g_utc_trace[6], (unsigned long long)li);
        atomicAdd(&g_utc_trace[7], t_busy);
      }
    }
  } else {
    // ---------------- epilogue (warpgroups of warps 2-5, 6-9, ...) ----------------
    // Warpgroup g < nwg takes the work items li = g, g + nwg, ...;
    // accumulator li mod nacc.  Warp w reads TMEM lanes 32 (w mod 4) .. + 31.
    const int g = (warp - 2) >> 2;
    const int qd = warp & 3;                 // TMEM lane quarter of this warp
    const int w = qd * 32 + lane;            // window row
    const int m = w - 1;                     // output of this thread
    const bool leader = threadIdx.x == 64 + 128 * g;
    const int bar_id = 1 + g;
    const int rowsz = p.ny + 2;
    unsigned long long t_wait = 0, t_busy = 0;
    int vote = 0;  // this warpgroup's vote slot, alternating
    for (int li = g, wk = blockIdx.x + g * gridDim.x; g < nwg && wk < nwork;
         li += nwg, wk += nwg * gridDim.x, vote ^= 1) {
      const int b = li & (nacc - 1);
      // one thread waits (bounded) and the 128 threads of the warpgroup take
      // its answer through their named barrier, so they all leave together
      if (leader)
        c->ep_ok[g][vote] =
            timed_wait(&c->acc_full[b], (uint32_t)((li >> lgacc) & 1), c, tr, t_wait) ? 1 : 0;
      named_sync(bar_id, 128);
      if (!*(volatile int *)&c->ep_ok[g][vote]) break;
      const long long t0 = (tr && leader) ? clock64() : 0;
      tc_fence_after();
      const int t = wk / p.nct;
      const int ctile = wk - t * p.nct;
      const int q = p.r0 + t * MOUT + m;
      const bool valid = m >= 0 && m < MOUT && q < p.rows;
      bool interior = false;
      if (valid) {
        const unsigned uq = (unsigned)q, r2 = uq / (unsigned)R;
        const unsigned k = uq - r2 * (unsigned)R;
        const unsigned i = r2 / (unsigned)rowsz, j = r2 - i * (unsigned)rowsz;
        interior = k >= 1 && k <= (unsigned)p.nz && j >= 1 && j <= (unsigned)p.ny && i >= 1 &&
                   i <= (unsigned)p.nx;
      }
      const uint32_t trow = tbase + ((uint32_t)(qd * 32) << 16) + (uint32_t)(b * ncol);
      for (int cb = 0; cb < p.ct; cb += 16) {
        // the dk = -1 and +1 blocks first, the centre block (x1) after the
        // shuffles have consumed them: at most 48 of these registers live
        float x0[16], x2[16];
        tmem_ld2x16(trow + (uint32_t)(0 * p.ct + cb), trow + (uint32_t)(2 * p.ct + cb), x0, x2);
        // D[w-1][dk=-1] and D[w+1][dk=+1]: neighbouring lanes by shuffles, the
        // rows across a lane-quarter boundary through shared memory (slot
        // (cb / 16) mod 2: a slot is written again only after every reader
        // of it has passed the barrier of the block in between)
        const int xs = (cb >> 4) & 1;
        // the boundary rows' blocks to shared memory first (x0, x2 then die
        // as the shuffles consume them)
        if (lane == 31) {
          float4 *d4 = reinterpret_cast<float4 *>(c->xch0[g][xs][qd]);
#pragma unroll
          for (int e4 = 0; e4 < 4; ++e4)
            d4[e4] = make_float4(x0[4 * e4], x0[4 * e4 + 1], x0[4 * e4 + 2], x0[4 * e4 + 3]);
        }
        if (lane == 0) {
          float4 *d4 = reinterpret_cast<float4 *>(c->xch2[g][xs][qd]);
#pragma unroll
          for (int e4 = 0; e4 < 4; ++e4)
            d4[e4] = make_float4(x2[4 * e4], x2[4 * e4 + 1], x2[4 * e4 + 2], x2[4 * e4 + 3]);
        }
        // v = (up + x1) + dn: a = up + x1 now (lane 0: x1, its up comes from
        // the quarter above), dn now (lane 31: from the quarter below)
        float a[16], dn[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          a[e] = __shfl_up_sync(0xffffffffu, x0[e], 1);
          dn[e] = __shfl_down_sync(0xffffffffu, x2[e], 1);
        }
        {
          float x1[16];
          tmem_ld1x16(trow + (uint32_t)(1 * p.ct + cb), x1);
#pragma unroll
          for (int e = 0; e < 16; ++e) a[e] = lane == 0 ? x1[e] : a[e] + x1[e];
        }
        named_sync(bar_id, 128);
        if (lane == 0) {
          const float4 *s4 = reinterpret_cast<const float4 *>(c->xch0[g][xs][qd > 0 ? qd - 1 : 0]);
#pragma unroll
          for (int e4 = 0; e4 < 4; ++e4) {
            const float4 t = qd > 0 ? s4[e4] : make_float4(0.f, 0.f, 0.f, 0.f);
            a[4 * e4] = t.x + a[4 * e4];
            a[4 * e4 + 1] = t.y + a[4 * e4 + 1];
            a[4 * e4 + 2] = t.z + a[4 * e4 + 2];
            a[4 * e4 + 3] = t.w + a[4 * e4 + 3];
          }
        }
        if (lane == 31) {
          const float4 *s4 = reinterpret_cast<const float4 *>(c->xch2[g][xs][qd < 3 ? qd + 1 : 3]);
#pragma unroll
          for (int e4 = 0; e4 < 4; ++e4) {
            const float4 t = qd < 3 ? s4[e4] : make_float4(0.f, 0.f, 0.f, 0.f);
            dn[4 * e4] = t.x;
            dn[4 * e4 + 1] = t.y;
            dn[4 * e4 + 2] = t.z;
            dn[4 * e4 + 3] = t.w;
          }
        }
        float v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = a[e] + dn[e];
        if (valid) {
          const int co0 = ctile * p.ct + cb;
          __nv_bfloat16 *dst = p.out + (size_t)q * p.cout + co0;
          uint32_t w[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};  // halo rows: zeros
          if (interior) {
            if (p.bias) {
              const float4 *b4 = reinterpret_cast<const float4 *>(p.bias + co0);
#pragma unroll
              for (int e4 = 0; e4 < 4; ++e4) {
                const float4 bb = __ldg(b4 + e4);
                v[4 * e4 + 0] += bb.x;
                v[4 * e4 + 1] += bb.y;
                v[4 * e4 + 2] += bb.z;
                v[4 * e4 + 3] += bb.w;
              }
            }
            if (p.relu) {
#pragma unroll
              for (int e = 0; e < 16; ++e) v[e] = fmaxf(v[e], 0.0f);
            }
            if (p.skip) {
              const uint4 *sk = reinterpret_cast<const uint4 *>(p.skip + (size_t)q * p.cout + co0);
              const uint4 s0 = __ldg(sk), s1 = __ldg(sk + 1);
              const uint32_t sw[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
#pragma unroll
              for (int e = 0; e < 16; ++e) {
                const uint32_t u = sw[e >> 1];
                const float sv = __uint_as_float((e & 1) ? (u & 0xffff0000u) : (u << 16));
                v[e] = __bfloat162float(__float2bfloat16(v[e])) + sv;
              }
            }
#pragma unroll
            for (int e = 0; e < 8; ++e) w[e] = pack_bf16x2(v[2 * e], v[2 * e + 1]);
          }
          reinterpret_cast<uint4 *>(dst)[0] = make_uint4(w[0], w[1], w[2], w[3]);
          reinterpret_cast<uint4 *>(dst)[1] = make_uint4(w[4], w[5], w[6], w[7]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&c->acc_empty[b]);
      if (tr && leader) t_busy += (unsigned long long)(clock64() - t0);
    }
    if (tr && leader) {
      atomicAdd(&g_utc_trace[3], t_wait);
      atomicAdd(&g_utc_trace[4], t_busy);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase),
                 "r"(tcols)
                 : "memory");
  if (tr && threadIdx.x == 0)
    atomicAdd(&g_utc_trace[5], (unsigned long long)(clock64() - t_start));
}

// ---- weight image ---------------------------------------------------------------------
// wimg[ct][kc][s][h][n][8], n = dki * CT + col (dki 0..2 for dk = -1, 0, +1),
// co = ct * CT + col, ci = 16 kc + 8 h + e; from w[tap][co][ci] with
// tap = (di+1) 9 + (dj+1) 3 + (dk+1) and s = (di+1) 3 + (dj+1).
__global__ void weight_image_kernel(__nv_bfloat16 *__restrict__ wimg,
                                    const __nv_bfloat16 *__restrict__ w, int cin, int cout,
                                    int CT) {
  const int64_t total = 27LL * cin * cout;
  const int N = 3 * CT;
  const int nchunk = cin / 16;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = q;
    const int e = (int)(r % 8);
    r /= 8;
    const int n = (int)(r % N);
    r /= N;
    const int h = (int)(r % 2);
    r /= 2;
    const int s = (int)(r % 9);
    r /= 9;
    const int kc = (int)(r % nchunk);
    const int ct = (int)(r / nchunk);
    const int dki = n / CT, col = n % CT;
    const int co = ct * CT + col, ci = 16 * kc + 8 * h + e;
    const int tap = (s / 3) * 9 + (s % 3) * 3 + dki;
    wimg[q] = w[((int64_t)tap * cout + co) * cin + ci];
  }
}

// ---- padded-layout helpers (pack, pool, upsample, head) --------------------------------------
__device__ __forceinline__ bool unpad(int64_t q, int nx, int ny, int nz, int &i, int &j, int &k) {
  const int64_t R = nz + 2;
  const int64_t kk = q % R, r2 = q / R;
  const int64_t jj = r2 % (ny + 2), ii = r2 / (ny + 2);
  i = (int)ii - 1;
  j = (int)jj - 1;
  k = (int)kk - 1;
  return i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz;
}
__device__ __forceinline__ int64_t padrow(int i, int j, int k, int ny, int nz) {
  return ((int64_t)(i + 1) * (ny + 2) + (j + 1)) * (nz + 2) + (k + 1);
}

// x[q][0] = div / s on fluid, x[q][1] = fluid flag, x[q][2] = solid flag, other
// channels and halo rows 0 (16 channels).
__global__ void pack_pad_kernel(__nv_bfloat16 *__restrict__ x, const float *__restrict__ div,
                                const uint8_t *__restrict__ mask, int nx, int ny, int nz,
                                const float *__restrict__ s_dev, int64_t rows) {
  const float inv_scale = 1.0f / s_dev[0];
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < rows;
       q += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    uint4 v[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
    if (unpad(q, nx, ny, nz, i, j, k)) {
      const int64_t c = ((int64_t)i * ny + j) * nz + k;
      const uint8_t m = mask[c];
      const bool fl = (m & BSP_CLASS_FLUID) != 0;
      __nv_bfloat16 *h = reinterpret_cast<__nv_bfloat16 *>(v);
      h[0] = __float2bfloat16(fl ? div[c] * inv_scale : 0.0f);
      h[1] = __float2bfloat16(fl ? 1.0f : 0.0f);
      h[2] = __float2bfloat16((m & BSP_CLASS_SOLID) ? 1.0f : 0.0f);
    }
    uint4 *o = reinterpret_cast<uint4 *>(x + q * 16);
    o[0] = v[0];
    o[1] = v[1];
  }
}

// 2x2x2 average of the fine level (nx, ny, nz) into the coarse padded level;
// 8 channels per thread.  Halo rows of the output get zeros.
__global__ void pool_pad_kernel(__nv_bfloat16 *__restrict__ out,
                                const __nv_bfloat16 *__restrict__ in, int nx, int ny, int nz,
                                int c) {
  const int ox = nx / 2, oy = ny / 2, oz = nz / 2;
  const int g = c / 8;
  const int64_t rows = (int64_t)(ox + 2) * (oy + 2) * (oz + 2);
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < rows * g;
       u += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = u / g;
    const int cg = (int)(u - q * g);
    int i, j, k;
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const bool in_ = unpad(q, ox, oy, oz, i, j, k);
    if (in_) {
      for (int a = 0; a < 8; ++a) {
        const int64_t qf = padrow(2 * i + (a >> 2), 2 * j + ((a >> 1) & 1), 2 * k + (a & 1), ny, nz);
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(in + qf * c) + cg);
        const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] += __bfloat162float(h[e]);
      }
    }
    uint4 o;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
    for (int e = 0; e < 4; ++e) h[e] = __floats2bfloat162_rn(0.125f * s[2 * e], 0.125f * s[2 * e + 1]);
    reinterpret_cast<uint4 *>(out + q * c)[cg] = o;
  }
}

// nearest x2 upsampling of the coarse padded level onto the fine padded level
// (nx, ny, nz); halo rows get zeros.
__global__ void up_pad_kernel(__nv_bfloat16 *__restrict__ out, const __nv_bfloat16 *__restrict__ in,
                              int nx, int ny, int nz, int c) {
  const int g = c / 8;
  const int64_t rows = (int64_t)(nx + 2) * (ny + 2) * (nz + 2);
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < rows * g;
       u += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = u / g;
    const int cg = (int)(u - q * g);
    int i, j, k;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (unpad(q, nx, ny, nz, i, j, k))
      v = __ldg(reinterpret_cast<const uint4 *>(in + padrow(i >> 1, j >> 1, k >> 1, ny / 2,
                                                             nz / 2) * c) + cg);
    reinterpret_cast<uint4 *>(out + q * c)[cg] = v;
  }
}

// p[v] = scale (hb + hw . x[q]) on fluid cells, 0 elsewhere (unpadded FP32 out).
__global__ void head_pad_kernel(float *__restrict__ p, const __nv_bfloat16 *__restrict__ x,
                                const float *__restrict__ hw, const float *__restrict__ hb,
                                const uint8_t *__restrict__ mask, int nx, int ny, int nz,
                                const float *__restrict__ s_dev, float factor) {
  const float scale = factor * s_dev[0];
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(v % nz);
    const int64_t r = v / nz;
    const int j = (int)(r % ny), i = (int)(r / ny);
    const uint4 *xr = reinterpret_cast<const uint4 *>(x + padrow(i, j, k, ny, nz) * 16);
    const uint4 a = __ldg(xr), b = __ldg(xr + 1);
    const __nv_bfloat16 *h0 = reinterpret_cast<const __nv_bfloat16 *>(&a);
    const __nv_bfloat16 *h1 = reinterpret_cast<const __nv_bfloat16 *>(&b);
    float y = hb[0];
#pragma unroll
    for (int e = 0; e < 8; ++e) y = fmaf(hw[e], __bfloat162float(h0[e]), y);
#pragma unroll
    for (int e = 0; e < 8; ++e) y = fmaf(hw[8 + e], __bfloat162float(h1[e]), y);
    p[v] = (mask[v] & BSP_CLASS_FLUID) ? scale * y : 0.0f;
  }
}

// Divergence of the grid coarsened 2x in each direction: the mean over the
// fluid children of a coarse fluid cell (mask_c marks the coarse classes);
// 0 elsewhere.  (nx, ny, nz) is the fine size (even).
__global__ void restrict_div_kernel(float *__restrict__ divc, const uint8_t *__restrict__ maskc,
                                    const float *__restrict__ div,
                                    const uint8_t *__restrict__ mask, int nx, int ny, int nz) {
  // 32-bit index arithmetic (the host checks nx ny nz < 2^31)
  const int ox = nx / 2, oy = ny / 2, oz = nz / 2;
  const unsigned n = (unsigned)ox * (unsigned)oy * (unsigned)oz;
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const unsigned r = v / (unsigned)oz;
    const int k = (int)(v - r * (unsigned)oz);
    const unsigned ii = r / (unsigned)oy;
    const int j = (int)(r - ii * (unsigned)oy), i = (int)ii;
    float s = 0.0f;
    int cnt = 0;
    for (int a = 0; a < 8; ++a) {
      const unsigned c = ((unsigned)(2 * i + (a >> 2)) * (unsigned)ny + 2 * j + ((a >> 1) & 1)) *
                             (unsigned)nz +
                         2 * k + (a & 1);
      if (mask[c] & BSP_CLASS_FLUID) {
        s += div[c];
        ++cnt;
      }
    }
    divc[v] = ((maskc[v] & BSP_CLASS_FLUID) && cnt) ? s / (float)cnt : 0.0f;
  }
}

// Trilinear interpolation of a cell-centred coarse field (nx/2, ny/2, nz/2)
// onto the fine cells (half-cell offsets, edge values held), on fluid cells
// only; 0 elsewhere.
__device__ __forceinline__ void lin2(int d, int nc, int &a, int &b, float &wa) {
  // fine index d -> coarse position d/2 - 1/4, clamped to [0, nc - 1]
  if (d & 1) {
    a = d >> 1;
    b = min(a + 1, nc - 1);
    wa = 0.75f;
  } else {
    b = d >> 1;
    a = max(b - 1, 0);
    wa = 0.25f;
  }
}
__global__ void prolong_kernel(float *__restrict__ p, const float *__restrict__ pc,
                               const uint8_t *__restrict__ mask, int nx, int ny, int nz) {
  // 32-bit index arithmetic (the host checks nx ny nz < 2^31)
  const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
  const unsigned n = (unsigned)nx * (unsigned)ny * (unsigned)nz;
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (!(mask[v] & BSP_CLASS_FLUID)) {
      p[v] = 0.0f;
      continue;
    }
    const unsigned r = v / (unsigned)nz;
    const int k = (int)(v - r * (unsigned)nz);
    const unsigned ii = r / (unsigned)ny;
    const int j = (int)(r - ii * (unsigned)ny), i = (int)ii;
    int i0, i1, j0, j1, k0, k1;
    float wi, wj, wk;
    lin2(i, cx, i0, i1, wi);
    lin2(j, cy, j0, j1, wj);
    lin2(k, cz, k0, k1, wk);
    auto at = [&](int a, int b, int c) {
      return __ldg(pc + ((unsigned)a * (unsigned)cy + (unsigned)b) * (unsigned)cz + (unsigned)c);
    };
    const float c00 = wk * at(i0, j0, k0) + (1.0f - wk) * at(i0, j0, k1);
    const float c01 = wk * at(i0, j1, k0) + (1.0f - wk) * at(i0, j1, k1);
    const float c10 = wk * at(i1, j0, k0) + (1.0f - wk) * at(i1, j0, k1);
    const float c11 = wk * at(i1, j1, k0) + (1.0f - wk) * at(i1, j1, k1);
    const float c0 = wj * c00 + (1.0f - wj) * c01, c1 = wj * c10 + (1.0f - wj) * c11;
    p[v] = wi * c0 + (1.0f - wi) * c1;
  }
}

// The same interpolation for four consecutive k cells per thread (nz % 4 ==
// 0, p 16-byte aligned): the row and column terms and the index divisions once
// per four cells, the mask read as one word, p written as one float4.
__global__ void prolong4_kernel(float *__restrict__ p, const float *__restrict__ pc,
                                const uint8_t *__restrict__ mask, int nx, int ny, int nz) {
  const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
  const unsigned nzq = (unsigned)nz / 4u;
  const unsigned nq = (unsigned)nx * (unsigned)ny * nzq;
  for (unsigned u = blockIdx.x * blockDim.x + threadIdx.x; u < nq; u += gridDim.x * blockDim.x) {
    const unsigned v = 4u * u;
    const uint32_t mw = *reinterpret_cast<const uint32_t *>(mask + v);
    float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (mw & 0x80808080u) {
      const unsigned r = u / nzq;
      const int k = 4 * (int)(u - r * nzq);
      const unsigned ii = r / (unsigned)ny;
      const int j = (int)(r - ii * (unsigned)ny), i = (int)ii;
      int i0, i1, j0, j1;
      float wi, wj;
      lin2(i, cx, i0, i1, wi);
      lin2(j, cy, j0, j1, wj);
      const float *r00 = pc + ((unsigned)i0 * (unsigned)cy + (unsigned)j0) * (unsigned)cz;
      const float *r01 = pc + ((unsigned)i0 * (unsigned)cy + (unsigned)j1) * (unsigned)cz;
      const float *r10 = pc + ((unsigned)i1 * (unsigned)cy + (unsigned)j0) * (unsigned)cz;
      const float *r11 = pc + ((unsigned)i1 * (unsigned)cy + (unsigned)j1) * (unsigned)cz;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (!((mw >> (8 * q)) & BSP_CLASS_FLUID)) continue;
        int k0, k1;
        float wk;
        lin2(k + q, cz, k0, k1, wk);
        const float c00 = wk * __ldg(r00 + k0) + (1.0f - wk) * __ldg(r00 + k1);
        const float c01 = wk * __ldg(r01 + k0) + (1.0f - wk) * __ldg(r01 + k1);
        const float c10 = wk * __ldg(r10 + k0) + (1.0f - wk) * __ldg(r10 + k1);
        const float c11 = wk * __ldg(r11 + k0) + (1.0f - wk) * __ldg(r11 + k1);
        const float c0 = wj * c00 + (1.0f - wj) * c01, c1 = wj * c10 + (1.0f - wj) * c11;
        o[q] = wi * c0 + (1.0f - wi) * c1;
      }
    }
    *reinterpret_cast<float4 *>(p + v) = make_float4(o[0], o[1], o[2], o[3]);
  }
}

// s = RMS of div over the fluid cells (1 when there is none or it is 0): the
// network's input scale, on the device.  Per-block FP64 partials of
// (sum div^2, count) in a fixed order, then one block sums them in order.
constexpr int RMS_BLOCKS = 592;
__global__ void __launch_bounds__(256) rms_partial_kernel(double *__restrict__ part,
                                                          const float *__restrict__ div,
                                                          const uint8_t *__restrict__ mask,
                                                          int64_t n) {
  __shared__ double sh[2][8];
  double a = 0.0, c = 0.0;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    if (mask[v] & BSP_CLASS_FLUID) {
      const double d = div[v];
      a += d * d;
      c += 1.0;
    }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = a;
    sh[1][threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0.0, sc = 0.0;
    for (int w = 0; w < 8; ++w) {
      sa += sh[0][w];
      sc += sh[1][w];
    }
    part[2 * blockIdx.x] = sa;
    part[2 * blockIdx.x + 1] = sc;
  }
}
__global__ void rms_final_kernel(float *__restrict__ s_out, const double *__restrict__ part,
                                 int nb) {
  // one warp: lane l sums blocks l, l + 32, ..., then a fixed shuffle tree
  double a = 0.0, c = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) {
    a += part[2 * b];
    c += part[2 * b + 1];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if (threadIdx.x == 0) {
    const double r = c > 0.0 ? sqrt(a / c) : 0.0;
    s_out[0] = r > 0.0 ? (float)r : 1.0f;
  }
}

// Energy-optimal scale of a starting pressure: with b = factor div on fluid
// cells, gamma = (b . p) / (p . A p) minimises ||p* - gamma p||_A, so the
// scaled guess is never farther from the solution than zero in the A-norm.
// Partials of (b . p, p . Ap, b . b, b . Ap, Ap . Ap) per block in FP64,
// fixed order; the last three give the residual of the scaled guess,
// ||b - gamma A p||^2 = b.b - 2 gamma b.Ap + gamma^2 Ap.Ap.
constexpr int EN_SUMS = 5;
__global__ void __launch_bounds__(256) energy_partial_kernel(double *__restrict__ part,
                                                             const float *__restrict__ p,
                                                             const float *__restrict__ Ap,
                                                             const float *__restrict__ div,
                                                             const uint8_t *__restrict__ mask,
                                                             int64_t n, float factor) {
  // four cells per step (float4 loads, one mask word): the four products
  // summed in FP32, widened once, the sums over steps, threads and blocks in
  // FP64 and a fixed order
  __shared__ double sh[EN_SUMS][8];
  double acc[EN_SUMS] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int64_t n4 = n >> 2;
  const float4 *p4 = reinterpret_cast<const float4 *>(p);
  const float4 *a4 = reinterpret_cast<const float4 *>(Ap);
  const float4 *d4 = reinterpret_cast<const float4 *>(div);
  const uint32_t *m4 = reinterpret_cast<const uint32_t *>(mask);
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n4;
       v += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t mw = __ldg(m4 + v);
    if (!(mw & 0x80808080u)) continue;  // no fluid cell among the four
    const float4 pv = __ldg(p4 + v), av = __ldg(a4 + v), dv = __ldg(d4 + v);
    // values of non-fluid cells selected away (never multiplied by 0, so a
    // non-finite value there cannot leak in)
    const bool q0 = mw & 0x80u, q1 = mw & 0x8000u, q2 = mw & 0x800000u, q3 = mw & 0x80000000u;
    const float b0 = q0 ? factor * dv.x : 0.0f, b1 = q1 ? factor * dv.y : 0.0f;
    const float b2 = q2 ? factor * dv.z : 0.0f, b3 = q3 ? factor * dv.w : 0.0f;
    const float p0 = q0 ? pv.x : 0.0f, p1 = q1 ? pv.y : 0.0f, p2 = q2 ? pv.z : 0.0f,
                p3 = q3 ? pv.w : 0.0f;
    const float A0 = q0 ? av.x : 0.0f, A1 = q1 ? av.y : 0.0f, A2 = q2 ? av.z : 0.0f,
                A3 = q3 ? av.w : 0.0f;
    acc[0] += (double)((b0 * p0 + b1 * p1) + (b2 * p2 + b3 * p3));
    acc[1] += (double)((p0 * A0 + p1 * A1) + (p2 * A2 + p3 * A3));
    acc[2] += (double)((b0 * b0 + b1 * b1) + (b2 * b2 + b3 * b3));
    acc[3] += (double)((b0 * A0 + b1 * A1) + (b2 * A2 + b3 * A3));
    acc[4] += (double)((A0 * A0 + A1 * A1) + (A2 * A2 + A3 * A3));
  }
  // the n mod 4 tail cells, by block 0
  if (blockIdx.x == 0 && threadIdx.x < (int)(n & 3)) {
    const int64_t v = (n4 << 2) + threadIdx.x;
    if (mask[v] & BSP_CLASS_FLUID) {
      const float b = factor * div[v];
      acc[0] += (double)(b * p[v]);
      acc[1] += (double)(p[v] * Ap[v]);
      acc[2] += (double)(b * b);
      acc[3] += (double)(b * Ap[v]);
      acc[4] += (double)(Ap[v] * Ap[v]);
    }
  }
#pragma unroll
  for (int k = 0; k < EN_SUMS; ++k)
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < EN_SUMS; ++k) sh[k][threadIdx.x >> 5] = acc[k];
  __syncthreads();
  if (threadIdx.x < EN_SUMS) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[threadIdx.x][w];
    part[EN_SUMS * blockIdx.x + threadIdx.x] = t;
  }
}
// gamma from the partials (0 when p . A p is not positive), then p *= gamma.
// With keep_below > 0 the guess is dropped (gamma = 0: the solve starts from
// zero) unless the relative residual of the scaled guess,
// ||b - gamma A p|| / ||b||, is below keep_below.  The first warp of each
// block sums the partials: lane l takes blocks l, l + 32, ..., then a fixed
// shuffle tree (the same order in every block).
__global__ void energy_scale_kernel(float *__restrict__ p, const double *__restrict__ part,
                                    int nb, int64_t n, float keep_below,
                                    float *__restrict__ gamma_out,
                                    float *__restrict__ relres_out) {
  __shared__ float g;
  if (threadIdx.x < 32) {
    double t[EN_SUMS] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += 32)
#pragma unroll
      for (int k = 0; k < EN_SUMS; ++k) t[k] += part[EN_SUMS * b + k];
#pragma unroll
    for (int k = 0; k < EN_SUMS; ++k)
      for (int o = 16; o > 0; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
    if (threadIdx.x == 0) {
      const double a = t[0], c = t[1], bb = t[2], bA = t[3], AA = t[4];
      const double gd = (c > 0.0 && a == a) ? a / c : 0.0;
      const double rr = fmax(bb - 2.0 * gd * bA + gd * gd * AA, 0.0);
      const double rel = bb > 0.0 ? sqrt(rr / bb) : 0.0;
      const bool keep = keep_below <= 0.0f || rel < (double)keep_below;
      g = keep ? (float)gd : 0.0f;
      if (blockIdx.x == 0 && gamma_out) *gamma_out = g;
      if (blockIdx.x == 0 && relres_out) *relres_out = (float)rel;
    }
  }
  __syncthreads();
  const float gg = g;
  const int64_t n4 = n >> 2;
  float4 *p4 = reinterpret_cast<float4 *>(p);
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n4;
       v += (int64_t)gridDim.x * blockDim.x) {
    float4 x = p4[v];
    x.x *= gg;
    x.y *= gg;
    x.z *= gg;
    x.w *= gg;
    p4[v] = x;
  }
  if (blockIdx.x == 0 && threadIdx.x < (int)(n & 3)) p[(n4 << 2) + threadIdx.x] *= gg;
}

inline int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

static bool encode_rows(CUtensorMap *m, const void *base, int c, int64_t rows) {
  auto fn = encode_tiled();
  if (!fn || ((uintptr_t)base & 15u)) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)c, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)c * 2};
  const cuuint32_t box[2] = {16, (cuuint32_t)M};  // 32-byte rows: one sector each
  const cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
            es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static int g_utc_trace_on = 0;  // host switch of the cycle accounting
// BSP_TUNE_CONV_EPILOGUE: epilogue warpgroups (1 = two CTAs per SM, 2, 3 or
// 4); 0 (default) chooses per layer: two CTAs per SM for 16 output channels
// (N = 48: the issue streams, not the epilogue, limit those layers; measured
// 0.252 -> 0.195 ms for 16 -> 16 at 192x192x128), else two warpgroups
int g_utc_nepi = 0;

int cout_tile(int cout) { return cout % 64 == 0 ? 64 : (cout % 32 == 0 ? 32 : 16); }

int num_sms_dev() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

}  // namespace utc
}  // namespace bsp

using namespace bsp;
using namespace bsp::utc;

extern "C" int64_t bsp_unet_tc_rows(int nx, int ny, int nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
  return (int64_t)(nx + 2) * (ny + 2) * (nz + 2);
}

extern "C" int bsp_unet_tc_weights(bsp_bf16_t *wimg, const bsp_bf16_t *w, int cin, int cout,
                                   cudaStream_t s) {
  if (!wimg || !w) return BSP_ERR_NULL;
  if (cin <= 0 || cin % 16 || cout <= 0 || cout % 16) return BSP_ERR_SHAPE;
  ProfScope ps(PROF_UNET, s);
  weight_image_kernel<<<grid_for(27LL * cin * cout), 256, 0, s>>>(
      reinterpret_cast<__nv_bfloat16 *>(wimg), reinterpret_cast<const __nv_bfloat16 *>(w), cin,
      cout, cout_tile(cout));
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_tc_conv3(bsp_bf16_t *out, const bsp_bf16_t *in, const bsp_bf16_t *wimg,
                                 const float *bias, const bsp_bf16_t *skip, int nx, int ny, int nz,
                                 int cin, int cout, int relu, cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!out || !in || !wimg) return BSP_ERR_NULL;
  if (cin <= 0 || cin % 16 || cout <= 0 || cout % 16 || cin > 1024) return BSP_ERR_SHAPE;
  if (((uintptr_t)in & 15u) || ((uintptr_t)out & 15u) || ((uintptr_t)wimg & 15u) ||
      ((uintptr_t)skip & 15u))
    return BSP_ERR_ALIGN;
  if ((const void *)out == (const void *)in || (skip && (const void *)skip == (const void *)out))
    return BSP_ERR_ALIAS;
  if (((uintptr_t)bias & 15u)) return BSP_ERR_ALIGN;
  const int64_t rows = bsp_unet_tc_rows(nx, ny, nz);
  if (rows >= ROWS_MAX) return BSP_ERR_SHAPE;  // 32-bit row arithmetic, TMA coordinates
  Params p{};
  p.out = reinterpret_cast<__nv_bfloat16 *>(out);
  p.wimg = reinterpret_cast<const __nv_bfloat16 *>(wimg);
  p.bias = bias;
  p.skip = reinterpret_cast<const __nv_bfloat16 *>(skip);
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  p.cin = cin;
  p.cout = cout;
  p.ct = cout_tile(cout);
  p.nct = cout / p.ct;
  p.relu = relu;
  const int64_t R = nz + 2, P = (int64_t)(ny + 2) * R;
  p.r0 = (int)(P + R + 1);
  const int64_t rlast = (int64_t)nx * P + ny * R + nz;
  p.rows = (int)rows;
  const int64_t ntiles = (rlast - p.r0 + MOUT) / MOUT;
  p.nwork = (int)(ntiles * p.nct);
  p.trace = g_utc_trace_on;
  const int N = 3 * p.ct;
  p.w_bytes_chunk = 9 * 2 * N * 16;
  const int nchunk = cin / 16;
  const int wtotal = p.w_bytes_chunk * nchunk;
  const int ctl = (int)((sizeof(Ctl) + 127) / 128 * 128);
  // one CTA per SM with up to 227 KB, or (one epilogue warpgroup) two CTAs per
  // SM with 112 KB each; weights stay resident when they leave room for two
  // stages
  // (a layer whose streamed weights leave no room for two stages in half the
  // shared memory runs one CTA per SM with two epilogue warpgroups)
  int nepi = g_utc_nepi > 0 ? g_utc_nepi : (cout == 16 ? 1 : 2);
  int per_sm = 1, budget = SMEM_MAX, wres_max = WRES_MAX;
  for (int pass = 0; pass < 2; ++pass) {
    per_sm = nepi == 1 ? 2 : 1;
    budget = per_sm == 2 ? SMEM_PAIR : SMEM_MAX;
    wres_max = per_sm == 2 ? budget - 1024 - ctl - 2 * A_STAGE : WRES_MAX;
    p.resident = (p.nct == 1 && round1k(wtotal) <= wres_max) ? 1 : 0;
    const int stage = round1k(A_STAGE + (p.resident ? 0 : p.w_bytes_chunk));
    p.nst = (budget - 1024 - ctl - (p.resident ? round1k(wtotal) : 0)) / stage;
    if (p.nst >= 2 || nepi != 1) break;
    nepi = 2;
  }
  if (p.nst > 8) p.nst = 8;
  if (p.nst < 2) return BSP_ERR_SHAPE;
  const int stage = round1k(A_STAGE + (p.resident ? 0 : p.w_bytes_chunk));
  int bytes = 1024 + (p.resident ? round1k(wtotal) : 0) + p.nst * stage + ctl;
  if (per_sm == 1 && bytes < SMEM_MIN) bytes = SMEM_MIN;
  CUtensorMap amap;
  if (!encode_rows(&amap, in, cin, rows)) return BSP_ERR_ARG;
  const int slots = per_sm * num_sms_dev();
  const int grid = p.nwork < slots ? p.nwork : slots;
  ProfScope ps(PROF_UNET, s);
  if (nepi == 1) {
    if (!smem_opt_in((const void *)conv_tc_kernel<1>, SMEM_MAX)) return BSP_ERR_ARG;
    conv_tc_kernel<1><<<grid, conv_threads(1), bytes, s>>>(amap, p);
  } else if (nepi == 3) {
    if (!smem_opt_in((const void *)conv_tc_kernel<3>, SMEM_MAX)) return BSP_ERR_ARG;
    conv_tc_kernel<3><<<grid, conv_threads(3), bytes, s>>>(amap, p);
  } else if (nepi == 2) {
    if (!smem_opt_in((const void *)conv_tc_kernel<2>, SMEM_MAX)) return BSP_ERR_ARG;
    conv_tc_kernel<2><<<grid, conv_threads(2), bytes, s>>>(amap, p);
  } else {
    if (!smem_opt_in((const void *)conv_tc_kernel<4>, SMEM_MAX)) return BSP_ERR_ARG;
    conv_tc_kernel<4><<<grid, conv_threads(4), bytes, s>>>(amap, p);
  }
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_tc_trace(unsigned long long *counters_host, int enable) {
  cudaError_t e = cudaSuccess;
  if (counters_host) e = cudaMemcpyFromSymbol(counters_host, g_utc_trace, sizeof(g_utc_trace));
  if (e == cudaSuccess) {
    const unsigned long long zero[8] = {};
    e = cudaMemcpyToSymbol(g_utc_trace, zero, sizeof(zero));
  }
  g_utc_trace_on = enable ? 1 : 0;
  return (int)e;
}

extern "C" int bsp_unet_tc_error(int *flag_host) {
  if (!flag_host) return BSP_ERR_NULL;
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_utc_err, sizeof(int));
  if (e == cudaSuccess) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_utc_err, &zero, sizeof(int));
  }
  *flag_host = v;
  return (int)e;
}

extern "C" size_t bsp_unet_scale_workspace_bytes(void) {
  return sizeof(double) * EN_SUMS * RMS_BLOCKS;
}

extern "C" int bsp_unet_input_scale(float *s_dev, const float *div, const uint8_t *mask, int nx,
                                    int ny, int nz, void *workspace, size_t workspace_bytes,
                                    cudaStream_t s) {
  if (!s_dev || !div || !mask || !workspace) return BSP_ERR_NULL;
  if (workspace_bytes < bsp_unet_scale_workspace_bytes() || ((uintptr_t)workspace & 7u))
    return BSP_ERR_WORKSPACE;
  ProfScope ps(PROF_UNET, s);
  rms_partial_kernel<<<RMS_BLOCKS, 256, 0, s>>>(static_cast<double *>(workspace), div, mask,
                                                (int64_t)nx * ny * nz);
  rms_final_kernel<<<1, 32, 0, s>>>(s_dev, static_cast<const double *>(workspace), RMS_BLOCKS);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_tc_pack(bsp_bf16_t *x, const float *div, const uint8_t *mask, int nx,
                                int ny, int nz, const float *s_dev, cudaStream_t s) {
  if (!x || !div || !mask || !s_dev) return BSP_ERR_NULL;
  const int64_t rows = bsp_unet_tc_rows(nx, ny, nz);
  ProfScope ps(PROF_UNET, s);
  pack_pad_kernel<<<grid_for(rows), 256, 0, s>>>(reinterpret_cast<__nv_bfloat16 *>(x), div, mask,
                                                 nx, ny, nz, s_dev, rows);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_tc_pool(bsp_bf16_t *out, const bsp_bf16_t *in, int nx, int ny, int nz,
                                int c, cudaStream_t s) {
  if (!out || !in) return BSP_ERR_NULL;
  if (nx % 2 || ny % 2 || nz % 2 || c % 8) return BSP_ERR_SHAPE;
  const int64_t rows = bsp_unet_tc_rows(nx / 2, ny / 2, nz / 2);
  ProfScope ps(PROF_UNET, s);
  pool_pad_kernel<<<grid_for(rows * (c / 8)), 256, 0, s>>>(
      reinterpret_cast<__nv_bfloat16 *>(out), reinterpret_cast<const __nv_bfloat16 *>(in), nx,
      ny, nz, c);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_tc_up(bsp_bf16_t *out, const bsp_bf16_t *in, int nx, int ny, int nz,
                              int c, cudaStream_t s) {
  if (!out || !in) return BSP_ERR_NULL;
  if (nx % 2 || ny % 2 || nz % 2 || c % 8) return BSP_ERR_SHAPE;
  const int64_t rows = bsp_unet_tc_rows(nx, ny, nz);
  ProfScope ps(PROF_UNET, s);
  up_pad_kernel<<<grid_for(rows * (c / 8)), 256, 0, s>>>(
      reinterpret_cast<__nv_bfloat16 *>(out), reinterpret_cast<const __nv_bfloat16 *>(in), nx,
      ny, nz, c);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_tc_head(float *p, const bsp_bf16_t *x, const float *hw, const float *hb,
                                const uint8_t *mask, int nx, int ny, int nz, const float *s_dev,
                                float factor, cudaStream_t s) {
  if (!p || !x || !hw || !hb || !mask || !s_dev) return BSP_ERR_NULL;
  ProfScope ps(PROF_UNET, s);
  head_pad_kernel<<<grid_for((int64_t)nx * ny * nz), 256, 0, s>>>(
      p, reinterpret_cast<const __nv_bfloat16 *>(x), hw, hb, mask, nx, ny, nz, s_dev, factor);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_restrict_div(float *divc, const uint8_t *maskc, const float *div,
                                     const uint8_t *mask, int nx, int ny, int nz,
                                     cudaStream_t s) {
  if (!divc || !maskc || !div || !mask) return BSP_ERR_NULL;
  if (nx % 2 || ny % 2 || nz % 2 || nx <= 0 || ny <= 0 || nz <= 0) return BSP_ERR_SHAPE;
  if ((int64_t)nx * ny * nz >= ((int64_t)1 << 31)) return BSP_ERR_SHAPE;
  ProfScope ps(PROF_UNET, s);
  restrict_div_kernel<<<grid_for((int64_t)nx * ny * nz / 8), 256, 0, s>>>(divc, maskc, div, mask,
                                                                            nx, ny, nz);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_prolong(float *p, const float *pc, const uint8_t *mask, int nx, int ny,
                                int nz, cudaStream_t s) {
  if (!p || !pc || !mask) return BSP_ERR_NULL;
  if (nx % 2 || ny % 2 || nz % 2 || nx <= 0 || ny <= 0 || nz <= 0) return BSP_ERR_SHAPE;
  if ((int64_t)nx * ny * nz >= ((int64_t)1 << 31)) return BSP_ERR_SHAPE;
  if ((const void *)p == (const void *)pc) return BSP_ERR_ALIAS;
  ProfScope ps(PROF_UNET, s);
  if (nz % 4 == 0 && ((uintptr_t)p & 15u) == 0 && ((uintptr_t)mask & 3u) == 0)
    prolong4_kernel<<<grid_for((int64_t)nx * ny * nz / 4), 256, 0, s>>>(p, pc, mask, nx, ny, nz);
  else
    prolong_kernel<<<grid_for((int64_t)nx * ny * nz), 256, 0, s>>>(p, pc, mask, nx, ny, nz);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_energy_scale_keep(float *p, const float *Ap, const float *div,
                                          const uint8_t *mask, int nx, int ny, int nz,
                                          float factor, float keep_below, void *workspace,
                                          size_t workspace_bytes, float *gamma_dev,
                                          float *relres_dev, cudaStream_t s);

extern "C" int bsp_unet_energy_scale(float *p, const float *Ap, const float *div,
                                     const uint8_t *mask, int nx, int ny, int nz, float factor,
                                     void *workspace, size_t workspace_bytes, float *gamma_dev,
                                     cudaStream_t s) {
  return bsp_unet_energy_scale_keep(p, Ap, div, mask, nx, ny, nz, factor, 0.0f, workspace,
                                    workspace_bytes, gamma_dev, nullptr, s);
}

extern "C" int bsp_unet_energy_scale_keep(float *p, const float *Ap, const float *div,
                                          const uint8_t *mask, int nx, int ny, int nz,
                                          float factor, float keep_below, void *workspace,
                                          size_t workspace_bytes, float *gamma_dev,
                                          float *relres_dev, cudaStream_t s) {
  if (!p || !Ap || !div || !mask || !workspace) return BSP_ERR_NULL;
  if (workspace_bytes < bsp_unet_scale_workspace_bytes() || ((uintptr_t)workspace & 7u))
    return BSP_ERR_WORKSPACE;
  if ((const void *)p == (const void *)Ap) return BSP_ERR_ALIAS;
  // float4 / 4-byte mask-word access
  if (((uintptr_t)p | (uintptr_t)Ap | (uintptr_t)div) & 15u || ((uintptr_t)mask & 3u))
    return BSP_ERR_ALIGN;
  const int64_t n = (int64_t)nx * ny * nz;
  if (n <= 0) return BSP_OK;
  ProfScope ps(PROF_UNET, s);
  energy_partial_kernel<<<RMS_BLOCKS, 256, 0, s>>>(static_cast<double *>(workspace), p, Ap, div,
                                                   mask, n, factor);
  // every block first sums the partials: two blocks per SM, grid-stride
  const int sblocks = std::min(grid_for((n + 3) / 4), 2 * num_sms_dev());
  energy_scale_kernel<<<sblocks, 256, 0, s>>>(
      p, static_cast<const double *>(workspace), RMS_BLOCKS, n, keep_below, gamma_dev,
      relres_dev);
  return (int)cudaGetLastError();
}
