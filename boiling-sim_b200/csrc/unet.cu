// unet.cu -- kernels of the learned warm start: a small 3-D U-Net over the
// pot grid, trained and run on the GPU by these kernels alone.
//
// Activations are channels-last BF16, act[v][c] with v = (i*ny + j)*nz + k;
// weights of a 3x3x3 convolution are BF16 w[tap][co][ci] (tap = (di+1)*9 +
// (dj+1)*3 + (dk+1)), with an FP32 master copy kept by the optimiser.
//
// The convolution is an implicit GEMM on the tensor cores (mma.sync
// m16n8k16, BF16 operands, FP32 accumulate): M = voxels, N = output
// channels, K = 27 taps x input channels in chunks of 16.  A CTA of 4 warps
// owns 128 voxels x NT output channels; per K chunk the 128 x 16 activation
// tile (gathered through the tap's neighbour offset, zero outside the grid)
// and the NT x 16 weight tile are staged in shared memory by cp.async and
// read with ldmatrix.  The backward pass of the data is the same kernel on
// the output gradient with the weights flipped in space and transposed in
// channels; the weight gradient is a second implicit GEMM (M = output
// channels, N = input channels, K = voxels) accumulated per voxel chunk into
// FP32 partials that a fixed-order reduction sums (deterministic).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "bsproj.h"

namespace bsp {
namespace unet {

constexpr int CT = 128;     // threads per conv CTA (4 warps)
constexpr int MT = 128;     // voxels per conv CTA
constexpr int ROWB = 48;    // smem row stride in bytes for 16 bf16 (32 B) + pad: conflict-free ldmatrix

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid) {
  // src-size 0 zero-fills the 16 destination bytes
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void ldsm_x4(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3,
                                        const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_addr(p)));
}
__device__ __forceinline__ void ldsm_x2(uint32_t &r0, uint32_t &r1, const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];"
               : "=r"(r0), "=r"(r1)
               : "r"(smem_addr(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3,
                                          const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_addr(p)));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ---- convolution, forward (and backward data with flipped weights) ------------------------
// out[v][co] = act(bias[co] + sum_{tap, ci} in[v + d(tap)][ci] * w[tap][co][ci])
// NT output channels per CTA (16, 32 or 64); cin % 16 == 0; cout % NT == 0.
template <int NT>
__global__ void __launch_bounds__(CT) conv3_fwd_kernel(__nv_bfloat16 *__restrict__ out,
                                                       const __nv_bfloat16 *__restrict__ in,
                                                       const __nv_bfloat16 *__restrict__ w,
                                                       const float *__restrict__ bias, int nx,
                                                       int ny, int nz, int cin, int cout,
                                                       int relu) {
  __shared__ __align__(128) unsigned char sA[2][MT * ROWB];
  __shared__ __align__(128) unsigned char sB[2][NT * ROWB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t nvox = (int64_t)nx * ny * nz;
  const int64_t v0 = (int64_t)blockIdx.x * MT;
  const int co0 = blockIdx.y * NT;
  // this thread stages rows tid (A: one 32-byte row = 2 x 16 B per thread)
  const int64_t va = v0 + tid;
  const bool vin = va < nvox;
  int ia = 0, ja = 0, ka = 0;
  if (vin) {
    ka = (int)(va % nz);
    const int64_t rj = va / nz;
    ja = (int)(rj % ny);
    ia = (int)(rj / ny);
  }
  const int nchunk = cin >> 4;
  const int ksteps = 27 * nchunk;
  auto stage = [&](int s, int buf) {
    const int tap = s / nchunk, c0 = (s - tap * nchunk) << 4;
    const int di = tap / 9 - 1, dj = (tap / 3) % 3 - 1, dk = tap % 3 - 1;
    const int ii = ia + di, jj = ja + dj, kk = ka + dk;
    const bool ok = vin && ii >= 0 && ii < nx && jj >= 0 && jj < ny && kk >= 0 && kk < nz;
    const __nv_bfloat16 *src = ok ? in + (((int64_t)ii * ny + jj) * nz + kk) * cin + c0 : in;
    unsigned char *dst = sA[buf] + tid * ROWB;
    cp_async16(dst, src, ok);
    cp_async16(dst + 16, src + 8, ok);
    // weights: NT rows of 32 bytes
    for (int r = tid; r < NT * 2; r += CT) {
      const int row = r >> 1, half = r & 1;
      const __nv_bfloat16 *ws = w + ((int64_t)tap * cout + co0 + row) * cin + c0 + half * 8;
      cp_async16(sB[buf] + row * ROWB + half * 16, ws, true);
    }
    cp_async_commit();
  };
  float acc[2][NT / 8][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int n = 0; n < NT / 8; ++n)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[m][n][q] = 0.0f;
  stage(0, 0);
  for (int s = 0; s < ksteps; ++s) {
    const int buf = s & 1;
    if (s + 1 < ksteps) {
      stage(s + 1, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    uint32_t a[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int row = warp * 32 + m * 16 + (lane & 15);
      ldsm_x4(a[m][0], a[m][1], a[m][2], a[m][3], sA[buf] + row * ROWB + (lane >> 4) * 16);
    }
#pragma unroll
    for (int n = 0; n < NT / 8; ++n) {
      uint32_t b0, b1;
      // rows n*8 + (lane & 7), k half (lane >> 3) & 1
      ldsm_x2(b0, b1, sB[buf] + (n * 8 + (lane & 7)) * ROWB + ((lane >> 3) & 1) * 16);
#pragma unroll
      for (int m = 0; m < 2; ++m) mma_bf16(acc[m][n], a[m][0], a[m][1], a[m][2], a[m][3], b0, b1);
    }
    __syncthreads();
  }
  // epilogue: rows g and g + 8 of each m16 tile, columns 2t, 2t+1 of each n8 tile
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t v = v0 + warp * 32 + m * 16 + g + h * 8;
      if (v >= nvox) continue;
#pragma unroll
      for (int n = 0; n < NT / 8; ++n) {
        const int co = co0 + n * 8 + t4 * 2;
        float x0 = acc[m][n][2 * h], x1 = acc[m][n][2 * h + 1];
        if (bias) {
          x0 += bias[co];
          x1 += bias[co + 1];
        }
        if (relu) {
          x0 = fmaxf(x0, 0.0f);
          x1 = fmaxf(x1, 0.0f);
        }
        *reinterpret_cast<__nv_bfloat162 *>(out + v * cout + co) = __floats2bfloat162_rn(x0, x1);
      }
    }
}

// ---- convolution, weight gradient -----------------------------------------------------------
// part[chunk][tap][co][ci] = sum over the chunk's voxels v of g[v][co] * in[v + d(tap)][ci]
// (FP32).  CTA: 4 warps, a 64 x 64 (co x ci) tile of one tap, VCH voxels.
constexpr int WG_VCH = 2048;  // voxels per chunk
constexpr int WG_KV = 32;     // voxels per staged step
constexpr int WG_ROW = 144;   // 64 bf16 (128 B) + 16 B pad per staged voxel row

__global__ void __launch_bounds__(CT) conv3_wgrad_kernel(float *__restrict__ part,
                                                         const __nv_bfloat16 *__restrict__ g,
                                                         const __nv_bfloat16 *__restrict__ in,
                                                         int nx, int ny, int nz, int cin,
                                                         int cout) {
  __shared__ __align__(128) unsigned char sG[2][WG_KV * WG_ROW];
  __shared__ __align__(128) unsigned char sI[2][WG_KV * WG_ROW];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t nvox = (int64_t)nx * ny * nz;
  const int chunk = blockIdx.x;
  const int tap = blockIdx.z;
  const int ntile_ci = (cin + 63) / 64;
  const int co0 = (blockIdx.y / ntile_ci) * 64, ci0 = (blockIdx.y % ntile_ci) * 64;
  const int nco = min(64, cout - co0), nci = min(64, cin - ci0);
  const int di = tap / 9 - 1, dj = (tap / 3) % 3 - 1, dk = tap % 3 - 1;
  const int64_t vbeg = (int64_t)chunk * WG_VCH;
  const int64_t vend = min(vbeg + WG_VCH, nvox);
  // staging: WG_KV voxel rows x 64 channels = 8 x 16 B per row for g and for in;
  // 128 threads: each stages 2 segments of g and 2 of in per step
  auto stage = [&](int64_t vs, int buf) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int idx = tid + q * CT;  // 0 .. 255
      const int row = idx >> 3, seg = idx & 7;
      const int64_t v = vs + row;
      const bool vok = v < vend;
      // gradient of the output at v
      const bool gok = vok && seg * 8 < nco;
      cp_async16(sG[buf] + row * WG_ROW + seg * 16, gok ? g + v * cout + co0 + seg * 8 : g, gok);
      // input at v + d(tap)
      bool iok = vok && seg * 8 < nci;
      const __nv_bfloat16 *src = in;
      if (iok) {
        const int k = (int)(v % nz);
        const int64_t rj = v / nz;
        const int j = (int)(rj % ny), i = (int)(rj / ny);
        const int ii = i + di, jj = j + dj, kk = k + dk;
        iok = ii >= 0 && ii < nx && jj >= 0 && jj < ny && kk >= 0 && kk < nz;
        if (iok) src = in + (((int64_t)ii * ny + jj) * nz + kk) * cin + ci0 + seg * 8;
      }
      cp_async16(sI[buf] + row * WG_ROW + seg * 16, src, iok);
    }
    cp_async_commit();
  };
  // warp tile: co rows warp*16 .. +16 (M), all 64 ci (8 n8 tiles)
  float acc[8][4];
#pragma unroll
  for (int n = 0; n < 8; ++n)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[n][q] = 0.0f;
  const int nsteps = (int)((vend - vbeg + WG_KV - 1) / WG_KV);
  if (nsteps > 0) stage(vbeg, 0);
  for (int s = 0; s < nsteps; ++s) {
    const int buf = s & 1;
    if (s + 1 < nsteps) {
      stage(vbeg + (int64_t)(s + 1) * WG_KV, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < WG_KV; kk += 16) {
      // A = g^T (co x v): 8x8 blocks of sG (rows v, cols co) read transposed
      uint32_t a0, a1, a2, a3;
      {
        // matrices: (v kk..kk+7, co m..m+7), (v kk..+7, co m+8..), (v kk+8.., co m..), (v kk+8.., co m+8..)
        const int mat = lane >> 3, r = lane & 7;
        const int vrow = kk + (mat >> 1) * 8 + r;
        const int col = warp * 16 + (mat & 1) * 8;
        ldsm_x4_t(a0, a1, a2, a3, sG[buf] + vrow * WG_ROW + col * 2);
      }
#pragma unroll
      for (int n = 0; n < 8; n += 2) {
        // B = in (v x ci), col layout: 8x8 blocks (rows v, cols ci) read transposed
        uint32_t b0, b1, b2, b3;
        const int mat = lane >> 3, r = lane & 7;
        const int vrow = kk + (mat & 1) * 8 + r;
        const int col = (n + (mat >> 1)) * 8;
        ldsm_x4_t(b0, b1, b2, b3, sI[buf] + vrow * WG_ROW + col * 2);
        mma_bf16(acc[n], a0, a1, a2, a3, b0, b1);
        mma_bf16(acc[n + 1], a0, a1, a2, a3, b2, b3);
      }
    }
    __syncthreads();
  }
  const int gq = lane >> 2, t4 = lane & 3;
  float *dst = part + ((int64_t)chunk * 27 + tap) * cout * cin;
#pragma unroll
  for (int n = 0; n < 8; ++n)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int co = co0 + warp * 16 + gq + h * 8;
      const int ci = ci0 + n * 8 + t4 * 2;
      if (co < cout && ci < cin) {
        dst[(int64_t)co * cin + ci] = acc[n][2 * h];
        dst[(int64_t)co * cin + ci + 1] = acc[n][2 * h + 1];
      }
    }
}

// out[q] = sum over chunks of part[chunk][q] in chunk order (deterministic)
__global__ void sum_chunks_kernel(float *__restrict__ out, const float *__restrict__ part,
                                  int nchunk, int64_t n, float scale, int accumulate) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int c = 0; c < nchunk; ++c) s += part[(int64_t)c * n + q];
    out[q] = accumulate ? out[q] + scale * s : scale * s;
  }
}

__global__ void sum_slots_kernel(float *__restrict__ out, const float *__restrict__ partials,
                                 int nblocks) {
  float acc = 0.0f;
  for (int b = 0; b < nblocks; ++b) acc += partials[(int64_t)threadIdx.x * nblocks + b];
  out[threadIdx.x] = acc;
}

// bias gradient: db[co] = sum_v g[v][co]; one block per channel group, fixed order
__global__ void bias_grad_kernel(float *__restrict__ db, const __nv_bfloat16 *__restrict__ g,
                                 int64_t nvox, int cout) {
  __shared__ float sh[256];
  const int co = blockIdx.x;
  float s = 0.0f;
  for (int64_t v = threadIdx.x; v < nvox; v += blockDim.x) s += __bfloat162float(g[v * cout + co]);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[co] = sh[0];
}

// wt[tap'][ci][co] = w[26 - tap'][co][ci]: weights of the data-gradient convolution
__global__ void flip_weights_kernel(__nv_bfloat16 *__restrict__ wt,
                                    const __nv_bfloat16 *__restrict__ w, int cin, int cout) {
  const int64_t n = 27LL * cin * cout;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int co = (int)(q % cout);
    const int64_t r = q / cout;
    const int ci = (int)(r % cin);
    const int tp = (int)(r / cin);
    wt[q] = w[((int64_t)(26 - tp) * cout + co) * cin + ci];
  }
}

// g[v][c] *= (act[v][c] > 0): gradient through ReLU (act is the ReLU output)
__global__ void relu_bwd_kernel(__nv_bfloat16 *__restrict__ g, const __nv_bfloat16 *__restrict__ act,
                                int64_t n) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    if (!(__bfloat162float(act[q]) > 0.0f)) g[q] = __float2bfloat16(0.0f);
}

// 2x2x2 average pooling (channels-last); output dims (nx/2, ny/2, nz/2)
__global__ void pool_fwd_kernel(__nv_bfloat16 *__restrict__ out, const __nv_bfloat16 *__restrict__ in,
                                int nx, int ny, int nz, int c) {
  const int ox = nx / 2, oy = ny / 2, oz = nz / 2;
  const int64_t n = (int64_t)ox * oy * oz * c;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % c);
    int64_t v = q / c;
    const int k = (int)(v % oz);
    v /= oz;
    const int j = (int)(v % oy), i = (int)(v / oy);
    float s = 0.0f;
    for (int a = 0; a < 8; ++a) {
      const int ii = 2 * i + (a >> 2), jj = 2 * j + ((a >> 1) & 1), kk = 2 * k + (a & 1);
      s += __bfloat162float(in[(((int64_t)ii * ny + jj) * nz + kk) * c + ch]);
    }
    out[q] = __float2bfloat16(0.125f * s);
  }
}
// gradient of the pooling: gin[child] = gout[parent] / 8 (+= when accumulate)
__global__ void pool_bwd_kernel(__nv_bfloat16 *__restrict__ gin, const __nv_bfloat16 *__restrict__ gout,
                                int nx, int ny, int nz, int c, int accumulate) {
  const int64_t n = (int64_t)nx * ny * nz * c;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % c);
    int64_t v = q / c;
    const int k = (int)(v % nz);
    v /= nz;
    const int j = (int)(v % ny), i = (int)(v / ny);
    const int64_t p = ((((int64_t)(i >> 1) * (ny / 2) + (j >> 1)) * (nz / 2)) + (k >> 1)) * c + ch;
    float x = 0.125f * __bfloat162float(gout[p]);
    if (accumulate) x += __bfloat162float(gin[q]);
    gin[q] = __float2bfloat16(x);
  }
}
// nearest-neighbour x2 upsampling to (nx, ny, nz) from (nx/2, ny/2, nz/2), plus an
// optional skip tensor of the output's shape: out = up(in) + skip
__global__ void up_fwd_kernel(__nv_bfloat16 *__restrict__ out, const __nv_bfloat16 *__restrict__ in,
                              int nx, int ny, int nz, int c) {
  const int64_t n = (int64_t)nx * ny * nz * c;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % c);
    int64_t v = q / c;
    const int k = (int)(v % nz);
    v /= nz;
    const int j = (int)(v % ny), i = (int)(v / ny);
    const int64_t p = ((((int64_t)(i >> 1) * (ny / 2) + (j >> 1)) * (nz / 2)) + (k >> 1)) * c + ch;
    out[q] = in[p];
  }
}
// gradient of the upsampling: gin[parent] = sum of the 8 children's gout
__global__ void up_bwd_kernel(__nv_bfloat16 *__restrict__ gin, const __nv_bfloat16 *__restrict__ gout,
                              int nx, int ny, int nz, int c) {
  const int ox = nx / 2, oy = ny / 2, oz = nz / 2;
  const int64_t n = (int64_t)ox * oy * oz * c;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % c);
    int64_t v = q / c;
    const int k = (int)(v % oz);
    v /= oz;
    const int j = (int)(v % oy), i = (int)(v / oy);
    float s = 0.0f;
    for (int a = 0; a < 8; ++a) {
      const int ii = 2 * i + (a >> 2), jj = 2 * j + ((a >> 1) & 1), kk = 2 * k + (a & 1);
      s += __bfloat162float(gout[(((int64_t)ii * ny + jj) * nz + kk) * c + ch]);
    }
    gin[q] = __float2bfloat16(s);
  }
}
// a += b (BF16, elementwise; skip connections and gradient sums)
__global__ void add_kernel(__nv_bfloat16 *__restrict__ a, const __nv_bfloat16 *__restrict__ b,
                           int64_t n) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    a[q] = __float2bfloat16(__bfloat162float(a[q]) + __bfloat162float(b[q]));
}

// Network input: x[v][0] = rhs[v] / scale on fluid cells, x[v][1] = fluid flag,
// x[v][2] = solid flag, channels 3..15 zero.
__global__ void pack_input_kernel(__nv_bfloat16 *__restrict__ x, const float *__restrict__ div,
                                  const uint8_t *__restrict__ mask, int64_t nvox, float inv_scale) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t m = mask[v];
    const bool fl = (m & BSP_CLASS_FLUID) != 0;
    __nv_bfloat16 *o = x + v * 16;
    o[0] = __float2bfloat16(fl ? div[v] * inv_scale : 0.0f);
    o[1] = __float2bfloat16(fl ? 1.0f : 0.0f);
    o[2] = __float2bfloat16((m & BSP_CLASS_SOLID) ? 1.0f : 0.0f);
    for (int c = 3; c < 16; ++c) o[c] = __float2bfloat16(0.0f);
  }
}

// Head: y[v] = hb + sum_c hw[c] * x[v][c] (16 channels), masked to fluid cells;
// p[v] = scale * y[v] (FP32)
__global__ void head_fwd_kernel(float *__restrict__ p, const __nv_bfloat16 *__restrict__ x,
                                const float *__restrict__ hw, const float *__restrict__ hb,
                                const uint8_t *__restrict__ mask, int64_t nvox, float scale) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    float y = hb[0];
    for (int c = 0; c < 16; ++c) y = fmaf(hw[c], __bfloat162float(x[v * 16 + c]), y);
    p[v] = (mask[v] & BSP_CLASS_FLUID) ? scale * y : 0.0f;
  }
}

// Loss and head gradient: with y = prediction / scale and t = target / scale on
// fluid cells, loss = mean (y - t)^2; gx[v][c] = dL/dx = 2 (y - t) hw[c] / nfl;
// per-block partials of loss, dhw[16], dhb (FP32, deterministic order).
__global__ void __launch_bounds__(256) head_loss_kernel(
    __nv_bfloat16 *__restrict__ gx, float *__restrict__ partials, const float *__restrict__ pred,
    const float *__restrict__ target, const __nv_bfloat16 *__restrict__ x,
    const float *__restrict__ hw, const uint8_t *__restrict__ mask, int64_t nvox, float inv_scale,
    float inv_nfl) {
  float lsum = 0.0f, dhw[16], dhb = 0.0f;
#pragma unroll
  for (int c = 0; c < 16; ++c) dhw[c] = 0.0f;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    const bool fl = (mask[v] & BSP_CLASS_FLUID) != 0;
    const float d = fl ? (pred[v] - target[v]) * inv_scale : 0.0f;
    lsum += d * d;
    const float gy = 2.0f * d * inv_nfl;
    dhb += gy;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const float xc = __bfloat162float(x[v * 16 + c]);
      dhw[c] = fmaf(gy, xc, dhw[c]);
      gx[v * 16 + c] = __float2bfloat16(gy * hw[c]);
    }
  }
  __shared__ float sh[256];
  auto reduce = [&](float val, int slot) {
    sh[threadIdx.x] = val;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) partials[(int64_t)slot * gridDim.x + blockIdx.x] = sh[0];
    __syncthreads();
  };
  reduce(lsum * inv_nfl, 0);
  reduce(dhb, 1);
  for (int c = 0; c < 16; ++c) reduce(dhw[c], 2 + c);
}

// Head gradient for a given output gradient gy (dL/dy per voxel, 0 off fluid):
// gx[v][c] = gy[v] hw[c]; per-block partials of dhb (slot 0) and dhw (1..16).
__global__ void __launch_bounds__(256) head_bwd_kernel(
    __nv_bfloat16 *__restrict__ gx, float *__restrict__ partials, const float *__restrict__ gy,
    const __nv_bfloat16 *__restrict__ x, const float *__restrict__ hw,
    const uint8_t *__restrict__ mask, int64_t nvox) {
  float dhw[16], dhb = 0.0f;
#pragma unroll
  for (int c = 0; c < 16; ++c) dhw[c] = 0.0f;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    const float g = (mask[v] & BSP_CLASS_FLUID) ? gy[v] : 0.0f;
    dhb += g;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      dhw[c] = fmaf(g, __bfloat162float(x[v * 16 + c]), dhw[c]);
      gx[v * 16 + c] = __float2bfloat16(g * hw[c]);
    }
  }
  __shared__ float sh[256];
  auto reduce = [&](float val, int slot) {
    sh[threadIdx.x] = val;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) partials[(int64_t)slot * gridDim.x + blockIdx.x] = sh[0];
    __syncthreads();
  };
  reduce(dhb, 0);
  for (int c = 0; c < 16; ++c) reduce(dhw[c], 1 + c);
}

// Adam step on FP32 master weights, refreshing the BF16 copy.
__global__ void adam_kernel(float *__restrict__ w, __nv_bfloat16 *__restrict__ wb,
                            float *__restrict__ m, float *__restrict__ vv,
                            const float *__restrict__ g, int64_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * vv[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    vv[q] = vq;
    const float upd = lr * (mq * c1) / (sqrtf(vq * c2) + eps);
    const float wq = w[q] - upd;
    w[q] = wq;
    if (wb) wb[q] = __float2bfloat16(wq);
  }
}

inline int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

}  // namespace unet
}  // namespace bsp

using namespace bsp::unet;

extern "C" int bsp_unet_conv3_fwd(bsp_bf16_t *out_, const bsp_bf16_t *in_,
                                  const bsp_bf16_t *w_, const float *bias, int nx, int ny,
                                  int nz, int cin, int cout, int relu, cudaStream_t s) {
  __nv_bfloat16 *out = reinterpret_cast<__nv_bfloat16 *>(out_);
  const __nv_bfloat16 *in = reinterpret_cast<const __nv_bfloat16 *>(in_);
  const __nv_bfloat16 *w = reinterpret_cast<const __nv_bfloat16 *>(w_);
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!out || !in || !w) return BSP_ERR_NULL;
  if (cin <= 0 || cin % 16 || cout <= 0 || cout % 16) return BSP_ERR_SHAPE;
  if (((uintptr_t)in & 15u) || ((uintptr_t)w & 15u) || ((uintptr_t)out & 3u)) return BSP_ERR_ALIGN;
  const int64_t nvox = (int64_t)nx * ny * nz;
  const int nt = cout % 64 == 0 ? 64 : (cout % 32 == 0 ? 32 : 16);
  dim3 grid((unsigned)((nvox + MT - 1) / MT), cout / nt);
  if (nt == 64)
    conv3_fwd_kernel<64><<<grid, CT, 0, s>>>(out, in, w, bias, nx, ny, nz, cin, cout, relu);
  else if (nt == 32)
    conv3_fwd_kernel<32><<<grid, CT, 0, s>>>(out, in, w, bias, nx, ny, nz, cin, cout, relu);
  else
    conv3_fwd_kernel<16><<<grid, CT, 0, s>>>(out, in, w, bias, nx, ny, nz, cin, cout, relu);
  return (int)cudaGetLastError();
}

extern "C" size_t bsp_unet_wgrad_workspace_bytes(int nx, int ny, int nz, int cin, int cout) {
  const int64_t nvox = (int64_t)nx * ny * nz;
  const int64_t nchunk = (nvox + WG_VCH - 1) / WG_VCH;
  return (size_t)nchunk * 27 * cin * cout * sizeof(float);
}

extern "C" int bsp_unet_conv3_wgrad(float *dw, float *db, const bsp_bf16_t *g_,
                                    const bsp_bf16_t *in_, int nx, int ny, int nz, int cin,
                                    int cout, float *workspace, size_t workspace_bytes,
                                    cudaStream_t s) {
  const __nv_bfloat16 *g = reinterpret_cast<const __nv_bfloat16 *>(g_);
  const __nv_bfloat16 *in = reinterpret_cast<const __nv_bfloat16 *>(in_);
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!dw || !g || !in || !workspace) return BSP_ERR_NULL;
  if (cin <= 0 || cin % 16 || cout <= 0 || cout % 16) return BSP_ERR_SHAPE;
  if (workspace_bytes < bsp_unet_wgrad_workspace_bytes(nx, ny, nz, cin, cout))
    return BSP_ERR_WORKSPACE;
  if (((uintptr_t)in & 15u) || ((uintptr_t)g & 15u)) return BSP_ERR_ALIGN;
  const int64_t nvox = (int64_t)nx * ny * nz;
  const int nchunk = (int)((nvox + WG_VCH - 1) / WG_VCH);
  dim3 grid(nchunk, ((cout + 63) / 64) * ((cin + 63) / 64), 27);
  conv3_wgrad_kernel<<<grid, CT, 0, s>>>(workspace, g, in, nx, ny, nz, cin, cout);
  const int64_t n = 27LL * cin * cout;
  sum_chunks_kernel<<<grid_for(n), 256, 0, s>>>(dw, workspace, nchunk, n, 1.0f, 0);
  if (db) bias_grad_kernel<<<cout, 256, 0, s>>>(db, g, nvox, cout);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_flip_weights(bsp_bf16_t *wt_, const bsp_bf16_t *w_, int cin,
                                     int cout, cudaStream_t s) {
  __nv_bfloat16 *wt = reinterpret_cast<__nv_bfloat16 *>(wt_);
  const __nv_bfloat16 *w = reinterpret_cast<const __nv_bfloat16 *>(w_);
  if (!wt || !w) return BSP_ERR_NULL;
  flip_weights_kernel<<<grid_for(27LL * cin * cout), 256, 0, s>>>(wt, w, cin, cout);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_relu_bwd(bsp_bf16_t *g_, const bsp_bf16_t *act_, int64_t n,
                                 cudaStream_t s) {
  __nv_bfloat16 *g = reinterpret_cast<__nv_bfloat16 *>(g_);
  const __nv_bfloat16 *act = reinterpret_cast<const __nv_bfloat16 *>(act_);
  if (n <= 0) return BSP_OK;
  relu_bwd_kernel<<<grid_for(n), 256, 0, s>>>(g, act, n);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_pool(bsp_bf16_t *out_, const bsp_bf16_t *in_, int nx, int ny,
                             int nz, int c, int backward, int accumulate, cudaStream_t s) {
  __nv_bfloat16 *out = reinterpret_cast<__nv_bfloat16 *>(out_);
  const __nv_bfloat16 *in = reinterpret_cast<const __nv_bfloat16 *>(in_);
  if (nx % 2 || ny % 2 || nz % 2) return BSP_ERR_SHAPE;
  if (backward)
    pool_bwd_kernel<<<grid_for((int64_t)nx * ny * nz * c), 256, 0, s>>>(out, in, nx, ny, nz, c,
                                                                         accumulate);
  else
    pool_fwd_kernel<<<grid_for((int64_t)nx * ny * nz * c / 8), 256, 0, s>>>(out, in, nx, ny, nz,
                                                                             c);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_up(bsp_bf16_t *out_, const bsp_bf16_t *in_, int nx, int ny, int nz,
                           int c, int backward, cudaStream_t s) {
  __nv_bfloat16 *out = reinterpret_cast<__nv_bfloat16 *>(out_);
  const __nv_bfloat16 *in = reinterpret_cast<const __nv_bfloat16 *>(in_);
  if (nx % 2 || ny % 2 || nz % 2) return BSP_ERR_SHAPE;
  if (backward)
    up_bwd_kernel<<<grid_for((int64_t)nx * ny * nz * c / 8), 256, 0, s>>>(out, in, nx, ny, nz, c);
  else
    up_fwd_kernel<<<grid_for((int64_t)nx * ny * nz * c), 256, 0, s>>>(out, in, nx, ny, nz, c);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_add(bsp_bf16_t *a_, const bsp_bf16_t *b_, int64_t n, cudaStream_t s) {
  __nv_bfloat16 *a = reinterpret_cast<__nv_bfloat16 *>(a_);
  const __nv_bfloat16 *b = reinterpret_cast<const __nv_bfloat16 *>(b_);
  if (n <= 0) return BSP_OK;
  add_kernel<<<grid_for(n), 256, 0, s>>>(a, b, n);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_pack_input(bsp_bf16_t *x_, const float *div, const uint8_t *mask,
                                   int64_t nvox, float inv_scale, cudaStream_t s) {
  __nv_bfloat16 *x = reinterpret_cast<__nv_bfloat16 *>(x_);
  pack_input_kernel<<<grid_for(nvox), 256, 0, s>>>(x, div, mask, nvox, inv_scale);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_head_fwd(float *p, const bsp_bf16_t *x_, const float *hw,
                                 const float *hb, const uint8_t *mask, int64_t nvox, float scale,
                                 cudaStream_t s) {
  const __nv_bfloat16 *x = reinterpret_cast<const __nv_bfloat16 *>(x_);
  head_fwd_kernel<<<grid_for(nvox), 256, 0, s>>>(p, x, hw, hb, mask, nvox, scale);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_head_loss(bsp_bf16_t *gx_, float *partials, int nblocks,
                                  const float *pred, const float *target, const bsp_bf16_t *x_,
                                  const float *hw, const uint8_t *mask, int64_t nvox,
                                  float inv_scale, float inv_nfl, cudaStream_t s) {
  __nv_bfloat16 *gx = reinterpret_cast<__nv_bfloat16 *>(gx_);
  const __nv_bfloat16 *x = reinterpret_cast<const __nv_bfloat16 *>(x_);
  if (nblocks <= 0 || nblocks > 4096) return BSP_ERR_ARG;
  head_loss_kernel<<<nblocks, 256, 0, s>>>(gx, partials, pred, target, x, hw, mask, nvox,
                                           inv_scale, inv_nfl);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_head_bwd(bsp_bf16_t *gx_, float *partials, int nblocks,
                                 const float *gy, const bsp_bf16_t *x_, const float *hw,
                                 const uint8_t *mask, int64_t nvox, cudaStream_t s) {
  __nv_bfloat16 *gx = reinterpret_cast<__nv_bfloat16 *>(gx_);
  const __nv_bfloat16 *x = reinterpret_cast<const __nv_bfloat16 *>(x_);
  if (nblocks <= 0 || nblocks > 4096) return BSP_ERR_ARG;
  head_bwd_kernel<<<nblocks, 256, 0, s>>>(gx, partials, gy, x, hw, mask, nvox);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_sum_partials(float *out, const float *partials, int nblocks, int nslots,
                                     cudaStream_t s) {
  // out[slot] = sum over blocks in block order; partials laid out [slot][block]
  if (nblocks <= 0 || nslots <= 0 || nslots > 1024) return BSP_ERR_ARG;
  sum_slots_kernel<<<1, nslots, 0, s>>>(out, partials, nblocks);
  return (int)cudaGetLastError();
}

extern "C" int bsp_unet_adam(float *w, bsp_bf16_t *wb_, float *m, float *v, const float *g,
                             int64_t n, float lr, float b1, float b2, float eps, int step,
                             cudaStream_t s) {
  __nv_bfloat16 *wb = reinterpret_cast<__nv_bfloat16 *>(wb_);
  if (n <= 0 || step <= 0) return BSP_ERR_ARG;
  const float c1 = 1.0f / (1.0f - powf(b1, (float)step));
  const float c2 = 1.0f / (1.0f - powf(b2, (float)step));
  adam_kernel<<<grid_for(n), 256, 0, s>>>(w, wb, m, v, g, n, lr, b1, b2, eps, c1, c2);
  return (int)cudaGetLastError();
}
