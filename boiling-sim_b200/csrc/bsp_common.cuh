// bsp_common.cuh -- shared device helpers for the B200 pressure-projection library.
//
// Grid layout (identical to the reference, crates/cuda-kernels/src/jacobi_pressure.cu:16-18):
// cell (i, j, k) of an (nx, ny, nz) field lives at (i*ny + j)*nz + k, k fastest.
// MAC faces: ux (nx+1, ny, nz), uy (nx, ny+1, nz), uz (nx, ny, nz+1).
//
// Cell classes.  The reference passes an int32 material id per cell plus the
// two ids it treats specially (mat_fluid, mat_air); every other id is a solid
// (python/boilingsim/fluid.py:222-240).  The product path stores one byte per
// cell instead: BSP_FLUID / BSP_AIR / BSP_SOLID.  Cells outside the grid are
// air (jacobi_pressure.cu:121-124).
#pragma once
#include <cstdint>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/bsproj.h"

#define BSP_FLUID 0
#define BSP_AIR 1
#define BSP_SOLID 2

namespace bsp {

// Programmatic dependent launch: a kernel launched with the programmatic-
// stream-serialization attribute may start while the kernel before it
// drains; it waits here, before touching anything that kernel wrote, until
// that kernel has completed and its writes are visible.  A no-op for kernels
// launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the dependent kernel launch once every CTA of this one has called it
// (or exited).
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// Host: launch `kernel` with the programmatic-stream-serialization attribute
// when `pdl` is set (BSP_TUNE_PDL), plainly otherwise.
template <class... Exp, class... Act>
inline cudaError_t launch_maybe_pdl(bool pdl, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                    void (*kernel)(Exp...), Act &&...args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<Act &&>(args)...);
}

__device__ __forceinline__ int64_t idx3(int i, int j, int k, int ny, int nz) {
  return ((int64_t)i * ny + j) * nz + k;
}

// uint8 mask byte: bit 7 = fluid, bit 6 = solid (air = neither, so a zero byte
// is air, like a cell outside the grid), bits 0-2 = number of solid face
// neighbours (the Jacobi preconditioner's 6 - n_solid, diag_inverse_apply.cu:62-78).
// Bit 7 and bit 6 let a warp turn four packed mask bytes into all-ones /
// all-zero select words with one prmt (sign replication) each.
#define BSP_MFLUID 0x80u
#define BSP_MSOLID 0x40u
__device__ __forceinline__ uint32_t mcls(uint32_t mbyte) {
  return (mbyte & BSP_MFLUID) ? BSP_FLUID : ((mbyte & BSP_MSOLID) ? BSP_SOLID : BSP_AIR);
}
__device__ __forceinline__ uint32_t mnsolid(uint32_t mbyte) { return mbyte & 7u; }
__device__ __forceinline__ uint32_t enc_cls(uint32_t cls) {
  return cls == BSP_FLUID ? BSP_MFLUID : (cls == BSP_SOLID ? BSP_MSOLID : 0u);
}

__device__ __forceinline__ uint32_t classify(int m, int mat_fluid, int mat_air) {
  return m == mat_fluid ? BSP_FLUID : (m == mat_air ? BSP_AIR : BSP_SOLID);
}

// Neighbour value under the mixed boundary rule: fluid -> its pressure,
// air (free surface) -> 0 (Dirichlet), solid -> p_self (Neumann ghost).
__device__ __forceinline__ float nbr(uint32_t cls, float p_n, float p_self) {
  return cls == BSP_FLUID ? p_n : (cls == BSP_AIR ? 0.0f : p_self);
}

// Correctly rounded x / 6 in three instructions.  Method: the
// Markstein-style correction for a divisor known in advance (Brisebarre,
// Muller, Raina, "Accelerating correctly rounded floating-point division when
// the divisor is known in advance", IEEE Trans. Computers 53(8), 2004):
// q0 = RN(x z) with z = RN(1/6), r = x - 6 q0 (exact by fma), q = RN(q0 + r z).
// Verified bit-identical to IEEE x / 6 for every one of the 2^32 float
// inputs once results below 8 * FLT_MIN, signed zero, inf and NaN take the
// IEEE division (the exhaustive check is bsp_selftest_div6 and the CPU test).
__device__ __forceinline__ float div6(float x) {
  const float z = 0.16666667163372039795f;  // RN(1/6)
  const float q0 = __fmul_rn(x, z);
  const float r = __fmaf_rn(-q0, 6.0f, x);
  const float q = __fmaf_rn(r, z, q0);
  const float ax = fabsf(x);
  if (ax >= 0x1p-120f && ax <= 3.40282347e38f) return q;
  return ax == 0.0f ? x : __fdiv_rn(x, 6.0f);  // +-0 / 6 = +-0; tiny, inf, NaN: IEEE
}

// Branch-free neighbour select on bit patterns: for the mask byte q of word
// mw (bit 7 fluid, bit 6 solid) return p_n if fluid, p_self if solid, +0 if air.
// sw is mw << 1 (solid bit moved to bit 7).
// prmt.b32 in its default mode: a selector nibble with bit 3 set replicates the
// sign bit of the selected byte over the output byte (__byte_perm ignores
// that bit, so the instruction is issued directly).
__device__ __forceinline__ uint32_t sign_bytes(uint32_t w, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, 0, %2;" : "=r"(d) : "r"(w), "r"(sel));
  return d;
}
__device__ __forceinline__ float sel_nbr(uint32_t mw, uint32_t sw, int q, float pn, float ps) {
  const uint32_t sel = (uint32_t)(8 | q) * 0x1111u;  // replicate the sign bit of byte q
  const uint32_t fm = sign_bytes(mw, sel);
  const uint32_t sm = sign_bytes(sw, sel);
  return __uint_as_float((__float_as_uint(pn) & fm) | (__float_as_uint(ps) & sm));
}
__device__ __forceinline__ uint32_t fluid_word(uint32_t mw, int q) {
  return sign_bytes(mw, (uint32_t)(8 | q) * 0x1111u);
}

// One Jacobi update of a fluid cell with the reference's exact operation
// order (fluid.py:273-276): s = l + r + d + u + b + f left to right,
// rhs = rho*dx*dx*div/dt, p = (s - rhs)/6.  rdd = (rho*dx)*dx.
__device__ __forceinline__ float jacobi_update(float l, float r, float d, float u, float b,
                                               float f, float div, float rdd, float dt) {
  float s = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(l, r), d), u), b), f);
  float rhs = __fdiv_rn(__fmul_rn(rdd, div), dt);
  return div6(__fsub_rn(s, rhs));
}

// A p for a fluid cell, laplacian_spmv.cu:140: 6 p_self - s, contracted to one
// fma as the reference's default nvcc build does.
__device__ __forceinline__ float spmv_update(float l, float r, float d, float u, float b,
                                             float f, float ps) {
  float s = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(l, r), d), u), b), f);
  return __fmaf_rn(6.0f, ps, -s);
}

__device__ __forceinline__ uint32_t byte_of(uint32_t w, int q) { return (w >> (8 * q)) & 0xffu; }

// Opt kernel `fn` into `bytes` of dynamic shared memory on the current
// device.  The attribute belongs to the device, so the answer is cached per
// (kernel, device): a second GPU in the same process gets its own opt-in.
// Callers pass one fixed size per kernel (the largest they launch it with).
// False when the device refuses (the caller then takes another path).
inline bool smem_opt_in(const void *fn, int bytes) {
  struct Entry {
    const void *fn;
    int dev;
    bool ok;
  };
  static std::mutex mu;
  static std::vector<Entry> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lk(mu);
  for (const Entry &e : done)
    if (e.fn == fn && e.dev == dev) return e.ok;
  const bool ok = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) ==
                  cudaSuccess;
  done.push_back(Entry{fn, dev, ok});
  return ok;
}

}  // namespace bsp
