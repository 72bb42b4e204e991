// Dense layers of the warm-start surrogate on the tensor cores (no reference counterpart).
//
// Every dense block of the network is a two-layer perceptron y = W2 silu(W1 x + b1) + b2 (+ r),
// hidden width 64, whose input row x is up to three row segments side by side, each read from
// its own array, directly or through a row index (the per-edge gathers of the message-passing
// layers are fused into the operand staging).  Operands are rounded to BF16 when they are staged
// into shared memory; the products accumulate in FP32 (mma.sync m16n8k16, BF16 inputs, FP32
// accumulators); bias, SiLU, residual and the SiLU derivative are FP32 epilogues.
//
//   k_mlp_fwd    y and the hidden pre-activation z1 (kept for the backward pass), one 64-row tile
//                per loop trip, weights staged once per block.
//   k_mlp_bwd    dz1 = (dy W2) * silu'(z1) and dx = dz1 W1 for a tile of rows (k_mlp_bwd_tc: the
//                same on tcgen05).
//   k_wgrad      dW = dz^T x and db = sum of dz over the rows: each block accumulates its tiles in
//                registers and writes one partial; k_wgrad_reduce sums the partials in block
//                order, so the gradients are the same on every run.
//
// The CPU FP64 restatement these kernels are checked against is oracle/mpnn_ref.py.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "cfd_b200.h"

namespace cfdb {
void set_last_error(const std::string &msg);
}

namespace {

constexpr int TM = 64;    // rows per tile
constexpr int HID = 64;   // hidden width
constexpr int KMAX = 192; // widest input row
constexpr int LDH = HID + 8;
constexpr int LDT = TM + 8;

struct SegDev {
  const float *src;
  const int *idx;
  int width, ld, silu;
};

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ uint16_t bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ uint32_t ld2(const uint16_t *p) { return *reinterpret_cast<const uint32_t *>(p); }

// D += A B with A 16x16 (row-major fragment), B 16x8 (column-major fragment), BF16 in, FP32 acc.
__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A fragment of rows [r, r+16), columns [k, k+16) of a row-major BF16 tile with leading dimension ld.
__device__ __forceinline__ void frag_a(const uint16_t *s, int ld, int r, int k, int g, int t, uint32_t a[4]) {
  a[0] = ld2(s + (r + g) * ld + k + 2 * t);
  a[1] = ld2(s + (r + g + 8) * ld + k + 2 * t);
  a[2] = ld2(s + (r + g) * ld + k + 2 * t + 8);
  a[3] = ld2(s + (r + g + 8) * ld + k + 2 * t + 8);
}
// B fragment of columns [n, n+8), rows [k, k+16) of B, stored as B^T row-major ([n][k], ld).
__device__ __forceinline__ void frag_b(const uint16_t *s, int ld, int n, int k, int g, int t, uint32_t b[2]) {
  b[0] = ld2(s + (n + g) * ld + k + 2 * t);
  b[1] = ld2(s + (n + g) * ld + k + 2 * t + 8);
}

// Value of column k of input row `row` (the segments side by side).
__device__ __forceinline__ float seg_value(const SegDev *seg, int nseg, int row, int k) {
  int off = 0;
  for (int s = 0; s < nseg; s++) {
    const int w = seg[s].width;
    if (k < off + w) {
      const int r = seg[s].idx ? seg[s].idx[row] : row;
      const float v = seg[s].src[(size_t)r * seg[s].ld + (k - off)];
      return seg[s].silu ? silu_f(v) : v;
    }
    off += w;
  }
  return 0.0f;
}

struct FwdArgs {
  int M, K, N2, nseg;
  SegDev seg[3];
  const float *w1, *b1, *w2, *b2, *resid;
  int ld_resid;
  float *z1, *y;
  int ld_y;
};

__global__ void __launch_bounds__(128) k_mlp_fwd(FwdArgs a) {
  extern __shared__ __align__(16) uint16_t sm[];
  const int Kp = (a.K + 15) & ~15, LDX = Kp + 8, N2p = (a.N2 + 7) & ~7;
  uint16_t *sW1 = sm;                // [HID][LDX]      W1 (B operand of GEMM 1, [n][k])
  uint16_t *sW2 = sW1 + HID * LDX;   // [N2p][LDH]      W2 (B operand of GEMM 2)
  uint16_t *sX = sW2 + N2p * LDH;    // [TM][LDX]       input rows
  uint16_t *sS = sX + TM * LDX;      // [TM][LDH]       silu(z1)
  for (int e = threadIdx.x; e < HID * Kp; e += blockDim.x) {
    const int n = e / Kp, k = e - n * Kp;
    sW1[n * LDX + k] = k < a.K ? bf(a.w1[n * a.K + k]) : 0;
  }
  for (int e = threadIdx.x; e < N2p * HID; e += blockDim.x) {
    const int n = e / HID, k = e - n * HID;
    sW2[n * LDH + k] = n < a.N2 ? bf(a.w2[n * HID + k]) : 0;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, wr = warp * 16;
  const int ntiles = (a.M + TM - 1) / TM;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * TM;
    __syncthreads();
    for (int e = threadIdx.x; e < TM * Kp; e += blockDim.x) {
      const int r = e / Kp, k = e - r * Kp, row = r0 + r;
      sX[r * LDX + k] = (row < a.M && k < a.K) ? bf(seg_value(a.seg, a.nseg, row, k)) : 0;
    }
    __syncthreads();
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
    for (int k0 = 0; k0 < Kp; k0 += 16) {
      uint32_t af[4];
      frag_a(sX, LDX, wr, k0, g, t, af);
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        uint32_t bfr[2];
        frag_b(sW1, LDX, nt * 8, k0, g, t, bfr);
        mma16816(acc[nt], af, bfr);
      }
    }
    const int ra = r0 + wr + g, rb = ra + 8;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const int col = nt * 8 + 2 * t;
      const float b0 = a.b1[col], b1v = a.b1[col + 1];
      const float z00 = acc[nt][0] + b0, z01 = acc[nt][1] + b1v, z10 = acc[nt][2] + b0, z11 = acc[nt][3] + b1v;
      if (a.z1) {
        if (ra < a.M) *reinterpret_cast<float2 *>(a.z1 + (size_t)ra * HID + col) = make_float2(z00, z01);
        if (rb < a.M) *reinterpret_cast<float2 *>(a.z1 + (size_t)rb * HID + col) = make_float2(z10, z11);
      }
      sS[(wr + g) * LDH + col] = bf(silu_f(z00));
      sS[(wr + g) * LDH + col + 1] = bf(silu_f(z01));
      sS[(wr + g + 8) * LDH + col] = bf(silu_f(z10));
      sS[(wr + g + 8) * LDH + col + 1] = bf(silu_f(z11));
    }
    __syncwarp();
    float acc2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) acc2[nt][0] = acc2[nt][1] = acc2[nt][2] = acc2[nt][3] = 0.0f;
#pragma unroll
    for (int k0 = 0; k0 < HID; k0 += 16) {
      uint32_t af[4];
      frag_a(sS, LDH, wr, k0, g, t, af);
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        if (nt * 8 < N2p) {
          uint32_t bfr[2];
          frag_b(sW2, LDH, nt * 8, k0, g, t, bfr);
          mma16816(acc2[nt], af, bfr);
        }
      }
    }
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const int col = nt * 8 + 2 * t;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int row = h ? rb : ra;
        if (row >= a.M) continue;
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = col + q;
          if (c >= a.N2) continue;
          float v = acc2[nt][2 * h + q] + a.b2[c];
          if (a.resid) v += a.resid[(size_t)row * a.ld_resid + c];
          a.y[(size_t)row * a.ld_y + c] = v;
        }
      }
    }
  }
}

// ---- The forward block on the 5th-generation tensor cores (tcgen05) ----
// One CTA of 128 threads per 128-row tile (persistent over tiles): the input rows and the
// weights are staged in shared memory as BF16 in the K-major, no-swizzle canonical layout of the
// tcgen05 matrix descriptors (8-row x 16-byte core matrices, consecutive rows 16 bytes apart,
// row groups SBO = 128 bytes apart, 8-column chunks LBO = rows x 16 bytes apart); one elected
// thread issues the M = 128 MMAs (kind::f16, BF16 operands, FP32 accumulators in tensor memory)
// and commits them to an mbarrier; each warp reads its 32 rows of the accumulator with
// tcgen05.ld, applies bias and SiLU in FP32, writes the hidden layer back to shared memory as the
// A operand of the second MMA, and so on.  The results equal the mma.sync kernel's up to the FP32
// summation order.  Every mbarrier wait is bounded; a wait that runs out records an error in
// g_tc_status (read by cfd_mpnn_status), and the CTA releases its tensor memory and returns.
constexpr int TM_TC = 128;
constexpr long long kTcSpin = 1ll << 22;
__device__ int g_tc_status = 0;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// Byte offset of element (row, k) of a rows x K tile in the canonical K-major layout.
__device__ __forceinline__ uint32_t canon_off(int row, int k, int rows) {
  return (uint32_t)((((k >> 3) * (rows >> 3) + (row >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}
// Shared-memory matrix descriptor: start address, LBO and SBO in 16-byte units, version 1,
// no swizzle.
__device__ __forceinline__ uint64_t make_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t make_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kTcSpin; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(64);
  }
  return false;
}
// 16 consecutive FP32 accumulator columns of this thread's row.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__global__ void __launch_bounds__(128) k_mlp_fwd_tc(FwdArgs a) {
  extern __shared__ __align__(1024) uint8_t smb[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  const int Kp = (a.K + 15) & ~15, N2p = a.N2 <= 16 ? 16 : 64;
  uint8_t *sX = smb;                                  // [128 x Kp]  input rows
  uint8_t *sW1 = sX + (size_t)TM_TC * Kp * 2;         // [64 x Kp]   W1
  uint8_t *sS = sW1 + (size_t)HID * Kp * 2;           // [128 x 64]  silu(z1)
  uint8_t *sW2 = sS + (size_t)TM_TC * HID * 2;        // [N2p x 64]  W2
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < HID * Kp; e += blockDim.x) {
    const int n = e / Kp, k = e - n * Kp;
    *reinterpret_cast<uint16_t *>(sW1 + canon_off(n, k, HID)) = k < a.K ? bf(a.w1[n * a.K + k]) : 0;
  }
  for (int e = tid; e < N2p * HID; e += blockDim.x) {
    const int n = e / HID, k = e - n * HID;
    *reinterpret_cast<uint16_t *>(sW2 + canon_off(n, k, N2p)) = n < a.N2 ? bf(a.w2[n * HID + k]) : 0;
  }
  const uint32_t bar_a = smem_u32(&bar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
    abort_sh = 0;
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  const uint32_t d1 = tmem, d2 = tmem + 64;
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
  const uint32_t idesc1 = make_idesc(TM_TC, HID), idesc2 = make_idesc(TM_TC, N2p);
  uint32_t parity = 0;
  const int ntiles = (a.M + TM_TC - 1) / TM_TC;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * TM_TC;
    for (int e = tid; e < TM_TC * Kp; e += blockDim.x) {
      const int r = e / Kp, k = e - r * Kp, row = r0 + r;
      *reinterpret_cast<uint16_t *>(sX + canon_off(r, k, TM_TC)) =
          (row < a.M && k < a.K) ? bf(seg_value(a.seg, a.nseg, row, k)) : 0;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t xa = smem_u32(sX), wa = smem_u32(sW1);
      for (int k0 = 0; k0 < Kp; k0 += 16) {
        const uint64_t da = make_sdesc(xa + (uint32_t)((k0 >> 3) * (TM_TC >> 3) * 128), TM_TC * 16, 128);
        const uint64_t db = make_sdesc(wa + (uint32_t)((k0 >> 3) * (HID >> 3) * 128), HID * 16, 128);
        tc_mma(d1, da, db, idesc1, k0 > 0 ? 1u : 0u);
      }
      tc_commit(bar_a);
    }
    if (!mbar_wait(bar_a, parity)) {
      if (tid == 0) atomicExch(&g_tc_status, 5 /* CFD_ERR_TIMEOUT */);
      abort_sh = 1;
    }
    parity ^= 1u;
    __syncthreads();
    if (abort_sh) break;
    tc_fence_after();
    const int r = 32 * warp + (tid & 31), row = r0 + r;
#pragma unroll
    for (int c0 = 0; c0 < HID; c0 += 16) {
      float v[16];
      tmem_ld16(d1 + lane_base + c0, v);
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const float z = v[j] + a.b1[c0 + j];
        if (a.z1 && row < a.M) a.z1[(size_t)row * HID + c0 + j] = z;
        *reinterpret_cast<uint16_t *>(sS + canon_off(r, c0 + j, TM_TC)) = bf(silu_f(z));
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t sa = smem_u32(sS), wa = smem_u32(sW2);
      for (int k0 = 0; k0 < HID; k0 += 16) {
        const uint64_t da = make_sdesc(sa + (uint32_t)((k0 >> 3) * (TM_TC >> 3) * 128), TM_TC * 16, 128);
        const uint64_t db = make_sdesc(wa + (uint32_t)((k0 >> 3) * (N2p >> 3) * 128), N2p * 16, 128);
        tc_mma(d2, da, db, idesc2, k0 > 0 ? 1u : 0u);
      }
      tc_commit(bar_a);
    }
    if (!mbar_wait(bar_a, parity)) {
      if (tid == 0) atomicExch(&g_tc_status, 5);
      abort_sh = 1;
    }
    parity ^= 1u;
    __syncthreads();
    if (abort_sh) break;
    tc_fence_after();
    for (int c0 = 0; c0 < N2p; c0 += 16) {
      float v[16];
      tmem_ld16(d2 + lane_base + c0, v);
      if (row < a.M) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int c = c0 + j;
          if (c >= a.N2) continue;
          float y = v[j] + a.b2[c];
          if (a.resid) y += a.resid[(size_t)row * a.ld_resid + c];
          a.y[(size_t)row * a.ld_y + c] = y;
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  // After a timed-out wait the MMAs may still be in flight: wait for them (bounded) before the
  // tensor memory is released.
  if (abort_sh) mbar_wait(bar_a, parity);
  tc_fence_after();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
}

struct BwdArgs {
  int M, K, N2;
  const float *dy;
  int ld_dy;
  const float *z1, *w1, *w2;
  float *dz1, *dx;
  int ld_dx;
};

__global__ void __launch_bounds__(128) k_mlp_bwd(BwdArgs a) {
  extern __shared__ __align__(16) uint16_t sm[];
  const int Kp = (a.K + 15) & ~15, N2p = (a.N2 + 15) & ~15, LDN = N2p + 8;
  uint16_t *sW2T = sm;                 // [HID][LDN]   W2^T: B operand of dS = dY W2
  uint16_t *sW1T = sW2T + HID * LDN;   // [Kp][LDH]    W1^T: B operand of dX = dZ1 W1
  uint16_t *sDY = sW1T + Kp * LDH;     // [TM][LDN]
  uint16_t *sDZ = sDY + TM * LDN;      // [TM][LDH]
  for (int e = threadIdx.x; e < HID * N2p; e += blockDim.x) {
    const int j = e / N2p, o = e - j * N2p;
    sW2T[j * LDN + o] = o < a.N2 ? bf(a.w2[o * HID + j]) : 0;
  }
  for (int e = threadIdx.x; e < Kp * HID; e += blockDim.x) {
    const int c = e / HID, j = e - c * HID;
    sW1T[c * LDH + j] = c < a.K ? bf(a.w1[j * a.K + c]) : 0;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, wr = warp * 16;
  const int ntiles = (a.M + TM - 1) / TM;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * TM;
    __syncthreads();
    for (int e = threadIdx.x; e < TM * N2p; e += blockDim.x) {
      const int r = e / N2p, o = e - r * N2p, row = r0 + r;
      sDY[r * LDN + o] = (row < a.M && o < a.N2) ? bf(a.dy[(size_t)row * a.ld_dy + o]) : 0;
    }
    __syncthreads();
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
    for (int k0 = 0; k0 < N2p; k0 += 16) {
      uint32_t af[4];
      frag_a(sDY, LDN, wr, k0, g, t, af);
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        uint32_t bfr[2];
        frag_b(sW2T, LDN, nt * 8, k0, g, t, bfr);
        mma16816(acc[nt], af, bfr);
      }
    }
    const int ra = r0 + wr + g, rb = ra + 8;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const int col = nt * 8 + 2 * t;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int row = h ? rb : ra;
        float d0 = 0.0f, d1 = 0.0f;
        if (row < a.M) {
          const float2 z = *reinterpret_cast<const float2 *>(a.z1 + (size_t)row * HID + col);
          d0 = acc[nt][2 * h] * dsilu_f(z.x);
          d1 = acc[nt][2 * h + 1] * dsilu_f(z.y);
          *reinterpret_cast<float2 *>(a.dz1 + (size_t)row * HID + col) = make_float2(d0, d1);
        }
        sDZ[(wr + g + 8 * h) * LDH + col] = bf(d0);
        sDZ[(wr + g + 8 * h) * LDH + col + 1] = bf(d1);
      }
    }
    __syncwarp();
    if (!a.dx) continue;
    for (int c0 = 0; c0 < Kp; c0 += 64) {
      float ax[8][4];
#pragma unroll
      for (int nt = 0; nt < 8; nt++) ax[nt][0] = ax[nt][1] = ax[nt][2] = ax[nt][3] = 0.0f;
#pragma unroll
      for (int k0 = 0; k0 < HID; k0 += 16) {
        uint32_t af[4];
        frag_a(sDZ, LDH, wr, k0, g, t, af);
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
          if (c0 + nt * 8 < Kp) {
            uint32_t bfr[2];
            frag_b(sW1T, LDH, c0 + nt * 8, k0, g, t, bfr);
            mma16816(ax[nt], af, bfr);
          }
        }
      }
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        const int col = c0 + nt * 8 + 2 * t;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int row = h ? rb : ra;
          if (row >= a.M) continue;
          if (col < a.K) a.dx[(size_t)row * a.ld_dx + col] = ax[nt][2 * h];
          if (col + 1 < a.K) a.dx[(size_t)row * a.ld_dx + col + 1] = ax[nt][2 * h + 1];
        }
      }
    }
  }
}

// The backward data path on the tensor cores: dS = dY W2 (M = 128 rows, N = 64, K = the block's
// output width rounded up to 16), dz1 = dS * silu'(z1), dX = dz1 W1 (N = the input width rounded up
// to 16, K = 64), the same two-MMA chain as the forward with the transposed weights as the B
// operands: W2^T as (n = 64, k = out) and W1^T as (n = in, k = 64), all BF16 in the canonical
// K-major layout, FP32 accumulators in 64 + in columns of tensor memory.  BF16 rounding of dY, the
// weights and dz1 as in k_mlp_bwd, so the results agree up to the FP32 summation order.
__global__ void __launch_bounds__(128) k_mlp_bwd_tc(BwdArgs a) {
  extern __shared__ __align__(1024) uint8_t smb[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  const int Kp = (a.K + 15) & ~15, N2p = (a.N2 + 15) & ~15;
  uint8_t *sDY = smb;                                 // [128 x N2p]  dY rows
  uint8_t *sW2T = sDY + (size_t)TM_TC * N2p * 2;      // [64 x N2p]   W2^T
  uint8_t *sDZ = sW2T + (size_t)HID * N2p * 2;        // [128 x 64]   dz1
  uint8_t *sW1T = sDZ + (size_t)TM_TC * HID * 2;      // [Kp x 64]    W1^T
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < HID * N2p; e += blockDim.x) {
    const int n = e / N2p, k = e - n * N2p;  // B(n, k) = W2[k][n]
    *reinterpret_cast<uint16_t *>(sW2T + canon_off(n, k, HID)) = k < a.N2 ? bf(a.w2[k * HID + n]) : 0;
  }
  for (int e = tid; e < Kp * HID; e += blockDim.x) {
    const int n = e / HID, k = e - n * HID;  // B(n, k) = W1[k][n]
    *reinterpret_cast<uint16_t *>(sW1T + canon_off(n, k, Kp)) = n < a.K ? bf(a.w1[k * a.K + n]) : 0;
  }
  const uint32_t bar_a = smem_u32(&bar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(256));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
    abort_sh = 0;
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  const uint32_t d1 = tmem, d2 = tmem + 64;
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
  const uint32_t idesc1 = make_idesc(TM_TC, HID), idesc2 = make_idesc(TM_TC, Kp);
  uint32_t parity = 0;
  const int ntiles = (a.M + TM_TC - 1) / TM_TC;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * TM_TC;
    for (int e = tid; e < TM_TC * N2p; e += blockDim.x) {
      const int r = e / N2p, k = e - r * N2p, row = r0 + r;
      *reinterpret_cast<uint16_t *>(sDY + canon_off(r, k, TM_TC)) =
          (row < a.M && k < a.N2) ? bf(a.dy[(size_t)row * a.ld_dy + k]) : 0;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t ya = smem_u32(sDY), wa = smem_u32(sW2T);
      for (int k0 = 0; k0 < N2p; k0 += 16) {
        const uint64_t da = make_sdesc(ya + (uint32_t)((k0 >> 3) * (TM_TC >> 3) * 128), TM_TC * 16, 128);
        const uint64_t db = make_sdesc(wa + (uint32_t)((k0 >> 3) * (HID >> 3) * 128), HID * 16, 128);
        tc_mma(d1, da, db, idesc1, k0 > 0 ? 1u : 0u);
      }
      tc_commit(bar_a);
    }
    if (!mbar_wait(bar_a, parity)) {
      if (tid == 0) atomicExch(&g_tc_status, 5 /* CFD_ERR_TIMEOUT */);
      abort_sh = 1;
    }
    parity ^= 1u;
    __syncthreads();
    if (abort_sh) break;
    tc_fence_after();
    const int r = 32 * warp + (tid & 31), row = r0 + r;
#pragma unroll
    for (int c0 = 0; c0 < HID; c0 += 16) {
      float v[16];
      tmem_ld16(d1 + lane_base + c0, v);
#pragma unroll
      for (int j = 0; j < 16; j++) {
        float d = 0.0f;
        if (row < a.M) {
          d = v[j] * dsilu_f(a.z1[(size_t)row * HID + c0 + j]);
          a.dz1[(size_t)row * HID + c0 + j] = d;
        }
        *reinterpret_cast<uint16_t *>(sDZ + canon_off(r, c0 + j, TM_TC)) = bf(d);
      }
    }
    if (a.dx) {
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t za = smem_u32(sDZ), wa = smem_u32(sW1T);
        for (int k0 = 0; k0 < HID; k0 += 16) {
          const uint64_t da = make_sdesc(za + (uint32_t)((k0 >> 3) * (TM_TC >> 3) * 128), TM_TC * 16, 128);
          const uint64_t db = make_sdesc(wa + (uint32_t)((k0 >> 3) * (Kp >> 3) * 128), Kp * 16, 128);
          tc_mma(d2, da, db, idesc2, k0 > 0 ? 1u : 0u);
        }
        tc_commit(bar_a);
      }
      if (!mbar_wait(bar_a, parity)) {
        if (tid == 0) atomicExch(&g_tc_status, 5);
        abort_sh = 1;
      }
      parity ^= 1u;
      __syncthreads();
      if (abort_sh) break;
      tc_fence_after();
      for (int c0 = 0; c0 < Kp; c0 += 16) {
        float v[16];
        tmem_ld16(d2 + lane_base + c0, v);
        if (row < a.M) {
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const int c = c0 + j;
            if (c < a.K) a.dx[(size_t)row * a.ld_dx + c] = v[j];
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  // After a timed-out wait the MMAs may still be in flight: wait for them (bounded) before the
  // tensor memory is released.
  if (abort_sh) mbar_wait(bar_a, parity);
  tc_fence_after();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
}

struct WgArgs {
  int M, N, K, nseg;
  SegDev seg[3];
  const float *dz;
  int ld_dz;
  float *partial;  // [gridDim.x][N*K + N]
};

// dW[n][c] = sum over rows of dz[row][n] x[row][c] as D = A B with A = dz^T (N x TM) and
// B = x (TM x K).  MT = number of 16-row tiles of N (1 or 4); the four warps split the N tiles
// and the 8-column tiles of K between them.
template <int MT>
__global__ void __launch_bounds__(128) k_wgrad(WgArgs a) {
  extern __shared__ __align__(16) uint16_t sm[];
  constexpr int WPM = 4 / MT;            // warps per N tile
  constexpr int NTW = (KMAX / 8 + WPM - 1) / WPM;  // K tiles per warp, at most
  const int Kp = (a.K + 15) & ~15, Np = MT * 16;
  uint16_t *sDZT = sm;                 // [Np][LDT]   dz^T
  uint16_t *sXT = sDZT + Np * LDT;     // [Kp][LDT]   x^T
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int mrow = (warp % MT) * 16, ntile0 = warp / MT;
  const int nkt = Kp / 8;
  float acc[NTW][4];
#pragma unroll
  for (int i = 0; i < NTW; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0f;
  float bsum = 0.0f;
  const int ntiles = (a.M + TM - 1) / TM;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * TM;
    __syncthreads();
    for (int e = threadIdx.x; e < TM * Np; e += blockDim.x) {
      const int m = e / Np, n = e - m * Np, row = r0 + m;
      sDZT[n * LDT + m] = (row < a.M && n < a.N) ? bf(a.dz[(size_t)row * a.ld_dz + n]) : 0;
    }
    for (int e = threadIdx.x; e < TM * Kp; e += blockDim.x) {
      const int m = e / Kp, c = e - m * Kp, row = r0 + m;
      sXT[c * LDT + m] = (row < a.M && c < a.K) ? bf(seg_value(a.seg, a.nseg, row, c)) : 0;
    }
    if (threadIdx.x < a.N) {
      const int rend = min(TM, a.M - r0);
      for (int m = 0; m < rend; m++) bsum += a.dz[(size_t)(r0 + m) * a.ld_dz + threadIdx.x];
    }
    __syncthreads();
#pragma unroll
    for (int k0 = 0; k0 < TM; k0 += 16) {
      uint32_t af[4];
      frag_a(sDZT, LDT, mrow, k0, g, t, af);
#pragma unroll
      for (int i = 0; i < NTW; i++) {
        const int kt = ntile0 + i * WPM;
        if (kt < nkt) {
          uint32_t bfr[2];
          frag_b(sXT, LDT, kt * 8, k0, g, t, bfr);
          mma16816(acc[i], af, bfr);
        }
      }
    }
  }
  float *out = a.partial + (size_t)blockIdx.x * (a.N * a.K + a.N);
#pragma unroll
  for (int i = 0; i < NTW; i++) {
    const int kt = ntile0 + i * WPM;
    if (kt >= nkt) continue;
    const int c = kt * 8 + 2 * t;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int n = mrow + g + 8 * h;
      if (n >= a.N) continue;
      if (c < a.K) out[n * a.K + c] = acc[i][2 * h];
      if (c + 1 < a.K) out[n * a.K + c + 1] = acc[i][2 * h + 1];
    }
  }
  if (threadIdx.x < a.N) out[a.N * a.K + threadIdx.x] = bsum;
}

// dw[j] (j < N*K) and db[j] (j < N) from the per-block partials, summed in block order.
__global__ void k_wgrad_reduce(const float *__restrict__ partial, int nblk, int N, int K, float *__restrict__ dw,
                               float *__restrict__ db, int accumulate) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = N * K + N;
  if (j >= stride) return;
  float s = 0.0f;
  for (int b = 0; b < nblk; b++) s += partial[(size_t)b * stride + j];
  float *o = j < N * K ? dw + j : db + (j - N * K);
  *o = accumulate ? *o + s : s;
}

// out[r][j] = a[r][j] + b[r][j] (j < width; leading dimensions given).
__global__ void k_add(float *out, int ldo, const float *a, int lda, const float *b, int ldb, int rows, int width) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)rows * width) return;
  const int r = (int)(e / width), j = (int)(e - (size_t)r * width);
  out[(size_t)r * ldo + j] = a[(size_t)r * lda + j] + b[(size_t)r * ldb + j];
}

// out[r][j] += src[idx[r]][j].
__global__ void k_gather_add(float *out, int ldo, const float *src, int lds, const int *idx, int rows, int width) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)rows * width) return;
  const int r = (int)(e / width), j = (int)(e - (size_t)r * width);
  out[(size_t)r * ldo + j] += src[(size_t)idx[r] * lds + j];
}

// out[r][:] (+)= sum over j in [ptr[r], ptr[r+1]) of x[idx[j]][:], in list order (warp per row).
__global__ void k_segment_sum_acc(const float *__restrict__ x, int ldx, const int *__restrict__ ptr,
                                  const int *__restrict__ idx, int n_rows, int width, float *__restrict__ out, int ldo,
                                  int accumulate) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n_rows) return;
  const int b = ptr[row], e = ptr[row + 1];
  for (int col = lane; col < width; col += 32) {
    float acc = 0.f;
    for (int j = b; j < e; j++) acc += x[(size_t)idx[j] * ldx + col];
    float *o = out + (size_t)row * ldo + col;
    *o = accumulate ? *o + acc : acc;
  }
}

// Mean-squared error: grad = 2 (pred - target) / n and loss = sum (pred - target)^2 / n, one block,
// fixed-order tree.
__global__ void __launch_bounds__(1024) k_mse(const float *pred, const float *target, int n, float *grad, float *loss) {
  __shared__ float sh[1024];
  float s = 0.0f;
  const float inv = 1.0f / (float)n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float d = pred[i] - target[i];
    grad[i] = 2.0f * d * inv;
    s += d * d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = sh[0] * inv;
}

cfd_status status_of(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return CFD_OK;
  cfdb::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return CFD_ERR_CUDA;
}

cfd_status bad(const char *what) {
  cfdb::set_last_error(what);
  return CFD_ERR_BAD_ARG;
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

bool copy_segs(int nseg, const cfd_mlp_seg *in, SegDev *out, int &K) {
  if (nseg < 1 || nseg > 3) return false;
  K = 0;
  for (int s = 0; s < nseg; s++) {
    if (!in[s].src || in[s].width < 1 || in[s].ld < in[s].width) return false;
    out[s] = SegDev{in[s].src, in[s].idx, in[s].width, in[s].ld, in[s].silu};
    K += in[s].width;
  }
  for (int s = nseg; s < 3; s++) out[s] = SegDev{nullptr, nullptr, 0, 0, 0};
  return K <= KMAX;
}

size_t fwd_smem(int K, int N2) {
  const int Kp = (K + 15) & ~15, LDX = Kp + 8, N2p = (N2 + 7) & ~7;
  return sizeof(uint16_t) * ((size_t)HID * LDX + (size_t)N2p * LDH + (size_t)TM * LDX + (size_t)TM * LDH);
}
size_t tc_smem(int K, int N2) {
  const int Kp = (K + 15) & ~15, N2p = N2 <= 16 ? 16 : 64;
  return 2 * ((size_t)TM_TC * Kp + (size_t)HID * Kp + (size_t)TM_TC * HID + (size_t)N2p * HID);
}
size_t bwd_tc_smem(int K, int N2) {
  const int Kp = (K + 15) & ~15, N2p = (N2 + 15) & ~15;
  return 2 * ((size_t)TM_TC * N2p + (size_t)HID * N2p + (size_t)TM_TC * HID + (size_t)Kp * HID);
}
size_t bwd_smem(int K, int N2) {
  const int Kp = (K + 15) & ~15, N2p = (N2 + 15) & ~15, LDN = N2p + 8;
  return sizeof(uint16_t) * ((size_t)HID * LDN + (size_t)Kp * LDH + (size_t)TM * LDN + (size_t)TM * LDH);
}
size_t wg_smem(int K, int MT) {
  const int Kp = (K + 15) & ~15;
  return sizeof(uint16_t) * ((size_t)MT * 16 * LDT + (size_t)Kp * LDT);
}

template <typename F>
void set_smem(F f, size_t bytes) {
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

extern "C" {

int cfd_mpnn_wgrad_blocks(void) { return CFD_MPNN_WGRAD_BLOCKS; }

cfd_status cfd_mpnn_status(int *status, int reset) {
  if (!status) return bad("cfd_mpnn_status: null argument");
  cudaError_t e = cudaMemcpyFromSymbol(status, g_tc_status, sizeof(int));
  if (e == cudaSuccess && reset) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_tc_status, &zero, sizeof(int));
  }
  if (e != cudaSuccess) {
    cfdb::set_last_error(std::string("cfd_mpnn_status: ") + cudaGetErrorString(e));
    return CFD_ERR_CUDA;
  }
  return CFD_OK;
}

cfd_status cfd_mpnn_mlp_forward(const cfd_mlp_fwd *p, void *stream) {
  if (!p || p->rows < 0 || p->out < 1 || p->out > HID || !p->w1 || !p->b1 || !p->w2 || !p->b2 || !p->y ||
      p->ld_y < p->out || (p->resid && p->ld_resid < p->out))
    return bad("cfd_mpnn_mlp_forward: bad argument");
  FwdArgs a{};
  if (!copy_segs(p->nseg, p->seg, a.seg, a.K)) return bad("cfd_mpnn_mlp_forward: bad input segments (total width <= 192)");
  if (p->rows == 0) return CFD_OK;
  a.M = p->rows;
  a.N2 = p->out;
  a.nseg = p->nseg;
  a.w1 = p->w1;
  a.b1 = p->b1;
  a.w2 = p->w2;
  a.b2 = p->b2;
  a.resid = p->resid;
  a.ld_resid = p->ld_resid;
  a.z1 = p->z1;
  a.y = p->y;
  a.ld_y = p->ld_y;
  if (p->engine == 1) {
    // tcgen05 form: the tiles plus 48 KB, and at least 80 KB, of shared memory per CTA, so that at
    // most two CTAs (2 x 128 tensor-memory columns of the SM's 512) share an SM.
    const size_t need = tc_smem(a.K, a.N2) + 48 * 1024, sm = need > 80 * 1024 ? need : 80 * 1024;
    set_smem(k_mlp_fwd_tc, sm);
    const int ntiles = (a.M + TM_TC - 1) / TM_TC;
    const int grid = ntiles < 2 * sm_count() ? ntiles : 2 * sm_count();
    k_mlp_fwd_tc<<<grid, 128, sm, static_cast<cudaStream_t>(stream)>>>(a);
    return status_of("cfd_mpnn_mlp_forward (tcgen05)");
  }
  const size_t sm = fwd_smem(a.K, a.N2);
  set_smem(k_mlp_fwd, sm);
  const int ntiles = (a.M + TM - 1) / TM;
  const int grid = ntiles < 3 * sm_count() ? ntiles : 3 * sm_count();
  k_mlp_fwd<<<grid, 128, sm, static_cast<cudaStream_t>(stream)>>>(a);
  return status_of("cfd_mpnn_mlp_forward");
}

cfd_status cfd_mpnn_mlp_backward(const cfd_mlp_bwd *p, void *stream) {
  if (!p || p->rows < 0 || p->in_width < 1 || p->in_width > KMAX || p->out < 1 || p->out > HID || !p->dy ||
      p->ld_dy < p->out || !p->z1 || !p->w1 || !p->w2 || !p->dz1 || (p->dx && p->ld_dx < p->in_width))
    return bad("cfd_mpnn_mlp_backward: bad argument");
  if (p->rows == 0) return CFD_OK;
  BwdArgs a{p->rows, p->in_width, p->out, p->dy, p->ld_dy, p->z1, p->w1, p->w2, p->dz1, p->dx, p->ld_dx};
  if (p->engine == 1) {
    // tcgen05 form: one CTA per SM (at least 120 KB of shared memory each), each holding 256 of
    // the SM's 512 tensor-memory columns.
    const size_t need = bwd_tc_smem(a.K, a.N2) + 16 * 1024, sm = need > 120 * 1024 ? need : 120 * 1024;
    set_smem(k_mlp_bwd_tc, sm);
    const int ntiles = (a.M + TM_TC - 1) / TM_TC;
    const int grid = ntiles < sm_count() ? ntiles : sm_count();
    k_mlp_bwd_tc<<<grid, 128, sm, static_cast<cudaStream_t>(stream)>>>(a);
    return status_of("cfd_mpnn_mlp_backward (tcgen05)");
  }
  const size_t sm = bwd_smem(a.K, a.N2);
  set_smem(k_mlp_bwd, sm);
  const int ntiles = (a.M + TM - 1) / TM;
  const int grid = ntiles < 3 * sm_count() ? ntiles : 3 * sm_count();
  k_mlp_bwd<<<grid, 128, sm, static_cast<cudaStream_t>(stream)>>>(a);
  return status_of("cfd_mpnn_mlp_backward");
}

cfd_status cfd_mpnn_weight_grad(const cfd_mlp_wgrad *p, void *stream) {
  if (!p || p->rows < 0 || !(p->n == HID || (p->n >= 1 && p->n <= 16)) || !p->dz || p->ld_dz < p->n || !p->dw ||
      !p->db || !p->workspace)
    return bad("cfd_mpnn_weight_grad: bad argument (n must be 64 or at most 16)");
  WgArgs a{};
  int K = 0;
  if (!copy_segs(p->nseg, p->seg, a.seg, K)) return bad("cfd_mpnn_weight_grad: bad input segments (total width <= 192)");
  a.M = p->rows;
  a.N = p->n;
  a.K = K;
  a.nseg = p->nseg;
  a.dz = p->dz;
  a.ld_dz = p->ld_dz;
  a.partial = p->workspace;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int ntiles = (a.M + TM - 1) / TM;
  const int grid = ntiles < 1 ? 1 : (ntiles < CFD_MPNN_WGRAD_BLOCKS ? ntiles : CFD_MPNN_WGRAD_BLOCKS);
  if (a.N == HID) {
    const size_t sm = wg_smem(K, 4);
    set_smem(k_wgrad<4>, sm);
    k_wgrad<4><<<grid, 128, sm, s>>>(a);
  } else {
    const size_t sm = wg_smem(K, 1);
    set_smem(k_wgrad<1>, sm);
    k_wgrad<1><<<grid, 128, sm, s>>>(a);
  }
  cfd_status st = status_of("cfd_mpnn_weight_grad");
  if (st != CFD_OK) return st;
  const int total = a.N * a.K + a.N;
  k_wgrad_reduce<<<(total + 255) / 256, 256, 0, s>>>(a.partial, grid, a.N, a.K, p->dw, p->db, p->accumulate);
  return status_of("cfd_mpnn_weight_grad (reduce)");
}

cfd_status cfd_mpnn_add(float *out, int ldo, const float *a, int lda, const float *b, int ldb, int rows, int width,
                        void *stream) {
  if (rows < 0 || width < 1 || ldo < width || lda < width || ldb < width || (rows > 0 && (!out || !a || !b)))
    return bad("cfd_mpnn_add: bad argument");
  if (rows == 0) return CFD_OK;
  const size_t n = (size_t)rows * width;
  k_add<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, ldo, a, lda, b, ldb, rows,
                                                                                    width);
  return status_of("cfd_mpnn_add");
}

cfd_status cfd_mpnn_gather_add(float *out, int ldo, const float *src, int lds, const int *idx, int rows, int width,
                               void *stream) {
  if (rows < 0 || width < 1 || ldo < width || lds < width || (rows > 0 && (!out || !src || !idx)))
    return bad("cfd_mpnn_gather_add: bad argument");
  if (rows == 0) return CFD_OK;
  const size_t n = (size_t)rows * width;
  k_gather_add<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, ldo, src, lds, idx,
                                                                                           rows, width);
  return status_of("cfd_mpnn_gather_add");
}

cfd_status cfd_mpnn_segment_sum_acc(const float *x, int ldx, const int *ptr, const int *idx, int n_rows, int width,
                                    float *out, int ldo, int accumulate, void *stream) {
  if (n_rows < 0 || width < 1 || ldx < width || ldo < width || (n_rows > 0 && (!x || !ptr || !idx || !out)))
    return bad("cfd_mpnn_segment_sum_acc: bad argument");
  if (n_rows == 0) return CFD_OK;
  const int rows_per_block = 256 / 32;
  k_segment_sum_acc<<<(n_rows + rows_per_block - 1) / rows_per_block, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      x, ldx, ptr, idx, n_rows, width, out, ldo, accumulate);
  return status_of("cfd_mpnn_segment_sum_acc");
}

cfd_status cfd_mpnn_mse(const float *pred, const float *target, int n, float *grad, float *loss, void *stream) {
  if (n < 1 || !pred || !target || !grad || !loss) return bad("cfd_mpnn_mse: bad argument");
  k_mse<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(pred, target, n, grad, loss);
  return status_of("cfd_mpnn_mse");
}

}  // extern "C"
