// RBF Gram tiles on the 5th-generation tensor cores (tcgen05), for the
// Gram-input sweeps (gram.cuh).  Same output as gram_kernel's RBF mode: the
// static-kernel values exp(-|x_i - y_j|^2 / max(2 s^2, 1e-12))
// (ksig/static/kernels.py:248-260, ksig/utils.py:138-157) of every point
// pair of a task, written into the task's Gram slot.
//
// One CTA (4 warps) computes a tile of 128 rows (x points) by kTcN columns
// (y points) of one pair:
//   1. Centre: every point of the tile is moved to the tile's first column
//      point c, so that |x'|^2 + |y'|^2 - 2 <x', y'> is formed from small
//      vectors near the diagonal of the pair (no FP32 cancellation of large
//      norms; see rbf_center_cols in common.cuh for the same argument).
//   2. Split each centred coordinate into a TF32 head and a TF32-rounded
//      tail (v = hi + lo + O(2^-22 |v|)) and write hi / lo of the 128 x KC row block (A) and the
//      kTcN x KC column block (B) to shared memory in the canonical K-major
//      no-swizzle layout of the UMMA descriptors.
//   3. One elected thread issues tcgen05.mma.kind::tf32 for the three
//      products hi*hi + hi*lo + lo*hi (3xTF32: FP32-level accuracy) into one
//      FP32 accumulator in tensor memory, K = 8 per instruction, and commits
//      to an mbarrier.
//   4. After the last K chunk, each warp reads its 32 accumulator lanes with
//      tcgen05.ld (thread t of warp w holds row 32 w + t), forms
//      arg = -a (|x'|^2 + |y'|^2 - 2 <x', y'>) and writes exp2(arg).
// Waits on the mbarrier are bounded: past the limit the tile records
// KSIG_ERR_DEVICE in the status word, waits (bounded again) for its own
// MMAs, frees its tensor memory and returns.
#pragma once

#include "gram.cuh"

namespace ksig {

constexpr int kTcM = 128;  // x points per tile (accumulator lanes)
constexpr int kTcN = 32;   // y points per tile (accumulator columns), one centre
constexpr int kTcKC = 64;  // coordinates per shared-memory chunk (multiple of 8)

__host__ __device__ constexpr size_t gram_tc_smem_bytes() {
  return (size_t)(2 * kTcM + 2 * kTcN) * kTcKC * 4 + (kTcM + kTcN) * 4 + 64;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (tcgen05), K-major, no swizzle.  Element
// (r, k) of an R x KC operand block lives at byte (k / 4) * R * 16 + r * 16 +
// (k % 4) * 4: 8 x 16-byte core matrices with rows 16 B apart, 8-row groups
// 128 B apart (stride byte offset) and 16-byte K chunks R * 16 B apart
// (leading byte offset).  Fields in 16-byte units; version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B,
// both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ float to_tf32(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

// Bounded wait on phase `parity` of an mbarrier; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(32);
  }
  return false;
}

__global__ void __launch_bounds__(128) gram_tc_kernel(const GramArgs<float> a) {
  extern __shared__ __align__(128) unsigned char tsm[];
  float* a_hi = reinterpret_cast<float*>(tsm);
  float* a_lo = a_hi + kTcM * kTcKC;
  float* b_hi = a_lo + kTcM * kTcKC;
  float* b_lo = b_hi + kTcN * kTcKC;
  float* yn = b_lo + kTcN * kTcKC;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(yn + kTcN + kTcM);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);

  const int slot = blockIdx.y;
  const int pos = a.task_base + slot;
  const int2 ab = decode_task(pos, a.mode, a.nY, a.list, a.order);
  if (ab.x < 0 || ab.x >= a.nX || ab.y < 0 || ab.y >= a.nYseq) {
    if (threadIdx.x == 0 && blockIdx.x == 0) set_status(a.status, KSIG_ERR_INVALID);
    return;
  }
  const int Lx = a.xlen[ab.x], Ly = a.ylen[ab.y];
  const int ti = blockIdx.x / a.tiles_y, tj = blockIdx.x - ti * a.tiles_y;
  const int i0 = ti * kTcM, j0 = tj * kTcN;
  if (i0 >= Lx || j0 >= Ly) return;  // the tile lies past this pair's lengths
  const float* xb = a.xr + a.xstart[ab.x] * a.rs;
  const float* yb = a.yr + a.ystart[ab.y] * a.rs;
  const float* cpt = yb + (long long)j0 * a.rs;  // the tile's centre (column j0)
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;

  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(tmem_slot)), "r"(kTcN) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const float* xrow = xb + (long long)min(i0 + t, Lx - 1) * a.rs;
  const float* yrow = yb + (long long)min(j0 + (t & (kTcN - 1)), Ly - 1) * a.rs;
  float xnorm = 0.f, ynorm = 0.f;
  const uint32_t idesc = umma_idesc_tf32(kTcM, kTcN);
  const uint32_t bar = smem_u32(mbar);
  bool ok = true;
  int nchunks = 0;
  for (int k0 = 0; k0 < a.kd; k0 += kTcKC, ++nchunks) {
    // Centred, split operand blocks of this chunk (thread t: row t of A;
    // threads 0 .. kTcN - 1 also row t of B).
#pragma unroll 4
    for (int q = 0; q < kTcKC / 4; ++q) {
      const int k = k0 + 4 * q;
      float4 c = make_float4(0.f, 0.f, 0.f, 0.f), x = c, y = c;
      if (k < a.kd) {  // kd and k are multiples of 4
        c = *reinterpret_cast<const float4*>(cpt + k);
        x = *reinterpret_cast<const float4*>(xrow + k);
        if (t < kTcN) y = *reinterpret_cast<const float4*>(yrow + k);
      }
      float4 v = make_float4(x.x - c.x, x.y - c.y, x.z - c.z, x.w - c.w);
      xnorm = fmaf(v.x, v.x, fmaf(v.y, v.y, fmaf(v.z, v.z, fmaf(v.w, v.w, xnorm))));
      float4 h = make_float4(to_tf32(v.x), to_tf32(v.y), to_tf32(v.z), to_tf32(v.w));
      *reinterpret_cast<float4*>(a_hi + (q * kTcM + t) * 4) = h;
      *reinterpret_cast<float4*>(a_lo + (q * kTcM + t) * 4) =
          make_float4(to_tf32(v.x - h.x), to_tf32(v.y - h.y), to_tf32(v.z - h.z),
                      to_tf32(v.w - h.w));
      if (t < kTcN) {
        v = make_float4(y.x - c.x, y.y - c.y, y.z - c.z, y.w - c.w);
        ynorm = fmaf(v.x, v.x, fmaf(v.y, v.y, fmaf(v.z, v.z, fmaf(v.w, v.w, ynorm))));
        h = make_float4(to_tf32(v.x), to_tf32(v.y), to_tf32(v.z), to_tf32(v.w));
        *reinterpret_cast<float4*>(b_hi + (q * kTcN + t) * 4) = h;
        *reinterpret_cast<float4*>(b_lo + (q * kTcN + t) * 4) =
            make_float4(to_tf32(v.x - h.x), to_tf32(v.y - h.y), to_tf32(v.z - h.z),
                        to_tf32(v.w - h.w));
      }
    }
    // Generic-proxy shared-memory writes -> visible to the tensor core.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
      const uint32_t bh = smem_u32(b_hi), bl = smem_u32(b_lo);
#pragma unroll
      for (int s = 0; s < kTcKC / 8; ++s) {  // K = 8 TF32 = two 16-byte chunks
        const uint64_t dah = umma_desc(ah + s * 2 * kTcM * 16, kTcM * 16, 128);
        const uint64_t dal = umma_desc(al + s * 2 * kTcM * 16, kTcM * 16, 128);
        const uint64_t dbh = umma_desc(bh + s * 2 * kTcN * 16, kTcN * 16, 128);
        const uint64_t dbl = umma_desc(bl + s * 2 * kTcN * 16, kTcN * 16, 128);
        const uint32_t acc = (k0 > 0 || s > 0) ? 1u : 0u;
        // hi*hi (overwrites the accumulator on the first step), hi*lo, lo*hi.
        asm volatile(
            "{\n\t.reg .pred p, q;\n\t"
            "setp.ne.b32 p, %6, 0;\n\t"
            "setp.eq.b32 q, %6, %6;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %3, %5, p;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %4, %5, q;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %2, %3, %5, q;\n\t}"
            ::"r"(tmem), "l"(dah), "l"(dal), "l"(dbh), "l"(dbl), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(bar) : "memory");
    }
    // The chunk's MMAs have read the operands once this phase completes;
    // the give-up decision is taken by the whole CTA together.
    if (!__syncthreads_and(mbar_wait(bar, nchunks & 1, 1LL << 22))) {
      ok = false;
      break;
    }
  }
  if (ok) {
    if (t < kTcN) yn[t] = ynorm;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    uint32_t r[kTcN];
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const int i = i0 + warp * 32 + lane;
    if (i < Lx) {
      float* out = a.gram + (long long)slot * a.slot + (long long)i * a.ld;
      const float na = -a.ralpha;
#pragma unroll
      for (int c = 0; c < kTcN; ++c) {
        const int j = j0 + c;
        if (j < Ly) {
          const float dot = __uint_as_float(r[c]);
          out[j] = kexp2(na * ((xnorm + yn[c]) - 2.f * dot));
        }
      }
    }
  } else {
    if (t == 0) set_status(a.status, KSIG_ERR_DEVICE);
    // Let this tile's own MMAs drain (bounded) before the memory goes.
    mbar_wait(bar, nchunks & 1, 1LL << 22);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcN)
                 : "memory");
  }
}

}  // namespace ksig
