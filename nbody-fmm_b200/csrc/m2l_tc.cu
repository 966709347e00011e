// M2L on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// A batch of 128 target cells of one level and one child class shares the
// same interaction offsets, so for each offset slot present in the batch
//   D[128 x N] += A_slot[128 x K] * B_slot[K x N]
// where A_slot gathers each target's source multipole at that offset (zero
// row if absent) and B_slot is the offset's M2L operator (transposed).  D
// lives in tensor memory (TMEM) across all slots of the batch and is added
// into the local expansions at the end.
//
// Precision: every FP32 operand x is split into three BF16 parts
// x = x1 + x2 + x3 (8 significant bits each, 24 in all), and the product is
// the sum of the six split products with total order <= 2
// (x1y1 + x1y2 + x2y1 + x1y3 + x2y2 + x3y1); the dropped terms are below
// 2^-24 relative.  The tensor core's own FP32 accumulation truncates at the
// accumulator's magnitude, so each slot starts a fresh accumulator and
// issues its split products smallest first; the slot's result is then read
// out of TMEM and summed across slots in FP32 registers (round to nearest),
// which keeps the contraction at FP32 accuracy.  The BF16 parts of the
// operators are prepared once per pass (k_tc_images); those of the gathered
// multipoles by the CTA.
//
// Shared-memory operands use the K-major layout without swizzle: 8-row x
// 16-byte core matrices, rows of a core matrix contiguous, 8-row groups
// SBO = 128 B apart and 16-byte K chunks LBO apart.  One thread issues the
// MMAs and commits them to an mbarrier that all threads wait on with an
// iteration limit; on timeout the kernel flags the device error word,
// releases its TMEM and returns.
#include <cuda_bf16.h>

#include "m2l_tc.cuh"

namespace fmm {

static constexpr int TC_M = 128;

__device__ inline uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// SM100 shared-memory matrix descriptor: start >> 4 [0,14), LBO >> 4
// [16,30), SBO >> 4 [32,46), version 1 [46,48), no swizzle [61,64) = 0.
__device__ inline uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ inline void split3(float v, uint16_t &h, uint16_t &m, uint16_t &l) {
  const __nv_bfloat16 bh = __float2bfloat16_rn(v);
  const float r1 = v - __bfloat162float(bh);
  const __nv_bfloat16 bm = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(bm);
  const __nv_bfloat16 bl = __float2bfloat16_rn(r2);
  h = __bfloat16_as_ushort(bh);
  m = __bfloat16_as_ushort(bm);
  l = __bfloat16_as_ushort(bl);
}

// Operator images: for each M2L table slot and split, element (n, k) of
// B = T^T (n: output, k: input) at ((k/8) * (P16/8) + n/8) * 64 + (n%8) * 8 + k%8.
__global__ void k_tc_images(const float *tab, int K, int KP, int P16, uint16_t *img) {
  const int slot = blockIdx.x;
  const size_t bsplit = (size_t)P16 * P16;
  const float *T = tab + (size_t)slot * K * KP;
  uint16_t *out = img + (size_t)slot * 3 * bsplit;
  for (int e = threadIdx.x; e < P16 * P16; e += blockDim.x) {
    const int n = e / P16, k = e % P16;
    const float v = (n < K && k < K) ? T[(size_t)k * KP + n] : 0.f;
    uint16_t h, m, l;
    split3(v, h, m, l);
    const size_t idx = ((size_t)(k / 8) * (P16 / 8) + n / 8) * 64 + (n % 8) * 8 + (k % 8);
    out[idx] = h;
    out[bsplit + idx] = m;
    out[2 * bsplit + idx] = l;
  }
}

__device__ inline void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ inline void tmem_ld16(uint32_t addr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}

template <int P16>
__global__ void __launch_bounds__(128, 1) k_m2l_tc(TcArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ int s_tgt[TC_M];
  __shared__ __align__(8) uint64_t s_mbar;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int KC = P16 / 8;
  float acc[P16];
#pragma unroll
  for (int j = 0; j < P16; ++j) acc[j] = 0.f;
  const size_t asplit = (size_t)KC * (TC_M / 8) * 64;  // elements per A split
  const size_t bsplit = (size_t)KC * (P16 / 8) * 64;
  uint16_t *As = (uint16_t *)smem;
  uint16_t *Bs = As + 3 * asplit;
  const int nslots = a.nslots[blockIdx.x];
  if (nslots == 0) return;
  const int4 bt = a.batches[blockIdx.x];
  s_tgt[tid] = tid < bt.y ? a.tlist[bt.x + tid] : -1;
  const uint32_t ncols = P16 <= 128 ? 128u : 256u;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s_tmem;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(P16 >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
  const uint32_t lboA = (TC_M / 8) * 128, lboB = (P16 / 8) * 128;
  const size_t tbase = (size_t)blockIdx.x * 189;
  uint32_t phase = 0;
  bool ok = true;
  for (int i = 0; i < nslots && ok; ++i) {
    const int slot = a.slot_list[tbase + i];
    const int ts = a.tslot_list[tbase + i];
    // operator image: 3 splits, contiguous
    const uint16_t *bsrc = a.bimg + (size_t)ts * 3 * bsplit;
    const int n16 = (int)(3 * bsplit * 2 / 16);
    for (int c = tid; c < n16; c += TC_M) {
      unsigned d = smem_u32(Bs + 8 * (size_t)c);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(bsrc + 8 * (size_t)c));
    }
    asm volatile("cp.async.commit_group;\n" ::);
    // gathered source multipole of this thread's target row, split in three
    const int src = a.src_tab[(tbase + slot) * TC_M + tid];
    const float *xr = src >= 0 ? a.X + (size_t)(src - a.cell0) * a.KS : nullptr;
    for (int kc = 0; kc < KC; ++kc) {
      float v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k = kc * 8 + j;
        v[j] = (xr && k < a.KS) ? xr[k] : 0.f;
      }
      uint16_t h[8], m[8], l[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) split3(v[j], h[j], m[j], l[j]);
      const size_t off = (size_t)kc * (TC_M / 8) * 64 + (size_t)(tid / 8) * 64 + (tid % 8) * 8;
      uint4 ph, pm, pl;
      ph.x = h[0] | ((uint32_t)h[1] << 16); ph.y = h[2] | ((uint32_t)h[3] << 16);
      ph.z = h[4] | ((uint32_t)h[5] << 16); ph.w = h[6] | ((uint32_t)h[7] << 16);
      pm.x = m[0] | ((uint32_t)m[1] << 16); pm.y = m[2] | ((uint32_t)m[3] << 16);
      pm.z = m[4] | ((uint32_t)m[5] << 16); pm.w = m[6] | ((uint32_t)m[7] << 16);
      pl.x = l[0] | ((uint32_t)l[1] << 16); pl.y = l[2] | ((uint32_t)l[3] << 16);
      pl.z = l[4] | ((uint32_t)l[5] << 16); pl.w = l[6] | ((uint32_t)l[7] << 16);
      *(uint4 *)(As + off) = ph;
      *(uint4 *)(As + asplit + off) = pm;
      *(uint4 *)(As + 2 * asplit + off) = pl;
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
      // smallest split products first: (x3,y1) (x2,y2) (x1,y3) (x2,y1) (x1,y2) (x1,y1)
      const int pa[6] = {2, 1, 0, 1, 0, 0}, pb[6] = {0, 1, 2, 0, 1, 0};
#pragma unroll
      for (int pr = 0; pr < 6; ++pr)
        for (int ks = 0; ks < P16 / 16; ++ks) {
          const uint64_t ad = smem_desc(a0 + (uint32_t)(pa[pr] * asplit * 2) + ks * 2 * lboA, lboA, 128);
          const uint64_t bd = smem_desc(b0 + (uint32_t)(pb[pr] * bsplit * 2) + ks * 2 * lboB, lboB, 128);
          mma_bf16(tmem, ad, bd, idesc, (ks > 0 || pr > 0) ? 1u : 0u);
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&s_mbar))
                   : "memory");
    }
    // the operands are reused for the next slot only after the MMAs finish
    uint32_t done = 0;
    for (long long it = 0; !done; ++it) {
      asm volatile(
          "{\n\t.reg .pred P1;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
          "selp.b32 %0, 1, 0, P1;\n\t}"
          : "=r"(done)
          : "r"(smem_u32(&s_mbar)), "r"(phase)
          : "memory");
      if (!done && it > (1ll << 22)) {
        ok = false;
        break;
      }
    }
    phase ^= 1u;
    // tcgen05.ld is warp-collective: read only when the whole warp saw the commit
    const bool wdone = __all_sync(0xffffffffu, done != 0);
    if (!wdone) ok = false;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (wdone) {
      // this slot's contribution, added in FP32 registers
#pragma unroll
      for (int c0 = 0; c0 < P16; c0 += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[c0 + j] += __uint_as_float(r[j]);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    ok = __syncthreads_and(ok);  // every thread leaves the loop at the same slot
  }
  if (ok) {
    const int tg = s_tgt[warp * 32 + lane];
    if (tg >= 0) {
      float *y = a.Y + (size_t)(tg - a.cell0) * a.KS;
#pragma unroll
      for (int j = 0; j < P16; ++j)
        if (j < a.K) y[j] += acc[j];
    }
  } else if (tid == 0) {
    atomicOr(a.err, FMM_DEV_ERR_TIMEOUT);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

size_t tc_smem_bytes(int P16) { return (size_t)3 * P16 * TC_M * 2 + (size_t)3 * P16 * P16 * 2; }

int tc_build_images(const float *tab, int n_m2l, int K, int KP, int P16, uint16_t *img, cudaStream_t st,
                    int64_t &launches) {
  k_tc_images<<<n_m2l, 256, 0, st>>>(tab, K, KP, P16, img);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

template <int P16>
static int tc_launch_p(const TcArgs &a, int nb, cudaStream_t st) {
  const size_t sh = tc_smem_bytes(P16);
  static size_t attr = 0;
  if (attr < sh) {
    if (cudaFuncSetAttribute(k_m2l_tc<P16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh) != cudaSuccess)
      return FMM_ERR_CUDA;
    attr = sh;
  }
  k_m2l_tc<P16><<<nb, TC_M, sh, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int tc_launch_m2l(const TcArgs &a, int nb, cudaStream_t st, int64_t &launches) {
  if (nb <= 0) return FMM_OK;
  launches += 1;
  switch (a.P16) {
    case 16: return tc_launch_p<16>(a, nb, st);
    case 32: return tc_launch_p<32>(a, nb, st);
    case 48: return tc_launch_p<48>(a, nb, st);
    case 64: return tc_launch_p<64>(a, nb, st);
    case 80: return tc_launch_p<80>(a, nb, st);
    case 96: return tc_launch_p<96>(a, nb, st);
    case 112: return tc_launch_p<112>(a, nb, st);
    case 128: return tc_launch_p<128>(a, nb, st);
    default: return FMM_ERR_UNSUPPORTED;
  }
}

}  // namespace fmm
