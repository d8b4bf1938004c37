// mlp_tc.cuh — the surrogate MLP ensemble on the 5th-generation tensor cores.
//
// One CTA (256 threads) evaluates 128 sites of one species through every
// ensemble member: four 128×64×64 products per member, each issued by one
// thread as tcgen05.mma (kind::tf32, operands in shared memory, the FP32
// accumulator in tensor memory), read back with tcgen05.ld for the epilogue:
//
//   Z1 = X·W1ᵀ        → H1 = SiLU(Z1 + b1), S1 = SiLU'(·)   (S1 stays in registers)
//   Z2 = H1·W2ᵀ       → y = w3·SiLU(Z2 + b2) + b3,  D2 = w3 ⊙ SiLU'(·)
//   G1 = (D2·W2) ⊙ S1
//   dX += G1·W1
//
// The weights are BF16 values, exact in TF32.  Every activation operand is
// split as a = hi + lo with hi its TF32 truncation (the bits the tensor core
// reads) and lo the FP32 remainder, and both halves are multiplied and
// accumulated into the same tensor-memory tile, so the products carry FP32
// accuracy.  Operand tiles use the K-major, non-swizzled canonical layout:
// 8-row × 16-byte core matrices, consecutive along K (128 B apart), row
// groups 2048 B apart.  Waits on the MMA barrier are bounded; a wait that
// runs out sets status bit 16, skips the rest and frees the tensor memory.
#pragma once
#include <cstdint>

namespace pfw {

constexpr int TC_TILE = 128;  // sites (MMA M)
constexpr int TC_W = 64;      // features and hidden units, padded (MMA N and K)
constexpr int TC_OPERAND = TC_TILE * TC_W * 4;  // bytes of one 128×64 FP32 operand tile
constexpr int TC_WEIGHT = TC_W * TC_W * 4;      // bytes of one 64×64 FP32 weight tile
// instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2),
// both K-major, N = 64 (bits 17-22 = N/8), M = 128 (bits 24-28 = M/16)
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_W >> 3) << 17) |
                              ((uint32_t)(TC_TILE >> 4) << 24);

// byte offset of element (row, k) in a K-major [rows][64] FP32 operand tile
__device__ __forceinline__ int tc_off(int row, int k) {
  return ((row >> 3) << 11) + ((k >> 2) << 7) + ((row & 7) << 4) + ((k & 3) << 2);
}

__device__ __forceinline__ uint32_t tc_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, LBO = 128 B (next core
// matrix along K), SBO = 2048 B (next 8 rows), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(2048 >> 4) << 32) |
         ((uint64_t)1 << 46);
}

__device__ __forceinline__ void tc_store(unsigned char* hi, unsigned char* lo, int row, int k, float v) {
  const float h = __uint_as_float(__float_as_uint(v) & 0xFFFFE000u);  // TF32 truncation
  const int o = tc_off(row, k);
  *reinterpret_cast<float*>(hi + o) = h;
  *reinterpret_cast<float*>(lo + o) = v - h;
}

// D[tmem] = A_hi·Bᵀ + A_lo·Bᵀ over K = 64 (8 steps of K = 8 per half)
__device__ __forceinline__ void tc_gemm_issue(uint32_t tmem, uint32_t a_hi, uint32_t a_lo, uint32_t b) {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const uint32_t a = half ? a_lo : a_hi;
#pragma unroll
    for (int s = 0; s < TC_W / 8; ++s) {
      const uint64_t ad = tc_desc(a + 256u * s), bd = tc_desc(b + 256u * s);
      const uint32_t acc = (half | s) ? 1u : 0u;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
          "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
          : "memory");
    }
  }
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

// bounded wait for the phase with this parity; false when it ran out
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 32 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tc_load32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr + 16u));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ float tc_bf16(unsigned short b) { return __uint_as_float((unsigned)b << 16); }

constexpr size_t tc_mlp_smem() {
  return 4 * (size_t)TC_OPERAND + 4 * (size_t)TC_WEIGHT +
         sizeof(float) * (3 * TC_W + 4 * TC_TILE + 2 * TC_TILE) + sizeof(int) * TC_TILE + 64;
}

__global__ void __launch_bounds__(256, 1)
    k_sur_mlp_tc(SurParams sp, int n, const int* __restrict__ count, const int* __restrict__ list,
                 int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char* Xh = tsm;  // X split (A of the first product)
  unsigned char* Xl = Xh + TC_OPERAND;
  unsigned char* Ah = Xl + TC_OPERAND;  // H1, then D2, then G1
  unsigned char* Al = Ah + TC_OPERAND;
  unsigned char* W1s = Al + TC_OPERAND;  // B tiles [n][k]: W1, W2, W2ᵀ, W1ᵀ
  unsigned char* W2s = W1s + TC_WEIGHT;
  unsigned char* W2t = W2s + TC_WEIGHT;
  unsigned char* W1t = W2t + TC_WEIGHT;
  float* vec = reinterpret_cast<float*>(W1t + TC_WEIGHT);  // b1, b2, w3
  float* ym = vec + 3 * TC_W;                              // [4][128]
  float* ypart = ym + 4 * TC_TILE;                         // [2][128]
  int* gate = reinterpret_cast<int*>(ypart + 2 * TC_TILE);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(gate + TC_TILE);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);

  const int z = blockIdx.y, tile = blockIdx.x;
  const int cnt = count[z];
  const int l0 = tile * TC_TILE;
  if (l0 >= cnt) return;
  const int rows = min(TC_TILE, cnt - l0);
  const int* L = list + (size_t)z * n + l0;
  const int nin = sp.nin, H = sp.H, M = sp.M;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t mb = tc_smem(mbar);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(tslot)),
                 "r"(TC_W)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mb), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // standardised features, split for the tensor core; the range gate
  for (int k = tid; k < TC_TILE * TC_W; k += 256) {
    const int r = k / TC_W, i = k - r * TC_W;
    float x = 0.f;
    if (r < rows && i < nin) {
      const double raw = sp.site_feat[(size_t)L[r] * nin + i];
      x = (float)((raw - sp.x_mean[z * nin + i]) / sp.x_std[z * nin + i]);
    }
    tc_store(Xh, Xl, r, i, x);
  }
  if (tid < TC_TILE) gate[tid] = 0;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  for (int k = tid; k < rows * nin; k += 256) {
    const int r = k / nin, i = k - r * nin;
    const float x = *reinterpret_cast<const float*>(Xh + tc_off(r, i)) + *reinterpret_cast<const float*>(Xl + tc_off(r, i));
    if (!(x >= sp.x_lo[z * nin + i] && x <= sp.x_hi[z * nin + i])) gate[r] = 1;  // NaN-safe
  }

  // this thread's accumulator lane (site row) and 32 columns
  const int row = 32 * (warp & 3) + lane, c0 = 32 * (warp >> 2);
  const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)c0;
  float s1[32], dx[32], acc[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) dx[k] = 0.f;
  uint32_t phase = 0;
  bool ok = true;
  const uint32_t xh = tc_smem(Xh), xl = tc_smem(Xl), ah = tc_smem(Ah), al = tc_smem(Al);

  // one product: operands written by all threads, issued by thread 0, read back by all
  auto gemm = [&](uint32_t a_hi, uint32_t a_lo, const unsigned char* b) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (ok) {  // uniform over the CTA
      if (tid == 0) {
        tc_gemm_issue(tmem, a_hi, a_lo, tc_smem(b));
        tc_commit(mb);
      }
      const bool done = tc_wait(mb, phase);
      ok = __syncthreads_and(done);
      if (ok) phase ^= 1u;
      else if (tid == 0) atomicOr(status, 16);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      tc_load32(taddr, acc);
    } else {
#pragma unroll
      for (int k = 0; k < 32; ++k) acc[k] = 0.f;
    }
  };

  for (int m = 0; m < M; ++m) {
    const size_t zm = (size_t)z * M + m;
    __syncthreads();  // the previous member's last product has been read
    for (int k = tid; k < TC_W * TC_W; k += 256) {
      const int o = k / TC_W, i = k - o * TC_W;
      const float w1 = (o < H && i < nin) ? tc_bf16(sp.W1[zm * H * nin + o * nin + i]) : 0.f;
      const float w2 = (o < H && i < H) ? tc_bf16(sp.W2[zm * H * H + o * H + i]) : 0.f;
      *reinterpret_cast<float*>(W1s + tc_off(o, i)) = w1;  // [n = out][k = in]
      *reinterpret_cast<float*>(W1t + tc_off(i, o)) = w1;  // [n = in][k = out]
      *reinterpret_cast<float*>(W2s + tc_off(o, i)) = w2;
      *reinterpret_cast<float*>(W2t + tc_off(i, o)) = w2;
    }
    for (int k = tid; k < TC_W; k += 256) {
      vec[k] = k < H ? sp.b1[zm * H + k] : 0.f;
      vec[TC_W + k] = k < H ? sp.b2[zm * H + k] : 0.f;
      vec[2 * TC_W + k] = k < H ? tc_bf16(sp.w3[zm * H + k]) : 0.f;
    }
    // layer 1
    gemm(xh, xl, W1s);
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      const float zz = acc[k] + vec[c0 + k];
      const float sg = 1.f / (1.f + expf(-zz));
      s1[k] = sg * (1.f + zz * (1.f - sg));
      tc_store(Ah, Al, row, c0 + k, zz * sg);
    }
    // layer 2 and the output
    gemm(ah, al, W2s);
    float yp = 0.f;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      const float zz = acc[k] + vec[TC_W + c0 + k];
      const float sg = 1.f / (1.f + expf(-zz));
      const float w3 = vec[2 * TC_W + c0 + k];
      yp = fmaf(w3, zz * sg, yp);
      tc_store(Ah, Al, row, c0 + k, w3 * (sg * (1.f + zz * (1.f - sg))));
    }
    ypart[(warp >> 2) * TC_TILE + row] = yp;
    // G1 = (D2·W2) ⊙ S1
    gemm(ah, al, W2t);
#pragma unroll
    for (int k = 0; k < 32; ++k) tc_store(Ah, Al, row, c0 + k, acc[k] * s1[k]);
    // dX += G1·W1
    gemm(ah, al, W1t);
#pragma unroll
    for (int k = 0; k < 32; ++k) dx[k] += acc[k];
    if (tid < TC_TILE) ym[m * TC_TILE + tid] = sp.b3[zm] + ypart[tid] + ypart[TC_TILE + tid];
  }
  __syncthreads();
  const double ysd = sp.y_std[z];
  if (ok && row < rows) {
    const size_t s = L[row];
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      const int c = c0 + k;
      if (c < nin) sp.site_df[s * nin + c] = ysd * (double)(dx[k] / (float)M) / sp.x_std[z * nin + c];
    }
  }
  if (ok && tid < rows) {
    float mean = 0.f;
    for (int m = 0; m < M; ++m) mean += ym[m * TC_TILE + tid];
    mean /= (float)M;
    float var = 0.f;
    for (int m = 0; m < M; ++m) var += (ym[m * TC_TILE + tid] - mean) * (ym[m * TC_TILE + tid] - mean);
    var /= (float)M;
    const int s = L[tid];
    sp.site_e[s] = sp.y_mean[z] + ysd * (double)mean;
    sp.flags[s] = (gate[tid] || !(ysd * (double)sqrtf(var) <= (double)sp.tau)) ? 1 : 0;
  }
  if (!ok) tc_wait(mb, phase);  // a product still in flight: one more bounded wait before freeing
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_W) : "memory");
  }
}

}  // namespace pfw
