// Block-level float64 products in 3xTF32 on the fifth-generation tensor
// cores (tcgen05), for kernels in which one thread block does all the work
// of a solve (the persistent AMEn kernel).
//
// C (M x N) = alpha * A (M x K) * B (K x N) + beta * C with float64 operands
// anywhere in global memory (strided views) and a float64 output view with
// split indices (OMat).  Every operand element x is split into two TF32
// values while it is staged into shared memory, hi = tf32(x) and
// lo = tf32(x - hi) (rounded to nearest), and each 128 x 64 output tile
// accumulates A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32 in tensor memory:
// about 22 significant bits per operand, relative errors near 1e-6 of
// |A| |B|, far below float64 accuracy; the callers use it only inside
// iterative refinement whose residuals are float64.
//
// One elected thread issues the MMAs (M = 128, N = 64, K = 8, three split
// products per K step) and commits them to the mbarrier of the shared-memory
// stage they read; the block stages the next K slab into the other stage
// meanwhile.  Stages, mbarriers and the accumulator's tensor-memory columns
// belong to the caller (TcState), which keeps them for the life of the
// block: the tile and K-step sequence of all products forms one pipeline
// whose mbarrier phases are counted in TcState, so a product may follow
// another without re-initialising anything.  Every mbarrier wait is bounded;
// a wait that gives up sets TcState::failed, after which the products are
// skipped (their outputs are left unwritten) and the caller reports an error.
//
// Shared-memory operands use the K-major layout without swizzle: 8-row x
// 16-byte core matrices, rows 16 bytes apart, core matrices 128 bytes apart
// along M/N (SBO) and M*16 (A) or N*16 (B) bytes apart along K (LBO).
#pragma once

#include <stdint.h>

#include "ttb_device.cuh"

namespace ttb {

constexpr int TC_M = 128, TC_N = 64, TC_K = 32;
constexpr int TC_A_FL = TC_M * TC_K;                      // floats of one A plane
constexpr int TC_B_FL = TC_N * TC_K;                      // floats of one B plane
constexpr int TC_STAGE_FL = 2 * TC_A_FL + 2 * TC_B_FL;    // A hi, A lo, B hi, B lo
constexpr int TC_STAGES = 2;
constexpr int TC_RING_BYTES = TC_STAGES * TC_STAGE_FL * 4;  // 96 KiB
constexpr uint32_t TC_TMEM_COLS = TC_N;                   // FP32 accumulator columns
constexpr unsigned TC_SPIN = 1u << 22;                    // mbarrier polls before giving up

// instruction descriptor: F32 accumulator, TF32 A and B, both K-major,
// N = TC_N, M = TC_M
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) |
                              ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);

struct TcState {
  float* ring;        // TC_RING_BYTES of shared memory, 16-byte aligned
  uint64_t* mbar;     // TC_STAGES mbarriers in shared memory
  uint32_t* slot;     // shared word receiving the tensor-memory address
  uint32_t tmem;      // accumulator columns (TC_TMEM_COLS)
  unsigned steps;     // K steps issued so far (all products): stage = step % 2
  int failed;         // a bounded wait gave up
};

static __device__ __forceinline__ uint32_t tc_smem(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor (no swizzle, descriptor version 1)
static __device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

static __device__ __forceinline__ void tc_split(double x, float& hi, float& lo) {
  const float f = __double2float_rn(x);
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(f));
  const float hf = __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(f - hf));
  hi = hf;
  lo = __uint_as_float(l);
}

static __device__ __forceinline__ bool tc_wait(uint32_t addr, uint32_t parity) {
  for (unsigned it = 0; it < TC_SPIN; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

static __device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(tmem), "l"(a), "l"(b), "r"(TC_IDESC), "r"(acc)
      : "memory");
}

// Allocates the accumulator columns and initialises the mbarriers; the whole
// block calls it once, before the first product.
static __device__ void tc_init(TcState& s) {
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc_smem(s.slot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < TC_STAGES; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(s.mbar + i)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  s.tmem = *s.slot;
  s.steps = 0;
  s.failed = 0;
}

// Waits (bounded) for every product issued so far, then frees the
// accumulator columns; the whole block calls it once, after the last
// product (also after a failure, so that no MMA is left reading freed
// tensor memory).
static __device__ void tc_release(TcState& s) {
  if (s.steps > 0) {
    const unsigned last = s.steps - 1;
    tc_wait(tc_smem(s.mbar + last % TC_STAGES), (last / TC_STAGES) & 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem),
                 "r"(TC_TMEM_COLS)
                 : "memory");
  }
}

// Converts the K slab k0 .. k0 + TC_K of the tile's A rows and B columns
// into the stage's four TF32 planes (zeros outside the matrices).  Element e
// of a plane lands at float e: each warp fills 8-row x 4-column core
// matrices (lane -> row lane / 4, column lane % 4).
static __device__ __forceinline__ void tc_stage(const CMat& A, const CMat& B, int M, int N, int K,
                                                int m0, int n0, int k0, float* st) {
  float* ahi = st;
  float* alo = st + TC_A_FL;
  float* bhi = st + 2 * TC_A_FL;
  float* blo = st + 2 * TC_A_FL + TC_B_FL;
  constexpr int NA = TC_M * TC_K / TTB_THREADS, NB = TC_N * TC_K / TTB_THREADS;
  static_assert(NA * TTB_THREADS == TC_M * TC_K && NB * TTB_THREADS == TC_N * TC_K,
                "stage loads must divide evenly");
  // all of a thread's loads first, so that they are in flight together
  double xa[NA], xb[NB];
#pragma unroll
  for (int t = 0; t < NA; ++t) {
    const int e = threadIdx.x + t * TTB_THREADS;
    const int u = e >> 5, ln = e & 31;
    const int r = (u % (TC_M / 8)) * 8 + (ln >> 2), c = (u / (TC_M / 8)) * 4 + (ln & 3);
    const int gm = m0 + r, gk = k0 + c;
    xa[t] = (gm < M && gk < K) ? A(gm, gk) : 0.0;
  }
#pragma unroll
  for (int t = 0; t < NB; ++t) {
    const int e = threadIdx.x + t * TTB_THREADS;
    const int u = e >> 5, ln = e & 31;
    const int j = (u % (TC_N / 8)) * 8 + (ln >> 2), c = (u / (TC_N / 8)) * 4 + (ln & 3);
    const int gn = n0 + j, gk = k0 + c;
    xb[t] = (gn < N && gk < K) ? B(gk, gn) : 0.0;
  }
#pragma unroll
  for (int t = 0; t < NA; ++t) {
    const int e = threadIdx.x + t * TTB_THREADS;
    float hi, lo;
    tc_split(xa[t], hi, lo);
    ahi[e] = hi;
    alo[e] = lo;
  }
#pragma unroll
  for (int t = 0; t < NB; ++t) {
    const int e = threadIdx.x + t * TTB_THREADS;
    float hi, lo;
    tc_split(xb[t], hi, lo);
    bhi[e] = hi;
    blo[e] = lo;
  }
}

// C = alpha * A B + beta * C on the tensor cores (see the file comment).
// K must be positive.  Block-uniform: every thread calls it with the same
// arguments.
static __device__ __noinline__ void cta_gemm_tc(TcState& s, CMat A, CMat B, OMat C, int M, int N,
                                                int K, double alpha, double beta) {
  if (M <= 0 || N <= 0 || K <= 0 || s.failed) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tm = (M + TC_M - 1) / TC_M, tn = (N + TC_N - 1) / TC_N;
  const int nk = (K + TC_K - 1) / TC_K;
  for (int tile = 0; tile < tm * tn; ++tile) {
    const int m0 = (tile / tn) * TC_M, n0 = (tile % tn) * TC_N;
    for (int kt = 0; kt < nk; ++kt) {
      const unsigned step = s.steps;
      const int buf = (int)(step % TC_STAGES);
      float* st = s.ring + buf * TC_STAGE_FL;
      bool ok = true;
      if (step >= TC_STAGES) {  // the MMAs that last read this stage
        const unsigned prev = step - TC_STAGES;
        ok = tc_wait(tc_smem(s.mbar + buf), (prev / TC_STAGES) & 1u);
      }
      if (!__syncthreads_and(ok)) {
        s.failed = 1;
        return;
      }
      tc_stage(A, B, M, N, K, m0, n0, kt * TC_K, st);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (threadIdx.x == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t ahi = tc_smem(st), alo = tc_smem(st + TC_A_FL);
        const uint32_t bhi = tc_smem(st + 2 * TC_A_FL), blo = tc_smem(st + 2 * TC_A_FL + TC_B_FL);
        for (int ks = 0; ks < TC_K / 8; ++ks) {
          const uint32_t ao = ks * 2 * (TC_M * 16), bo = ks * 2 * (TC_N * 16);
          const uint64_t dah = tc_sdesc(ahi + ao, TC_M * 16, 128);
          const uint64_t dal = tc_sdesc(alo + ao, TC_M * 16, 128);
          const uint64_t dbh = tc_sdesc(bhi + bo, TC_N * 16, 128);
          const uint64_t dbl = tc_sdesc(blo + bo, TC_N * 16, 128);
          tc_mma(s.tmem, dah, dbh, (kt > 0 || ks > 0) ? 1u : 0u);
          tc_mma(s.tmem, dah, dbl, 1u);
          tc_mma(s.tmem, dal, dbh, 1u);
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                tc_smem(s.mbar + buf))
            : "memory");
      }
      s.steps = step + 1;
    }
    // the tile's accumulator is complete once its last commit has arrived
    const unsigned last = s.steps - 1;
    const bool ok = tc_wait(tc_smem(s.mbar + last % TC_STAGES), (last / TC_STAGES) & 1u);
    if (!__syncthreads_and(ok)) {
      s.failed = 1;
      return;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (tile rows),
    // columns 32 (w / 4) .. + 31
    const uint32_t taddr =
        s.tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(32 * (warp >> 2));
    uint32_t v[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, "
        "%29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
          "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
          "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const int row = m0 + 32 * (warp & 3) + lane;
    const int col0 = n0 + 32 * (warp >> 2);
    if (row < M) {
      double* crow = C.p + C.row(row);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int col = col0 + i;
        if (col < N) {
          double* cp = crow + C.col(col);
          double val = alpha * (double)__uint_as_float(v[i]);
          if (beta != 0.0) val = fma(beta, *cp, val);
          *cp = val;
        }
      }
    }
    // the accumulator is read before the next tile's first MMA overwrites it
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
}

}  // namespace ttb
