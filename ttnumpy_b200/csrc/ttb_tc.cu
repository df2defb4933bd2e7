// Float64 products on the fifth-generation tensor cores (tcgen05) in 3xTF32.
//
// Each operand element x (float64) is split into two TF32 values,
// hi = tf32(x) and lo = tf32(x - hi) (both rounded to nearest), and the
// product is accumulated in FP32 in tensor memory (TMEM) as
// A_hi B_hi + A_hi B_lo + A_lo B_hi: about 22 significant bits per
// operand and FP32 accumulation, several orders of magnitude below FP64
// accuracy but eight times the tensor throughput of the FP64 path.
//
// One CTA of 256 threads computes a 128 x 64 tile of C.  K advances 32 at a
// time through two shared-memory stages: every thread converts its share of
// the A and B elements of the next stage while the tensor core works on the
// current one; one elected thread issues the twelve tcgen05.mma of a stage
// (4 K-steps of 8, three split products each) and commits them to the
// stage's mbarrier, which the threads wait on before overwriting the stage.
// The accumulator (128 lanes x 64 FP32 columns) is read back with
// tcgen05.ld by all eight warps and scaled into C in float64.
//
// Shared-memory operands use the K-major layout without swizzle: 8-row x
// 16-byte core matrices, rows of a core matrix 16 bytes apart, core
// matrices along M/N 128 bytes apart (SBO) and along K M*16 (A) or N*16
// (B) bytes apart (LBO).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "ttb200.h"

namespace ttb {
void count_launch();  // the library's launch counter (ttb200.cu)
constexpr int kMaxDevices = 64;
// per-device shared-memory limit set-up (ttb200.cu)
int smem_limit_once(const void* func, int bytes, int* done);
}

namespace {

typedef long long i64;

constexpr int TM = 128, TN = 64, TK = 32;
constexpr int THREADS = 256;
constexpr int A_FL = TM * TK;                  // floats of one A plane (hi or lo)
constexpr int B_FL = TN * TK;                  // floats of one B plane
constexpr int STAGE_FL = 2 * A_FL + 2 * B_FL;  // A hi, A lo, B hi, B lo
constexpr int NSTAGE = 2;
constexpr size_t kSmemBytes = (size_t)NSTAGE * STAGE_FL * 4 + 64;
constexpr unsigned kSpinLimit = 1u << 20;      // mbarrier polls before giving up
constexpr uint32_t kTmemCols = TN;             // FP32 accumulator columns

// instruction descriptor: F32 accumulator, TF32 A and B, both K-major,
// N = TN, M = TM
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

struct TcDesc {
  const double* a;
  const double* b;
  double* c;
  i64 a_rs, a_cs, a_bs, b_rs, b_cs, b_bs, c_rs, c_cs, c_bs;
  int m, n, k, tm, tn;
  double alpha, beta;
};
constexpr int kMaxTc = 24;
struct TcBatch {
  int count;
  int base[kMaxTc + 1];
  TcDesc d[kMaxTc];
};

int g_tc_configured[ttb::kMaxDevices];

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor (no swizzle, descriptor version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

__device__ __forceinline__ void split_tf32(double x, float& hi, float& lo) {
  const float f = __double2float_rn(x);
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(f));
  const float hf = __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(f - hf));
  hi = hf;
  lo = __uint_as_float(l);
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
  for (unsigned it = 0; it < kSpinLimit; ++it) {
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

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(tmem), "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
      : "memory");
}

// Converts the (k0 .. k0+TK) slab of the tile's A rows and B columns into
// the stage's four TF32 planes (zeros outside the matrices).
__device__ __forceinline__ void stage_in(const TcDesc& q, const double* A, const double* B, int m0,
                                         int n0, int k0, float* st) {
  float* ahi = st;
  float* alo = st + A_FL;
  float* bhi = st + 2 * A_FL;
  float* blo = st + 2 * A_FL + B_FL;
  // element e lands at float e of its plane: each warp fills one 8-row x
  // 4-column core matrix (lane -> row lane / 4, column lane % 4), so the
  // shared-memory stores are contiguous and the global loads read 4
  // neighbouring columns of 8 rows
  const int tid = threadIdx.x;
  for (int e = tid; e < TM * TK; e += THREADS) {
    const int u = e >> 5, ln = e & 31;
    const int r = (u % (TM / 8)) * 8 + (ln >> 2), c = (u / (TM / 8)) * 4 + (ln & 3);
    const int gm = m0 + r, gk = k0 + c;
    const double x = (gm < q.m && gk < q.k) ? A[gm * q.a_rs + gk * q.a_cs] : 0.0;
    float hi, lo;
    split_tf32(x, hi, lo);
    ahi[e] = hi;
    alo[e] = lo;
  }
  for (int e = tid; e < TN * TK; e += THREADS) {
    const int u = e >> 5, ln = e & 31;
    const int j = (u % (TN / 8)) * 8 + (ln >> 2), c = (u / (TN / 8)) * 4 + (ln & 3);
    const int gn = n0 + j, gk = k0 + c;
    const double x = (gn < q.n && gk < q.k) ? B[gk * q.b_rs + gn * q.b_cs] : 0.0;
    float hi, lo;
    split_tf32(x, hi, lo);
    bhi[e] = hi;
    blo[e] = lo;
  }
}

__global__ void __launch_bounds__(THREADS, 1) k_gemm_3xtf32(const __grid_constant__ TcBatch tb,
                                                            int* status) {
  extern __shared__ __align__(1024) float smem[];
  float* stages = smem;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + NSTAGE * STAGE_FL);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + NSTAGE);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // which problem, batch entry and tile
  const int t = blockIdx.x;
  int p = 0;
  while (p + 1 < tb.count && tb.base[p + 1] <= t) ++p;
  const TcDesc& q = tb.d[p];
  const int local = t - tb.base[p];
  const int per = q.tm * q.tn;
  const int bi = local / per, rr = local % per;
  const int m0 = (rr / q.tn) * TM, n0 = (rr % q.tn) * TN;
  const double* A = q.a + bi * q.a_bs;
  const double* B = q.b + bi * q.b_bs;
  double* C = q.c + bi * q.c_bs;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar + s)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int nk = q.k > 0 ? (q.k + TK - 1) / TK : 0;
  bool ok = true;
  for (int s = 0; s < nk; ++s) {
    const int buf = s % NSTAGE;
    float* st = stages + buf * STAGE_FL;
    bool w = true;
    if (s >= NSTAGE) w = mbar_wait(smem_u32(mbar + buf), (uint32_t)(((s - NSTAGE) / NSTAGE) & 1));
    if (!__syncthreads_and(w)) {  // the same decision in every thread
      ok = false;
      break;
    }
    stage_in(q, A, B, m0, n0, s * TK, st);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ahi = smem_u32(st), alo = smem_u32(st + A_FL);
      const uint32_t bhi = smem_u32(st + 2 * A_FL), blo = smem_u32(st + 2 * A_FL + B_FL);
      for (int ks = 0; ks < TK / 8; ++ks) {
        const uint32_t ao = ks * 2 * (TM * 16), bo = ks * 2 * (TN * 16);
        const uint64_t dah = sdesc(ahi + ao, TM * 16, 128), dal = sdesc(alo + ao, TM * 16, 128);
        const uint64_t dbh = sdesc(bhi + bo, TN * 16, 128), dbl = sdesc(blo + bo, TN * 16, 128);
        mma_tf32(tmem, dah, dbh, (s > 0 || ks > 0) ? 1u : 0u);
        mma_tf32(tmem, dah, dbl, 1u);
        mma_tf32(tmem, dal, dbh, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(mbar + buf))
                   : "memory");
    }
  }
  if (ok && nk > 0) {
    const bool w =
        mbar_wait(smem_u32(mbar + (nk - 1) % NSTAGE), (uint32_t)(((nk - 1) / NSTAGE) & 1));
    ok = __syncthreads_and(w);
  }
  if (!ok) {
    if (tid == 0 && status) atomicExch(status, 1);
    // let the tensor core drain whatever was issued before the TMEM goes away
    if (nk > 0) mbar_wait(smem_u32(mbar + (nk - 1) % NSTAGE), (uint32_t)(((nk - 1) / NSTAGE) & 1));
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (ok && nk == 0) {  // no K: C = beta * C
    for (int e = tid; e < TM * TN; e += THREADS) {
      const int row = m0 + e / TN, col = n0 + e % TN;
      if (row < q.m && col < q.n) {
        double* cp = C + row * q.c_rs + col * q.c_cs;
        *cp = q.beta != 0.0 ? q.beta * *cp : 0.0;
      }
    }
  } else if (ok) {
    // warp w reads TMEM lanes 32 (w % 4) .. + 31, columns 32 (w / 4) .. + 31
    const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(32 * (warp >> 2));
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
    if (row < q.m) {
      double* crow = C + row * q.c_rs;
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int col = col0 + i;
        if (col < q.n) {
          double val = q.alpha * (double)__uint_as_float(v[i]);
          if (q.beta != 0.0) val = fma(q.beta, crow[col * q.c_cs], val);
          crow[col * q.c_cs] = val;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
  }
}

}  // namespace

extern "C" {

int ttb_gemm_3xtf32(const ttb_gemm_t* ps, int count, int* status, void* stream) {
  if (int e = ttb::smem_limit_once((const void*)k_gemm_3xtf32, (int)kSmemBytes, g_tc_configured))
    return e;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int i = 0;
  while (i < count) {
    TcBatch tb;
    tb.count = 0;
    int blocks = 0;
    while (i < count && tb.count < kMaxTc) {
      const ttb_gemm_t& g = ps[i++];
      if (g.m <= 0 || g.n <= 0 || g.batch <= 0) continue;
      TcDesc& d = tb.d[tb.count];
      d.a = g.a;
      d.b = g.b;
      d.c = g.c;
      d.a_rs = g.a_rs;
      d.a_cs = g.a_cs;
      d.a_bs = g.a_bs;
      d.b_rs = g.b_rs;
      d.b_cs = g.b_cs;
      d.b_bs = g.b_bs;
      d.c_rs = g.c_rs;
      d.c_cs = g.c_cs;
      d.c_bs = g.c_bs;
      d.m = g.m;
      d.n = g.n;
      d.k = g.k;
      d.tm = (g.m + TM - 1) / TM;
      d.tn = (g.n + TN - 1) / TN;
      d.alpha = g.alpha;
      d.beta = g.beta;
      tb.base[tb.count] = blocks;
      blocks += d.tm * d.tn * g.batch;
      ++tb.count;
    }
    tb.base[tb.count] = blocks;
    if (blocks == 0) continue;
    k_gemm_3xtf32<<<blocks, THREADS, kSmemBytes, s>>>(tb, status);
    ttb::count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
  }
  return 0;
}

}  // extern "C"
