// CTA-level float64 building blocks shared by every kernel of libttb200.
//
// All routines here are executed cooperatively by one thread block of
// TTB_THREADS threads.  Matrices are addressed through generic pointers and
// explicit (row, column) element strides, so the same code runs on shared
// memory, on global memory and on transposed views.  Reductions are done in a
// fixed order (per-thread strided partials, a warp tree, then the warp sums
// in warp order), so a result never depends on scheduling and every thread
// of the block sees the same value.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#ifndef TTB_THREADS
#define TTB_THREADS 256
#endif
#define TTB_WARPS (TTB_THREADS / 32)

namespace ttb {

typedef long long i64;

// Host side (ttb200.cu): raise ``func``'s dynamic shared-memory limit to
// ``bytes`` on the current device the first time a launch there needs it.
// ``done`` holds one flag per device index (kMaxDevices); a flag is set only
// after cudaFuncSetAttribute succeeded, and its error is returned otherwise.
constexpr int kMaxDevices = 64;
int smem_limit_once(const void* func, int bytes, int* done);

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------

static __device__ __forceinline__ double warp_sum(double v) {
  // tree towards lane 0, then broadcast lane 0 so all lanes agree bitwise
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return __shfl_sync(0xffffffffu, v, 0);
}

// Sum over the block; every thread returns the same value.  ``red`` must
// hold TTB_WARPS doubles of shared memory.  Contains two __syncthreads.
static __device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int i = 0; i < TTB_WARPS; ++i) t += red[i];
  return t;
}

// Index of the entry of largest absolute value, first index on ties (the
// LAPACK idamax convention).  ``redv``/``redi`` hold TTB_WARPS entries.
static __device__ __forceinline__ int block_argmax_abs(double v, int idx, double* redv, int* redi) {
  double a = (idx >= 0) ? fabs(v) : -1.0;
  int i = idx;
  for (int o = 16; o > 0; o >>= 1) {
    double a2 = __shfl_down_sync(0xffffffffu, a, o);
    int i2 = __shfl_down_sync(0xffffffffu, i, o);
    if (a2 > a || (a2 == a && i2 >= 0 && (i < 0 || i2 < i))) { a = a2; i = i2; }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) { redv[wid] = a; redi[wid] = i; }
  __syncthreads();
  double best = -1.0;
  int bi = -1;
  for (int w = 0; w < TTB_WARPS; ++w) {
    double a2 = redv[w];
    int i2 = redi[w];
    if (a2 > best || (a2 == best && i2 >= 0 && (bi < 0 || i2 < bi))) { best = a2; bi = i2; }
  }
  return bi;
}

// ---------------------------------------------------------------------------
// strided matrix view
// ---------------------------------------------------------------------------

struct Mat {
  double* p;
  i64 rs, cs;  // element strides of a row step and a column step
  __device__ __forceinline__ double& operator()(int i, int j) const { return p[i * rs + j * cs]; }
};

struct CMat {
  const double* p;
  i64 rs, cs;
  __device__ __forceinline__ double operator()(int i, int j) const { return p[i * rs + j * cs]; }
};

// ---------------------------------------------------------------------------
// GEMM: one GBM x 64 output tile per call, K staged through shared memory,
// products on the FP64 tensor-core path (mma.sync m8n8k4 .f64)
// ---------------------------------------------------------------------------

// Tile rows: 32 per four warps (64 for 8 warps, 96 for 12), 64 columns.
// K depth of a staged slab (16, or 32 for half the block barriers per K)
#ifndef TTB_GBK
#define TTB_GBK 16
#endif
constexpr int GBM = 8 * TTB_WARPS, GBN = 64, GBK = TTB_GBK;
// Row pitches of the staged tiles: 4 more than a multiple of 16 doubles puts
// the four k-rows a fragment load touches on disjoint bank groups, so each
// load takes two wavefronts.
constexpr int GPITCH_A = GBM + 4, GPITCH_B = GBN + 4;
// loads per thread of one k-step's A and B tiles
constexpr int GNA = (GBM * GBK) / TTB_THREADS;
constexpr int GNB = (GBK * GBN + TTB_THREADS - 1) / TTB_THREADS;
static_assert(GNA * TTB_THREADS == GBM * GBK, "A tile loads must divide evenly");

struct GemmSmem {
  double a[GBK][GPITCH_A];  // a[k][m]
  double b[GBK][GPITCH_B];  // b[k][n]
};

// D += A(8x4, row) * B(4x8, col) in FP64; lane l holds A[l/4][l%4],
// B[l%4][l/4] and D[l/4][2(l%4) + {0,1}].
static __device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// GEMM output view whose row and column indices may each be split in two:
// (i, j) -> p + (i / rdiv) * rs_hi + (i % rdiv) * rs
//             + (j / cdiv) * cs_hi + (j % cdiv) * cs.
// A plain Mat converts to the unsplit form.  The split lets one product write
// a result whose two index groups interleave in memory (a tensor
// contraction's output permuted for the next contraction).
constexpr int kNoSplit = 1 << 30;

// Division of 0 <= n < 2^31 by an invariant d >= 1 as a multiply and a
// shift (Granlund and Montgomery, "Division by invariant integers using
// multiplication", 1994, theorem 4.2 with N = 32): with l = ceil(log2 d)
// and m = floor(2^32 (2^l - d) / d) + 1 (below 2^32),
// n / d = (mulhi(m, n) + n) >> l, the sum staying below 2^32 for n < 2^31.
// The split-index outputs divide every output index by their split sizes.
struct FastDiv {
  uint32_t m;
  int l, d;
  __device__ FastDiv() : m(1), l(0), d(1) {}
  __device__ explicit FastDiv(int d_) : d(d_) {
    l = 32 - __clz(d_ - 1);
    m = (uint32_t)(((1ull << 32) * ((1ull << l) - (unsigned long long)d_)) / (unsigned)d_ + 1);
  }
  __device__ __forceinline__ int div(int n) const {
    return (int)((__umulhi(m, (uint32_t)n) + (uint32_t)n) >> l);
  }
};

struct OMat {
  double* p;
  i64 rs, cs, rs_hi, cs_hi;
  int rdiv, cdiv;
  FastDiv rq, cq;  // rdiv and cdiv (when split)
  __device__ OMat(Mat m)
      : p(m.p), rs(m.rs), cs(m.cs), rs_hi(0), cs_hi(0), rdiv(kNoSplit), cdiv(kNoSplit) {}
  __device__ OMat(double* p_, int rdiv_, i64 rs_hi_, i64 rs_, int cdiv_, i64 cs_hi_, i64 cs_)
      : p(p_), rs(rs_), cs(cs_), rs_hi(rs_hi_), cs_hi(cs_hi_), rdiv(rdiv_), cdiv(cdiv_) {
    if (rdiv != kNoSplit) rq = FastDiv(rdiv);
    if (cdiv != kNoSplit) cq = FastDiv(cdiv);
  }
  __device__ __forceinline__ i64 row(int i) const {
    if (rdiv == kNoSplit) return i * rs;
    const int q = rq.div(i);
    return q * rs_hi + (i - q * rdiv) * rs;
  }
  __device__ __forceinline__ i64 col(int j) const {
    if (cdiv == kNoSplit) return j * cs;
    const int q = cq.div(j);
    return q * cs_hi + (j - q * cdiv) * cs;
  }
};

// C[m0:m0+GBM, n0:n0+64] = alpha * A * B + beta * C over the full K range.
// A is M x K, B is K x N.  beta == 0 never reads C.  The warps form a
// (TTB_WARPS / 4) x 4 grid of 32 x 16 warp tiles, each 4 x 2 MMA tiles of
// 8 x 8 (the tile is GBM = 8 * TTB_WARPS rows by 64 columns).
static __device__ void cta_gemm_tile(CMat A, CMat B, const OMat& C, int M, int N, int K, int m0,
                                     int n0, double alpha, double beta, GemmSmem& sm) {
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
  const int g = lane >> 2, t = lane & 3;
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // loads walk the unit-stride direction of each operand when there is one
  const bool a_kfast = (A.cs == 1);
  const bool b_nfast = (B.cs == 1) || (B.rs != 1);
  double ra[GNA], rb[GNB];
  auto load = [&](int k0) {
#pragma unroll
    for (int e = 0; e < GNA; ++e) {
      int idx = tid + e * TTB_THREADS;
      int mm, kk;
      if (a_kfast) { kk = idx % GBK; mm = idx / GBK; } else { mm = idx % GBM; kk = idx / GBM; }
      int gm = m0 + mm, gk = k0 + kk;
      ra[e] = (gm < M && gk < K) ? A(gm, gk) : 0.0;
    }
#pragma unroll
    for (int e = 0; e < GNB; ++e) {
      int idx = tid + e * TTB_THREADS;
      if (idx >= GBK * GBN) break;
      int nn, kb;
      if (b_nfast) { nn = idx % GBN; kb = idx / GBN; } else { kb = idx % GBK; nn = idx / GBK; }
      int gn = n0 + nn, gk2 = k0 + kb;
      rb[e] = (gn < N && gk2 < K) ? B(gk2, gn) : 0.0;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int e = 0; e < GNA; ++e) {
      int idx = tid + e * TTB_THREADS;
      int mm, kk;
      if (a_kfast) { kk = idx % GBK; mm = idx / GBK; } else { mm = idx % GBM; kk = idx / GBM; }
      sm.a[kk][mm] = ra[e];
    }
#pragma unroll
    for (int e = 0; e < GNB; ++e) {
      int idx = tid + e * TTB_THREADS;
      if (idx >= GBK * GBN) break;
      int nn, kb;
      if (b_nfast) { nn = idx % GBN; kb = idx / GBN; } else { kb = idx % GBK; nn = idx / GBK; }
      sm.b[kb][nn] = rb[e];
    }
  };

  if (K > 0) load(0);
  for (int k0 = 0; k0 < K; k0 += GBK) {
    __syncthreads();  // previous compute finished with the tile
    store();
    __syncthreads();
    if (k0 + GBK < K) load(k0 + GBK);  // prefetch overlaps the MMAs below
#pragma unroll
    for (int kk = 0; kk < GBK; kk += 4) {
      double av[4], bv[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = sm.a[kk + t][wm + 8 * i + g];
#pragma unroll
      for (int j = 0; j < 2; ++j) bv[j] = sm.b[kk + t][wn + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], av[i], bv[j]);
    }
  }
  i64 coff[2][2];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int h = 0; h < 2; ++h) coff[j][h] = C.col(n0 + wn + 8 * j + 2 * t + h);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + wm + 8 * i + g;
    if (gm >= M) continue;
    double* crow = C.p + C.row(gm);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gn = n0 + wn + 8 * j + 2 * t + h;
        if (gn >= N) continue;
        double v = alpha * acc[i][j][h];
        if (beta != 0.0) v = fma(beta, crow[coff[j][h]], v);
        crow[coff[j][h]] = v;
      }
  }
  __syncthreads();  // callers may reuse the staging buffers right away
}

// Whole product, looping over all output tiles with the one block.
static __device__ __noinline__ void cta_gemm(CMat A, CMat B, OMat C, int M, int N, int K, double alpha, double beta,
                         GemmSmem& sm) {
  for (int m0 = 0; m0 < M; m0 += GBM)
    for (int n0 = 0; n0 < N; n0 += GBN) cta_gemm_tile(A, B, C, M, N, K, m0, n0, alpha, beta, sm);
}

// ---------------------------------------------------------------------------
// Pipelined GEMM: the same 64x64 tiles and MMA fragments as cta_gemm_tile,
// with operands copied by cp.async into a ring of GSTAGES shared-memory
// stages.  The (output tile, k-tile) steps of the whole product form one
// sequence, so loads run GSTAGES - 1 steps ahead across tile boundaries and
// a tile's first operands arrive while the previous tile is finishing.
// ``ring`` holds GSTAGES * GSTAGE_D doubles of shared memory; its
// first stage has the layout of GemmSmem.  A and B may be anywhere (shared
// operands take the one-stage path); C must not overlap the ring.
// ---------------------------------------------------------------------------

constexpr int GSTAGES = 3;
constexpr int GSTAGE_D = GBK * (GPITCH_A + GPITCH_B);

static __device__ __forceinline__ void cp_async8(double* dst, const double* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = ok ? 8 : 0;  // 0 bytes read: the destination is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(sz)
               : "memory");
}
static __device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
static __device__ __forceinline__ void cp_async_wait_ahead() {
  asm volatile("cp.async.wait_group %0;" ::"n"(GSTAGES - 2) : "memory");
}
static __device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Split-K product for a small output and a long K range (the V^T V and
// V^T C products of the blocked factorisations: M, N <= 48, one of them <= 16,
// K in the thousands), where the tiled pipeline would spend one
// synchronised k-step per 16 of K on a mostly empty 64 x 64 tile.  Each warp
// takes a contiguous K slice and accumulates the whole MI*8 x NJ*8 product
// in DMMA fragments from direct global loads (32-byte runs along K), with no
// block barrier in the loop; the eight partial products are then added in
// warp order through ``scratch`` (TTB_WARPS * M * N doubles of shared
// memory), so the result does not depend on scheduling.
template <int MI, int NJ>
static __device__ __noinline__ void cta_gemm_skinny(CMat A, CMat B, OMat C, int M, int N, int K,
                                                    double alpha, double beta, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int mi = (M + 7) >> 3, nj = (N + 7) >> 3;
  double acc[MI][NJ][2];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int kper = (((K + TTB_WARPS - 1) / TTB_WARPS) + 3) & ~3;
  const int kb = warp * kper, ke = min(K, kb + kper);
  const double* ap[MI];
  const double* bp[NJ];
  bool aok[MI], bok[NJ];
#pragma unroll
  for (int i = 0; i < MI; ++i) {
    aok[i] = 8 * i + g < M;
    ap[i] = A.p + (aok[i] ? (i64)(8 * i + g) * A.rs : 0);
  }
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    bok[j] = 8 * j + g < N;
    bp[j] = B.p + (bok[j] ? (i64)(8 * j + g) * B.cs : 0);
  }
#pragma unroll 4
  for (int k0 = kb; k0 < ke; k0 += 4) {
    const int kk = k0 + t;
    const bool okk = kk < ke;
    double av[MI], bv[NJ];
#pragma unroll
    for (int i = 0; i < MI; ++i) av[i] = (okk && aok[i]) ? ap[i][(i64)kk * A.cs] : 0.0;
#pragma unroll
    for (int j = 0; j < NJ; ++j) bv[j] = (okk && bok[j]) ? bp[j][(i64)kk * B.rs] : 0.0;
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
        if (i < mi && j < nj) dmma_8x8x4(acc[i][j][0], acc[i][j][1], av[i], bv[j]);
  }
  const int mn = M * N;
  double* mine = scratch + (i64)warp * mn;
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = 8 * i + g, col = 8 * j + 2 * t + h;
        if (r < M && col < N) mine[r * N + col] = acc[i][j][h];
      }
  __syncthreads();
  for (int e = threadIdx.x; e < mn; e += TTB_THREADS) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < TTB_WARPS; ++w) v += scratch[(i64)w * mn + e];
    const int r = e / N, col = e % N;
    double* cp = C.p + C.row(r) + C.col(col);
    v *= alpha;
    if (beta != 0.0) v = fma(beta, *cp, v);
    *cp = v;
  }
  __syncthreads();  // callers may reuse the scratch and read C right away
}

// Output shapes and K lengths that take the split-K path.
constexpr int kSkinnyK = 128;
static_assert(TTB_WARPS * 16 * 48 <= GSTAGES * GSTAGE_D, "split-K scratch must fit the ring");

// True when cta_gemm_pipe takes its tiled path for these operands (not the
// one-stage tile or the split-K product), the path whose output tiles may be
// shared out between the blocks of a cluster (tile0, tstride below).
static __device__ __forceinline__ bool gemm_pipe_tiled(CMat A, CMat B, int M, int N, int K) {
  if (M <= 0 || N <= 0 || K <= 0 || __isShared(A.p) || __isShared(B.p)) return false;
  if (K >= kSkinnyK && A.cs == 1 && B.rs == 1 && ((M <= 16 && N <= 48) || (M <= 48 && N <= 16)))
    return false;
  return true;
}

// The tiled path of cta_gemm_pipe for TM x TN output tiles (eight warps of
// 32 x 16, TN / 16 of them along N), K staged TK at a time through an
// NS-stage cp.async ring.  Each output element accumulates its K range in
// steps of four (one DMMA each) in increasing order whatever the tile
// shape, so every shape gives the same bits.
template <int TM, int TN, int TK, int NS>
static __device__ __forceinline__ void gemm_tiles(CMat A, CMat B, OMat C, int M, int N, int K,
                                                  double alpha, double beta, double* ring,
                                                  int tile0, int tstride) {
  static_assert(TTB_WARPS == 8 && TM * TN == 8 * 32 * 16, "eight warps of 32 x 16");
  static_assert(TK % 4 == 0, "K steps of four");
  constexpr int PA = TM + 4, PB = TN + 4;  // pitches: see GPITCH_A
  constexpr int SD = TK * (PA + PB);       // doubles of a stage
  static_assert(NS * SD <= GSTAGES * GSTAGE_D, "stages must fit the ring");
  constexpr int NA = (TM * TK) / TTB_THREADS;
  constexpr int NB = (TK * TN + TTB_THREADS - 1) / TTB_THREADS;
  static_assert(NA * TTB_THREADS == TM * TK, "A tile loads must divide evenly");
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = (warp / (TN / 16)) * 32, wn = (warp % (TN / 16)) * 16;
  const int g = lane >> 2, t = lane & 3;
  const int tn = (N + TN - 1) / TN;
  const int nk = (K + TK - 1) / TK;
  const int tiles = ((M + TM - 1) / TM) * tn;
  const int nloc = tile0 < tiles ? (tiles - tile0 + tstride - 1) / tstride : 0;
  const int total = nloc * nk;
  const bool a_kfast = (A.cs == 1);
  const bool b_nfast = (B.cs == 1) || (B.rs != 1);
  auto issue = [&](int step) {
    if (step < total) {
      const int tile = tile0 + (step / nk) * tstride, kt = step % nk;
      const int m0 = (tile / tn) * TM, n0 = (tile % tn) * TN, k0 = kt * TK;
      double* sa = ring + (step % NS) * SD;
      double* sb = sa + TK * PA;
#pragma unroll
      for (int e = 0; e < NA; ++e) {
        const int idx = tid + e * TTB_THREADS;
        int mm, kk;
        if (a_kfast) { kk = idx % TK; mm = idx / TK; } else { mm = idx % TM; kk = idx / TM; }
        const int gm = m0 + mm, gk = k0 + kk;
        const bool oka = gm < M && gk < K;
        cp_async8(sa + kk * PA + mm, oka ? A.p + gm * A.rs + gk * A.cs : A.p, oka);
      }
#pragma unroll
      for (int e = 0; e < NB; ++e) {
        const int idx = tid + e * TTB_THREADS;
        if (idx >= TK * TN) break;
        int nn, kb;
        if (b_nfast) { nn = idx % TN; kb = idx / TN; } else { kb = idx % TK; nn = idx / TK; }
        const int gn = n0 + nn, gk2 = k0 + kb;
        const bool okb = gn < N && gk2 < K;
        cp_async8(sb + kb * PB + nn, okb ? B.p + gk2 * B.rs + gn * B.cs : B.p, okb);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int st = 0; st < NS - 1; ++st) issue(st);
  double acc[4][2][2];
  for (int step = 0; step < total; ++step) {
    const int kt = step % nk;
    if (kt == 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    }
    asm volatile("cp.async.wait_group %0;" ::"n"(NS - 2) : "memory");
    __syncthreads();  // this step's operands landed; the previous step's reads are done
    issue(step + NS - 1);
    const double* sa = ring + (step % NS) * SD;
    const double* sb = sa + TK * PA;
    const int kvalid = K - kt * TK;  // the last slab's groups of four past K are zeros: skipped
#pragma unroll
    for (int kk = 0; kk < TK; kk += 4) {
      if (kk >= kvalid) break;
      double av[4], bv[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = sa[(kk + t) * PA + wm + 8 * i + g];
#pragma unroll
      for (int j = 0; j < 2; ++j) bv[j] = sb[(kk + t) * PB + wn + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], av[i], bv[j]);
    }
    if (kt == nk - 1) {
      const int tile = tile0 + (step / nk) * tstride;
      const int m0 = (tile / tn) * TM, n0 = (tile % tn) * TN;
      i64 coff[2][2];
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) coff[j][h] = C.col(n0 + wn + 8 * j + 2 * t + h);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int gm = m0 + wm + 8 * i + g;
        if (gm >= M) continue;
        double* crow = C.p + C.row(gm);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int gn = n0 + wn + 8 * j + 2 * t + h;
            if (gn >= N) continue;
            double v = alpha * acc[i][j][h];
            if (beta != 0.0) v = fma(beta, crow[coff[j][h]], v);
            crow[coff[j][h]] = v;
          }
      }
    }
  }
  cp_async_wait_all();
}


// ``tile0`` and ``tstride``: on the tiled path, compute only the output
// tiles tile0, tile0 + tstride, ... (row-major tile order), each exactly as
// the whole product computes it.
static __device__ __noinline__ void cta_gemm_pipe(CMat A, CMat B, OMat C, int M, int N, int K,
                                                  double alpha, double beta, double* ring,
                                                  int tile0 = 0, int tstride = 1) {
  if (M <= 0 || N <= 0) return;
  // cp.async copies from global memory only: operands in shared memory, and
  // K == 0 (C = beta * C), go through the one-stage tile
  if (K <= 0 || __isShared(A.p) || __isShared(B.p)) {
    cta_gemm(A, B, C, M, N, K, alpha, beta, *reinterpret_cast<GemmSmem*>(ring));
    return;
  }
  // (operands contiguous along K only: the split-K loads read 32-byte runs of K)
  if (K >= kSkinnyK && A.cs == 1 && B.rs == 1) {
    if (M <= 16 && N <= 48) {
      cta_gemm_skinny<2, 6>(A, B, C, M, N, K, alpha, beta, ring);
      return;
    }
    if (M <= 48 && N <= 16) {
      cta_gemm_skinny<6, 2>(A, B, C, M, N, K, alpha, beta, ring);
      return;
    }
  }
  // 128 x 32 tiles where they cover the output with at least a fifth less
  // padded area than 64 x 64 tiles (N <= 32 with M > 64, or N just above a
  // multiple of 64, as 65-96): their operand loads per MMA are a fifth
  // higher, so a smaller saving would not pay
  const i64 pad64 = (i64)((M + 63) / 64 * 64) * ((N + 63) / 64 * 64);
  const i64 pad128 = (i64)((M + 127) / 128 * 128) * ((N + 31) / 32 * 32);
  if (5 * pad128 <= 4 * pad64)
    gemm_tiles<128, 32, 12, 3>(A, B, C, M, N, K, alpha, beta, ring, tile0, tstride);
  else
    gemm_tiles<GBM, GBN, GBK, GSTAGES>(A, B, C, M, N, K, alpha, beta, ring, tile0, tstride);
  __syncthreads();  // callers may reuse the ring and read C right away
}

// The blocked factorisations take an optional GEMM ring: with one, their
// trailing-update products are pipelined (cta_gemm_pipe), else they use the
// one-stage tile in ``gsm``.
static __device__ __forceinline__ void gemm_sel(CMat A, CMat B, OMat C, int M, int N, int K,
                                                double alpha, double beta, GemmSmem& gsm,
                                                double* ring) {
  if (ring)
    cta_gemm_pipe(A, B, C, M, N, K, alpha, beta, ring);
  else
    cta_gemm(A, B, C, M, N, K, alpha, beta, gsm);
}

// ---------------------------------------------------------------------------
// copies
// ---------------------------------------------------------------------------

static __device__ __forceinline__ void cta_copy(CMat src, Mat dst, int M, int N, double alpha = 1.0) {
  const int total = M * N;
  // walk the unit-stride direction of the destination when there is one
  const bool rowfast = (dst.cs == 1);
  for (int e = threadIdx.x; e < total; e += TTB_THREADS) {
    int i, j;
    if (rowfast) { i = e / N; j = e % N; } else { i = e % M; j = e / M; }
    dst(i, j) = alpha * src(i, j);
  }
}

static __device__ __forceinline__ void cta_fill(Mat dst, int M, int N, double v) {
  const int total = M * N;
  for (int e = threadIdx.x; e < total; e += TTB_THREADS) {
    int i = e % M, j = e / M;
    dst(i, j) = v;
  }
}

// ---------------------------------------------------------------------------
// Householder QR
// ---------------------------------------------------------------------------

// In-place Householder QR of the m x k matrix W (column step ``ldw``, unit
// row step), as LAPACK dgeqr2 lays it out: on return R is in the upper
// triangle and the reflector vectors v_j (v_j[j] = 1 implied) below the
// diagonal, with the scalars in tau[0 .. min(m,k)-1].  Each reflector is
// H = I - tau v v^T built as in dlarfg: beta = -sign(alpha) ||x||,
// tau = (beta - alpha) / beta, v = x / (alpha - beta); a column whose
// sub-diagonal part is exactly zero gets tau = 0.
static __device__ void cta_householder(double* W, int m, int k, i64 ldw, double* tau, double* red) {
  // The whole block works on every reflector: the trailing columns are
  // taken HC at a time, their dot products with v accumulated per thread
  // over a row stripe and reduced together, and the squared norm of the
  // next column is gathered during its update (one pass fewer per column).
  constexpr int HC = 16;
  __shared__ double hred[TTB_WARPS][HC];
  __shared__ double hw[HC];
  const int p = m < k ? m : k;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double part = 0.0;
  for (int i = 1 + tid; i < m; i += TTB_THREADS) part = fma(W[i], W[i], part);
  double sigma = block_sum(part, red);
  for (int j = 0; j < p; ++j) {
    double* col = W + j * ldw;
    const double alpha = col[j];
    double t = 0.0, beta = alpha, scale = 0.0;
    if (sigma != 0.0) {
      const double nrm = sqrt(alpha * alpha + sigma);
      beta = (alpha >= 0.0) ? -nrm : nrm;
      t = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    __syncthreads();  // everyone has read col[j] before it is overwritten
    if (sigma != 0.0) {
      for (int i = j + 1 + tid; i < m; i += TTB_THREADS) col[i] *= scale;
    }
    if (tid == 0) {
      col[j] = beta;
      tau[j] = t;
    }
    __syncthreads();
    double next = 0.0;  // this thread's part of |column j+1, rows > j+1|^2
    for (int c0 = j + 1; c0 < k; c0 += HC) {
      const int nc = min(HC, k - c0);
      double* cb = W + (i64)c0 * ldw;
      if (t != 0.0) {
        double w[HC];
#pragma unroll
        for (int q = 0; q < HC; ++q) w[q] = 0.0;
        for (int i = j + 1 + tid; i < m; i += TTB_THREADS) {
          const double v = col[i];
#pragma unroll
          for (int q = 0; q < HC; ++q)
            if (q < nc) w[q] = fma(v, cb[i + q * ldw], w[q]);
        }
#pragma unroll
        for (int q = 0; q < HC; ++q) {
          const double sw = warp_sum(w[q]);
          if (lane == 0) hred[wid][q] = sw;
        }
        __syncthreads();
        if (tid < nc) {
          double sw = 0.0;
          for (int q = 0; q < TTB_WARPS; ++q) sw += hred[q][tid];
          const double wv = t * (sw + cb[j + tid * ldw]);
          hw[tid] = wv;
          cb[j + tid * ldw] -= wv;
        }
        __syncthreads();
        for (int i = j + 1 + tid; i < m; i += TTB_THREADS) {
          const double v = col[i];
#pragma unroll
          for (int q = 0; q < HC; ++q) {
            if (q < nc) {
              const double x = fma(-hw[q], v, cb[i + q * ldw]);
              cb[i + q * ldw] = x;
              if (q == 0 && c0 == j + 1 && i > j + 1) next = fma(x, x, next);
            }
          }
        }
        __syncthreads();  // hred and hw are reused by the next chunk
      } else if (c0 == j + 1) {
        for (int i = j + 2 + tid; i < m; i += TTB_THREADS) next = fma(cb[i], cb[i], next);
      }
    }
    if (j + 1 < p) sigma = block_sum(next, red);
  }
}

// Overwrite the m x q matrix X (strided) with H_0 H_1 ... H_{p-1} X, the
// reflectors of cta_householder (applied last to first).
static __device__ void cta_apply_q(const double* W, int m, int p, i64 ldw, const double* tau, Mat X,
                            int q) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int j = p - 1; j >= 0; --j) {
    const double t = tau[j];
    if (t != 0.0) {
      const double* v = W + j * ldw;
      for (int c = wid; c < q; c += TTB_WARPS) {
        double w = 0.0;
        for (int i = j + 1 + lane; i < m; i += 32) w = fma(v[i], X(i, c), w);
        w = warp_sum(w) + X(j, c);
        w *= t;
        if (lane == 0) X(j, c) -= w;
        for (int i = j + 1 + lane; i < m; i += 32) X(i, c) = fma(-w, v[i], X(i, c));
      }
    }
    __syncthreads();
  }
}

// Economic QR of the m x k matrix ``A`` (any strides): Q (m x p) and R
// (p x k), p = min(m, k).  ``W`` is an m x k column-major work area (unit
// row step, column step m), ``tau`` p doubles; both may be shared or
// global memory.  Q and R may be NULL to skip them.
static __device__ void cta_qr(CMat A, int m, int k, double* W, double* tau, Mat Q, Mat R, double* red) {
  const int p = m < k ? m : k;
  cta_copy(A, Mat{W, 1, (i64)m}, m, k);
  __syncthreads();
  cta_householder(W, m, k, m, tau, red);
  if (R.p) {
    for (int e = threadIdx.x; e < p * k; e += TTB_THREADS) {
      int i = e % p, j = e / p;
      R(i, j) = (i <= j) ? W[i + (i64)j * m] : 0.0;
    }
  }
  if (Q.p) {
    for (int e = threadIdx.x; e < m * p; e += TTB_THREADS) {
      int i = e % m, j = e / m;
      Q(i, j) = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    cta_apply_q(W, m, p, m, tau, Q, p);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// one-sided Jacobi SVD of a small square matrix
// ---------------------------------------------------------------------------

// Hestenes one-sided Jacobi on the columns of the k x k matrix B (column
// major, leading dimension ldb): finds an orthogonal V with B V having
// orthogonal columns.  On return B holds B V and V (column major, ldv) the
// accumulated rotations.  Pairs are visited in round-robin tournament order
// (k/2 disjoint pairs per round, one warp per pair).  A pair is rotated when
// |b_p . b_q| > tol sqrt(|b_p|^2 |b_q|^2); sweeps stop when one sweep
// rotates nothing, or after ``max_sweeps``.  Returns the sweeps used, or -1
// when the cap was hit.
static __device__ int cta_jacobi(double* B, int k, i64 ldb, double* V, i64 ldv, int max_sweeps,
                          double tol, int* flag) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < k * k; e += TTB_THREADS) {
    int i = e % k, j = e / k;
    V[i + j * ldv] = (i == j) ? 1.0 : 0.0;
  }
  if (k < 2) {
    __syncthreads();
    return 0;
  }
  const int kk = (k + 1) & ~1;  // players, one dummy when k is odd
  const int half = kk / 2;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    if (threadIdx.x == 0) *flag = 0;
    __syncthreads();
    int rotated = 0;
    for (int round = 0; round < kk - 1; ++round) {
      for (int pr = wid; pr < half; pr += TTB_WARPS) {
        int pa = (pr == 0) ? 0 : ((pr - 1 + round) % (kk - 1)) + 1;
        int pos = kk - 1 - pr;
        int pb = ((pos - 1 + round) % (kk - 1)) + 1;
        int p = pa < pb ? pa : pb, q = pa < pb ? pb : pa;
        if (q >= k) continue;  // paired with the dummy player
        double* bp = B + p * ldb;
        double* bq = B + q * ldb;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = lane; i < k; i += 32) {
          double x = bp[i], y = bq[i];
          al = fma(x, x, al);
          be = fma(y, y, be);
          ga = fma(x, y, ga);
        }
        al = warp_sum(al);
        be = warp_sum(be);
        ga = warp_sum(ga);
        if (ga != 0.0 && fabs(ga) > tol * sqrt(al) * sqrt(be)) {
          double zeta = (be - al) / (2.0 * ga);
          double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          double c = 1.0 / sqrt(1.0 + t * t);
          double s = c * t;
          for (int i = lane; i < k; i += 32) {
            double x = bp[i], y = bq[i];
            bp[i] = c * x - s * y;
            bq[i] = s * x + c * y;
          }
          double* vp = V + p * ldv;
          double* vq = V + q * ldv;
          for (int i = lane; i < k; i += 32) {
            double x = vp[i], y = vq[i];
            vp[i] = c * x - s * y;
            vq[i] = s * x + c * y;
          }
          rotated = 1;
        }
      }
      __syncthreads();
    }
    if (rotated) *flag = 1;  // benign race: every writer stores 1
    __syncthreads();
    int any = *flag;
    __syncthreads();
    if (!any) return sweep + 1;
  }
  return -1;
}

// Thin SVD of the m x k matrix A (any strides), m >= k required, as
// A = U diag(S) Vh with S descending: Householder QR A = Q R, one-sided
// Jacobi on R (R V = B, columns of B orthogonal), singular values the
// column norms of B, U = Q [B diag(1/S); 0].  Work areas (shared or global):
// W (m x k, column major), tau (k), Bsq (k x k), V (k x k), sv (k),
// order (k ints), flag (1 int).  U (m x k), S (k) and Vh (k x k) are
// strided outputs; U is also used as the work area of the final Q product.
// Returns the Jacobi sweeps used, or -1 if the sweep cap was hit.
static __device__ int cta_svd_tall(CMat A, int m, int k, double* W, double* tau, double* Bsq, double* V,
                            double* sv, int* order, int* flag, Mat U, double* S, Mat Vh,
                            double* red) {
  cta_copy(A, Mat{W, 1, (i64)m}, m, k);
  __syncthreads();
  cta_householder(W, m, k, m, tau, red);
  for (int e = threadIdx.x; e < k * k; e += TTB_THREADS) {
    int i = e % k, j = e / k;
    Bsq[i + (i64)j * k] = (i <= j) ? W[i + (i64)j * m] : 0.0;
  }
  __syncthreads();
  const double tol = 4.0 * k * 2.220446049250313e-16;
  int status = cta_jacobi(Bsq, k, k, V, k, 60, tol, flag);
  for (int j = threadIdx.x; j < k; j += TTB_THREADS) {
    double s = 0.0;
    for (int i = 0; i < k; ++i) s = fma(Bsq[i + (i64)j * k], Bsq[i + (i64)j * k], s);
    sv[j] = sqrt(s);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < k; j += TTB_THREADS) {
    double sj = sv[j];
    int rank = 0;
    for (int i = 0; i < k; ++i) {
      double si = sv[i];
      rank += (si > sj) || (si == sj && i < j);
    }
    order[rank] = j;
  }
  __syncthreads();
  // U <- [B(:, order) / S ; 0], S and Vh in descending order
  for (int e = threadIdx.x; e < m * k; e += TTB_THREADS) {
    int i = e % m, r = e / m;
    int j = order[r];
    double sj = sv[j];
    double v;
    if (i < k) v = (sj > 0.0) ? Bsq[i + (i64)j * k] / sj : (i == r ? 1.0 : 0.0);
    else v = 0.0;
    U(i, r) = v;
  }
  for (int r = threadIdx.x; r < k; r += TTB_THREADS) S[r] = sv[order[r]];
  for (int e = threadIdx.x; e < k * k; e += TTB_THREADS) {
    int r = e % k, c = e / k;
    Vh(r, c) = V[c + (i64)order[r] * k];
  }
  __syncthreads();
  cta_apply_q(W, m, k, m, tau, U, k);
  return status;
}

// Gaussian elimination with partial pivoting on [W | b] (LAPACK getrf/getrs
// semantics: largest |pivot|, first index on ties), W column major with
// leading dimension ld, then back substitution.  b is overwritten with the
// solution and W with the factors.  Returns 0, or the 1-based index of the
// first exactly-zero pivot (the solve then stops, like gesv's info > 0).
static __device__ int cta_gepp_solve(double* W, i64 ld, double* b, int n, double* redv, int* redi) {
  for (int j = 0; j < n; ++j) {
    double best = -1.0;
    int bi = -1;
    for (int i = j + threadIdx.x; i < n; i += TTB_THREADS) {
      double a = fabs(W[i + j * ld]);
      if (a > best) { best = a; bi = i; }
    }
    int piv = block_argmax_abs(best, bi, redv, redi);
    if (piv != j) {
      for (int c = j + threadIdx.x; c < n; c += TTB_THREADS) {
        double t = W[j + c * ld];
        W[j + c * ld] = W[piv + c * ld];
        W[piv + c * ld] = t;
      }
      if (threadIdx.x == 0) {
        double t = b[j];
        b[j] = b[piv];
        b[piv] = t;
      }
    }
    __syncthreads();
    const double d = W[j + j * ld];
    if (d == 0.0) return j + 1;
    const double rd = 1.0 / d;
    for (int i = j + 1 + threadIdx.x; i < n; i += TTB_THREADS) W[i + j * ld] *= rd;
    __syncthreads();
    const int rows = n - j - 1;
    const int total = rows * rows;
    for (int e = threadIdx.x; e < total; e += TTB_THREADS) {
      int i = j + 1 + e % rows, c = j + 1 + e / rows;
      W[i + c * ld] = fma(-W[i + j * ld], W[j + c * ld], W[i + c * ld]);
    }
    const double bj = b[j];
    for (int i = j + 1 + threadIdx.x; i < n; i += TTB_THREADS) b[i] = fma(-W[i + j * ld], bj, b[i]);
    __syncthreads();
  }
  for (int j = n - 1; j >= 0; --j) {
    if (threadIdx.x == 0) b[j] = b[j] / W[j + j * ld];
    __syncthreads();
    const double xj = b[j];
    for (int i = threadIdx.x; i < j; i += TTB_THREADS) b[i] = fma(-W[i + j * ld], xj, b[i]);
    __syncthreads();
  }
  return 0;
}

// ---------------------------------------------------------------------------
// blocked factorisations for matrices that do not fit in shared memory
// ---------------------------------------------------------------------------

constexpr int LNB = 16;   // panel width of the blocked factorisations
constexpr int YCH = 512;  // columns per chunk of the blocked trailing updates

// Blocked Gaussian elimination with partial pivoting on [W | b] (W column
// major, leading dimension ld), panels of LNB columns factored in ``panel``
// (rows x LNB doubles, shared or global memory), trailing updates as GEMMs.
// Same pivot rule and result as cta_gepp_solve; b becomes the solution.
static __device__ int cta_gepp_blocked(double* W, i64 ld, double* b, int n, double* panel, double* redv,
                                int* redi, int* ipiv, GemmSmem& gsm, double* ring = nullptr) {
  const int tid = threadIdx.x;
  for (int j0 = 0; j0 < n; j0 += LNB) {
    const int jb = min(LNB, n - j0);
    const int rows = n - j0;
    double* P = panel;
    for (int e = tid; e < rows * jb; e += TTB_THREADS) {
      int i = e % rows, c = e / rows;
      P[i + (i64)c * rows] = W[(j0 + i) + (i64)(j0 + c) * ld];
    }
    __syncthreads();
    for (int c = 0; c < jb; ++c) {
      double best = -1.0;
      int bi = -1;
      for (int i = c + tid; i < rows; i += TTB_THREADS) {
        double a = fabs(P[i + (i64)c * rows]);
        if (a > best) { best = a; bi = i; }
      }
      const int piv = block_argmax_abs(best, bi, redv, redi);
      if (tid == 0) ipiv[c] = piv;
      if (piv != c) {
        for (int cc = tid; cc < jb; cc += TTB_THREADS) {
          double t = P[c + (i64)cc * rows];
          P[c + (i64)cc * rows] = P[piv + (i64)cc * rows];
          P[piv + (i64)cc * rows] = t;
        }
      }
      __syncthreads();
      const double d = P[c + (i64)c * rows];
      if (d == 0.0) return j0 + c + 1;
      const double rd = 1.0 / d;
      for (int i = c + 1 + tid; i < rows; i += TTB_THREADS) P[i + (i64)c * rows] *= rd;
      __syncthreads();
      const int rr = rows - c - 1, cw = jb - c - 1;
      for (int e = tid; e < rr * cw; e += TTB_THREADS) {
        int i = c + 1 + e % rr, cc = c + 1 + e / rr;
        P[i + (i64)cc * rows] = fma(-P[i + (i64)c * rows], P[c + (i64)cc * rows],
                                    P[i + (i64)cc * rows]);
      }
      __syncthreads();
    }
    for (int e = tid; e < rows * jb; e += TTB_THREADS) {
      int i = e % rows, c = e / rows;
      W[(j0 + i) + (i64)(j0 + c) * ld] = P[i + (i64)c * rows];
    }
    // row swaps and the unit-lower solve on the columns right of the panel
    // and on b; each thread owns whole columns, so no synchronisation
    const int ncols = n - j0 - jb;
    for (int col = tid; col <= ncols; col += TTB_THREADS) {
      double* x = (col < ncols) ? W + (i64)(j0 + jb + col) * ld + j0 : b + j0;
      for (int c = 0; c < jb; ++c) {
        const int piv = ipiv[c];
        if (piv != c) {
          double t = x[c];
          x[c] = x[piv];
          x[piv] = t;
        }
      }
      for (int r = 1; r < jb; ++r) {
        double acc = x[r];
        for (int q = 0; q < r; ++q) acc = fma(-P[r + (i64)q * rows], x[q], acc);
        x[r] = acc;
      }
    }
    __syncthreads();
    if (rows > jb) {
      // A22 -= L21 U12 ; b2 -= L21 u_b
      if (ncols > 0)
        gemm_sel(CMat{P + jb, 1, rows}, CMat{W + j0 + (i64)(j0 + jb) * ld, 1, ld},
                 Mat{W + (j0 + jb) + (i64)(j0 + jb) * ld, 1, ld}, rows - jb, ncols, jb, -1.0,
                 1.0, gsm, ring);
      for (int i = tid; i < rows - jb; i += TTB_THREADS) {
        double acc = b[j0 + jb + i];
        for (int q = 0; q < jb; ++q) acc = fma(-P[jb + i + (i64)q * rows], b[j0 + q], acc);
        b[j0 + jb + i] = acc;
      }
    }
    __syncthreads();
  }
  for (int j = n - 1; j >= 0; --j) {
    if (tid == 0) b[j] = b[j] / W[j + (i64)j * ld];
    __syncthreads();
    const double xj = b[j];
    for (int i = tid; i < j; i += TTB_THREADS) b[i] = fma(-W[i + (i64)j * ld], xj, b[i]);
    __syncthreads();
  }
  return 0;
}

// T factor (jb x jb, upper triangular, column major in Tm) of the block
// reflector H_0 ... H_{jb-1} = I - V T V^T, V the rows x jb explicit
// reflector block (unit diagonal, zeros above) in Wp with leading dim ldw
// (LAPACK dlarft, forward column-wise).  G is jb x jb scratch.
static __device__ void cta_block_t(const double* Wp, i64 ldw, int rows, int jb, const double* tau,
                            double* G, double* Tm, GemmSmem& gsm, double* ring = nullptr) {
  gemm_sel(CMat{Wp, ldw, 1}, CMat{Wp, 1, ldw}, Mat{G, 1, LNB}, jb, jb, rows, 1.0, 0.0, gsm, ring);
  if (threadIdx.x == 0) {
    for (int i = 0; i < jb; ++i) {
      for (int q = 0; q < i; ++q) {
        double acc = 0.0;
        for (int r = q; r < i; ++r) acc = fma(Tm[q + r * LNB], G[r + i * LNB], acc);
        Tm[q + i * LNB] = -tau[i] * acc;
      }
      Tm[i + i * LNB] = tau[i];
      for (int q = i + 1; q < LNB; ++q) Tm[q + i * LNB] = 0.0;
    }
  }
  __syncthreads();
}

// X (m x nx, strided) <- H_0 ... H_{p-1} X for the block reflectors left in
// W by cta_qr_blocked (explicit reflector blocks, leading dimension m),
// applied last block first; only rows >= the block's first row change.
// Columns of X left of a block are untouched (as for an identity start).
static __device__ void cta_apply_q_blocked(const double* W, int m, int p, const double* tau, Mat X,
                                    int nx, double* Y, double* G, double* Tm, GemmSmem& gsm, double* ring = nullptr) {
  const int tid = threadIdx.x;
  const int last = ((p - 1) / LNB) * LNB;
  for (int j0 = last; j0 >= 0; j0 -= LNB) {
    const int jb = min(LNB, p - j0);
    const int rows = m - j0;
    const double* Wp = W + j0 + (i64)j0 * m;
    cta_block_t(Wp, m, rows, jb, tau + j0, G, Tm, gsm, ring);
    for (int c0 = 0; c0 < nx; c0 += YCH) {
      const int nc = min(YCH, nx - c0);
      Mat Xs{X.p + j0 * X.rs + c0 * X.cs, X.rs, X.cs};
      gemm_sel(CMat{Wp, m, 1}, CMat{Xs.p, Xs.rs, Xs.cs}, Mat{Y, 1, LNB}, jb, nc, rows, 1.0, 0.0,
               gsm, ring);
      for (int col = tid; col < nc; col += TTB_THREADS) {
        double y[LNB];
        for (int i = 0; i < jb; ++i) y[i] = Y[i + (i64)col * LNB];
        for (int i = 0; i < jb; ++i) {
          double acc = 0.0;
          for (int q = i; q < jb; ++q) acc = fma(Tm[i + q * LNB], y[q], acc);
          Y[i + (i64)col * LNB] = acc;
        }
      }
      __syncthreads();
      gemm_sel(CMat{Wp, 1, m}, CMat{Y, 1, LNB}, Xs, rows, nc, jb, -1.0, 1.0, gsm, ring);
    }
  }
}

// Blocked (compact WY) economic QR of the m x k matrix A into the m x k
// column-major work area W (global), panels of LNB columns: Householder on
// the panel (cta_householder), the T factor, then the trailing update
// C -= V (T^T (V^T C)) as two GEMMs through Y (LNB x k, shared).  Q (m x p)
// and R (p x k) as in cta_qr; either may be NULL.  Same reflectors and R as
// the unblocked factorisation up to rounding.
static __device__ void cta_qr_blocked(CMat A, int m, int k, double* W, double* tau, Mat Q, Mat R,
                               double* Y, double* G, double* Tm, double* red, GemmSmem& gsm, double* ring = nullptr) {
  const int p = m < k ? m : k;
  const int tid = threadIdx.x;
  cta_copy(A, Mat{W, 1, (i64)m}, m, k);
  __syncthreads();
  for (int j0 = 0; j0 < p; j0 += LNB) {
    const int jb = min(LNB, p - j0);
    const int rows = m - j0;
    double* Wp = W + j0 + (i64)j0 * m;
    cta_householder(Wp, rows, jb, m, tau + j0, red);
    // R's diagonal block, then the explicit reflector form in its place
    for (int e = tid; e < jb * jb; e += TTB_THREADS) {
      int r = e % jb, c = e / jb;
      if (r <= c) {
        if (R.p) R(j0 + r, j0 + c) = Wp[r + (i64)c * m];
        Wp[r + (i64)c * m] = (r == c) ? 1.0 : 0.0;
      }
    }
    __syncthreads();
    const int nt = k - j0 - jb;
    if (nt > 0) {
      cta_block_t(Wp, m, rows, jb, tau + j0, G, Tm, gsm, ring);
      for (int c0 = 0; c0 < nt; c0 += YCH) {
        const int nc = min(YCH, nt - c0);
        double* C = W + j0 + (i64)(j0 + jb + c0) * m;
        // Y = V^T C (jb x nc), then Y = T^T Y, then C -= V Y
        gemm_sel(CMat{Wp, m, 1}, CMat{C, 1, m}, Mat{Y, 1, LNB}, jb, nc, rows, 1.0, 0.0, gsm, ring);
        for (int col = tid; col < nc; col += TTB_THREADS) {
          double y[LNB];
          for (int i = 0; i < jb; ++i) y[i] = Y[i + (i64)col * LNB];
          for (int i = jb - 1; i >= 0; --i) {
            double acc = 0.0;
            for (int q = 0; q <= i; ++q) acc = fma(Tm[q + i * LNB], y[q], acc);
            Y[i + (i64)col * LNB] = acc;
          }
        }
        __syncthreads();
        gemm_sel(CMat{Wp, 1, m}, CMat{Y, 1, LNB}, Mat{C, 1, m}, rows, nc, jb, -1.0, 1.0, gsm, ring);
      }
    }
  }
  if (R.p) {
    for (int e = tid; e < p * k; e += TTB_THREADS) {
      int i = e % p, j = e / p;
      int jp = (i / LNB) * LNB;  // panel of row i
      bool in_diag_block = (j >= jp && j < jp + LNB && j < p);
      if (i > j) R(i, j) = 0.0;
      else if (!in_diag_block) R(i, j) = W[i + (i64)j * m];
    }
  }
  if (Q.p) {
    for (int e = tid; e < m * p; e += TTB_THREADS) {
      int i = e % m, j = e / m;
      Q(i, j) = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    cta_apply_q_blocked(W, m, p, tau, Q, p, Y, G, Tm, gsm, ring);
  }
  __syncthreads();
}

// R factor only of the economic QR of the m x k view A, two-level blocked
// for tall operands: outer panels of LNB2 columns are factorised by the
// LNB-blocked Householder code (trailing updates inside the panel only),
// then the panel's LNB2 reflectors update the rest of the matrix as one
// compact-WY block, C -= V (T^T (V^T C)), whose products have 64-wide tiles
// and long K.  Same reflectors as cta_qr_blocked.  W (m x k column major)
// and tau (min(m, k)) are global work; ``pool`` (shared) holds
// 2 LNB2^2 + LNB2^2 + LNB * LNB2 + 2 LNB^2 doubles.
constexpr int LNB2 = 64;
static __device__ __noinline__ void cta_qr_r_blocked2(CMat A, int m, int k, double* W, double* tau,
                                                      Mat R, double* pool, double* red,
                                                      double* ring) {
  const int p = m < k ? m : k;
  const int tid = threadIdx.x;
  double* G2 = pool;                      // LNB2 x LNB2: V^T V, later T^T Y
  double* T2 = G2 + LNB2 * LNB2;          // LNB2 x LNB2 upper triangular
  double* Yo = T2 + LNB2 * LNB2;          // LNB2 x LNB2 chunk of V^T C
  double* Yi = Yo + LNB2 * LNB2;          // LNB x LNB2 (inner updates)
  double* Gi = Yi + LNB * LNB2;
  double* Ti = Gi + LNB * LNB;
  cta_copy(A, Mat{W, 1, (i64)m}, m, k);
  __syncthreads();
  for (int o0 = 0; o0 < p; o0 += LNB2) {
    const int ob = min(LNB2, p - o0);
    const int orows = m - o0;
    double* Wo = W + o0 + (i64)o0 * m;
    // inner LNB-blocked factorisation of the panel's ob columns
    for (int j0 = o0; j0 < o0 + ob; j0 += LNB) {
      const int jb = min(LNB, o0 + ob - j0);
      const int rows = m - j0;
      double* Wp = W + j0 + (i64)j0 * m;
      cta_householder(Wp, rows, jb, m, tau + j0, red);
      for (int e = tid; e < jb * jb; e += TTB_THREADS) {
        int r = e % jb, c = e / jb;
        if (r <= c) {
          R(j0 + r, j0 + c) = Wp[r + (i64)c * m];
          Wp[r + (i64)c * m] = (r == c) ? 1.0 : 0.0;
        }
      }
      __syncthreads();
      const int nt = o0 + ob - j0 - jb;
      if (nt > 0) {
        // T of the block (as cta_block_t), column by column over the block
        cta_gemm_pipe(CMat{Wp, m, 1}, CMat{Wp, 1, m}, Mat{Gi, 1, LNB}, jb, jb, rows, 1.0, 0.0,
                      ring);
        for (int e = tid; e < LNB * LNB; e += TTB_THREADS) Ti[e] = 0.0;
        __syncthreads();
        for (int i = 0; i < jb; ++i) {
          if (tid < i) {
            double acc = 0.0;
            for (int r = tid; r < i; ++r) acc = fma(Ti[tid + r * LNB], Gi[r + i * LNB], acc);
            Ti[tid + i * LNB] = -tau[j0 + i] * acc;
          }
          if (tid == 0) Ti[i + i * LNB] = tau[j0 + i];
          __syncthreads();
        }
        double* C = W + j0 + (i64)(j0 + jb) * m;
        cta_gemm_pipe(CMat{Wp, m, 1}, CMat{C, 1, m}, Mat{Yi, 1, LNB}, jb, nt, rows, 1.0, 0.0,
                      ring);
        for (int col = tid; col < nt; col += TTB_THREADS) {
          double y[LNB];
          for (int i = 0; i < jb; ++i) y[i] = Yi[i + (i64)col * LNB];
          for (int i = jb - 1; i >= 0; --i) {
            double acc = 0.0;
            for (int q = 0; q <= i; ++q) acc = fma(Ti[q + i * LNB], y[q], acc);
            Yi[i + (i64)col * LNB] = acc;
          }
        }
        __syncthreads();
        cta_gemm_pipe(CMat{Wp, 1, m}, CMat{Yi, 1, LNB}, Mat{C, 1, m}, rows, nt, jb, -1.0, 1.0,
                      ring);
      }
    }
    // R entries above the inner diagonal blocks move out; V gets zeros there
    for (int e = tid; e < ob * ob; e += TTB_THREADS) {
      int r = e % ob, c = e / ob;
      if (r < c && (r / LNB) != (c / LNB)) {
        R(o0 + r, o0 + c) = Wo[r + (i64)c * m];
        Wo[r + (i64)c * m] = 0.0;
      }
    }
    __syncthreads();
    const int nt = k - o0 - ob;
    if (nt <= 0) continue;
    // T of the panel: T[i, i] = tau_i, T[0:i, i] = -tau_i T[0:i, 0:i] (V^T V)[0:i, i]
    cta_gemm_pipe(CMat{Wo, m, 1}, CMat{Wo, 1, m}, Mat{G2, 1, LNB2}, ob, ob, orows, 1.0, 0.0, ring);
    for (int e = tid; e < LNB2 * LNB2; e += TTB_THREADS) T2[e] = 0.0;
    __syncthreads();
    for (int i = 0; i < ob; ++i) {
      const double ti = tau[o0 + i];
      for (int q = tid; q < i; q += TTB_THREADS) {
        double acc = 0.0;
        for (int r = q; r < i; ++r) acc = fma(T2[q + r * LNB2], G2[r + i * LNB2], acc);
        T2[q + i * LNB2] = -ti * acc;
      }
      if (tid == 0) T2[i + i * LNB2] = ti;
      __syncthreads();
    }
    for (int c0 = 0; c0 < nt; c0 += LNB2) {
      const int nc = min(LNB2, nt - c0);
      double* C = W + o0 + (i64)(o0 + ob + c0) * m;
      // Yo = V^T C, G2 = T^T Yo, C -= V G2
      cta_gemm_pipe(CMat{Wo, m, 1}, CMat{C, 1, m}, Mat{Yo, 1, LNB2}, ob, nc, orows, 1.0, 0.0, ring);
      cta_gemm_pipe(CMat{T2, LNB2, 1}, CMat{Yo, 1, LNB2}, Mat{G2, 1, LNB2}, ob, nc, ob, 1.0, 0.0,
                    ring);
      cta_gemm_pipe(CMat{Wo, 1, m}, CMat{G2, 1, LNB2}, Mat{C, 1, m}, orows, nc, ob, -1.0, 1.0,
                    ring);
    }
  }
  // the rest of R: below the diagonal zero, right of each outer panel from W
  for (int e = tid; e < p * k; e += TTB_THREADS) {
    int i = e % p, j = e / p;
    if (i > j) {
      R(i, j) = 0.0;
    } else if (j >= min((i / LNB2) * LNB2 + LNB2, p)) {
      R(i, j) = W[i + (i64)j * m];
    }
  }
  __syncthreads();
}

// cta_svd_tall for matrices that do not fit in shared memory: blocked QR
// into the global work area W, Jacobi on R in Bsq/V (global or shared), U
// by the blocked reflector product.  Y needs LNB * max(k, 1) doubles, G and
// Tm LNB * LNB each (shared).
static __device__ int cta_svd_tall_blocked(CMat A, int m, int k, double* W, double* tau, double* Bsq,
                                    double* V, double* sv, int* order, int* flag, Mat U, double* S,
                                    Mat Vh, double* Y, double* G, double* Tm, double* red,
                                    GemmSmem& gsm, double* ring = nullptr) {
  cta_qr_blocked(A, m, k, W, tau, Mat{nullptr, 0, 0}, Mat{Bsq, 1, (i64)k}, Y, G, Tm, red, gsm, ring);
  __syncthreads();
  const double tol = 4.0 * k * 2.220446049250313e-16;
  int status = cta_jacobi(Bsq, k, k, V, k, 60, tol, flag);
  for (int j = threadIdx.x; j < k; j += TTB_THREADS) {
    double s2 = 0.0;
    for (int i = 0; i < k; ++i) s2 = fma(Bsq[i + (i64)j * k], Bsq[i + (i64)j * k], s2);
    sv[j] = sqrt(s2);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < k; j += TTB_THREADS) {
    double sj = sv[j];
    int rank = 0;
    for (int i = 0; i < k; ++i) {
      double si = sv[i];
      rank += (si > sj) || (si == sj && i < j);
    }
    order[rank] = j;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < m * k; e += TTB_THREADS) {
    int i = e % m, r = e / m;
    int j = order[r];
    double sj = sv[j];
    double v;
    if (i < k) v = (sj > 0.0) ? Bsq[i + (i64)j * k] / sj : (i == r ? 1.0 : 0.0);
    else v = 0.0;
    U(i, r) = v;
  }
  for (int r = threadIdx.x; r < k; r += TTB_THREADS) S[r] = sv[order[r]];
  for (int e = threadIdx.x; e < k * k; e += TTB_THREADS) {
    int r = e % k, c = e / k;
    Vh(r, c) = V[c + (i64)order[r] * k];
  }
  __syncthreads();
  cta_apply_q_blocked(W, m, k, tau, U, k, Y, G, Tm, gsm, ring);
  return status;
}

}  // namespace ttb
