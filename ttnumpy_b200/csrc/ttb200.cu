// libttb200: grouped float64 kernels and the C ABI of include/ttb200.h.
//
// Every entry point takes a host array of problems, packs them into
// by-value launch descriptors (no device allocation, no host-device copy of
// descriptors) and issues grouped launches on the caller's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cfloat>
#include <cstring>
#include <vector>

#include "ttb200.h"
#include "ttb_device.cuh"

using namespace ttb;

namespace {

std::atomic<long long> g_launches{0};
inline void counted() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ---------------------------------------------------------------------------
// optional per-kernel-class timing with CUDA events (ttb_profile_*)
// ---------------------------------------------------------------------------

enum { P_GEMM = 0, P_COPY, P_KRON, P_NORM, P_LOCALMAT, P_QR, P_SVD, P_LU, P_RANK, P_MINRES,
       P_GMRES, P_ROUND, P_CLASSES };

struct ProfRec {
  cudaEvent_t a, b;
  int cls;
  double flops, bytes;
};

std::atomic<int> g_prof_mask{0};
std::vector<ProfRec> g_prof;
std::vector<cudaEvent_t> g_event_pool;
double g_prof_ms[P_CLASSES], g_prof_flops[P_CLASSES], g_prof_bytes[P_CLASSES];
long long g_prof_n[P_CLASSES];

cudaEvent_t pool_event() {
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// Brackets one launch of class ``cls`` when that class is being profiled.
struct ProfScope {
  bool on;
  ProfRec r;
  cudaStream_t s;
  ProfScope(int cls, cudaStream_t st, double flops, double bytes) : on(false), s(st) {
    if (!(g_prof_mask.load(std::memory_order_relaxed) & (1 << cls))) return;
    on = true;
    r.cls = cls;
    r.flops = flops;
    r.bytes = bytes;
    r.a = pool_event();
    r.b = pool_event();
    cudaEventRecord(r.a, s);
  }
  ~ProfScope() {
    if (!on) return;
    cudaEventRecord(r.b, s);
    g_prof.push_back(r);
  }
};

void prof_collect() {
  for (auto& r : g_prof) {
    float ms = 0.f;
    cudaEventSynchronize(r.b);
    cudaEventElapsedTime(&ms, r.a, r.b);
    g_prof_ms[r.cls] += ms;
    g_prof_n[r.cls] += 1;
    g_prof_flops[r.cls] += r.flops;
    g_prof_bytes[r.cls] += r.bytes;
    g_event_pool.push_back(r.a);
    g_event_pool.push_back(r.b);
  }
  g_prof.clear();
}

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

inline int last_error() {
  cudaError_t e = cudaGetLastError();
  return (int)e;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// shared memory the one-CTA factorisations may use (B200: 227 KB per block)
constexpr int kSmemCap = 200 * 1024;

int g_smem_qr[kMaxDevices], g_smem_svd[kMaxDevices], g_smem_lu[kMaxDevices],
    g_smem_round[kMaxDevices];

// ---------------------------------------------------------------------------
// grouped GEMM
// ---------------------------------------------------------------------------

struct GDesc {
  const double* a;
  const double* b;
  double* c;
  int m, n, k, batch;
  i64 a_rs, a_cs, a_bs, b_rs, b_cs, b_bs, c_rs, c_cs, c_bs;
  double alpha, beta;
  int tm, tn;
};

constexpr int kMaxG = 48;
struct GBatch {
  int count;
  int base[kMaxG + 1];
  GDesc d[kMaxG];
};

__global__ void __launch_bounds__(TTB_THREADS) k_gemm(const __grid_constant__ GBatch gb) {
  __shared__ GemmSmem sm;
  const int t = blockIdx.x;
  int p = 0;
  while (p + 1 < gb.count && gb.base[p + 1] <= t) ++p;
  const GDesc& g = gb.d[p];
  const int local = t - gb.base[p];
  const int per = g.tm * g.tn;
  const int bi = local / per, r = local % per;
  const int m0 = (r / g.tn) * GBM, n0 = (r % g.tn) * GBN;
  CMat A{g.a + bi * g.a_bs, g.a_rs, g.a_cs};
  CMat B{g.b + bi * g.b_bs, g.b_rs, g.b_cs};
  Mat C{g.c + bi * g.c_bs, g.c_rs, g.c_cs};
  cta_gemm_tile(A, B, C, g.m, g.n, g.k, m0, n0, g.alpha, g.beta, sm);
}

GDesc make_gemm(const double* a, i64 a_rs, i64 a_cs, i64 a_bs, const double* b, i64 b_rs,
                i64 b_cs, i64 b_bs, double* c, i64 c_rs, i64 c_cs, i64 c_bs, int m, int n, int k,
                int batch, double alpha, double beta) {
  GDesc d;
  d.a = a; d.b = b; d.c = c;
  d.m = m; d.n = n; d.k = k; d.batch = batch;
  d.a_rs = a_rs; d.a_cs = a_cs; d.a_bs = a_bs;
  d.b_rs = b_rs; d.b_cs = b_cs; d.b_bs = b_bs;
  d.c_rs = c_rs; d.c_cs = c_cs; d.c_bs = c_bs;
  d.alpha = alpha; d.beta = beta;
  d.tm = d.tn = 0;
  return d;
}

int launch_gemms(const std::vector<GDesc>& ds, cudaStream_t s) {
  size_t i = 0;
  while (i < ds.size()) {
    GBatch gb;
    gb.count = 0;
    long long tiles = 0;
    while (i < ds.size() && gb.count < kMaxG) {
      GDesc d = ds[i++];
      if (d.m <= 0 || d.n <= 0 || d.batch <= 0) continue;
      d.tm = cdiv(d.m, GBM);
      d.tn = cdiv(d.n, GBN);
      gb.base[gb.count] = (int)tiles;
      gb.d[gb.count++] = d;
      tiles += (long long)d.tm * d.tn * d.batch;
    }
    if (gb.count == 0) continue;
    gb.base[gb.count] = (int)tiles;
    double fl = 0.0, by = 0.0;
    if (g_prof_mask.load(std::memory_order_relaxed) & (1 << P_GEMM)) {
      for (int j = 0; j < gb.count; ++j) {
        const GDesc& g = gb.d[j];
        fl += 2.0 * g.m * g.n * (double)g.k * g.batch;
        const double na = g.a_bs ? g.batch : 1, nb = g.b_bs ? g.batch : 1;
        by += 8.0 * ((double)g.m * g.k * na + (double)g.k * g.n * nb + 2.0 * g.m * g.n * g.batch);
      }
    }
    ProfScope ps(P_GEMM, s, fl, by);
    k_gemm<<<(unsigned)tiles, TTB_THREADS, 0, s>>>(gb);
    counted();
  }
  return last_error();
}

// ---------------------------------------------------------------------------
// strided copy, Kronecker cores, norms
// ---------------------------------------------------------------------------

constexpr int kMaxC = 32;
struct CBatch {
  int count;
  ttb_copy_t d[kMaxC];
};

__global__ void __launch_bounds__(TTB_THREADS) k_copy(const __grid_constant__ CBatch cb) {
  const ttb_copy_t& c = cb.d[blockIdx.y];
  const i64 total = (i64)c.d0 * c.d1 * c.d2 * c.d3;
  for (i64 e = (i64)blockIdx.x * TTB_THREADS + threadIdx.x; e < total;
       e += (i64)gridDim.x * TTB_THREADS) {
    i64 r = e;
    int i3 = (int)(r % c.d3); r /= c.d3;
    int i2 = (int)(r % c.d2); r /= c.d2;
    int i1 = (int)(r % c.d1); r /= c.d1;
    int i0 = (int)r;
    double v = c.alpha;
    if (c.scale) {
      const int ia = c.scale_axis == 0 ? i0 : c.scale_axis == 1 ? i1 : c.scale_axis == 2 ? i2 : i3;
      v *= c.scale[ia];
    }
    if (c.src) v *= c.src[i0 * c.s0 + i1 * c.s1 + i2 * c.s2 + i3 * c.s3];
    c.dst[i0 * c.t0 + i1 * c.t1 + i2 * c.t2 + i3 * c.t3] = v;
  }
}

constexpr int kMaxK = 32;
struct KBatch {
  int count;
  ttb_kron_t d[kMaxK];
};

__global__ void __launch_bounds__(TTB_THREADS) k_kron(const __grid_constant__ KBatch kb) {
  const ttb_kron_t& q = kb.d[blockIdx.y];
  const i64 rows = (i64)q.ra * q.rx, cols = (i64)q.ra2 * q.rx2;
  const i64 total = rows * q.n * q.kk * cols;
  for (i64 e = (i64)blockIdx.x * TTB_THREADS + threadIdx.x; e < total;
       e += (i64)gridDim.x * TTB_THREADS) {
    i64 r = e;
    int y = (int)(r % q.rx2); r /= q.rx2;
    int b = (int)(r % q.ra2); r /= q.ra2;
    int kk = (int)(r % q.kk); r /= q.kk;
    int i = (int)(r % q.n); r /= q.n;
    int x = (int)(r % q.rx); r /= q.rx;
    int a = (int)r;
    const double* op = q.op + (((i64)a * q.n + i) * q.m) * q.ra2 + b;  // op[a, i, j, b]
    const double* cr = q.core + ((i64)x * q.m) * q.kk * q.rx2 + (i64)kk * q.rx2 + y;
    double s = 0.0;
    for (int j = 0; j < q.m; ++j) s = fma(op[(i64)j * q.ra2], cr[(i64)j * q.kk * q.rx2], s);
    q.out[e] = s;
  }
}

struct HBatch {
  int count;
  ttb_hadamard_t d[kMaxK];
};

// One output element per thread and step, written in order (coalesced
// stores); the two factors' entries are re-read from L1/L2.
__global__ void __launch_bounds__(TTB_THREADS) k_hadamard(const __grid_constant__ HBatch hb) {
  const ttb_hadamard_t& q = hb.d[blockIdx.y];
  const i64 total = (i64)q.ra * q.rx * q.modes * q.ra2 * q.rx2;
  for (i64 e = (i64)blockIdx.x * TTB_THREADS + threadIdx.x; e < total;
       e += (i64)gridDim.x * TTB_THREADS) {
    i64 r = e;
    int y = (int)(r % q.rx2); r /= q.rx2;
    int b = (int)(r % q.ra2); r /= q.ra2;
    int p = (int)(r % q.modes); r /= q.modes;
    int x = (int)(r % q.rx); r /= q.rx;
    int a = (int)r;
    q.out[e] = q.lhs[((i64)a * q.modes + p) * q.ra2 + b] * q.rhs[((i64)x * q.modes + p) * q.rx2 + y];
  }
}

constexpr int kMaxN = 64;
struct NBatch {
  int count;
  ttb_norm_t d[kMaxN];
};

__global__ void __launch_bounds__(TTB_THREADS) k_norm(const __grid_constant__ NBatch nb) {
  __shared__ double red[TTB_WARPS];
  const ttb_norm_t& q = nb.d[blockIdx.x];
  double s = 0.0;
  if (q.y) {
    for (i64 i = threadIdx.x; i < q.n; i += TTB_THREADS) {
      double v = q.x[i] - q.y[i];
      s = fma(v, v, s);
    }
  } else {
    for (i64 i = threadIdx.x; i < q.n; i += TTB_THREADS) s = fma(q.x[i], q.x[i], s);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) q.out[0] = sqrt(s);
}

// ---------------------------------------------------------------------------
// explicit local matrix
// ---------------------------------------------------------------------------

constexpr int kMaxLM = 16;
struct LMBatch {
  int count;
  ttb_local_matrix_t d[kMaxLM];
};

__global__ void __launch_bounds__(TTB_THREADS) k_local_matrix(const __grid_constant__ LMBatch lb) {
  const ttb_local_matrix_t& q = lb.d[blockIdx.y];
  const i64 rows = (i64)q.lf * q.n * q.rf, cols = (i64)q.lt * q.m * q.rt;
  const i64 total = rows * cols;
  for (i64 e = (i64)blockIdx.x * TTB_THREADS + threadIdx.x; e < total;
       e += (i64)gridDim.x * TTB_THREADS) {
    i64 row = e % rows, col = e / rows;
    int nf = (int)(row % q.rf);
    int kr = (int)((row / q.rf) % q.n);
    int j = (int)(row / ((i64)q.rf * q.n));
    int mt = (int)(col % q.rt);
    int l = (int)((col / q.rt) % q.m);
    int i = (int)(col / ((i64)q.rt * q.m));
    double s = 0.0;
    for (int a = 0; a < q.R; ++a) {
      const double la = q.left[((i64)i * q.R + a) * q.lf + j];
      if (la == 0.0) continue;
      const double* op = q.op + (((i64)a * q.n + kr) * q.m + l) * q.R2;
      double t = 0.0;
      for (int b = 0; b < q.R2; ++b) t = fma(op[b], q.right[((i64)mt * q.R2 + b) * q.rf + nf], t);
      s = fma(la, t, s);
    }
    q.out[e] = s;
  }
}

// ---------------------------------------------------------------------------
// QR, SVD, LU: one thread block per problem
// ---------------------------------------------------------------------------

constexpr int kMaxQ = 24;
struct QBatch {
  int count;
  int mode[kMaxQ];  // 0: whole factorisation in shared memory, 1: blocked (work in global)
  ttb_qr_t d[kMaxQ];
};

__global__ void __launch_bounds__(TTB_THREADS) k_qr(const __grid_constant__ QBatch qb) {
  extern __shared__ double dsm[];
  __shared__ double red[TTB_WARPS];
  __shared__ GemmSmem gsm;
  const ttb_qr_t& q = qb.d[blockIdx.x];
  const int m = q.m, k = q.k;
  if (m <= 0 || k <= 0) return;
  if (qb.mode[blockIdx.x] == 0) {
    double* W = dsm;
    double* tau = W + (i64)m * k;
    cta_qr(CMat{q.a, q.a_rs, q.a_cs}, m, k, W, tau, Mat{q.q, q.q_rs, q.q_cs},
           Mat{q.r, q.r_rs, q.r_cs}, red);
  } else {
    double* Y = dsm;
    double* G = Y + (i64)LNB * min(k, YCH);
    double* Tm = G + LNB * LNB;
    cta_qr_blocked(CMat{q.a, q.a_rs, q.a_cs}, m, k, q.work, q.work + (i64)m * k,
                   Mat{q.q, q.q_rs, q.q_cs}, Mat{q.r, q.r_rs, q.r_cs}, Y, G, Tm, red, gsm);
  }
}

i64 qr_need(int m, int k) { return (i64)m * k + std::min(m, k); }
i64 blocked_smem(int k) { return (i64)LNB * std::min(std::max(k, 1), YCH) + 2 * LNB * LNB; }

constexpr int kMaxS = 16;
struct SBatch {
  int count;
  int mode[kMaxS];  // 0: shared memory, 1: blocked with the work area in global memory
  ttb_svd_t d[kMaxS];
};

// doubles of the tall SVD work area for an M x K (M >= K) problem
i64 svd_tall_need(int M, int K) { return (i64)M * K + 2 * (i64)K * K + 3 * (i64)K + 2; }

__global__ void __launch_bounds__(TTB_THREADS) k_svd(const __grid_constant__ SBatch sb) {
  extern __shared__ double dsm[];
  __shared__ double red[TTB_WARPS];
  __shared__ GemmSmem gsm;
  const ttb_svd_t& q = sb.d[blockIdx.x];
  if (q.m <= 0 || q.k <= 0) return;
  const bool tall = q.m >= q.k;
  const int M = tall ? q.m : q.k, K = tall ? q.k : q.m;
  const int mode = sb.mode[blockIdx.x];
  double* base = mode == 0 ? dsm : q.work;
  double* W = base;
  double* tau = W + (i64)M * K;
  double* Bsq = tau + K;
  double* V = Bsq + (i64)K * K;
  double* sv = V + (i64)K * K;
  int* order = reinterpret_cast<int*>(sv + K);
  int* flag = reinterpret_cast<int*>(sv + 2 * K);
  CMat A = tall ? CMat{q.a, q.a_rs, q.a_cs} : CMat{q.a, q.a_cs, q.a_rs};
  // a^T = U' S Vh'  =>  a = Vh'^T S U'^T : U' goes to vh^T, Vh' to u^T
  Mat U = tall ? Mat{q.u, q.u_rs, q.u_cs} : Mat{q.vh, q.vh_cs, q.vh_rs};
  Mat Vh = tall ? Mat{q.vh, q.vh_rs, q.vh_cs} : Mat{q.u, q.u_cs, q.u_rs};
  int st;
  if (mode == 0) {
    st = cta_svd_tall(A, M, K, W, tau, Bsq, V, sv, order, flag, U, q.s, Vh, red);
  } else {
    double* Y = dsm;
    double* G = Y + (i64)LNB * min(K, YCH);
    double* Tm = G + LNB * LNB;
    st = cta_svd_tall_blocked(A, M, K, W, tau, Bsq, V, sv, order, flag, U, q.s, Vh, Y, G, Tm,
                              red, gsm);
  }
  if (q.status && threadIdx.x == 0) *q.status = st;
}

constexpr int kMaxL = 24;
struct LBatch {
  int count;
  int mode[kMaxL];  // 0: all in shared memory, 1: blocked, panel shared, 2: blocked, panel global
  ttb_lu_t d[kMaxL];
};

__global__ void __launch_bounds__(TTB_THREADS) k_lu(const __grid_constant__ LBatch lb) {
  extern __shared__ double dsm[];
  __shared__ double redv[TTB_WARPS];
  __shared__ int redi[TTB_WARPS];
  __shared__ int ipiv[LNB];
  __shared__ GemmSmem gsm;
  const ttb_lu_t& q = lb.d[blockIdx.x];
  const int n = q.n;
  if (n <= 0) return;
  const int mode = lb.mode[blockIdx.x];
  int info;
  if (mode == 0) {
    double* W = dsm;
    double* b = dsm + (i64)n * n;
    for (i64 e = threadIdx.x; e < (i64)n * n; e += TTB_THREADS) {
      i64 i = e % n, j = e / n;
      W[e] = q.a[i + j * q.lda];
    }
    for (int i = threadIdx.x; i < n; i += TTB_THREADS) b[i] = q.b[i];
    __syncthreads();
    info = cta_gepp_solve(W, n, b, n, redv, redi);
    __syncthreads();
    if (info == 0)
      for (int i = threadIdx.x; i < n; i += TTB_THREADS) q.b[i] = b[i];
  } else {
    double* panel = mode == 1 ? dsm : q.work;
    info = cta_gepp_blocked(q.a, q.lda, q.b, n, panel, redv, redi, ipiv, gsm);
  }
  if (q.info && threadIdx.x == 0) *q.info = info;
}

// the one-CTA factorisations' shared-memory limit on the current device
int configure_smem() {
  int e = smem_limit_once((const void*)k_qr, kSmemCap, g_smem_qr);
  if (!e) e = smem_limit_once((const void*)k_svd, kSmemCap, g_smem_svd);
  if (!e) e = smem_limit_once((const void*)k_lu, kSmemCap, g_smem_lu);
  return e;
}

// ---------------------------------------------------------------------------
// truncation-rank rules
// ---------------------------------------------------------------------------

constexpr int kRankRows = 8;  // rows per thread in the prefix-norm pass
constexpr int kRankChunk = kRankRows * TTB_THREADS;

constexpr int kMaxR = 16;
struct RBatch {
  int count;
  int chunks[kMaxR];
  ttb_rank_t d[kMaxR];
};

// part[c * (limit + 1) + r] = sum over the chunk of (prefix r)^2, and
// part[c * (limit + 1) + limit] = sum over the chunk of b^2
__global__ void __launch_bounds__(TTB_THREADS) k_rank_partial(const __grid_constant__ RBatch rb) {
  __shared__ double red[TTB_WARPS];
  const ttb_rank_t& q = rb.d[blockIdx.y];
  const int chunk = blockIdx.x;
  if (chunk >= rb.chunks[blockIdx.y]) return;
  const i64 row0 = (i64)chunk * kRankChunk;
  double run[kRankRows];
  double bsq = 0.0;
#pragma unroll
  for (int e = 0; e < kRankRows; ++e) {
    i64 i = row0 + threadIdx.x + (i64)e * TTB_THREADS;
    double bv = (i < q.n) ? q.b[i] : 0.0;
    run[e] = -bv;
    bsq = fma(bv, bv, bsq);
  }
  double* part = q.work + (i64)chunk * (q.limit + 1);
  for (int r = 0; r < q.limit; ++r) {
    const double* c = q.contrib + (i64)r * q.n;
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < kRankRows; ++e) {
      i64 i = row0 + threadIdx.x + (i64)e * TTB_THREADS;
      if (i < q.n) run[e] += c[i];
      s = fma(run[e], run[e], s);
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[r] = s;
  }
  bsq = block_sum(bsq, red);
  if (threadIdx.x == 0) part[q.limit] = bsq;
}

__global__ void k_rank_select(const __grid_constant__ RBatch rb) {
  const ttb_rank_t& q = rb.d[blockIdx.x];
  if (threadIdx.x != 0) return;
  const int chunks = rb.chunks[blockIdx.x];
  if (q.s[0] == 0.0) {
    q.rank[0] = 1;
    return;
  }
  double bsq = 0.0;
  for (int c = 0; c < chunks; ++c) bsq += q.work[(i64)c * (q.limit + 1) + q.limit];
  const double thr = fmax(q.damp * q.exact[0], 0.5 * q.tol * sqrt(bsq));
  for (int r = 0; r < q.limit; ++r) {
    double s = 0.0;
    for (int c = 0; c < chunks; ++c) s += q.work[(i64)c * (q.limit + 1) + r];
    if (sqrt(s) <= thr) {
      q.rank[0] = r + 1;
      return;
    }
  }
  q.rank[0] = q.limit;
}

constexpr int kMaxRR = 64;
struct RRBatch {
  int count;
  ttb_rank_rule_t d[kMaxRR];
};

__global__ void k_rank_rule(const __grid_constant__ RRBatch rb) {
  const ttb_rank_rule_t& q = rb.d[blockIdx.x];
  if (threadIdx.x != 0) return;
  const double* s = q.s;
  int rank;
  if (q.p <= 0 || s[0] == 0.0) {
    rank = 1;
  } else if (q.mode == 0) {
    int c = 0;
    for (int i = 0; i < q.p; ++i) c += (s[i] / s[0] > q.value);
    rank = c > 1 ? c : 1;
  } else {
    const double floor_ = 2.220446049250313e-16 * q.p * s[0];
    // tail[i] = sum_{j >= i} s_j^2 (noise-floored), accumulated from the end
    const double d2 = q.value * q.value;
    double tail = 0.0;
    int c = 0;
    for (int i = q.p - 1; i >= 0; --i) {
      double v = (s[i] <= floor_) ? 0.0 : s[i];
      tail += v * v;
      if (tail > d2) c++;
    }
    rank = c > 1 ? c : 1;
  }
  if (q.max_rank > 0 && rank > q.max_rank) rank = q.max_rank;
  q.rank[0] = rank;
}

// ---------------------------------------------------------------------------
// local operator GEMM chain (shared by ttb_local_apply and the Krylov solvers)
// ---------------------------------------------------------------------------

i64 local_work(const ttb_local_t& q) {
  return (i64)q.cols * q.lt * q.m * q.R2 * q.rf + (i64)q.cols * q.lt * q.R * q.n * q.rf;
}

void local_descs(const ttb_local_t& q, std::vector<GDesc>& s1, std::vector<GDesc>& s2,
                 std::vector<GDesc>& s3) {
  const int lt = q.lt, lf = q.lf, R = q.R, R2 = q.R2, n = q.n, m = q.m, rt = q.rt, rf = q.rf;
  const int cols = q.cols;
  double* T1 = q.work;
  double* T2 = q.work + (i64)cols * lt * m * R2 * rf;
  // T1 (cols*lt*m, R2*rf) = x (cols*lt*m, rt) @ right (rt, R2*rf)
  s1.push_back(make_gemm(q.x, rt, 1, 0, q.right, (i64)R2 * rf, 1, 0, T1, (i64)R2 * rf, 1, 0,
                         cols * lt * m, R2 * rf, rt, 1, 1.0, 0.0));
  // per (c, i): T2 (R*n, rf) = op (R*n, m*R2) @ T1_ci (m*R2, rf)
  s2.push_back(make_gemm(q.op, (i64)m * R2, 1, 0, T1, rf, 1, (i64)m * R2 * rf, T2, rf, 1,
                         (i64)R * n * rf, R * n, rf, m * R2, cols * lt, 1.0, 0.0));
  // per c: y_c (lf, n*rf) = alpha * left^T (lf, lt*R) @ T2_c (lt*R, n*rf) + beta * y_c
  s3.push_back(make_gemm(q.left, 1, lf, 0, T2, (i64)n * rf, 1, (i64)lt * R * n * rf, q.y,
                         (i64)n * rf, 1, (i64)lf * n * rf, lf, n * rf, lt * R, cols, q.alpha,
                         q.beta));
}

int run_local(const ttb_local_t* ps, int count, cudaStream_t s) {
  std::vector<GDesc> s1, s2, s3;
  for (int i = 0; i < count; ++i) local_descs(ps[i], s1, s2, s3);
  int e;
  if ((e = launch_gemms(s1, s))) return e;
  if ((e = launch_gemms(s2, s))) return e;
  return launch_gemms(s3, s);
}

// ---------------------------------------------------------------------------
// MINRES (Paige & Saunders, with SciPy 1.18.1's stopping rules)
// ---------------------------------------------------------------------------

constexpr int kKryRows = 4;  // rows per thread
constexpr int kKryChunk = kKryRows * TTB_THREADS;
constexpr int kStateDoubles = 32;

// scalar state, one copy per parity of the iteration counter
enum {
  S_BETA1 = 0, S_BNORM, S_BETA, S_OLDB, S_DBAR, S_EPSLN, S_PHIBAR, S_RHS1, S_RHS2, S_TNORM2,
  S_GMAX, S_GMIN, S_CS, S_SN, S_ROOT, S_ANORM, S_ITN, S_ISTOP, S_DONE, S_RTOL, S_MAXIT, S_PEND,
  S_ALFA
};

struct KDesc {
  const double* b;
  double* x;
  double* vec;   // r1 r2 y v w w1 w2, n each
  double* part;  // chunks * 4 partial sums
  double* st;    // 2 * kStateDoubles
  int* istop;
  int* iters;
  i64 n;
  int chunks;
  double rtol;
  int maxit;
};

constexpr int kMaxKry = 32;
struct KBatchM {
  int count;
  KDesc d[kMaxKry];
};

__device__ __forceinline__ double sum_parts(const double* part, int chunks, int slot) {
  double s = 0.0;
  for (int c = 0; c < chunks; ++c) s += part[c * 4 + slot];
  return s;
}

// r1 = b - y (y = A x0, or 0 when cold), y = r1; partials |r1|^2, |b|^2
__global__ void __launch_bounds__(TTB_THREADS) k_minres_init(const __grid_constant__ KBatchM kb,
                                                             int warm) {
  __shared__ double red[TTB_WARPS];
  const KDesc& q = kb.d[blockIdx.y];
  if ((int)blockIdx.x >= q.chunks) return;
  const i64 n = q.n;
  double* r1 = q.vec;
  double* r2 = q.vec + n;
  double* y = q.vec + 2 * n;
  double s1 = 0.0, s2 = 0.0;
  for (int e = 0; e < kKryRows; ++e) {
    i64 i = (i64)blockIdx.x * kKryChunk + threadIdx.x + (i64)e * TTB_THREADS;
    if (i >= n) break;
    double bv = q.b[i];
    double r = warm ? bv - y[i] : bv;
    if (!warm) q.x[i] = 0.0;
    r1[i] = r;
    r2[i] = r;
    y[i] = r;
    s1 = fma(r, r, s1);
    s2 = fma(bv, bv, s2);
  }
  s1 = block_sum(s1, red);
  s2 = block_sum(s2, red);
  if (threadIdx.x == 0) {
    q.part[blockIdx.x * 4 + 0] = s1;
    q.part[blockIdx.x * 4 + 1] = s2;
  }
}

// state[0] from the init partials; v = y / beta1; w = w2 = 0
__global__ void __launch_bounds__(TTB_THREADS) k_minres_start(const __grid_constant__ KBatchM kb,
                                                              double rtol_unused) {
  const KDesc& q = kb.d[blockIdx.y];
  if ((int)blockIdx.x >= q.chunks) return;
  const i64 n = q.n;
  double* st = q.st;
  const double beta1sq = sum_parts(q.part, q.chunks, 0);
  const double bnorm = sqrt(sum_parts(q.part, q.chunks, 1));
  const double beta1 = sqrt(beta1sq);
  const int done = (beta1sq == 0.0 || bnorm == 0.0) ? 1 : 0;
  double* y = q.vec + 2 * n;
  double* v = q.vec + 3 * n;
  double* w = q.vec + 4 * n;
  double* w2 = q.vec + 6 * n;
  const double s = done ? 0.0 : 1.0 / beta1;
  for (int e = 0; e < kKryRows; ++e) {
    i64 i = (i64)blockIdx.x * kKryChunk + threadIdx.x + (i64)e * TTB_THREADS;
    if (i >= n) break;
    v[i] = s * y[i];
    w[i] = 0.0;
    w2[i] = 0.0;
    if (bnorm == 0.0) q.x[i] = q.b[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st[S_BETA1] = beta1;
    st[S_BNORM] = bnorm;
    st[S_BETA] = beta1;
    st[S_OLDB] = 0.0;
    st[S_DBAR] = 0.0;
    st[S_EPSLN] = 0.0;
    st[S_PHIBAR] = beta1;
    st[S_RHS1] = beta1;
    st[S_RHS2] = 0.0;
    st[S_TNORM2] = 0.0;
    st[S_GMAX] = 0.0;
    st[S_GMIN] = DBL_MAX;
    st[S_CS] = -1.0;
    st[S_SN] = 0.0;
    st[S_ROOT] = 0.0;
    st[S_ANORM] = 0.0;
    st[S_ITN] = 0.0;
    st[S_ISTOP] = 0.0;
    st[S_DONE] = done;
    st[S_PEND] = 0.0;
    if (q.istop) *q.istop = 0;
    if (q.iters) *q.iters = 0;
  }
}

// Stop test of the iteration that just finished (state in st), SciPy's
// order of checks.  Returns istop (0 = continue).
__device__ int minres_test(const double* st, double ynorm, double rtol, int maxiter) {
  const double eps = 2.220446049250313e-16;
  const double Anorm = st[S_ANORM];
  const double beta1 = st[S_BETA1];
  const double rnorm = st[S_PHIBAR];
  const double epsx = Anorm * ynorm * eps;
  double test1, test2;
  if (ynorm == 0.0 || Anorm == 0.0) test1 = INFINITY;
  else test1 = rnorm / (Anorm * ynorm);
  if (Anorm == 0.0) test2 = INFINITY;
  else test2 = st[S_ROOT] / Anorm;
  const double Acond = st[S_GMAX] / st[S_GMIN];
  const int itn = (int)st[S_ITN];
  int istop = (int)st[S_PEND];
  if (istop == 0) {
    const double t1 = 1.0 + test1, t2 = 1.0 + test2;
    if (t2 <= 1.0) istop = 2;
    if (t1 <= 1.0) istop = 1;
    if (itn >= maxiter) istop = 6;
    if (Acond >= 0.1 / eps) istop = 4;
    if (epsx >= beta1) istop = 3;
    if (test2 <= rtol) istop = 2;
    if (test1 <= rtol) istop = 1;
  }
  return istop;
}

// Iteration ``it`` (0-based), first half: finish the previous iteration's
// stop test, then y -= (beta/oldb) r1 and the partial v.y.
__global__ void __launch_bounds__(TTB_THREADS) k_minres_a(const __grid_constant__ KBatchM kb, int it) {
  __shared__ double red[TTB_WARPS];
  const KDesc& q = kb.d[blockIdx.y];
  if ((int)blockIdx.x >= q.chunks) return;
  const i64 n = q.n;
  double* st = q.st + (it & 1) * kStateDoubles;
  if (st[S_DONE] != 0.0) return;
  if (it >= 1) {
    const double ynorm = sqrt(sum_parts(q.part, q.chunks, 3));
    const int istop = minres_test(st, ynorm, q.rtol, q.maxit);
    if (istop != 0) {
      // every block of the system reaches the same stopping decision from the same
      // partial sums; block 0 records it
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (q.istop) *q.istop = istop;
        if (q.iters) *q.iters = (int)st[S_ITN];
        st[S_DONE] = 1.0;
      }
      return;
    }
  }
  const double itn = st[S_ITN] + 1.0;
  const double ratio = (itn >= 2.0) ? st[S_BETA] / st[S_OLDB] : 0.0;
  const double* r1 = q.vec;
  double* y = q.vec + 2 * n;
  const double* v = q.vec + 3 * n;
  double s = 0.0;
  for (int e = 0; e < kKryRows; ++e) {
    i64 i = (i64)blockIdx.x * kKryChunk + threadIdx.x + (i64)e * TTB_THREADS;
    if (i >= n) break;
    double yi = y[i];
    if (itn >= 2.0) yi = yi - ratio * r1[i];
    y[i] = yi;
    s = fma(v[i], yi, s);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) q.part[blockIdx.x * 4 + 0] = s;
}

// second half: alfa; y -= (alfa/beta) r2; r1 = r2; r2 = y; partial |y|^2
__global__ void __launch_bounds__(TTB_THREADS) k_minres_b(const __grid_constant__ KBatchM kb, int it) {
  __shared__ double red[TTB_WARPS];
  const KDesc& q = kb.d[blockIdx.y];
  if ((int)blockIdx.x >= q.chunks) return;
  const i64 n = q.n;
  const double* st = q.st + (it & 1) * kStateDoubles;
  if (st[S_DONE] != 0.0) return;
  const double alfa = sum_parts(q.part, q.chunks, 0);
  const double f = alfa / st[S_BETA];
  double* r1 = q.vec;
  double* r2 = q.vec + n;
  double* y = q.vec + 2 * n;
  double s = 0.0;
  for (int e = 0; e < kKryRows; ++e) {
    i64 i = (i64)blockIdx.x * kKryChunk + threadIdx.x + (i64)e * TTB_THREADS;
    if (i >= n) break;
    double yi = y[i] - f * r2[i];
    r1[i] = r2[i];
    r2[i] = yi;
    y[i] = yi;
    s = fma(yi, yi, s);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) q.part[blockIdx.x * 4 + 1] = s;
}

// third part: scalar recurrences, w and x updates, v for the next
// iteration, partial |x|^2; writes the next state copy
__global__ void __launch_bounds__(TTB_THREADS) k_minres_c(const __grid_constant__ KBatchM kb, int it) {
  __shared__ double red[TTB_WARPS];
  const KDesc& q = kb.d[blockIdx.y];
  if ((int)blockIdx.x >= q.chunks) return;
  const i64 n = q.n;
  const double* st = q.st + (it & 1) * kStateDoubles;
  double* nx = q.st + ((it + 1) & 1) * kStateDoubles;
  if (st[S_DONE] != 0.0) {
    // keep the finished flag visible in the copy the next iteration reads
    if (blockIdx.x == 0 && threadIdx.x == 0) nx[S_DONE] = 1.0;
    return;
  }
  const double eps = 2.220446049250313e-16;
  const double alfa = sum_parts(q.part, q.chunks, 0);
  const double itn = st[S_ITN] + 1.0;
  const double oldb = st[S_BETA];
  const double beta = sqrt(sum_parts(q.part, q.chunks, 1));
  const double tnorm2 = st[S_TNORM2] + alfa * alfa + oldb * oldb + beta * beta;
  double pend = st[S_PEND];
  if (itn == 1.0 && beta / st[S_BETA1] <= 10.0 * eps) pend = -1.0;
  const double oldeps = st[S_EPSLN];
  const double cs0 = st[S_CS], sn0 = st[S_SN], dbar0 = st[S_DBAR];
  const double delta = cs0 * dbar0 + sn0 * alfa;
  const double gbar = sn0 * dbar0 - cs0 * alfa;
  const double epsln = sn0 * beta;
  const double dbar = -cs0 * beta;
  const double root = hypot(gbar, dbar);
  double gamma = hypot(gbar, beta);
  gamma = fmax(gamma, eps);
  const double cs = gbar / gamma;
  const double sn = beta / gamma;
  const double phi = cs * st[S_PHIBAR];
  const double phibar = sn * st[S_PHIBAR];
  const double denom = 1.0 / gamma;
  const double z = st[S_RHS1] / gamma;
  const double rhs1 = st[S_RHS2] - delta * z;
  const double rhs2 = -epsln * z;
  const double rbeta = 1.0 / beta;
  const double* y = q.vec + 2 * n;
  double* v = q.vec + 3 * n;
  double* w = q.vec + 4 * n;
  double* w1 = q.vec + 5 * n;
  double* w2 = q.vec + 6 * n;
  double s = 0.0;
  for (int e = 0; e < kKryRows; ++e) {
    i64 i = (i64)blockIdx.x * kKryChunk + threadIdx.x + (i64)e * TTB_THREADS;
    if (i >= n) break;
    double w1n = w2[i];
    double w2n = w[i];
    double wn = (v[i] - oldeps * w1n - delta * w2n) * denom;
    w1[i] = w1n;
    w2[i] = w2n;
    w[i] = wn;
    double xi = q.x[i] + phi * wn;
    q.x[i] = xi;
    s = fma(xi, xi, s);
    v[i] = rbeta * y[i];
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) q.part[blockIdx.x * 4 + 3] = s;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    nx[S_BETA1] = st[S_BETA1];
    nx[S_BNORM] = st[S_BNORM];
    nx[S_BETA] = beta;
    nx[S_OLDB] = oldb;
    nx[S_DBAR] = dbar;
    nx[S_EPSLN] = epsln;
    nx[S_PHIBAR] = phibar;
    nx[S_RHS1] = rhs1;
    nx[S_RHS2] = rhs2;
    nx[S_TNORM2] = tnorm2;
    nx[S_GMAX] = fmax(st[S_GMAX], gamma);
    nx[S_GMIN] = fmin(st[S_GMIN], gamma);
    nx[S_CS] = cs;
    nx[S_SN] = sn;
    nx[S_ROOT] = root;
    nx[S_ANORM] = sqrt(tnorm2);
    nx[S_ITN] = itn;
    nx[S_ISTOP] = 0.0;
    nx[S_DONE] = 0.0;
    nx[S_PEND] = pend;
  }
}

// final stop test for systems still running when the loop ends (the test of
// the last iteration is otherwise evaluated at the start of the next one)
__global__ void k_minres_final(const __grid_constant__ KBatchM kb, int it, int* done_out) {
  const KDesc& q = kb.d[blockIdx.x];
  if (threadIdx.x != 0) return;
  double* st = q.st + (it & 1) * kStateDoubles;
  if (st[S_DONE] != 0.0) {
    done_out[blockIdx.x] = 1;
    return;
  }
  if (it == 0) {
    done_out[blockIdx.x] = 0;
    return;
  }
  const double ynorm = sqrt(sum_parts(q.part, q.chunks, 3));
  const int istop = minres_test(st, ynorm, q.rtol, q.maxit);
  if (istop != 0) {
    st[S_DONE] = 1.0;
    if (q.istop) *q.istop = istop;
    if (q.iters) *q.iters = (int)st[S_ITN];
  }
  done_out[blockIdx.x] = istop != 0;
}


// ---------------------------------------------------------------------------
// GMRES(restart) with SciPy 1.18.1's gmres control flow
// ---------------------------------------------------------------------------

// scalar state slots
enum {
  G_BNRM2 = 0, G_ATOL, G_PTOL, G_PMF, G_PRESID, G_RNORM, G_COL, G_BREAK, G_DONE, G_INNER,
  G_CONV, G_NSTATE = 16
};

struct GmDesc {
  const double* b;
  double* x;
  double* V;      // (restart + 1) x n basis
  double* w;      // n
  double* r;      // n
  double* h;      // restart x (restart + 1), h[col * (restart + 1) + row]
  double* giv;    // restart x 2
  double* S;      // restart + 1
  double* st;     // G_NSTATE scalars
  int* istop;
  int* iters;
  i64 n;
  double rtol;
  int restart;
};

constexpr int kMaxGm = 16;
struct GmBatch {
  int count;
  GmDesc d[kMaxGm];
};

// LAPACK dlartg convention (unscaled branch): [c s; -s c] [f; g] = [r; 0]
__device__ __forceinline__ void lartg(double f, double g, double& c, double& s, double& r) {
  if (g == 0.0) { c = 1.0; s = 0.0; r = f; return; }
  if (f == 0.0) { c = 0.0; s = (g >= 0.0) ? 1.0 : -1.0; r = fabs(g); return; }
  double d = sqrt(f * f + g * g);
  c = fabs(f) / d;
  r = copysign(d, f);
  s = g / r;
}

// bnrm2, atol, ptol; r = b - y (warm) or b; done when ||r|| < atol or b == 0
__global__ void __launch_bounds__(TTB_THREADS) k_gm_init(const __grid_constant__ GmBatch gb, int warm_mask_lo, int warm_mask_hi) {
  __shared__ double red[TTB_WARPS];
  const GmDesc& q = gb.d[blockIdx.x];
  const int j = blockIdx.x;
  const int warm = (j < 32) ? ((warm_mask_lo >> j) & 1) : ((warm_mask_hi >> (j - 32)) & 1);
  double sb = 0.0, sr = 0.0;
  for (i64 i = threadIdx.x; i < q.n; i += TTB_THREADS) {
    double bv = q.b[i];
    double rv = warm ? bv - q.w[i] : bv;
    if (!warm) q.x[i] = 0.0;
    q.r[i] = rv;
    sb = fma(bv, bv, sb);
    sr = fma(rv, rv, sr);
  }
  sb = block_sum(sb, red);
  sr = block_sum(sr, red);
  if (threadIdx.x == 0) {
    const double bnrm2 = sqrt(sb);
    const double atol = fmax(0.0, q.rtol * bnrm2);
    double* st = q.st;
    st[G_BNRM2] = bnrm2;
    st[G_ATOL] = atol;
    st[G_PMF] = 1.0;
    st[G_PTOL] = (bnrm2 > 0.0) ? bnrm2 * fmin(1.0, atol / bnrm2) : 0.0;
    st[G_PRESID] = 0.0;
    st[G_INNER] = 0.0;
    st[G_DONE] = 0.0;
    st[G_CONV] = 0.0;
    if (bnrm2 == 0.0) { st[G_DONE] = 1.0; st[G_CONV] = 1.0; }
    else if (sqrt(sr) < atol) { st[G_DONE] = 1.0; st[G_CONV] = 1.0; }
    if (q.iters) *q.iters = 0;
    if (q.istop) *q.istop = 1;
  }
  __syncthreads();
  if (sb == 0.0)
    for (i64 i = threadIdx.x; i < q.n; i += TTB_THREADS) q.x[i] = q.b[i];
}

// start of an outer cycle: v0 = r / ||r||, S = [||r||, 0, ...]
__global__ void __launch_bounds__(TTB_THREADS) k_gm_cycle(const __grid_constant__ GmBatch gb) {
  __shared__ double red[TTB_WARPS];
  const GmDesc& q = gb.d[blockIdx.x];
  if (q.st[G_DONE] != 0.0) return;
  double s = 0.0;
  for (i64 i = threadIdx.x; i < q.n; i += TTB_THREADS) s = fma(q.r[i], q.r[i], s);
  s = block_sum(s, red);
  const double tmp = sqrt(s);
  const double inv = 1.0 / tmp;
  for (i64 i = threadIdx.x; i < q.n; i += TTB_THREADS) q.V[i] = q.r[i] * inv;
  for (int i = threadIdx.x; i <= q.restart; i += TTB_THREADS) q.S[i] = (i == 0) ? tmp : 0.0;
  if (threadIdx.x == 0) {
    q.st[G_COL] = 0.0;
    q.st[G_BREAK] = 0.0;
  }
}

// one Arnoldi column (w = A v_col on entry): modified Gram-Schmidt, the
// breakdown test, past and new Givens rotations, presid; flags the end of
// the inner loop in st[G_COL] = -1 - col
__global__ void __launch_bounds__(TTB_THREADS) k_gm_arnoldi(const __grid_constant__ GmBatch gb, int col) {
  __shared__ double red[TTB_WARPS];
  const GmDesc& q = gb.d[blockIdx.x];
  if (q.st[G_DONE] != 0.0 || q.st[G_COL] < 0.0) return;
  const double eps = 2.220446049250313e-16;
  const i64 n = q.n;
  const int R1 = q.restart + 1;
  double* h = q.h + (i64)col * R1;
  double* w = q.w;
  double s = 0.0;
  for (i64 i = threadIdx.x; i < n; i += TTB_THREADS) s = fma(w[i], w[i], s);
  const double h0 = sqrt(block_sum(s, red));
  for (int k = 0; k <= col; ++k) {
    const double* vk = q.V + (i64)k * n;
    double d = 0.0;
    for (i64 i = threadIdx.x; i < n; i += TTB_THREADS) d = fma(vk[i], w[i], d);
    d = block_sum(d, red);
    if (threadIdx.x == 0) h[k] = d;
    for (i64 i = threadIdx.x; i < n; i += TTB_THREADS) w[i] -= d * vk[i];
    __syncthreads();
  }
  s = 0.0;
  for (i64 i = threadIdx.x; i < n; i += TTB_THREADS) s = fma(w[i], w[i], s);
  const double h1 = sqrt(block_sum(s, red));
  double* vn = q.V + (i64)(col + 1) * n;
  const bool brk = h1 <= eps * h0;
  const double inv = brk ? 1.0 : 1.0 / h1;
  for (i64 i = threadIdx.x; i < n; i += TTB_THREADS) vn[i] = brk ? w[i] : w[i] * inv;
  __syncthreads();
  if (threadIdx.x == 0) {
    h[col + 1] = brk ? 0.0 : h1;
    for (int k = 0; k < col; ++k) {
      const double c = q.giv[2 * k], sn = q.giv[2 * k + 1];
      const double n0 = h[k], n1 = h[k + 1];
      h[k] = c * n0 + sn * n1;
      h[k + 1] = -sn * n0 + c * n1;
    }
    double c, sn, mag;
    lartg(h[col], h[col + 1], c, sn, mag);
    q.giv[2 * col] = c;
    q.giv[2 * col + 1] = sn;
    h[col] = mag;
    h[col + 1] = 0.0;
    const double tmp = -sn * q.S[col];
    q.S[col] = c * q.S[col];
    q.S[col + 1] = tmp;
    const double presid = fabs(tmp);
    q.st[G_PRESID] = presid;
    q.st[G_INNER] += 1.0;
    if (brk) q.st[G_BREAK] = 1.0;
    if (presid <= q.st[G_PTOL] || brk || col == q.restart - 1) q.st[G_COL] = -1.0 - col;
    else q.st[G_COL] = col + 1;
  }
}

// end of the inner loop: back substitution on the rotated Hessenberg
// factor and x += y V
__global__ void __launch_bounds__(TTB_THREADS) k_gm_update(const __grid_constant__ GmBatch gb) {
  __shared__ double y[64];
  const GmDesc& q = gb.d[blockIdx.x];
  if (q.st[G_DONE] != 0.0) return;
  const int col = (int)(-q.st[G_COL] - 1.0);
  const int R1 = q.restart + 1;
  if (threadIdx.x == 0) {
    if (q.h[(i64)col * R1 + col] == 0.0) q.S[col] = 0.0;
    for (int k = 0; k <= col; ++k) y[k] = q.S[k];
    for (int k = col; k > 0; --k) {
      if (y[k] != 0.0) {
        y[k] /= q.h[(i64)k * R1 + k];
        const double t = y[k];
        for (int i = 0; i < k; ++i) y[i] -= t * q.h[(i64)k * R1 + i];
      }
    }
    if (y[0] != 0.0) y[0] /= q.h[0];
  }
  __syncthreads();
  for (i64 i = threadIdx.x; i < q.n; i += TTB_THREADS) {
    double acc = 0.0;
    for (int k = 0; k <= col; ++k) acc = fma(y[k], q.V[(i64)k * q.n + i], acc);
    q.x[i] += acc;
  }
}

// after w = A x: r = b - w, rnorm, the outer convergence and ptol updates
__global__ void __launch_bounds__(TTB_THREADS) k_gm_outer(const __grid_constant__ GmBatch gb, int iteration, int maxiter) {
  __shared__ double red[TTB_WARPS];
  const GmDesc& q = gb.d[blockIdx.x];
  if (q.st[G_DONE] != 0.0) return;
  double s = 0.0;
  for (i64 i = threadIdx.x; i < q.n; i += TTB_THREADS) {
    double rv = q.b[i] - q.w[i];
    q.r[i] = rv;
    s = fma(rv, rv, s);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) {
    const double eps = 2.220446049250313e-16;
    double* st = q.st;
    const double rnorm = sqrt(s);
    st[G_RNORM] = rnorm;
    const double atol = st[G_ATOL];
    const double presid = st[G_PRESID];
    if (rnorm <= atol) {
      st[G_DONE] = 1.0;
      st[G_CONV] = 1.0;
    } else if (st[G_BREAK] != 0.0) {
      st[G_DONE] = 1.0;
    } else {
      double pmf = st[G_PMF];
      if (presid <= st[G_PTOL]) pmf = fmax(eps, 0.25 * pmf);
      else pmf = fmin(1.0, 1.5 * pmf);
      st[G_PMF] = pmf;
      st[G_PTOL] = presid * fmin(pmf, atol / rnorm);
      if (iteration + 1 >= maxiter) st[G_DONE] = 1.0;
    }
    if (st[G_DONE] != 0.0) {
      if (q.istop) *q.istop = st[G_CONV] != 0.0 ? 0 : 1;
      if (q.iters) *q.iters = (int)st[G_INNER];
    }
  }
}

// flags[j] = inner loop ended (mode 0) / solve finished (mode 1)
__global__ void k_gm_flags(const __grid_constant__ GmBatch gb, int* flags, int mode) {
  const GmDesc& q = gb.d[blockIdx.x];
  if (threadIdx.x != 0) return;
  if (mode == 0) flags[blockIdx.x] = (q.st[G_DONE] != 0.0 || q.st[G_COL] < 0.0) ? 1 : 0;
  else flags[blockIdx.x] = q.st[G_DONE] != 0.0 ? 1 : 0;
}

// ---------------------------------------------------------------------------
// batched TT rounding of p + q, one block per pair
// ---------------------------------------------------------------------------

constexpr int kRoundMaxBond = 64;
constexpr int kRoundMaxRows = 256;
constexpr int kRoundMaxD = 64;

__device__ int round_truncated_bond(const double* S, int p, double delta, int max_rank) {
  const double floor_ = 2.220446049250313e-16 * p * S[0];
  const double d2 = delta * delta;
  double tail = 0.0;
  int c = 0;
  for (int i = p - 1; i >= 0; --i) {
    double v = (S[i] <= floor_) ? 0.0 : S[i];
    tail += v * v;
    if (tail > d2) c++;
  }
  int r = c > 1 ? c : 1;
  if (max_rank > 0 && r > max_rank) r = max_rank;
  return r;
}

__global__ void __launch_bounds__(TTB_THREADS) k_round(const __grid_constant__ ttb_round_t P,
                                                       i64 slot, i64 qslot) {
  extern __shared__ double dsm[];
  __shared__ double red[TTB_WARPS];
  __shared__ GemmSmem gsm;
  __shared__ int rows_of[kRoundMaxD];
  __shared__ int nb_sh;
  const int pair = blockIdx.x;
  const int d = P.d;
  const double* pb = P.p + pair * P.p_stride;
  const double* qb = P.q + pair * P.q_stride;
  double* work = P.work + pair * P.work_stride;
  double* out = P.out + pair * P.out_stride;
  // global per-pair work: Q cores (d slots), X, Rm, U, Vh, S
  double* qcores = work;
  double* X = qcores + (i64)d * qslot;
  double* Rm = X + qslot;
  double* U = Rm + (i64)kRoundMaxBond * kRoundMaxBond;
  double* Vh = U + qslot;
  double* Sv = Vh + qslot;
  // shared factorisation area
  double* W = dsm;
  double* tau = W + (i64)kRoundMaxRows * kRoundMaxBond;
  double* Bsq = tau + kRoundMaxBond;
  double* V = Bsq + kRoundMaxBond * kRoundMaxBond;
  double* sv = V + kRoundMaxBond * kRoundMaxBond;
  int* order = reinterpret_cast<int*>(sv + kRoundMaxBond);
  int* flag = reinterpret_cast<int*>(sv + 2 * kRoundMaxBond);
  int status = 0;
  const int RS = kRoundMaxBond;  // row stride of Rm
  // shapes outside the shared-memory plan are refused (status -2)
  for (int k = 0; k < d; ++k) {
    const int n = P.modes[k];
    const int rin = (k == 0) ? 1 : P.p_bonds[k] + P.q_bonds[k];
    const int rout = (k == d - 1) ? 1 : P.p_bonds[k + 1] + P.q_bonds[k + 1];
    if (rin > kRoundMaxBond || rout > kRoundMaxBond || n * rin > kRoundMaxRows ||
        n * rout > kRoundMaxRows) {
      if (threadIdx.x == 0 && P.status) P.status[pair] = -2;
      return;
    }
  }

  if (threadIdx.x == 0) Rm[0] = 1.0;
  __syncthreads();
  int rl = 1;
  // ---- left QR sweep of the block-diagonal sum
  for (int k = 0; k < d; ++k) {
    const int n = P.modes[k];
    const int rp = P.p_bonds[k], rq = P.q_bonds[k];
    const int rp2 = P.p_bonds[k + 1], rq2 = P.q_bonds[k + 1];
    const int r_out = (k == d - 1) ? 1 : rp2 + rq2;
    const double* pk = pb + P.p_off[k];
    const double* qk = qb + P.q_off[k];
    const int m = rl * n;
    for (int e = threadIdx.x; e < m * r_out; e += TTB_THREADS) X[e] = 0.0;
    __syncthreads();
    for (int i = 0; i < n; ++i) {
      // X[(a, i), b] += Rm[a, :rp] p[:, i, b]
      cta_gemm(CMat{Rm, RS, 1}, CMat{pk + (i64)i * rp2, (i64)n * rp2, 1},
               Mat{X + (i64)i * r_out, (i64)n * r_out, 1}, rl, rp2, (k == 0) ? 1 : rp, 1.0, 1.0,
               gsm);
      cta_gemm(CMat{Rm + ((k == 0) ? 0 : rp), RS, 1}, CMat{qk + (i64)i * rq2, (i64)n * rq2, 1},
               Mat{X + (i64)i * r_out + ((k == d - 1) ? 0 : rp2), (i64)n * r_out, 1}, rl, rq2,
               (k == 0) ? 1 : rq, 1.0, 1.0, gsm);
    }
    rows_of[k] = rl;  // rows of core k before its factorisation
    if (k == d - 1) break;
    const int pq = m < r_out ? m : r_out;
    cta_qr(CMat{X, r_out, 1}, m, r_out, W, tau, Mat{qcores + (i64)k * qslot, pq, 1},
           Mat{Rm, RS, 1}, red);
    rl = pq;
  }
  // ---- norm of the last core and the per-split budget
  const int nl = P.modes[d - 1];
  double s2 = 0.0;
  for (int e = threadIdx.x; e < rl * nl; e += TTB_THREADS) s2 = fma(X[e], X[e], s2);
  const double nrm = sqrt(block_sum(s2, red));
  const double delta = P.error / sqrt((double)(d - 1)) * nrm;
  // ---- right SVD sweep
  int bond = 1;
  int r = rl;  // rows of the current matrix X (r x n*bond), row major
  if (threadIdx.x == 0) {
    P.bonds[(i64)pair * (d + 1) + d] = 1;
    P.bonds[(i64)pair * (d + 1)] = 1;
  }
  for (int i = d - 1; i >= 1; --i) {
    const int n = P.modes[i];
    const int c = n * bond;
    const int p = r < c ? r : c;
    int st;
    if (r >= c) {
      st = cta_svd_tall(CMat{X, c, 1}, r, c, W, tau, Bsq, V, sv, order, flag, Mat{U, p, 1}, Sv,
                        Mat{Vh, c, 1}, red);
    } else {
      st = cta_svd_tall(CMat{X, 1, c}, c, r, W, tau, Bsq, V, sv, order, flag, Mat{Vh, 1, c}, Sv,
                        Mat{U, 1, p}, red);
    }
    if (st < 0) status = -1;
    __syncthreads();
    if (threadIdx.x == 0) nb_sh = round_truncated_bond(Sv, p, delta, P.max_rank);
    __syncthreads();
    const int nb = nb_sh;
    // core i = Vh[:nb] as (nb, n, bond)
    double* oc = out + (i64)i * slot;
    for (int e = threadIdx.x; e < nb * c; e += TTB_THREADS) oc[e] = Vh[e];
    // U[:, :nb] *= S[:nb]
    for (int e = threadIdx.x; e < r * nb; e += TTB_THREADS) {
      int a = e / nb, j = e % nb;
      U[(i64)a * p + j] *= Sv[j];
    }
    __syncthreads();
    // X <- Qcore_{i-1} (rows*n_{i-1} x r) @ U[:, :nb]
    const int rows = rows_of[i - 1];
    const int mprev = rows * P.modes[i - 1];
    cta_gemm(CMat{qcores + (i64)(i - 1) * qslot, r, 1}, CMat{U, p, 1}, Mat{X, nb, 1}, mprev, nb, r,
             1.0, 0.0, gsm);
    if (threadIdx.x == 0) P.bonds[(i64)pair * (d + 1) + i] = nb;
    bond = nb;
    r = rows;
  }
  // core 0
  {
    const int c = P.modes[0] * bond;
    for (int e = threadIdx.x; e < c; e += TTB_THREADS) out[e] = X[e];
  }
  for (int k = threadIdx.x; k < d; k += TTB_THREADS) P.out_off[(i64)pair * d + k] = (i64)k * slot;
  if (threadIdx.x == 0 && P.status) P.status[pair] = status;
}


// FP64 FMA throughput probe: 8 independent chains per thread
__global__ void __launch_bounds__(TTB_THREADS) k_fma_peak(double* out, int iters) {
  double a[8];
  const double m = 1.0 + 1e-9 * threadIdx.x, c = 1e-12;
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = j * 1e-3 + blockIdx.x * 1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = fma(a[j], m, c);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += a[j];
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

}  // namespace

// ---------------------------------------------------------------------------
// Fixed scratch for ttb_qr_static: one array in the module's own device
// memory (it exists on every device the module is loaded on), so the entry
// point needs no allocator.  Nothing in it has to start at zero: the blocked
// factorisation copies the input into its slice and writes every tau before
// reading it.  Calls that overlap in time (other streams, other host
// threads) share it and race; they must be serialised by the caller.
// ---------------------------------------------------------------------------

static __device__ __align__(256) double g_qr_static[TTB_QR_STATIC_DOUBLES];

namespace {

constexpr int kStaticDevices = 64;
constexpr i64 kStaticAlign = 32;  // doubles: every slice starts on 256 bytes
std::atomic<double*> g_qr_static_base[kStaticDevices];

// Device address of g_qr_static on the current device, looked up on the
// first call there (with that device current) and kept.
int qr_static_base(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kStaticDevices) return (int)cudaErrorInvalidDevice;
  double* p = g_qr_static_base[dev].load(std::memory_order_acquire);
  if (!p) {
    void* addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_qr_static);
    if (e != cudaSuccess) return (int)e;
    e = cudaFuncSetAttribute(k_qr, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap);
    if (e != cudaSuccess) return (int)e;
    p = static_cast<double*>(addr);
    g_qr_static_base[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return 0;
}

}  // namespace

namespace ttb {
void count_launch() { counted(); }

int smem_limit_once(const void* func, int bytes, int* done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kMaxDevices) return (int)cudaErrorInvalidDevice;
  if (__atomic_load_n(&done[dev], __ATOMIC_ACQUIRE)) return 0;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return (int)e;
  __atomic_store_n(&done[dev], 1, __ATOMIC_RELEASE);
  return 0;
}
}  // namespace ttb

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

int ttb_version(void) { return 1; }

long long ttb_launch_count(void) { return g_launches.load(); }

int ttb_gemm(const ttb_gemm_t* ps, int count, void* stream) {
  std::vector<GDesc> ds;
  ds.reserve(count);
  for (int i = 0; i < count; ++i) {
    const ttb_gemm_t& p = ps[i];
    ds.push_back(make_gemm(p.a, p.a_rs, p.a_cs, p.a_bs, p.b, p.b_rs, p.b_cs, p.b_bs, p.c, p.c_rs,
                           p.c_cs, p.c_bs, p.m, p.n, p.k, p.batch, p.alpha, p.beta));
  }
  return launch_gemms(ds, as_stream(stream));
}

long long ttb_env_work_doubles(const ttb_env_t* q) {
  if (q->op) {
    if (q->side == 0) return (i64)q->t * q->R * q->n * q->f2 + (i64)q->t * q->m * q->R2 * q->f2;
    return (i64)q->t2 * q->m * q->R * q->f + (i64)q->t2 * q->R2 * q->n * q->f;
  }
  if (q->side == 0) return (i64)q->t * q->n * q->f2;
  return (i64)q->t2 * q->n * q->f;
}

int ttb_env_update(const ttb_env_t* ps, int count, void* stream) {
  std::vector<GDesc> s1, s2, s3;
  for (int i = 0; i < count; ++i) {
    const ttb_env_t& q = ps[i];
    const int f = q.f, f2 = q.f2, t = q.t, t2 = q.t2, R = q.R, R2 = q.R2, n = q.n, m = q.m;
    if (q.op && q.side == 0) {
      double* S1 = q.work;
      double* S2 = q.work + (i64)t * R * n * f2;
      s1.push_back(make_gemm(q.env, f, 1, 0, q.frame, (i64)n * f2, 1, 0, S1, (i64)n * f2, 1, 0,
                             t * R, n * f2, f, 1, 1.0, 0.0));
      s2.push_back(make_gemm(q.op, 1, (i64)m * R2, 0, S1, f2, 1, (i64)R * n * f2, S2, f2, 1,
                             (i64)m * R2 * f2, m * R2, f2, R * n, t, 1.0, 0.0));
      s3.push_back(make_gemm(q.target, 1, t2, 0, S2, (i64)R2 * f2, 1, 0, q.out, (i64)R2 * f2, 1, 0,
                             t2, R2 * f2, t * m, 1, 1.0, 0.0));
    } else if (q.op) {
      double* S1 = q.work;
      double* S2 = q.work + (i64)t2 * m * R * f;
      s1.push_back(make_gemm(q.target, t, 1, 0, q.env, (i64)R * f, 1, 0, S1, (i64)R * f, 1, 0,
                             t2 * m, R * f, t, 1, 1.0, 0.0));
      s2.push_back(make_gemm(q.op, (i64)m * R, 1, 0, S1, f, 1, (i64)m * R * f, S2, f, 1,
                             (i64)R2 * n * f, R2 * n, f, m * R, t2, 1.0, 0.0));
      s3.push_back(make_gemm(S2, (i64)n * f, 1, 0, q.frame, 1, (i64)n * f, 0, q.out, f2, 1, 0,
                             t2 * R2, f2, n * f, 1, 1.0, 0.0));
    } else if (q.side == 0) {
      double* S1 = q.work;
      s1.push_back(make_gemm(q.env, f, 1, 0, q.frame, (i64)n * f2, 1, 0, S1, (i64)n * f2, 1, 0, t,
                             n * f2, f, 1, 1.0, 0.0));
      s2.push_back(make_gemm(q.target, 1, t2, 0, S1, f2, 1, 0, q.out, f2, 1, 0, t2, f2, t * n, 1,
                             1.0, 0.0));
    } else {
      double* S1 = q.work;
      s1.push_back(make_gemm(q.target, t, 1, 0, q.env, f, 1, 0, S1, f, 1, 0, t2 * n, f, t, 1, 1.0,
                             0.0));
      s2.push_back(make_gemm(S1, (i64)n * f, 1, 0, q.frame, 1, (i64)n * f, 0, q.out, f2, 1, 0, t2,
                             f2, n * f, 1, 1.0, 0.0));
    }
  }
  cudaStream_t s = as_stream(stream);
  int e;
  if ((e = launch_gemms(s1, s))) return e;
  if ((e = launch_gemms(s2, s))) return e;
  return launch_gemms(s3, s);
}

long long ttb_local_work_doubles(const ttb_local_t* q) { return local_work(*q); }

int ttb_local_apply(const ttb_local_t* ps, int count, void* stream) {
  return run_local(ps, count, as_stream(stream));
}

int ttb_local_matrix(const ttb_local_matrix_t* ps, int count, void* stream) {
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxLM) {
    LMBatch lb;
    lb.count = std::min(kMaxLM, count - i0);
    long long most = 1;
    for (int j = 0; j < lb.count; ++j) {
      lb.d[j] = ps[i0 + j];
      const ttb_local_matrix_t& q = lb.d[j];
      most = std::max(most, (long long)q.lf * q.n * q.rf * q.lt * q.m * q.rt);
    }
    dim3 grid((unsigned)std::min<long long>(cdiv(most, TTB_THREADS), 4096), lb.count);
    ProfScope ps(P_LOCALMAT, s, 0.0, 0.0);
    k_local_matrix<<<grid, TTB_THREADS, 0, s>>>(lb);
    counted();
  }
  return last_error();
}

int ttb_project(const ttb_project_t* ps, int count, void* stream) {
  std::vector<GDesc> s1, s2;
  for (int i = 0; i < count; ++i) {
    const ttb_project_t& q = ps[i];
    // W (a*n, l) = core (a*n, c) @ right (c, l)
    s1.push_back(make_gemm(q.core, q.c, 1, 0, q.right, q.l, 1, 0, q.work, q.l, 1, 0, q.a * q.n,
                           q.l, q.c, 1, 1.0, 0.0));
    // out (i, n*l) = alpha * left^T (i, a) @ W (a, n*l) + beta * out
    s2.push_back(make_gemm(q.left, 1, q.i, 0, q.work, (i64)q.n * q.l, 1, 0, q.out, (i64)q.n * q.l,
                           1, 0, q.i, q.n * q.l, q.a, 1, q.alpha, q.beta));
  }
  cudaStream_t s = as_stream(stream);
  int e;
  if ((e = launch_gemms(s1, s))) return e;
  return launch_gemms(s2, s);
}

long long ttb_qr_work_doubles(int m, int k) { return qr_need(m, k); }

int ttb_qr(const ttb_qr_t* ps, int count, void* stream) {
  if (int e = configure_smem()) return e;
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxQ) {
    QBatch qb;
    qb.count = std::min(kMaxQ, count - i0);
    i64 smem = 0;
    for (int j = 0; j < qb.count; ++j) {
      qb.d[j] = ps[i0 + j];
      const i64 whole = qr_need(qb.d[j].m, qb.d[j].k) * 8;
      const i64 blk = blocked_smem(qb.d[j].k) * 8;
      if (whole <= kSmemCap) {
        qb.mode[j] = 0;
        smem = std::max(smem, whole);
      } else {
        if (blk > kSmemCap) return (int)cudaErrorInvalidValue;
        qb.mode[j] = 1;
        smem = std::max(smem, blk);
      }
    }
    double fl = 0.0;
    for (int j = 0; j < qb.count; ++j) {
      // Householder R: 2mk^2 - 2k^3/3 (p = k), and as much again to form Q
      const double m = qb.d[j].m, k = std::min(qb.d[j].m, qb.d[j].k), kk = qb.d[j].k;
      fl += 2.0 * m * k * kk - 2.0 / 3.0 * k * k * k;
      if (qb.d[j].q) fl += 2.0 * m * k * k - 2.0 / 3.0 * k * k * k;
    }
    ProfScope ps(P_QR, s, fl, 0.0);
    k_qr<<<qb.count, TTB_THREADS, (size_t)smem, s>>>(qb);
    counted();
  }
  return last_error();
}

int ttb_qr_static(const ttb_qr_t* ps, int count, void* stream) {
  double* base = nullptr;
  int e = qr_static_base(&base);
  if (e) return e;
  if (count <= 0) return 0;
  // pass 0 checks every problem before anything is launched; pass 1 gives
  // each blocked problem its own slice (in call order) and launches
  for (int pass = 0; pass < 2; ++pass) {
    i64 used = 0;
    for (int i0 = 0; i0 < count; i0 += kMaxQ) {
      QBatch qb;
      qb.count = std::min(kMaxQ, count - i0);
      i64 smem = 0;
      for (int j = 0; j < qb.count; ++j) {
        qb.d[j] = ps[i0 + j];
        const i64 whole = qr_need(qb.d[j].m, qb.d[j].k) * 8;
        if (whole <= kSmemCap) {
          qb.mode[j] = 0;
          qb.d[j].work = nullptr;
          smem = std::max(smem, whole);
        } else {
          const i64 blk = blocked_smem(qb.d[j].k) * 8;
          if (blk > kSmemCap) return (int)cudaErrorInvalidValue;
          const i64 need = (qr_need(qb.d[j].m, qb.d[j].k) + kStaticAlign - 1) / kStaticAlign *
                           kStaticAlign;
          if (need > TTB_QR_STATIC_DOUBLES - used) return TTB_ERR_STATIC_SCRATCH;
          qb.mode[j] = 1;
          qb.d[j].work = base + used;
          used += need;
          smem = std::max(smem, blk);
        }
      }
      if (pass == 1) {
        k_qr<<<qb.count, TTB_THREADS, (size_t)smem, as_stream(stream)>>>(qb);
        counted();
      }
    }
  }
  return last_error();
}

long long ttb_svd_work_doubles(int m, int k) {
  int M = std::max(m, k), K = std::min(m, k);
  return svd_tall_need(M, K);
}

int ttb_svd(const ttb_svd_t* ps, int count, void* stream) {
  if (int e = configure_smem()) return e;
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxS) {
    SBatch sb;
    sb.count = std::min(kMaxS, count - i0);
    i64 smem = 0;
    for (int j = 0; j < sb.count; ++j) {
      sb.d[j] = ps[i0 + j];
      const i64 whole = ttb_svd_work_doubles(sb.d[j].m, sb.d[j].k) * 8;
      const i64 blk = blocked_smem(std::min(sb.d[j].m, sb.d[j].k)) * 8;
      if (whole <= kSmemCap) {
        sb.mode[j] = 0;
        smem = std::max(smem, whole);
      } else {
        if (blk > kSmemCap) return (int)cudaErrorInvalidValue;
        sb.mode[j] = 1;
        smem = std::max(smem, blk);
      }
    }
    double fl = 0.0;
    for (int j = 0; j < sb.count; ++j) {
      // QR of the tall orientation, U = Q [U_R; 0] (Jacobi rotations not counted)
      const double M = std::max(sb.d[j].m, sb.d[j].k), k = std::min(sb.d[j].m, sb.d[j].k);
      fl += 4.0 * M * k * k - 4.0 / 3.0 * k * k * k;
    }
    ProfScope ps(P_SVD, s, fl, 0.0);
    k_svd<<<sb.count, TTB_THREADS, (size_t)smem, s>>>(sb);
    counted();
  }
  return last_error();
}

long long ttb_lu_work_doubles(int n) { return (long long)n * LNB; }

int ttb_lu_solve(const ttb_lu_t* ps, int count, void* stream) {
  if (int e = configure_smem()) return e;
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxL) {
    LBatch lb;
    lb.count = std::min(kMaxL, count - i0);
    i64 smem = 0;
    for (int j = 0; j < lb.count; ++j) {
      lb.d[j] = ps[i0 + j];
      const i64 n = lb.d[j].n;
      const i64 whole = (n * n + n) * 8, panel = n * LNB * 8;
      if (whole <= kSmemCap) {
        lb.mode[j] = 0;
        smem = std::max(smem, whole);
      } else if (panel <= kSmemCap) {
        lb.mode[j] = 1;
        smem = std::max(smem, panel);
      } else {
        if (lb.d[j].work == nullptr) return (int)cudaErrorInvalidValue;
        lb.mode[j] = 2;
      }
    }
    double fl = 0.0;
    for (int j = 0; j < lb.count; ++j) fl += 2.0 / 3.0 * std::pow((double)lb.d[j].n, 3.0);
    ProfScope ps(P_LU, s, fl, 0.0);
    k_lu<<<lb.count, TTB_THREADS, (size_t)smem, s>>>(lb);
    counted();
  }
  return last_error();
}

int ttb_copy(const ttb_copy_t* ps, int count, void* stream) {
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxC) {
    CBatch cb;
    cb.count = std::min(kMaxC, count - i0);
    long long most = 1;
    for (int j = 0; j < cb.count; ++j) {
      cb.d[j] = ps[i0 + j];
      most = std::max(most, (long long)cb.d[j].d0 * cb.d[j].d1 * cb.d[j].d2 * cb.d[j].d3);
    }
    dim3 grid((unsigned)std::min<long long>(cdiv(most, TTB_THREADS), 2048), cb.count);
    ProfScope ps(P_COPY, s, 0.0, 0.0);
    k_copy<<<grid, TTB_THREADS, 0, s>>>(cb);
    counted();
  }
  return last_error();
}

int ttb_kron(const ttb_kron_t* ps, int count, void* stream) {
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxK) {
    KBatch kb;
    kb.count = std::min(kMaxK, count - i0);
    long long most = 1;
    for (int j = 0; j < kb.count; ++j) {
      kb.d[j] = ps[i0 + j];
      const ttb_kron_t& q = kb.d[j];
      most = std::max(most, (long long)q.ra * q.rx * q.n * q.kk * q.ra2 * q.rx2);
    }
    dim3 grid((unsigned)std::min<long long>(cdiv(most, TTB_THREADS), 2048), kb.count);
    ProfScope ps(P_KRON, s, 0.0, 0.0);
    k_kron<<<grid, TTB_THREADS, 0, s>>>(kb);
    counted();
  }
  return last_error();
}

int ttb_hadamard(const ttb_hadamard_t* ps, int count, void* stream) {
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxK) {
    HBatch hb;
    hb.count = std::min(kMaxK, count - i0);
    long long most = 1;
    for (int j = 0; j < hb.count; ++j) {
      hb.d[j] = ps[i0 + j];
      const ttb_hadamard_t& q = hb.d[j];
      if (q.ra < 0 || q.ra2 < 0 || q.rx < 0 || q.rx2 < 0 || q.modes < 0) return (int)cudaErrorInvalidValue;
      most = std::max(most, (long long)q.ra * q.rx * q.modes * q.ra2 * q.rx2);
    }
    dim3 grid((unsigned)std::min<long long>(cdiv(most, TTB_THREADS), 2048), hb.count);
    ProfScope ps(P_KRON, s, 0.0, 0.0);
    k_hadamard<<<grid, TTB_THREADS, 0, s>>>(hb);
    counted();
  }
  return last_error();
}

int ttb_norm(const ttb_norm_t* ps, int count, void* stream) {
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxN) {
    NBatch nb;
    nb.count = std::min(kMaxN, count - i0);
    for (int j = 0; j < nb.count; ++j) nb.d[j] = ps[i0 + j];
    ProfScope ps(P_NORM, s, 0.0, 0.0);
    k_norm<<<nb.count, TTB_THREADS, 0, s>>>(nb);
    counted();
  }
  return last_error();
}

long long ttb_rank_work_doubles(long long n, int limit) {
  return (long long)cdiv(n, kRankChunk) * (limit + 1);
}

int ttb_rank_residual(const ttb_rank_t* ps, int count, void* stream) {
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxR) {
    RBatch rb;
    rb.count = std::min(kMaxR, count - i0);
    int most = 1;
    for (int j = 0; j < rb.count; ++j) {
      rb.d[j] = ps[i0 + j];
      rb.chunks[j] = std::max(1, cdiv(rb.d[j].n, kRankChunk));
      most = std::max(most, rb.chunks[j]);
    }
    ProfScope ps(P_RANK, s, 0.0, 0.0);
    k_rank_partial<<<dim3(most, rb.count), TTB_THREADS, 0, s>>>(rb);
    counted();
    k_rank_select<<<rb.count, 32, 0, s>>>(rb);
    counted();
  }
  return last_error();
}

int ttb_rank_threshold(const ttb_rank_rule_t* ps, int count, void* stream) {
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxRR) {
    RRBatch rb;
    rb.count = std::min(kMaxRR, count - i0);
    for (int j = 0; j < rb.count; ++j) rb.d[j] = ps[i0 + j];
    k_rank_rule<<<rb.count, 32, 0, s>>>(rb);
    counted();
  }
  return last_error();
}

long long ttb_minres_work_doubles(const ttb_krylov_t* p) {
  ttb_local_t op = p->op;
  op.cols = 1;
  const long long chunks = std::max(1, cdiv(p->n, kKryChunk));
  return 7 * p->n + chunks * 4 + 2 * kStateDoubles + local_work(op);
}

int ttb_minres(const ttb_krylov_t* ps, int count, int* flags, void* stream) {
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < count; i0 += kMaxKry) {
    const int nb = std::min(kMaxKry, count - i0);
    KBatchM kb, warm_b, cold_b;
    kb.count = nb;
    std::vector<ttb_local_t> mv(nb), warm_ops;
    int most = 1, maxit_all = 0;
    for (int j = 0; j < nb; ++j) {
      const ttb_krylov_t& p = ps[i0 + j];
      KDesc& d = kb.d[j];
      d.b = p.b;
      d.x = p.x;
      d.n = p.n;
      d.chunks = std::max(1, cdiv(p.n, kKryChunk));
      d.vec = p.work;
      d.part = p.work + 7 * p.n;
      d.st = d.part + (i64)d.chunks * 4;
      d.istop = p.istop;
      d.iters = p.iters;
      d.rtol = p.rtol;
      d.maxit = p.maxiter > 0 ? p.maxiter : (int)std::min<long long>(5 * p.n, 1 << 30);
      most = std::max(most, d.chunks);
      maxit_all = std::max(maxit_all, d.maxit);
      ttb_local_t op = p.op;
      op.cols = 1;
      op.alpha = 1.0;
      op.beta = 0.0;
      op.work = d.st + 2 * kStateDoubles;
      // iterations apply the operator to v and write y
      mv[j] = op;
      mv[j].x = d.vec + 3 * p.n;
      mv[j].y = d.vec + 2 * p.n;
      if (p.warm) {
        ttb_local_t w0 = op;
        w0.x = p.x;
        w0.y = d.vec + 2 * p.n;
        warm_ops.push_back(w0);
      }
    }
    warm_b = kb;
    cold_b = kb;
    for (int j = 0; j < nb; ++j) {
      if (ps[i0 + j].warm) cold_b.d[j].chunks = 0;
      else warm_b.d[j].chunks = 0;
    }
    int e;
    if (!warm_ops.empty() && (e = run_local(warm_ops.data(), (int)warm_ops.size(), s))) return e;
    k_minres_init<<<dim3(most, nb), TTB_THREADS, 0, s>>>(warm_b, 1);
    counted();
    k_minres_init<<<dim3(most, nb), TTB_THREADS, 0, s>>>(cold_b, 0);
    counted();
    k_minres_start<<<dim3(most, nb), TTB_THREADS, 0, s>>>(kb, 0.0);
    counted();
    std::vector<int> done_host(nb, 0);
    const int check_every = 8;
    for (int it = 0; it < maxit_all; ++it) {
      if ((e = run_local(mv.data(), nb, s))) return e;
      {
        double by = 0.0;
        for (int j = 0; j < nb; ++j) by += 8.0 * 19.0 * kb.d[j].n;  // vector reads + writes
        ProfScope ps(P_MINRES, s, 0.0, by);
        k_minres_a<<<dim3(most, nb), TTB_THREADS, 0, s>>>(kb, it);
        counted();
        k_minres_b<<<dim3(most, nb), TTB_THREADS, 0, s>>>(kb, it);
        counted();
        k_minres_c<<<dim3(most, nb), TTB_THREADS, 0, s>>>(kb, it);
        counted();
      }
      if ((it + 1) % check_every == 0 || it + 1 == maxit_all) {
        // evaluates the stop test of iteration ``it`` (state copy it + 1)
        k_minres_final<<<nb, 32, 0, s>>>(kb, it + 1, flags + i0);
        counted();
        if ((e = (int)cudaMemcpyAsync(done_host.data(), flags + i0, nb * sizeof(int),
                                      cudaMemcpyDeviceToHost, s)))
          return e;
        if ((e = (int)cudaStreamSynchronize(s))) return e;
        bool all = true;
        for (int j = 0; j < nb; ++j) all = all && done_host[j];
        if (all) break;
      }
    }
    if ((e = last_error())) return e;
  }
  return 0;
}


long long ttb_gmres_work_doubles(const ttb_krylov_t* p, int restart) {
  if (restart <= 0) restart = 20;
  ttb_local_t op = p->op;
  op.cols = 1;
  const long long R1 = restart + 1;
  return R1 * p->n + 2 * p->n + (long long)restart * R1 + 2LL * restart + R1 + G_NSTATE +
         local_work(op);
}

int ttb_gmres(const ttb_krylov_t* ps, int count, int restart, int* flags, void* stream) {
  cudaStream_t s = as_stream(stream);
  if (restart <= 0) restart = 20;
  if (restart > 63) return (int)cudaErrorInvalidValue;
  for (int i0 = 0; i0 < count; i0 += kMaxGm) {
    const int nb = std::min(kMaxGm, count - i0);
    GmBatch gb;
    gb.count = nb;
    std::vector<ttb_local_t> mv(nb), warm_ops, xo(nb);
    int warm_lo = 0, warm_hi = 0, maxiter = 0;
    for (int j = 0; j < nb; ++j) {
      const ttb_krylov_t& p = ps[i0 + j];
      GmDesc& g = gb.d[j];
      const int rs = std::min<long long>(restart, p.n) > 0 ? (int)std::min<long long>(restart, p.n) : 1;
      const i64 R1 = rs + 1;
      g.b = p.b;
      g.x = p.x;
      g.n = p.n;
      g.restart = rs;
      g.rtol = p.rtol;
      g.istop = p.istop;
      g.iters = p.iters;
      g.V = p.work;
      g.w = g.V + R1 * p.n;
      g.r = g.w + p.n;
      g.h = g.r + p.n;
      g.giv = g.h + (i64)rs * R1;
      g.S = g.giv + 2 * rs;
      g.st = g.S + R1;
      ttb_local_t op = p.op;
      op.cols = 1;
      op.alpha = 1.0;
      op.beta = 0.0;
      op.work = g.st + G_NSTATE;
      mv[j] = op;
      mv[j].y = g.w;
      xo[j] = op;
      xo[j].x = p.x;
      xo[j].y = g.w;
      if (p.warm) {
        warm_ops.push_back(xo[j]);
        if (j < 32) warm_lo |= 1 << j; else warm_hi |= 1 << (j - 32);
      }
      const int mi = p.maxiter > 0 ? p.maxiter : (int)std::min<long long>(10 * p.n, 1 << 30);
      maxiter = std::max(maxiter, mi);
    }
    int e;
    if (!warm_ops.empty() && (e = run_local(warm_ops.data(), (int)warm_ops.size(), s))) return e;
    k_gm_init<<<nb, TTB_THREADS, 0, s>>>(gb, warm_lo, warm_hi);
    counted();
    std::vector<int> fl(nb);
    for (int iteration = 0; iteration < maxiter; ++iteration) {
      k_gm_cycle<<<nb, TTB_THREADS, 0, s>>>(gb);
      counted();
      for (int col = 0; col < restart; ++col) {
        for (int j = 0; j < nb; ++j) mv[j].x = gb.d[j].V + (i64)std::min(col, gb.d[j].restart - 1) * gb.d[j].n;
        if ((e = run_local(mv.data(), nb, s))) return e;
        k_gm_arnoldi<<<nb, TTB_THREADS, 0, s>>>(gb, col);
        counted();
        k_gm_flags<<<nb, 32, 0, s>>>(gb, flags + i0, 0);
        counted();
        if ((e = (int)cudaMemcpyAsync(fl.data(), flags + i0, nb * sizeof(int),
                                      cudaMemcpyDeviceToHost, s)))
          return e;
        if ((e = (int)cudaStreamSynchronize(s))) return e;
        bool all = true;
        for (int j = 0; j < nb; ++j) all = all && fl[j];
        if (all) break;
      }
      k_gm_update<<<nb, TTB_THREADS, 0, s>>>(gb);
      counted();
      if ((e = run_local(xo.data(), nb, s))) return e;
      k_gm_outer<<<nb, TTB_THREADS, 0, s>>>(gb, iteration, maxiter);
      counted();
      k_gm_flags<<<nb, 32, 0, s>>>(gb, flags + i0, 1);
      counted();
      if ((e = (int)cudaMemcpyAsync(fl.data(), flags + i0, nb * sizeof(int),
                                    cudaMemcpyDeviceToHost, s)))
        return e;
      if ((e = (int)cudaStreamSynchronize(s))) return e;
      bool all = true;
      for (int j = 0; j < nb; ++j) all = all && fl[j];
      if (all) break;
    }
    if ((e = last_error())) return e;
  }
  return 0;
}

long long ttb_round_work_doubles(int d, int max_mode, int max_bond) {
  (void)max_mode;
  (void)max_bond;
  const long long qslot = (long long)kRoundMaxRows * kRoundMaxBond;
  return (long long)d * qslot + 3 * qslot + (long long)kRoundMaxBond * kRoundMaxBond +
         kRoundMaxRows;
}

int ttb_round_batch(const ttb_round_t* P, void* stream) {
  if (P->pairs <= 0) return 0;
  if (P->d < 2 || P->d > kRoundMaxD) return (int)cudaErrorInvalidValue;
  const size_t smem = ((size_t)kRoundMaxRows * kRoundMaxBond + kRoundMaxBond +
                       2 * (size_t)kRoundMaxBond * kRoundMaxBond + 3 * kRoundMaxBond + 2) *
                      sizeof(double);
  if (int e = smem_limit_once((const void*)k_round, (int)smem, g_smem_round)) return e;
  const long long qslot = (long long)kRoundMaxRows * kRoundMaxBond;
  const long long slot = qslot;
  ProfScope ps(P_ROUND, as_stream(stream), 0.0, 0.0);
  k_round<<<P->pairs, TTB_THREADS, smem, as_stream(stream)>>>(*P, slot, qslot);
  counted();
  return last_error();
}


void ttb_profile_enable(int mask) {
  if (mask == 0) prof_collect();
  g_prof_mask.store(mask);
}

int ttb_profile_read(int cls, double* ms, long long* launches, double* flops, double* bytes) {
  if (cls < 0 || cls >= P_CLASSES) return (int)cudaErrorInvalidValue;
  prof_collect();
  *ms = g_prof_ms[cls];
  *launches = g_prof_n[cls];
  *flops = g_prof_flops[cls];
  *bytes = g_prof_bytes[cls];
  return 0;
}

void ttb_profile_reset(void) {
  prof_collect();
  for (int i = 0; i < P_CLASSES; ++i) {
    g_prof_ms[i] = g_prof_flops[i] = g_prof_bytes[i] = 0.0;
    g_prof_n[i] = 0;
  }
}


int ttb_fma_peak(double* out, int blocks, int iters, void* stream) {
  k_fma_peak<<<blocks, TTB_THREADS, 0, as_stream(stream)>>>(out, iters);
  counted();
  return last_error();
}

}  // extern "C"
