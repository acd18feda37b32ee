// Matvec driver and device-resident GMRES.
//
// GMRES restated from BEEP::gmres (src/beep/beep.cpp:1262-1483): residual
// r = A x - b, classical Gram-Schmidt Arnoldi (two dgemv per step), Givens
// rotations on a packed upper-triangular U (column j starts at j(j+1)/2),
// stop when |y_j| <= tol * ||b||, back substitution and x -= V y.  The
// reference runs a single cycle of max_iters; a positive `restart` repeats
// cycles of that length until convergence or max_iters.
//
// Everything stays on the device in FP64: V is (m+1) columns of 2N doubles,
// the dot products are deterministic two-pass reductions (fixed block
// partials, then one block per column), and the 2x2 rotations run in a
// single-thread step.  An Arnoldi step is five kernels (load v_j, V^T w
// partials, their sums, orthogonalisation fused with the partials of |w|^2,
// and the norm + Givens + stop test) plus the matvec, all reading the step
// index from device memory, so one cycle's whole loop is one CUDA graph: a
// WHILE conditional node whose body is the step, continued while j < cycle
// and |y_j| > tol ||b||.  The kernels after the matvec are programmatic
// dependent launches.  The host waits once per cycle.  Where the
// conditional graph cannot be built the host launches the same kernels
// step by step and reads the stop flag after each.
//
// A batch problem runs one GMRES per scenario in the same launches: every
// kernel takes the scenario from blockIdx.y (or one block per scenario)
// and works on the scenario's part of the vector, with its own control
// block, Hessenberg column, Givens rotations and stop test; a scenario that
// has converged sits out the rest of the steps, and the WHILE node goes on
// while any scenario does.  A solve from x = 0 starts from r = -b without
// the first matvec.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "engine.h"

namespace bp {

namespace {

constexpr int kThreads = 256;
constexpr int kDotBlocks = 296;  // 2 per SM on a 148-SM part

// DBL_MIN guard used by the reference to avoid 0/0 (src/beep/beep.cpp:1360)
__device__ __forceinline__ double near0(double v) { return v == 0.0 ? 2.2250738585072014e-308 : v; }

// r = -b: the residual of x = 0, where A x is exactly zero (every term of
// the near field and of the far field is a product with an entry of x)
__global__ void negate_into(double* __restrict__ r, const double* __restrict__ b, int64_t len) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = -b[i];
}

// flag = 1 if some entry of x is not zero
__global__ void any_nonzero(const double* __restrict__ x, int64_t len, int* __restrict__ flag) {
  int nz = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    nz |= x[i] != 0.0;
  if (__syncthreads_or(nz) && threadIdx.x == 0) *flag = 1;
}

// r = r - b ; then v0 = r / near0(||r||) is done by seg_scale_by_norm
__global__ void sub_inplace(double* __restrict__ r, const double* __restrict__ b, int64_t len) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    r[i] -= b[i];
}

// Scenarios of a batch problem each run their own GMRES on their part of
// the vector: scenario s owns entries [a, a+n) (the f half) and
// [N+a, N+a+n) (the h half); its local index i in [0, 2n) maps to a + i or
// N + a + i - n.  An ordinary problem is one scenario (a = 0, n = N).
struct Seg {
  int a, n;
};
__device__ __forceinline__ int64_t seg_at(Seg sg, int64_t N, int64_t i) {
  return i < sg.n ? sg.a + i : N + sg.a + (i - sg.n);
}

// Programmatic dependent launch (PTX griddepcontrol.wait): a kernel of the
// Arnoldi step launched as a programmatic dependent starts as the previous
// kernel on the stream retires its CTAs and waits here for that grid's
// completion and writes; it touches no memory before the wait.  Launched
// without the attribute the instruction does nothing.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
void launch_dependent(void (*kernel)(KArgs...), dim3 grid, unsigned block, cudaStream_t q, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(block);
  cfg.stream = q;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BP_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
}

// fixed-order block sum; the total is valid in thread 0
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;
}

// Control block of one scenario's solver (after the scalars in d_scal).
struct KrylovCtl {
  double nrm_b;  // ||b||
  double h;      // norm of the newest Arnoldi vector before it is normalised
  double stop;   // tol * ||b||
  double last;   // |y_j| after the newest step
  int j;         // Arnoldi steps done in this cycle
  int cycle;     // step limit of this cycle (0: the scenario sits it out)
  int cont;      // 1 while the cycle goes on
  int done;      // converged in an earlier step
  int iters;     // Arnoldi steps over all cycles
  int pad;
};
struct KrylovAll {
  int any;  // some scenario goes on
  int pad;
};

// partial[s * nbs + b] = block b's share of |v|^2 over scenario s
__global__ void seg_sq_partials(const double* __restrict__ v, const Seg* __restrict__ seg, int64_t N,
                                double* __restrict__ partial) {
  const int sc = blockIdx.y;
  const Seg sg = seg[sc];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 2 * (int64_t)sg.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double t = v[seg_at(sg, N, i)];
    s += t * t;
  }
  __shared__ double red[kThreads / 32];
  s = block_sum(s, red);
  if (threadIdx.x == 0) partial[(int64_t)sc * gridDim.x + blockIdx.x] = s;
}

// ctl[s].nrm_b = sqrt(sum of the partials); the stop level; a fresh solve
__global__ void norm_b_finish(const double* __restrict__ partial, int nbs, KrylovCtl* __restrict__ ctl, double tol) {
  const int sc = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nbs; b += blockDim.x) s += partial[(int64_t)sc * nbs + b];
  __shared__ double red[kThreads / 32];
  s = block_sum(s, red);
  if (threadIdx.x == 0) {
    KrylovCtl& c = ctl[sc];
    c.nrm_b = sqrt(s);
    c.stop = tol * c.nrm_b;
    c.done = 0;
    c.iters = 0;
    c.last = 0.0;
  }
}

// ctl[s].h = ||r|| of the scenario
__global__ void norm_r_finish(const double* __restrict__ partial, int nbs, KrylovCtl* __restrict__ ctl) {
  const int sc = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nbs; b += blockDim.x) s += partial[(int64_t)sc * nbs + b];
  __shared__ double red[kThreads / 32];
  s = block_sum(s, red);
  if (threadIdx.x == 0) ctl[sc].h = sqrt(s);
}

// v0 = r / near0(||r||) for the scenarios still solving
__global__ void seg_scale_by_norm(double* __restrict__ v, const Seg* __restrict__ seg, int64_t N,
                                  const KrylovCtl* __restrict__ ctl) {
  const int sc = blockIdx.y;
  if (ctl[sc].done) return;
  const Seg sg = seg[sc];
  const double inv = 1.0 / near0(ctl[sc].h);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 2 * (int64_t)sg.n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[seg_at(sg, N, i)] *= inv;
}

// y[0] = beta = ||r||; a new cycle starts at step 0 for every scenario not
// yet converged
__global__ void cycle_start(KrylovCtl* __restrict__ ctl, int n_scen, double* __restrict__ y0, int64_t ks,
                            int64_t y_off, int cycle, KrylovAll* __restrict__ all) {
  const int sc = blockIdx.x * blockDim.x + threadIdx.x;
  if (sc == 0) all->any = 1;
  if (sc >= n_scen) return;
  KrylovCtl& c = ctl[sc];
  y0[sc * ks + y_off] = c.h;
  c.j = 0;
  c.cycle = c.done ? 0 : cycle;
  c.cont = c.done ? 0 : 1;
}

// gx = v_j; for j > 0 the newest column is normalised here first (by 1/h)
__global__ void arnoldi_load(double* __restrict__ V, int64_t len, const Seg* __restrict__ seg,
                             const KrylovCtl* __restrict__ ctl, double* __restrict__ gx) {
  const int sc = blockIdx.y;
  if (!ctl[sc].cont) return;
  const Seg sg = seg[sc];
  const int64_t N = len / 2;
  const int j = ctl[sc].j;
  double* vj = V + len * j;
  const double inv = j > 0 ? 1.0 / near0(ctl[sc].h) : 1.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 2 * (int64_t)sg.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = seg_at(sg, N, i);
    double v = vj[g];
    if (j > 0) {
      v *= inv;
      vj[g] = v;
    }
    gx[g] = v;
  }
}

// partial_s[k * nbs + b] = block b's share of V[:, k] . w over scenario s,
// k <= j (partial_s = partial + s * (m+1) * nbs)
__global__ void arnoldi_dots(const double* __restrict__ V, int64_t len, const double* __restrict__ w,
                             const Seg* __restrict__ seg, const KrylovCtl* __restrict__ ctl, int m,
                             double* __restrict__ partial) {
  pdl_wait();
  const int sc = blockIdx.y;
  if (!ctl[sc].cont) return;
  const Seg sg = seg[sc];
  const int64_t N = len / 2;
  const int j = ctl[sc].j, nbs = gridDim.x;
  double* part = partial + (int64_t)sc * (m + 1) * nbs;
  __shared__ double red[kThreads / 32];
  for (int k = 0; k <= j; ++k) {
    const double* v = V + len * k;
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 2 * (int64_t)sg.n;
         i += (int64_t)gridDim.x * blockDim.x) {
      const int64_t g = seg_at(sg, N, i);
      s += v[g] * w[g];
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[(int64_t)k * nbs + blockIdx.x] = s;
  }
}

// U_s[j(j+1)/2 + k] = sum_b partial_s[k * nbs + b] (fixed order), block k <= j
__global__ void arnoldi_reduce(const double* __restrict__ partial, int nbs, const KrylovCtl* __restrict__ ctl, int m,
                               double* __restrict__ U0, int64_t ks) {
  pdl_wait();
  const int k = blockIdx.x, sc = blockIdx.y;
  if (!ctl[sc].cont) return;
  const int j = ctl[sc].j;
  if (k > j) return;
  const double* part = partial + (int64_t)sc * (m + 1) * nbs;
  double s = 0.0;
  for (int b = threadIdx.x; b < nbs; b += blockDim.x) s += part[(int64_t)k * nbs + b];
  __shared__ double red[kThreads / 32];
  s = block_sum(s, red);
  if (threadIdx.x == 0) U0[sc * ks + j * (j + 1) / 2 + k] = s;
}

// V[:, j+1] = w - V[:, 0..j] u (u = U_s's column j) over scenario s, and
// block b's share of |V[:, j+1]|^2 into partial_s[b] (the slices of
// arnoldi_dots)
__global__ void arnoldi_orth(double* __restrict__ V, int64_t len, const double* __restrict__ w,
                             const double* __restrict__ U0, int64_t ks, const Seg* __restrict__ seg,
                             const KrylovCtl* __restrict__ ctl, int m, double* __restrict__ partial) {
  pdl_wait();
  const int sc = blockIdx.y;
  if (!ctl[sc].cont) return;
  const Seg sg = seg[sc];
  const int64_t N = len / 2;
  const int j = ctl[sc].j;
  const double* u = U0 + sc * ks + j * (j + 1) / 2;
  double* out = V + len * (j + 1);
  double s2 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 2 * (int64_t)sg.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = seg_at(sg, N, i);
    double s = 0.0;
    for (int k = 0; k <= j; ++k) s += V[len * k + g] * u[k];
    const double v = w[g] - s;
    out[g] = v;
    s2 += v * v;
  }
  __shared__ double red[kThreads / 32];
  s2 = block_sum(s2, red);
  if (threadIdx.x == 0) partial[(int64_t)sc * (m + 1) * gridDim.x + blockIdx.x] = s2;
}

// One block per scenario: h = ||V[:, j+1]|| from the partials (fixed order);
// the Givens step of column j (src/beep/beep.cpp:1399-1416); j += 1; the
// stop test (src/beep/beep.cpp:1421).  With a conditional handle and one
// scenario the decision drives the graph's WHILE node (with several,
// any_continue does).
__global__ void arnoldi_finish(const double* __restrict__ partial, int nbs, int m, double* __restrict__ U0,
                               int64_t ks, KrylovCtl* __restrict__ ctl, cudaGraphConditionalHandle handle,
                               int use_handle) {
  pdl_wait();
  const int sc = blockIdx.x;
  if (!ctl[sc].cont) return;
  const double* part = partial + (int64_t)sc * (m + 1) * nbs;
  double acc = 0.0;
  for (int b = threadIdx.x; b < nbs; b += blockDim.x) acc += part[b];
  __shared__ double red[kThreads / 32];
  acc = block_sum(acc, red);
  if (threadIdx.x != 0) return;
  double* U = U0 + sc * ks;
  double* c = U + m * (m + 1) / 2;
  double* s = c + m;
  double* y = s + m;
  KrylovCtl& C = ctl[sc];
  const double h = sqrt(acc);
  const int j = C.j;
  int uij = j * (j + 1) / 2;
  for (int i = 0; i < j; ++i) {
    const double tmp = c[i] * U[uij] - s[i] * U[uij + 1];
    U[uij + 1] = s[i] * U[uij] + c[i] * U[uij + 1];
    U[uij] = tmp;
    ++uij;
  }
  const double rd = U[uij];
  const double dd = sqrt(rd * rd + h * h);
  c[j] = rd / near0(dd);
  s[j] = -h / near0(dd);
  U[uij] = dd;
  y[j + 1] = s[j] * y[j];
  y[j] = c[j] * y[j];
  const double last = fabs(y[j + 1]);
  const int cont = (j + 1 < C.cycle && last > C.stop) ? 1 : 0;
  C.h = h;
  C.j = j + 1;
  C.last = last;
  C.cont = cont;
  if (last <= C.stop) C.done = 1;
  if (use_handle && gridDim.x == 1) cudaGraphSetConditional(handle, cont);
}

// all->any = some scenario goes on; drives the WHILE node of a batch
__global__ void any_continue(const KrylovCtl* __restrict__ ctl, int n_scen, KrylovAll* __restrict__ all,
                             cudaGraphConditionalHandle handle, int use_handle) {
  pdl_wait();
  int any = 0;
  for (int sc = threadIdx.x; sc < n_scen; sc += blockDim.x) any |= ctl[sc].cont;
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    all->any = any;
    if (use_handle) cudaGraphSetConditional(handle, any);
  }
}

// Per scenario: solve the packed upper-triangular U y = y (column-major,
// first j columns) unless U and y are both zero (src/beep/beep.cpp:1422-1426);
// count the cycle's steps.
__global__ void packed_back_substitution(double* __restrict__ U0, int64_t ks, int m, KrylovCtl* __restrict__ ctl,
                                         int n_scen) {
  const int sc = blockIdx.x * blockDim.x + threadIdx.x;
  if (sc >= n_scen) return;
  const double* U = U0 + sc * ks;
  double* y = U0 + sc * ks + m * (m + 1) / 2 + 2 * m;
  const int j = ctl[sc].j;
  ctl[sc].iters += j;
  double su = 0.0, sy = 0.0;
  const int uij = j * (j + 1) / 2;
  for (int k = 0; k < uij; ++k) su += fabs(U[k]);
  for (int k = 0; k < j; ++k) sy += fabs(y[k]);
  if (su == 0.0 && sy == 0.0) return;
  for (int i = j - 1; i >= 0; --i) {
    double t = y[i];
    for (int k = i + 1; k < j; ++k) t -= U[k * (k + 1) / 2 + i] * y[k];
    y[i] = t / U[i * (i + 1) / 2 + i];
  }
}

// x -= V[:, 0..j) y over each scenario
__global__ void update_x(const double* __restrict__ V, int64_t len, const Seg* __restrict__ seg,
                         const KrylovCtl* __restrict__ ctl, const double* __restrict__ U0, int64_t ks, int m,
                         double* __restrict__ x) {
  const int sc = blockIdx.y;
  const int j = ctl[sc].j;
  if (j == 0) return;
  const Seg sg = seg[sc];
  const int64_t N = len / 2;
  const double* y = U0 + sc * ks + m * (m + 1) / 2 + 2 * m;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 2 * (int64_t)sg.n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = seg_at(sg, N, i);
    double s = 0.0;
    for (int k = 0; k < j; ++k) s += V[len * k + g] * y[k];
    x[g] -= s;
  }
}

inline int grid_for(int64_t len) {
  int64_t g = (len + kThreads - 1) / kThreads;
  if (g > 4 * 148) g = 4 * 148;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace

void ensure_dynamic_smem(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> granted;
  // the default limit holds static and dynamic shared memory together
  cudaFuncAttributes fa;
  BP_CUDA(cudaFuncGetAttributes(&fa, kernel));
  if (bytes + fa.sharedSizeBytes <= 48 * 1024) return;
  int dev = 0;
  BP_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = granted[{dev, kernel}];
  if (bytes <= cur) return;
  BP_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  // kernels with this much shared memory run more blocks per SM with the
  // largest shared-memory carveout
  BP_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  cur = bytes;
}

void matvec_setup(Problem& P) {
  Ctx* c = P.ctx;
  const size_t bytes = sizeof(double) * 2 * (size_t)P.n;
  P.d_yfar.alloc(c, bytes);
  P.d_gx.alloc(c, bytes);
  P.d_gy.alloc(c, bytes);
  // the FMM stream carries the far field's critical chain (P2M, M2M, L2L,
  // L2P) and has the highest priority; the per-level streams it forks (M2X,
  // X2L) have lower ones
  int lo = 0, hi = 0;
  BP_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  BP_CUDA(cudaStreamCreateWithPriority(&P.side, cudaStreamNonBlocking, hi));
  BP_CUDA(cudaEventCreateWithFlags(&P.ev_fork, cudaEventDisableTiming));
  BP_CUDA(cudaEventCreateWithFlags(&P.ev_join, cudaEventDisableTiming));
  // a pinned word, so that reading the status behind a result is a plain
  // asynchronous copy, not a staged one
  BP_CUDA(cudaHostAlloc((void**)&P.h_status, sizeof(int), cudaHostAllocDefault));
}

// One matvec as kernel launches: the near field on `main` (writes y), the
// FMM on `side` into the far-field buffer, joined and added on `main`.  With
// side == main everything is serial (the profiling path).
static void matvec_launches(Problem& P, const double* x, double* y, cudaStream_t main, cudaStream_t side,
                            StageTimes* st) {
  const bool far = fmm_active(P);
  const int64_t len = 2 * (int64_t)P.n;
  // The far field first, then the near field, which adds it in its store.
  // They do not run side by side: the near field is an HBM-bound stream of
  // about a gigabyte that evicts the FMM's L2-resident expansions, operators
  // and plane waves and raises the memory latency the FMM's small kernels
  // wait on, so together they take longer than one after the other.
  if (far) {
    if (side != main) {
      // the FMM runs on its own stream (and one stream per level inside)
      BP_CUDA(cudaEventRecord(P.ev_fork, main));
      BP_CUDA(cudaStreamWaitEvent(side, P.ev_fork, 0));
      fmm_apply(P, x, P.d_yfar.as<double>(), st, side);  // assigns every far-field entry
      BP_CUDA(cudaEventRecord(P.ev_join, side));
      BP_CUDA(cudaStreamWaitEvent(main, P.ev_join, 0));
    } else {
      fmm_apply(P, x, P.d_yfar.as<double>(), st, main);
    }
  }
  if (st) st->begin(0, main);
  const int launches = nf_apply(P, x, y, far ? P.d_yfar.as<double>() : nullptr, main);  // writes every y entry
  if (!launches) {  // no near-field work (not produced by the tree builder): y = far field only
    if (far)
      BP_CUDA(cudaMemcpyAsync(y, P.d_yfar.get(), sizeof(double) * len, cudaMemcpyDeviceToDevice, main));
    else
      BP_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * len, main));
  }
  if (st) st->end(launches);
  (void)len;
}

// Captures matvec_launches(d_gx -> d_gy) as a CUDA graph on first use.
static bool ensure_graph(Problem& P) {
  if (P.graph) return true;
  if (P.graph_failed) return false;
  cudaStream_t s = P.ctx->stream;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    P.graph_failed = true;
    return false;
  }
  bool ok = true;
  try {
    matvec_launches(P, P.d_gx.as<double>(), P.d_gy.as<double>(), s, P.side, nullptr);
  } catch (const CudaError&) {
    ok = false;
  }
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (!ok || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    P.graph_failed = true;
    return false;
  }
  // node priorities (taken from the capturing streams) are kept in the graph
  e = cudaGraphInstantiateWithFlags(&P.graph, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    P.graph = nullptr;
    P.graph_failed = true;
    return false;
  }
  return true;
}

void matvec_device(Problem& P, const double* x_dev, double* y_dev, StageTimes* st) {
  cudaStream_t s = P.ctx->stream;
  if (st) {  // profiling: serial launches with per-stage events
    matvec_launches(P, x_dev, y_dev, s, s, st);
    return;
  }
  if (ensure_graph(P)) {
    const size_t bytes = sizeof(double) * 2 * (size_t)P.n;
    if (x_dev != P.d_gx.as<double>())
      BP_CUDA(cudaMemcpyAsync(P.d_gx.get(), x_dev, bytes, cudaMemcpyDeviceToDevice, s));
    BP_CUDA(cudaGraphLaunch(P.graph, s));
    if (y_dev != P.d_gy.as<double>())
      BP_CUDA(cudaMemcpyAsync(y_dev, P.d_gy.get(), bytes, cudaMemcpyDeviceToDevice, s));
    return;
  }
  matvec_launches(P, x_dev, y_dev, s, P.side, nullptr);
}

namespace {

// Scalar block of the solver, per scenario s: U (m(m+1)/2), c (m), s (m),
// y (m+1) at s * ks; then the dot partials ((m+1) * nbs per scenario), the
// control blocks and the batch flag.
struct KrylovView {
  double* U0;  // scenario s's U at U0 + s * ks, then its c, s, y
  int64_t ks;
  double* partial;
  KrylovCtl* ctl;
  KrylovAll* all;
  int nbs;  // dot-product blocks per scenario
  int gx;   // elementwise blocks per scenario
};
int dot_blocks(int n_scen) { return n_scen == 1 ? kDotBlocks : std::max(16, kDotBlocks / n_scen); }
int64_t scal_stride(int m) { return (int64_t)m * (m + 1) / 2 + 2 * (int64_t)m + (m + 1); }
size_t krylov_scalar_bytes(int m, int n_scen) {
  const size_t nd = (size_t)n_scen * (scal_stride(m) + (size_t)(m + 1) * dot_blocks(n_scen));
  return sizeof(double) * nd + sizeof(KrylovCtl) * n_scen + sizeof(KrylovAll);
}
KrylovView krylov_view(Problem& P, int m) {
  const int S = P.n_scen();
  KrylovView v;
  v.ks = scal_stride(m);
  v.nbs = dot_blocks(S);
  v.U0 = P.d_scal.as<double>();
  v.partial = v.U0 + S * v.ks;
  v.ctl = reinterpret_cast<KrylovCtl*>(v.partial + (size_t)S * (m + 1) * v.nbs);
  v.all = reinterpret_cast<KrylovAll*>(v.ctl + S);
  int nmax = 1;
  for (int s = 0; s < S; ++s) nmax = std::max(nmax, P.scen_first[s + 1] - P.scen_first[s]);
  v.gx = std::max(1, std::min(grid_for(2 * (int64_t)nmax), S == 1 ? 4 * 148 : std::max(4, 4 * 148 / S)));
  return v;
}

// One Arnoldi step of every scenario still solving, on stream st: v_j -> gx,
// the matvec into gy, the CGS orthogonalisation of gy into V[:, j+1] and the
// Givens step.  With a handle the last kernel sets the enclosing WHILE
// node's condition.
void arnoldi_step_launches(Problem& P, int m, cudaStream_t st, cudaGraphConditionalHandle handle, int use_handle) {
  const int64_t len = 2 * (int64_t)P.n;
  const int S = P.n_scen();
  const KrylovView kv = krylov_view(P, m);
  const Seg* seg = P.d_seg.as<Seg>();
  double* V = P.d_V.as<double>();
  double* gx = P.d_gx.as<double>();
  double* gy = P.d_gy.as<double>();
  arnoldi_load<<<dim3(kv.gx, S), kThreads, 0, st>>>(V, len, seg, kv.ctl, gx);
  BP_LAUNCH_CHECK();
  matvec_launches(P, gx, gy, st, P.side, nullptr);
  // the dot products follow the near-field kernel on st; the rest of the
  // step is a chain of dependent launches
  launch_dependent(arnoldi_dots, dim3(kv.nbs, S), kThreads, st, (const double*)V, len, (const double*)gy, seg,
                   (const KrylovCtl*)kv.ctl, m, kv.partial);
  launch_dependent(arnoldi_reduce, dim3(m, S), kThreads, st, (const double*)kv.partial, kv.nbs,
                   (const KrylovCtl*)kv.ctl, m, kv.U0, kv.ks);
  launch_dependent(arnoldi_orth, dim3(kv.nbs, S), kThreads, st, V, len, (const double*)gy, (const double*)kv.U0,
                   kv.ks, seg, (const KrylovCtl*)kv.ctl, m, kv.partial);
  launch_dependent(arnoldi_finish, dim3(S), kThreads, st, (const double*)kv.partial, kv.nbs, m, kv.U0, kv.ks, kv.ctl,
                   handle, use_handle);
  if (S > 1)
    launch_dependent(any_continue, dim3(1), kThreads, st, (const KrylovCtl*)kv.ctl, S, kv.all, handle, use_handle);
}

// The Arnoldi loop of one cycle as a graph: a WHILE node (condition 1 at
// every launch) whose body is one step.  False when this CUDA build or
// device cannot make it; the caller then drives the same step from the host.
bool ensure_gmres_graph(Problem& P, int m) {
  if (P.gmres_graph && P.gmres_graph_m == m && P.gmres_graph_v == P.d_V.get()) return true;
  if (P.gmres_graph_failed) return false;
  if (P.gmres_graph) {
    cudaGraphExecDestroy(P.gmres_graph);
    P.gmres_graph = nullptr;
  }
  cudaStream_t s = P.ctx->stream;
  cudaGraph_t g = nullptr;
  bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
  cudaGraphConditionalHandle handle{};
  cudaGraphNode_t node{};
  cudaGraphNodeParams cp = {};
  if (ok) ok = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
  if (ok) {
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    ok = cudaGraphAddNode(&node, g, nullptr, 0, &cp) == cudaSuccess;
  }
  if (ok) ok = cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    bool launched = true;
    try {
      arnoldi_step_launches(P, m, s, handle, 1);
    } catch (const CudaError&) {
      launched = false;
    }
    cudaGraph_t body = nullptr;
    ok = cudaStreamEndCapture(s, &body) == cudaSuccess && launched;
  }
  if (ok) ok = cudaGraphInstantiateWithFlags(&P.gmres_graph, g, cudaGraphInstantiateFlagUseNodePriority) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    cudaGetLastError();
    if (P.gmres_graph) cudaGraphExecDestroy(P.gmres_graph);
    P.gmres_graph = nullptr;
    P.gmres_graph_failed = true;
    return false;
  }
  P.gmres_graph_m = m;
  P.gmres_graph_v = P.d_V.get();
  return true;
}

}  // namespace

bool device_all_zero(Problem& P, const double* x_dev, int64_t len) {
  cudaStream_t st = P.ctx->stream;
  DevBuf flag(P.ctx, sizeof(int));
  BP_CUDA(cudaMemsetAsync(flag.get(), 0, sizeof(int), st));
  any_nonzero<<<grid_for(len), kThreads, 0, st>>>(x_dev, len, flag.as<int>());
  BP_LAUNCH_CHECK();
  int h = 0;
  BP_CUDA(cudaMemcpyAsync(&h, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  return h == 0;
}

int gmres_device(Problem& P, const double* b_dev, double* x_dev, double tol, int max_iters, int restart,
                 double* rel_resid, int* iters, bool x_is_zero) {
  Ctx* ctx = P.ctx;
  cudaStream_t st = ctx->stream;
  const int64_t len = 2 * (int64_t)P.n;
  const int S = P.n_scen();
  if (max_iters <= 0) throw std::invalid_argument("max_iters must be positive");
  const int m = (restart > 0 && restart < max_iters) ? restart : max_iters;
  if (P.krylov_m != m || !P.d_V.get()) {
    P.d_V.alloc(ctx, sizeof(double) * (size_t)len * (m + 1));
    P.d_scal.alloc(ctx, krylov_scalar_bytes(m, S));
    P.krylov_m = m;
  }
  if (!P.d_seg.get()) {
    std::vector<Seg> seg(S);
    for (int s = 0; s < S; ++s) seg[s] = {P.scen_first[s], P.scen_first[s + 1] - P.scen_first[s]};
    P.d_seg = upload(ctx, seg);
  }
  const Seg* seg = P.d_seg.as<Seg>();
  double* V = P.d_V.as<double>();
  const KrylovView kv = krylov_view(P, m);
  const int sb = (S + kThreads - 1) / kThreads;
  seg_sq_partials<<<dim3(kv.nbs, S), kThreads, 0, st>>>(b_dev, seg, P.n, kv.partial);
  norm_b_finish<<<S, kThreads, 0, st>>>(kv.partial, kv.nbs, kv.ctl, tol);
  BP_LAUNCH_CHECK();
  const bool graph = ensure_gmres_graph(P, m);
  int total = 0;
  std::vector<KrylovCtl> h_ctl(S);
  bool x_zero = x_is_zero;
  while (true) {
    BP_CUDA(cudaMemsetAsync(kv.U0, 0, sizeof(double) * (size_t)S * kv.ks, st));
    // r = A x - b into V[:,0], normalised per scenario; y[0] = beta (for
    // x = 0, -b: the same bits without the matvec)
    if (x_zero) {
      negate_into<<<grid_for(len), kThreads, 0, st>>>(V, b_dev, len);
      x_zero = false;
    } else {
      matvec_device(P, x_dev, V);
      sub_inplace<<<grid_for(len), kThreads, 0, st>>>(V, b_dev, len);
    }
    seg_sq_partials<<<dim3(kv.nbs, S), kThreads, 0, st>>>(V, seg, P.n, kv.partial);
    norm_r_finish<<<S, kThreads, 0, st>>>(kv.partial, kv.nbs, kv.ctl);
    seg_scale_by_norm<<<dim3(kv.gx, S), kThreads, 0, st>>>(V, seg, P.n, kv.ctl);
    cycle_start<<<sb, kThreads, 0, st>>>(kv.ctl, S, kv.U0, kv.ks, (int64_t)m * (m + 1) / 2 + 2 * m,
                                         std::min(m, max_iters - total), kv.all);
    BP_LAUNCH_CHECK();
    if (graph) {
      BP_CUDA(cudaGraphLaunch(P.gmres_graph, st));
    } else {
      while (true) {
        arnoldi_step_launches(P, m, st, cudaGraphConditionalHandle{}, 0);
        int cont = 0;
        if (S == 1)
          BP_CUDA(cudaMemcpyAsync(&cont, &kv.ctl->cont, sizeof(int), cudaMemcpyDeviceToHost, st));
        else
          BP_CUDA(cudaMemcpyAsync(&cont, &kv.all->any, sizeof(int), cudaMemcpyDeviceToHost, st));
        BP_CUDA(cudaStreamSynchronize(st));
        if (!cont) break;
      }
    }
    packed_back_substitution<<<sb, kThreads, 0, st>>>(kv.U0, kv.ks, m, kv.ctl, S);
    update_x<<<dim3(kv.gx, S), kThreads, 0, st>>>(V, len, seg, kv.ctl, kv.U0, kv.ks, m, x_dev);
    BP_LAUNCH_CHECK();
    BP_CUDA(cudaMemcpyAsync(h_ctl.data(), kv.ctl, sizeof(KrylovCtl) * S, cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    int steps = 0;
    bool all_done = true;
    for (const KrylovCtl& c : h_ctl) {
      steps = std::max(steps, c.j);
      all_done = all_done && c.last <= c.stop;
    }
    total += steps;
    if (all_done || total >= max_iters || restart <= 0) break;
  }
  int worst = 0;
  for (int s = 0; s < S; ++s) {
    const KrylovCtl& c = h_ctl[s];
    if (rel_resid) rel_resid[s] = c.nrm_b > 0 ? c.last / c.nrm_b : 0.0;
    if (iters) iters[s] = c.iters;
    worst = std::max(worst, c.iters);
  }
  return worst;
}

}  // namespace bp
