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
// WHILE conditional node whose body is the step, continued by the last
// kernel while j < cycle and |y_j| > tol ||b||.  The host waits once per
// cycle.  Where the conditional graph cannot be built the host launches the
// same kernels step by step and reads the stop flag after each.
#include <cuda_runtime.h>

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

// partial[k * gridDim.x + b] = sum over block b's slice of V[:,k] . w
__global__ void dot_partials(const double* __restrict__ V, int64_t ld, const double* __restrict__ w, int64_t len,
                             double* __restrict__ partial) {
  const int k = blockIdx.y;
  const double* v = V + ld * k;
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    s += v[i] * w[i];
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[(int64_t)k * gridDim.x + blockIdx.x] = s;
  }
}

// out[k] = sum_b partial[k * nb + b] (fixed order), optionally sqrt
__global__ void reduce_partials(const double* __restrict__ partial, int nb, double* __restrict__ out, int take_sqrt) {
  const int k = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(int64_t)k * nb + b];
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[k] = take_sqrt ? sqrt(s) : s;
  }
}

// r = r - b ; then v0 = r / near0(||r||) is done by scale_by_norm
__global__ void sub_inplace(double* __restrict__ r, const double* __restrict__ b, int64_t len) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    r[i] -= b[i];
}

__global__ void scale_by_norm(double* __restrict__ v, const double* __restrict__ norm, int64_t len) {
  const double inv = 1.0 / near0(*norm);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    v[i] *= inv;
}

// Control block of the device-resident solver (after the scalars in d_scal).
struct KrylovCtl {
  double nrm_b;  // ||b||
  double h;      // norm of the newest Arnoldi vector before it is normalised
  double stop;   // tol * ||b||
  double last;   // |y_j| after the newest step
  int j;         // Arnoldi steps done in this cycle
  int cycle;     // step limit of this cycle
  int cont;      // 1 while the cycle goes on
  int pad;
};

__global__ void set_stop(KrylovCtl* ctl, double tol) { ctl->stop = tol * ctl->nrm_b; }

// y[0] = beta = ||r||; a new cycle starts at step 0
__global__ void cycle_start(KrylovCtl* ctl, double* y, int cycle) {
  y[0] = ctl->h;
  ctl->j = 0;
  ctl->cycle = cycle;
  ctl->cont = 1;
}

// gx = v_j; for j > 0 the newest column is normalised here first (by 1/h)
__global__ void arnoldi_load(double* __restrict__ V, int64_t len, const KrylovCtl* __restrict__ ctl,
                             double* __restrict__ gx) {
  const int j = ctl->j;
  double* vj = V + len * j;
  const double inv = j > 0 ? 1.0 / near0(ctl->h) : 1.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    double v = vj[i];
    if (j > 0) {
      v *= inv;
      vj[i] = v;
    }
    gx[i] = v;
  }
}

// partial[k * gridDim.x + b] = block b's share of V[:, k] . w for k <= j
__global__ void arnoldi_dots(const double* __restrict__ V, int64_t len, const double* __restrict__ w,
                             const KrylovCtl* __restrict__ ctl, double* __restrict__ partial) {
  const int j = ctl->j;
  __shared__ double red[kThreads / 32];
  for (int k = 0; k <= j; ++k) {
    const double* v = V + len * k;
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
      s += v[i] * w[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
      s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (threadIdx.x == 0) partial[(int64_t)k * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
  }
}

// U[j(j+1)/2 + k] = sum_b partial[k * nb + b] (fixed order), block k <= j
__global__ void arnoldi_reduce(const double* __restrict__ partial, int nb, const KrylovCtl* __restrict__ ctl,
                               double* __restrict__ U) {
  const int k = blockIdx.x, j = ctl->j;
  if (k > j) return;
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(int64_t)k * nb + b];
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) U[j * (j + 1) / 2 + k] = s;
  }
}

// V[:, j+1] = w - V[:, 0..j] u (u = U's column j), and block b's share of
// |V[:, j+1]|^2 into partial[b] (the same slices as arnoldi_dots)
__global__ void arnoldi_orth(double* __restrict__ V, int64_t len, const double* __restrict__ w,
                             const double* __restrict__ U, const KrylovCtl* __restrict__ ctl,
                             double* __restrict__ partial) {
  const int j = ctl->j;
  const double* u = U + j * (j + 1) / 2;
  double* out = V + len * (j + 1);
  double s2 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k <= j; ++k) s += V[len * k + i] * u[k];
    const double v = w[i] - s;
    out[i] = v;
    s2 += v * v;
  }
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
  __syncthreads();
  if (threadIdx.x < 32) {
    s2 = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s2;
  }
}

// h = ||V[:, j+1]|| from the partials (fixed order); the Givens step of
// column j (src/beep/beep.cpp:1399-1416); j += 1; the stop test
// (src/beep/beep.cpp:1421).  With a conditional handle the decision drives
// the graph's WHILE node.
__global__ void arnoldi_finish(const double* __restrict__ partial, int nb, double* __restrict__ U,
                               double* __restrict__ c, double* __restrict__ s, double* __restrict__ y,
                               KrylovCtl* __restrict__ ctl, cudaGraphConditionalHandle handle, int use_handle) {
  double acc = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) acc += partial[b];
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x != 0) return;
  acc = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) acc += red[w];
  const double h = sqrt(acc);
  const int j = ctl->j;
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
  const int cont = (j + 1 < ctl->cycle && last > ctl->stop) ? 1 : 0;
  ctl->h = h;
  ctl->j = j + 1;
  ctl->last = last;
  ctl->cont = cont;
  if (use_handle) cudaGraphSetConditional(handle, cont);
}

// Solve the packed upper-triangular U y = y (column-major, first j columns)
// unless U and y are both zero (src/beep/beep.cpp:1422-1426).
__global__ void packed_back_substitution(const double* __restrict__ U, const KrylovCtl* __restrict__ ctl,
                                         double* __restrict__ y) {
  const int j = ctl->j;
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

// x -= V[:, 0..j) y
__global__ void update_x(const double* __restrict__ V, int64_t ld, const KrylovCtl* __restrict__ ctl,
                         const double* __restrict__ y, double* __restrict__ x, int64_t len) {
  const int j = ctl->j;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < j; ++k) s += V[ld * k + i] * y[k];
    x[i] -= s;
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
  if (bytes <= 48 * 1024) return;  // the default limit
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

// Scalar block of the solver: U (m(m+1)/2), c (m), s (m), y (m+1), partial
// sums (kDotBlocks * (m+1)), then the control block.
struct KrylovView {
  double *U, *c, *s, *y, *partial;
  KrylovCtl* ctl;
};
size_t krylov_scalar_bytes(int m) {
  const size_t nd = (size_t)m * (m + 1) / 2 + 2 * (size_t)m + (m + 1) + (size_t)kDotBlocks * (m + 1);
  return sizeof(double) * nd + sizeof(KrylovCtl);
}
KrylovView krylov_view(Problem& P, int m) {
  KrylovView v;
  v.U = P.d_scal.as<double>();
  v.c = v.U + (size_t)m * (m + 1) / 2;
  v.s = v.c + m;
  v.y = v.s + m;
  v.partial = v.y + (m + 1);
  v.ctl = reinterpret_cast<KrylovCtl*>(v.partial + (size_t)kDotBlocks * (m + 1));
  return v;
}

// One Arnoldi step on stream st: v_j -> gx, the matvec into gy, the CGS
// orthogonalisation of gy into V[:, j+1] and the Givens step.  With a handle
// the last kernel sets the enclosing WHILE node's condition.
void arnoldi_step_launches(Problem& P, int m, cudaStream_t st, cudaGraphConditionalHandle handle, int use_handle) {
  const int64_t len = 2 * (int64_t)P.n;
  const KrylovView kv = krylov_view(P, m);
  double* V = P.d_V.as<double>();
  double* gx = P.d_gx.as<double>();
  double* gy = P.d_gy.as<double>();
  arnoldi_load<<<grid_for(len), kThreads, 0, st>>>(V, len, kv.ctl, gx);
  BP_LAUNCH_CHECK();
  matvec_launches(P, gx, gy, st, P.side, nullptr);
  arnoldi_dots<<<kDotBlocks, kThreads, 0, st>>>(V, len, gy, kv.ctl, kv.partial);
  arnoldi_reduce<<<m, kThreads, 0, st>>>(kv.partial, kDotBlocks, kv.ctl, kv.U);
  arnoldi_orth<<<kDotBlocks, kThreads, 0, st>>>(V, len, gy, kv.U, kv.ctl, kv.partial);
  arnoldi_finish<<<1, kThreads, 0, st>>>(kv.partial, kDotBlocks, kv.U, kv.c, kv.s, kv.y, kv.ctl, handle,
                                         use_handle);
  BP_LAUNCH_CHECK();
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

int gmres_device(Problem& P, const double* b_dev, double* x_dev, double tol, int max_iters, int restart,
                 double* rel_resid) {
  Ctx* ctx = P.ctx;
  cudaStream_t st = ctx->stream;
  const int64_t len = 2 * (int64_t)P.n;
  if (max_iters <= 0) throw std::invalid_argument("max_iters must be positive");
  const int m = (restart > 0 && restart < max_iters) ? restart : max_iters;
  if (P.krylov_m != m || !P.d_V.get()) {
    P.d_V.alloc(ctx, sizeof(double) * (size_t)len * (m + 1));
    P.d_scal.alloc(ctx, krylov_scalar_bytes(m));
    P.krylov_m = m;
  }
  double* V = P.d_V.as<double>();
  const KrylovView kv = krylov_view(P, m);
  auto norm_into = [&](const double* v, double* out) {
    dot_partials<<<dim3(kDotBlocks, 1), kThreads, 0, st>>>(v, len, v, len, kv.partial);
    reduce_partials<<<1, kThreads, 0, st>>>(kv.partial, kDotBlocks, out, 1);
  };
  const int g = grid_for(len);
  norm_into(b_dev, &kv.ctl->nrm_b);
  set_stop<<<1, 1, 0, st>>>(kv.ctl, tol);
  BP_LAUNCH_CHECK();
  const bool graph = ensure_gmres_graph(P, m);
  int total = 0;
  KrylovCtl h_ctl{};
  while (true) {
    BP_CUDA(cudaMemsetAsync(kv.U, 0, sizeof(double) * ((size_t)m * (m + 1) / 2 + 2 * m + (m + 1)), st));
    // r = A x - b into V[:,0], normalised; y[0] = beta
    matvec_device(P, x_dev, V);
    sub_inplace<<<g, kThreads, 0, st>>>(V, b_dev, len);
    norm_into(V, &kv.ctl->h);
    scale_by_norm<<<g, kThreads, 0, st>>>(V, &kv.ctl->h, len);
    cycle_start<<<1, 1, 0, st>>>(kv.ctl, kv.y, std::min(m, max_iters - total));
    BP_LAUNCH_CHECK();
    if (graph) {
      BP_CUDA(cudaGraphLaunch(P.gmres_graph, st));
    } else {
      while (true) {
        arnoldi_step_launches(P, m, st, cudaGraphConditionalHandle{}, 0);
        int cont = 0;
        BP_CUDA(cudaMemcpyAsync(&cont, &kv.ctl->cont, sizeof(int), cudaMemcpyDeviceToHost, st));
        BP_CUDA(cudaStreamSynchronize(st));
        if (!cont) break;
      }
    }
    packed_back_substitution<<<1, 1, 0, st>>>(kv.U, kv.ctl, kv.y);
    update_x<<<g, kThreads, 0, st>>>(V, len, kv.ctl, kv.y, x_dev, len);
    BP_LAUNCH_CHECK();
    BP_CUDA(cudaMemcpyAsync(&h_ctl, kv.ctl, sizeof(KrylovCtl), cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    total += h_ctl.j;
    if (h_ctl.last <= h_ctl.stop || total >= max_iters || restart <= 0) break;
  }
  if (rel_resid) *rel_resid = h_ctl.nrm_b > 0 ? h_ctl.last / h_ctl.nrm_b : 0.0;
  return total;
}

}  // namespace bp
