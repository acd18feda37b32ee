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
// single-thread kernel.  The host only reads the residual estimate once per
// Arnoldi step to decide whether to stop.
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

// w -= V[:, 0..ncols) * u
__global__ void orth_update(const double* __restrict__ V, int64_t ld, int ncols, const double* __restrict__ u,
                            double* __restrict__ w, int64_t len) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < ncols; ++k) s += V[ld * k + i] * u[k];
    w[i] -= s;
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

// x -= V[:, 0..j) y
__global__ void update_x(const double* __restrict__ V, int64_t ld, int j, const double* __restrict__ y,
                         double* __restrict__ x, int64_t len) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < j; ++k) s += V[ld * k + i] * y[k];
    x[i] -= s;
  }
}

// Givens step for Arnoldi column j (src/beep/beep.cpp:1399-1416).
// U[u0j .. u0j+j] holds V^T w; h = ||w|| after orthogonalisation.
__global__ void givens_step(double* __restrict__ U, int u0j, int j, const double* __restrict__ hptr,
                            double* __restrict__ c, double* __restrict__ s, double* __restrict__ y) {
  int uij = u0j;
  const double h = *hptr;
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
}

// Solve the packed upper-triangular U y = y (column-major, first j columns)
// unless U and y are both zero (src/beep/beep.cpp:1422-1426).
__global__ void packed_back_substitution(const double* __restrict__ U, int j, double* __restrict__ y) {
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

__global__ void set_scalar(double* p, const double* src) { *p = *src; }

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

int gmres_device(Problem& P, const double* b_dev, double* x_dev, double tol, int max_iters, int restart,
                 double* rel_resid) {
  Ctx* ctx = P.ctx;
  cudaStream_t st = ctx->stream;
  const int64_t len = 2 * (int64_t)P.n;
  if (max_iters <= 0) throw std::invalid_argument("max_iters must be positive");
  const int m = (restart > 0 && restart < max_iters) ? restart : max_iters;
  if (P.krylov_m != m || !P.d_V.get()) {
    P.d_V.alloc(ctx, sizeof(double) * (size_t)len * (m + 1));
    // scalars: U (m(m+1)/2), c (m), s (m), y (m+1), norms (4), partials
    size_t nscal = (size_t)m * (m + 1) / 2 + 2 * m + (m + 1) + 8 + (size_t)kDotBlocks * (m + 1);
    P.d_scal.alloc(ctx, sizeof(double) * nscal);
    P.krylov_m = m;
  }
  double* V = P.d_V.as<double>();
  double* U = P.d_scal.as<double>();
  double* c = U + (size_t)m * (m + 1) / 2;
  double* s = c + m;
  double* y = s + m;
  double* norms = y + (m + 1);  // [0] = ||b||, [1] = scratch norm
  double* partial = norms + 8;
  auto dots = [&](const double* Vb, int ncols, const double* w, double* out, bool take_sqrt) {
    dim3 g(kDotBlocks, ncols);
    dot_partials<<<g, kThreads, 0, st>>>(Vb, len, w, len, partial);
    reduce_partials<<<ncols, kThreads, 0, st>>>(partial, kDotBlocks, out, take_sqrt ? 1 : 0);
  };
  const int g = grid_for(len);
  // ||b||
  dots(b_dev, 1, b_dev, norms, true);
  double nrm2b = 0.0;
  BP_CUDA(cudaMemcpyAsync(&nrm2b, norms, sizeof(double), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  const double stop = tol * nrm2b;
  int total = 0;
  double last = 0.0;
  while (true) {
    BP_CUDA(cudaMemsetAsync(U, 0, sizeof(double) * ((size_t)m * (m + 1) / 2 + 2 * m + (m + 1)), st));
    // r = A x - b into V[:,0], normalise, y[0] = beta
    matvec_device(P, x_dev, V);
    sub_inplace<<<g, kThreads, 0, st>>>(V, b_dev, len);
    dots(V, 1, V, norms + 1, true);
    set_scalar<<<1, 1, 0, st>>>(y, norms + 1);
    scale_by_norm<<<g, kThreads, 0, st>>>(V, norms + 1, len);
    BP_LAUNCH_CHECK();
    int j = 0, uij = 0;
    const int cycle = std::min(m, max_iters - total);
    while (true) {
      const int u0j = uij;
      double* vj = V + len * j;
      double* w = V + len * (j + 1);
      matvec_device(P, vj, w);
      dots(V, j + 1, w, U + u0j, false);
      orth_update<<<g, kThreads, 0, st>>>(V, len, j + 1, U + u0j, w, len);
      dots(w, 1, w, norms + 1, true);
      scale_by_norm<<<g, kThreads, 0, st>>>(w, norms + 1, len);
      givens_step<<<1, 1, 0, st>>>(U, u0j, j, norms + 1, c, s, y);
      BP_LAUNCH_CHECK();
      uij += j + 1;
      ++j;
      double yj = 0.0;
      BP_CUDA(cudaMemcpyAsync(&yj, y + j, sizeof(double), cudaMemcpyDeviceToHost, st));
      BP_CUDA(cudaStreamSynchronize(st));
      last = std::fabs(yj);
      if (!(j < cycle && last > stop)) break;
    }
    packed_back_substitution<<<1, 1, 0, st>>>(U, j, y);
    update_x<<<g, kThreads, 0, st>>>(V, len, j, y, x_dev, len);
    BP_LAUNCH_CHECK();
    total += j;
    if (last <= stop || total >= max_iters || restart <= 0) break;
  }
  BP_CUDA(cudaStreamSynchronize(st));
  if (rel_resid) *rel_resid = nrm2b > 0 ? last / nrm2b : 0.0;
  return total;
}

}  // namespace bp
