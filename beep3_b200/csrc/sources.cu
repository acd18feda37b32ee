// Point-charge sources: right-hand side and energy coefficients.
//
// RHS (BEEP::set_rhs, src/beep/beep.cpp:1124-1260): at every qualocation
// point q of patch i, phi(q) = sum_c q_c/|x_q - x_c| and grad phi;
//   f_rhs[i] = sum_q w_q phi(q) / (4 pi eps_solvent)
//   h_rhs[i] = sum_q w_q grad phi(q) . n_q / (4 pi eps_solvent).
// The reference evaluates phi with its 6-figure vanilla FMM; here the sum is
// direct (exact in FP64), tiled through shared memory.
//
// Energy coefficients (Mesh::init_energy_precalcs, src/bem/mesh.cpp:730-925):
// at the galerkin points of each patch, from the charges of its own mesh,
//   ec_f[i] = sum_g (grad phi . n_g) w_g / (4 pi),  ec_h[i] = sum_g phi w_g / (4 pi)
// followed by the Gauss-law renormalisation of ec_f
// (Mesh::renormalise_energy_precalcs, src/bem/mesh.cpp:905-925).
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "engine.h"

namespace bp {

namespace {

constexpr int kThreads = 256;
constexpr double kOneOver4Pi = 0.07957747154594767;

// 1/sqrt(d2) for d2 > 0 in double precision: the single-precision estimate
// refined by two Newton-Raphson steps y <- y (3 - d2 y^2) / 2 (each step
// roughly squares the relative error: ~2^-22 -> ~2^-44 -> double rounding),
// far cheaper than the double-precision reciprocal square root.
__device__ __forceinline__ double rsqrt_newton(double d2) {
  double y = (double)rsqrtf((float)d2);
  y = y * (1.5 - 0.5 * d2 * y * y);
  y = y * (1.5 - 0.5 * d2 * y * y);
  return y;
}

// One thread per point; charges staged through shared memory in tiles.
// out[2*p] = w * phi * scale, out[2*p+1] = w * (grad phi . n) * scale,
// exact in FP64.
__global__ void point_potential_kernel(const double* __restrict__ pts, int npts, int first_pt, int count_pts,
                                       const double* __restrict__ charges, int nc, double scale,
                                       double* __restrict__ out) {
  __shared__ double4 tile[kThreads];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = k < count_pts;
  const int p = first_pt + k;
  double x = 0, y = 0, z = 0;
  if (active) {
    x = pts[p];
    y = pts[(size_t)npts + p];
    z = pts[2 * (size_t)npts + p];
  }
  double phi = 0, gx = 0, gy = 0, gz = 0;
  for (int base = 0; base < nc; base += kThreads) {
    const int c = base + threadIdx.x;
    if (c < nc) tile[threadIdx.x] = make_double4(charges[4 * c], charges[4 * c + 1], charges[4 * c + 2], charges[4 * c + 3]);
    __syncthreads();
    const int lim = min(kThreads, nc - base);
    if (active)
      for (int t = 0; t < lim; ++t) {
        const double4 ch = tile[t];
        const double dx = x - ch.x, dy = y - ch.y, dz = z - ch.z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 > 2.220446049250313e-16) {
          const double id = rsqrt_newton(d2);
          const double pt = ch.w * id;
          const double ft = -pt * id * id;
          phi += pt;
          gx += ft * dx;
          gy += ft * dy;
          gz += ft * dz;
        }
      }
    __syncthreads();
  }
  if (active) {
    const double w = pts[6 * (size_t)npts + p];
    const double nx = pts[3 * (size_t)npts + p], ny = pts[4 * (size_t)npts + p], nz = pts[5 * (size_t)npts + p];
    out[2 * k] = w * phi * scale;
    out[2 * k + 1] = w * (gx * nx + gy * ny + gz * nz) * scale;
  }
}

// The mixed engine's right-hand side terms: the same sums with FP32 terms.
// Points and charges are held as two-float (hi + lo) offsets from the
// block's first point, converted once, so the coordinate differences come
// out to FP32 rounding without any per-term conversion; the reciprocal
// distance and the terms are FP32, summed per tile in FP32 and across tiles
// in FP64 -- about 1e-7 relative per term, in line with the reference, whose
// right-hand side comes from a 6-figure FMM.  Each thread takes two points
// (kPtsPerThread), so every charge read from shared memory serves both, and
// a coincident charge and point give a zero term by a select, not a branch.
constexpr int kPtsPerThread = 2;
__global__ void __launch_bounds__(kThreads) point_potential_fast_kernel(const double* __restrict__ pts, int npts,
                                                                        const double* __restrict__ charges, int nc,
                                                                        double scale, double* __restrict__ out) {
  __shared__ float4 th[kThreads], tl[kThreads];
  constexpr int P = kPtsPerThread;
  const int p0 = blockIdx.x * (P * kThreads);  // the block's first point: origin of the offsets
  const double ox = pts[min(p0, npts - 1)], oy = pts[(size_t)npts + min(p0, npts - 1)],
               oz = pts[2 * (size_t)npts + min(p0, npts - 1)];
  auto split = [](double v, float& hi, float& lo) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
  };
  float xh[P], xl[P], yh[P], yl[P], zh[P], zl[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int p = min(p0 + j * kThreads + (int)threadIdx.x, npts - 1);
    split(pts[p] - ox, xh[j], xl[j]);
    split(pts[(size_t)npts + p] - oy, yh[j], yl[j]);
    split(pts[2 * (size_t)npts + p] - oz, zh[j], zl[j]);
  }
  double phi[P], gx[P], gy[P], gz[P];
#pragma unroll
  for (int j = 0; j < P; ++j) phi[j] = gx[j] = gy[j] = gz[j] = 0.0;
  for (int base = 0; base < nc; base += kThreads) {
    const int c = base + threadIdx.x;
    if (c < nc) {
      float4 h, l;
      split(charges[4 * c] - ox, h.x, l.x);
      split(charges[4 * c + 1] - oy, h.y, l.y);
      split(charges[4 * c + 2] - oz, h.z, l.z);
      h.w = (float)charges[4 * c + 3];
      l.w = 0.f;
      th[threadIdx.x] = h;
      tl[threadIdx.x] = l;
    }
    __syncthreads();
    const int lim = min(kThreads, nc - base);
    float fphi[P], fgx[P], fgy[P], fgz[P];
#pragma unroll
    for (int j = 0; j < P; ++j) fphi[j] = fgx[j] = fgy[j] = fgz[j] = 0.f;
#pragma unroll 4
    for (int t = 0; t < lim; ++t) {
      const float4 h = th[t], l = tl[t];
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const float dx = (xh[j] - h.x) + (xl[j] - l.x), dy = (yh[j] - h.y) + (yl[j] - l.y),
                    dz = (zh[j] - h.z) + (zl[j] - l.z);
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float id = d2 > 2.220446049250313e-16f ? rsqrtf(d2) : 0.f;
        const float pt = h.w * id;
        const float ft = -pt * id * id;
        fphi[j] += pt;
        fgx[j] = fmaf(ft, dx, fgx[j]);
        fgy[j] = fmaf(ft, dy, fgy[j]);
        fgz[j] = fmaf(ft, dz, fgz[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < P; ++j) {
      phi[j] += fphi[j];
      gx[j] += fgx[j];
      gy[j] += fgy[j];
      gz[j] += fgz[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int p = p0 + j * kThreads + (int)threadIdx.x;
    if (p >= npts) continue;
    const double w = pts[6 * (size_t)npts + p];
    const double nx = pts[3 * (size_t)npts + p], ny = pts[4 * (size_t)npts + p], nz = pts[5 * (size_t)npts + p];
    out[2 * (size_t)p] = w * phi[j] * scale;
    out[2 * (size_t)p + 1] = w * (gx[j] * nx + gy[j] * ny + gz[j] * nz) * scale;
  }
}

// Per-patch sums of the per-point values (fixed order: deterministic).
__global__ void sum_points_kernel(const int32_t* __restrict__ off, int first, int count, int pt_base,
                                  const double* __restrict__ vals, double* __restrict__ a, double* __restrict__ b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int i = first + k;
  double s0 = 0, s1 = 0;
  for (int p = off[i]; p < off[i + 1]; ++p) {
    s0 += vals[2 * (p - pt_base)];
    s1 += vals[2 * (p - pt_base) + 1];
  }
  a[k] = s0;
  b[k] = s1;
}

}  // namespace

void rhs_device(Problem& P, const double* charges_dev, int n_charges, double eps_solvent, double* rhs_dev) {
  // FP64 engine: exact FP64 sum; mixed engine: the fast FP32 terms
  Ctx* ctx = P.ctx;
  const int nq = P.n_qual_pts;
  DevBuf& vals = P.scratch_vals;
  if (vals.bytes() < sizeof(double) * 2 * (size_t)nq) vals.alloc(ctx, sizeof(double) * 2 * (size_t)nq);
  const double scale = kOneOver4Pi / eps_solvent;
  if (P.fp64)
    point_potential_kernel<<<(nq + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(
        P.d_qual.as<double>(), nq, 0, nq, charges_dev, n_charges, scale, vals.as<double>());
  else
    point_potential_fast_kernel<<<(nq + kPtsPerThread * kThreads - 1) / (kPtsPerThread * kThreads), kThreads, 0,
                                  ctx->stream>>>(P.d_qual.as<double>(), nq, charges_dev, n_charges, scale,
                                                 vals.as<double>());
  BP_LAUNCH_CHECK();
  sum_points_kernel<<<(P.n + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(
      P.d_qual_off.as<int32_t>(), 0, P.n, 0, vals.as<double>(), rhs_dev, rhs_dev + P.n);
  BP_LAUNCH_CHECK();
  BP_CUDA(cudaStreamSynchronize(ctx->stream));
}

void energy_coefficients_device(Problem& P, int first, int count, const double* charges_dev, int n_charges,
                                double* cf_dev, double* ch_dev) {
  Ctx* ctx = P.ctx;
  const int ng = P.n_gal_pts;
  const int p0 = P.h_gal_off[first], p1 = P.h_gal_off[first + count];
  DevBuf vals(ctx, sizeof(double) * 2 * (size_t)std::max(1, p1 - p0));
  if (p1 > p0) {
    point_potential_kernel<<<(p1 - p0 + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(
        P.d_gal.as<double>(), ng, p0, p1 - p0, charges_dev, n_charges, kOneOver4Pi, vals.as<double>());
    BP_LAUNCH_CHECK();
  }
  // vals[2p] -> ec_h (potential), vals[2p+1] -> ec_f (normal field)
  sum_points_kernel<<<(count + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(
      P.d_gal_off.as<int32_t>(), first, count, p0, vals.as<double>(), ch_dev, cf_dev);
  BP_LAUNCH_CHECK();
  BP_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace bp

// ---------------------------------------------------------------------------
// Right-hand side without any device allocation.
//
// For callers that cannot allocate device memory themselves: code running
// inside a host application whose allocator owns the whole GPU (a pooled
// or pre-reserved heap), code that must not call cudaMalloc while another
// thread may be capturing a CUDA graph, or embedded users given fixed
// device buffers.  The per-point scratch of the right-hand-side kernels
// lives in a fixed file-scope device array instead of a cudaMalloc'd
// buffer; the caller passes inputs and outputs as device pointers.
//
// The array holds kNoAllocMaxPoints points (2 doubles each, 16 MiB) on every
// GPU that loads this library, until the process exits.  Every call shares
// it: calls that overlap on the GPU (different streams, or different host
// threads on the same device) race on it and must be serialised by the
// caller.  Each call writes every scratch entry it later reads, so nothing
// has to start at zero.
namespace bp {
namespace {

constexpr int kNoAllocMaxPoints = 1 << 20;
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxPoints];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array for the current device.  Host code
// cannot use the symbol itself as a device pointer, so the address is
// looked up once per device, with that device current, and cached.
double* noalloc_scratch_for_current_device() {
  int dev = -1;
  BP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw std::invalid_argument("device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    BP_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_addr[dev];
}

}  // namespace
}  // namespace bp

extern "C" BP_API int32_t bp_rhs_noalloc(int32_t n_patches, const int32_t* qual_offsets_dev,
                                         const double* qual_points_soa_dev, int32_t n_qual_points,
                                         const double* charges_xyzq_dev, int32_t n_charges, double eps_solvent,
                                         double* rhs_dev, void* cuda_stream) {
  using namespace bp;
  return guarded_engine([&]() -> int32_t {
    if (n_patches <= 0 || n_qual_points <= 0 || !qual_offsets_dev || !qual_points_soa_dev || !rhs_dev ||
        n_charges < 0 || (n_charges > 0 && !charges_xyzq_dev) || !(eps_solvent > 0))
      return fail(BP_ERR_INVALID, "bp_rhs_noalloc: bad argument");
    if (n_qual_points > kNoAllocMaxPoints)
      return fail(BP_ERR_INVALID, "bp_rhs_noalloc: " + std::to_string(n_qual_points) +
                                      " qualocation points exceed the fixed scratch of " +
                                      std::to_string(kNoAllocMaxPoints) + " points");
    double* scratch = noalloc_scratch_for_current_device();
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    const double scale = kOneOver4Pi / eps_solvent;
    point_potential_kernel<<<(n_qual_points + kThreads - 1) / kThreads, kThreads, 0, st>>>(
        qual_points_soa_dev, n_qual_points, 0, n_qual_points, charges_xyzq_dev, n_charges, scale, scratch);
    BP_LAUNCH_CHECK();
    sum_points_kernel<<<(n_patches + kThreads - 1) / kThreads, kThreads, 0, st>>>(
        qual_offsets_dev, 0, n_patches, 0, scratch, rhs_dev, rhs_dev + n_patches);
    BP_LAUNCH_CHECK();
    return BP_OK;
  });
}

