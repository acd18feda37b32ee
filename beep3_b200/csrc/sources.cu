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

#include <algorithm>
#include <cstring>

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
// For point p = first_pt + k: out[2k] = w * phi * scale, out[2k+1] =
// w * (grad phi . n) * scale, exact in FP64, plus add[2k], add[2k+1] when
// add is set.
__global__ void point_potential_kernel(const double* __restrict__ pts, int npts, int first_pt, int count_pts,
                                       const double* __restrict__ charges, int nc, double scale,
                                       double* __restrict__ out, const double* __restrict__ add) {
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
    const size_t o = 2 * (size_t)k;
    const double a0 = add ? add[o] : 0.0, a1 = add ? add[o + 1] : 0.0;
    out[o] = w * phi * scale + a0;
    out[o + 1] = w * (gx * nx + gy * ny + gz * nz) * scale + a1;
  }
}

// The mixed engine's right-hand side terms: the same sums with FP32 terms.
// Points and charges are held as two-float (hi + lo) offsets from the
// block's first point, converted once, so the coordinate differences come
// out to FP32 rounding without any per-term conversion; the reciprocal
// distance (the hardware approximation, PTX rsqrt.approx.ftz: r^2 below the
// FP32 normal range is a coincident pair, zeroed by the guard anyway) and
// the terms are FP32, summed in FP32 over runs of kFp32Run charges and
// across runs in FP64 -- about 1e-7 relative per term, 6e-7 on a whole sum
// of 2000 charges of mixed signs, in line with the reference, whose
// right-hand side comes from a 6-figure FMM.  Each thread takes four points
// (kPtsPerThread), so every charge read from shared memory serves all four,
// and a coincident charge and point give a zero term by a select, not a
// branch.  Measured on 1.97 M points x 2000 charges: 2.8 ms, against 3.45 ms
// with two points per thread, rsqrtf and FP32 runs of 256.
constexpr int kPtsPerThread = 4;
constexpr int kFp32Run = 64;
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// Points first_pt .. first_pt + count_pts - 1 of the list (stride npts);
// outputs and the optional addend are indexed from first_pt.
__global__ void __launch_bounds__(kThreads) point_potential_fast_kernel(const double* __restrict__ pts, int npts,
                                                                        int first_pt, int count_pts,
                                                                        const double* __restrict__ charges, int nc,
                                                                        double scale, double* __restrict__ out,
                                                                        const double* __restrict__ add) {
  __shared__ float4 th[kThreads], tl[kThreads];
  constexpr int P = kPtsPerThread;
  const int p0 = blockIdx.x * (P * kThreads);  // the block's first point: origin of the offsets
  const int po = first_pt + min(p0, count_pts - 1);
  const double ox = pts[po], oy = pts[(size_t)npts + po], oz = pts[2 * (size_t)npts + po];
  auto split = [](double v, float& hi, float& lo) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
  };
  float xh[P], xl[P], yh[P], yl[P], zh[P], zl[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int p = first_pt + min(p0 + j * kThreads + (int)threadIdx.x, count_pts - 1);
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
    for (int t0 = 0; t0 < lim; t0 += kFp32Run) {
      const int t1 = min(lim, t0 + kFp32Run);
      float fphi[P], fgx[P], fgy[P], fgz[P];
#pragma unroll
      for (int j = 0; j < P; ++j) fphi[j] = fgx[j] = fgy[j] = fgz[j] = 0.f;
#pragma unroll 4
      for (int t = t0; t < t1; ++t) {
        const float4 h = th[t], l = tl[t];
#pragma unroll
        for (int j = 0; j < P; ++j) {
          const float dx = (xh[j] - h.x) + (xl[j] - l.x), dy = (yh[j] - h.y) + (yl[j] - l.y),
                      dz = (zh[j] - h.z) + (zl[j] - l.z);
          const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          float id = rsqrt_ftz(d2);
          id = d2 > 2.220446049250313e-16f ? id : 0.f;
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
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int k = p0 + j * kThreads + (int)threadIdx.x;
    if (k >= count_pts) continue;
    const int p = first_pt + k;
    const double w = pts[6 * (size_t)npts + p];
    const double nx = pts[3 * (size_t)npts + p], ny = pts[4 * (size_t)npts + p], nz = pts[5 * (size_t)npts + p];
    const double a0 = add ? add[2 * (size_t)k] : 0.0, a1 = add ? add[2 * (size_t)k + 1] : 0.0;
    out[2 * (size_t)k] = w * phi[j] * scale + a0;
    out[2 * (size_t)k + 1] = w * (gx[j] * nx + gy[j] * ny + gz[j] * nz) * scale + a1;
  }
}

// Per-patch sums of the per-point values (fixed order: deterministic).
// vals holds n_vals points starting at point pt_base; a patch's offsets are
// clamped to that range, so offsets that do not describe the list (not
// non-decreasing, or past its end) never read outside it.
__global__ void sum_points_kernel(const int32_t* __restrict__ off, int first, int count, int pt_base, int n_vals,
                                  const double* __restrict__ vals, double* __restrict__ a, double* __restrict__ b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int i = first + k;
  const int lo = max(off[i] - pt_base, 0), hi = min(off[i + 1] - pt_base, n_vals);
  double s0 = 0, s1 = 0;
  for (int p = lo; p < hi; ++p) {
    s0 += vals[2 * (size_t)p];
    s1 += vals[2 * (size_t)p + 1];
  }
  a[k] = s0;
  b[k] = s1;
}

// The mixed engine's terms over points taken in spatial order (an order
// list; outputs at the points' own indices), each block splitting the
// charges by distance.  The block's origin is the centre of its points' box
// (half-diagonal rho).  A charge farther than kFarRatio x rho from it has a
// coordinate offset about as large as the distance itself, so one FP32 word
// per offset keeps the difference to ~1.5e-7 of the distance, and it cannot
// coincide with a point: those charges take a loop without the low words and
// without the coincidence guard (about 14 instead of 22 instructions a
// term).  Nearer charges take the two-word loop of
// point_potential_fast_kernel.  A block whose points are scattered (no
// spatial order) has a large rho and sends every charge down the near loop:
// slower, never less accurate.  The near and far lists are compacted by
// ballots in charge order, so the sums are deterministic.  Measured on
// 1.97 M points in patch clusters x 2000 charges: 2.23 ms (96% far) against
// 2.83 ms for point_potential_fast_kernel.
constexpr float kFarRatio = 3.f;
__global__ void __launch_bounds__(kThreads) point_potential_split_kernel(
    const double* __restrict__ pts, int npts, const int32_t* __restrict__ order, int first_pt, int count_pts,
    const double* __restrict__ charges, int nc, double scale, double* __restrict__ out,
    const double* __restrict__ add) {
  constexpr int P = kPtsPerThread;
  constexpr int W = kThreads / 32;
  __shared__ float4 nh[kThreads], nl[kThreads], fh[kThreads];
  __shared__ double red[6][W];
  __shared__ int wcnt[2][W];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b0 = blockIdx.x * (P * kThreads);
  auto split = [](double v, float& hi, float& lo) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
  };
  int idx[P];
  double px[P], py[P], pz[P];
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
#pragma unroll
  for (int j = 0; j < P; ++j) {
    idx[j] = order[first_pt + min(b0 + j * kThreads + tid, count_pts - 1)];
    px[j] = pts[idx[j]];
    py[j] = pts[(size_t)npts + idx[j]];
    pz[j] = pts[2 * (size_t)npts + idx[j]];
    mn[0] = fmin(mn[0], px[j]);
    mn[1] = fmin(mn[1], py[j]);
    mn[2] = fmin(mn[2], pz[j]);
    mx[0] = fmax(mx[0], px[j]);
    mx[1] = fmax(mx[1], py[j]);
    mx[2] = fmax(mx[2], pz[j]);
  }
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  if (lane == 0)
    for (int d = 0; d < 3; ++d) {
      red[d][warp] = mn[d];
      red[3 + d][warp] = mx[d];
    }
  __syncthreads();
  for (int d = 0; d < 3; ++d) {
    mn[d] = red[d][0];
    mx[d] = red[3 + d][0];
    for (int w = 1; w < W; ++w) {
      mn[d] = fmin(mn[d], red[d][w]);
      mx[d] = fmax(mx[d], red[3 + d][w]);
    }
  }
  const double cx = 0.5 * (mn[0] + mx[0]), cy = 0.5 * (mn[1] + mx[1]), cz = 0.5 * (mn[2] + mx[2]);
  const double ex = mx[0] - mn[0], ey = mx[1] - mn[1], ez = mx[2] - mn[2];
  const double far = fmax((double)kFarRatio * 0.5 * sqrt(ex * ex + ey * ey + ez * ez), 1e-6);
  const double far2 = far * far;
  float xh[P], xl[P], yh[P], yl[P], zh[P], zl[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    split(px[j] - cx, xh[j], xl[j]);
    split(py[j] - cy, yh[j], yl[j]);
    split(pz[j] - cz, zh[j], zl[j]);
  }
  double phi[P], gx[P], gy[P], gz[P];
#pragma unroll
  for (int j = 0; j < P; ++j) phi[j] = gx[j] = gy[j] = gz[j] = 0.0;
  for (int base = 0; base < nc; base += kThreads) {
    const int c = base + tid;
    const bool valid = c < nc;
    double ox = 0, oy = 0, oz = 0, q = 0;
    bool is_far = false;
    if (valid) {
      ox = charges[4 * (size_t)c] - cx;
      oy = charges[4 * (size_t)c + 1] - cy;
      oz = charges[4 * (size_t)c + 2] - cz;
      q = charges[4 * (size_t)c + 3];
      is_far = ox * ox + oy * oy + oz * oz > far2;
    }
    const unsigned mf = __ballot_sync(0xffffffffu, valid && is_far);
    const unsigned mnr = __ballot_sync(0xffffffffu, valid && !is_far);
    if (lane == 0) {
      wcnt[0][warp] = __popc(mf);
      wcnt[1][warp] = __popc(mnr);
    }
    __syncthreads();
    int of = 0, on = 0, tf = 0, tn = 0;
    for (int w = 0; w < W; ++w) {
      if (w < warp) {
        of += wcnt[0][w];
        on += wcnt[1][w];
      }
      tf += wcnt[0][w];
      tn += wcnt[1][w];
    }
    const unsigned below = (1u << lane) - 1u;
    if (valid && is_far) fh[of + __popc(mf & below)] = make_float4((float)ox, (float)oy, (float)oz, (float)q);
    if (valid && !is_far) {
      float4 h, l;
      split(ox, h.x, l.x);
      split(oy, h.y, l.y);
      split(oz, h.z, l.z);
      h.w = (float)q;
      l.w = 0.f;
      const int pos = on + __popc(mnr & below);
      nh[pos] = h;
      nl[pos] = l;
    }
    __syncthreads();
    for (int t0 = 0; t0 < tf; t0 += kFp32Run) {
      const int t1 = min(tf, t0 + kFp32Run);
      float fphi[P], fgx[P], fgy[P], fgz[P];
#pragma unroll
      for (int j = 0; j < P; ++j) fphi[j] = fgx[j] = fgy[j] = fgz[j] = 0.f;
#pragma unroll 4
      for (int t = t0; t < t1; ++t) {
        const float4 h = fh[t];
#pragma unroll
        for (int j = 0; j < P; ++j) {
          const float dx = xh[j] - h.x, dy = yh[j] - h.y, dz = zh[j] - h.z;
          const float id = rsqrt_ftz(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
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
    }
    for (int t0 = 0; t0 < tn; t0 += kFp32Run) {
      const int t1 = min(tn, t0 + kFp32Run);
      float fphi[P], fgx[P], fgy[P], fgz[P];
#pragma unroll
      for (int j = 0; j < P; ++j) fphi[j] = fgx[j] = fgy[j] = fgz[j] = 0.f;
      for (int t = t0; t < t1; ++t) {
        const float4 h = nh[t], l = nl[t];
#pragma unroll
        for (int j = 0; j < P; ++j) {
          const float dx = (xh[j] - h.x) + (xl[j] - l.x), dy = (yh[j] - h.y) + (yl[j] - l.y),
                      dz = (zh[j] - h.z) + (zl[j] - l.z);
          const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          float id = rsqrt_ftz(d2);
          id = d2 > 2.220446049250313e-16f ? id : 0.f;
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
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < P; ++j) {
    if (b0 + j * kThreads + tid >= count_pts) continue;
    const int p = idx[j];
    const size_t k = 2 * (size_t)(p - first_pt);
    const double w = pts[6 * (size_t)npts + p];
    const double nx = pts[3 * (size_t)npts + p], ny = pts[4 * (size_t)npts + p], nz = pts[5 * (size_t)npts + p];
    const double a0 = add ? add[k] : 0.0, a1 = add ? add[k + 1] : 0.0;
    out[k] = w * phi[j] * scale + a0;
    out[k + 1] = w * (gx[j] * nx + gy[j] * ny + gz[j] * nz) * scale + a1;
  }
}

// order[start[k] + i] = off[patch[k]] + i: the points of the patches in the
// given order
__global__ void expand_order_kernel(int n, const int32_t* __restrict__ patch, const int32_t* __restrict__ start,
                                    const int32_t* __restrict__ off, int32_t* __restrict__ order) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int p = patch[k], a = off[p], c = off[p + 1] - a, s = start[k];
  for (int i = 0; i < c; ++i) order[s + i] = a + i;
}

// The spatial point order of P (built once): per instance (all patches for a
// problem without instances), its patches in the tree's leaf order, so the
// order list keeps every instance's points in the instance's own range.
const int32_t* qual_order(Problem& P) {
  if (P.d_qual_order.get()) return P.d_qual_order.as<int32_t>();
  const int n = P.n;
  std::vector<int> inst_of(n, 0), inst_first{0};
  for (const Placement& pl : P.placements) inst_first.push_back(inst_first.back() + pl.mesh->n);
  if (P.placements.empty()) inst_first.push_back(n);
  const int ni = (int)inst_first.size() - 1;
  for (int k = 0; k < ni; ++k)
    for (int i = inst_first[k]; i < inst_first[k + 1]; ++i) inst_of[i] = k;
  std::vector<std::vector<int32_t>> by_inst(ni);
  std::vector<char> seen(n, 0);
  for (const TreeNode& nd : P.tree.nodes) {
    if (!(nd.flags & TREE_LEAF)) continue;
    for (int32_t c = 0; c < nd.content_count; ++c) {
      const int p = P.tree.contents[nd.content_start + c];
      if (!seen[p]) by_inst[inst_of[p]].push_back(p);
      seen[p] = 1;
    }
  }
  for (int p = 0; p < n; ++p)
    if (!seen[p]) by_inst[inst_of[p]].push_back(p);  // leaves partition the patches; kept for safety
  std::vector<int32_t> patch, start;
  patch.reserve(n);
  start.reserve(n);
  for (int k = 0; k < ni; ++k) {
    int s = P.h_qual_off[inst_first[k]];
    for (int p : by_inst[k]) {
      patch.push_back(p);
      start.push_back(s);
      s += P.h_qual_off[p + 1] - P.h_qual_off[p];
    }
  }
  Ctx* ctx = P.ctx;
  DevBuf d_patch = upload(ctx, patch), d_start = upload(ctx, start);
  P.d_qual_order.alloc(ctx, sizeof(int32_t) * (size_t)std::max(1, P.n_qual_pts));
  expand_order_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(
      n, d_patch.as<int32_t>(), d_start.as<int32_t>(), P.d_qual_off.as<int32_t>(), P.d_qual_order.as<int32_t>());
  BP_LAUNCH_CHECK();
  BP_CUDA(cudaStreamSynchronize(ctx->stream));  // the host lists go out of scope
  return P.d_qual_order.as<int32_t>();
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
        P.d_qual.as<double>(), nq, 0, nq, charges_dev, n_charges, scale, vals.as<double>(), nullptr);
  else
    point_potential_split_kernel<<<(nq + kPtsPerThread * kThreads - 1) / (kPtsPerThread * kThreads), kThreads, 0,
                                   ctx->stream>>>(P.d_qual.as<double>(), nq, qual_order(P), 0, nq, charges_dev,
                                                  n_charges, scale, vals.as<double>(), nullptr);
  BP_LAUNCH_CHECK();
  sum_points_kernel<<<(P.n + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(
      P.d_qual_off.as<int32_t>(), 0, P.n, 0, nq, vals.as<double>(), rhs_dev, rhs_dev + P.n);
  BP_LAUNCH_CHECK();
  BP_CUDA(cudaStreamSynchronize(ctx->stream));
}

namespace {

// Per-point values of points [first, first + count) of a SoA list (stride
// npts) into out (indexed from first), plus add when set: the FP64 or the
// fast kernel.
void launch_point_potential(bool fp64, const double* pts, int npts, int first, int count, const double* charges,
                            int nc, double scale, double* out, const double* add, cudaStream_t st) {
  if (count <= 0) return;
  if (fp64)
    point_potential_kernel<<<(count + kThreads - 1) / kThreads, kThreads, 0, st>>>(pts, npts, first, count, charges,
                                                                                 nc, scale, out, add);
  else
    point_potential_fast_kernel<<<(count + kPtsPerThread * kThreads - 1) / (kPtsPerThread * kThreads), kThreads, 0,
                                  st>>>(pts, npts, first, count, charges, nc, scale, out, add);
  BP_LAUNCH_CHECK();
}

// The potential of a charge list (mesh frame) at the mesh's qualocation
// points, from the mesh's cache or computed into it.  Rotation and
// translation leave distances and normal derivatives unchanged, so the
// values serve every placement of the mesh.
const double* mesh_self_potential(DevMesh& m, const double* charges, int nc, double scale, bool fp64,
                                  cudaStream_t st) {
  std::lock_guard<std::mutex> lk(m.mu);
  auto& list = m.self_potential;
  for (size_t k = 0; k < list.size(); ++k) {
    const DevMesh::SelfPotential& e = list[k];
    if (e.fp64 == fp64 && e.scale == scale && e.charges.size() == 4 * (size_t)nc &&
        (nc == 0 || std::memcmp(e.charges.data(), charges, sizeof(double) * 4 * (size_t)nc) == 0)) {
      std::rotate(list.begin() + k, list.begin() + k + 1, list.end());  // most recently used last
      return list.back().vals.as<double>();
    }
  }
  if (list.size() >= DevMesh::kSelfPotentials) list.erase(list.begin());
  DevMesh::SelfPotential e;
  e.charges.assign(charges, charges + 4 * (size_t)nc);
  e.scale = scale;
  e.fp64 = fp64;
  e.vals.alloc(m.ctx, sizeof(double) * 2 * (size_t)std::max(1, m.n_qual_pts));
  DevBuf dch(m.ctx, sizeof(double) * 4 * (size_t)std::max(1, nc));
  if (nc) BP_CUDA(cudaMemcpyAsync(dch.get(), charges, sizeof(double) * 4 * (size_t)nc, cudaMemcpyHostToDevice, st));
  launch_point_potential(fp64, m.d_qual.as<double>(), m.n_qual_pts, 0, m.n_qual_pts, dch.as<double>(), nc, scale,
                         e.vals.as<double>(), nullptr, st);
  list.push_back(std::move(e));
  return list.back().vals.as<double>();
}

}  // namespace

void rhs_posed_device(Problem& P, const double* const* charges_host, const int32_t* n_charges, double eps_solvent,
                      double* rhs_dev) {
  Ctx* ctx = P.ctx;
  cudaStream_t st = ctx->stream;
  const int ni = (int)P.placements.size();
  const double scale = kOneOver4Pi / eps_solvent;
  // every instance's charges in the problem's frame
  std::vector<size_t> wstart(ni + 1, 0);
  for (int k = 0; k < ni; ++k) wstart[k + 1] = wstart[k] + (size_t)n_charges[k];
  std::vector<double> world(4 * wstart[ni]);
  for (int k = 0; k < ni; ++k) {
    const Placement& pl = P.placements[k];
    for (int i = 0; i < n_charges[k]; ++i) {
      const double* ch = charges_host[k] + 4 * (size_t)i;
      const double x = ch[0] - pl.c[0], y = ch[1] - pl.c[1], z = ch[2] - pl.c[2];
      double* w = &world[4 * (wstart[k] + i)];
      for (int r = 0; r < 3; ++r) w[r] = pl.R[3 * r] * x + pl.R[3 * r + 1] * y + pl.R[3 * r + 2] * z + pl.o[r];
      w[3] = ch[3];
    }
  }
  // per instance the other instances' charges of its scenario, one list
  // after another
  std::vector<size_t> ostart(ni + 1, 0);
  std::vector<double> others;
  for (int k = 0; k < ni; ++k) {
    for (int j = 0; j < ni; ++j)
      if (j != k && P.placements[j].scenario == P.placements[k].scenario) others.insert(others.end(), world.begin() + 4 * wstart[j], world.begin() + 4 * wstart[j + 1]);
    ostart[k + 1] = others.size() / 4;
  }
  DevBuf& dch = P.scratch_charges;
  const size_t cbytes = sizeof(double) * std::max<size_t>(4, others.size());
  if (dch.bytes() < cbytes) dch.alloc(ctx, cbytes);
  if (!others.empty())
    BP_CUDA(cudaMemcpyAsync(dch.get(), others.data(), sizeof(double) * others.size(), cudaMemcpyHostToDevice, st));
  const int nq = P.n_qual_pts;
  DevBuf& vals = P.scratch_vals;
  if (vals.bytes() < sizeof(double) * 2 * (size_t)nq) vals.alloc(ctx, sizeof(double) * 2 * (size_t)nq);
  for (int k = 0; k < ni; ++k) {
    const Placement& pl = P.placements[k];
    const double* self = mesh_self_potential(*pl.mesh, charges_host[k], n_charges[k], scale, P.fp64, st);
    if (P.fp64 || pl.q_count <= 0)
      launch_point_potential(P.fp64, P.d_qual.as<double>(), nq, pl.q_begin, pl.q_count,
                             dch.as<double>() + 4 * ostart[k], (int)(ostart[k + 1] - ostart[k]), scale,
                             vals.as<double>() + 2 * (size_t)pl.q_begin, self, st);
    else {
      point_potential_split_kernel<<<(pl.q_count + kPtsPerThread * kThreads - 1) / (kPtsPerThread * kThreads),
                                     kThreads, 0, st>>>(P.d_qual.as<double>(), nq, qual_order(P), pl.q_begin,
                                                        pl.q_count, dch.as<double>() + 4 * ostart[k],
                                                        (int)(ostart[k + 1] - ostart[k]), scale,
                                                        vals.as<double>() + 2 * (size_t)pl.q_begin, self);
      BP_LAUNCH_CHECK();
    }
  }
  sum_points_kernel<<<(P.n + kThreads - 1) / kThreads, kThreads, 0, st>>>(
      P.d_qual_off.as<int32_t>(), 0, P.n, 0, nq, vals.as<double>(), rhs_dev, rhs_dev + P.n);
  BP_LAUNCH_CHECK();
  BP_CUDA(cudaStreamSynchronize(st));
}

void energy_coefficients_device(Problem& P, int first, int count, const double* charges_dev, int n_charges,
                                double* cf_dev, double* ch_dev) {
  Ctx* ctx = P.ctx;
  const int ng = P.n_gal_pts;
  const int p0 = P.h_gal_off[first], p1 = P.h_gal_off[first + count];
  DevBuf vals(ctx, sizeof(double) * 2 * (size_t)std::max(1, p1 - p0));
  if (p1 > p0) {
    point_potential_kernel<<<(p1 - p0 + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(
        P.d_gal.as<double>(), ng, p0, p1 - p0, charges_dev, n_charges, kOneOver4Pi, vals.as<double>(), nullptr);
    BP_LAUNCH_CHECK();
  }
  // vals[2p] -> ec_h (potential), vals[2p+1] -> ec_f (normal field)
  sum_points_kernel<<<(count + kThreads - 1) / kThreads, kThreads, 0, ctx->stream>>>(
      P.d_gal_off.as<int32_t>(), first, count, p0, p1 - p0, vals.as<double>(), ch_dev, cf_dev);
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
    // the scratch array used is the current device's: every buffer must be
    // on that device
    int dev = -1;
    BP_CUDA(cudaGetDevice(&dev));
    const void* bufs[4] = {qual_offsets_dev, qual_points_soa_dev, rhs_dev, n_charges > 0 ? charges_xyzq_dev : nullptr};
    for (const void* b : bufs) {
      if (!b) continue;
      cudaPointerAttributes at{};
      if (cudaPointerGetAttributes(&at, b) != cudaSuccess) {
        cudaGetLastError();
        return fail(BP_ERR_INVALID, "bp_rhs_noalloc: a buffer is not CUDA memory");
      }
      if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != dev)
        return fail(BP_ERR_INVALID, "bp_rhs_noalloc: every buffer must be device memory of the current device");
    }
    double* scratch = noalloc_scratch_for_current_device();
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    const double scale = kOneOver4Pi / eps_solvent;
    point_potential_kernel<<<(n_qual_points + kThreads - 1) / kThreads, kThreads, 0, st>>>(
        qual_points_soa_dev, n_qual_points, 0, n_qual_points, charges_xyzq_dev, n_charges, scale, scratch, nullptr);
    BP_LAUNCH_CHECK();
    sum_points_kernel<<<(n_patches + kThreads - 1) / kThreads, kThreads, 0, st>>>(
        qual_offsets_dev, 0, n_patches, 0, n_qual_points, scratch, rhs_dev, rhs_dev + n_patches);
    BP_LAUNCH_CHECK();
    return BP_OK;
  });
}

