// Near field of the BEM matvec on sm_100a.
//
// What it computes (reference: src/bem/bem_kernels.h:18-251,
// src/bem/local_integrations.h:98-130, src/beep/beep.cpp:768-1064):
//   for every leaf L of the adaptive octree and every pair (i, j) with i a
//   patch of L (collocation, "src" in the reference) and j a patch of the
//   27-box neighbourhood of L (integration, "targ"), i != j:
//     A_ij = sum_q w_q sum_p w_p (G - u)
//     B_ij = sum_q w_q sum_p w_p n_p . (grad G / eps_j - grad u)
//     C_ij = -sum_q w_q sum_p w_p n_q . (grad G - grad u / eps_j)
//     D_ij = -(1/eps_j) sum_q w_q sum_p w_p n_q^T (Hess G - Hess u) n_p  (kappa != 0)
//   with G = 1/(4 pi r), u = exp(-kappa r)/(4 pi r), r = x_p - x_q, q over
//   the qualocation points of i, p over the quadrature points of j, and
//   pairs with |r|^2 < 1e-9 skipped.  The diagonal (i, i) slot holds the
//   singular self-patch integral plus the geometric corrections
//   (src/bem/bem_kernels.cpp:123-136, src/beep/beep.cpp:829-843); it is
//   computed and applied in FP64 in every precision mode.
//   Per matvec: y_f[i] += B_ij f_j - A_ij h_j ; y_h[i] += D_ij f_j - C_ij h_j.
//
// Layout: one dense block of (A,B,C,D) per leaf, rows = the leaf's patches,
// cols = the concatenated patches of its neighbours in neighbour order
// 0..26.  The column list is stored once per leaf, so a pair costs 16 bytes
// (FP32) or 32 bytes (FP64) of coefficients instead of the reference's
// 24-byte (src, targ, A, B, C, D) record.  The apply kernel stages the
// leaf's x values in shared memory once and streams each row's
// coefficients with 16/32-byte vector loads, one warp per row, reduced with
// warp shuffles: the per-iteration floor is the coefficient stream (HBM).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "engine.h"

namespace bp {

namespace {

constexpr int kAsmRows = 8;      // rows per assembly work item
constexpr int kAsmThreads = 256;
constexpr int kApplyRows = 64;   // rows per apply work item
constexpr int kApplyThreads = 256;
constexpr int kApplyBlocksPerSm = 8;  // resident apply blocks per SM (persistent grid)
constexpr double kOneOver4Pi = 0.07957747154594767;  // 1/(4 pi)

template <typename T>
struct Vec4 {};
template <>
struct Vec4<float> {
  using type = float4;
};
template <>
struct Vec4<double> {
  using type = double4;
};

// Streaming (evict-first) loads of one coefficient quadruple.
__device__ __forceinline__ float4 ld_stream(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ double4 ld_stream(const double4* p) {
  const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// Compact near field (BP_FLAG_COMPACT_NEARFIELD): each FP32 coefficient
// rounded to its top 24 bits (sign, exponent and a 15-bit fraction: a 16-bit
// significand, relative rounding error at most 2^-17) and the four of a pair
// packed into 12 bytes, kept as two planes of one buffer so that every warp
// load is contiguous: plane 0 holds (w0, w1) per pair, plane 1 w2, with
//   w0 = a | b << 24,  w1 = b >> 8 | c << 16,  w2 = c >> 16 | d << 8
// for the 24-bit values a, b, c, d.
__device__ __forceinline__ uint32_t round24(float v) {
  return (__float_as_uint(v) + 0x80u) >> 8;  // to nearest on the magnitude; carries into the exponent
}
__device__ __forceinline__ void pack24(float4 v, uint2& w01, uint32_t& w2) {
  const uint32_t a = round24(v.x), b = round24(v.y), c = round24(v.z), d = round24(v.w);
  w01.x = a | (b << 24);
  w01.y = (b >> 8) | (c << 16);
  w2 = (c >> 16) | (d << 8);
}
__device__ __forceinline__ float4 unpack24(uint2 w01, uint32_t w2) {
  float4 v;
  v.x = __uint_as_float(w01.x << 8);
  v.y = __uint_as_float(((w01.x >> 16) & 0xFF00u) | (w01.y << 16));
  v.z = __uint_as_float(((w01.y >> 8) & 0xFFFF00u) | (w2 << 24));
  v.w = __uint_as_float(w2 & 0xFFFFFF00u);
  return v;
}

// The coefficient quadruple of pair index k: FP32 / FP64 records, or the
// compact planes: plane 0 holds each pair's first two words (8 bytes), plane
// 1, starting 2 n_pairs words later, its third word (4 bytes).  A warp's 32
// consecutive pairs read 256 contiguous bytes of plane 0 and 128 of plane 1
// (measured: groups of 32 pairs with both parts side by side, 384 bytes a
// group, split each warp's reads over two groups and ran the apply at 0.183
// against 0.141 ms on the 40962-patch star).
template <typename T, bool kCompact>
struct CoefReader {
  const typename Vec4<T>::type* rec;
  __device__ __forceinline__ typename Vec4<T>::type operator()(int64_t k) const { return ld_stream(rec + k); }
};
template <>
struct CoefReader<float, true> {
  const uint2* p01;
  const uint32_t* p2;
  __device__ __forceinline__ float4 operator()(int64_t k) const { return unpack24(__ldcs(p01 + k), __ldcs(p2 + k)); }
};
template <typename T, bool kCompact>
struct CoefWriter {
  typename Vec4<T>::type* rec;
  __device__ __forceinline__ void operator()(int64_t k, typename Vec4<T>::type v) const { rec[k] = v; }
};
template <>
struct CoefWriter<float, true> {
  uint2* p01;
  uint32_t* p2;
  __device__ __forceinline__ void operator()(int64_t k, float4 v) const {
    uint2 w01;
    uint32_t w2;
    pack24(v, w01, w2);
    p01[k] = w01;
    p2[k] = w2;
  }
};

// FP32: the hardware approximations with denormals flushed (PTX
// rsqrt.approx.ftz / ex2.approx.ftz).  The arguments here are normal
// numbers (r^2 >= 1e-9 and exponents above -126), where flushing changes
// nothing and saves the denormal handling of rsqrtf / exp2f.
__device__ __forceinline__ float fast_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double fast_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float fexp(float x) { return expf(x); }
__device__ __forceinline__ double fexp(double x) { return exp(x); }

// One (collocation point, quadrature point) term of the four kernels,
// accumulated into a, b, c, d (src/bem/bem_kernels.h:187-240).
template <typename T>
__device__ __forceinline__ void pair_term(T qx, T qy, T qz, T qnx, T qny, T qnz, T px, T py, T pz, T pnx, T pny,
                                          T pnz, T pw, T kappa, T ie, bool with_d, T& a, T& b, T& c, T& d) {
  const T dx = px - qx, dy = py - qy, dz = pz - qz;
  const T r2 = dx * dx + dy * dy + dz * dz;
  if (fabs(r2) < T(1e-9)) return;
  const T ir = fast_rsqrt(r2);
  const T r = r2 * ir;
  const T ir2 = ir * ir;
  const T ir3 = ir2 * ir;
  const T gr0 = T(kOneOver4Pi);
  const T gr1 = gr0 * ir;
  const T gr3 = gr0 * ir3;
  const T ur0 = fexp(-kappa * r) * gr0;
  const T ur1 = ur0 * ir;
  const T ur2 = ur0 * ir2;
  const T ur3 = ur0 * ir3;
  const T ur3ur2 = ur3 + kappa * ur2;
  // gd = -dx*gr3 ; ud = -dx*ur3ur2
  const T ndx = pnx * dx + pny * dy + pnz * dz;   // n_p . dx
  const T n0dx = qnx * dx + qny * dy + qnz * dz;  // n_q . dx
  a += pw * (gr1 - ur1);
  b += pw * (-(ie * gr3) + ur3ur2) * ndx;
  c += -pw * (-gr3 + ie * ur3ur2) * n0dx;
  if (with_d) {
    const T ir4 = ir2 * ir2;
    const T ir5 = ir4 * ir;
    const T gr5 = gr0 * ir5;
    const T ur4 = ur0 * ir4;
    const T ur5 = ur0 * ir5;
    const T pur4ur3 = kappa * (T(3) * ur4 + kappa * ur3) + T(3) * ur5;
    const T nn0 = pnx * qnx + pny * qny + pnz * qnz;
    // sum_jk n0_k n_j (gdd_jk - udd_jk)
    const T s = ndx * n0dx * (T(3) * gr5 - pur4ur3) - nn0 * (gr3 - ur3ur2);
    d -= pw * s;
  }
}

// The same four kernels without the quadrature weight, rearranged to share
// factors: with g = 1/(4 pi r), e = exp(-kappa r) and t = 1/r^2,
//   G - u                     = g (1 - e)
//   grad G . d / |d|^2 terms  : g3 = g t,  u3 = e g (t + kappa/r)
//   Hessian terms             : gr5 = g3 t, pu = e g t (3 kappa/r + kappa^2 + 3 t)
// (the expressions of pair_term, factored).  `ek` is the exponent scale:
// -kappa log2(e) for FP32, where e = 2^(ek r) (exp2f), and -kappa for FP64.
__device__ __forceinline__ float exp_scaled(float ek, float r) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(ek * r));
  return y;
}
__device__ __forceinline__ double exp_scaled(double ek, double r) { return exp(ek * r); }
template <typename T>
__device__ __forceinline__ T exp_scale(T kappa);
template <>
__device__ __forceinline__ float exp_scale<float>(float kappa) {
  return -kappa * 1.4426950408889634f;  // log2(e)
}
template <>
__device__ __forceinline__ double exp_scale<double>(double kappa) {
  return -kappa;
}

template <typename T>
__device__ __forceinline__ void pair_term_unit(T qx, T qy, T qz, T qnx, T qny, T qnz, T px, T py, T pz, T pnx,
                                               T pny, T pnz, T kappa, T ek, T ie, bool with_d, T& a, T& b, T& c,
                                               T& d) {
  const T dx = px - qx, dy = py - qy, dz = pz - qz;
  const T r2 = dx * dx + dy * dy + dz * dz;
  if (fabs(r2) < T(1e-9)) return;
  const T ir = fast_rsqrt(r2);
  const T r = r2 * ir;
  const T e = exp_scaled(ek, r);
  const T g = T(kOneOver4Pi) * ir;
  const T eg = e * g;
  const T t = ir * ir;
  const T g3 = g * t;
  const T u3 = eg * (t + kappa * ir);
  const T ndx = pnx * dx + pny * dy + pnz * dz;   // n_p . dx
  const T n0dx = qnx * dx + qny * dy + qnz * dz;  // n_q . dx
  a += g - eg;
  b += (u3 - ie * g3) * ndx;
  c += (g3 - ie * u3) * n0dx;
  if (with_d) {
    const T pu = eg * t * (kappa * (T(3) * ir + kappa) + T(3) * t);
    const T nn0 = pnx * qnx + pny * qny + pnz * qnz;
    d -= ndx * n0dx * (T(3) * g3 * t - pu) - nn0 * (g3 - u3);
  }
}

// Singular self-patch integrals in FP64, one warp per patch
// (src/bem/bem_kernels.h:18-132): all ordered pairs of distinct galerkin
// points of the patch, normalised by the sum of the outer weights; then the
// geometric corrections B += (1-gc) + gc/eps, C -= gc + (1-gc)/eps.
__global__ void singular_kernel(int n, const int32_t* __restrict__ off, const double* __restrict__ g, int ng,
                                const double* __restrict__ eps, const double* __restrict__ gcv, double kappa,
                                double* __restrict__ diag) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int s = off[warp], e = off[warp + 1];
  const double* X = g;
  const double* Y = g + ng;
  const double* Z = g + 2 * (size_t)ng;
  const double* NX = g + 3 * (size_t)ng;
  const double* NY = g + 4 * (size_t)ng;
  const double* NZ = g + 5 * (size_t)ng;
  const double* W = g + 6 * (size_t)ng;
  const double ie = 1.0 / eps[warp];
  double A = 0, B = 0, C = 0, D = 0, wsum = 0;
  for (int q = s + lane; q < e; q += 32) {
    double a = 0, b = 0, c = 0, d = 0;
    for (int p = s; p < e; ++p) {
      pair_term<double>(X[q], Y[q], Z[q], NX[q], NY[q], NZ[q], X[p], Y[p], Z[p], NX[p], NY[p], NZ[p], W[p], kappa,
                        ie, kappa != 0.0, a, b, c, d);
    }
    A += a * W[q];
    B += b * W[q];
    C += c * W[q];
    D += d * W[q];
    wsum += W[q];
  }
  for (int o = 16; o > 0; o >>= 1) {
    A += __shfl_xor_sync(0xffffffffu, A, o);
    B += __shfl_xor_sync(0xffffffffu, B, o);
    C += __shfl_xor_sync(0xffffffffu, C, o);
    D += __shfl_xor_sync(0xffffffffu, D, o);
    wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
  }
  if (lane == 0) {
    const double epsr = eps[warp];
    const double gc = gcv[warp];
    A /= wsum;
    B /= wsum;
    C /= wsum;
    D *= ie / wsum;
    const double fgc = (1.0 - gc) + gc / epsr;
    const double hgc = gc + (1.0 - gc) / epsr;
    diag[4 * warp + 0] = A;
    diag[4 * warp + 1] = B + fgc;
    diag[4 * warp + 2] = C - hgc;
    diag[4 * warp + 3] = D;
  }
}

// One staged qualocation point: position, normal and weight, stored 8 wide
// so that a point is two 16-byte (FP32) or four 16-byte (FP64) shared loads.
__device__ __forceinline__ void load_qpoint(const float* s, int q, float (&v)[7]) {
  const float4 a = reinterpret_cast<const float4*>(s)[2 * q];
  const float4 b = reinterpret_cast<const float4*>(s)[2 * q + 1];
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z;
}
__device__ __forceinline__ void load_qpoint(const double* s, int q, double (&v)[7]) {
  const double2* p = reinterpret_cast<const double2*>(s) + 4 * q;
  const double2 a = p[0], b = p[1], c = p[2], d = p[3];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y; v[6] = d.x;
}

// Coefficient assembly.  A work item is <= kAsmRows rows of one leaf; their
// qualocation points are staged in shared memory; each thread walks the
// leaf's columns and produces the (A,B,C,D) of every staged row for its
// column, so one row's stores are contiguous across the block.  A column
// with one quadrature point (quadrature rule 0) keeps it in registers for
// all of its rows x qualocation points.
template <typename T, bool kCompact>
__global__ void __launch_bounds__(kAsmThreads) assemble_kernel(
    const NfItem* __restrict__ items, const int32_t* __restrict__ rows, const int64_t* __restrict__ row_off,
    const int32_t* __restrict__ cols, const int64_t* __restrict__ col_off, const int64_t* __restrict__ coef_off,
    const int32_t* __restrict__ qoff, const T* __restrict__ qual, int nq, const int32_t* __restrict__ poff,
    const T* __restrict__ quad, int np, const double* __restrict__ eps, T kappa, const double* __restrict__ diag,
    const CoefWriter<T, kCompact> out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sq = reinterpret_cast<T*>(smem_raw);  // [qual_total][8]
  __shared__ int s_start[kAsmRows + 1];
  __shared__ int s_row[kAsmRows];
  const NfItem it = items[blockIdx.x];
  const int64_t r0 = row_off[it.leaf] + it.row_begin;
  const int64_t c0 = col_off[it.leaf];
  const int ncols = (int)(col_off[it.leaf + 1] - c0);
  const int64_t block = coef_off[it.leaf];
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int r = 0; r < it.row_count; ++r) {
      const int i = rows[r0 + r];
      s_row[r] = i;
      s_start[r] = acc;
      acc += qoff[i + 1] - qoff[i];
    }
    s_start[it.row_count] = acc;
  }
  __syncthreads();
  for (int r = 0; r < it.row_count; ++r) {
    const int i = s_row[r];
    const int base = qoff[i];
    const int cnt = s_start[r + 1] - s_start[r];
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      T* dst = sq + 8 * (s_start[r] + k);
      for (int f = 0; f < 7; ++f) dst[f] = qual[(size_t)f * nq + base + k];
      dst[7] = T(0);
    }
  }
  __syncthreads();
  const bool with_d = kappa != T(0);
  const T ek = exp_scale<T>(kappa);
  using V4 = typename Vec4<T>::type;
  for (int cc = threadIdx.x; cc < ncols; cc += blockDim.x) {
    const int j = cols[c0 + cc];
    const T ie = T(1.0 / eps[j]);
    const int ps = poff[j], pe = poff[j + 1];
    const bool one_point = pe - ps == 1;
    T p1[7] = {0, 0, 0, 0, 0, 0, 0};
    if (one_point)
      for (int f = 0; f < 7; ++f) p1[f] = quad[(size_t)f * np + ps];
    for (int r = 0; r < it.row_count; ++r) {
      const int i = s_row[r];
      const int64_t o = block + (int64_t)(it.row_begin + r) * ncols + cc;
      V4 v;
      if (i == j) {  // self pair: applied in FP64 from the singular diagonal
        v.x = T(0);
        v.y = T(0);
        v.z = T(0);
        v.w = T(0);
        out(o, v);
        continue;
      }
      T A = 0, B = 0, C = 0, D = 0;
      const int qs = s_start[r], qe = s_start[r + 1];
      if (one_point) {  // the column's weight multiplies the row's sums
#pragma unroll 4
        for (int q = qs; q < qe; ++q) {
          T u[7];
          load_qpoint(sq, q, u);
          T a = 0, b = 0, c = 0, d = 0;
          pair_term_unit<T>(u[0], u[1], u[2], u[3], u[4], u[5], p1[0], p1[1], p1[2], p1[3], p1[4], p1[5], kappa, ek,
                            ie, with_d, a, b, c, d);
          A += a * u[6];
          B += b * u[6];
          C += c * u[6];
          D += d * u[6];
        }
        A *= p1[6];
        B *= p1[6];
        C *= p1[6];
        D *= p1[6];
      } else {
        for (int q = qs; q < qe; ++q) {
          T u[7];
          load_qpoint(sq, q, u);
          T a = 0, b = 0, c = 0, d = 0;
          for (int p = ps; p < pe; ++p) {
            pair_term<T>(u[0], u[1], u[2], u[3], u[4], u[5], quad[p], quad[(size_t)np + p],
                         quad[2 * (size_t)np + p], quad[3 * (size_t)np + p], quad[4 * (size_t)np + p],
                         quad[5 * (size_t)np + p], quad[6 * (size_t)np + p], kappa, ie, with_d, a, b, c, d);
          }
          A += a * u[6];
          B += b * u[6];
          C += c * u[6];
          D += d * u[6];
        }
      }
      v.x = A;
      v.y = B;
      v.z = C;
      v.w = D * ie;
      out(o, v);
    }
  }
}

// ---------------------------------------------------------------------------
// Mesh pair cache (BP_FLAG_MESH_PAIR_CACHE).  The coefficients of a pair of
// patches of one rigid mesh depend only on the mesh, kappa and the
// instance's dielectric ratio, not on where the instance sits, so a scan
// that places the same meshes pose after pose integrates them once, in the
// mesh's frame, for every pair of patches closer than a radius, and each
// pose's assembly looks them up.  Pairs beyond the radius, pairs of two
// instances and the self pairs go through the integration as before.

// One term of pair_term_unit with the dielectric factor left out: B and C
// as their two parts (B = Bu - ie Bg, C = Cg - ie Cu) and D before its
// factor ie.
__device__ __forceinline__ void pair_term_parts(float qx, float qy, float qz, float qnx, float qny, float qnz, float px,
                                                float py, float pz, float pnx, float pny, float pnz, float kappa,
                                                float ek, bool with_d, float (&acc)[6]) {
  const float dx = px - qx, dy = py - qy, dz = pz - qz;
  const float r2 = dx * dx + dy * dy + dz * dz;
  if (fabsf(r2) < 1e-9f) return;
  const float ir = fast_rsqrt(r2);
  const float r = r2 * ir;
  const float e = exp_scaled(ek, r);
  const float g = float(kOneOver4Pi) * ir;
  const float eg = e * g;
  const float t = ir * ir;
  const float g3 = g * t;
  const float u3 = eg * (t + kappa * ir);
  const float ndx = pnx * dx + pny * dy + pnz * dz;
  const float n0dx = qnx * dx + qny * dy + qnz * dz;
  acc[0] += g - eg;
  acc[1] += u3 * ndx;
  acc[2] += g3 * ndx;
  acc[3] += g3 * n0dx;
  acc[4] += u3 * n0dx;
  if (with_d) {
    const float pu = eg * t * (kappa * (3.f * ir + kappa) + 3.f * t);
    const float nn0 = pnx * qnx + pny * qny + pnz * qnz;
    acc[5] -= ndx * n0dx * (3.f * g3 * t - pu) - nn0 * (g3 - u3);
  }
}

// Partners j != i of every patch i with |c_i - c_j|^2 < r2: their count
// (js == nullptr) or their list, ascending (from off[i]).  Every thread
// scans all centroids through shared-memory tiles; both passes make the
// same comparisons, so the lists have the counted lengths.
__global__ void __launch_bounds__(256) pair_cache_scan_kernel(int n, const float4* __restrict__ c, float r2,
                                                              int32_t* __restrict__ count,
                                                              const int64_t* __restrict__ off,
                                                              int32_t* __restrict__ js) {
  __shared__ float4 tile[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const float4 ci = i < n ? c[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  int64_t w = (js && i < n) ? off[i] : 0;
  int cnt = 0;
  for (int base = 0; base < n; base += 256) {
    const int jj = base + threadIdx.x;
    tile[threadIdx.x] = jj < n ? c[jj] : make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    const int lim = min(256, n - base);
    if (i < n)
      for (int t = 0; t < lim; ++t) {
        // rounded operations only (no contraction), so both passes decide alike
        const float dx = __fsub_rn(tile[t].x, ci.x), dy = __fsub_rn(tile[t].y, ci.y), dz = __fsub_rn(tile[t].z, ci.z);
        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
        if (d2 < r2 && base + t != i) {
          if (!js)
            ++cnt;
          else if (w < off[i + 1])
            js[w++] = base + t;
        }
      }
    __syncthreads();
  }
  if (!js && i < n) count[i] = cnt;
}

// The six parts of every listed pair, one block per patch i of the mesh:
// i's qualocation points staged in shared memory (FP32, as the mixed
// assembly converts them), one thread per partner j (one quadrature point
// per patch), weights applied as in assemble_kernel.
__global__ void __launch_bounds__(kAsmThreads) pair_cache_coef_kernel(
    const int64_t* __restrict__ off, const int32_t* __restrict__ js, const int32_t* __restrict__ qoff,
    const double* __restrict__ qual, int nq, const int32_t* __restrict__ poff, const double* __restrict__ quad, int np,
    float kappa, float* __restrict__ vals) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* sq = reinterpret_cast<float*>(smem_raw);
  const int i = blockIdx.x;
  const int qs = qoff[i], nqi = qoff[i + 1] - qs;
  for (int k = threadIdx.x; k < nqi; k += blockDim.x) {
    for (int f = 0; f < 7; ++f) sq[8 * k + f] = (float)qual[(size_t)f * nq + qs + k];
    sq[8 * k + 7] = 0.f;
  }
  __syncthreads();
  const bool with_d = kappa != 0.f;
  const float ek = exp_scale<float>(kappa);
  for (int64_t k = off[i] + threadIdx.x; k < off[i + 1]; k += blockDim.x) {
    const int p = poff[js[k]];
    float p1[7];
    for (int f = 0; f < 7; ++f) p1[f] = (float)quad[(size_t)f * np + p];
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
    for (int q = 0; q < nqi; ++q) {
      float u[7];
      load_qpoint(sq, q, u);
      float a[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      pair_term_parts(u[0], u[1], u[2], u[3], u[4], u[5], p1[0], p1[1], p1[2], p1[3], p1[4], p1[5], kappa, ek, with_d,
                      a);
      for (int f = 0; f < 6; ++f) acc[f] += a[f] * u[6];
    }
    float2* o = reinterpret_cast<float2*>(vals + 6 * k);
    o[0] = make_float2(acc[0] * p1[6], acc[1] * p1[6]);
    o[1] = make_float2(acc[2] * p1[6], acc[3] * p1[6]);
    o[2] = make_float2(acc[4] * p1[6], acc[5] * p1[6]);
  }
}

// One placement's cache as the assembly sees it (off == nullptr: none).
struct CacheView {
  const int64_t* off;
  const int32_t* js;
  const float* vals;
  int first;  // the placement's first patch in the problem
};

constexpr int kMissCap = 4096;  // pairs a block integrates in one pass

// One (row, column) pair integrated as assemble_kernel does it (FP32).
__device__ __forceinline__ float4 pair_integrated(const float* sq, int qs, int qe, int j, const int32_t* poff,
                                                  const float* quad, int np, float kappa, float ek, float ie,
                                                  bool with_d) {
  const int ps = poff[j], pe = poff[j + 1];
  float A = 0, B = 0, C = 0, D = 0;
  if (pe - ps == 1) {
    float p1[7];
    for (int f = 0; f < 7; ++f) p1[f] = quad[(size_t)f * np + ps];
    for (int q = qs; q < qe; ++q) {
      float u[7];
      load_qpoint(sq, q, u);
      float a = 0, b = 0, c = 0, d = 0;
      pair_term_unit<float>(u[0], u[1], u[2], u[3], u[4], u[5], p1[0], p1[1], p1[2], p1[3], p1[4], p1[5], kappa, ek,
                            ie, with_d, a, b, c, d);
      A += a * u[6];
      B += b * u[6];
      C += c * u[6];
      D += d * u[6];
    }
    A *= p1[6];
    B *= p1[6];
    C *= p1[6];
    D *= p1[6];
  } else {
    for (int q = qs; q < qe; ++q) {
      float u[7];
      load_qpoint(sq, q, u);
      float a = 0, b = 0, c = 0, d = 0;
      for (int p = ps; p < pe; ++p)
        pair_term<float>(u[0], u[1], u[2], u[3], u[4], u[5], quad[p], quad[(size_t)np + p], quad[2 * (size_t)np + p],
                         quad[3 * (size_t)np + p], quad[4 * (size_t)np + p], quad[5 * (size_t)np + p],
                         quad[6 * (size_t)np + p], kappa, ie, with_d, a, b, c, d);
      A += a * u[6];
      B += b * u[6];
      C += c * u[6];
      D += d * u[6];
    }
  }
  return make_float4(A, B, C, D * ie);
}

// assemble_kernel with the mesh pair caches (mixed engine): for each row,
// its cached partner list is staged in shared memory; a thread takes the
// row's columns, finds a column of the same placement by binary search and
// combines its six parts with the column's dielectric factor.  Columns not
// found (farther than the cache radius, of another placement, or of a
// placement without a cache) are queued in shared memory and integrated
// when the queue is full and at the end of the item, one pair per thread,
// so that the integration runs on full warps.  Self pairs are zero, as in
// assemble_kernel.
template <bool kCompact>
__global__ void __launch_bounds__(kAsmThreads) assemble_cached_kernel(
    const NfItem* __restrict__ items, const int32_t* __restrict__ rows, const int64_t* __restrict__ row_off,
    const int32_t* __restrict__ cols, const int64_t* __restrict__ col_off, const int64_t* __restrict__ coef_off,
    const int32_t* __restrict__ qoff, const float* __restrict__ qual, int nq, const int32_t* __restrict__ poff,
    const float* __restrict__ quad, int np, const double* __restrict__ eps, float kappa,
    const int32_t* __restrict__ inst_of, const CacheView* __restrict__ views, int max_list, int qual_cap,
    const CoefWriter<float, kCompact> out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* sq = reinterpret_cast<float*>(smem_raw);              // [qual_cap][8]
  int32_t* s_js = reinterpret_cast<int32_t*>(sq + 8 * (size_t)qual_cap);  // [max_list]
  __shared__ int s_miss[kMissCap];
  __shared__ int s_nmiss;
  __shared__ int s_start[kAsmRows + 1];
  __shared__ int s_row[kAsmRows];
  const NfItem it = items[blockIdx.x];
  const int64_t r0 = row_off[it.leaf] + it.row_begin;
  const int64_t c0 = col_off[it.leaf];
  const int ncols = (int)(col_off[it.leaf + 1] - c0);
  const int64_t block = coef_off[it.leaf];
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int r = 0; r < it.row_count; ++r) {
      const int i = rows[r0 + r];
      s_row[r] = i;
      s_start[r] = acc;
      acc += qoff[i + 1] - qoff[i];
    }
    s_start[it.row_count] = acc;
    s_nmiss = 0;
  }
  __syncthreads();
  for (int r = 0; r < it.row_count; ++r) {
    const int i = s_row[r];
    const int base = qoff[i];
    const int cnt = s_start[r + 1] - s_start[r];
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      float* dst = sq + 8 * (s_start[r] + k);
      for (int f = 0; f < 7; ++f) dst[f] = qual[(size_t)f * nq + base + k];
      dst[7] = 0.f;
    }
  }
  __syncthreads();
  const bool with_d = kappa != 0.f;
  const float ek = exp_scale<float>(kappa);
  // integrates the queued pairs (called by every thread, after a barrier)
  auto flush = [&]() {
    const int nm = s_nmiss;
    for (int m = threadIdx.x; m < nm; m += blockDim.x) {
      const int r = s_miss[m] >> 24, cc = s_miss[m] & 0xFFFFFF;
      const int j = cols[c0 + cc];
      const float ie = float(1.0 / eps[j]);
      out(block + (int64_t)(it.row_begin + r) * ncols + cc,
          pair_integrated(sq, s_start[r], s_start[r + 1], j, poff, quad, np, kappa, ek, ie, with_d));
    }
    __syncthreads();
    if (threadIdx.x == 0) s_nmiss = 0;
    __syncthreads();
  };
  for (int r = 0; r < it.row_count; ++r) {
    const int i = s_row[r];
    const int pi = inst_of[i];
    const CacheView v = views[pi];
    int len = 0;
    int64_t lbase = 0;
    if (v.off) {
      lbase = v.off[i - v.first];
      len = (int)(v.off[i - v.first + 1] - lbase);
      for (int k = threadIdx.x; k < len; k += blockDim.x) s_js[k] = v.js[lbase + k];
    }
    __syncthreads();
    for (int lo = 0; lo < ncols; lo += kMissCap) {
      const int hi = min(ncols, lo + kMissCap);
      if (s_nmiss + (hi - lo) > kMissCap) flush();  // s_nmiss is the same for every thread here
      for (int cc = lo + threadIdx.x; cc < hi; cc += blockDim.x) {
        const int j = cols[c0 + cc];
        const int64_t o = block + (int64_t)(it.row_begin + r) * ncols + cc;
        if (j == i) {
          out(o, make_float4(0.f, 0.f, 0.f, 0.f));
          continue;
        }
        bool found = false;
        if (len > 0 && inst_of[j] == pi) {
          const int jl = j - v.first;
          int a = 0, b = len;  // first entry >= jl
          while (a < b) {
            const int m = (a + b) >> 1;
            if (s_js[m] < jl)
              a = m + 1;
            else
              b = m;
          }
          if (a < len && s_js[a] == jl) {
            const float2* pv = reinterpret_cast<const float2*>(v.vals + 6 * (lbase + a));
            const float2 x0 = pv[0], x1 = pv[1], x2 = pv[2];
            const float ie = float(1.0 / eps[j]);
            out(o, make_float4(x0.x, x0.y - ie * x1.x, x1.y - ie * x2.x, x2.y * ie));
            found = true;
          }
        }
        if (!found) s_miss[atomicAdd(&s_nmiss, 1)] = (r << 24) | cc;
      }
      __syncthreads();
    }
  }
  flush();
}

// The near field without cached coefficients (the reference's
// BEM_kernels_instant + processBEMBlockResults for its uncached OpenCL path,
// src/bem/opencl_bem_kernels.cl:237-352, src/beep/beep.cpp:999-1008): the
// work items and point staging of assemble_kernel, but each thread applies
// the (A, B, C, D) of a pair to x at once and keeps, per staged row, the sums
// over its columns; the block then adds them in a fixed order (warp
// shuffles, then warps in order) and writes the rows with the FP64 diagonal
// and, when given, the far field.  Every row of a leaf belongs to one work
// item, so no two blocks write the same row.  The cost is the assembly's,
// every matvec; the memory is that of the points only.
template <typename T>
__global__ void __launch_bounds__(kAsmThreads) instant_kernel(
    const NfItem* __restrict__ items, const int32_t* __restrict__ rows, const int64_t* __restrict__ row_off,
    const int32_t* __restrict__ cols, const int64_t* __restrict__ col_off, const int32_t* __restrict__ qoff,
    const T* __restrict__ qual, int nq, const int32_t* __restrict__ poff, const T* __restrict__ quad, int np,
    const double* __restrict__ eps, T kappa, const double* __restrict__ diag, int n, const double* __restrict__ x,
    const double* __restrict__ yfar, double* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sq = reinterpret_cast<T*>(smem_raw);  // [qual_total][8]
  __shared__ int s_start[kAsmRows + 1];
  __shared__ int s_row[kAsmRows];
  __shared__ double s_red[kAsmThreads / 32][kAsmRows][2];
  const NfItem it = items[blockIdx.x];
  const int64_t r0 = row_off[it.leaf] + it.row_begin;
  const int64_t c0 = col_off[it.leaf];
  const int ncols = (int)(col_off[it.leaf + 1] - c0);
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int r = 0; r < it.row_count; ++r) {
      const int i = rows[r0 + r];
      s_row[r] = i;
      s_start[r] = acc;
      acc += qoff[i + 1] - qoff[i];
    }
    s_start[it.row_count] = acc;
  }
  __syncthreads();
  for (int r = 0; r < it.row_count; ++r) {
    const int i = s_row[r];
    const int base = qoff[i];
    const int cnt = s_start[r + 1] - s_start[r];
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      T* dst = sq + 8 * (s_start[r] + k);
      for (int f = 0; f < 7; ++f) dst[f] = qual[(size_t)f * nq + base + k];
      dst[7] = T(0);
    }
  }
  __syncthreads();
  const bool with_d = kappa != T(0);
  const T ek = exp_scale<T>(kappa);
  T accf[kAsmRows], acch[kAsmRows];
#pragma unroll
  for (int r = 0; r < kAsmRows; ++r) accf[r] = acch[r] = T(0);
  for (int cc = threadIdx.x; cc < ncols; cc += blockDim.x) {
    const int j = cols[c0 + cc];
    const T ie = T(1.0 / eps[j]);
    const T fj = T(x[j]), hj = T(x[n + j]);
    const int ps = poff[j], pe = poff[j + 1];
    const bool one_point = pe - ps == 1;
    T p1[7] = {0, 0, 0, 0, 0, 0, 0};
    if (one_point)
      for (int f = 0; f < 7; ++f) p1[f] = quad[(size_t)f * np + ps];
#pragma unroll
    for (int r = 0; r < kAsmRows; ++r) {
      if (r >= it.row_count || s_row[r] == j) continue;  // the self pair is the FP64 diagonal
      T A = 0, B = 0, C = 0, D = 0;
      const int qs = s_start[r], qe = s_start[r + 1];
      if (one_point) {
        for (int q = qs; q < qe; ++q) {
          T u[7];
          load_qpoint(sq, q, u);
          T a = 0, b = 0, c = 0, d = 0;
          pair_term_unit<T>(u[0], u[1], u[2], u[3], u[4], u[5], p1[0], p1[1], p1[2], p1[3], p1[4], p1[5], kappa, ek,
                            ie, with_d, a, b, c, d);
          A += a * u[6];
          B += b * u[6];
          C += c * u[6];
          D += d * u[6];
        }
        A *= p1[6];
        B *= p1[6];
        C *= p1[6];
        D *= p1[6];
      } else {
        for (int q = qs; q < qe; ++q) {
          T u[7];
          load_qpoint(sq, q, u);
          T a = 0, b = 0, c = 0, d = 0;
          for (int p = ps; p < pe; ++p) {
            pair_term<T>(u[0], u[1], u[2], u[3], u[4], u[5], quad[p], quad[(size_t)np + p],
                         quad[2 * (size_t)np + p], quad[3 * (size_t)np + p], quad[4 * (size_t)np + p],
                         quad[5 * (size_t)np + p], quad[6 * (size_t)np + p], kappa, ie, with_d, a, b, c, d);
          }
          A += a * u[6];
          B += b * u[6];
          C += c * u[6];
          D += d * u[6];
        }
      }
      accf[r] += B * fj - A * hj;
      acch[r] += (D * ie) * fj - C * hj;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < kAsmRows; ++r) {
    double df = (double)accf[r], dh = (double)acch[r];
    for (int o = 16; o > 0; o >>= 1) {
      df += __shfl_xor_sync(0xffffffffu, df, o);
      dh += __shfl_xor_sync(0xffffffffu, dh, o);
    }
    if (lane == 0) {
      s_red[warp][r][0] = df;
      s_red[warp][r][1] = dh;
    }
  }
  __syncthreads();
  if (threadIdx.x < it.row_count) {
    const int r = threadIdx.x, i = s_row[r];
    double df = 0.0, dh = 0.0;
    for (int w = 0; w < kAsmThreads / 32; ++w) {
      df += s_red[w][r][0];
      dh += s_red[w][r][1];
    }
    const double fi = x[i], hi = x[n + i];
    double yf = df + (diag[4 * i + 1] * fi - diag[4 * i + 0] * hi);
    double yh = dh + (diag[4 * i + 3] * fi - diag[4 * i + 2] * hi);
    if (yfar) {
      yf += yfar[i];
      yh += yfar[n + i];
    }
    y[i] = yf;
    y[n + i] = yh;
  }
}

// y_f[i] = sum_j B_ij f_j - A_ij h_j ; y_h[i] = sum_j D_ij f_j - C_ij h_j
// over the leaf's columns (the cached-coefficient stream of
// src/beep/beep.cpp:1049-1062).  Accumulation type AccT.
template <typename T, bool kCompact>
__global__ void __launch_bounds__(kApplyThreads) apply_kernel(
    const NfItem* __restrict__ items, const int32_t* __restrict__ rows, const int64_t* __restrict__ row_off,
    const int32_t* __restrict__ cols, const int64_t* __restrict__ col_off, const int64_t* __restrict__ coef_off,
    const CoefReader<T, kCompact> rd, const double* __restrict__ diag, int n, const double* __restrict__ x,
    const double* __restrict__ yfar, double* __restrict__ y, int n_items, int stage_cols) {
  extern __shared__ unsigned char smem_raw[];
  T* sf = reinterpret_cast<T*>(smem_raw);
  // persistent: a few blocks per SM stride over the items, leaving room on
  // every SM for the far-field kernels that run beside the near field
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
  if (item != blockIdx.x) __syncthreads();  // the previous item's readers of sf / sh are done
  const NfItem it = items[item];
  const int64_t c0 = col_off[it.leaf];
  const int ncols = (int)(col_off[it.leaf + 1] - c0);
  if (ncols > stage_cols) {
    // a neighbourhood beyond the shared-memory staging: x gathered through
    // the column ids (x is L2-resident), one coefficient per lane and step
    using V4 = typename Vec4<T>::type;
    const int64_t blk = coef_off[it.leaf];
    const int lane = threadIdx.x & 31;
    const int64_t r0 = row_off[it.leaf] + it.row_begin;
    for (int r = threadIdx.x >> 5; r < it.row_count; r += blockDim.x >> 5) {
      const int64_t rowp = blk + (int64_t)(it.row_begin + r) * ncols;
      T accf = 0, acch = 0;
      for (int cc = lane; cc < ncols; cc += 32) {
        const V4 v = rd(rowp + cc);
        const int j = cols[c0 + cc];
        const T xf = T(x[j]), xh = T(x[n + j]);
        accf += v.y * xf - v.x * xh;
        acch += v.w * xf - v.z * xh;
      }
      double df = (double)accf, dh = (double)acch;
      for (int o = 16; o > 0; o >>= 1) {
        df += __shfl_xor_sync(0xffffffffu, df, o);
        dh += __shfl_xor_sync(0xffffffffu, dh, o);
      }
      if (lane == 0) {
        const int i = rows[r0 + r];
        const double fi = x[i], hi = x[n + i];
        double yf = df + (diag[4 * i + 1] * fi - diag[4 * i + 0] * hi);
        double yh = dh + (diag[4 * i + 3] * fi - diag[4 * i + 2] * hi);
        if (yfar) {
          yf += yfar[i];
          yh += yfar[n + i];
        }
        y[i] = yf;
        y[n + i] = yh;
      }
    }
    continue;
  }
  T* sh = sf + ncols;
  for (int cc = threadIdx.x; cc < ncols; cc += blockDim.x) {
    const int j = cols[c0 + cc];
    sf[cc] = T(x[j]);
    sh[cc] = T(x[n + j]);
  }
  __syncthreads();
  using V4 = typename Vec4<T>::type;
  const int64_t blk = coef_off[it.leaf];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int64_t r0 = row_off[it.leaf] + it.row_begin;
  for (int r = warp; r < it.row_count; r += nwarps) {
    const int64_t rowp = blk + (int64_t)(it.row_begin + r) * ncols;
    T accf = 0, acch = 0;
    int cc = lane;
    // eight 16-byte (FP32) / 32-byte (FP64) / 12-byte (compact) coefficient
    // loads in flight per lane (compact: twelve ran the apply at 0.148
    // against 0.141 ms on the 40962-patch star)
    constexpr int kU = 8;
    for (; cc + 32 * (kU - 1) < ncols; cc += 32 * kU) {
      V4 v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) v[u] = rd(rowp + cc + 32 * u);
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        accf += v[u].y * sf[cc + 32 * u] - v[u].x * sh[cc + 32 * u];
        acch += v[u].w * sf[cc + 32 * u] - v[u].z * sh[cc + 32 * u];
      }
    }
    for (; cc + 96 < ncols; cc += 128) {
      V4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = rd(rowp + cc + 32 * u);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        accf += v[u].y * sf[cc + 32 * u] - v[u].x * sh[cc + 32 * u];
        acch += v[u].w * sf[cc + 32 * u] - v[u].z * sh[cc + 32 * u];
      }
    }
    for (; cc < ncols; cc += 32) {
      const V4 v = rd(rowp + cc);
      accf += v.y * sf[cc] - v.x * sh[cc];
      acch += v.w * sf[cc] - v.z * sh[cc];
    }
    double df = (double)accf, dh = (double)acch;
    for (int o = 16; o > 0; o >>= 1) {
      df += __shfl_xor_sync(0xffffffffu, df, o);
      dh += __shfl_xor_sync(0xffffffffu, dh, o);
    }
    if (lane == 0) {
      const int i = rows[r0 + r];
      const double fi = x[i], hi = x[n + i];
      double yf = df + (diag[4 * i + 1] * fi - diag[4 * i + 0] * hi);
      double yh = dh + (diag[4 * i + 3] * fi - diag[4 * i + 2] * hi);
      if (yfar) {  // the far field of the same matvec, added in the store
        yf += yfar[i];
        yh += yfar[n + i];
      }
      y[i] = yf;
      y[n + i] = yh;
    }
  }
  }
}

// Columns of a leaf whose x values the apply kernel stages in shared memory
// (2 values each): up to the per-block limit of 227 KB
int apply_stage_cols(size_t elem) { return (int)(227 * 1024 / (2 * elem)); }

}  // namespace

void nf_build_structure(Problem& P) {
  const TreeInfo& T = P.tree;
  NearField& nf = P.nf;
  nf.h_row_off.assign(1, 0);
  nf.h_col_off.assign(1, 0);
  nf.h_coef_off.assign(1, 0);
  nf.h_rows.clear();
  nf.h_cols.clear();
  std::vector<int> seen(P.n, 0);
  std::vector<int> leaves;
  for (size_t k = 0; k < T.nodes.size(); ++k) {
    const TreeNode& nd = T.nodes[k];
    if (!(nd.flags & TREE_LEAF) || nd.content_count == 0) continue;
    leaves.push_back((int)k);
  }
  nf.max_cols = 0;
  for (int leaf : leaves) {
    const TreeNode& nd = T.nodes[leaf];
    for (int c = 0; c < nd.content_count; ++c) {
      int i = T.contents[nd.content_start + c];
      nf.h_rows.push_back(i);
      seen[i]++;
    }
    for (int nb = 0; nb < 27; ++nb) {
      int m = nd.neighbours[nb];
      if (m < 0) continue;
      const TreeNode& mn = T.nodes[m];
      for (int c = 0; c < mn.content_count; ++c) nf.h_cols.push_back(T.contents[mn.content_start + c]);
    }
    int64_t nrows = (int64_t)nf.h_rows.size() - nf.h_row_off.back();
    int64_t ncols = (int64_t)nf.h_cols.size() - nf.h_col_off.back();
    nf.max_cols = std::max<int>(nf.max_cols, (int)ncols);
    nf.h_coef_off.push_back(nf.h_coef_off.back() + nrows * ncols);
    nf.h_row_off.push_back((int64_t)nf.h_rows.size());
    nf.h_col_off.push_back((int64_t)nf.h_cols.size());
  }
  for (int i = 0; i < P.n; ++i)
    if (seen[i] != 1) throw std::runtime_error("octree leaves do not partition the patches");
  nf.n_leaves = (int)leaves.size();
  nf.n_pairs = nf.h_coef_off.back();
  Ctx* ctx = P.ctx;
  nf.rows = upload(ctx, nf.h_rows);
  nf.cols = upload(ctx, nf.h_cols);
  nf.row_off = upload(ctx, nf.h_row_off);
  nf.col_off = upload(ctx, nf.h_col_off);
  nf.coef_off = upload(ctx, nf.h_coef_off);
}

namespace {

constexpr float kCacheRadiusEdges = 4.4f;  // cache radius in edges of the problem's smallest leaf
constexpr double kCacheMaxBytes = 8e9;     // per mesh and kappa

// The mesh's pair cache for kappa, built on `st` if missing (radius shrunk
// while the cache would exceed kCacheMaxBytes).  The caller holds m.mu.
// False when the mesh cannot have one (more than one quadrature point on a
// patch, nothing within the radius).
bool ensure_pair_cache(DevMesh& m, double kappa, float radius, cudaStream_t st) {
  DevMesh::PairCache& pc = m.pair_cache;
  if (pc.kappa == kappa && pc.n_pairs > 0) return true;
  for (int i = 0; i < m.n; ++i)
    if (m.h_quad_off[i + 1] - m.h_quad_off[i] != 1) return false;
  Ctx* ctx = m.ctx;
  pc.off.reset();
  pc.js.reset();
  pc.vals.reset();
  pc.kappa = -1;
  pc.n_pairs = 0;
  const int n = m.n;
  std::vector<float4> hc((size_t)n);
  for (int i = 0; i < n; ++i)
    hc[i] = make_float4((float)m.h_centroid[3 * (size_t)i], (float)m.h_centroid[3 * (size_t)i + 1],
                        (float)m.h_centroid[3 * (size_t)i + 2], 0.f);
  DevBuf dc = upload(ctx, hc);
  DevBuf dcount(ctx, sizeof(int32_t) * (size_t)n);
  std::vector<int32_t> cnt((size_t)n);
  const int grid = (n + 255) / 256;
  // the list pass below must use exactly the r2 of the accepted count
  float R = 0.f, r2 = 0.f;
  int64_t total = -1;
  for (int attempt = 0; attempt < 6 && total < 0; ++attempt) {
    R = radius * std::pow(0.85f, (float)attempt);
    r2 = R * R;
    pair_cache_scan_kernel<<<grid, 256, 0, st>>>(n, dc.as<float4>(), r2, dcount.as<int32_t>(), nullptr, nullptr);
    BP_LAUNCH_CHECK();
    BP_CUDA(cudaMemcpyAsync(cnt.data(), dcount.get(), sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    int64_t t = 0;
    for (int32_t c : cnt) t += c;
    if ((double)t * (sizeof(int32_t) + 6 * sizeof(float)) <= kCacheMaxBytes) total = t;
  }
  if (total <= 0) return false;
  std::vector<int64_t> off((size_t)n + 1, 0);
  int max_row = 0;
  for (int i = 0; i < n; ++i) {
    off[i + 1] = off[i] + cnt[i];
    max_row = std::max(max_row, (int)cnt[i]);
  }
  pc.off = upload(ctx, off);
  pc.js.alloc(ctx, sizeof(int32_t) * (size_t)total);
  BP_CUDA(cudaMemsetAsync(pc.js.get(), 0, sizeof(int32_t) * (size_t)total, st));
  pc.vals.alloc(ctx, 6 * sizeof(float) * (size_t)total);
  pair_cache_scan_kernel<<<grid, 256, 0, st>>>(n, dc.as<float4>(), r2, nullptr, pc.off.as<int64_t>(),
                                               pc.js.as<int32_t>());
  BP_LAUNCH_CHECK();
  DevBuf dq = upload(ctx, m.h_qual_off), dp = upload(ctx, m.h_quad_off);
  int max_q = 0;
  for (int i = 0; i < n; ++i) max_q = std::max(max_q, m.h_qual_off[i + 1] - m.h_qual_off[i]);
  const size_t smem = sizeof(float) * 8 * (size_t)std::max(1, max_q);
  if (smem > 200 * 1024) throw std::invalid_argument("too many qualocation points per patch");
  ensure_dynamic_smem((const void*)pair_cache_coef_kernel, smem);
  pair_cache_coef_kernel<<<n, kAsmThreads, smem, st>>>(pc.off.as<int64_t>(), pc.js.as<int32_t>(), dq.as<int32_t>(),
                                                       m.d_qual.as<double>(), m.n_qual_pts, dp.as<int32_t>(),
                                                       m.d_quad.as<double>(), m.n_quad_pts, (float)kappa,
                                                       pc.vals.as<float>());
  BP_LAUNCH_CHECK();
  BP_CUDA(cudaStreamSynchronize(st));  // the temporaries go back to the context
  pc.kappa = kappa;
  pc.radius = R;
  pc.n_pairs = total;
  pc.max_row = max_row;
  return true;
}

}  // namespace

static std::vector<NfItem> make_items(const Problem& P, int chunk) {
  const NearField& nf = P.nf;
  std::vector<NfItem> items;
  for (int l = 0; l < nf.n_leaves; ++l) {
    int nrows = (int)(nf.h_row_off[l + 1] - nf.h_row_off[l]);
    for (int r = 0; r < nrows; r += chunk) {
      NfItem it;
      it.leaf = l;
      it.row_begin = r;
      it.row_count = std::min(chunk, nrows - r);
      int tq = 0;
      for (int k = 0; k < it.row_count; ++k) {
        int i = nf.h_rows[nf.h_row_off[l] + r + k];
        tq += P.h_qual_off[i + 1] - P.h_qual_off[i];
      }
      it.qual_total = tq;
      items.push_back(it);
    }
  }
  return items;
}

void nf_assemble(Problem& P) {
  Ctx* ctx = P.ctx;
  NearField& nf = P.nf;
  if (!P.asm_stream) {
    BP_CUDA(cudaStreamCreateWithFlags(&P.asm_stream, cudaStreamNonBlocking));
    BP_CUDA(cudaEventCreateWithFlags(&P.asm_in, cudaEventDisableTiming));
    BP_CUDA(cudaEventCreate(&P.asm_t0));
    BP_CUDA(cudaEventCreate(&P.asm_t1));
  }
  std::vector<NfItem> asm_items = make_items(P, kAsmRows);
  int max_tq = 0;
  for (auto& it : asm_items) max_tq = std::max(max_tq, it.qual_total);
  const size_t elem = P.fp64 ? sizeof(double) : sizeof(float);
  const int nq = P.n_qual_pts;
  const int np = P.n_quad_pts;
  const size_t smem = elem * 8 * (size_t)max_tq;
  if (smem > 200 * 1024) throw std::invalid_argument("too many qualocation points per patch");
  // inputs and outputs are placed on the context's stream; the kernels run
  // on the assembly stream once they are
  nf.on_demand = (P.params.flags & BP_FLAG_NEARFIELD_ON_DEMAND) != 0;
  P.asm_gc = upload(ctx, P.h_gc);  // geometric correction per patch
  P.asm_items = upload(ctx, asm_items);
  P.d_diag.alloc(ctx, sizeof(double) * 4 * (size_t)P.n);
  nf.compact = !P.fp64 && (P.params.flags & BP_FLAG_COMPACT_NEARFIELD) != 0;
  if (!nf.on_demand) nf.coef.alloc(ctx, (nf.compact ? 12 : elem * 4) * (size_t)nf.n_pairs);
  // mesh pair caches (built on the context's stream, before the assembly
  // stream is released): a view per placement, the placement of each patch
  int max_list = 0;
  bool use_cache = false;
  if (!P.fp64 && !nf.on_demand && (P.params.flags & BP_FLAG_MESH_PAIR_CACHE) && !P.placements.empty() &&
      nf.max_cols < (1 << 24) && !asm_items.empty()) {
    double hmin = 0;
    for (const TreeNode& nd : P.tree.nodes)
      if ((nd.flags & TREE_LEAF) && nd.content_count > 0) hmin = hmin > 0 ? std::min(hmin, nd.edge) : nd.edge;
    const float radius = kCacheRadiusEdges * (float)hmin;
    std::vector<CacheView> views;
    std::vector<int32_t> inst_of((size_t)P.n, 0);
    int first = 0;
    for (size_t k = 0; k < P.placements.size(); ++k) {
      DevMesh& m = *P.placements[k].mesh;
      CacheView v{nullptr, nullptr, nullptr, first};
      {
        std::lock_guard<std::mutex> lk(m.mu);
        bool ok = false;
        try {
          ok = radius > 0 && ensure_pair_cache(m, P.params.kappa, radius, ctx->stream);
        } catch (const std::exception&) {  // no room for it: integrate as usual
          m.pair_cache.off.reset();
          m.pair_cache.js.reset();
          m.pair_cache.vals.reset();
          m.pair_cache.kappa = -1;
          m.pair_cache.n_pairs = 0;
        }
        if (ok) {
          v.off = m.pair_cache.off.as<int64_t>();
          v.js = m.pair_cache.js.as<int32_t>();
          v.vals = m.pair_cache.vals.as<float>();
          max_list = std::max(max_list, m.pair_cache.max_row);
          use_cache = true;
        }
      }
      for (int i = 0; i < m.n && first + i < P.n; ++i) inst_of[(size_t)first + i] = (int32_t)k;
      first += m.n;
      views.push_back(v);
    }
    if (first != P.n || smem + sizeof(int32_t) * (size_t)max_list > 180 * 1024) use_cache = false;
    if (use_cache) {
      P.d_inst_of = upload(ctx, inst_of);
      P.asm_views = upload(ctx, views);
    }
  }
  BP_CUDA(cudaEventRecord(P.asm_in, ctx->stream));
  const cudaStream_t st = P.asm_stream;
  BP_CUDA(cudaStreamWaitEvent(st, P.asm_in, 0));
  BP_CUDA(cudaEventRecord(P.asm_t0, st));
  {
    const int ng = P.n_gal_pts;
    const int threads = 256;
    const int blocks = (P.n * 32 + threads - 1) / threads;
    singular_kernel<<<blocks, threads, 0, st>>>(P.n, P.d_gal_off.as<int32_t>(), P.d_gal.as<double>(), ng,
                                               P.d_eps.as<double>(), P.asm_gc.as<double>(), P.params.kappa,
                                               P.d_diag.as<double>());
    BP_LAUNCH_CHECK();
  }
  const DevBuf& d_asm_items = P.asm_items;
  if (nf.on_demand) {
    // only the singular diagonal is assembled; every matvec recomputes the
    // pairs over the assembly's work items
    BP_CUDA(cudaEventRecord(P.asm_t1, st));
    nf.instant_smem = smem;
    if (P.fp64)
      ensure_dynamic_smem((const void*)instant_kernel<double>, smem);
    else
      ensure_dynamic_smem((const void*)instant_kernel<float>, smem);
    nf.h_items = asm_items;
    nf.items = upload(ctx, nf.h_items);
    nf.n_items = (int)nf.h_items.size();
    return;
  }
  if (!asm_items.empty()) {
    if (P.fp64) {
      ensure_dynamic_smem((const void*)assemble_kernel<double, false>, smem);
      assemble_kernel<double, false><<<(int)asm_items.size(), kAsmThreads, smem, st>>>(
          d_asm_items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
          nf.col_off.as<int64_t>(), nf.coef_off.as<int64_t>(), P.d_qual_off.as<int32_t>(), P.d_qual.as<double>(), nq,
          P.d_quad_off.as<int32_t>(), P.d_quad.as<double>(), np, P.d_eps.as<double>(), P.params.kappa,
          P.d_diag.as<double>(), CoefWriter<double, false>{nf.coef.as<double4>()});
    } else if (use_cache) {
      const size_t csmem = smem + sizeof(int32_t) * (size_t)max_list;
      auto launch = [&](auto kernel, auto out) {
        ensure_dynamic_smem((const void*)kernel, csmem);
        kernel<<<(int)asm_items.size(), kAsmThreads, csmem, st>>>(
            d_asm_items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
            nf.col_off.as<int64_t>(), nf.coef_off.as<int64_t>(), P.d_qual_off.as<int32_t>(), P.d_qual_f.as<float>(),
            nq, P.d_quad_off.as<int32_t>(), P.d_quad_f.as<float>(), np, P.d_eps.as<double>(), (float)P.params.kappa,
            P.d_inst_of.as<int32_t>(), P.asm_views.as<CacheView>(), max_list, max_tq, out);
      };
      if (nf.compact) {
        uint2* p01 = nf.coef.as<uint2>();
        launch(assemble_cached_kernel<true>, CoefWriter<float, true>{p01, reinterpret_cast<uint32_t*>(p01 + nf.n_pairs)});
      } else {
        launch(assemble_cached_kernel<false>, CoefWriter<float, false>{nf.coef.as<float4>()});
      }
    } else if (nf.compact) {
      uint2* p01 = nf.coef.as<uint2>();
      const CoefWriter<float, true> out{p01, reinterpret_cast<uint32_t*>(p01 + nf.n_pairs)};
      ensure_dynamic_smem((const void*)assemble_kernel<float, true>, smem);
      assemble_kernel<float, true><<<(int)asm_items.size(), kAsmThreads, smem, st>>>(
          d_asm_items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
          nf.col_off.as<int64_t>(), nf.coef_off.as<int64_t>(), P.d_qual_off.as<int32_t>(), P.d_qual_f.as<float>(), nq,
          P.d_quad_off.as<int32_t>(), P.d_quad_f.as<float>(), np, P.d_eps.as<double>(), (float)P.params.kappa,
          P.d_diag.as<double>(), out);
    } else {
      ensure_dynamic_smem((const void*)assemble_kernel<float, false>, smem);
      assemble_kernel<float, false><<<(int)asm_items.size(), kAsmThreads, smem, st>>>(
          d_asm_items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
          nf.col_off.as<int64_t>(), nf.coef_off.as<int64_t>(), P.d_qual_off.as<int32_t>(), P.d_qual_f.as<float>(), nq,
          P.d_quad_off.as<int32_t>(), P.d_quad_f.as<float>(), np, P.d_eps.as<double>(), (float)P.params.kappa,
          P.d_diag.as<double>(), CoefWriter<float, false>{nf.coef.as<float4>()});
    }
    BP_LAUNCH_CHECK();
  }
  BP_CUDA(cudaEventRecord(P.asm_t1, st));
  // apply work items; the apply kernel's shared memory holds the x values of
  // a leaf's columns (leaves with more columns than fit gather x instead)
  const size_t apply_smem = 2 * elem * (size_t)std::min(nf.max_cols, apply_stage_cols(elem));
  if (P.fp64)
    ensure_dynamic_smem((const void*)apply_kernel<double, false>, apply_smem);
  else if (nf.compact)
    ensure_dynamic_smem((const void*)apply_kernel<float, true>, apply_smem);
  else
    ensure_dynamic_smem((const void*)apply_kernel<float, false>, apply_smem);
  // rows per apply item: 64, halved (down to 8) while the grid would hold
  // fewer than 8 blocks per SM, so small problems still fill the GPU
  int rows_per_item = kApplyRows;
  nf.h_items = make_items(P, rows_per_item);
  while (rows_per_item > 8 && (int)nf.h_items.size() < 8 * ctx->sm_count) {
    rows_per_item /= 2;
    nf.h_items = make_items(P, rows_per_item);
  }
  // largest items (rows x neighbourhood columns) first: the persistent grid
  // starts the long ones early instead of ending on them (measured: the
  // apply 0.170 against 0.179 ms on the 40962-patch star).  Every item
  // writes its own rows, so the order changes no result.
  std::stable_sort(nf.h_items.begin(), nf.h_items.end(), [&](const NfItem& a, const NfItem& b) {
    const long long wa = (long long)a.row_count * (nf.h_col_off[a.leaf + 1] - nf.h_col_off[a.leaf]);
    const long long wb = (long long)b.row_count * (nf.h_col_off[b.leaf + 1] - nf.h_col_off[b.leaf]);
    return wa > wb;
  });
  nf.items = upload(ctx, nf.h_items);
  nf.n_items = (int)nf.h_items.size();
}

void nf_join(Problem& P) {
  if (!P.asm_stream) return;
  BP_CUDA(cudaStreamWaitEvent(P.ctx->stream, P.asm_t1, 0));
  // later users of these blocks run on the context's stream, after the join
  P.asm_gc.reset();
  P.asm_items.reset();
  P.asm_views.reset();
}

int nf_apply(Problem& P, const double* x_dev, double* y_dev, const double* yfar_dev, cudaStream_t stream) {
  NearField& nf = P.nf;
  if (nf.n_items == 0) return 0;
  if (nf.on_demand) {
    const int nq = P.n_qual_pts, np = P.n_quad_pts;
    if (P.fp64)
      instant_kernel<double><<<nf.n_items, kAsmThreads, nf.instant_smem, stream>>>(
          nf.items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
          nf.col_off.as<int64_t>(), P.d_qual_off.as<int32_t>(), P.d_qual.as<double>(), nq, P.d_quad_off.as<int32_t>(),
          P.d_quad.as<double>(), np, P.d_eps.as<double>(), P.params.kappa, P.d_diag.as<double>(), P.n, x_dev,
          yfar_dev, y_dev);
    else
      instant_kernel<float><<<nf.n_items, kAsmThreads, nf.instant_smem, stream>>>(
          nf.items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
          nf.col_off.as<int64_t>(), P.d_qual_off.as<int32_t>(), P.d_qual_f.as<float>(), nq, P.d_quad_off.as<int32_t>(),
          P.d_quad_f.as<float>(), np, P.d_eps.as<double>(), (float)P.params.kappa, P.d_diag.as<double>(), P.n, x_dev,
          yfar_dev, y_dev);
    BP_LAUNCH_CHECK();
    return 1;
  }
  const size_t elem = P.fp64 ? sizeof(double) : sizeof(float);
  const int stage = apply_stage_cols(elem);
  const size_t smem = 2 * elem * (size_t)std::min(nf.max_cols, stage);
  const int grid = std::min(nf.n_items, kApplyBlocksPerSm * P.ctx->sm_count);
  if (P.fp64) {
    apply_kernel<double, false><<<grid, kApplyThreads, smem, stream>>>(
        nf.items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
        nf.col_off.as<int64_t>(), nf.coef_off.as<int64_t>(), CoefReader<double, false>{nf.coef.as<double4>()},
        P.d_diag.as<double>(), P.n, x_dev, yfar_dev, y_dev, nf.n_items, stage);
  } else if (nf.compact) {
    apply_kernel<float, true><<<grid, kApplyThreads, smem, stream>>>(
        nf.items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
        nf.col_off.as<int64_t>(), nf.coef_off.as<int64_t>(),
        CoefReader<float, true>{nf.coef.as<uint2>(), reinterpret_cast<const uint32_t*>(nf.coef.as<uint2>() + nf.n_pairs)},
        P.d_diag.as<double>(), P.n, x_dev, yfar_dev, y_dev, nf.n_items, stage);
  } else {
    apply_kernel<float, false><<<grid, kApplyThreads, smem, stream>>>(
        nf.items.as<NfItem>(), nf.rows.as<int32_t>(), nf.row_off.as<int64_t>(), nf.cols.as<int32_t>(),
        nf.col_off.as<int64_t>(), nf.coef_off.as<int64_t>(), CoefReader<float, false>{nf.coef.as<float4>()},
        P.d_diag.as<double>(), P.n, x_dev, yfar_dev, y_dev, nf.n_items, stage);
  }
  BP_LAUNCH_CHECK();
  return 1;
}

}  // namespace bp
