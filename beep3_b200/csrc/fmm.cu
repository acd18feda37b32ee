// Far field of the BEM matvec on sm_100a: the 12-channel screened-Coulomb
// plane-wave FMM of the reference (FMM_BEM_Octree::solve,
// src/fmm/fmm_bem_hybrid.h:183-279; operators in src/fmm/fmm.h).
//
// Channels (src/bem/node_patch.h:339-394): with a = patch area, n its normal,
// eps the dielectric ratio, charges [a f n, a h] and [a f n/eps, a h/eps]
// are screened with kappa (channels 0-7), [a f n/eps, a h] with beta0 = 1e-10
// (channels 8-11, standing in for Laplace).  Each matvec runs:
//   P2M   one launch for all non-empty childless nodes (yformmp)
//   M2M   one launch per level, bottom-up, one block per parent gathering its
//         children (ympshift: rotate, z-shift, rotate back)
//   M2X   one launch for all non-empty nodes below the root: multipole ->
//         6 directional plane waves (rotate z->y / z->x, ympoletoexp,
//         yftophys), with the parent level's tables
//   X2L   one launch for all parents that are neither leaf nor shadow: the
//         diagonal plane-wave translations of the 1512-entry interaction list
//         (translate_up/down_wave) accumulated in shared memory per target
//         child, then converted to local expansions (yphystof,
//         yexptolocal, rotate back) -- translation and conversion fused, no
//         accumulator ever goes to HBM
//   L2L   one launch per level, top-down (ylcshift)
//   L2P   one launch over leaves: potential, field and Hessian of the 12
//         local expansions at each patch centroid, reduced on the fly to the
//         f and h results of FMM_results_to_BEM (src/bem/bem_kernels.cpp:12-121)
// Precision: T = double (FP64 engine) or float (mixed engine); tables are
// computed on the host in FP64 (fmm_tables.cpp) and rounded to T.
// Expansions are stored [node][channel][tri(n, m)] as complex T; plane waves
// [node][direction][channel][i].
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "engine.h"
#include "fmm_tables.h"

namespace bp {

namespace {

constexpr int kCh = 12;
constexpr int kMaxNT = 18;

template <typename T>
struct C2T;
template <>
struct C2T<float> {
  using type = float2;
};
template <>
struct C2T<double> {
  using type = double2;
};

template <typename C>
__device__ __forceinline__ C cmk(decltype(C::x) a, decltype(C::x) b) {
  C c;
  c.x = a;
  c.y = b;
  return c;
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
  return cmk<C>(a.x + b.x, a.y + b.y);
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
  return cmk<C>(a.x - b.x, a.y - b.y);
}
template <typename C>
__device__ __forceinline__ C cconj(C a) {
  return cmk<C>(a.x, -a.y);
}
template <typename C, typename T>
__device__ __forceinline__ C cscale(C a, T s) {
  return cmk<C>(a.x * s, a.y * s);
}

__host__ __device__ __forceinline__ int tri(int n, int m) { return m + n * (n + 1) / 2; }

// Device view of the tables; arrays indexed by lg = 2*level + group
// (group 0: kappa, group 1: beta0).
template <typename T>
struct Tables {
  using C = typename C2T<T>::type;
  int nt, E, nl, np_max, nlev;
  const T* rot;     // 4 rotations [rdpi2, rdmpi2, rdsq3, rdmsq3], each (nt+1)^2 (2nt+1)
  const T* sfac;    // [E]
  const T* weights; // [nl]
  const int* numfour;    // [nl]
  const int* numphys;    // [lg][nl]
  const int* nexptot;    // [lg]
  const int* nexptotp;   // [lg]
  const T* scale;        // [lg]
  const T* betascal;     // [lg]
  const T* beta;         // [2]
  const T* rlsc;         // [lg][E][nl]
  const C* fexpe;        // concatenated per lg
  const C* fexpo;
  const C* fexpback;
  const int* fexpe_off;  // [lg]
  const int* fexpo_off;
  const int* fexpback_off;
  const C* xs;           // [lg][3][np_max]
  const C* ys;
  const T* zs;
  const T* mpshift;      // [lg][(nt+1)^3]
  const T* lcshift;
  __device__ const T* R(int which) const { return rot + (size_t)which * (nt + 1) * (nt + 1) * (2 * nt + 1); }
  __device__ T rd(const T* r, int l, int mp, int m) const {
    return r[((size_t)l * (nt + 1) + mp) * (2 * nt + 1) + m + nt];
  }
};

enum { ROT_PI2 = 0, ROT_MPI2 = 1, ROT_SQ3 = 2, ROT_MSQ3 = 3 };

// ---------------------------------------------------------------- device helpers
// scaled modified spherical Bessel functions b[n] = i_n(x)/scal^n, n <= nb
// (series for x <= 1e-4, zero above 100, else Miller's backward recurrence
// normalised with sinh(x)/x), as the host tables.
template <typename T>
__device__ void bessel_in_dev(T scal, T x, int nb, T* b) {
  const T inv = T(1) / scal;
  if (x <= T(1e-4)) {
    const T xs = x * inv, t2 = T(0.5) * x * x;
    T t1 = 1;
    b[0] = T(1) + t2 / T(3);
    for (int i = 1; i <= nb; ++i) {
      t1 *= xs / T(2 * i + 1);
      if (t1 <= T(1e-300)) t1 = 0;
      b[i] = t1 * (T(1) + t2 / T(2 * i + 3));
    }
    return;
  }
  if (x > T(100)) {
    for (int i = 0; i <= nb; ++i) b[i] = 0;
    return;
  }
  // backward recurrence in double for range, result rounded to T
  const int top = nb + 30 + (int)(2.0 * (double)x);
  double vp1 = 0.0, v = 1e-300, scale_acc = 1.0;
  double keep[kMaxNT + 4];
  const double xd = (double)x;
  for (int n = top; n >= 1; --n) {
    double vm1 = vp1 + (2.0 * n + 1.0) / xd * v;
    vp1 = v;
    v = vm1;
    if (n - 1 <= nb) keep[n - 1] = v;
    if (fabs(v) > 1e250) {
      v *= 1e-250;
      vp1 *= 1e-250;
      for (int k = n - 1; k <= nb; ++k) keep[k] *= 1e-250;
    }
  }
  (void)scale_acc;
  const double norm = (sinh(xd) / xd) / keep[0];
  double c = 1.0;
  const double invd = 1.0 / (double)scal;
  for (int i = 0; i <= nb; ++i) {
    const double bi = keep[i] * norm * c;
    b[i] = (T)bi;
    c *= invd;
    if (fabs(bi) <= 1e-300) c = 0.0;
  }
}

// P_n^m(x) with the Condon-Shortley phase into p[tri(n, m)], n <= nmax
template <typename T>
__device__ void legendre_dev(int nmax, T x, T* p) {
  const T u = -sqrt(T(1) - x * x);
  p[0] = 1;
  for (int m = 0; m <= nmax; ++m) {
    if (m > 0) p[tri(m, m)] = p[tri(m - 1, m - 1)] * u * T(2 * m - 1);
    if (m < nmax) p[tri(m + 1, m)] = T(2 * m + 1) * x * p[tri(m, m)];
    for (int n = m + 2; n <= nmax; ++n)
      p[tri(n, m)] = ((T(2) * n - T(1)) * x * p[tri(n - 1, m)] - T(n + m - 1) * p[tri(n - 2, m)]) / T(n - m);
  }
}

// BasicNodePatch::get_fmm_charge_equiv for all 12 channels
template <typename T>
__device__ __forceinline__ void patch_charges(const double* area, const double* normal, const double* eps,
                                              const double* x, int n, int i, T q[kCh]) {
  const double a = area[i], e = eps[i], f = x[i], h = x[n + i];
  const double nx = normal[3 * i], ny = normal[3 * i + 1], nz = normal[3 * i + 2];
  q[0] = (T)(a * f * nx);
  q[1] = (T)(a * f * ny);
  q[2] = (T)(a * f * nz);
  q[3] = (T)(a * h);
  q[4] = (T)(a * f * nx / e);
  q[5] = (T)(a * f * ny / e);
  q[6] = (T)(a * f * nz / e);
  q[7] = (T)(a * h / e);
  q[8] = (T)(a * f * nx / e);
  q[9] = (T)(a * f * ny / e);
  q[10] = (T)(a * f * nz / e);
  q[11] = (T)(a * h);
}

// ---------------------------------------------------------------- P2M
struct P2mItem {
  int node, level, start, count;
  double c[3];
};

constexpr int kP2mChunk = 32;

template <typename T>
__global__ void __launch_bounds__(256) p2m_kernel(const __grid_constant__ Tables<T> tb, const P2mItem* __restrict__ items,
                                                  const int32_t* __restrict__ contents,
                                                  const double* __restrict__ centroid, const double* __restrict__ area,
                                                  const double* __restrict__ normal, const double* __restrict__ eps,
                                                  const double* __restrict__ x, int n,
                                                  typename C2T<T>::type* __restrict__ M) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E, NT = tb.nt;
  C* basis = reinterpret_cast<C*>(smem_raw);                       // [chunk][2][E]
  T* q = reinterpret_cast<T*>(basis + 2 * kP2mChunk * E);          // [chunk][12]
  const P2mItem it = items[blockIdx.x];
  C acc[(kCh * ((kMaxNT + 1) * (kMaxNT + 2) / 2) + 255) / 256];
  const int nout = kCh * E;
  for (int k = 0; k < (nout + 255) / 256; ++k) acc[k] = cmk<C>(0, 0);
  for (int base = 0; base < it.count; base += kP2mChunk) {
    const int cnt = min(kP2mChunk, it.count - base);
    const int t = threadIdx.x;
    if (t < 2 * cnt) {
      const int pl = t >> 1, g = t & 1;
      const int i = contents[it.start + base + pl];
      const double rx = centroid[3 * i] - it.c[0], ry = centroid[3 * i + 1] - it.c[1],
                   rz = centroid[3 * i + 2] - it.c[2];
      double proj = rx * rx + ry * ry;
      const double rr = proj + rz * rz;
      proj = sqrt(proj);
      const double d = sqrt(rr);
      const double PREC = 2.220446049250313e-16;
      const T ct = (T)((d <= PREC) ? 1.0 : rz / d);
      C e1 = (proj <= PREC * d) ? cmk<C>(1, 0) : cmk<C>((T)(rx / proj), (T)(-ry / proj));
      const int lg = 2 * it.level + g;
      T bi[kMaxNT + 2];
      bessel_in_dev<T>(tb.scale[lg], (T)(d * (double)tb.beta[g]), NT, bi);
      T p[(kMaxNT + 1) * (kMaxNT + 2) / 2];
      legendre_dev<T>(NT, ct, p);
      C* bs = basis + ((size_t)pl * 2 + g) * E;
      bs[0] = cmk<C>(bi[0], 0);
      C ephi = e1;  // e^{-i m phi} for m = 1
      for (int m = 1; m <= NT; ++m) {
        for (int l = m; l <= NT; ++l) {
          const T cp = bi[l] * tb.sfac[tri(l, m)] * p[tri(l, m)];
          bs[tri(l, m)] = cscale(ephi, cp);
        }
        ephi = cmul(ephi, e1);
      }
      for (int l = 1; l <= NT; ++l) bs[tri(l, 0)] = cmk<C>(p[tri(l, 0)] * bi[l] * tb.sfac[tri(l, 0)], 0);
    } else if (t >= 64 && t < 64 + cnt) {
      const int pl = t - 64;
      const int i = contents[it.start + base + pl];
      T qq[kCh];
      patch_charges<T>(area, normal, eps, x, n, i, qq);
      for (int c = 0; c < kCh; ++c) q[pl * kCh + c] = qq[c];
    }
    __syncthreads();
    for (int k = 0; k < (nout + 255) / 256; ++k) {
      const int o = threadIdx.x + 256 * k;
      if (o < nout) {
        const int ch = o / E, e = o - ch * E;
        const int g = ch >= 8 ? 1 : 0;
        C a = acc[k];
        for (int pl = 0; pl < cnt; ++pl) {
          const C b = basis[((size_t)pl * 2 + g) * E + e];
          const T qc = q[pl * kCh + ch];
          a.x += b.x * qc;
          a.y += b.y * qc;
        }
        acc[k] = a;
      }
    }
    __syncthreads();
  }
  for (int k = 0; k < (nout + 255) / 256; ++k) {
    const int o = threadIdx.x + 256 * k;
    if (o < nout) M[(size_t)it.node * nout + o] = acc[k];
  }
}

// ---------------------------------------------------------------- M2M / L2L
// out += shift of `in` for one child octant: conj(ephi) phase, rotation,
// z-shift (coefficients dc[m][n][n']), signed rotation back, ephi phase
// (ympshift / ylcshift, src/fmm/fmm.h:1718-2051).  All threads of the block
// take part; w1, w2 are [12][E] shared buffers; out is a shared accumulator.
template <typename T>
__device__ void shift_block(const Tables<T>& tb, int ifl, bool multipole, int level, const typename C2T<T>::type* in,
                            typename C2T<T>::type* w1, typename C2T<T>::type* w2, typename C2T<T>::type* out,
                            const T* rd, int c0, int nc) {
  using C = typename C2T<T>::type;
  const int E = tb.E, NT = tb.nt, nout = nc * E;
  const T arg = T(0.70710678118654752440);
  C e1;
  if (multipole) {
    if (ifl == 4 || ifl == 8) e1 = cmk<C>(-arg, arg);
    else if (ifl == 3 || ifl == 7) e1 = cmk<C>(arg, arg);
    else if (ifl == 1 || ifl == 5) e1 = cmk<C>(arg, -arg);
    else e1 = cmk<C>(-arg, -arg);
  } else {
    if (ifl == 4 || ifl == 8) e1 = cmk<C>(arg, -arg);
    else if (ifl == 3 || ifl == 7) e1 = cmk<C>(-arg, -arg);
    else if (ifl == 1 || ifl == 5) e1 = cmk<C>(-arg, arg);
    else e1 = cmk<C>(arg, arg);
  }
  // ephi[m] = e1^m
  auto ephi = [&](int m) {
    C r = cmk<C>(1, 0);
    for (int k = 0; k < m; ++k) r = cmul(r, e1);
    return r;
  };
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    const int e = o % E;
    int l = 0;
    while (tri(l + 1, 0) <= e) ++l;
    const int m = e - tri(l, 0);
    w1[o] = cmul(cconj(ephi(m)), in[o]);
  }
  __syncthreads();
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    const int ch = o / E, e = o - ch * E;
    int l = 0;
    while (tri(l + 1, 0) <= e) ++l;
    const int m = e - tri(l, 0);
    const C* src = w1 + ch * E;
    C v = cscale(src[tri(l, 0)], tb.rd(rd, l, 0, m));
    for (int mp = 1; mp <= l; ++mp) {
      const C s = src[tri(l, mp)];
      v = cadd(v, cadd(cscale(s, tb.rd(rd, l, mp, m)), cscale(cconj(s), tb.rd(rd, l, mp, -m))));
    }
    w2[o] = v;
  }
  __syncthreads();
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    const int ch = o / E, e = o - ch * E;
    int nn = 0;
    while (tri(nn + 1, 0) <= e) ++nn;
    const int m = e - tri(nn, 0);
    const int lg = 2 * level + (c0 + ch >= 8 ? 1 : 0);
    const T* dc = (multipole ? tb.mpshift : tb.lcshift) + (size_t)lg * (NT + 1) * (NT + 1) * (NT + 1);
    const C* src = w2 + ch * E;
    C v = cmk<C>(0, 0);
    for (int nd = m; nd <= NT; ++nd) {
      const T c = dc[((size_t)m * (NT + 1) + nn) * (NT + 1) + nd];
      v = cadd(v, cscale(src[tri(nd, m)], c));
    }
    w1[o] = v;
  }
  __syncthreads();
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    const int ch = o / E, e = o - ch * E;
    int l = 0;
    while (tri(l + 1, 0) <= e) ++l;
    const int m = e - tri(l, 0);
    const C* src = w1 + ch * E;
    C v = cscale(src[tri(l, 0)], tb.rd(rd, l, 0, m));
    if (m & 1) v = cmk<C>(-v.x, -v.y);
    for (int mp = 1; mp <= l; ++mp) {
      const C s = src[tri(l, mp)];
      const C t = cadd(cscale(s, tb.rd(rd, l, mp, m)), cscale(cconj(s), tb.rd(rd, l, mp, -m)));
      // even m: minus for odd mp, plus for even mp; odd m: the reverse
      const bool plus = ((mp & 1) == 0) != ((m & 1) == 1);
      v = plus ? cadd(v, t) : csub(v, t);
    }
    out[o] = cadd(out[o], cmul(ephi(m), v));
  }
  __syncthreads();
}

struct ShiftItem {
  int parent, first_child, n_children;  // children listed in shift_children
};
struct ShiftChild {
  int node, octant;
};

// M2M: one block per (parent, channel) gathering its children in order
template <typename T>
__global__ void __launch_bounds__(64) m2m_kernel(const __grid_constant__ Tables<T> tb, const ShiftItem* __restrict__ items,
                                                 const ShiftChild* __restrict__ children, int child_level,
                                                 typename C2T<T>::type* __restrict__ M) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E;
  C* w1 = reinterpret_cast<C*>(smem_raw);
  C* w2 = w1 + E;
  C* acc = w2 + E;
  C* in = acc + E;
  const ShiftItem it = items[blockIdx.x / kCh];
  const int ch = blockIdx.x % kCh;
  for (int o = threadIdx.x; o < E; o += blockDim.x) acc[o] = cmk<C>(0, 0);
  for (int c = 0; c < it.n_children; ++c) {
    const ShiftChild sc = children[it.first_child + c];
    __syncthreads();
    for (int o = threadIdx.x; o < E; o += blockDim.x) in[o] = M[((size_t)sc.node * kCh + ch) * E + o];
    __syncthreads();
    const T* rd = tb.R(sc.octant > 4 ? ROT_MSQ3 : ROT_SQ3);
    shift_block<T>(tb, sc.octant, true, child_level, in, w1, w2, acc, rd, ch, 1);
  }
  __syncthreads();
  for (int o = threadIdx.x; o < E; o += blockDim.x) M[((size_t)it.parent * kCh + ch) * E + o] = acc[o];
}

// L2L: one block per (child, channel), local_child += shift(local_parent)
template <typename T>
__global__ void __launch_bounds__(64) l2l_kernel(const __grid_constant__ Tables<T> tb, const ShiftItem* __restrict__ items,
                                                 const ShiftChild* __restrict__ children, int parent_level,
                                                 typename C2T<T>::type* __restrict__ L) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E;
  C* w1 = reinterpret_cast<C*>(smem_raw);
  C* w2 = w1 + E;
  C* acc = w2 + E;
  C* in = acc + E;
  const ShiftItem it = items[blockIdx.x / kCh];
  const int ch = blockIdx.x % kCh;
  const ShiftChild sc = children[it.first_child];
  for (int o = threadIdx.x; o < E; o += blockDim.x) {
    in[o] = L[((size_t)it.parent * kCh + ch) * E + o];
    acc[o] = L[((size_t)sc.node * kCh + ch) * E + o];
  }
  __syncthreads();
  const T* rd = tb.R(sc.octant > 4 ? ROT_SQ3 : ROT_MSQ3);
  shift_block<T>(tb, sc.octant, false, parent_level, in, w1, w2, acc, rd, ch, 1);
  for (int o = threadIdx.x; o < E; o += blockDim.x) L[((size_t)sc.node * kCh + ch) * E + o] = acc[o];
}

// ---------------------------------------------------------------- M2X
// rotation application out(l,m) = in(l,0) d(l,0,m) + sum_mp in(l,mp) d(l,mp,m) + conj(in(l,mp)) d(l,mp,-m)
template <typename T>
__device__ __forceinline__ typename C2T<T>::type rotate_one(const Tables<T>& tb, const typename C2T<T>::type* in,
                                                            const T* rd, int l, int m) {
  using C = typename C2T<T>::type;
  C v = cscale(in[tri(l, 0)], tb.rd(rd, l, 0, m));
  for (int mp = 1; mp <= l; ++mp) {
    const C s = in[tri(l, mp)];
    v = cadd(v, cadd(cscale(s, tb.rd(rd, l, mp, m)), cscale(cconj(s), tb.rd(rd, l, mp, -m))));
  }
  return v;
}

struct M2xItem {
  int node, level;  // level of the node; tables of level-1
};

constexpr int kM2xThreads = 128;

// one block per (node, channel): three multipole -> (Fourier -> physical)
// conversions, one per direction pair
template <typename T>
__global__ void __launch_bounds__(kM2xThreads) m2x_kernel(const __grid_constant__ Tables<T> tb,
                                                          const M2xItem* __restrict__ items,
                                                          const typename C2T<T>::type* __restrict__ M,
                                                          typename C2T<T>::type* __restrict__ W) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E, NT = tb.nt, nl = tb.nl;
  C* mp = reinterpret_cast<C*>(smem_raw);  // [E]
  C* rot = mp + E;                          // [E]
  C* fu = rot + E;                          // [nexptot]
  C* fd = fu + 64;                          // [nexptot]
  const M2xItem it = items[blockIdx.x / kCh];
  const int ch = blockIdx.x % kCh;
  const int lg = 2 * (it.level - 1) + (ch >= 8 ? 1 : 0);
  const int nexptot = tb.nexptot[lg], np = tb.nexptotp[lg];
  const int* numphys = tb.numphys + (size_t)lg * nl;
  const T* rl = tb.rlsc + (size_t)lg * E * nl;
  const C* fexpe = tb.fexpe + tb.fexpe_off[lg];
  const C* fexpo = tb.fexpo + tb.fexpo_off[lg];
  for (int e = threadIdx.x; e < E; e += blockDim.x) mp[e] = M[((size_t)it.node * kCh + ch) * E + e];
  __syncthreads();
  for (int pair = 0; pair < 3; ++pair) {
    // rotated multipole: pair 0 none, 1 rotate_ztoy(rdmpi2), 2 rotate_ztox(rdpi2)
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
      if (pair == 0) {
        rot[e] = mp[e];
      } else {
        int l = 0;
        while (tri(l + 1, 0) <= e) ++l;
        const int m = e - tri(l, 0);
        if (pair == 1) {
          // mwork = (-i)^m mpole, then rotation by rdmpi2
          C v = cscale(mp[tri(l, 0)], tb.rd(tb.R(ROT_MPI2), l, 0, m));
          for (int q = 1; q <= l; ++q) {
            C s = mp[tri(l, q)];
            // (-i)^q
            switch (q & 3) {
              case 1: s = cmk<C>(s.y, -s.x); break;
              case 2: s = cmk<C>(-s.x, -s.y); break;
              case 3: s = cmk<C>(-s.y, s.x); break;
              default: break;
            }
            v = cadd(v, cadd(cscale(s, tb.rd(tb.R(ROT_MPI2), l, q, m)), cscale(cconj(s), tb.rd(tb.R(ROT_MPI2), l, q, -m))));
          }
          rot[e] = v;
        } else {
          rot[e] = rotate_one<T>(tb, mp, tb.R(ROT_PI2), l, m);
        }
      }
    }
    __syncthreads();
    // ympoletoexp: Fourier modes (up, down)
    for (int j = threadIdx.x; j < nexptot; j += blockDim.x) {
      int l = 0, ntot = 0;
      while (ntot + tb.numfour[l] <= j) {
        ntot += tb.numfour[l];
        ++l;
      }
      const int mth = j - ntot;
      C z1 = cmk<C>(0, 0), z2 = cmk<C>(0, 0);
      for (int nm = mth; nm <= NT; nm += 2) z1 = cadd(z1, cscale(rot[tri(nm, mth)], rl[(size_t)tri(nm, mth) * nl + l]));
      for (int nm = mth + 1; nm <= NT; nm += 2) z2 = cadd(z2, cscale(rot[tri(nm, mth)], rl[(size_t)tri(nm, mth) * nl + l]));
      fu[j] = cadd(z1, z2);
      const T sgn = (mth & 1) ? T(-1) : T(1);
      fd[j] = cscale(csub(z1, z2), sgn);
    }
    __syncthreads();
    // yftophys for both
    for (int o = threadIdx.x; o < 2 * np; o += blockDim.x) {
      const int which = o / np, iw = o - which * np;
      const C* mf = which ? fd : fu;
      int l = 0, nptot = 0, nftot = 0, be = 0, bo = 0;
      while (nptot + numphys[l] / 2 <= iw) {
        nptot += numphys[l] / 2;
        nftot += tb.numfour[l];
        be += (numphys[l] / 2) * (tb.numfour[l] / 2);
        bo += (numphys[l] / 2) * ((tb.numfour[l] - 1) / 2);
        ++l;
      }
      const int iv = iw - nptot;
      const int nfo = tb.numfour[l];
      C val = mf[nftot];
      int k = 0;
      for (int mm = 1; mm < nfo; mm += 2, ++k) {
        const T s = (k & 1) ? T(-2) : T(2);
        const C fe = fexpe[be + iv * (nfo / 2) + k];
        const C pm = mf[nftot + mm];
        val.y += s * (fe.x * pm.x - fe.y * pm.y);
      }
      k = 0;
      for (int mm = 2; mm < nfo; mm += 2, ++k) {
        const T s = (k & 1) ? T(2) : T(-2);
        const C fo = fexpo[bo + iv * ((nfo - 1) / 2) + k];
        const C pm = mf[nftot + mm];
        val.x += s * (fo.x * pm.x - fo.y * pm.y);
      }
      const int dir = 2 * pair + which;  // 0 up 1 down 2 north 3 south 4 east 5 west
      W[(((size_t)it.node * 6 + dir) * kCh + ch) * tb.np_max + iw] = val;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- X2L
struct XlItem {
  int parent_level;
  int first_entry[3], n_entries[3];  // entries of each direction pair (UP/DOWN, N/S, E/W)
  int targets[8];                    // target child node ids (-1 absent or shadow)
};
struct XlEntry {
  int src;          // source node id
  signed char dir, targ, a, b, c, up;
};

constexpr int kXlGroup = 96;  // threads per direction pair (>= nexptotp)
constexpr int kXlThreads = 3 * kXlGroup;

// One block per (parent, channel); thread group g handles direction pair g:
// its diagonal translations accumulated in shared memory per (direction,
// target child), then yphystof + yexptolocal + rotation back per target;
// the three pairs' local expansions are summed in a fixed order.
template <typename T>
__global__ void __launch_bounds__(kXlThreads) x2l_kernel(const __grid_constant__ Tables<T> tb,
                                                         const XlItem* __restrict__ items,
                                                         const XlEntry* __restrict__ entries,
                                                         const typename C2T<T>::type* __restrict__ W,
                                                         typename C2T<T>::type* __restrict__ L) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E, nl = tb.nl, NPM = tb.np_max;
  C* acc = reinterpret_cast<C*>(smem_raw);  // [6 dirs][8 targets][NPM]
  C* mf = acc + 6 * 8 * NPM;                 // [3 pairs][2][64]
  C* loc = mf + 3 * 2 * 64;                  // [3][E]
  C* out = loc + 3 * E;                      // [3][E]
  const XlItem it = items[blockIdx.x / kCh];
  const int ch = blockIdx.x % kCh;
  const int lg = 2 * it.parent_level + (ch >= 8 ? 1 : 0);
  const int np = tb.nexptotp[lg], nexptot = tb.nexptot[lg];
  const int g = threadIdx.x / kXlGroup, lt = threadIdx.x - g * kXlGroup;
  for (int o = threadIdx.x; o < 6 * 8 * NPM; o += blockDim.x) acc[o] = cmk<C>(0, 0);
  __syncthreads();
  // translations of pair g
  if (lt < np) {
    const int i = lt;
    const C* xs = tb.xs + (size_t)lg * 3 * NPM;
    const C* ys = tb.ys + (size_t)lg * 3 * NPM;
    const T* zs = tb.zs + (size_t)lg * 3 * NPM;
    const int e0 = it.first_entry[g], ne = it.n_entries[g];
    for (int k = 0; k < ne; ++k) {
      const XlEntry en = entries[e0 + k];
      const C w = W[(((size_t)en.src * 6 + en.dir) * kCh + ch) * NPM + i];
      C t;
      if (en.up) {
        T tr = 1;
        if (en.c > 0) tr = zs[(en.c - 1) * NPM + i];
        t = cmk<C>(tr, 0);
        if (en.b > 0) t = cmul(t, ys[(en.b - 1) * NPM + i]);
        else if (en.b < 0) t = cmul(t, cconj(ys[(-en.b - 1) * NPM + i]));
        if (en.a > 0) t = cmul(t, xs[(en.a - 1) * NPM + i]);
        else if (en.a < 0) t = cmul(t, cconj(xs[(-en.a - 1) * NPM + i]));
      } else {
        T tr = 1;
        if (en.c < 0) tr = zs[(-en.c - 1) * NPM + i];
        t = cmk<C>(tr, 0);
        if (en.b > 0) t = cmul(t, cconj(ys[(en.b - 1) * NPM + i]));
        else if (en.b < 0) t = cmul(t, ys[(-en.b - 1) * NPM + i]);
        if (en.a > 0) t = cmul(t, cconj(xs[(en.a - 1) * NPM + i]));
        else if (en.a < 0) t = cmul(t, xs[(-en.a - 1) * NPM + i]);
      }
      C& a = acc[((size_t)en.dir * 8 + en.targ) * NPM + i];
      a = cadd(a, cmul(w, t));
    }
  }
  const int* numphys = tb.numphys + (size_t)lg * nl;
  const C* fb = tb.fexpback + tb.fexpback_off[lg];
  const T* rl = tb.rlsc + (size_t)lg * E * nl;
  for (int t = 0; t < 8; ++t) {
    const int tn = it.targets[t];
    if (tn < 0) continue;
    __syncthreads();
    // yphystof of the pair's up (2g) and down (2g+1) waves
    for (int o = lt; o < 2 * 64; o += kXlGroup) {
      const int which = o / 64, j = o - which * 64;
      if (j >= nexptot) continue;
      int l = 0, nftot = 0, nptot = 0, bb = 0;
      while (nftot + tb.numfour[l] <= j) {
        nftot += tb.numfour[l];
        nptot += numphys[l] / 2;
        bb += (tb.numfour[l] - 1) * (numphys[l] / 2);
        ++l;
      }
      const int mm = j - nftot + 1;
      const int na = numphys[l], na2 = na / 2;
      const C* ph = acc + ((size_t)(2 * g + which) * 8 + t) * NPM + nptot;
      C sum = cmk<C>(0, 0);
      if (mm == 1) {
        for (int iv = 0; iv < na2; ++iv) sum.x += T(2) * ph[iv].x;
      } else if (mm & 1) {
        const C* f = fb + bb + ((mm - 3) / 2) * na2;
        for (int iv = 0; iv < na2; ++iv) sum = cadd(sum, cscale(f[iv], T(2) * ph[iv].x));
      } else {
        const int nodd = (tb.numfour[l] - 1) / 2;
        const C* f = fb + bb + nodd * na2 + ((mm - 2) / 2) * na2;
        for (int iv = 0; iv < na2; ++iv) sum = cadd(sum, cmul(f[iv], cmk<C>(0, T(2) * ph[iv].y)));
      }
      mf[(g * 2 + which) * 64 + j] = cscale(sum, T(1) / T(na));
    }
    __syncthreads();
    // yexptolocal
    for (int e = lt; e < E; e += kXlGroup) {
      int nm = 0;
      while (tri(nm + 1, 0) <= e) ++nm;
      const int mth = e - tri(nm, 0);
      const C* fu = mf + (g * 2 + 0) * 64;
      const C* fd = mf + (g * 2 + 1) * 64;
      C v = cmk<C>(0, 0);
      int ntot = 0;
      for (int l = 0; l < nl; ++l) {
        const int mmax = tb.numfour[l] - 1 > nm ? nm : tb.numfour[l] - 1;
        if (mth <= mmax) {
          const C pm = (nm & 1) ? csub(fd[ntot + mth], fu[ntot + mth]) : cadd(fd[ntot + mth], fu[ntot + mth]);
          v = cadd(v, cscale(pm, rl[(size_t)e * nl + l] * tb.weights[l]));
        }
        ntot += tb.numfour[l];
      }
      const T rs = T(3.14159265358979323846) / (tb.betascal[lg] * T(2)) * tb.sfac[e];
      v = cscale(v, rs);
      switch (mth & 3) {  // * i^m
        case 1: v = cmk<C>(-v.y, v.x); break;
        case 2: v = cmk<C>(-v.x, -v.y); break;
        case 3: v = cmk<C>(v.y, -v.x); break;
        default: break;
      }
      loc[g * E + e] = v;
    }
    __syncthreads();
    // rotate back
    for (int e = lt; e < E; e += kXlGroup) {
      if (g == 0) {
        out[e] = loc[e];
        continue;
      }
      int l = 0;
      while (tri(l + 1, 0) <= e) ++l;
      const int m = e - tri(l, 0);
      if (g == 1) {  // rotate_ytoz(rdpi2): rotate then * i^m
        C v = rotate_one<T>(tb, loc + E, tb.R(ROT_PI2), l, m);
        switch (m & 3) {
          case 1: v = cmk<C>(-v.y, v.x); break;
          case 2: v = cmk<C>(-v.x, -v.y); break;
          case 3: v = cmk<C>(v.y, -v.x); break;
          default: break;
        }
        out[E + e] = v;
      } else {  // rotate_ztox(rdmpi2)
        out[2 * E + e] = rotate_one<T>(tb, loc + 2 * E, tb.R(ROT_MPI2), l, m);
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < E; e += blockDim.x)
      L[((size_t)tn * kCh + ch) * E + e] = cadd(cadd(out[e], out[E + e]), out[2 * E + e]);
  }
}

// ---------------------------------------------------------------- L2P
// evaluate_local_expansion_at_xyz computes, per target point, q(n,m) =
// i_n P_n^m e^{im phi}, its gradient gq and Hessian g2q through the ladder
// relations of grad_q / grad2_q (src/fmm/fmm.h:128-415), and contracts them
// with the local coefficients.  Every quantity FMM_results_to_BEM needs is
// linear in q, so the ladders are transposed onto the coefficients once per
// leaf (l2p_prep_kernel): per screening group one expansion F for f and three
// H_j for h, and a target only evaluates q and four dot products per group
// (l2p_eval_kernel).  Same mathematics, summed in a different order.
struct LeafItem {
  int node, level, start, count;
  int leaf;  // index of the leaf's derivative expansions (eval chunks of a leaf share it)
  double c[3];
};

// One term of a ladder output: coef * S(a, b) or coef * conj(S(a, b)).
template <typename T>
struct LTerm {
  int a, b;
  T re, im;
  bool conj;
};

// Terms of component d of the ladder at output (n, m) (grad_q, src/fmm/fmm.h:128-208).
template <typename T>
__device__ int ladder_terms(int n, int m, int d, T sc, T isc, T beta, LTerm<T> out[4]) {
  // l0, l1, l2, r0, r1, r2 as (scale, a, b, conj, valid)
  struct P {
    T s;
    int a, b;
    bool c, v;
  } l[3] = {{0, 0, 0, false, false}, {0, 0, 0, false, false}, {0, 0, 0, false, false}},
    r[3] = {{0, 0, 0, false, false}, {0, 0, 0, false, false}, {0, 0, 0, false, false}};
  if (n == 0 && m == 0) {
    r[0] = {-sc, 1, 1, true, true};
    r[1] = {-sc, 1, 0, false, true};
    r[2] = {sc, 1, 1, false, true};
  } else if (n == 1 && m == 0) {
    l[1] = {isc, 0, 0, false, true};
    r[0] = {-sc, 2, 1, true, true};
    r[1] = {-T(2) * sc, 2, 0, false, true};
    r[2] = {sc, 2, 1, false, true};
  } else if (m == 0) {
    l[0] = {-isc, n - 1, 1, true, true};
    l[1] = {T(n) * isc, n - 1, 0, false, true};
    l[2] = {isc, n - 1, 1, false, true};
    r[0] = {-sc, n + 1, 1, true, true};
    r[1] = {-T(n + 1) * sc, n + 1, 0, false, true};
    r[2] = {sc, n + 1, 1, false, true};
  } else if (n == 1 && m == 1) {
    l[0] = {T(2) * isc, 0, 0, false, true};
    r[0] = {T(2) * sc, 2, 0, false, true};
    r[1] = {-sc, 2, 1, false, true};
    r[2] = {sc, 2, 2, false, true};
  } else if (m == n) {
    l[0] = {T((n + n - 1) * (n + n)) * isc, n - 1, n - 1, false, true};
    r[0] = {T(2) * sc, n + 1, n - 1, false, true};
    r[1] = {-sc, n + 1, n, false, true};
    r[2] = {sc, n + 1, n + 1, false, true};
  } else if (m == n - 1) {
    l[0] = {T((n + m - 1) * (n + m)) * isc, n - 1, n - 2, false, true};
    l[1] = {T(n + m) * isc, n - 1, n - 1, false, true};
    r[0] = {T(6) * sc, n + 1, m - 1, false, true};
    r[1] = {-T(2) * sc, n + 1, m, false, true};
    r[2] = {sc, n + 1, m + 1, false, true};
  } else {
    l[0] = {T((n + m - 1) * (n + m)) * isc, n - 1, m - 1, false, true};
    l[1] = {T(n + m) * isc, n - 1, m, false, true};
    l[2] = {isc, n - 1, m + 1, false, true};
    r[0] = {T((n - m + 1) * (n - m + 2)) * sc, n + 1, m - 1, false, true};
    r[1] = {-T(n - m + 1) * sc, n + 1, m, false, true};
    r[2] = {sc, n + 1, m + 1, false, true};
  }
  const T pb = T(-0.5) / T(2 * n + 1) * beta;
  int k = 0;
  auto add = [&](const P& p, T fr, T fi) {
    if (!p.v) return;
    out[k++] = {p.a, p.b, p.s * fr, p.s * fi, p.c};
  };
  if (d == 0) {  // pb ((l0 - r0) - (l2 - r2))
    add(l[0], pb, 0);
    add(r[0], -pb, 0);
    add(l[2], -pb, 0);
    add(r[2], pb, 0);
  } else if (d == 1) {  // i pb ((l0 - r0) + (l2 - r2))
    add(l[0], 0, pb);
    add(r[0], 0, -pb);
    add(l[2], 0, pb);
    add(r[2], 0, -pb);
  } else {  // -2 pb (l1 - r1)
    add(l[1], -T(2) * pb, 0);
    add(r[1], T(2) * pb, 0);
  }
  return k;
}

// D += adjoint of ladder component d applied to W (outputs n <= nin):
// sum_{n,m} Re[ladder_d(S)(n,m) W(n,m)] = sum Re[S(a,b) D(a,b)].
// Sequential scatter by the calling thread (deterministic).
template <typename T>
__device__ void adjoint_ladder(const typename C2T<T>::type* W, int nin, int d, T sc, T isc, T beta,
                               typename C2T<T>::type* D) {
  using C = typename C2T<T>::type;
  LTerm<T> t[4];
  for (int n = 0; n <= nin; ++n)
    for (int m = 0; m <= n; ++m) {
      const C w = W[tri(n, m)];
      const int k = ladder_terms<T>(n, m, d, sc, isc, beta, t);
      for (int j = 0; j < k; ++j) {
        // kappa * w, conjugated for conj terms
        const T re = t[j].re * w.x - t[j].im * w.y;
        const T im = t[j].re * w.y + t[j].im * w.x;
        C& dst = D[tri(t[j].a, t[j].b)];
        dst.x += re;
        dst.y += t[j].conj ? -im : im;
      }
    }
}

// Per leaf and screening group g: F = A_x[V_a] + A_y[V_a+1] + A_z[V_a+2] + V_a+3
// and H_j = 1/2 sum_k (A_k[A_j[V_b+k]] + A_j[A_k[V_b+k]]) + A_j[V_last], with
// V_c = w_m L_c (w_0 = 1, w_m>0 = 2), all scaled by sign_g * 2 beta_g / pi.
// Output [leaf][g][4][EQ]: F then H_0, H_1, H_2.
template <typename T>
__global__ void __launch_bounds__(64) l2p_prep_kernel(const __grid_constant__ Tables<T> tb,
                                                      const LeafItem* __restrict__ items,
                                                      const typename C2T<T>::type* __restrict__ L,
                                                      typename C2T<T>::type* __restrict__ D) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int NT = tb.nt, E = tb.E;
  const int EQ = (NT + 3) * (NT + 4) / 2;
  const LeafItem it = items[blockIdx.x];
  // per group: V (6 channels used: a..a+3 for f, b..b+2 and last for h) [8][EQ],
  // first level buffers F-part [3][EQ] and U[3][3][EQ], result [4][EQ]
  C* base = reinterpret_cast<C*>(smem_raw);
  const int per_group = (8 + 3 + 9 + 4) * EQ;
  for (int o = threadIdx.x; o < 2 * per_group; o += blockDim.x) base[o] = cmk<C>(0, 0);
  __syncthreads();
  for (int o = threadIdx.x; o < 2 * 8 * E; o += blockDim.x) {
    const int g = o / (8 * E), rem = o - g * 8 * E, slot = rem / E, e = rem - slot * E;
    // slots: 0..3 -> f channels, 4..6 -> h channels, 7 -> last
    const int ch = g == 0 ? (slot < 4 ? slot : (slot < 7 ? 4 + (slot - 4) : 7))
                          : (slot < 4 ? 8 + slot : (slot < 7 ? 8 + (slot - 4) : 11));
    int n = 0;
    while (tri(n + 1, 0) <= e) ++n;
    const int m = e - tri(n, 0);
    const C v = L[((size_t)it.node * kCh + ch) * E + e];
    base[(size_t)g * per_group + slot * EQ + e] = cscale(v, m ? T(2) : T(1));
  }
  __syncthreads();
  // first level: 3 F parts + 9 U per group = 24 passes
  if (threadIdx.x < 24) {
    const int g = threadIdx.x / 12, p = threadIdx.x % 12;
    C* G = base + (size_t)g * per_group;
    const int lg = 2 * it.level + g;
    const T beta = tb.beta[g], sc = tb.scale[lg], isc = T(1) / sc;
    if (p < 3) {
      adjoint_ladder<T>(G + p * EQ, NT, p, sc, isc, beta, G + (8 + p) * EQ);
    } else {
      const int j = (p - 3) / 3, k = (p - 3) % 3;  // U_{j,k} = A_j[V_{b+k}]
      adjoint_ladder<T>(G + (4 + k) * EQ, NT, j, sc, isc, beta, G + (11 + 3 * j + k) * EQ);
    }
  }
  __syncthreads();
  // second level: F sum (1 thread) and H_j (3 threads) per group
  if (threadIdx.x < 8) {
    const int g = threadIdx.x / 4, p = threadIdx.x % 4;
    C* G = base + (size_t)g * per_group;
    C* R = G + 20 * EQ;
    const int lg = 2 * it.level + g;
    const T beta = tb.beta[g], sc = tb.scale[lg], isc = T(1) / sc;
    if (p == 0) {
      for (int e = 0; e < EQ; ++e) {
        C v = cadd(cadd(G[8 * EQ + e], G[9 * EQ + e]), G[10 * EQ + e]);
        if (e < E) v = cadd(v, G[3 * EQ + e]);
        R[e] = v;
      }
    } else {
      const int j = p - 1;
      C* H = R + p * EQ;
      // A_k[U_{j,k}] and A_j[U_{k,k}] at weight 1/2 each: accumulate into H
      // with a scratch buffer of the same size
      for (int k = 0; k < 3; ++k) {
        adjoint_ladder<T>(G + (11 + 3 * j + k) * EQ, NT + 1, k, sc * T(1), isc, beta * T(0.5), H);
        adjoint_ladder<T>(G + (11 + 3 * k + k) * EQ, NT + 1, j, sc, isc, beta * T(0.5), H);
      }
      adjoint_ladder<T>(G + 7 * EQ, NT, j, sc, isc, beta, H);
    }
  }
  __syncthreads();
  // scale by sign_g * 2 beta_g / pi and store
  for (int o = threadIdx.x; o < 2 * 4 * EQ; o += blockDim.x) {
    const int g = o / (4 * EQ), rem = o - g * 4 * EQ;
    const T f = (g ? T(-1) : T(1)) * tb.beta[g] * T(0.63661977236758134308);
    D[((size_t)blockIdx.x * 2 + g) * 4 * EQ + rem] = cscale(base[(size_t)g * per_group + 20 * EQ + rem], f);
  }
}

// One thread per target patch: q(n, m) generated on the fly (Bessel,
// Legendre recurrence in n for each m, e^{i m phi}) and contracted with the
// leaf's F and H_j; y_f += f / 4 pi, y_h += n . h / 4 pi.
constexpr int kEvalChunk = 64;  // targets per l2p_eval block

template <typename T>
__global__ void __launch_bounds__(kEvalChunk) l2p_eval_kernel(const __grid_constant__ Tables<T> tb,
                                                       const LeafItem* __restrict__ items,
                                                       const int32_t* __restrict__ contents,
                                                       const double* __restrict__ centroid,
                                                       const double* __restrict__ normal,
                                                       const typename C2T<T>::type* __restrict__ D, int n,
                                                       double* __restrict__ y) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int NT = tb.nt, N2 = NT + 2;
  const int EQ = (NT + 3) * (NT + 4) / 2;
  C* Ds = reinterpret_cast<C*>(smem_raw);  // [2][4][EQ]
  const LeafItem it = items[blockIdx.x];
  for (int o = threadIdx.x; o < 8 * EQ; o += blockDim.x) Ds[o] = D[(size_t)it.leaf * 8 * EQ + o];
  __syncthreads();
  for (int k = threadIdx.x; k < it.count; k += blockDim.x) {
    const int i = contents[it.start + k];
    const double rx = centroid[3 * i] - it.c[0], ry = centroid[3 * i + 1] - it.c[1], rz = centroid[3 * i + 2] - it.c[2];
    double proj = rx * rx + ry * ry;
    const double rr = proj + rz * rz;
    proj = sqrt(proj);
    const double d = sqrt(rr);
    const double PREC = 2.220446049250313e-16;
    const T x = (T)((d <= PREC) ? 0.0 : rz / d);
    const C e1 = (proj <= PREC * d) ? cmk<C>(1, 0) : cmk<C>((T)(rx / proj), (T)(ry / proj));
    const T u = -sqrt(T(1) - x * x);
    T f = 0, h0 = 0, h1 = 0, h2 = 0;
    T bi[kMaxNT + 4];
    for (int g = 0; g < 2; ++g) {
      const int lg = 2 * it.level + g;
      bessel_in_dev<T>(tb.scale[lg], (T)(d * (double)tb.beta[g]), N2, bi);
      const C* F = Ds + g * 4 * EQ;
      const C* H0 = F + EQ;
      const C* H1 = F + 2 * EQ;
      const C* H2 = F + 3 * EQ;
      C em = cmk<C>(1, 0);  // e^{i m phi}
      T pmm = 1;            // P_m^m
      for (int m = 0; m <= N2; ++m) {
        if (m > 0) {
          pmm = pmm * u * T(2 * m - 1);
          em = cmul(em, e1);
        }
        T p0 = 0, p1 = pmm;  // P_{n-1}^m, P_n^m at n = m
        for (int nn = m; nn <= N2; ++nn) {
          T pn;
          if (nn == m) {
            pn = pmm;
          } else if (nn == m + 1) {
            pn = T(2 * m + 1) * x * pmm;
          } else {
            pn = ((T(2) * nn - T(1)) * x * p1 - T(nn + m - 1) * p0) / T(nn - m);
          }
          if (nn > m) {
            p0 = p1;
            p1 = pn;
          }
          const T amp = (nn == 0) ? bi[0] : bi[nn] * pn;
          const C q = cscale(em, amp);
          const int e = tri(nn, m);
          if (nn <= NT + 1) f += q.x * F[e].x - q.y * F[e].y;
          h0 += q.x * H0[e].x - q.y * H0[e].y;
          h1 += q.x * H1[e].x - q.y * H1[e].y;
          h2 += q.x * H2[e].x - q.y * H2[e].y;
        }
      }
    }
    const double k4 = 0.07957747154594767;
    const double h = normal[3 * i] * (double)h0 + normal[3 * i + 1] * (double)h1 + normal[3 * i + 2] * (double)h2;
    y[i] = (double)f * k4;  // far-field buffer: every patch is in exactly one leaf
    y[n + i] = h * k4;
  }
}

template <typename C, typename S>
void to_dev_c(std::vector<C>& out, const std::vector<S>& in) {
  out.resize(in.size());
  for (size_t k = 0; k < in.size(); ++k) {
    out[k].x = (decltype(out[k].x))in[k].real();
    out[k].y = (decltype(out[k].x))in[k].imag();
  }
}

}  // namespace

// ---------------------------------------------------------------- host state
// ---------------------------------------------------------------- operator form
// The M2M and L2L shifts of one channel are R-linear maps of the 2E reals of
// an expansion, fixed per (level, screening group, child octant); the L2P
// preparation is an R-linear map from the 12 x 2E reals of a leaf's locals to
// its 8 x 2EQ derivative-expansion reals, fixed per (level).  They are
// tabulated once per problem by applying the kernels above to unit vectors
// (same arithmetic, so the same operators), then applied as dense (shifts)
// or sparse (preparation) matrix-vector products: no shared-memory phases
// and no serial chains per output.
template <typename T>
__global__ void __launch_bounds__(64) shift_basis_kernel(const __grid_constant__ Tables<T> tb, int nlev,
                                                         T* __restrict__ ops) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E, R = 2 * E;
  C* w1 = reinterpret_cast<C*>(smem_raw);
  C* w2 = w1 + E;
  C* acc = w2 + E;
  C* in = acc + E;
  const int k = blockIdx.x % R;
  const int op = blockIdx.x / R;  // ((kind * nlev + level) * 2 + group) * 8 + octant-1
  const int oct = op % 8 + 1, g = (op / 8) % 2, level = (op / 16) % nlev, kind = op / (16 * nlev);
  for (int o = threadIdx.x; o < E; o += blockDim.x) {
    in[o] = cmk<C>(2 * o == k ? T(1) : T(0), 2 * o + 1 == k ? T(1) : T(0));
    acc[o] = cmk<C>(0, 0);
  }
  __syncthreads();
  const bool multipole = kind == 0;
  const T* rd = multipole ? tb.R(oct > 4 ? ROT_MSQ3 : ROT_SQ3) : tb.R(oct > 4 ? ROT_SQ3 : ROT_MSQ3);
  shift_block<T>(tb, oct, multipole, level, in, w1, w2, acc, rd, g ? 8 : 0, 1);
  T* col = ops + ((size_t)op * R + k) * R;  // column k: [op][k][r]
  for (int o = threadIdx.x; o < E; o += blockDim.x) {
    col[2 * o] = acc[o].x;
    col[2 * o + 1] = acc[o].y;
  }
}

struct DenseShift {
  int target, first_src, n_src;  // sources listed in DenseSrc
};
struct DenseSrc {
  int node, op;  // source expansion node and operator index
};

// y[target][ch] (=, or += for L2L) sum over sources of A_op x[source][ch];
// one block per (target, channel), thread per output real
template <typename T>
__global__ void __launch_bounds__(128) dense_shift_kernel(int E, const DenseShift* __restrict__ items,
                                                          const DenseSrc* __restrict__ srcs,
                                                          const T* __restrict__ ops, const T* __restrict__ X,
                                                          T* __restrict__ Y, int accumulate) {
  extern __shared__ unsigned char smem_raw[];
  const int R = 2 * E;
  T* xs = reinterpret_cast<T*>(smem_raw);  // [8][R]
  const DenseShift it = items[blockIdx.x / kCh];
  const int ch = blockIdx.x % kCh;
  for (int o = threadIdx.x; o < it.n_src * R; o += blockDim.x) {
    const DenseSrc sc = srcs[it.first_src + o / R];
    xs[o] = X[((size_t)sc.node * kCh + ch) * R + o % R];
  }
  __syncthreads();
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    T acc = accumulate ? Y[((size_t)it.target * kCh + ch) * R + r] : T(0);
    for (int c = 0; c < it.n_src; ++c) {
      const T* A = ops + (size_t)(srcs[it.first_src + c].op + (ch >= 8 ? 8 : 0)) * R * R;  // group offset
      const T* x = xs + c * R;
      for (int k = 0; k < R; ++k) acc += A[(size_t)k * R + r] * x[k];
    }
    Y[((size_t)it.target * kCh + ch) * R + r] = acc;
  }
}

// Unit-vector inputs for tabulating the L2P preparation: item b of level l
// has local expansions zero except real component k of channel c
// (b = c * 2E + k).
template <typename T>
__global__ void prep_basis_inputs(int E, int nb, typename C2T<T>::type* __restrict__ Lb) {
  const int b = blockIdx.x;
  const int R = 2 * E;
  const int c = b / R, k = b % R;
  for (int o = threadIdx.x; o < kCh * E; o += blockDim.x) {
    const int ch = o / E, e = o % E;
    T re = (ch == c && 2 * e == k) ? T(1) : T(0);
    T im = (ch == c && 2 * e + 1 == k) ? T(1) : T(0);
    Lb[(size_t)b * kCh * E + o] = cmk<typename C2T<T>::type>(re, im);
  }
  (void)nb;
}

// D[leaf][row] = sum over the row's nonzeros of val * Lreal[leaf][col]
template <typename T>
__global__ void __launch_bounds__(256) prep_csr_kernel(int E, int EQ, const LeafItem* __restrict__ items,
                                                       const int* __restrict__ rowptr, const int* __restrict__ cols,
                                                       const T* __restrict__ vals, const T* __restrict__ Lr,
                                                       T* __restrict__ D) {
  extern __shared__ unsigned char smem_raw[];
  const int R = 2 * E, rows = 8 * 2 * EQ;
  T* x = reinterpret_cast<T*>(smem_raw);  // [12 * R]
  const LeafItem it = items[blockIdx.x];
  for (int o = threadIdx.x; o < kCh * R; o += blockDim.x) x[o] = Lr[(size_t)it.node * kCh * R + o];
  __syncthreads();
  const int* rp = rowptr + (size_t)it.level * (rows + 1);
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    T acc = 0;
    for (int z = rp[r]; z < rp[r + 1]; ++z) acc += vals[z] * x[cols[z]];
    D[(size_t)blockIdx.x * rows + r] = acc;
  }
}

struct FmmState {
  int nt = 9, E = 55, nlev = 0, np_max = 0, nl = 0;
  bool fp64 = true;
  DevBuf tables_buf;  // one allocation holding every table
  Tables<double> tb_d{};
  Tables<float> tb_f{};
  DevBuf M, L, W;  // expansions and plane waves
  DevBuf p2m_items, m2x_items, xl_items, xl_entries, leaf_items, m2m_items, m2m_children, l2l_items, l2l_children;
  int n_p2m = 0, n_m2x = 0, n_xl = 0, n_leaf = 0;
  std::vector<int> m2m_first, m2m_count;  // per child level
  std::vector<int> l2l_first, l2l_count;  // per parent level
  size_t smem_p2m = 0, smem_shift = 0, smem_m2x = 0, smem_xl = 0, smem_prep = 0, smem_eval = 0;
  DevBuf leaf_exp;  // per leaf: [2 groups][F, H0, H1, H2][EQ]
  DevBuf eval_items;
  int n_eval = 0;
  // operator form of M2M / L2L and of the L2P preparation
  DevBuf shift_ops;                       // [op][k][r], op = ((kind*nlev + level)*2 + group)*8 + octant-1
  DevBuf m2m_dense, m2m_src, l2l_dense, l2l_src;
  std::vector<int> m2m_dfirst, m2m_dcount, l2l_dfirst, l2l_dcount;
  DevBuf prep_rowptr, prep_cols, prep_vals;
  size_t smem_dense = 0, smem_csr = 0;
  bool use_operators = true;
};

void fmm_destroy(FmmState* s) { delete s; }

bool fmm_active(const Problem& P) { return P.tree.n_levels - 1 >= 2; }

namespace {

// Generates the 1512 interaction entries (src/fmm/interaction_list.h):
// source = child of a non-self neighbour of the parent, target = child of
// the parent, separated by >= 2 child boxes along some axis; the direction
// is UP/DOWN by dz, else NORTH/SOUTH by dy, else EAST/WEST by dx.
struct RawInteraction {
  int nb, dir, targ, src, dx, dy, dz;
};
std::vector<RawInteraction> interaction_table() {
  std::vector<RawInteraction> out;
  for (int nb = 0; nb < 27; ++nb) {
    if (nb == 13) continue;
    const int pz = nb / 9 - 1, py = (nb % 9) / 3 - 1, px = nb % 3 - 1;
    for (int t = 0; t < 8; ++t) {
      const int tx = t & 1, ty = (t >> 1) & 1, tz = t >> 2;
      for (int s = 0; s < 8; ++s) {
        const int sx = 2 * px + (s & 1), sy = 2 * py + ((s >> 1) & 1), sz = 2 * pz + (s >> 2);
        const int dx = tx - sx, dy = ty - sy, dz = tz - sz;
        if (std::abs(dx) < 2 && std::abs(dy) < 2 && std::abs(dz) < 2) continue;
        int dir;
        if (dz >= 2) dir = 0;
        else if (dz <= -2) dir = 1;
        else if (dy >= 2) dir = 2;
        else if (dy <= -2) dir = 3;
        else if (dx >= 2) dir = 4;
        else dir = 5;
        out.push_back({nb, dir, t, s, dx, dy, dz});
      }
    }
  }
  return out;
}

template <typename T>
void fill_tables(FmmState& S, const Problem& P, Tables<T>& tb) {
  using C = typename C2T<T>::type;
  const int nt = S.nt, E = S.E, nlev = S.nlev;
  GlobalTables G;
  G.build(nt);
  std::vector<LevelTables> LT(2 * nlev);
  const double beta = std::max(P.params.kappa, P.params.beta0);
  for (int l = 0; l < nlev; ++l) {
    LT[2 * l].build(nt, beta, l, P.params.cube_edge);
    LT[2 * l + 1].build(nt, P.params.beta0, l, P.params.cube_edge);
  }
  S.nl = LT[0].nl;
  int npm = 0;
  for (auto& t : LT) npm = std::max(npm, t.nexptotp);
  S.np_max = npm;
  // pack everything into one byte buffer with aligned sub-arrays
  std::vector<unsigned char> blob;
  auto put = [&](const void* src, size_t bytes) -> size_t {
    size_t off = (blob.size() + 255) & ~size_t(255);
    blob.resize(off + bytes);
    if (bytes) std::memcpy(blob.data() + off, src, bytes);
    return off;
  };
  auto putT = [&](const std::vector<double>& v) {
    std::vector<T> t(v.begin(), v.end());
    return put(t.data(), t.size() * sizeof(T));
  };
  auto putC = [&](const std::vector<cplx>& v) {
    std::vector<C> t;
    to_dev_c(t, v);
    return put(t.data(), t.size() * sizeof(C));
  };
  auto putI = [&](const std::vector<int>& v) { return put(v.data(), v.size() * sizeof(int)); };
  std::vector<double> rot;
  for (auto* r : {&G.rdpi2, &G.rdmpi2, &G.rdsq3, &G.rdmsq3}) rot.insert(rot.end(), r->begin(), r->end());
  size_t o_rot = putT(rot), o_sfac = putT(G.scale_factors), o_w = putT(LT[0].weights), o_nf = putI(LT[0].numfour);
  std::vector<int> numphys, nexptot, nexptotp, fe_off, fo_off, fb_off;
  std::vector<double> scale, betascal, rlsc, zs, mps, lcs;
  std::vector<cplx> fexpe, fexpo, fexpback, xs, ys;
  for (auto& t : LT) {
    numphys.insert(numphys.end(), t.numphys.begin(), t.numphys.end());
    nexptot.push_back(t.nexptot);
    nexptotp.push_back(t.nexptotp);
    scale.push_back(t.scale);
    betascal.push_back(t.betascal);
    rlsc.insert(rlsc.end(), t.rlsc.begin(), t.rlsc.end());
    fe_off.push_back((int)fexpe.size());
    fexpe.insert(fexpe.end(), t.fexpe.begin(), t.fexpe.end());
    fo_off.push_back((int)fexpo.size());
    fexpo.insert(fexpo.end(), t.fexpo.begin(), t.fexpo.end());
    fb_off.push_back((int)fexpback.size());
    fexpback.insert(fexpback.end(), t.fexpback.begin(), t.fexpback.end());
    for (int k = 0; k < 3; ++k) {
      for (int i = 0; i < npm; ++i) {
        const bool ok = i < t.nexptotp;
        xs.push_back(ok ? t.xs[(size_t)k * t.nexptotp + i] : cplx(0));
        ys.push_back(ok ? t.ys[(size_t)k * t.nexptotp + i] : cplx(0));
        zs.push_back(ok ? t.zs[(size_t)k * t.nexptotp + i] : 0.0);
      }
    }
    mps.insert(mps.end(), t.mpshift.begin(), t.mpshift.end());
    lcs.insert(lcs.end(), t.lcshift.begin(), t.lcshift.end());
  }
  if (fexpe.empty()) fexpe.push_back(0);
  if (fexpo.empty()) fexpo.push_back(0);
  size_t o_np = putI(numphys), o_ne = putI(nexptot), o_nep = putI(nexptotp), o_sc = putT(scale),
         o_bs = putT(betascal), o_beta = putT(std::vector<double>{beta, P.params.beta0}), o_rl = putT(rlsc),
         o_fe = putC(fexpe), o_fo = putC(fexpo), o_fb = putC(fexpback), o_feo = putI(fe_off), o_foo = putI(fo_off),
         o_fbo = putI(fb_off), o_xs = putC(xs), o_ys = putC(ys), o_zs = putT(zs), o_mps = putT(mps),
         o_lcs = putT(lcs);
  S.tables_buf.alloc(P.ctx, blob.size());
  BP_CUDA(cudaMemcpyAsync(S.tables_buf.get(), blob.data(), blob.size(), cudaMemcpyHostToDevice, P.ctx->stream));
  BP_CUDA(cudaStreamSynchronize(P.ctx->stream));
  unsigned char* base = S.tables_buf.as<unsigned char>();
  tb.nt = nt;
  tb.E = E;
  tb.nl = S.nl;
  tb.np_max = npm;
  tb.nlev = nlev;
  tb.rot = reinterpret_cast<const T*>(base + o_rot);
  tb.sfac = reinterpret_cast<const T*>(base + o_sfac);
  tb.weights = reinterpret_cast<const T*>(base + o_w);
  tb.numfour = reinterpret_cast<const int*>(base + o_nf);
  tb.numphys = reinterpret_cast<const int*>(base + o_np);
  tb.nexptot = reinterpret_cast<const int*>(base + o_ne);
  tb.nexptotp = reinterpret_cast<const int*>(base + o_nep);
  tb.scale = reinterpret_cast<const T*>(base + o_sc);
  tb.betascal = reinterpret_cast<const T*>(base + o_bs);
  tb.beta = reinterpret_cast<const T*>(base + o_beta);
  tb.rlsc = reinterpret_cast<const T*>(base + o_rl);
  tb.fexpe = reinterpret_cast<const C*>(base + o_fe);
  tb.fexpo = reinterpret_cast<const C*>(base + o_fo);
  tb.fexpback = reinterpret_cast<const C*>(base + o_fb);
  tb.fexpe_off = reinterpret_cast<const int*>(base + o_feo);
  tb.fexpo_off = reinterpret_cast<const int*>(base + o_foo);
  tb.fexpback_off = reinterpret_cast<const int*>(base + o_fbo);
  tb.xs = reinterpret_cast<const C*>(base + o_xs);
  tb.ys = reinterpret_cast<const C*>(base + o_ys);
  tb.zs = reinterpret_cast<const T*>(base + o_zs);
  tb.mpshift = reinterpret_cast<const T*>(base + o_mps);
  tb.lcshift = reinterpret_cast<const T*>(base + o_lcs);
  for (auto& t : LT)
    if (t.nexptot > 64) throw std::invalid_argument("FMM order with more than 64 Fourier modes is not supported");
}

}  // namespace


template <typename T>
static void build_operators(Problem& P, FmmState& S, const Tables<T>& tb, const std::vector<ShiftItem>& m2m,
                            const std::vector<ShiftChild>& m2m_ch, const std::vector<ShiftItem>& l2l,
                            const std::vector<ShiftChild>& l2l_ch, const std::vector<LeafItem>& leaves) {
  using C = typename C2T<T>::type;
  Ctx* c = P.ctx;
  cudaStream_t st = c->stream;
  const int E = S.E, R = 2 * E, nlev = S.nlev, NT = S.nt;
  const int EQ = (NT + 3) * (NT + 4) / 2;
  // shifts: kind 0 = M2M (level = child level), kind 1 = L2L (level = parent level)
  const int n_ops = 2 * nlev * 2 * 8;
  S.shift_ops.alloc(c, sizeof(T) * (size_t)n_ops * R * R);
  shift_basis_kernel<T><<<n_ops * R, 64, S.smem_shift, st>>>(tb, nlev, S.shift_ops.as<T>());
  BP_LAUNCH_CHECK();
  auto op_base = [&](int kind, int level, int oct) { return ((kind * nlev + level) * 2) * 8 + oct - 1; };
  std::vector<DenseShift> md, ld;
  std::vector<DenseSrc> ms, ls;
  S.m2m_dfirst.assign(nlev, 0);
  S.m2m_dcount.assign(nlev, 0);
  for (int lev = nlev - 1; lev >= 1; --lev) {
    S.m2m_dfirst[lev] = (int)md.size();
    for (int q = S.m2m_first[lev]; q < S.m2m_first[lev] + S.m2m_count[lev]; ++q) {
      const ShiftItem& it = m2m[q];
      DenseShift d{it.parent, (int)ms.size(), it.n_children};
      for (int k = 0; k < it.n_children; ++k) {
        const ShiftChild& ch = m2m_ch[it.first_child + k];
        ms.push_back({ch.node, op_base(0, lev, ch.octant)});
      }
      md.push_back(d);
    }
    S.m2m_dcount[lev] = (int)md.size() - S.m2m_dfirst[lev];
  }
  S.l2l_dfirst.assign(nlev, 0);
  S.l2l_dcount.assign(nlev, 0);
  for (int lev = 0; lev < nlev - 1; ++lev) {
    S.l2l_dfirst[lev] = (int)ld.size();
    for (int q = S.l2l_first[lev]; q < S.l2l_first[lev] + S.l2l_count[lev]; ++q) {
      const ShiftItem& it = l2l[q];
      const ShiftChild& ch = l2l_ch[it.first_child];
      ld.push_back({ch.node, (int)ls.size(), 1});
      ls.push_back({it.parent, op_base(1, lev, ch.octant)});
    }
    S.l2l_dcount[lev] = (int)ld.size() - S.l2l_dfirst[lev];
  }
  S.m2m_dense = upload(c, md);
  S.m2m_src = upload(c, ms);
  S.l2l_dense = upload(c, ld);
  S.l2l_src = upload(c, ls);
  S.smem_dense = sizeof(T) * 8 * (size_t)R;
  // L2P preparation operator per level that holds leaves
  const int nb = kCh * R, rows = 8 * 2 * EQ;
  std::vector<int> levels_with_leaves(nlev, 0);
  for (const LeafItem& lf : leaves) levels_with_leaves[lf.level] = 1;
  DevBuf Lb(c, sizeof(C) * (size_t)nb * kCh * E);
  DevBuf Db(c, sizeof(C) * (size_t)nb * 8 * EQ);
  prep_basis_inputs<T><<<nb, 128, 0, st>>>(E, nb, Lb.as<C>());
  BP_LAUNCH_CHECK();
  std::vector<int> rowptr((size_t)nlev * (rows + 1), 0), cols;
  std::vector<T> vals;
  std::vector<T> host((size_t)nb * rows);
  for (int lev = 0; lev < nlev; ++lev) {
    int* rp = rowptr.data() + (size_t)lev * (rows + 1);
    if (!levels_with_leaves[lev]) {
      for (int r = 0; r <= rows; ++r) rp[r] = (int)vals.size();
      continue;
    }
    std::vector<LeafItem> bi(nb);
    for (int b = 0; b < nb; ++b) bi[b] = LeafItem{b, lev, 0, 0, b, {0, 0, 0}};
    DevBuf d_bi = upload(c, bi);
    l2p_prep_kernel<T><<<nb, 64, S.smem_prep, st>>>(tb, d_bi.as<LeafItem>(), Lb.as<C>(), Db.as<C>());
    BP_LAUNCH_CHECK();
    BP_CUDA(cudaMemcpyAsync(host.data(), Db.get(), sizeof(T) * host.size(), cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    for (int r = 0; r < rows; ++r) {
      rp[r] = (int)vals.size();
      for (int b = 0; b < nb; ++b) {
        const T v = host[(size_t)b * rows + r];
        if (v != T(0)) {
          cols.push_back(b);
          vals.push_back(v);
        }
      }
    }
    rp[rows] = (int)vals.size();
  }
  if (vals.empty()) {
    vals.push_back(0);
    cols.push_back(0);
  }
  S.prep_rowptr = upload(c, rowptr);
  S.prep_cols = upload(c, cols);
  S.prep_vals = upload(c, vals);
  S.smem_csr = sizeof(T) * (size_t)kCh * R;
  BP_CUDA(cudaStreamSynchronize(st));
}

void fmm_setup(Problem& P) {
  auto S = new FmmState();
  P.fmm.reset(S);
  const TreeInfo& T = P.tree;
  S->nt = P.params.nterms;
  S->E = (S->nt + 1) * (S->nt + 2) / 2;
  S->nlev = T.n_levels;
  S->fp64 = P.fp64;
  if (S->fp64)
    fill_tables<double>(*S, P, S->tb_d);
  else
    fill_tables<float>(*S, P, S->tb_f);
  const int nn = (int)T.nodes.size();
  const size_t celem = S->fp64 ? sizeof(double2) : sizeof(float2);
  const size_t exp_bytes = (size_t)nn * kCh * S->E * celem;
  S->M.alloc(P.ctx, exp_bytes);
  S->L.alloc(P.ctx, exp_bytes);
  BP_CUDA(cudaMemsetAsync(S->L.get(), 0, exp_bytes, P.ctx->stream));
  S->W.alloc(P.ctx, (size_t)nn * 6 * kCh * S->np_max * celem);
  BP_CUDA(cudaMemsetAsync(S->W.get(), 0, S->W.bytes(), P.ctx->stream));
  auto flags = [&](int k) { return T.nodes[k].flags; };
  auto cnt = [&](int k) { return T.nodes[k].content_count; };
  auto octant = [&](int k) { return 1 + (T.nodes[k].ix & 1) + 2 * (T.nodes[k].iy & 1) + 4 * (T.nodes[k].iz & 1); };
  // P2M items
  std::vector<P2mItem> p2m;
  for (int k = 0; k < nn; ++k) {
    if ((flags(k) & TREE_HAS_CHILDREN) || cnt(k) == 0) continue;
    P2mItem it{k, T.nodes[k].level, (int)T.nodes[k].content_start, cnt(k), {0, 0, 0}};
    for (int d = 0; d < 3; ++d) it.c[d] = T.nodes[k].centre[d];
    p2m.push_back(it);
  }
  // M2M per child level: parents with non-empty children
  std::vector<ShiftItem> m2m;
  std::vector<ShiftChild> m2m_ch;
  S->m2m_first.assign(S->nlev, 0);
  S->m2m_count.assign(S->nlev, 0);
  for (int lev = S->nlev - 1; lev >= 1; --lev) {
    S->m2m_first[lev] = (int)m2m.size();
    for (int k = T.level_start[lev - 1]; k < T.level_start[lev]; ++k) {
      if (!(flags(k) & TREE_HAS_CHILDREN) || cnt(k) == 0) continue;
      ShiftItem it{k, (int)m2m_ch.size(), 0};
      for (int c = 0; c < 8; ++c) {
        const int ck = T.nodes[k].children[c];
        if (ck < 0 || cnt(ck) == 0) continue;
        m2m_ch.push_back(ShiftChild{ck, (int)octant(ck)});
        it.n_children++;
      }
      if (it.n_children) m2m.push_back(it);
    }
    S->m2m_count[lev] = (int)m2m.size() - S->m2m_first[lev];
  }
  // M2X items: non-empty nodes below the root
  std::vector<M2xItem> m2x;
  for (int k = 0; k < nn; ++k)
    if (T.nodes[k].level >= 1 && cnt(k) > 0) m2x.push_back({k, T.nodes[k].level});
  // X2L: parents neither leaf nor shadow, levels 0..bottom-1
  const auto table = interaction_table();
  std::vector<XlItem> xl;
  std::vector<XlEntry> xle;
  for (int k = 0; k < nn; ++k) {
    const TreeNode& nd = T.nodes[k];
    if (nd.level >= S->nlev - 1) continue;
    if ((nd.flags & TREE_LEAF) || (nd.flags & TREE_SHADOW)) continue;
    XlItem it;
    it.parent_level = nd.level;
    bool any_target = false;
    for (int c = 0; c < 8; ++c) {
      const int ck = nd.children[c];
      it.targets[c] = (ck >= 0 && !(flags(ck) & TREE_SHADOW)) ? ck : -1;
      any_target |= it.targets[c] >= 0;
    }
    if (!any_target) continue;
    for (int pair = 0; pair < 3; ++pair) {
      it.first_entry[pair] = (int)xle.size();
      for (const RawInteraction& r : table) {
        if (r.dir / 2 != pair) continue;
        if (it.targets[r.targ] < 0) continue;
        const int nbk = nd.neighbours[r.nb];
        if (nbk < 0 || cnt(nbk) == 0) continue;
        const int sk = T.nodes[nbk].children[r.src];
        if (sk < 0 || cnt(sk) == 0) continue;
        XlEntry e;
        e.src = sk;
        e.dir = (signed char)r.dir;
        e.targ = (signed char)r.targ;
        int a, b, c;
        switch (r.dir) {
          case 0: case 1: a = r.dx; b = r.dy; c = r.dz; break;
          case 2: case 3: a = r.dz; b = r.dx; c = r.dy; break;
          default: a = -r.dz; b = r.dy; c = r.dx; break;
        }
        e.a = (signed char)a;
        e.b = (signed char)b;
        e.c = (signed char)c;
        e.up = (r.dir % 2 == 0) ? 1 : 0;
        xle.push_back(e);
      }
      it.n_entries[pair] = (int)xle.size() - it.first_entry[pair];
    }
    xl.push_back(it);
  }
  // L2L per parent level: one item per (parent, child)
  std::vector<ShiftItem> l2l;
  std::vector<ShiftChild> l2l_ch;
  S->l2l_first.assign(S->nlev, 0);
  S->l2l_count.assign(S->nlev, 0);
  for (int lev = 0; lev < S->nlev - 1; ++lev) {
    S->l2l_first[lev] = (int)l2l.size();
    for (int k = T.level_start[lev]; k < T.level_start[lev + 1]; ++k) {
      if (!(flags(k) & TREE_HAS_CHILDREN) || (flags(k) & TREE_LEAF)) continue;
      for (int c = 0; c < 8; ++c) {
        const int ck = T.nodes[k].children[c];
        if (ck < 0 || cnt(ck) == 0 || (flags(ck) & TREE_SHADOW)) continue;
        l2l.push_back({k, (int)l2l_ch.size(), 1});
        l2l_ch.push_back({ck, c + 1});
      }
    }
    S->l2l_count[lev] = (int)l2l.size() - S->l2l_first[lev];
  }
  // leaves
  std::vector<LeafItem> leaves, evals;
  for (int k = 0; k < nn; ++k) {
    if (!(flags(k) & TREE_LEAF) || cnt(k) == 0) continue;
    LeafItem it{k, T.nodes[k].level, (int)T.nodes[k].content_start, cnt(k), (int)leaves.size(), {0, 0, 0}};
    for (int d = 0; d < 3; ++d) it.c[d] = T.nodes[k].centre[d];
    leaves.push_back(it);
    for (int off = 0; off < it.count; off += kEvalChunk) {
      LeafItem ev = it;
      ev.start = it.start + off;
      ev.count = std::min(kEvalChunk, it.count - off);
      evals.push_back(ev);
    }
  }
  Ctx* c = P.ctx;
  S->p2m_items = upload(c, p2m);
  S->n_p2m = (int)p2m.size();
  S->m2m_items = upload(c, m2m);
  S->m2m_children = upload(c, m2m_ch);
  S->m2x_items = upload(c, m2x);
  S->n_m2x = (int)m2x.size();
  S->xl_items = upload(c, xl);
  S->xl_entries = upload(c, xle);
  S->n_xl = (int)xl.size();
  S->l2l_items = upload(c, l2l);
  S->l2l_children = upload(c, l2l_ch);
  S->leaf_items = upload(c, leaves);
  S->n_leaf = (int)leaves.size();
  S->eval_items = upload(c, evals);
  S->n_eval = (int)evals.size();
  // contents on the device (node-major patch lists)
  const int E = S->E, NT = S->nt;
  S->smem_p2m = celem * 2 * kP2mChunk * E + (S->fp64 ? 8 : 4) * kP2mChunk * kCh;
  S->smem_shift = 4 * celem * E;
  S->smem_m2x = celem * (2 * E + 128);
  S->smem_xl = celem * (6 * 8 * (size_t)S->np_max + 3 * 2 * 64 + 6 * E);
  if (S->np_max > kXlGroup) throw std::invalid_argument("FMM order too large for the X2L thread layout");
  const int EQ = (NT + 3) * (NT + 4) / 2, EG = (NT + 2) * (NT + 3) / 2;
  S->smem_prep = celem * 2 * 24 * (size_t)EQ;
  S->smem_eval = celem * 8 * (size_t)EQ;
  S->leaf_exp.alloc(P.ctx, celem * 8 * (size_t)EQ * std::max(1, S->n_leaf));
  (void)EG;
  auto attr = [&](const void* fn, size_t bytes) {
    ensure_dynamic_smem(fn, bytes);
  };
  if (S->fp64) {
    attr((const void*)p2m_kernel<double>, S->smem_p2m);
    attr((const void*)m2m_kernel<double>, S->smem_shift);
    attr((const void*)l2l_kernel<double>, S->smem_shift);
    attr((const void*)m2x_kernel<double>, S->smem_m2x);
    attr((const void*)x2l_kernel<double>, S->smem_xl);
    attr((const void*)l2p_prep_kernel<double>, S->smem_prep);
    attr((const void*)l2p_eval_kernel<double>, S->smem_eval);
  } else {
    attr((const void*)p2m_kernel<float>, S->smem_p2m);
    attr((const void*)m2m_kernel<float>, S->smem_shift);
    attr((const void*)l2l_kernel<float>, S->smem_shift);
    attr((const void*)m2x_kernel<float>, S->smem_m2x);
    attr((const void*)x2l_kernel<float>, S->smem_xl);
    attr((const void*)l2p_prep_kernel<float>, S->smem_prep);
    attr((const void*)l2p_eval_kernel<float>, S->smem_eval);
  }
  if (S->smem_xl > 227 * 1024 || S->smem_prep > 227 * 1024)
    throw std::invalid_argument("FMM order too large for the shared-memory layout");
  // device copy of the tree contents (node-major)
  P.fmm_contents = upload(c, T.contents);
  BP_CUDA(cudaStreamSynchronize(c->stream));
  if (S->fp64)
    build_operators<double>(P, *S, S->tb_d, m2m, m2m_ch, l2l, l2l_ch, leaves);
  else
    build_operators<float>(P, *S, S->tb_f, m2m, m2m_ch, l2l, l2l_ch, leaves);
}

template <typename T>
static void run_fmm(Problem& P, FmmState& S, const Tables<T>& tb, const double* x, double* y, StageTimes* st,
                    cudaStream_t s) {
  using C = typename C2T<T>::type;
  C* M = S.M.as<C>();
  C* Lx = S.L.as<C>();
  C* W = S.W.as<C>();
  const int32_t* contents = P.fmm_contents.as<int32_t>();
  auto begin = [&](int stage) {
    if (st) st->begin(stage, s);
  };
  auto end = [&](int launches) {
    if (st) st->end(launches);
  };
  if (S.n_p2m == 0 || S.n_m2x == 0 || S.n_xl == 0 || S.n_leaf == 0)
    throw std::runtime_error("inconsistent FMM schedule (empty stage)");
  begin(1);
  p2m_kernel<T><<<S.n_p2m, 256, S.smem_p2m, s>>>(tb, S.p2m_items.as<P2mItem>(), contents, P.d_centroid.as<double>(),
                                                 P.d_area.as<double>(), P.d_normal.as<double>(), P.d_eps.as<double>(),
                                                 x, P.n, M);
  BP_LAUNCH_CHECK();
  end(1);
  begin(2);
  int l_m2m = 0;
  for (int lev = S.nlev - 1; lev >= 1; --lev) {
    if (S.use_operators) {
      if (!S.m2m_dcount[lev]) continue;
      dense_shift_kernel<T><<<S.m2m_dcount[lev] * kCh, 128, S.smem_dense, s>>>(
          S.E, S.m2m_dense.as<DenseShift>() + S.m2m_dfirst[lev], S.m2m_src.as<DenseSrc>(), S.shift_ops.as<T>(),
          reinterpret_cast<const T*>(M), reinterpret_cast<T*>(M), 0);
    } else {
      if (!S.m2m_count[lev]) continue;
      m2m_kernel<T><<<S.m2m_count[lev] * kCh, 64, S.smem_shift, s>>>(
          tb, S.m2m_items.as<ShiftItem>() + S.m2m_first[lev], S.m2m_children.as<ShiftChild>(), lev, M);
    }
    BP_LAUNCH_CHECK();
    ++l_m2m;
  }
  end(l_m2m);
  begin(3);
  m2x_kernel<T><<<S.n_m2x * kCh, kM2xThreads, S.smem_m2x, s>>>(tb, S.m2x_items.as<M2xItem>(), M, W);
  BP_LAUNCH_CHECK();
  end(1);
  begin(4);
  x2l_kernel<T><<<S.n_xl * kCh, kXlThreads, S.smem_xl, s>>>(tb, S.xl_items.as<XlItem>(),
                                                                     S.xl_entries.as<XlEntry>(), W, Lx);
  BP_LAUNCH_CHECK();
  end(1);
  begin(6);
  int l_l2l = 0;
  for (int lev = 0; lev < S.nlev - 1; ++lev) {
    if (S.use_operators) {
      if (!S.l2l_dcount[lev]) continue;
      dense_shift_kernel<T><<<S.l2l_dcount[lev] * kCh, 128, S.smem_dense, s>>>(
          S.E, S.l2l_dense.as<DenseShift>() + S.l2l_dfirst[lev], S.l2l_src.as<DenseSrc>(), S.shift_ops.as<T>(),
          reinterpret_cast<const T*>(Lx), reinterpret_cast<T*>(Lx), 1);
    } else {
      if (!S.l2l_count[lev]) continue;
      l2l_kernel<T><<<S.l2l_count[lev] * kCh, 64, S.smem_shift, s>>>(
          tb, S.l2l_items.as<ShiftItem>() + S.l2l_first[lev], S.l2l_children.as<ShiftChild>(), lev, Lx);
    }
    BP_LAUNCH_CHECK();
    ++l_l2l;
  }
  end(l_l2l);
  begin(5);
  if (S.use_operators) {
    const int NT = S.nt, EQ = (NT + 3) * (NT + 4) / 2;
    prep_csr_kernel<T><<<S.n_leaf, 256, S.smem_csr, s>>>(S.E, EQ, S.leaf_items.as<LeafItem>(), S.prep_rowptr.as<int>(),
                                                          S.prep_cols.as<int>(), S.prep_vals.as<T>(),
                                                          reinterpret_cast<const T*>(Lx),
                                                          reinterpret_cast<T*>(S.leaf_exp.as<C>()));
  } else {
    l2p_prep_kernel<T><<<S.n_leaf, 64, S.smem_prep, s>>>(tb, S.leaf_items.as<LeafItem>(), Lx, S.leaf_exp.as<C>());
  }
  BP_LAUNCH_CHECK();
  end(1);
  begin(7);
  l2p_eval_kernel<T><<<S.n_eval, kEvalChunk, S.smem_eval, s>>>(tb, S.eval_items.as<LeafItem>(), contents,
                                                        P.d_centroid.as<double>(), P.d_normal.as<double>(),
                                                        S.leaf_exp.as<C>(), P.n, y);
  BP_LAUNCH_CHECK();
  end(1);
}

void fmm_apply(Problem& P, const double* x_dev, double* y_dev, StageTimes* st, cudaStream_t stream) {
  FmmState* S = P.fmm.get();
  if (!S) return;
  if (S->fp64)
    run_fmm<double>(P, *S, S->tb_d, x_dev, y_dev, st, stream);
  else
    run_fmm<float>(P, *S, S->tb_f, x_dev, y_dev, st, stream);
}

}  // namespace bp
