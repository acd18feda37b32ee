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
constexpr int kXlCh = 2;  // channels per X2L block
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
                            const T* rd) {
  using C = typename C2T<T>::type;
  const int E = tb.E, NT = tb.nt, nout = kCh * E;
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
    const int lg = 2 * level + (ch >= 8 ? 1 : 0);
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

template <typename T>
__global__ void __launch_bounds__(256) m2m_kernel(const __grid_constant__ Tables<T> tb, const ShiftItem* __restrict__ items,
                                                  const ShiftChild* __restrict__ children, int child_level,
                                                  typename C2T<T>::type* __restrict__ M) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int nout = kCh * tb.E;
  C* w1 = reinterpret_cast<C*>(smem_raw);
  C* w2 = w1 + nout;
  C* acc = w2 + nout;
  C* in = acc + nout;
  const ShiftItem it = items[blockIdx.x];
  for (int o = threadIdx.x; o < nout; o += blockDim.x) acc[o] = cmk<C>(0, 0);
  for (int c = 0; c < it.n_children; ++c) {
    const ShiftChild ch = children[it.first_child + c];
    __syncthreads();
    for (int o = threadIdx.x; o < nout; o += blockDim.x) in[o] = M[(size_t)ch.node * nout + o];
    __syncthreads();
    const T* rd = tb.R(ch.octant > 4 ? ROT_MSQ3 : ROT_SQ3);
    shift_block<T>(tb, ch.octant, true, child_level, in, w1, w2, acc, rd);
  }
  __syncthreads();
  for (int o = threadIdx.x; o < nout; o += blockDim.x) M[(size_t)it.parent * nout + o] = acc[o];
}

// L2L: one block per child, local_child += shift(local_parent)
template <typename T>
__global__ void __launch_bounds__(256) l2l_kernel(const __grid_constant__ Tables<T> tb, const ShiftItem* __restrict__ items,
                                                  const ShiftChild* __restrict__ children, int parent_level,
                                                  typename C2T<T>::type* __restrict__ L) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int nout = kCh * tb.E;
  C* w1 = reinterpret_cast<C*>(smem_raw);
  C* w2 = w1 + nout;
  C* acc = w2 + nout;
  C* in = acc + nout;
  const ShiftItem it = items[blockIdx.x];
  const ShiftChild ch = children[it.first_child];
  for (int o = threadIdx.x; o < nout; o += blockDim.x) {
    in[o] = L[(size_t)it.parent * nout + o];
    acc[o] = L[(size_t)ch.node * nout + o];
  }
  __syncthreads();
  const T* rd = tb.R(ch.octant > 4 ? ROT_SQ3 : ROT_MSQ3);
  shift_block<T>(tb, ch.octant, false, parent_level, in, w1, w2, acc, rd);
  for (int o = threadIdx.x; o < nout; o += blockDim.x) L[(size_t)ch.node * nout + o] = acc[o];
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
  int parent_level, first_entry, n_entries;
  int targets[8];  // target child node ids (-1 absent or shadow)
};
struct XlEntry {
  int src;          // source node id
  signed char dir, targ, a, b, c, up;
};

constexpr int kXlThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kXlThreads) x2l_kernel(const __grid_constant__ Tables<T> tb,
                                                         const XlItem* __restrict__ items,
                                                         const XlEntry* __restrict__ entries,
                                                         const typename C2T<T>::type* __restrict__ W,
                                                         typename C2T<T>::type* __restrict__ L) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E, NT = tb.nt, nl = tb.nl, NPM = tb.np_max;
  C* acc = reinterpret_cast<C*>(smem_raw);  // [6][8][kXlCh][NPM]
  const XlItem it = items[blockIdx.x / (kCh / kXlCh)];
  const int ch0 = (blockIdx.x % (kCh / kXlCh)) * kXlCh;
  const int total = 6 * 8 * kXlCh * NPM;
  for (int o = threadIdx.x; o < total; o += blockDim.x) acc[o] = cmk<C>(0, 0);
  __syncthreads();
  // translations: thread owns (channel, i) pairs
  for (int o = threadIdx.x; o < kXlCh * NPM; o += blockDim.x) {
    const int cl = o / NPM, i = o - cl * NPM;
    const int ch = ch0 + cl;
    const int lg = 2 * it.parent_level + (ch >= 8 ? 1 : 0);
    const int np = tb.nexptotp[lg];
    if (i >= np) continue;
    const C* xs = tb.xs + (size_t)lg * 3 * NPM;
    const C* ys = tb.ys + (size_t)lg * 3 * NPM;
    const T* zs = tb.zs + (size_t)lg * 3 * NPM;
    for (int k = 0; k < it.n_entries; ++k) {
      const XlEntry en = entries[it.first_entry + k];
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
      C& a = acc[(((size_t)en.dir * 8 + en.targ) * kXlCh + cl) * NPM + i];
      a = cadd(a, cmul(w, t));
    }
  }
  __syncthreads();
  // conversion of the accumulated waves of each target to its local expansion
  C* mf = acc + total;          // [kXlCh][2][64]
  C* loc = mf + kXlCh * 2 * 64;  // [kXlCh][E]
  C* out = loc + kXlCh * E;      // [kXlCh][E]
  for (int t = 0; t < 8; ++t) {
    const int tn = it.targets[t];
    if (tn < 0) continue;
    for (int o = threadIdx.x; o < kXlCh * E; o += blockDim.x) out[o] = cmk<C>(0, 0);
    for (int pair = 0; pair < 3; ++pair) {
      __syncthreads();
      // yphystof (up = dir 2*pair, down = 2*pair+1)
      for (int o = threadIdx.x; o < kXlCh * 2 * 64; o += blockDim.x) {
        const int cl = o / 128, rem = o - cl * 128, which = rem / 64, j = rem - which * 64;
        const int ch = ch0 + cl;
        const int lg = 2 * it.parent_level + (ch >= 8 ? 1 : 0);
        if (j >= tb.nexptot[lg]) continue;
        const int* numphys = tb.numphys + (size_t)lg * nl;
        const C* fb = tb.fexpback + tb.fexpback_off[lg];
        int l = 0, nftot = 0, nptot = 0, bb = 0;
        while (nftot + tb.numfour[l] <= j) {
          nftot += tb.numfour[l];
          nptot += numphys[l] / 2;
          bb += (tb.numfour[l] - 1) * (numphys[l] / 2);
          ++l;
        }
        const int mm = j - nftot + 1;  // mode number 1..numfour
        const int na = numphys[l], na2 = na / 2;
        const C* ph = acc + (((size_t)(2 * pair + which) * 8 + t) * kXlCh + cl) * NPM + nptot;
        C s = cmk<C>(0, 0);
        if (mm == 1) {
          for (int iv = 0; iv < na2; ++iv) s.x += T(2) * ph[iv].x;
        } else if (mm & 1) {  // odd mm >= 3
          const C* f = fb + bb + ((mm - 3) / 2) * na2;
          for (int iv = 0; iv < na2; ++iv) s = cadd(s, cscale(f[iv], T(2) * ph[iv].x));
        } else {  // even mm
          const int nodd = (tb.numfour[l] - 1) / 2;
          const C* f = fb + bb + nodd * na2 + ((mm - 2) / 2) * na2;
          for (int iv = 0; iv < na2; ++iv) s = cadd(s, cmul(f[iv], cmk<C>(0, T(2) * ph[iv].y)));
        }
        mf[(cl * 2 + which) * 64 + j] = cscale(s, T(1) / T(na));
      }
      __syncthreads();
      // yexptolocal
      for (int o = threadIdx.x; o < kXlCh * E; o += blockDim.x) {
        const int cl = o / E, e = o - cl * E;
        const int ch = ch0 + cl;
        const int lg = 2 * it.parent_level + (ch >= 8 ? 1 : 0);
        const T* rl = tb.rlsc + (size_t)lg * E * nl;
        int nm = 0;
        while (tri(nm + 1, 0) <= e) ++nm;
        const int mth = e - tri(nm, 0);
        const C* fu = mf + (cl * 2 + 0) * 64;
        const C* fd = mf + (cl * 2 + 1) * 64;
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
        loc[o] = v;
      }
      __syncthreads();
      // rotate back and accumulate
      for (int o = threadIdx.x; o < kXlCh * E; o += blockDim.x) {
        const int cl = o / E, e = o - cl * E;
        if (pair == 0) {
          out[o] = cadd(out[o], loc[o]);
          continue;
        }
        int l = 0;
        while (tri(l + 1, 0) <= e) ++l;
        const int m = e - tri(l, 0);
        if (pair == 1) {  // rotate_ytoz(rdpi2): rotate then * i^m
          C v = rotate_one<T>(tb, loc + cl * E, tb.R(ROT_PI2), l, m);
          switch (m & 3) {
            case 1: v = cmk<C>(-v.y, v.x); break;
            case 2: v = cmk<C>(-v.x, -v.y); break;
            case 3: v = cmk<C>(v.y, -v.x); break;
            default: break;
          }
          out[o] = cadd(out[o], v);
        } else {  // rotate_ztox(rdmpi2)
          out[o] = cadd(out[o], rotate_one<T>(tb, loc + cl * E, tb.R(ROT_MPI2), l, m));
        }
      }
    }
    __syncthreads();
    for (int o = threadIdx.x; o < kXlCh * E; o += blockDim.x) {
      const int cl = o / E, e = o - cl * E;
      L[((size_t)tn * kCh + ch0 + cl) * E + e] = out[o];
    }
  }
  (void)NT;
}

// ---------------------------------------------------------------- L2P
struct LeafItem {
  int node, level, start, count;
  double c[3];
};

constexpr int kL2pWarps = 4;

// per-warp evaluation of the channel sums of FMM_results_to_BEM for one
// screening group; lanes over coefficients; returns (f, h) partial sums
template <typename T>
__device__ void l2p_group(const Tables<T>& tb, int g, int level, double d, double ctheta,
                          const typename C2T<T>::type& e1, const double nrm[3], const typename C2T<T>::type* Lc,
                          typename C2T<T>::type* q, typename C2T<T>::type* gq, typename C2T<T>::type* g2,
                          T* bi, T* p, double& f_acc, double& h_acc) {
  using C = typename C2T<T>::type;
  const int lane = threadIdx.x & 31;
  const int NT = tb.nt, N2 = NT + 2, E = tb.E;
  const int EQ = (N2 + 1) * (N2 + 2) / 2;      // q: n <= NT+2
  const int EG = (NT + 2) * (NT + 3) / 2;      // gq: n <= NT+1
  const int lg = 2 * level + g;
  const T beta = tb.beta[g], scale = tb.scale[lg], isc = T(1) / scale;
  if (lane == 0) bessel_in_dev<T>(scale, (T)(d * (double)beta), N2, bi);
  // Legendre: lane m computes column m
  {
    const T x = (T)ctheta;
    const T u = -sqrt(T(1) - x * x);
    if (lane <= N2) {
      const int m = lane;
      T pmm = 1;
      for (int k = 1; k <= m; ++k) pmm = pmm * u * T(2 * k - 1);
      p[tri(m, m)] = pmm;
      if (m < N2) {
        T p1 = T(2 * m + 1) * x * pmm;
        p[tri(m + 1, m)] = p1;
        T p0 = pmm;
        for (int n = m + 2; n <= N2; ++n) {
          const T pn = ((T(2) * n - T(1)) * x * p1 - T(n + m - 1) * p0) / T(n - m);
          p[tri(n, m)] = pn;
          p0 = p1;
          p1 = pn;
        }
      }
    }
  }
  __syncwarp();
  for (int e = lane; e < EQ; e += 32) {
    int n = 0;
    while (tri(n + 1, 0) <= e) ++n;
    const int m = e - tri(n, 0);
    if (n == 0) {
      q[e] = cmk<C>(bi[0], 0);
    } else {
      C ph = cmk<C>(1, 0);
      for (int k = 0; k < m; ++k) ph = cmul(ph, e1);
      q[e] = cscale(ph, bi[n] * p[e]);
    }
  }
  __syncwarp();
  // ladder (grad_q) from a source array src(n, m) with triangle width
  auto ladder = [&](const C* src, int n, int m, C out[3]) {
    C left[3], right[3];
    auto S = [&](int a, int b) { return src[tri(a, b)]; };
    const T sc = scale;
    if (n == 0 && m == 0) {
      left[0] = left[1] = left[2] = cmk<C>(0, 0);
      right[0] = cscale(cconj(S(1, 1)), -sc);
      right[1] = cscale(S(1, 0), -sc);
      right[2] = cscale(S(1, 1), sc);
    } else if (n == 1 && m == 0) {
      left[0] = cmk<C>(0, 0);
      left[1] = cscale(S(0, 0), isc);
      left[2] = cmk<C>(0, 0);
      right[0] = cscale(cconj(S(2, 1)), -sc);
      right[1] = cscale(S(2, 0), -T(2) * sc);
      right[2] = cscale(S(2, 1), sc);
    } else if (m == 0) {
      left[0] = cscale(cconj(S(n - 1, 1)), -isc);
      left[1] = cscale(S(n - 1, 0), T(n) * isc);
      left[2] = cscale(S(n - 1, 1), isc);
      right[0] = cscale(cconj(S(n + 1, 1)), -sc);
      right[1] = cscale(S(n + 1, 0), -T(n + 1) * sc);
      right[2] = cscale(S(n + 1, 1), sc);
    } else if (n == 1 && m == 1) {
      left[0] = cscale(S(0, 0), T(2) * isc);
      left[1] = left[2] = cmk<C>(0, 0);
      right[0] = cscale(S(2, 0), T(2) * sc);
      right[1] = cscale(S(2, 1), -sc);
      right[2] = cscale(S(2, 2), sc);
    } else if (m == n) {
      left[0] = cscale(S(n - 1, n - 1), T((n + n - 1) * (n + n)) * isc);
      left[1] = left[2] = cmk<C>(0, 0);
      right[0] = cscale(S(n + 1, n - 1), T(2) * sc);
      right[1] = cscale(S(n + 1, n), -sc);
      right[2] = cscale(S(n + 1, n + 1), sc);
    } else if (m == n - 1) {
      left[0] = cscale(S(n - 1, n - 2), T((n + m - 1) * (n + m)) * isc);
      left[1] = cscale(S(n - 1, n - 1), T(n + m) * isc);
      left[2] = cmk<C>(0, 0);
      right[0] = cscale(S(n + 1, m - 1), T(6) * sc);
      right[1] = cscale(S(n + 1, m), -T(2) * sc);
      right[2] = cscale(S(n + 1, m + 1), sc);
    } else {
      left[0] = cscale(S(n - 1, m - 1), T((n + m - 1) * (n + m)) * isc);
      left[1] = cscale(S(n - 1, m), T(n + m) * isc);
      left[2] = cscale(S(n - 1, m + 1), isc);
      right[0] = cscale(S(n + 1, m - 1), T((n - m + 1) * (n - m + 2)) * sc);
      right[1] = cscale(S(n + 1, m), -T(n - m + 1) * sc);
      right[2] = cscale(S(n + 1, m + 1), sc);
    }
    const T pre = T(-0.5) / T(2 * n + 1);
    const C a0 = csub(left[0], right[0]), a2 = csub(left[2], right[2]), a1 = csub(left[1], right[1]);
    out[0] = cscale(csub(a0, a2), pre * beta);
    const C s = cadd(a0, a2);
    out[1] = cmk<C>(-s.y * pre * beta, s.x * pre * beta);
    out[2] = cscale(a1, pre * beta * T(-2));
  };
  for (int e = lane; e < EG; e += 32) {
    int n = 0;
    while (tri(n + 1, 0) <= e) ++n;
    const int m = e - tri(n, 0);
    C o[3];
    ladder(q, n, m, o);
    gq[e] = o[0];
    gq[EG + e] = o[1];
    gq[2 * EG + e] = o[2];
  }
  __syncwarp();
  for (int e = lane; e < E; e += 32) {
    int n = 0;
    while (tri(n + 1, 0) <= e) ++n;
    const int m = e - tri(n, 0);
    for (int i = 0; i < 3; ++i) {
      C o[3];
      ladder(gq + i * EG, n, m, o);
      for (int c = 0; c < 3; ++c) g2[(c * 3 + i) * E + e] = o[c];  // g2q(c, i)
    }
  }
  __syncwarp();
  // channel sums of FMM_results_to_BEM (per group)
  const int c0 = g ? 8 : 0;
  double fp = 0, hp = 0;
  for (int e = lane; e < E; e += 32) {
    int n = 0;
    while (tri(n + 1, 0) <= e) ++n;
    const int m = e - tri(n, 0);
    const double w = m ? 2.0 : 1.0;
    auto re = [&](C a, C b) { return (double)a.x * (double)b.x - (double)a.y * (double)b.y; };
    const C* Lg = Lc;  // [12][E]
    // f: d/dx of ch0 + d/dy of ch1 + d/dz of ch2 + pot of ch3 (group 0); channels 8-11 for group 1
    double f = re(gq[e], Lg[(c0 + 0) * E + e]) + re(gq[EG + e], Lg[(c0 + 1) * E + e]) +
               re(gq[2 * EG + e], Lg[(c0 + 2) * E + e]) + re(q[e], Lg[(c0 + 3) * E + e]);
    // h: sum_j n_j (H_jk + H_kj)/2 on channels c0h+k, plus n . grad on the last channel
    const int c0h = g ? 8 : 4, clast = g ? 11 : 7;
    double h = 0;
    for (int k = 0; k < 3; ++k) {
      for (int j = 0; j < 3; ++j) {
        const C hjk = g2[(j * 3 + k) * E + e], hkj = g2[(k * 3 + j) * E + e];
        h += 0.5 * nrm[j] * (re(hjk, Lg[(c0h + k) * E + e]) + re(hkj, Lg[(c0h + k) * E + e]));
      }
    }
    h += nrm[0] * re(gq[e], Lg[clast * E + e]) + nrm[1] * re(gq[EG + e], Lg[clast * E + e]) +
         nrm[2] * re(gq[2 * EG + e], Lg[clast * E + e]);
    fp += w * f;
    hp += w * h;
  }
  const double tbp = (double)beta * (2.0 / 3.14159265358979323846);
  f_acc += (g ? -1.0 : 1.0) * fp * tbp;
  h_acc += (g ? -1.0 : 1.0) * hp * tbp;
  __syncwarp();
}

template <typename T>
__global__ void __launch_bounds__(32 * kL2pWarps) l2p_kernel(const __grid_constant__ Tables<T> tb,
                                                             const LeafItem* __restrict__ items,
                                                             const int32_t* __restrict__ contents,
                                                             const double* __restrict__ centroid,
                                                             const double* __restrict__ normal,
                                                             const typename C2T<T>::type* __restrict__ L, int n,
                                                             double* __restrict__ y) {
  using C = typename C2T<T>::type;
  extern __shared__ unsigned char smem_raw[];
  const int E = tb.E, NT = tb.nt;
  const int EQ = (NT + 3) * (NT + 4) / 2, EG = (NT + 2) * (NT + 3) / 2;
  C* Lc = reinterpret_cast<C*>(smem_raw);  // [12][E]
  const int per_warp = EQ + 3 * EG + 9 * E;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C* ws = Lc + kCh * E + (size_t)warp * per_warp;
  C* q = ws;
  C* gq = q + EQ;
  C* g2 = gq + 3 * EG;
  T* scal = reinterpret_cast<T*>(Lc + kCh * E + (size_t)kL2pWarps * per_warp) + (size_t)warp * (EQ + NT + 4);
  T* p = scal;
  T* bi = p + EQ;
  const LeafItem it = items[blockIdx.x];
  for (int o = threadIdx.x; o < kCh * E; o += blockDim.x) Lc[o] = L[(size_t)it.node * kCh * E + o];
  __syncthreads();
  for (int k = warp; k < it.count; k += kL2pWarps) {
    const int i = contents[it.start + k];
    const double rx = centroid[3 * i] - it.c[0], ry = centroid[3 * i + 1] - it.c[1], rz = centroid[3 * i + 2] - it.c[2];
    double proj = rx * rx + ry * ry;
    const double rr = proj + rz * rz;
    proj = sqrt(proj);
    const double d = sqrt(rr);
    const double PREC = 2.220446049250313e-16;
    const double ct = (d <= PREC) ? 0.0 : rz / d;
    const C e1 = (proj <= PREC * d) ? cmk<C>(1, 0) : cmk<C>((T)(rx / proj), (T)(ry / proj));
    const double nrm[3] = {normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]};
    double f = 0, h = 0;
    l2p_group<T>(tb, 0, it.level, d, ct, e1, nrm, Lc, q, gq, g2, bi, p, f, h);
    l2p_group<T>(tb, 1, it.level, d, ct, e1, nrm, Lc, q, gq, g2, bi, p, f, h);
    for (int o = 16; o > 0; o >>= 1) {
      f += __shfl_xor_sync(0xffffffffu, f, o);
      h += __shfl_xor_sync(0xffffffffu, h, o);
    }
    if (lane == 0) {
      const double k4 = 0.07957747154594767;
      y[i] += f * k4;
      y[n + i] += h * k4;
    }
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
  size_t smem_p2m = 0, smem_shift = 0, smem_m2x = 0, smem_xl = 0, smem_l2p = 0;
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
    it.first_entry = (int)xle.size();
    bool any_target = false;
    for (int c = 0; c < 8; ++c) {
      const int ck = nd.children[c];
      it.targets[c] = (ck >= 0 && !(flags(ck) & TREE_SHADOW)) ? ck : -1;
      any_target |= it.targets[c] >= 0;
    }
    if (!any_target) continue;
    for (const RawInteraction& r : table) {
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
    it.n_entries = (int)xle.size() - it.first_entry;
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
  std::vector<LeafItem> leaves;
  for (int k = 0; k < nn; ++k) {
    if (!(flags(k) & TREE_LEAF) || cnt(k) == 0) continue;
    LeafItem it{k, T.nodes[k].level, (int)T.nodes[k].content_start, cnt(k), {0, 0, 0}};
    for (int d = 0; d < 3; ++d) it.c[d] = T.nodes[k].centre[d];
    leaves.push_back(it);
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
  // contents on the device (node-major patch lists)
  const int E = S->E, NT = S->nt;
  S->smem_p2m = celem * 2 * kP2mChunk * E + (S->fp64 ? 8 : 4) * kP2mChunk * kCh;
  S->smem_shift = 4 * celem * kCh * E;
  S->smem_m2x = celem * (2 * E + 128);
  S->smem_xl = celem * (6 * 8 * kXlCh * (size_t)S->np_max + kXlCh * 2 * 64 + 2 * kXlCh * E);
  const int EQ = (NT + 3) * (NT + 4) / 2, EG = (NT + 2) * (NT + 3) / 2;
  S->smem_l2p = celem * (kCh * E + (size_t)kL2pWarps * (EQ + 3 * EG + 9 * E)) +
                (S->fp64 ? 8 : 4) * (size_t)kL2pWarps * (EQ + NT + 4);
  auto attr = [&](const void* fn, size_t bytes) {
    if (bytes > 48 * 1024) BP_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  };
  if (S->fp64) {
    attr((const void*)p2m_kernel<double>, S->smem_p2m);
    attr((const void*)m2m_kernel<double>, S->smem_shift);
    attr((const void*)l2l_kernel<double>, S->smem_shift);
    attr((const void*)m2x_kernel<double>, S->smem_m2x);
    attr((const void*)x2l_kernel<double>, S->smem_xl);
    attr((const void*)l2p_kernel<double>, S->smem_l2p);
  } else {
    attr((const void*)p2m_kernel<float>, S->smem_p2m);
    attr((const void*)m2m_kernel<float>, S->smem_shift);
    attr((const void*)l2l_kernel<float>, S->smem_shift);
    attr((const void*)m2x_kernel<float>, S->smem_m2x);
    attr((const void*)x2l_kernel<float>, S->smem_xl);
    attr((const void*)l2p_kernel<float>, S->smem_l2p);
  }
  if (S->smem_xl > 227 * 1024 || S->smem_l2p > 227 * 1024)
    throw std::invalid_argument("FMM order too large for the shared-memory layout");
  // device copy of the tree contents (node-major)
  P.fmm_contents = upload(c, T.contents);
  BP_CUDA(cudaStreamSynchronize(c->stream));
}

template <typename T>
static void run_fmm(Problem& P, FmmState& S, const Tables<T>& tb, const double* x, double* y, StageTimes* st) {
  using C = typename C2T<T>::type;
  cudaStream_t s = P.ctx->stream;
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
    if (!S.m2m_count[lev]) continue;
    m2m_kernel<T><<<S.m2m_count[lev], 256, S.smem_shift, s>>>(
        tb, S.m2m_items.as<ShiftItem>() + S.m2m_first[lev], S.m2m_children.as<ShiftChild>(), lev, M);
    BP_LAUNCH_CHECK();
    ++l_m2m;
  }
  end(l_m2m);
  begin(3);
  m2x_kernel<T><<<S.n_m2x * kCh, kM2xThreads, S.smem_m2x, s>>>(tb, S.m2x_items.as<M2xItem>(), M, W);
  BP_LAUNCH_CHECK();
  end(1);
  begin(4);
  x2l_kernel<T><<<S.n_xl * (kCh / kXlCh), kXlThreads, S.smem_xl, s>>>(tb, S.xl_items.as<XlItem>(),
                                                                     S.xl_entries.as<XlEntry>(), W, Lx);
  BP_LAUNCH_CHECK();
  end(1);
  begin(6);
  int l_l2l = 0;
  for (int lev = 0; lev < S.nlev - 1; ++lev) {
    if (!S.l2l_count[lev]) continue;
    l2l_kernel<T><<<S.l2l_count[lev], 256, S.smem_shift, s>>>(
        tb, S.l2l_items.as<ShiftItem>() + S.l2l_first[lev], S.l2l_children.as<ShiftChild>(), lev, Lx);
    BP_LAUNCH_CHECK();
    ++l_l2l;
  }
  end(l_l2l);
  begin(7);
  l2p_kernel<T><<<S.n_leaf, 32 * kL2pWarps, S.smem_l2p, s>>>(tb, S.leaf_items.as<LeafItem>(), contents,
                                                             P.d_centroid.as<double>(), P.d_normal.as<double>(), Lx,
                                                             P.n, y);
  BP_LAUNCH_CHECK();
  end(1);
}

void fmm_apply(Problem& P, const double* x_dev, double* y_dev, StageTimes* st) {
  FmmState* S = P.fmm.get();
  if (!S) return;
  if (S->fp64)
    run_fmm<double>(P, *S, S->tb_d, x_dev, y_dev, st);
  else
    run_fmm<float>(P, *S, S->tb_f, x_dev, y_dev, st);
}

}  // namespace bp
